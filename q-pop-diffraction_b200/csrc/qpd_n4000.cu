// Register-resident 4000-point axis passes of the float32 fused schedule.
//
// A 4000-point transform is done by 200 threads that hold 20 values each in registers, in three
// self-sorting (Stockham) stages of radix 10, 20 and 20:
//   stage 1 (radix 10, no twiddles): thread t holds x[t + 200 r] (r = 0..19); butterflies j = t and
//           t + 200 take x[j + 400 r'];
//   stage 2 (radix 20, twiddles exp(-2 pi i r k / 200), k = t mod 10) and
//   stage 3 (radix 20, twiddles exp(-2 pi i r t / 4000)) read their butterflies from a shared-memory
//           exchange buffer; stage 3 leaves X[t + 200 r] in the thread's registers.
// The radix-10 and radix-20 butterflies are prime-factor (Good-Thomas) transforms, 2 x 5 and 4 x 5,
// with no twiddles inside.  Stages 2 and 3 form the powers w^1..w^19 of their thread's root from the
// exact w^1, w^5, w^10 and w^15 of a small shared-memory table by at most three complex
// multiplications each.  A transform costs two shared-memory round trips and two CTA barriers; the
// exchange buffers are padded (one slot after every 80 and every 100 values) so the stage writes and
// reads of a half-warp of consecutive t are free of bank conflicts, and every thread's addresses
// reduce to a few bases plus compile-time offsets.
//
// The fold coefficients are formed in registers from two small factors (Pass4k: a per-thread root read
// once per input and 20 constants per input in shared memory).  CTAs are persistent: each walks its
// pencils input by input, and the next input's pencil (or tile of two pencils) arrives by TMA in a
// staging buffer while the current one is transformed, completing on an mbarrier whose waits are
// bounded (a copy that never lands records QPD_DEVERR_TIMEOUT in the status word and ends the CTA).
#include "qpd_n4000.h"
#include "qpd_tma.cuh"

namespace qpd {
namespace {

constexpr int kN = 4000, kT = 200;
constexpr int kSA = kN + kN / 80;   // exchange buffer after stage 1
constexpr int kSB = kN + kN / 100;  // after stage 2
constexpr int kT2 = 4 * 10;         // stage-2 seeds [e][k], k = t mod 10
constexpr int kS3 = 4 * kT;         // stage-3 seeds [e][t]
constexpr int kTW = kT2 + kS3;      // twiddle seeds of a CTA

// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}

// 5-point DFT, natural order, exp(-2 pi i / 5) convention
__device__ __forceinline__ void dft5(float2& x0, float2& x1, float2& x2, float2& x3, float2& x4) {
    const float c1 = 0.309016994374947424f;   // cos(2 pi / 5)
    const float c2 = -0.809016994374947424f;  // cos(4 pi / 5)
    const float s1 = 0.951056516295153572f;   // sin(2 pi / 5)
    const float s2 = 0.587785252292473129f;   // sin(4 pi / 5)
    const float2 a1 = cadd(x1, x4), a2 = cadd(x2, x3), b1 = csub(x1, x4), b2 = csub(x2, x3);
    float2 A1 = x0, A2 = x0;
    caxpy(A1, c1, a1);
    caxpy(A1, c2, a2);
    caxpy(A2, c2, a1);
    caxpy(A2, c1, a2);
    float2 B1 = cscale(b1, s1);
    caxpy(B1, s2, b2);
    float2 B2 = cscale(b1, s2);
    caxpy(B2, -s1, b2);
    x0 = cadd(x0, cadd(a1, a2));
    x1 = cadd_mi(A1, B1);
    x4 = cadd_pi(A1, B1);
    x2 = cadd_mi(A2, B2);
    x3 = cadd_pi(A2, B2);
}

// 10-point DFT as 2 x 5: input n = (5 n1 + 2 n2) mod 10, output k = (5 k1 + 6 k2) mod 10
__device__ __forceinline__ void dft10(float2 (&x)[10]) {
    float2 a0[5], a1[5];
#pragma unroll
    for (int n2 = 0; n2 < 5; n2++) {
        const float2 p = x[(2 * n2) % 10], q = x[(5 + 2 * n2) % 10];
        a0[n2] = cadd(p, q);
        a1[n2] = csub(p, q);
    }
    dft5(a0[0], a0[1], a0[2], a0[3], a0[4]);
    dft5(a1[0], a1[1], a1[2], a1[3], a1[4]);
#pragma unroll
    for (int k2 = 0; k2 < 5; k2++) {
        x[(6 * k2) % 10] = a0[k2];
        x[(5 + 6 * k2) % 10] = a1[k2];
    }
}

// 20-point DFT as 4 x 5: input n = (5 n1 + 4 n2) mod 20, output k = (5 k1 + 16 k2) mod 20
__device__ __forceinline__ void dft20(float2 (&x)[20]) {
    float2 a[4][5];
#pragma unroll
    for (int n2 = 0; n2 < 5; n2++) {
        float2 x0 = x[(4 * n2) % 20], x1 = x[(5 + 4 * n2) % 20], x2 = x[(10 + 4 * n2) % 20],
               x3 = x[(15 + 4 * n2) % 20];
        const float2 p = cadd(x0, x2), q = csub(x0, x2), r = cadd(x1, x3), s = csub(x1, x3);
        a[0][n2] = cadd(p, r);
        a[2][n2] = csub(p, r);
        a[1][n2] = cadd_mi(q, s);
        a[3][n2] = cadd_pi(q, s);
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
        dft5(a[k1][0], a[k1][1], a[k1][2], a[k1][3], a[k1][4]);
#pragma unroll
        for (int k2 = 0; k2 < 5; k2++) x[(5 * k1 + 16 * k2) % 20] = a[k1][k2];
    }
}

// v[r] *= w^r (r = 1..19) from the exact seeds s = {w, w^5, w^10, w^15}
__device__ __forceinline__ void twiddle20(float2 (&v)[20], const float2 (&s)[4]) {
    const float2 w1 = s[0], w5 = s[1], w10 = s[2], w15 = s[3];
    const float2 w2 = cmul(w1, w1);
    const float2 w3 = cmul(w2, w1);
    const float2 w4 = cmulc(w5, w1);
    v[1] = cmul(v[1], w1);
    v[2] = cmul(v[2], w2);
    v[3] = cmul(v[3], w3);
    v[4] = cmul(v[4], w4);
    v[5] = cmul(v[5], w5);
    v[6] = cmul(v[6], cmul(w5, w1));
    v[7] = cmul(v[7], cmul(w5, w2));
    v[8] = cmul(v[8], cmulc(w10, w2));
    v[9] = cmul(v[9], cmulc(w10, w1));
    v[10] = cmul(v[10], w10);
    v[11] = cmul(v[11], cmul(w10, w1));
    v[12] = cmul(v[12], cmul(w10, w2));
    v[13] = cmul(v[13], cmulc(w15, w2));
    v[14] = cmul(v[14], cmulc(w15, w1));
    v[15] = cmul(v[15], w15);
    v[16] = cmul(v[16], cmul(w15, w1));
    v[17] = cmul(v[17], cmul(w15, w2));
    v[18] = cmul(v[18], cmul(w15, w3));
    v[19] = cmul(v[19], cmul(w15, w4));
}

// The CTA's twiddle seeds in shared memory, filled from tw[m] = exp(-2 pi i m / 4000), e = 1, 5, 10, 15:
// t2[10 i + k] = exp(-2 pi i k e_i / 200) = tw[20 k e_i] and s3[200 i + t] = tw[t e_i].
struct Twiddles {
    float2* t2;
    float2* s3;
    __device__ __forceinline__ void fill(const float2* tw, int tid, int nthreads) const {
        const int e[4] = {1, 5, 10, 15};
        for (int i = tid; i < kT2; i += nthreads) t2[i] = tw[20 * (i % 10) * e[i / 10]];
        for (int i = tid; i < kS3; i += nthreads) s3[i] = tw[(i % kT) * e[i / kT]];
    }
};

// Thread t's shared-memory bases for the exchanges.  Buffer A holds stage-1 outputs at
// p + p / 80, buffer B stage-2 outputs at p + p / 100 (p the Stockham position), which reduces to:
//   stage-1 write, butterfly j:  A + 10 j + j / 8 + r           (r < 10)
//   stage-2 read, r = 0..19:     A + t + t / 80 + 202 r + r / 2 (+ 1 for odd r when t mod 80 >= 40)
//   stage-2 write:               B + 202 (t / 10) + t mod 10 + 10 r + [r >= 10]
//   stage-3 read:                B + t + t / 100 + 202 r
struct Lanes {
    float2* w1[2];
    const float2* r2[2];  // even, odd r
    float2* w2;
    const float2* r3;
    int t, k;
    __device__ __forceinline__ Lanes(float2* A, float2* B, int t_) : t(t_), k(t_ % 10) {
        for (int js = 0; js < 2; js++) {
            const int j = t + 200 * js;
            w1[js] = A + 10 * j + j / 8;
        }
        r2[0] = A + t + t / 80;
        r2[1] = r2[0] + ((t % 80) >= 40 ? 1 : 0);
        w2 = B + 202 * (t / 10) + k;
        r3 = B + t + t / 100;
    }
};

// Stage 1: v[r] = x[t + 200 r] -> A.
__device__ __forceinline__ void stage1(float2 (&v)[20], const Lanes& L) {
#pragma unroll
    for (int js = 0; js < 2; js++) {
        float2 x[10];
#pragma unroll
        for (int r = 0; r < 10; r++) x[r] = v[2 * r + js];
        dft10(x);
#pragma unroll
        for (int r = 0; r < 10; r++) L.w1[js][r] = x[r];
    }
}

// Stage 2: A -> B (after the barrier that follows stage 1).
__device__ __forceinline__ void stage2(float2 (&v)[20], const Lanes& L, const Twiddles& tw) {
#pragma unroll
    for (int r = 0; r < 20; r++) v[r] = L.r2[r & 1][202 * r + r / 2];
    const float2 seeds[4] = {tw.t2[L.k], tw.t2[10 + L.k], tw.t2[20 + L.k], tw.t2[30 + L.k]};
    twiddle20(v, seeds);
    dft20(v);
#pragma unroll
    for (int r = 0; r < 20; r++) L.w2[10 * r + (r >= 10 ? 1 : 0)] = v[r];
}

// Stage 3: B -> v[r] = X[t + 200 r] (after the barrier that follows stage 2).
__device__ __forceinline__ void stage3(float2 (&v)[20], const Lanes& L, const Twiddles& tw) {
#pragma unroll
    for (int r = 0; r < 20; r++) v[r] = L.r3[202 * r];
    const float2 seeds[4] = {tw.s3[L.t], tw.s3[kT + L.t], tw.s3[2 * kT + L.t], tw.s3[3 * kT + L.t]};
    twiddle20(v, seeds);
    dft20(v);
}

// acc[r] += u V[r] (-i k_m when ik) v[r], m = t + 200 r
__device__ __forceinline__ void fold20(float2 (&acc)[20], const float2 (&v)[20], float2 u, const float2* V, bool ik,
                                       float kscale, int t) {
#pragma unroll
    for (int r = 0; r < 20; r++) {
        float2 cf = cmul(u, V[r]);
        if (ik) {
            const float k = kscale * (float)(t + 200 * r - (r >= 10 ? kN : 0));
            cf = make_float2(k * cf.y, -k * cf.x);
        }
        cfma(acc[r], cf, v[r]);
    }
}

__device__ __forceinline__ void fill_v(float2* Vs, const Pass4k& p, int tid, int nthreads) {
    for (int i = tid; i < 20 * p.n; i += nthreads) Vs[i] = p.V[i / 20][i % 20];
}

__device__ __forceinline__ int shift_at(int k, int n) {
    const int v = k + n / 2;
    return v >= n ? v - n : v;
}

// ---------------------------------------------------------------------------------------
// y pass over (x, k_z, y) fields: pencil q = x nz + k_z holds N contiguous values in every field.
// 200 threads; shared memory: staging S (one pencil, 1-D bulk copies), A, B, seeds, V factors.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kT, 2) ypass4000(AxisArgs<float> a, const __grid_constant__ Pass4k p,
                                                   long long npencils) {
    extern __shared__ __align__(128) unsigned char sm_raw[];
    float2* S = reinterpret_cast<float2*>(sm_raw);
    float2* A = S + kN;
    float2* B = A + kSA;
    const Twiddles tw{B + kSB, B + kSB + kT2};
    float2* Vs = B + kSB + kTW;
    __shared__ __align__(8) uint64_t bar;
    const int t = threadIdx.x;
    if (smem_u32(sm_raw) % 16 != 0 || reinterpret_cast<uintptr_t>(a.in) % 16 != 0 || (a.fstride * 8) % 16 != 0) {
        if (t == 0) atomicExch(a.status, QPD_DEVERR_ALIGN);  // bulk copies need 16-byte alignment: do not load
        return;
    }
    long long pen = blockIdx.x;
    if (pen >= npencils) return;
    tw.fill(static_cast<const float2*>(a.ap.tw), t, kT);
    fill_v(Vs, p, t, kT);
    const Lanes L(A, B, t);
    auto issue = [&](long long q, int fl) {
        const float2* src = a.in + (long long)p.field[fl] * a.fstride + q * kN;
        mbar_expect_tx(&bar, kN * sizeof(float2));
#pragma unroll
        for (int k = 0; k < 4; k++) bulk_load(S + k * (kN / 4), src + k * (kN / 4), kN / 4 * sizeof(float2), &bar);
    };
    if (t == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
        issue(pen, 0);
    }
    __syncthreads();
    uint32_t phase = 0;
    int fl = 0;
    float2 acc[20];
#pragma unroll
    for (int r = 0; r < 20; r++) acc[r] = make_float2(0.f, 0.f);
    for (;;) {
        const float2 u = p.u[fl][t];
        long long npen = pen;
        int nfl = fl + 1;
        if (nfl == p.n) {
            nfl = 0;
            npen += gridDim.x;
        }
        const bool more = npen < npencils;
        const bool ok = mbar_wait(&bar, phase, a.status);
        if (!__syncthreads_and(ok)) return;  // a copy never landed; the status word records it
        phase ^= 1;
        float2 v[20];
#pragma unroll
        for (int r = 0; r < 20; r++) v[r] = S[t + 200 * r];
        stage1(v, L);
        __syncthreads();  // A written, S consumed
        if (t == 0 && more) {
            fence_proxy_async();
            issue(npen, nfl);
        }
        stage2(v, L, tw);
        __syncthreads();
        stage3(v, L, tw);
        fold20(acc, v, u, Vs + 20 * fl, (p.ik >> fl) & 1, p.kscale, t);
        if ((p.last >> fl) & 1) {
            float2* dst = a.out + (long long)p.out[fl] * a.fstride + pen * kN + t;
#pragma unroll
            for (int r = 0; r < 20; r++) {
                dst[200 * r] = acc[r];
                acc[r] = make_float2(0.f, 0.f);
            }
        }
        if (!more) break;
        pen = npen;
        fl = nfl;
    }
}

// Named barrier `id` over the n threads (a multiple of 32) of one pencil group.
__device__ __forceinline__ void group_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }

// The same barrier, returning whether p holds in every thread of the group.
__device__ __forceinline__ bool group_and(bool p, int id, int n) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred pi, po;\n\t"
        "setp.ne.u32 pi, %1, 0;\n\t"
        "bar.red.and.pred po, %2, %3, pi;\n\t"
        "selp.u32 %0, 1, 0, po;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)p), "r"(id), "r"(n)
        : "memory");
    return r != 0;
}

// ---------------------------------------------------------------------------------------
// Strided pass: a tile is the two pencils of inner values 2 b and 2 b + 1 at one outer index o (the
// value at transform index x of pencil (o, i) is element (o, i, x) of the map's view); it arrives as
// 20 tensor boxes of 200 rows x 16 bytes in the staging buffer, S[2 x + c].  The CTA is two groups of
// 7 warps, group c transforming pencil c (thread 32 w + l of the group at t = 32 w + l < 200), each with
// its own exchange buffers and named barrier, so one pencil's barrier waits do not hold the other's
// warps.  The groups share only the staging buffer: a group's leader counts its release in `released`
// after the group's stage-1 reads, and the leader that completes the pair issues the next tile.
// MID: the rows run along the map's middle dimension and tile (o, b) reads boxes at (4 b, 200 j,
// f nouter + o); otherwise along the outer dimension, boxes at (4 b, o, f nx + 200 j).
// EPI false (MID): the z-fastest y pass (o = x); the folded segments are stored in place.
// EPI true: the x pass with the |S Amp|^2 + fftshift epilogue, YZ for y-fastest fields (o = k_z,
// i = k_y; MID: (k_z, x, y) fields, whose x rows are ny values apart), else (x, y, z) fields (o = k_y,
// i = k_z, i fastest).  YZ tiles go in groups of 40 k_y pairs x 4 k_z (k_y pair fastest) when the
// extents allow, so the tiles in flight read 640 contiguous bytes of each x row per k_z.  With YZ and
// AxisArgs::Istage set, each pencil's intensities go whole into the staged (k_z, k_y, k_x) rows and
// unstage_intensity moves them to I afterwards: written here, the fftshifted I (k_z fastest) would
// take every value in a sector of its own.
// ---------------------------------------------------------------------------------------
constexpr int kGT = 7 * 32;                  // threads of one pencil group
constexpr int kXT = 2 * kGT;                  // two groups
constexpr int kTile = 2 * kN;                 // staging: two pencils, interleaved
constexpr int kPen = kSA + kSB + 8;           // one pencil's exchange buffers, the second 8 banks over

template <bool EPI, bool YZ, bool MID>
__global__ void __launch_bounds__(kXT, 1) strided4000(const __grid_constant__ CUtensorMap map, AxisArgs<float> a,
                                                      const __grid_constant__ Pass4k p, int nouter, int ntiles) {
    extern __shared__ __align__(128) unsigned char sm_raw[];
    float2* S = reinterpret_cast<float2*>(sm_raw);
    const int tid = threadIdx.x;
    const int c = tid / kGT;
    const int t = tid - c * kGT;
    const int gbar = 1 + c;  // the group's named barrier (0 is __syncthreads)
    const bool act = t < kT;
    const int tt = act ? t : 0;
    float2* A = S + kTile + c * kPen;
    float2* B = A + kSA;
    const Twiddles tw{S + kTile + 2 * kPen, S + kTile + 2 * kPen + kT2};
    float2* Vs = S + kTile + 2 * kPen + kTW;
    __shared__ __align__(8) uint64_t bar;
    __shared__ unsigned int released;  // +1 per group and tile once the group has read the staging buffer
    if (smem_u32(sm_raw) % 128 != 0) {  // TMA destinations must be 128-byte aligned: refuse, do not load
        if (tid == 0) atomicExch(a.status, QPD_DEVERR_ALIGN);
        return;
    }
    int q = blockIdx.x;
    if (q >= ntiles) return;
    tw.fill(static_cast<const float2*>(a.ap.tw), tid, kXT);
    fill_v(Vs, p, tid, kXT);
    const Lanes L(A, B, tt);
    const int npairs = a.nz / 2;
    const int nfx = (int)a.nx;
    constexpr int GB = 40, GO = 4;  // YZ tile groups: k_y pairs x k_z
    const bool grouped = npairs % GB == 0 && nouter % GO == 0;
    auto tile_of = [&](int qq, int* o, int* b) {  // 32-bit: ntiles < 2^31 (checked at launch)
        if (EPI && YZ) {
            if (grouped) {
                const int in = qq % (GB * GO);
                const int g = qq / (GB * GO);
                const int nog = nouter / GO;
                *b = (g / nog) * GB + in % GB;
                *o = (g % nog) * GO + in / GB;
            } else {
                *o = qq % nouter;
                *b = qq / nouter;
            }
        } else {
            *o = qq / npairs;
            *b = qq % npairs;
        }
    };
    auto issue = [&](int qq, int fl) {
        int o, b;
        tile_of(qq, &o, &b);
        const int f = p.field[fl];
        mbar_expect_tx(&bar, kTile * sizeof(float2));
#pragma unroll
        for (int j = 0; j < 20; j++) {
            if (MID) tma_load_3d(S + 400 * j, &map, &bar, 4 * b, 200 * j, f * nouter + o);
            else tma_load_3d(S + 400 * j, &map, &bar, 4 * b, o, f * nfx + 200 * j);
        }
    };
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
        released = 0;
        issue(q, 0);
    }
    __syncthreads();
    uint32_t phase = 0;
    int fl = 0;
    float2 acc[20];
#pragma unroll
    for (int r = 0; r < 20; r++) acc[r] = make_float2(0.f, 0.f);
    for (;;) {
        const float2 u = p.u[fl][tt];
        int nq = q;
        int nfl = fl + 1;
        if (nfl == p.n) {
            nfl = 0;
            nq += gridDim.x;
        }
        const bool more = nq < ntiles;
        const bool ok = mbar_wait(&bar, phase, a.status);
        if (!group_and(ok, gbar, kGT)) return;  // a copy never landed; the status word records it
        phase ^= 1;
        float2 v[20];
        if (act) {
#pragma unroll
            for (int r = 0; r < 20; r++) v[r] = S[2 * (tt + 200 * r) + c];
            stage1(v, L);
        }
        group_sync(gbar, kGT);  // A written, this group's reads of S done
        if (t == 0 && more) {
            // the second group to release the staging buffer issues the next tile into it
            __threadfence_block();
            const unsigned int before = atomicAdd(&released, 1u);
            __threadfence_block();
            if (before & 1u) {
                fence_proxy_async();
                issue(nq, nfl);
            }
        }
        if (act) stage2(v, L, tw);
        group_sync(gbar, kGT);
        if (act) {
            stage3(v, L, tw);
            fold20(acc, v, u, Vs + 20 * fl, (p.ik >> fl) & 1, p.kscale, tt);
            if ((p.last >> fl) & 1) {
                int o, b;
                tile_of(q, &o, &b);
                const int i = 2 * b + c;
                if constexpr (EPI) {
                    const int ky = YZ ? i : o, kz = YZ ? o : i;
                    const int NY = (int)a.ny, NZ = YZ ? nouter : a.nz;
                    const long long sy = shift_at(ky, NY);
                    const long long sz = shift_at(kz, NZ);
                    const double syz = a.S[1][ky] * a.S[2][kz];
                    double* srow = YZ && a.Istage ? a.Istage + ((long long)kz * NY + ky) * nfx : nullptr;
#pragma unroll
                    for (int r = 0; r < 20; r++) {
                        const int kx = tt + 200 * r;
                        const double Sx = a.S[0][kx] * syz;
                        const double re = (double)acc[r].x, im = (double)acc[r].y;
                        const double val = floor_1e50(Sx * Sx * (re * re + im * im) * a.scale2);
                        if (srow) srow[kx] = val;
                        else a.I[((long long)shift_at(kx, nfx) * NY + sy) * NZ + sz] = val;
                    }
                } else {
                    float2* dst = a.out + (long long)p.out[fl] * a.fstride + (long long)o * a.ostride + i +
                                  (long long)tt * a.stride;
                    const long long step = 200LL * a.stride;
#pragma unroll
                    for (int r = 0; r < 20; r++) dst[r * step] = acc[r];
                }
#pragma unroll
                for (int r = 0; r < 20; r++) acc[r] = make_float2(0.f, 0.f);
            }
        }
        if (!more) break;
        q = nq;
        fl = nfl;
    }
}

// ---------------------------------------------------------------------------------------
// Staged intensity -> I: I[shift(k_x)][shift(k_y)][shift(k_z)] = T[k_z][k_y][k_x] (shift(k) = (k + n / 2) mod n).
// A tile is one k_y and kUX neighbouring k_x over all k_z: 8 warps read its k_z rows of kUX values (512
// bytes each), then write its kUX I rows of nz values (contiguous, k_z fastest).  CTAs are persistent.
// ---------------------------------------------------------------------------------------
constexpr int kUT = 256, kUX = 64, kUP = kUX + 1;  // threads, k_x per tile, padded shared row

__global__ void __launch_bounds__(kUT) unstage_intensity(const double* __restrict__ T, double* __restrict__ I, int nx,
                                                         int ny, int nz, int ntiles) {
    extern __shared__ __align__(16) double tile[];  // [k_z][kUP]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nxb = (nx + kUX - 1) / kUX;
    for (int q = blockIdx.x; q < ntiles; q += gridDim.x) {
        const int ky = q / nxb;
        const int x0 = (q - ky * nxb) * kUX;
        for (int kz = warp; kz < nz; kz += kUT / 32) {
            const double* row = T + ((long long)kz * ny + ky) * nx;
#pragma unroll
            for (int h = 0; h < kUX; h += 32)
                if (x0 + h + lane < nx) tile[kz * kUP + h + lane] = row[x0 + h + lane];
        }
        __syncthreads();
        const long long sy = shift_at(ky, ny);
        for (int j = warp; j < kUX && x0 + j < nx; j += kUT / 32) {
            double* row = I + ((long long)shift_at(x0 + j, nx) * ny + sy) * nz;
            for (int kz = lane; kz < nz; kz += 32) row[shift_at(kz, nz)] = tile[kz * kUP + j];
        }
        __syncthreads();
    }
}

int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            n = 148;
    }
    return n;
}

template <bool EPI, bool YZ, bool MID>
cudaError_t launch_strided(const CUtensorMap& map, const AxisArgs<float>& a, const Pass4k& p, int nouter,
                           cudaStream_t st) {
    if (a.N != kN || a.nx < 1 || a.nz % 2 != 0 || nouter < 1 || p.n < 1 || p.n > kPass4kMax)
        return cudaErrorInvalidValue;
    const size_t smem = sizeof(float2) * (kTile + 2 * kPen + kTW + 20 * p.n);
    cudaError_t e = cudaFuncSetAttribute(strided4000<EPI, YZ, MID>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const long long ntiles = (long long)nouter * (a.nz / 2);
    if (ntiles + sm_count() >= (1LL << 31)) return cudaErrorInvalidValue;  // tiles index in 32 bits
    const long long grid = std::min<long long>(ntiles, sm_count());
    strided4000<EPI, YZ, MID><<<(unsigned)grid, kXT, smem, st>>>(map, a, p, nouter, (int)ntiles);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_unstage_intensity(const double* T, double* I, long long nx, long long ny, long long nz,
                                     cudaStream_t st) {
    const long long ntiles = ny * ((nx + kUX - 1) / kUX);
    if (nx < 1 || ny < 1 || nz < 1 || nz > 256 || ntiles >= (1LL << 31)) return cudaErrorInvalidValue;
    const size_t smem = sizeof(double) * kUP * nz;
    cudaError_t e = cudaFuncSetAttribute(unstage_intensity, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const long long grid = std::min<long long>(ntiles, 4LL * sm_count());
    unstage_intensity<<<(unsigned)grid, kUT, smem, st>>>(T, I, (int)nx, (int)ny, (int)nz, (int)ntiles);
    return cudaGetLastError();
}

cudaError_t launch_ypass4000(const AxisArgs<float>& a, const Pass4k& p, long long npencils, cudaStream_t st) {
    if (p.n < 1 || p.n > kPass4kMax || npencils < 1) return cudaErrorInvalidValue;
    const size_t smem = sizeof(float2) * (kN + kSA + kSB + kTW + 20 * p.n);
    cudaError_t e = cudaFuncSetAttribute(ypass4000, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const long long grid = std::min<long long>(npencils, 2LL * sm_count());
    ypass4000<<<(unsigned)grid, kT, smem, st>>>(a, p, npencils);
    return cudaGetLastError();
}

cudaError_t launch_strided4000(const CUtensorMap& map, const AxisArgs<float>& a, const Pass4k& p, int nouter,
                               Strided4k kind, cudaStream_t st) {
    switch (kind) {
        case Strided4k::YPassZFast: return launch_strided<false, false, true>(map, a, p, nouter, st);
        case Strided4k::XPassZFast: return launch_strided<true, false, false>(map, a, p, nouter, st);
        case Strided4k::XPassYFast: return launch_strided<true, true, true>(map, a, p, nouter, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace qpd
