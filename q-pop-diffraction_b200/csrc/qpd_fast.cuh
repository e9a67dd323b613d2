// Compile-time specialised fused kernels for the axis lengths of the measured workloads.
//
// Same work as zstage_kernel / axis_kernel in qpd_kernels.cuh, with the axis length, its radix
// stages, the tile shape and the thread count fixed at compile time: index arithmetic folds to
// shifts and multiplies, register arrays are sized exactly, and global accesses move two
// complex64 values (16 bytes) per thread when the z extent is even.  qpd_api.cu picks these
// kernels when a plan's axis lengths have an instantiation and falls back to the generic ones.
#pragma once

#include "qpd_kernels.cuh"
#include "qpd_tma.cuh"

namespace qpd {

// Position of index k (< n) after fftshift: (k + n / 2) mod n with one conditional subtraction.
__device__ __forceinline__ int fftshift_at(int k, int n) {
    const int v = k + n / 2;
    return v >= n ? v - n : v;
}

// ---------------------------------------------------------------------------------------
// z stage: source + FFT along z + fold, M columns of NZ cells per CTA
// ---------------------------------------------------------------------------------------
template <typename T, int NZ, int M, int NT, class RAD>
__global__ void __launch_bounds__(NT) zstage_fast(ZArgs<T> a) {
    using C = C_t<T>;
    constexpr int PS = NZ % 2 ? NZ : NZ + 1;
    constexpr int PLANE = M * PS;
    constexpr int CELLS = M * NZ;
    constexpr int CPT = cdiv(CELLS, NT);
    using GE = Geo<4 * M, 4 * M, PS, 0, 1, NT>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    AtomPhase<T>* apc = reinterpret_cast<AtomPhase<T>*>(buf + 4 * PLANE);
    const int tid = threadIdx.x;
    const int nap = a.in.nPhase * a.nAtom;
    for (int i = tid; i < nap; i += NT) apc[i] = a.apc[i];

    const long long c0 = (long long)blockIdx.x * M;
    const int ncell = (int)min((long long)M, a.ncols - c0) * NZ;
    const long long g0 = c0 * NZ;
    const C* tw = static_cast<const C*>(a.zp.tw);

    CellIn<T> cell[CPT];
    int ph[CPT];
    T wt[CPT];
    C accE[CPT], accX[CPT], accY[CPT];
#pragma unroll
    for (int q = 0; q < CPT; q++) {
        const int e = tid + q * NT;
        accE[q] = accX[q] = accY[q] = cmake<C>(0, 0);
        ph[q] = -1;
        wt[q] = T(0);
        if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
            const long long g = g0 + e;
            load_cell<T>(a.in, g, a.tq, cell[q]);
            if (!a.in.wdense) {
                ph[q] = a.in.phase[g];
                wt[q] = a.in.weight ? a.in.weight[g] : T(1);
            }
        }
    }
    __syncthreads();

    for (int at = 0; at < a.nAtom; at++) {
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            const int e = tid + q * NT;
            if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
                const int m = e / NZ;
                const int s = m * PS + (e - m * NZ);
                C E, X, Y, Z;
                cell_source<T>(a.in, g0 + e, cell[q], ph[q], wt[q], apc, a.nAtom, at, E, X, Y, Z);
                buf[s] = E;
                buf[PLANE + s] = X;
                buf[2 * PLANE + s] = Y;
                buf[3 * PLANE + s] = Z;
            }
        }
        __syncthreads();
        fft_ct<T, NZ, GE>(buf, tw, tid, RAD{});
        const C* ce = a.coefE + (long long)at * NZ;
        const C* cu = a.coefUz + (long long)at * NZ;
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            const int e = tid + q * NT;
            if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
                const int m = e / NZ;
                const int kz = e - m * NZ;
                const int s = m * PS + kz;
                const C e1 = ce[kz], u1 = cu[kz];
                cfma(accE[q], e1, buf[s]);
                cfma(accE[q], u1, buf[3 * PLANE + s]);
                cfma(accX[q], e1, buf[PLANE + s]);
                cfma(accY[q], e1, buf[2 * PLANE + s]);
            }
        }
        const int g = a.grp[at];
        if (at == a.nAtom - 1 || a.grp[at + 1] != g) {
            C* o = a.out + 3LL * g * a.fstride + g0;
#pragma unroll
            for (int q = 0; q < CPT; q++) {
                const int e = tid + q * NT;
                if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
                    o[e] = accE[q];
                    o[a.fstride + e] = accX[q];
                    o[2 * a.fstride + e] = accY[q];
                }
                accE[q] = accX[q] = accY[q] = cmake<C>(0, 0);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Strided axis pass on an N x CZ tile (rows along the axis, CZ contiguous z values).
// VEC complex values per global access (2: 16-byte float4 for complex64 when nz is even).
// ---------------------------------------------------------------------------------------
template <typename T, int N, int CZ, int NT, int VEC, bool EPI, class RAD>
__global__ void __launch_bounds__(NT) axis_fast(AxisArgs<T> a) {
    using C = C_t<T>;
    static_assert(CZ % VEC == 0, "chunk must hold whole vectors");
    constexpr int GROUPS = N * CZ / VEC;          // vector slots in the tile
    constexpr int EP = cdiv(GROUPS, NT);          // slots per thread
    constexpr int CV = CZ / VEC;                  // slots per row
    using GE = Geo<CZ, CZ, 1, 0, CZ, NT>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    const int tid = threadIdx.x;
    const long long outer = blockIdx.x / a.nzc;
    const int z0 = (int)(blockIdx.x % a.nzc) * CZ;
    const int cz = min(CZ, a.nz - z0);
    const long long base = outer * a.ostride + z0;
    const C* tw = static_cast<const C*>(a.ap.tw);

    for (int sg = 0; sg < a.nseg; sg++) {
        const Segment<T>& seg = a.segs[sg];
        C acc[2][EP][VEC];
#pragma unroll
        for (int q = 0; q < EP; q++)
#pragma unroll
            for (int w = 0; w < VEC; w++) acc[0][q][w] = acc[1][q][w] = cmake<C>(0, 0);
        for (int fi = 0; fi < seg.nin; fi++) {
            const C* src = a.in + seg.in[fi] * a.fstride + base;
#pragma unroll
            for (int q = 0; q < EP; q++) {
                const int e = tid + q * NT;
                if (GROUPS % NT == 0 || e < GROUPS) {
                    const int i = e / CV;
                    const int c = (e - i * CV) * VEC;
                    C* d = buf + i * CZ + c;
                    if (c < cz) {
                        if constexpr (VEC == 2) {
                            const float4 v = *reinterpret_cast<const float4*>(src + i * a.stride + c);
                            *reinterpret_cast<float4*>(d) = v;
                        } else {
                            d[0] = src[i * a.stride + c];
                        }
                    } else {
#pragma unroll
                        for (int w = 0; w < VEC; w++) d[w] = cmake<C>(0, 0);
                    }
                }
            }
            __syncthreads();
            fft_ct<T, N, GE>(buf, tw, tid, RAD{});
#pragma unroll
            for (int o = 0; o < 2; o++) {
                if (o >= seg.nout) break;
                const C* cf = seg.coef[o][fi];
                const bool mine = seg.ident ? (fi == o) : (cf != nullptr);
                if (!mine) continue;
#pragma unroll
                for (int q = 0; q < EP; q++) {
                    const int e = tid + q * NT;
                    if (GROUPS % NT == 0 || e < GROUPS) {
                        const int k = e / CV;
                        const int c = (e - k * CV) * VEC;
                        const C* s = buf + k * CZ + c;
                        if (seg.ident) {
#pragma unroll
                            for (int w = 0; w < VEC; w++) acc[o][q][w] = cadd(acc[o][q][w], s[w]);
                        } else {
                            const C f = cf[k];
#pragma unroll
                            for (int w = 0; w < VEC; w++) cfma(acc[o][q][w], f, s[w]);
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (EPI) {
            const long long ky = outer;
            const long long sy = (ky + a.ny / 2) % a.ny;
            const double syv = a.S[1][ky];
#pragma unroll
            for (int q = 0; q < EP; q++) {
                const int e = tid + q * NT;
                if (GROUPS % NT == 0 || e < GROUPS) {
                    const int kx = e / CV;
                    const int c = (e - kx * CV) * VEC;
                    const double sxy = a.S[0][kx] * syv;
                    const long long row = ((long long)fftshift_at(kx, (int)a.nx) * a.ny + sy) * a.nz;
#pragma unroll
                    for (int w = 0; w < VEC; w++) {
                        const int kz = z0 + c + w;
                        if (c + w < cz) {
                            const double S = sxy * a.S[2][kz];
                            const double re = (double)acc[0][q][w].x, im = (double)acc[0][q][w].y;
                            const double v = floor_1e50(S * S * (re * re + im * im) * a.scale2);
                            a.I[row + fftshift_at(kz, a.nz)] = v;
                        }
                    }
                }
            }
        } else {
#pragma unroll
            for (int o = 0; o < 2; o++) {
                if (o >= seg.nout) break;
                C* dst = a.out + seg.out[o] * a.fstride + base;
#pragma unroll
                for (int q = 0; q < EP; q++) {
                    const int e = tid + q * NT;
                    if (GROUPS % NT == 0 || e < GROUPS) {
                        const int i = e / CV;
                        const int c = (e - i * CV) * VEC;
                        if (c < cz) {
                            C* d = dst + i * a.stride + c;
                            C v[VEC];
#pragma unroll
                            for (int w = 0; w < VEC; w++) v[w] = acc[o][q][w];
                            if (a.accumulate) {
#pragma unroll
                                for (int w = 0; w < VEC; w++) v[w] = cadd(v[w], d[w]);
                            }
                            if constexpr (VEC == 2) {
                                *reinterpret_cast<float4*>(d) = *reinterpret_cast<const float4*>(v);
                            } else {
                                d[0] = v[0];
                            }
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Strided axis pass with TMA: the N x CZ tile of every input field arrives by
// cp.async.bulk.tensor into one of two shared-memory buffers, the next field's load in flight
// while the current one is transformed and folded.  The tensor map views the field array as
// (2 nz reals, ny, nfields * nx); XPASS selects rows along x (box 2CZ x 1 x BOX) instead of
// along y (box 2CZ x BOX x 1).  Out-of-range z of a partial chunk arrives as zeros.
// ---------------------------------------------------------------------------------------
// Rows per TMA box: the largest divisor of N that is at most 256 (a box dimension's limit) and whose
// box of `row_bytes`-byte rows is a multiple of 128 bytes, since every box lands at a 128-byte
// aligned shared-memory address.  0 when no such divisor exists.
__host__ __device__ constexpr int tma_rows(int N, int row_bytes) {
    for (int b = N < 256 ? N : 256; b > 0; b--)
        if (N % b == 0 && (b * row_bytes) % 128 == 0) return b;
    return 0;
}

// OOP: out-of-place Stockham stages through one more tile of shared memory (one barrier per stage,
// one butterfly in registers at a time); the in-place stages otherwise.
// YZ (x pass with EPI only): the fields are laid out (x, k_z, y) with y fastest, so a tile holds CZ
// values of k_y at one k_z; CTAs take k_z fastest, so the CTAs writing neighbouring z of I run together.
// PRE (the adjoint's passes, one input per segment): the coefficients multiply the tile before the
// transform and the transformed tile is the output.
// SEED (with EPI): the adjoint's seed instead of the intensity, D = dL/dI S^2 conj(Amp) / (n V) (0 where
// I is at its floor) written as field seg.out[0] of a.out, in the unshifted field layout.
template <typename T, int N, int CZ, int NT, int VEC, bool EPI, bool XPASS, class RAD, int NBUF, bool OOP = false,
          bool YZ = false, bool PRE = false, bool SEED = false>
__global__ void __launch_bounds__(NT, NT <= 512 && sizeof(C_t<T>) * (N * CZ * (NBUF + (OOP ? 1 : 0)) + N) <= 110 * 1024 ? 2 : 1)
    axis_tma(const __grid_constant__ CUtensorMap map, AxisArgs<T> a) {
    using C = C_t<T>;
    static_assert(CZ % VEC == 0, "chunk must hold whole vectors");
    constexpr int NO = 1;  // the host builds single-output segments for this kernel
    constexpr int TILE = N * CZ;
    constexpr int GROUPS = TILE / VEC;
    constexpr int EP = cdiv(GROUPS, NT);
    constexpr int CV = CZ / VEC;
    constexpr int BOX = tma_rows(N, CZ * (int)sizeof(C));
    static_assert(BOX > 0 && N % BOX == 0, "rows must split into whole boxes of 128-byte multiples");
    static_assert((TILE * sizeof(C)) % 128 == 0, "tile buffers must start 128-byte aligned");
    constexpr uint32_t BYTES = TILE * sizeof(C);
    using GE = Geo<CZ, CZ, 1, 0, CZ, NT>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* bufs = reinterpret_cast<C*>(smem_raw);
    C* tw = bufs + NBUF * TILE;  // twiddles, N values
    C* scratch = tw + N;         // OOP: the second buffer of the out-of-place stages
    __shared__ __align__(8) uint64_t bar[NBUF];
    static_assert(!YZ || (EPI && XPASS), "the y-fastest layout is read by the x pass only");
    static_assert(!PRE || (!EPI && !YZ), "the pre-multiplied passes store fields");
    static_assert(!SEED || (EPI && XPASS && !YZ), "the seed is an x-pass epilogue");
    const int tid = threadIdx.x;
    const long long outer = YZ ? blockIdx.x % a.nouter : blockIdx.x / a.nzc;
    const int z0 = (int)(YZ ? blockIdx.x / a.nouter : blockIdx.x % a.nzc) * CZ;
    const int cz = min(CZ, a.nz - z0);
    const long long base = outer * a.ostride + z0;
    for (int i = tid; i < N; i += NT) tw[i] = static_cast<const C*>(a.ap.tw)[i];
    const int nfx = (int)(XPASS ? a.nx : a.nx);  // rows of one field in the map's outer dimension: nx

    int total = 0;
    for (int sg = 0; sg < a.nseg; sg++) total += a.segs[sg].nin;

    // field of the flat input index fl
    auto field_of = [&](int fl) {
        for (int sg = 0; sg < a.nseg; sg++) {
            const int k = a.segs[sg].nin;
            if (fl < k) return a.segs[sg].in[fl];
            fl -= k;
        }
        return 0;
    };
    auto issue = [&](int fl, int b) {
        const int f = field_of(fl);
        C* dst = bufs + b * TILE;
        mbar_expect_tx(&bar[b], BYTES);
#pragma unroll
        for (int k = 0; k < N / BOX; k++) {
            if (XPASS) tma_load_3d(dst + k * BOX * CZ, &map, &bar[b], 2 * z0, (int)outer, f * nfx + k * BOX);
            else tma_load_3d(dst + k * BOX * CZ, &map, &bar[b], 2 * z0, k * BOX, f * nfx + (int)outer);
        }
    };

    if (smem_u32(smem_raw) % 128 != 0) {  // TMA destinations must be 128-byte aligned: refuse, do not load
        if (tid == 0) atomicExch(a.status, QPD_DEVERR_ALIGN);
        return;
    }
    if (tid == 0) {
        for (int b = 0; b < NBUF; b++) mbar_init(&bar[b], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int b = 0; b < NBUF && b < total; b++) issue(b, b);

    int fl = 0;
    for (int sg = 0; sg < a.nseg; sg++) {
        const Segment<T>& seg = a.segs[sg];
        C acc[NO][EP][VEC];
#pragma unroll
        for (int o = 0; o < NO; o++)
#pragma unroll
            for (int q = 0; q < EP; q++)
#pragma unroll
                for (int w = 0; w < VEC; w++) acc[o][q][w] = cmake<C>(0, 0);
        for (int fi = 0; fi < seg.nin; fi++, fl++) {
            const int b = fl % NBUF;
            C* buf = bufs + b * TILE;
            // this thread's coefficients for the field, fetched before the wait
            const C* cf = seg.coef[0][fi];
            C cfr[EP];
            if (!seg.ident && cf) {
#pragma unroll
                for (int q = 0; q < EP; q++) {
                    const int e = tid + q * NT;
                    cfr[q] = (GROUPS % NT == 0 || e < GROUPS) ? cf[e / CV] : cmake<C>(0, 0);
                }
            }
            const bool ok = mbar_wait(&bar[b], (fl / NBUF) & 1, a.status);
            if (!__syncthreads_and(ok)) {
                // a load never completed: give the other buffers' loads a bounded chance to land, then stop
                if (tid == 0)
                    for (int k = 1; k < NBUF && fl + k < total; k++)
                        mbar_wait(&bar[(fl + k) % NBUF], ((fl + k) / NBUF) & 1, nullptr);
                return;
            }
            if constexpr (PRE) {
                if (cf) {
                    for (int e = tid; e < TILE; e += NT) buf[e] = cmul(cf[e / CZ], buf[e]);
                    __syncthreads();
                }
            }
            C* res = buf;
            if constexpr (OOP) res = fft_oop<T, N, GE>(buf, scratch, TwFull<C>{tw}, tid, RAD{});
            else fft_ct<T, N, GE>(buf, tw, tid, RAD{});
            const bool mine = seg.ident ? (fi == 0) : (cf != nullptr);
            if (mine) {
#pragma unroll
                for (int q = 0; q < EP; q++) {
                    const int e = tid + q * NT;
                    if (GROUPS % NT == 0 || e < GROUPS) {
                        const int k = e / CV;
                        const int c = (e - k * CV) * VEC;
                        const C* s = res + (OOP ? oop_swz(k) : k) * CZ + c;
                        if (PRE || seg.ident) {
#pragma unroll
                            for (int w = 0; w < VEC; w++) acc[0][q][w] = cadd(acc[0][q][w], s[w]);
                        } else {
#pragma unroll
                            for (int w = 0; w < VEC; w++) cfma(acc[0][q][w], cfr[q], s[w]);
                        }
                    }
                }
            }
            __syncthreads();  // buffer b free again
            if (tid == 0 && fl + NBUF < total) {
                fence_proxy_async();
                issue(fl + NBUF, b);
            }
        }
        if constexpr (EPI && SEED) {
            const long long ky = outer;
            const int sy = fftshift_at((int)ky, (int)a.ny);
            const double syv = a.S[1][ky];
            C* dst = a.out + seg.out[0] * a.fstride + base;
#pragma unroll
            for (int q = 0; q < EP; q++) {
                const int e = tid + q * NT;
                if (GROUPS % NT == 0 || e < GROUPS) {
                    const int kx = e / CV;
                    const int c = (e - kx * CV) * VEC;
                    const double sxy = a.S[0][kx] * syv;
                    const long long row = ((long long)fftshift_at(kx, (int)a.nx) * a.ny + sy) * a.nz;
#pragma unroll
                    for (int w = 0; w < VEC; w++) {
                        const int kz = z0 + c + w;
                        if (c + w < cz) {
                            const double S = sxy * a.S[2][kz];
                            const double S2 = S * S * a.scale2;
                            const double re = (double)acc[0][q][w].x, im = (double)acc[0][q][w].y;
                            double f = 0.0;
                            if (S2 * (re * re + im * im) > 1e-50) f = a.gI[row + fftshift_at(kz, a.nz)] * S2;
                            dst[kx * a.stride + c + w] = cmake<C>(T(f * re), T(-f * im));
                        }
                    }
                }
            }
        } else if constexpr (EPI && YZ) {
            // outer = k_z, z0 + c + w = k_y; I is (x, y, z) with z fastest
            const long long nzr = a.nouter;
            const long long kz = outer;
            const long long sz = (kz + nzr / 2) % nzr;
            const double szv = a.S[2][kz];
#pragma unroll
            for (int q = 0; q < EP; q++) {
                const int e = tid + q * NT;
                if (GROUPS % NT == 0 || e < GROUPS) {
                    const int kx = e / CV;
                    const int c = (e - kx * CV) * VEC;
                    const double sxz = a.S[0][kx] * szv;
                    const long long row = (long long)fftshift_at(kx, (int)a.nx) * a.ny;
#pragma unroll
                    for (int w = 0; w < VEC; w++) {
                        const int ky = z0 + c + w;
                        if (c + w < cz) {
                            const double S = sxz * a.S[1][ky];
                            const double re = (double)acc[0][q][w].x, im = (double)acc[0][q][w].y;
                            const double v = floor_1e50(S * S * (re * re + im * im) * a.scale2);
                            a.I[(row + fftshift_at(ky, (int)a.ny)) * nzr + sz] = v;
                        }
                    }
                }
            }
        } else if (EPI) {
            const long long ky = outer;
            const long long sy = (ky + a.ny / 2) % a.ny;
            const double syv = a.S[1][ky];
#pragma unroll
            for (int q = 0; q < EP; q++) {
                const int e = tid + q * NT;
                if (GROUPS % NT == 0 || e < GROUPS) {
                    const int kx = e / CV;
                    const int c = (e - kx * CV) * VEC;
                    const double sxy = a.S[0][kx] * syv;
                    const long long row = ((long long)fftshift_at(kx, (int)a.nx) * a.ny + sy) * a.nz;
#pragma unroll
                    for (int w = 0; w < VEC; w++) {
                        const int kz = z0 + c + w;
                        if (c + w < cz) {
                            const double S = sxy * a.S[2][kz];
                            const double re = (double)acc[0][q][w].x, im = (double)acc[0][q][w].y;
                            const double v = floor_1e50(S * S * (re * re + im * im) * a.scale2);
                            a.I[row + fftshift_at(kz, a.nz)] = v;
                        }
                    }
                }
            }
        } else {
#pragma unroll
            for (int o = 0; o < NO; o++) {
                if (o >= seg.nout) break;
                C* dst = a.out + seg.out[o] * a.fstride + base;
#pragma unroll
                for (int q = 0; q < EP; q++) {
                    const int e = tid + q * NT;
                    if (GROUPS % NT == 0 || e < GROUPS) {
                        const int i = e / CV;
                        const int c = (e - i * CV) * VEC;
                        if (c < cz) {
                            C* d = dst + i * a.stride + c;
                            C v[VEC];
#pragma unroll
                            for (int w = 0; w < VEC; w++) v[w] = acc[o][q][w];
                            if (a.accumulate) {
#pragma unroll
                                for (int w = 0; w < VEC; w++) v[w] = cadd(v[w], d[w]);
                            }
                            if constexpr (VEC == 2) {
                                *reinterpret_cast<float4*>(d) = *reinterpret_cast<const float4*>(v);
                            } else {
                                d[0] = v[0];
                            }
                        }
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// Adjoint z stage with a compile-time transform (the adj_zstage_kernel of qpd_kernels.cuh for the
// lengths the forward specialises): per atom, the group's 3 conjugate adjoint fields times the z
// factors become 4 pencils per column, transformed along z in shared memory; each cell then adds
// its source transpose to dL/du and dL/dP held in registers.  The next atom's 3 fields arrive in a
// second staging buffer by per-thread asynchronous copies while the current atom is transformed.
// ---------------------------------------------------------------------------------------
template <typename T, int NZ, int M, int NT, class RAD>
__global__ void __launch_bounds__(NT, 2) adj_zstage_fast(AdjZArgs<T> a) {
    using C = C_t<T>;
    constexpr int PS = NZ % 2 ? NZ : NZ + 1;
    constexpr int PLANE = M * PS;
    constexpr int CELLS = M * NZ;
    constexpr int CPT = cdiv(CELLS, NT);
    using GE = Geo<4 * M, 4 * M, PS, 0, 1, NT>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    C* stg = buf + 4 * PLANE;  // 2 stages x 3 fields x CELLS: each thread's cells of one atom's fields
    const ZArgs<T>& z = a.z;
    AtomPhase<T>* apc = reinterpret_cast<AtomPhase<T>*>(stg + 6 * CELLS);
    const int tid = threadIdx.x;
    const int nap = z.in.nPhase * z.nAtom;
    for (int i = tid; i < nap; i += NT) apc[i] = z.apc[i];
    const long long c0 = (long long)blockIdx.x * M;
    const int ncell = (int)min((long long)M, z.ncols - c0) * NZ;
    const long long g0 = c0 * NZ;
    const C* tw = static_cast<const C*>(z.zp.tw);

    CellIn<T> cell[CPT];
    int ph[CPT];
    T wt[CPT], dU[CPT][3], dP[CPT][3];
#pragma unroll
    for (int q = 0; q < CPT; q++) {
        const int e = tid + q * NT;
        ph[q] = -1;
        wt[q] = T(0);
#pragma unroll
        for (int d = 0; d < 3; d++) dU[q][d] = dP[q][d] = T(0);
        if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
            const long long g = g0 + e;
            load_cell<T>(z.in, g, z.tq, cell[q]);
            ph[q] = z.in.phase[g];
            wt[q] = z.in.weight ? z.in.weight[g] : T(1);
        }
    }
    // atom at's 3 fields at this thread's cells into stage sb (the thread later reads only these slots)
    auto stage = [&](int at, int sb) {
        const C* fa = a.fin + 3LL * z.grp[at] * z.fstride + g0;
        C* d = stg + sb * 3 * CELLS;
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            const int e = tid + q * NT;
            if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
                cp_async<sizeof(C)>(d + e, fa + e);
                cp_async<sizeof(C)>(d + CELLS + e, fa + z.fstride + e);
                cp_async<sizeof(C)>(d + 2 * CELLS + e, fa + 2 * z.fstride + e);
            }
        }
        cp_async_commit();
    };
    if (z.nAtom > 0) stage(0, 0);
    __syncthreads();
    for (int at = 0; at < z.nAtom; at++) {
        // the next atom's copies go into the other stage (last read two barriers ago); an empty group
        // after the last atom keeps the count, so waiting for all but one group is atom at's data
        if (at + 1 < z.nAtom) stage(at + 1, (at + 1) & 1);
        else cp_async_commit();
        cp_async_wait<1>();
        const C* sa = stg + (at & 1) * 3 * CELLS;
        const C* ce = z.coefE + (long long)at * NZ;
        const C* cu = z.coefUz + (long long)at * NZ;
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            const int e = tid + q * NT;
            if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
                const int m = e / NZ;
                const int kz = e - m * NZ;
                const int s = m * PS + kz;
                const C A = sa[e], X = sa[CELLS + e], Y = sa[2 * CELLS + e];
                const C e1 = ce[kz], u1 = cu[kz];
                buf[s] = cmul(e1, A);
                buf[PLANE + s] = cmul(e1, X);
                buf[2 * PLANE + s] = cmul(e1, Y);
                buf[3 * PLANE + s] = cmul(u1, A);
            }
        }
        __syncthreads();
        fft_ct<T, NZ, GE>(buf, tw, tid, RAD{});
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            const int e = tid + q * NT;
            if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
                const int m = e / NZ;
                const int s = m * PS + OutPos<RAD>::at(e - m * NZ);
                if (ph[q] >= 0 && ph[q] < z.in.nPhase)
                    add_adjoint<T>(cell[q], apc[ph[q] * z.nAtom + at], wt[q], a.qc, buf[s], buf[PLANE + s],
                                   buf[2 * PLANE + s], buf[3 * PLANE + s], dU[q], dP[q]);
            }
        }
        __syncthreads();
    }
    cp_async_wait<0>();
#pragma unroll
    for (int q = 0; q < CPT; q++) {
        const int e = tid + q * NT;
        if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
            const long long g = g0 + e;
#pragma unroll
            for (int d = 0; d < 3; d++) {
                a.dU[d * z.in.n + g] = dU[q][d];
                a.dP[d * z.in.n + g] = d < z.in.nStruc ? dP[q][d] : T(0);
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// y pass over fields laid out (x, k_z, y), y fastest: one pencil (x, k_z) of N contiguous values per
// CTA.  Each input field's pencil arrives by 1-D bulk copies in one of two buffers while the
// previous field is transformed (out-of-place swizzled stages through a third buffer, twiddles from
// a two-level table) and folded into this thread's accumulators; the outputs go back in place, in
// the same layout (the CTA owns its pencil in every field).  Three pencils of shared memory, so two
// CTAs share an SM even for N = 4000.
// ---------------------------------------------------------------------------------------
template <typename T, int N, int NT, class RAD>
__global__ void __launch_bounds__(NT, 2) axis_bulk(AxisArgs<T> a) {
    using C = C_t<T>;
    constexpr int NBUF = 2, PIECES = 4;
    constexpr int EP = cdiv(N, NT);
    constexpr uint32_t BYTES = N * sizeof(C);
    static_assert(BYTES % (16 * PIECES) == 0 && N % PIECES == 0, "bulk copies of 16-byte multiples");
    constexpr int NHI = (N + 63) / 64;
    using GE = Geo<1, 1, 0, 0, 1, NT>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* bufs = reinterpret_cast<C*>(smem_raw);
    C* scratch = bufs + NBUF * N;
    C* thi = scratch + N;
    C* tlo = thi + NHI;
    __shared__ __align__(8) uint64_t bar[NBUF];
    const int tid = threadIdx.x;
    const long long pencil = blockIdx.x;  // x nz + k_z; its values start at pencil * N in every field
    const C* twg = static_cast<const C*>(a.ap.tw);
    for (int i = tid; i < NHI; i += NT) thi[i] = twg[64 * i];
    for (int i = tid; i < 64; i += NT) tlo[i] = twg[i];
    int total = 0;
    for (int sg = 0; sg < a.nseg; sg++) total += a.segs[sg].nin;
    auto field_of = [&](int fl) {
        for (int sg = 0; sg < a.nseg; sg++) {
            const int k = a.segs[sg].nin;
            if (fl < k) return a.segs[sg].in[fl];
            fl -= k;
        }
        return 0;
    };
    auto issue = [&](int fl, int b) {
        const C* src = a.in + (long long)field_of(fl) * a.fstride + pencil * N;
        C* dst = bufs + b * N;
        mbar_expect_tx(&bar[b], BYTES);
#pragma unroll
        for (int k = 0; k < PIECES; k++) bulk_load(dst + k * (N / PIECES), src + k * (N / PIECES), BYTES / PIECES, &bar[b]);
    };
    if (smem_u32(smem_raw) % 16 != 0 || reinterpret_cast<uintptr_t>(a.in) % 16 != 0 ||
        (a.fstride * sizeof(C)) % 16 != 0) {  // bulk copies need 16-byte aligned addresses: refuse, do not load
        if (tid == 0) atomicExch(a.status, QPD_DEVERR_ALIGN);
        return;
    }
    if (tid == 0) {
        for (int b = 0; b < NBUF; b++) mbar_init(&bar[b], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int b = 0; b < NBUF && b < total; b++) issue(b, b);
    const TwTwoLevel<C> tw{thi, tlo};

    int fl = 0;
    for (int sg = 0; sg < a.nseg; sg++) {
        const Segment<T>& seg = a.segs[sg];
        C acc[EP];
#pragma unroll
        for (int q = 0; q < EP; q++) acc[q] = cmake<C>(0, 0);
        for (int fi = 0; fi < seg.nin; fi++, fl++) {
            const int b = fl % NBUF;
            C* buf = bufs + b * N;
            const C* cf = seg.coef[0][fi];
            const bool ok = mbar_wait(&bar[b], (fl / NBUF) & 1, a.status);
            if (!__syncthreads_and(ok)) {
                if (tid == 0)
                    for (int k = 1; k < NBUF && fl + k < total; k++)
                        mbar_wait(&bar[(fl + k) % NBUF], ((fl + k) / NBUF) & 1, nullptr);
                return;
            }
            const C* res = fft_oop<T, N, GE>(buf, scratch, tw, tid, RAD{});
            if (cf) {  // coefficients read after the transform: fewer live registers
#pragma unroll
                for (int q = 0; q < EP; q++) {
                    const int e = tid + q * NT;
                    if (N % NT == 0 || e < N) cfma(acc[q], cf[e], res[oop_swz(e)]);
                }
            }
            __syncthreads();  // buffer b and the scratch buffer are free again
            if (tid == 0 && fl + NBUF < total) {
                fence_proxy_async();
                issue(fl + NBUF, b);
            }
        }
        C* dst = a.out + (long long)seg.out[0] * a.fstride + pencil * N;
#pragma unroll
        for (int q = 0; q < EP; q++) {
            const int e = tid + q * NT;
            if (N % NT == 0 || e < N) dst[e] = acc[q];
        }
    }
}

// ---------------------------------------------------------------------------------------
// z stage, persistent and pipelined: each CTA walks tiles of M columns (blockIdx.x, + gridDim.x,
// ...).  A tile's inputs (P, U, the phase index and weight) arrive in one of two shared-memory
// buffers by 1-D bulk copies issued a tile ahead, so the loads of tile i+1 overlap the source
// evaluation, the z transforms and the fold of tile i.  Each thread keeps only its cells'
// accumulators in registers.  A tile whose planes are not 16-byte aligned (only a partial last
// tile can be) is loaded by the threads instead.
// ---------------------------------------------------------------------------------------
template <typename T, int NZ, int M> struct ZLayout {
    static constexpr int PS = NZ % 2 ? NZ : NZ + 1;
    static constexpr int PLANE = M * PS;
    static constexpr int CELLS = M * NZ;
    static constexpr int CELLS16 = (CELLS + 15) / 16 * 16;
    // one input buffer: P, U (6 CELLS T) | weight (CELLS T) | phase (CELLS16 int8), 16-byte multiple
    static constexpr size_t INB = (sizeof(T) * 7 * CELLS + CELLS16 + 15) / 16 * 16;
    static constexpr size_t BUF = sizeof(C_t<T>) * 4 * PLANE;
    static constexpr size_t bytes(int nap, int nAtom) {
        return BUF + 2 * INB + sizeof(double) * CELLS + sizeof(C_t<T>) * NZ + sizeof(AtomPhase<T>) * nap +
               sizeof(C_t<T>) * 2 * nAtom * NZ + 64;
    }
};

template <typename T, int NZ, int M, int NT, class RAD, bool REGIN = false>
__global__ void __launch_bounds__(NT, 2) zstage_pipe(ZArgs<T> a) {
    using C = C_t<T>;
    using L = ZLayout<T, NZ, M>;
    constexpr int PS = L::PS, PLANE = L::PLANE, CELLS = L::CELLS;
    constexpr int CPT = cdiv(CELLS, NT);
    using GE = Geo<4 * M, 4 * M, PS, 0, 1, NT>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    unsigned char* inb = smem_raw + L::BUF;  // two input buffers of L::INB bytes
    double* stu = reinterpret_cast<double*>(inb + 2 * L::INB);
    C* stw = reinterpret_cast<C*>(stu + CELLS);
    AtomPhase<T>* apc = reinterpret_cast<AtomPhase<T>*>(stw + NZ);
    C* sce = reinterpret_cast<C*>(apc + a.in.nPhase * a.nAtom);  // [at][kz] exp(-i (k_z + G_z) R_z)
    C* scu = sce + a.nAtom * NZ;                                  // [at][kz] -i k_z times that
    __shared__ __align__(8) uint64_t bar[2];
    const int tid = threadIdx.x;
    const int nap = a.in.nPhase * a.nAtom;
    for (int i = tid; i < nap; i += NT) apc[i] = a.apc[i];
    for (int i = tid; i < NZ; i += NT) stw[i] = static_cast<const C*>(a.zp.tw)[i];
    for (int i = tid; i < a.nAtom * NZ; i += NT) {
        sce[i] = a.coefE[i];
        scu[i] = a.coefUz[i];
    }

    if (smem_u32(smem_raw) % 16 != 0) {  // bulk-copy destinations must be 16-byte aligned: refuse, do not load
        if (tid == 0) atomicExch(a.status, QPD_DEVERR_ALIGN);
        return;
    }
    const bool single = a.in.wdense == nullptr;
    const long long ntiles = (a.ncols + M - 1) / M;
    const bool aligned = (a.in.n * sizeof(T)) % 16 == 0 && a.in.nStruc == 3 &&
                         (reinterpret_cast<uintptr_t>(a.in.P) | reinterpret_cast<uintptr_t>(a.in.U) |
                          reinterpret_cast<uintptr_t>(a.in.phase) | reinterpret_cast<uintptr_t>(a.in.weight)) % 16 == 0;
    auto ncell_of = [&](long long t) { return (int)min((long long)M, a.ncols - t * M) * NZ; };
    // Every full tile starts at a multiple of CELLS, so whether full tiles can use bulk copies is a
    // property of the tile shape: all of a CTA's full tiles do, or none does.  That keeps the
    // barrier phases in step with the tile count; only the partial last tile loads by threads.
    constexpr bool TILE_BULK = (CELLS * sizeof(T)) % 16 == 0;
    const bool bulk_mode = aligned && TILE_BULK && (!single || CELLS % 16 == 0);
    auto bulk_ok = [&](long long t) { return bulk_mode && ncell_of(t) == CELLS; };
    auto issue = [&](long long t, int b) {
        const int nc = ncell_of(t);
        const long long g0 = t * M * NZ;
        T* sin_ = reinterpret_cast<T*>(inb + b * L::INB);
        T* swt = sin_ + 6 * CELLS;
        signed char* sph = reinterpret_cast<signed char*>(swt + CELLS);
        const uint32_t pb = nc * sizeof(T);
        mbar_expect_tx(&bar[b], 6 * pb + (single ? nc + (a.in.weight ? pb : 0) : 0));
        for (int k = 0; k < 3; k++) {
            bulk_load(sin_ + k * CELLS, a.in.P + k * a.in.n + g0, pb, &bar[b]);
            bulk_load(sin_ + (3 + k) * CELLS, a.in.U + k * a.in.n + g0, pb, &bar[b]);
        }
        if (single) {
            bulk_load(sph, a.in.phase + g0, nc, &bar[b]);
            if (a.in.weight) bulk_load(swt, a.in.weight + g0, pb, &bar[b]);
        }
    };

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0) {
        for (int k = 0; k < 2; k++) {
            const long long t = blockIdx.x + (long long)k * gridDim.x;
            if (t < ntiles && bulk_ok(t)) issue(t, k);
        }
    }

    // this thread's cells: source slot and output slot in the tile (atom-independent)
    int ssrc[CPT], sout[CPT];
#pragma unroll
    for (int q = 0; q < CPT; q++) {
        const int e = tid + q * NT;
        const int m = e / NZ;
        const int z = e - m * NZ;
        ssrc[q] = m * PS + z;
        sout[q] = m * PS + OutPos<RAD>::at(z);
    }

    for (int it = 0;; it++) {
        const long long t = blockIdx.x + (long long)it * gridDim.x;
        if (t >= ntiles) break;
        const int b = it & 1;
        const int ncell = ncell_of(t);
        const long long g0 = t * M * NZ;
        T* sin_ = reinterpret_cast<T*>(inb + b * L::INB);
        T* swt = sin_ + 6 * CELLS;
        signed char* sph = reinterpret_cast<signed char*>(swt + CELLS);
        if (bulk_ok(t)) {
            const bool ok = mbar_wait(&bar[b], (it >> 1) & 1, a.status);
            if (!__syncthreads_and(ok)) {
                if (tid == 0) {
                    const long long t2 = t + gridDim.x;
                    if (t2 < ntiles && bulk_ok(t2)) mbar_wait(&bar[b ^ 1], ((it + 1) >> 1) & 1, nullptr);
                }
                return;
            }
        } else {
            for (int e = tid; e < ncell; e += NT) {
                for (int k = 0; k < 3; k++) {
                    sin_[k * CELLS + e] = k < a.in.nStruc ? a.in.P[k * a.in.n + g0 + e] : T(0);
                    sin_[(3 + k) * CELLS + e] = a.in.U[k * a.in.n + g0 + e];
                }
                if (single) {
                    sph[e] = a.in.phase[g0 + e];
                    if (a.in.weight) swt[e] = a.in.weight[g0 + e];
                }
            }
            __syncthreads();
        }
        for (int e = tid; e < ncell; e += NT) {
            stu[e] = a.tq[0] * (double)sin_[3 * CELLS + e] + a.tq[1] * (double)sin_[4 * CELLS + e] +
                     a.tq[2] * (double)sin_[5 * CELLS + e];
            if (single && !a.in.weight) swt[e] = T(1);
        }
        __syncthreads();

        C accE[CPT], accX[CPT], accY[CPT];
#pragma unroll
        for (int q = 0; q < CPT; q++) accE[q] = accX[q] = accY[q] = cmake<C>(0, 0);
        // REGIN: each thread's cells' inputs stay in registers for all atoms
        CellIn<T> rcl[REGIN ? CPT : 1];
        int rph[REGIN ? CPT : 1];
        T rwt[REGIN ? CPT : 1];
        if constexpr (REGIN) {
#pragma unroll
            for (int q = 0; q < CPT; q++) {
                const int e = tid + q * NT;
                if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        rcl[q].p[k] = sin_[k * CELLS + e];
                        rcl[q].u[k] = sin_[(3 + k) * CELLS + e];
                    }
                    rcl[q].tu = stu[e];
                    rph[q] = single ? (int)sph[e] : -1;
                    rwt[q] = single ? swt[e] : T(0);
                }
            }
        }

        for (int at = 0; at < a.nAtom; at++) {
#pragma unroll
            for (int q = 0; q < CPT; q++) {
                const int e = tid + q * NT;
                if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
                    C E, X, Y, Z;
                    if constexpr (REGIN) {
                        cell_source<T>(a.in, g0 + e, rcl[q], rph[q], rwt[q], apc, a.nAtom, at, E, X, Y, Z);
                    } else {
                        CellIn<T> cl;
#pragma unroll
                        for (int k = 0; k < 3; k++) {
                            cl.p[k] = sin_[k * CELLS + e];
                            cl.u[k] = sin_[(3 + k) * CELLS + e];
                        }
                        cl.tu = stu[e];
                        cell_source<T>(a.in, g0 + e, cl, single ? (int)sph[e] : -1, single ? swt[e] : T(0), apc,
                                       a.nAtom, at, E, X, Y, Z);
                    }
                    const int s = ssrc[q];
                    buf[s] = E;
                    buf[PLANE + s] = X;
                    buf[2 * PLANE + s] = Y;
                    buf[3 * PLANE + s] = Z;
                }
            }
            __syncthreads();
            fft_ct<T, NZ, GE>(buf, stw, tid, RAD{});
            const C* ce = sce + at * NZ;
            const C* cu = scu + at * NZ;
#pragma unroll
            for (int q = 0; q < CPT; q++) {
                const int e = tid + q * NT;
                if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
                    const int kz = e % NZ;
                    const int s = sout[q];
                    const C e1 = ce[kz], u1 = cu[kz];
                    cfma(accE[q], e1, buf[s]);
                    cfma(accE[q], u1, buf[3 * PLANE + s]);
                    cfma(accX[q], e1, buf[PLANE + s]);
                    cfma(accY[q], e1, buf[2 * PLANE + s]);
                }
            }
            const int g = a.grp[at];
            if (at == a.nAtom - 1 || a.grp[at + 1] != g) {
                C* o = a.out + 3LL * g * a.fstride + g0;
#pragma unroll
                for (int q = 0; q < CPT; q++) {
                    const int e = tid + q * NT;
                    if ((CELLS % NT == 0 || e < CELLS) && e < ncell) {
                        o[e] = accE[q];
                        o[a.fstride + e] = accX[q];
                        o[2 * a.fstride + e] = accY[q];
                    }
                    accE[q] = accX[q] = accY[q] = cmake<C>(0, 0);
                }
            }
            __syncthreads();
        }
        // input buffer b is free: fetch the tile two steps ahead into it
        if (tid == 0) {
            const long long t2 = t + 2LL * gridDim.x;
            if (t2 < ntiles && bulk_ok(t2)) {
                fence_proxy_async();
                issue(t2, b);
            }
        }
    }
}

}  // namespace qpd
