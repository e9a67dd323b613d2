// Mixed-radix Stockham FFT over pencils held in shared memory.
//
// A CTA holds a tile of `count` pencils of length N in shared memory and transforms all of
// them together, forward (exp(-2 pi i j k / N)), unnormalised, results in natural order.
// Each radix-R stage reads a thread's butterflies into registers, applies the stage twiddles
// and the R-point DFT, waits at a CTA barrier, and writes the results back in place in
// Stockham (self-sorting) order: out[(j / Ns) Ns R + j % Ns + s Ns] = DFT_R(...)[s].
// Butterflies are numbered pencil-fastest, so neighbouring threads touch neighbouring
// pencils; tiles are laid out so that this is bank-conflict free (pencils contiguous,
// or pencil strides odd in 8-byte words).
#pragma once

#include "qpd_common.cuh"
#include "qpd_roots.cuh"

namespace qpd {

constexpr int kMaxStages = 24;

// One axis of the transform, passed to kernels by value.  tw points to N complex values
// exp(-2 pi i m / N), m = 0..N-1, computed in double on the host and stored in the kernel
// precision.  radix[] multiplies out to N; an axis of length 1 has no stage.
struct AxisPlan {
    int N;
    int nstages;
    int radix[kMaxStages];
    const void* tw;
};

// Where the pencils of a tile sit in shared memory: pencil pc starts at
// (pc / group) * gstride + (pc % group) * pstride and its elements are estride apart.
struct Pencils {
    int count;
    int group;
    int gstride;
    int pstride;
    int estride;
    __device__ __forceinline__ int base(int pc) const { return (pc / group) * gstride + (pc % group) * pstride; }
};

template <int R, typename C> struct Dft {
    // Odd R: pair r with R - r, y[s] = x0 + sum_r (cos a_r - i sin b_r), y[R - s] = x0 + sum_r (cos a_r + i sin b_r),
    // with a_r = x_r + x_{R-r}, b_r = x_r - x_{R-r}, angles 2 pi r s / R; the roots come from constant memory.
    __device__ __forceinline__ static void run(C (&x)[R]) {
        static_assert(R % 2 == 1 && root_offset(R) >= 0, "odd radix without a root table");
        using T = decltype(C::x);
        constexpr int H = (R - 1) / 2;
        C a[H], b[H];
#pragma unroll
        for (int r = 1; r <= H; r++) {
            a[r - 1] = cadd(x[r], x[R - r]);
            b[r - 1] = csub(x[r], x[R - r]);
        }
        C y0 = x[0];
#pragma unroll
        for (int r = 0; r < H; r++) y0 = cadd(y0, a[r]);
#pragma unroll
        for (int s = 1; s <= H; s++) {
            C A = x[0];
            C B = cmake<C>(0, 0);
#pragma unroll
            for (int r = 1; r <= H; r++) {
                const C w = unit_root<T>(root_offset(R) + (r * s) % R);
                const T c = w.x;
                const T sn = -w.y;
                caxpy(A, c, a[r - 1]);
                caxpy(B, sn, b[r - 1]);
            }
            x[s] = cadd_mi(A, B);
            x[R - s] = cadd_pi(A, B);
        }
        x[0] = y0;
    }
};

template <typename C> struct Dft<2, C> {
    __device__ __forceinline__ static void run(C (&x)[2]) {
        C a = x[0];
        x[0] = cadd(a, x[1]);
        x[1] = csub(a, x[1]);
    }
};

template <typename C> struct Dft<3, C> {
    __device__ __forceinline__ static void run(C (&x)[3]) {
        using R_t = decltype(C::x);
        const R_t h = R_t(0.86602540378443864676);  // sqrt(3) / 2
        C t = cadd(x[1], x[2]);
        C m = cmake<C>(x[0].x - R_t(0.5) * t.x, x[0].y - R_t(0.5) * t.y);
        C d = cscale(csub(x[1], x[2]), h);
        x[0] = cadd(x[0], t);
        x[1] = cadd_mi(m, d);
        x[2] = cadd_pi(m, d);
    }
};

template <typename C> __device__ __forceinline__ void dft4(C& x0, C& x1, C& x2, C& x3) {
    C a = cadd(x0, x2), b = csub(x0, x2), c = cadd(x1, x3), d = csub(x1, x3);
    x0 = cadd(a, c);
    x2 = csub(a, c);
    x1 = cadd_mi(b, d);  // b - i d
    x3 = cadd_pi(b, d);
}

template <typename C> struct Dft<4, C> {
    __device__ __forceinline__ static void run(C (&x)[4]) { dft4(x[0], x[1], x[2], x[3]); }
};

template <typename C> struct Dft<8, C> {
    __device__ __forceinline__ static void run(C (&x)[8]) {
        using R_t = decltype(C::x);
        const R_t r2 = R_t(0.70710678118654752440);  // 1 / sqrt(2)
        C e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6];
        C o0 = x[1], o1 = x[3], o2 = x[5], o3 = x[7];
        dft4(e0, e1, e2, e3);
        dft4(o0, o1, o2, o3);
        C t1 = cmake<C>((o1.x + o1.y) * r2, (o1.y - o1.x) * r2);   // exp(-i pi / 4) o1
        C t3 = cmake<C>((o3.y - o3.x) * r2, -(o3.x + o3.y) * r2);  // exp(-3 i pi / 4) o3
        x[0] = cadd(e0, o0);
        x[4] = csub(e0, o0);
        x[1] = cadd(e1, t1);
        x[5] = csub(e1, t1);
        x[2] = cadd_mi(e2, o2);  // exp(-i pi / 2) o2
        x[6] = cadd_pi(e2, o2);
        x[3] = cadd(e3, t3);
        x[7] = csub(e3, t3);
    }
};

__host__ __device__ constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }

// One radix-R stage over all pencils of the tile, in place.  BPT bounds the butterflies
// per thread: count * N <= EPT * nthreads with BPT = ceil(EPT / R).
template <typename T, int R, int BPT>
__device__ __forceinline__ void stage_r(C_t<T>* buf, const Pencils& pg, int N, int Ns, const C_t<T>* __restrict__ tw,
                                        int tid, int nt) {
    using C = C_t<T>;
    const int L = N / R;
    const int nb = pg.count * L;
    const int tstep = N / (Ns * R);
    C v[BPT][R];
    int ob[BPT];
#pragma unroll
    for (int q = 0; q < BPT; q++) {
        const int b = tid + q * nt;
        if (b < nb) {
            const int pc = b % pg.count;
            const int j = b / pg.count;
            const int k = j % Ns;
            const int pb = pg.base(pc);
#pragma unroll
            for (int r = 0; r < R; r++) v[q][r] = buf[pb + (j + r * L) * pg.estride];
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) v[q][r] = cmul(v[q][r], tw[r * k * tstep]);
            }
            Dft<R, C>::run(v[q]);
            ob[q] = pb + ((j / Ns) * Ns * R + k) * pg.estride;
        }
    }
    __syncthreads();
    const int os = Ns * pg.estride;
#pragma unroll
    for (int q = 0; q < BPT; q++) {
        const int b = tid + q * nt;
        if (b < nb) {
#pragma unroll
            for (int r = 0; r < R; r++) buf[ob[q] + r * os] = v[q][r];
        }
    }
    __syncthreads();
}

// Any radix, one thread per output: y_s = sum_r x_r W_N^(r k N/(Ns R) + (r s mod R) N/R).
// Used for prime factors without a specialised butterfly.
template <typename T, int EPT>
__device__ __noinline__ void stage_direct(C_t<T>* buf, const Pencils& pg, int N, int Ns, int R,
                                          const C_t<T>* __restrict__ tw, int tid, int nt) {
    using C = C_t<T>;
    const int L = N / R;
    const int ne = pg.count * N;
    const int tstep = N / (Ns * R);
    C out[EPT];
    int oa[EPT];
#pragma unroll
    for (int q = 0; q < EPT; q++) {
        const int e = tid + q * nt;
        if (e < ne) {
            const int pc = e % pg.count;
            const int rest = e / pg.count;
            const int j = rest % L;
            const int s = rest / L;
            const int k = j % Ns;
            const int pb = pg.base(pc);
            C acc = cmake<C>(0, 0);
            for (int r = 0; r < R; r++) {
                int idx = r * k * tstep + ((r * s) % R) * L;
                if (idx >= N) idx -= N;
                cfma(acc, buf[pb + (j + r * L) * pg.estride], tw[idx]);
            }
            out[q] = acc;
            oa[q] = pb + ((j / Ns) * Ns * R + k + s * Ns) * pg.estride;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < EPT; q++) {
        const int e = tid + q * nt;
        if (e < ne) buf[oa[q]] = out[q];
    }
    __syncthreads();
}

// Radices with a register butterfly; any other factor goes through stage_direct.
__host__ __device__ constexpr bool fast_radix(int r) {
    return r == 2 || r == 3 || r == 4 || r == 5 || r == 7 || r == 8 || r == 11 || r == 13 || r == 17;
}

// Forward FFT of every pencil of the tile.  All threads of the CTA must call it.
template <typename T, int EPT>
__device__ void fft_pencils(C_t<T>* buf, const Pencils& pg, const AxisPlan& ap, int tid, int nt) {
    using C = C_t<T>;
    const C* tw = static_cast<const C*>(ap.tw);
    const int N = ap.N;
    int Ns = 1;
    for (int s = 0; s < ap.nstages; s++) {
        const int R = ap.radix[s];
        switch (R) {
            case 2: stage_r<T, 2, cdiv(EPT, 2)>(buf, pg, N, Ns, tw, tid, nt); break;
            case 3: stage_r<T, 3, cdiv(EPT, 3)>(buf, pg, N, Ns, tw, tid, nt); break;
            case 4: stage_r<T, 4, cdiv(EPT, 4)>(buf, pg, N, Ns, tw, tid, nt); break;
            case 5: stage_r<T, 5, cdiv(EPT, 5)>(buf, pg, N, Ns, tw, tid, nt); break;
            case 7: stage_r<T, 7, cdiv(EPT, 7)>(buf, pg, N, Ns, tw, tid, nt); break;
            case 8: stage_r<T, 8, cdiv(EPT, 8)>(buf, pg, N, Ns, tw, tid, nt); break;
            case 11: stage_r<T, 11, cdiv(EPT, 11)>(buf, pg, N, Ns, tw, tid, nt); break;
            case 13: stage_r<T, 13, cdiv(EPT, 13)>(buf, pg, N, Ns, tw, tid, nt); break;
            case 17: stage_r<T, 17, cdiv(EPT, 17)>(buf, pg, N, Ns, tw, tid, nt); break;
            default: stage_direct<T, EPT>(buf, pg, N, Ns, R, tw, tid, nt); break;
        }
        Ns *= R;
    }
}

// ---------------------------------------------------------------------------------------
// Compile-time FFT: the axis length, the radices and the tile geometry are template
// parameters, so index arithmetic folds to constants and register arrays are exact.
// ---------------------------------------------------------------------------------------

// Tile geometry: COUNT pencils, pencil pc at (pc % G) * PSTR + (pc / G) * GSTR, elements ES apart,
// NT threads.
template <int COUNT_, int G_, int PSTR_, int GSTR_, int ES_, int NT_> struct Geo {
    static constexpr int COUNT = COUNT_, G = G_, PSTR = PSTR_, GSTR = GSTR_, ES = ES_, NT = NT_;
    __device__ __forceinline__ static int base(int pc) { return (pc % G) * PSTR + (pc / G) * GSTR; }
};

template <typename T, int N, int NS, int R, class GE>
__device__ __forceinline__ void stage_ct(C_t<T>* buf, const C_t<T>* __restrict__ tw, int t) {
    using C = C_t<T>;
    constexpr int L = N / R;
    constexpr int NB = GE::COUNT * L;
    constexpr int BPT = cdiv(NB, GE::NT);
    constexpr int TSTEP = N / (NS * R);
    C v[BPT][R];
    int ob[BPT];
#pragma unroll
    for (int q = 0; q < BPT; q++) {
        const int b = t + q * GE::NT;
        if (NB % GE::NT == 0 || b < NB) {
            const int pc = b % GE::COUNT;
            const int j = b / GE::COUNT;
            const int k = j % NS;
            const int pb = GE::base(pc);
#pragma unroll
            for (int r = 0; r < R; r++) v[q][r] = buf[pb + (j + r * L) * GE::ES];
            if (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) v[q][r] = cmul(v[q][r], tw[r * k * TSTEP]);
            }
            Dft<R, C>::run(v[q]);
            ob[q] = pb + ((j / NS) * NS * R + k) * GE::ES;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < BPT; q++) {
        const int b = t + q * GE::NT;
        if (NB % GE::NT == 0 || b < NB) {
#pragma unroll
            for (int r = 0; r < R; r++) buf[ob[q] + r * NS * GE::ES] = v[q][r];
        }
    }
    __syncthreads();
}

template <int... Rs> struct Radix {};

template <typename T, int N, int NS, class GE, int R, int... Rest>
__device__ __forceinline__ void fft_ct_(C_t<T>* buf, const C_t<T>* __restrict__ tw, int t) {
    stage_ct<T, N, NS, R, GE>(buf, tw, t);
    if constexpr (sizeof...(Rest) > 0) fft_ct_<T, N, NS * R, GE, Rest...>(buf, tw, t);
}

template <typename T, int N, class GE, int... Rs>
__device__ __forceinline__ void fft_ct(C_t<T>* buf, const C_t<T>* __restrict__ tw, int t, Radix<Rs...>) {
    if constexpr (sizeof...(Rs) > 0) fft_ct_<T, N, 1, GE, Rs...>(buf, tw, t);
}

// Out-of-place Stockham: stage s reads one buffer and writes the other, so a thread needs one
// butterfly in registers at a time and a stage needs a single barrier (its writes go to the buffer
// the previous stage read, whose reads all finished at that stage's barrier).  Returns the buffer
// that holds the result: `a` after an even number of stages, `b` after an odd one.
//
// Every buffer a stage writes holds element i at position oop_swz(i): the first stage writes
// elements R apart from neighbouring threads, which would put them on the same bank; the XOR of
// the element's block index into its low 3 bits spreads them.  It permutes within aligned blocks of
// 8 (N % 8 == 0), so contiguous reads stay conflict-free.  The input of the first stage (the loaded
// tile) is in natural order.
__device__ __forceinline__ int oop_swz(int i) { return i ^ ((i >> 3) & 7); }

// Twiddle exp(-2 pi i m / N): from a full table, or as the product of a coarse and a fine table
// (exp(-2 pi i 64 (m >> 6) / N) exp(-2 pi i (m & 63) / N), about N / 64 + 64 values in shared memory).
template <typename C> struct TwFull {
    const C* t;
    __device__ __forceinline__ C operator()(int m) const { return t[m]; }
};
template <typename C> struct TwTwoLevel {
    const C* hi;
    const C* lo;
    __device__ __forceinline__ C operator()(int m) const { return cmul(hi[m >> 6], lo[m & 63]); }
};

template <typename T, int N, int NS, int R, class GE, bool SWZ_IN, class TW>
__device__ __forceinline__ void stage_oop(const C_t<T>* __restrict__ src, C_t<T>* __restrict__ dst, const TW& tw,
                                          int t) {
    static_assert(N % 8 == 0, "the stage swizzle permutes blocks of 8");
    using C = C_t<T>;
    constexpr int L = N / R;
    constexpr int NB = GE::COUNT * L;
    constexpr int BPT = cdiv(NB, GE::NT);
    constexpr int TSTEP = N / (NS * R);
#pragma unroll 2
    for (int q = 0; q < BPT; q++) {
        const int b = t + q * GE::NT;
        if (NB % GE::NT == 0 || b < NB) {
            const int pc = b % GE::COUNT;
            const int j = b / GE::COUNT;
            const int k = j % NS;
            const int pb = GE::base(pc);
            C v[R];
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int i = j + r * L;
                v[r] = src[pb + (SWZ_IN ? oop_swz(i) : i) * GE::ES];
            }
            if (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) v[r] = cmul(v[r], tw(r * k * TSTEP));
            }
            Dft<R, C>::run(v);
            const int ob = (j / NS) * NS * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) dst[pb + oop_swz(ob + r * NS) * GE::ES] = v[r];
        }
    }
    __syncthreads();
}

template <typename T, int N, int NS, class GE, class TW, int R, int... Rest>
__device__ __forceinline__ C_t<T>* fft_oop_(C_t<T>* a, C_t<T>* b, const TW& tw, int t) {
    stage_oop<T, N, NS, R, GE, (NS > 1)>(a, b, tw, t);
    if constexpr (sizeof...(Rest) > 0) return fft_oop_<T, N, NS * R, GE, TW, Rest...>(b, a, tw, t);
    else return b;
}

// Result element k of pencil p sits at oop_swz(k) (see stage_oop).
template <typename T, int N, class GE, class TW, int... Rs>
__device__ __forceinline__ C_t<T>* fft_oop(C_t<T>* a, C_t<T>* b, const TW& tw, int t, Radix<Rs...>) {
    static_assert(sizeof...(Rs) > 0, "at least one stage");
    return fft_oop_<T, N, 1, GE, TW, Rs...>(a, b, tw, t);
}

// ---------------------------------------------------------------------------------------
// Prime-factor (Good-Thomas) FFT for N = N1 N2 with gcd(N1, N2) = 1: a 2-D DFT without twiddle
// factors.  Input x[n] is read as A0[n1][n2] = x[(N2 n1 + N1 n2) mod N]; stage A transforms over
// n1, stage B over n2, and X[k] ends at position (N2 (k mod N1) + N1 (k mod N2)) mod N.  Each
// butterfly writes back exactly the positions it read, so a stage needs no barrier between its
// loads and stores; one barrier separates the two stages.
// ---------------------------------------------------------------------------------------
template <int N1, int N2> struct Pfa {
    static constexpr int N = N1 * N2;
    // a < N1, b < N2, so N2 a + N1 b < 2 N: one conditional subtraction reduces it
    __host__ __device__ static constexpr int pos(int a, int b) {
        const int v = N2 * a + N1 * b;
        return v >= N ? v - N : v;
    }
    // where X[k] sits after the transform
    __host__ __device__ static constexpr int out_pos(int k) { return pos(k % N1, k % N2); }
};

template <typename T, int R, int OTHER, bool OVER_FIRST, class GE, class P>
__device__ __forceinline__ void pfa_stage(C_t<T>* buf, int t) {
    using C = C_t<T>;
    constexpr int NB = GE::COUNT * OTHER;  // butterflies: one per pencil and index of the other factor
    constexpr int BPT = cdiv(NB, GE::NT);
#pragma unroll
    for (int q = 0; q < BPT; q++) {
        const int b = t + q * GE::NT;
        if (NB % GE::NT == 0 || b < NB) {
            const int pc = b % GE::COUNT;
            const int o = b / GE::COUNT;
            const int pb = GE::base(pc);
            C v[R];
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = buf[pb + (OVER_FIRST ? P::pos(r, o) : P::pos(o, r)) * GE::ES];
            Dft<R, C>::run(v);
#pragma unroll
            for (int r = 0; r < R; r++) buf[pb + (OVER_FIRST ? P::pos(r, o) : P::pos(o, r)) * GE::ES] = v[r];
        }
    }
}

template <typename T, int N, class GE, int N1, int N2>
__device__ __forceinline__ void fft_ct(C_t<T>* buf, const C_t<T>* __restrict__, int t, Pfa<N1, N2>) {
    static_assert(N1 * N2 == N, "factors must multiply to N");
    pfa_stage<T, N1, N2, true, GE, Pfa<N1, N2>>(buf, t);
    __syncthreads();
    pfa_stage<T, N2, N1, false, GE, Pfa<N1, N2>>(buf, t);
    __syncthreads();
}

// Position of output k after fft_ct: natural order for Stockham, the CRT map for Pfa.
template <class RAD> struct OutPos {
    __host__ __device__ static constexpr int at(int k) { return k; }
};
template <int N1, int N2> struct OutPos<Pfa<N1, N2>> {
    __host__ __device__ static constexpr int at(int k) { return Pfa<N1, N2>::out_pos(k); }
};

}  // namespace qpd
