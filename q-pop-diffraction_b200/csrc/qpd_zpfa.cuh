// Fused z stage for prime-factor lengths nz = N1 * N2 (104 = 8 * 13, 68 = 4 * 17), single-phase
// packed inputs: source, z transform and fold with one trip through shared memory per value.
//
// The Good-Thomas transform of a column is a 2-D DFT without twiddles: with x[(N2 a + N1 b) mod N]
// as element (a, b), stage 1 transforms over a for every b, stage 2 over b for every a, and X[k]
// is element (k mod N1, k mod N2).  Between the stages element (a, b) sits at a N2 + b of its
// column, so stage-2 rows are contiguous and every index below is a constant offset.  Here
//   phase A (one item per (column, b) and lane half): the item's cells are exactly the inputs of
//     one stage-1 DFT, so each thread evaluates the 4 source components of its cells in
//     registers (their inputs stay in registers for every atom of the tile), transforms them
//     (for N1 = 8 as two 4-point halves on adjacent lanes joined by shuffles) and stores the
//     results once;
//   phase B (one item per (column, a, component)): loads N2 values, transforms them and folds
//     them straight into per-thread accumulators with exp(-i (k_z + G_z) R_z) (or -i k_z times it
//     for the z displacement component), across the atoms of an (R_x, R_y) group;
//   at the end of a group the accumulators go through shared memory once more so the group's 3
//     fields leave in coalesced rows (E = the E and U_z items' sum, X, Y).
// Shared memory is written and read once per value and atom (the Stockham z stage does it three
// times).  The fold coefficients are permuted into the same (a, r) order once per CTA.  Item orders
// and the pencil stride were chosen with a bank model so that the phase-B loads are conflict-free.
// Two exchange buffers let phase A of the next atom run in the same barrier interval as phase B of
// the current one (one CTA barrier per atom); the tile's inputs move to registers at its start, so a
// single input buffer takes the next tile's bulk copies while the atoms run.
#pragma once

#include "qpd_fast.cuh"

namespace qpd {

template <int N1, int N2> struct ZPfa;

template <> struct ZPfa<8, 13> {
    static constexpr int M = 8, NT = 256, SPLIT = 2, PS = 105;
    // phase A item t -> (column m, b, half h): h fastest, then m, then b
    __device__ static void itemA(int t, int& m, int& b, int& h) {
        h = t & 1;
        m = (t >> 1) % M;
        b = (t >> 1) / M;
    }
    // phase B item t -> (component, column m, a): a fastest, then the component, then m
    __device__ static void itemB(int t, int& comp, int& m, int& a) {
        a = t % 8;
        comp = (t / 8) % 4;
        m = t / 32;
    }
};

template <> struct ZPfa<4, 17> {
    static constexpr int M = 12, NT = 224, SPLIT = 1, PS = 81;
    __device__ static void itemA(int t, int& m, int& b, int& h) {
        h = 0;
        b = t % 17;
        m = t / 17;
    }
    __device__ static void itemB(int t, int& comp, int& m, int& a) {
        a = t % 4;
        comp = (t / 4) % 4;
        m = t / 16;
    }
};

// CRT idempotents: e1 = 1 mod N1, 0 mod N2; e2 = 0 mod N1, 1 mod N2
__host__ __device__ constexpr int crt_e(int Na, int Nb) {
    int e = 0;
    while ((e % Na) != 1 % Na) e += Nb;
    return e;
}

template <typename T, int N1, int N2> struct ZPfaLayout {
    using TR = ZPfa<N1, N2>;
    static constexpr int NZ = N1 * N2, M = TR::M, PS = TR::PS, PLANE = M * PS, CELLS = M * NZ;
    static constexpr int CELLS16 = (CELLS + 15) / 16 * 16;
    static constexpr size_t BUF = sizeof(C_t<T>) * 4 * PLANE;
    static constexpr size_t INB = (sizeof(T) * 7 * CELLS + CELLS16 + 15) / 16 * 16;
    // two exchange buffers (one per atom in flight), one input buffer
    static size_t bytes(int nap, int nAtom) {
        return 2 * BUF + INB + sizeof(AtomPhase<T>) * nap + sizeof(C_t<T>) * 2 * nAtom * NZ + 64;
    }
};

template <typename T, int N1, int N2>
__global__ void __launch_bounds__(ZPfa<N1, N2>::NT, 2) zstage_pfa(ZArgs<T> a) {
    using C = C_t<T>;
    using TR = ZPfa<N1, N2>;
    using L = ZPfaLayout<T, N1, N2>;
    constexpr int NZ = L::NZ, M = L::M, PS = L::PS, PLANE = L::PLANE, CELLS = L::CELLS, NT = TR::NT;
    constexpr int SPLIT = TR::SPLIT, CPA = N1 / SPLIT;
    constexpr int IA = SPLIT * M * N2, IB = 4 * M * N1;
    constexpr int E1 = crt_e(N1, N2), E2 = crt_e(N2, N1);
    static_assert(IA <= NT && IB <= NT && NT % 32 == 0, "one phase-A and one phase-B item per thread");
    static_assert(SPLIT == 1 || (SPLIT == 2 && N1 == 8), "lane pairs split an 8-point DFT only");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* const xb0 = reinterpret_cast<C*>(smem_raw);  // exchange buffers: atom at uses xb[at & 1]
    C* const xb1 = xb0 + 4 * PLANE;
    unsigned char* inb = smem_raw + 2 * L::BUF;
    AtomPhase<T>* apc = reinterpret_cast<AtomPhase<T>*>(inb + L::INB);
    C* sce = reinterpret_cast<C*>(apc + a.in.nPhase * a.nAtom);
    C* scu = sce + a.nAtom * NZ;
    __shared__ __align__(8) uint64_t bar;
    const int tid = threadIdx.x;
    const int nap = a.in.nPhase * a.nAtom;
    for (int i = tid; i < nap; i += NT) apc[i] = a.apc[i];
    for (int i = tid; i < a.nAtom * NZ; i += NT) {  // [at][a][r] = table[at][k], k = (a mod N1, r mod N2)
        const int at = i / NZ, rem = i - at * NZ, ia = rem / N2, r = rem - ia * N2;
        const int k = (ia * E1 + r * E2) % NZ;
        sce[i] = a.coefE[at * NZ + k];
        scu[i] = a.coefUz[at * NZ + k];
    }
    if (smem_u32(smem_raw) % 16 != 0) {
        if (tid == 0) atomicExch(a.status, QPD_DEVERR_ALIGN);
        return;
    }
    const long long ntiles = (a.ncols + M - 1) / M;
    const bool aligned = (a.in.n * sizeof(T)) % 16 == 0 && a.in.nStruc == 3 &&
                         (reinterpret_cast<uintptr_t>(a.in.P) | reinterpret_cast<uintptr_t>(a.in.U) |
                          reinterpret_cast<uintptr_t>(a.in.phase) | reinterpret_cast<uintptr_t>(a.in.weight)) % 16 == 0;
    auto ncell_of = [&](long long t) { return (int)min((long long)M, a.ncols - t * M) * NZ; };
    constexpr bool TILE_BULK = (CELLS * sizeof(T)) % 16 == 0 && CELLS % 16 == 0;
    const bool bulk_mode = aligned && TILE_BULK;
    auto bulk_ok = [&](long long t) { return bulk_mode && ncell_of(t) == CELLS; };
    T* const sin_ = reinterpret_cast<T*>(inb);
    T* const swt = sin_ + 6 * CELLS;
    signed char* const sph = reinterpret_cast<signed char*>(swt + CELLS);
    auto issue = [&](long long t) {
        const long long g0 = t * M * NZ;
        const uint32_t pb = CELLS * sizeof(T);
        mbar_expect_tx(&bar, 6 * pb + CELLS + (a.in.weight ? pb : 0));
        for (int k = 0; k < 3; k++) {
            bulk_load(sin_ + k * CELLS, a.in.P + k * a.in.n + g0, pb, &bar);
            bulk_load(sin_ + (3 + k) * CELLS, a.in.U + k * a.in.n + g0, pb, &bar);
        }
        bulk_load(sph, a.in.phase + g0, CELLS, &bar);
        if (a.in.weight) bulk_load(swt, a.in.weight + g0, pb, &bar);
    };
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0 && (long long)blockIdx.x < ntiles && bulk_ok(blockIdx.x)) issue(blockIdx.x);

    // this thread's items
    int am, ab, ah;
    TR::itemA(tid, am, ab, ah);
    const bool actA = tid < IA;
    const bool warpA = (tid & ~31) < IA;  // some lane of this warp has a phase-A item
    int bc, bm, ba;
    TR::itemB(tid, bc, bm, ba);
    const bool actB = tid < IB;
    int zc[CPA];  // z of each phase-A cell
#pragma unroll
    for (int j = 0; j < CPA; j++) {
        const int r = SPLIT == 2 ? 2 * j + ah : j;
        const int v = N2 * r + N1 * ab;
        zc[j] = v >= NZ ? v - NZ : v;
    }

    // phase A of atom at: sources of this thread's cells, stage-1 DFT, one store per value into dst
    auto phase_a = [&](int at, C* dst, const CellIn<T> (&cl)[CPA], const int (&cph)[CPA], const T (&cwt)[CPA]) {
        if (!warpA) return;
        C src[4][CPA];
#pragma unroll
        for (int j = 0; j < CPA; j++) {
            C E = cmake<C>(0, 0), X = E, Y = E, Z = E;
            if (cph[j] >= 0 && cph[j] < a.in.nPhase) add_source<T>(cl[j], apc[cph[j] * a.nAtom + at], cwt[j], E, X, Y, Z);
            src[0][j] = E;
            src[1][j] = X;
            src[2][j] = Y;
            src[3][j] = Z;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            C* plane = dst + q * PLANE + am * PS;
            if constexpr (SPLIT == 2) {
                C v[4] = {src[q][0], src[q][1], src[q][2], src[q][3]};
                dft4(v[0], v[1], v[2], v[3]);
                if (ah) {  // odd half: exp(-2 pi i k / 8) O_k
                    using R_t = decltype(C::x);
                    const R_t r2 = R_t(0.70710678118654752440);
                    const C o1 = v[1], o3 = v[3];
                    v[1] = cmake<C>((o1.x + o1.y) * r2, (o1.y - o1.x) * r2);
                    v[2] = cmul_mi(v[2]);
                    v[3] = cmake<C>((o3.y - o3.x) * r2, -(o3.x + o3.y) * r2);
                }
                C* row = plane + 4 * N2 * ah + ab;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    C p;
                    p.x = __shfl_xor_sync(0xffffffffu, v[k].x, 1);
                    p.y = __shfl_xor_sync(0xffffffffu, v[k].y, 1);
                    // even lane: X_k = E_k + O'_k; odd lane: X_{k+4} = E_k - O'_k
                    const C x = ah ? csub(p, v[k]) : cadd(v[k], p);
                    if (actA) row[k * N2] = x;
                }
            } else {
                C v[N1];
#pragma unroll
                for (int j = 0; j < N1; j++) v[j] = src[q][j];
                Dft<N1, C>::run(v);
#pragma unroll
                for (int k = 0; k < N1; k++)
                    if (actA) plane[k * N2 + ab] = v[k];
            }
        }
    };

    for (int it = 0;; it++) {
        const long long t = blockIdx.x + (long long)it * gridDim.x;
        if (t >= ntiles) break;
        const int ncell = ncell_of(t);
        const long long g0 = t * M * NZ;
        if (bulk_ok(t)) {
            // every tile but a partial last one is bulk-loaded, so this is the CTA's it-th use of bar
            const bool ok = mbar_wait(&bar, it & 1, a.status);
            if (!__syncthreads_and(ok)) return;  // the copy never landed (nothing else is in flight)
        } else {
            for (int e = tid; e < ncell; e += NT) {
                for (int k = 0; k < 3; k++) {
                    sin_[k * CELLS + e] = k < a.in.nStruc ? a.in.P[k * a.in.n + g0 + e] : T(0);
                    sin_[(3 + k) * CELLS + e] = a.in.U[k * a.in.n + g0 + e];
                }
                sph[e] = a.in.phase[g0 + e];
                if (a.in.weight) swt[e] = a.in.weight[g0 + e];
            }
            __syncthreads();
        }
        // phase-A cells' inputs into registers for every atom of the tile
        CellIn<T> cl[CPA];
        int cph[CPA];
        T cwt[CPA];
#pragma unroll
        for (int j = 0; j < CPA; j++) {
            const int e = am * NZ + zc[j];
            cph[j] = -1;
            cwt[j] = T(0);
            if (actA && e < ncell) {
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    cl[j].p[k] = sin_[k * CELLS + e];
                    cl[j].u[k] = sin_[(3 + k) * CELLS + e];
                }
                cph[j] = sph[e];
                cwt[j] = a.in.weight ? swt[e] : T(1);
            } else {
#pragma unroll
                for (int k = 0; k < 3; k++) cl[j].p[k] = cl[j].u[k] = T(0);
            }
            cl[j].tu = a.tq[0] * (double)cl[j].u[0] + a.tq[1] * (double)cl[j].u[1] + a.tq[2] * (double)cl[j].u[2];
        }
        phase_a(0, xb0, cl, cph, cwt);
        __syncthreads();
        // the input buffer is free: fetch the next tile into it while this one's atoms run
        if (tid == 0) {
            const long long t2 = t + gridDim.x;
            if (t2 < ntiles && bulk_ok(t2)) {
                fence_proxy_async();
                issue(t2);
            }
        }

        C acc[N2];
#pragma unroll
        for (int r = 0; r < N2; r++) acc[r] = cmake<C>(0, 0);

        for (int at = 0; at < a.nAtom; at++) {
            C* const cur = (at & 1) ? xb1 : xb0;
            // phase A of the next atom into the other buffer, then phase B of this one: one barrier per atom
            if (at + 1 < a.nAtom) phase_a(at + 1, (at & 1) ? xb0 : xb1, cl, cph, cwt);
            // ---- phase B: stage-2 DFT of one component, folded into the accumulators
            if (actB) {
                const C* row = cur + bc * PLANE + bm * PS + ba * N2;
                C v[N2];
#pragma unroll
                for (int r = 0; r < N2; r++) v[r] = row[r];
                Dft<N2, C>::run(v);
                const C* cf = (bc == 3 ? scu : sce) + at * NZ + ba * N2;
#pragma unroll
                for (int r = 0; r < N2; r++) cfma(acc[r], cf[r], v[r]);
            }
            __syncthreads();
            const int g = a.grp[at];
            if (at == a.nAtom - 1 || a.grp[at + 1] != g) {
                // the group's fields: accumulators in natural k_z order through this atom's buffer (its
                // phase-B reads are done), then coalesced rows out
                C* const ob = cur;
                if (actB) {
                    C* row = ob + bc * PLANE + bm * PS + ba * N2;
#pragma unroll
                    for (int r = 0; r < N2; r++) {
                        row[r] = acc[r];
                        acc[r] = cmake<C>(0, 0);
                    }
                }
                __syncthreads();
                if (a.yfast == 2) {
                    // (k_z, x, y) layout: column c = x ny + y of k_z sits at k_z ncols + c, and the tile's columns
                    // are t M .. t M + M - 1, so neighbouring threads write neighbouring columns of one k_z
                    C* o = a.out + 3LL * g * a.fstride + t * M;
                    const int mcols = ncell / NZ;
                    for (int e = tid; e < ncell; e += NT) {
                        const int kz = mcols == M ? e / M : e / mcols;  // full tiles divide by a constant
                        const int m = e - kz * mcols;
                        const long long d = kz * a.ncols + m;
                        const int s = m * PS + (kz % N1) * N2 + kz % N2;
                        o[d] = cadd(ob[s], ob[3 * PLANE + s]);
                        o[a.fstride + d] = ob[PLANE + s];
                        o[2 * a.fstride + d] = ob[2 * PLANE + s];
                    }
                } else if (a.yfast) {
                    // (x, k_z, y) layout: column c = x ny + y goes to (x nz + k_z) ny + y; neighbouring threads
                    // take neighbouring columns of one k_z (runs of up to M values)
                    C* o = a.out + 3LL * g * a.fstride;
                    const int mcols = ncell / NZ;
                    const long long x0 = t * M / a.ny, y0 = t * M - x0 * a.ny;  // the tile's first column
                    for (int e = tid; e < ncell; e += NT) {
                        const int kz = mcols == M ? e / M : e / mcols;  // full tiles divide by a constant
                        const int m = e - kz * mcols;
                        long long x = x0, y = y0 + m;
                        if (y >= a.ny) {  // M < ny: a tile wraps into the next x row at most once
                            y -= a.ny;
                            x += 1;
                        }
                        const long long d = (x * NZ + kz) * a.ny + y;
                        const int s = m * PS + (kz % N1) * N2 + kz % N2;
                        o[d] = cadd(ob[s], ob[3 * PLANE + s]);
                        o[a.fstride + d] = ob[PLANE + s];
                        o[2 * a.fstride + d] = ob[2 * PLANE + s];
                    }
                } else {
                    C* o = a.out + 3LL * g * a.fstride + g0;
                    for (int e = tid; e < ncell; e += NT) {
                        const int m = e / NZ;
                        const int kz = e - m * NZ;
                        const int s = m * PS + (kz % N1) * N2 + kz % N2;
                        o[e] = cadd(ob[s], ob[3 * PLANE + s]);
                        o[a.fstride + e] = ob[PLANE + s];
                        o[2 * a.fstride + e] = ob[2 * PLANE + s];
                    }
                }
                __syncthreads();  // the buffer is phase A's again two atoms on
            }
        }
    }
}

}  // namespace qpd
