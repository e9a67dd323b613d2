// Kernels of the diffraction hot path.
//
// Grid layout in HBM: every field is (nx, ny, nz) in C order, z fastest, the layout the
// reference's standard build hands over (src/python/io_utils.py:40) and the FFT order of
// its numpy.fft.fftn.  A "column" is one (x, y) pencil of nz contiguous cells.
//
// Fused schedule (three kernels per volume):
//   zstage_kernel  reads P, u and the phase weights once, evaluates the source of every atom
//                  (4 components), transforms them along z in shared memory and folds them,
//                  per group of atoms sharing (R_x, R_y), into 3 fields with the z factors
//                  exp(-i (k_z + G_z) R_z) and -i k_z applied;
//   axis_kernel    (y pass) transforms those along y and folds them, per group sharing R_x,
//                  into 2 fields with exp(-i (k_y + G_y) R_y) and -i k_y applied, in place;
//   axis_kernel    (x pass, EPI) transforms along x, forms Amp with exp(-i (k_x + G_x) R_x)
//                  and -i k_x, and writes max(|S Amp|^2, 1e-50) fftshifted as float64.
// This is exact by linearity of the FFT: the reference's factors are separable per axis
// (src/python/diffraction.py:107-109).
//
// Plain schedule (the reference's own loop, src/heffte/qpop_diffraction_mgpu.cu:169-186):
//   per atom and component: source_kernel -> fftz_kernel -> axis_kernel (y) -> axis_kernel (x)
//   -> accumulate_kernel; then intensity_kernel.
#pragma once

#include "qpd_common.cuh"
#include "qpd_fft.cuh"

namespace qpd {

constexpr int kMaxAtoms = 64;
constexpr int kMaxPhases = 8;
constexpr int kMaxSegIn = 24;
constexpr int kMaxSegs = 32;

// Per (phase, atom) constants, index p * nAtom + a (atoms in processing order); 16-byte
// aligned so a thread reads one with vector loads.
template <typename T> struct alignas(16) AtomPhase {
    double bq[3];  // sum_d qC_d su[d][k] / (2 pi): the P part of the phase, in turns
    T su[9];       // su[d * 3 + k]: shift of the atom along d per unit P_k, nm per C/m^2
    T fr, fi;      // form factor
};

// exp(-2 pi i t) for |t| <= 1/2 (already reduced in double).  float: the hardware sin / cos of an
// argument in [-pi, pi] (absolute error about 4e-7); double: sincospi.
__device__ __forceinline__ void expm2pi(double t, float* s, float* c) { __sincosf(6.283185307179586f * (float)t, s, c); }
__device__ __forceinline__ void expm2pi(double t, double* s, double* c) { sincospi(2.0 * t, s, c); }

// ---------------------------------------------------------------------------------------
// Inputs
// ---------------------------------------------------------------------------------------

// float64 reference-layout planes -> packed kernel inputs for cells [g0, g0 + cnt).
template <typename T> struct PackArgs {
    long long cnt, g0, n;
    int nStruc, nPhase;
    const double* ost[3];             // order parameter planes (nStruc of them)
    const double* uu[3];              // displacement planes, nm; null -> 0
    const double* oph[kMaxPhases];    // phase-fraction planes
    const double* region;             // scattering weight; null -> 1
    T* P;                             // 3 planes of n
    T* U;                             // 3 planes of n
    signed char* phase;               // single mode: the phase of the cell, -1 if it does not scatter
    T* weight;                        // single mode: its weight
    T* wdense;                        // dense mode: nPhase planes of n (phase fraction x region)
    unsigned int* flags;              // bit 0: a cell has >1 phases with weight; bit 1: a weight != 0, 1
};

template <typename T> __global__ void pack_kernel(PackArgs<T> a) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= a.cnt) return;
    const long long g = a.g0 + i;
    for (int k = 0; k < 3; k++) {
        a.P[k * a.n + g] = k < a.nStruc ? T(a.ost[k][i]) : T(0);
        a.U[k * a.n + g] = a.uu[k] ? T(a.uu[k][i]) : T(0);
    }
    const double r = a.region ? a.region[i] : 1.0;
    unsigned int f = 0;
    if (a.wdense) {
        for (int p = 0; p < a.nPhase; p++) a.wdense[p * a.n + g] = T(a.oph[p][i] * r);
    } else {
        int which = -1;
        double w = 0.0;
        for (int p = 0; p < a.nPhase; p++) {
            const double wp = a.oph[p][i] * r;
            if (wp != 0.0) {
                if (which >= 0) f |= 1u;
                else {
                    which = p;
                    w = wp;
                }
            }
        }
        if (which >= 0 && w != 1.0) f |= 2u;
        a.phase[g] = (signed char)which;
        a.weight[g] = T(w);
    }
    if (f) atomicOr(a.flags, f);
}

// Source of atom `at` at one cell: E = sum_p w_p f_pa exp(-2 pi i t_p), U_d = E_p u_ap[d].
template <typename T> struct CellIn {
    T p[3], u[3];
    double tu;  // qC . u / (2 pi)
};

template <typename T>
__device__ __forceinline__ void add_source(const CellIn<T>& c, const AtomPhase<T>& k, T w, C_t<T>& E, C_t<T>& X,
                                           C_t<T>& Y, C_t<T>& Z) {
    double t = c.tu + k.bq[0] * (double)c.p[0] + k.bq[1] * (double)c.p[1] + k.bq[2] * (double)c.p[2];
    t -= rint(t);  // reduced in double: the phase in turns, |t| <= 1/2
    T sn, cs;
    expm2pi(t, &sn, &cs);  // exp(-i qC . u_ap) = cs - i sn
    const T er = w * (k.fr * cs + k.fi * sn);
    const T ei = w * (k.fi * cs - k.fr * sn);
    const T ua0 = c.u[0] + k.su[0] * c.p[0] + k.su[1] * c.p[1] + k.su[2] * c.p[2];
    const T ua1 = c.u[1] + k.su[3] * c.p[0] + k.su[4] * c.p[1] + k.su[5] * c.p[2];
    const T ua2 = c.u[2] + k.su[6] * c.p[0] + k.su[7] * c.p[1] + k.su[8] * c.p[2];
    E.x += er;
    E.y += ei;
    X.x += er * ua0;
    X.y += ei * ua0;
    Y.x += er * ua1;
    Y.y += ei * ua1;
    Z.x += er * ua2;
    Z.y += ei * ua2;
}

// Packed inputs as the kernels read them.
template <typename T> struct Inputs {
    const T* P;               // 3 planes of n
    const T* U;               // 3 planes of n
    const signed char* phase; // single mode (with weight, null -> 1)
    const T* weight;
    const T* wdense;          // dense mode: nPhase planes of n
    long long n;
    int nStruc, nPhase;
};

template <typename T> __device__ __forceinline__ void load_cell(const Inputs<T>& in, long long g, const double tq[3],
                                                                CellIn<T>& c) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        c.p[k] = k < in.nStruc ? in.P[k * in.n + g] : T(0);
        c.u[k] = in.U[k * in.n + g];
    }
    c.tu = tq[0] * (double)c.u[0] + tq[1] * (double)c.u[1] + tq[2] * (double)c.u[2];
}

// Source of atom `at` (processing order) at cell g; the four components.
template <typename T>
__device__ __forceinline__ void cell_source(const Inputs<T>& in, long long g, const CellIn<T>& c, int ph, T wt,
                                            const AtomPhase<T>* apc, int nAtom, int at, C_t<T>& E, C_t<T>& X,
                                            C_t<T>& Y, C_t<T>& Z) {
    using C = C_t<T>;
    E = X = Y = Z = cmake<C>(0, 0);
    if (in.wdense) {
        for (int p = 0; p < in.nPhase; p++) {
            const T w = in.wdense[p * in.n + g];
            if (w != T(0)) add_source<T>(c, apc[p * nAtom + at], w, E, X, Y, Z);
        }
    } else if (ph >= 0 && ph < in.nPhase) {  // an index outside the phases does not scatter
        add_source<T>(c, apc[ph * nAtom + at], wt, E, X, Y, Z);
    }
}

// ---------------------------------------------------------------------------------------
// Fused z stage: source + FFT along z + fold of the atoms into 3 fields per (R_x, R_y) group
// ---------------------------------------------------------------------------------------

template <typename T> struct ZArgs {
    Inputs<T> in;
    long long ncols;  // nx * ny
    int nz, M, ps;    // z extent, columns per CTA, shared-memory pencil stride (odd)
    int nAtom;
    const AtomPhase<T>* apc;      // nPhase * nAtom
    const C_t<T>* coefE;          // [at * nz + kz] = exp(-i (k_z + G_z) R_z)
    const C_t<T>* coefUz;         // [at * nz + kz] = -i k_z exp(-i (k_z + G_z) R_z)
    int grp[kMaxAtoms];           // group of each atom in processing order (non-decreasing)
    C_t<T>* out;                  // field f = 3 g + {0: E, 1: X, 2: Y} at out + f * fstride
    long long fstride;
    double tq[3];                 // qC / (2 pi)
    AxisPlan zp;
    int* status;                  // device status word: bounded waits record timeouts here
    long long ny;                 // yfast: the y extent
    int yfast;                    // fields y fastest (zstage_pfa only): 1 (x, k_z, y), 2 (k_z, x, y)
};

template <typename T, int NT, int EPT>
__global__ void __launch_bounds__(NT) zstage_kernel(ZArgs<T> a) {
    using C = C_t<T>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    const int plane = a.M * a.ps;
    AtomPhase<T>* apc = reinterpret_cast<AtomPhase<T>*>(buf + 4 * plane);
    const int tid = threadIdx.x;
    const int nap = a.in.nPhase * a.nAtom;
    for (int i = tid; i < nap; i += NT) apc[i] = a.apc[i];

    constexpr int CPT = EPT / 4;
    const long long c0 = (long long)blockIdx.x * a.M;
    const int mcols = (int)min((long long)a.M, a.ncols - c0);
    const int ncell = mcols * a.nz;
    const long long g0 = c0 * a.nz;

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
        if (e < ncell) {
            const long long g = g0 + e;
            load_cell<T>(a.in, g, a.tq, cell[q]);
            if (!a.in.wdense) {
                ph[q] = a.in.phase[g];
                wt[q] = a.in.weight ? a.in.weight[g] : T(1);
            }
        }
    }
    const Pencils pg{4 * a.M, 4 * a.M, 0, a.ps, 1};
    __syncthreads();

    for (int at = 0; at < a.nAtom; at++) {
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            const int e = tid + q * NT;
            if (e < ncell) {
                const int m = e / a.nz;
                const int s = m * a.ps + (e - m * a.nz);
                C E, X, Y, Z;
                cell_source<T>(a.in, g0 + e, cell[q], ph[q], wt[q], apc, a.nAtom, at, E, X, Y, Z);
                buf[s] = E;
                buf[plane + s] = X;
                buf[2 * plane + s] = Y;
                buf[3 * plane + s] = Z;
            }
        }
        __syncthreads();
        fft_pencils<T, EPT>(buf, pg, a.zp, tid, NT);
        const C* ce = a.coefE + (long long)at * a.nz;
        const C* cu = a.coefUz + (long long)at * a.nz;
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            const int e = tid + q * NT;
            if (e < ncell) {
                const int m = e / a.nz;
                const int kz = e - m * a.nz;
                const int s = m * a.ps + kz;
                const C e1 = ce[kz], u1 = cu[kz];
                cfma(accE[q], e1, buf[s]);
                cfma(accE[q], u1, buf[3 * plane + s]);
                cfma(accX[q], e1, buf[plane + s]);
                cfma(accY[q], e1, buf[2 * plane + s]);
            }
        }
        const int g = a.grp[at];
        if (at == a.nAtom - 1 || a.grp[at + 1] != g) {
            C* o = a.out + 3LL * g * a.fstride + g0;
#pragma unroll
            for (int q = 0; q < CPT; q++) {
                const int e = tid + q * NT;
                if (e < ncell) {
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
// Strided axis pass (y or x): FFT of input fields along the axis, linear fold into outputs
// ---------------------------------------------------------------------------------------

// out_o(k) = sum_i coef[o][i](k) FFT(in_i)(k); a null coefficient means no contribution,
// ident means out_o = FFT(in_o) with no coefficient.
template <typename T> struct Segment {
    int nin, nout, ident;
    int in[kMaxSegIn];
    int out[2];
    const C_t<T>* coef[2][kMaxSegIn];
};

template <typename T> struct AxisArgs {
    int N;              // axis length
    long long stride;   // element stride along the axis
    long long ostride;  // stride of the outer index (x for the y pass, y for the x pass)
    int nz, Cz, nzc;    // z extent, z chunk per CTA, chunks
    const C_t<T>* in;
    C_t<T>* out;        // may alias in: every CTA reads all its inputs before writing
    long long fstride;
    const Segment<T>* segs;
    int nseg;
    int accumulate;
    AxisPlan ap;
    // epilogue of the x pass
    double* I;
    const double* S[3];
    double scale2;      // (1 / (n V))^2
    long long nx, ny;
    int* status;        // device status word: bounded waits record timeouts here
    const double* gI;   // adjoint seed (EPI 2): dL/dI, fftshifted like I
    int nouter;         // y-fastest x pass: the k_z extent (CTAs take k_z fastest)
    double* Istage;     // y-fastest 4000-point x pass: intensity rows (k_z, k_y, k_x), k_x fastest, unshifted;
                        // a separate kernel moves them to I (null: the epilogue writes I directly)
};

// EPI 0: store the folded fields; 1: intensity epilogue; 2: adjoint seed, the conjugate gradient
// D(k) = dL/dI S^2 conj(Amp) / (n V) written as field seg.out[0] (zero where I is at its floor).
template <typename T, int NT, int EPT, int EPI>
__global__ void __launch_bounds__(NT) axis_kernel(AxisArgs<T> a) {
    using C = C_t<T>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    const int tid = threadIdx.x;
    const long long outer = blockIdx.x / a.nzc;
    const int z0 = (int)(blockIdx.x % a.nzc) * a.Cz;
    const int cz = min(a.Cz, a.nz - z0);
    const int ne = a.N * cz;
    const long long base = outer * a.ostride + z0;
    const Pencils pg{cz, cz, 0, 1, a.Cz};

    for (int sg = 0; sg < a.nseg; sg++) {
        const Segment<T>& seg = a.segs[sg];
        C acc[2][EPT];
#pragma unroll
        for (int q = 0; q < EPT; q++) acc[0][q] = acc[1][q] = cmake<C>(0, 0);
        for (int fi = 0; fi < seg.nin; fi++) {
            const C* src = a.in + seg.in[fi] * a.fstride + base;
#pragma unroll
            for (int q = 0; q < EPT; q++) {
                const int e = tid + q * NT;
                if (e < ne) {
                    const int i = e / cz;
                    const int c = e - i * cz;
                    buf[i * a.Cz + c] = src[i * a.stride + c];
                }
            }
            __syncthreads();
            fft_pencils<T, EPT>(buf, pg, a.ap, tid, NT);
#pragma unroll
            for (int o = 0; o < 2; o++) {
                if (o >= seg.nout) break;
                const C* cf = seg.coef[o][fi];
                const bool mine = seg.ident ? (fi == o) : (cf != nullptr);
                if (!mine) continue;
#pragma unroll
                for (int q = 0; q < EPT; q++) {
                    const int e = tid + q * NT;
                    if (e < ne) {
                        const int k = e / cz;
                        const int c = e - k * cz;
                        const C v = buf[k * a.Cz + c];
                        if (seg.ident) acc[o][q] = cadd(acc[o][q], v);
                        else cfma(acc[o][q], cf[k], v);
                    }
                }
            }
            __syncthreads();
        }
        if (EPI == 2) {
            const long long ky = outer;
            const long long sy = (ky + a.ny / 2) % a.ny;
            const double syv = a.S[1][ky];
            C* dst = a.out + seg.out[0] * a.fstride + base;
#pragma unroll
            for (int q = 0; q < EPT; q++) {
                const int e = tid + q * NT;
                if (e < ne) {
                    const int kx = e / cz;
                    const int c = e - kx * cz;
                    const int kz = z0 + c;
                    const double S = a.S[0][kx] * syv * a.S[2][kz];
                    const double re = (double)acc[0][q].x, im = (double)acc[0][q].y;
                    const double S2 = S * S * a.scale2;
                    const long long sx = (kx + a.nx / 2) % a.nx;
                    const long long sz = (kz + a.nz / 2) % a.nz;
                    double f = 0.0;
                    if (S2 * (re * re + im * im) > 1e-50) f = a.gI[(sx * a.ny + sy) * a.nz + sz] * S2;
                    dst[kx * a.stride + c] = cmake<C>(T(f * re), T(-f * im));
                }
            }
        } else if (EPI == 1) {
            const long long ky = outer;
            const long long sy = (ky + a.ny / 2) % a.ny;
            const double syv = a.S[1][ky];
#pragma unroll
            for (int q = 0; q < EPT; q++) {
                const int e = tid + q * NT;
                if (e < ne) {
                    const int kx = e / cz;
                    const int c = e - kx * cz;
                    const int kz = z0 + c;
                    const double S = a.S[0][kx] * syv * a.S[2][kz];
                    const double re = (double)acc[0][q].x, im = (double)acc[0][q].y;
                    double v = S * S * (re * re + im * im) * a.scale2;
                    v = floor_1e50(v);
                    const long long sx = (kx + a.nx / 2) % a.nx;
                    const long long sz = (kz + a.nz / 2) % a.nz;
                    a.I[(sx * a.ny + sy) * a.nz + sz] = v;
                }
            }
        } else {
#pragma unroll
            for (int o = 0; o < 2; o++) {
                if (o >= seg.nout) break;
                C* dst = a.out + seg.out[o] * a.fstride + base;
#pragma unroll
                for (int q = 0; q < EPT; q++) {
                    const int e = tid + q * NT;
                    if (e < ne) {
                        const int i = e / cz;
                        const int c = e - i * cz;
                        C v = acc[o][q];
                        if (a.accumulate) v = cadd(v, dst[i * a.stride + c]);
                        dst[i * a.stride + c] = v;
                    }
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Adjoint (fused schedule).  With B = dL/dconj(Amp) = dL/dI S^2 Amp, the gradient of the
// source fields is G = ifftn(conj(phi) B ...), phi the separable per-atom factors.  Its conjugate
// conj(G) = fftn(phi conj(B)) / n runs the forward transforms with the forward tables, in the
// reverse axis order, unfolding the groups instead of folding them:
//   seed (axis_kernel, EPI 2)  D = dL/dI S^2 conj(Amp) / (n V)     (x pass of the recomputed forward)
//   adj_axis_kernel (x)        per R_x group: ex D, -i k_x ex D     -> FFT along x
//   adj_axis_kernel (y)        per (R_x, R_y) group: ey B, -i k_y ey B, ey X -> FFT along y
//   adj_zstage_kernel          per atom: ez A, -i k_z ez A, ez X, ez Y -> FFT along z = conj(G_E),
//                              conj(G_Uz), conj(G_Ux), conj(G_Uy), then the transpose of the source:
//   h_c = 2 qC_c Im(Q) + 2 Re(e conj(G_Uc)),  Q = e (conj(G_E) + sum_d u_d conj(G_Ud)),
//   e = w f exp(-i qC . u_ap);  dL/du_c += h_c,  dL/dP_s += sum_c su[c][s] h_c.
// ---------------------------------------------------------------------------------------

// out_o = FFT(sum_i coef[o][i](k) in_i(k)) along the axis: multiply first, then transform.
template <typename T, int NT, int EPT>
__global__ void __launch_bounds__(NT) adj_axis_kernel(AxisArgs<T> a) {
    using C = C_t<T>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    const int tid = threadIdx.x;
    const long long outer = blockIdx.x / a.nzc;
    const int z0 = (int)(blockIdx.x % a.nzc) * a.Cz;
    const int cz = min(a.Cz, a.nz - z0);
    const int ne = a.N * cz;
    const long long base = outer * a.ostride + z0;
    const Pencils pg{cz, cz, 0, 1, a.Cz};
    for (int sg = 0; sg < a.nseg; sg++) {
        const Segment<T>& seg = a.segs[sg];
        C acc[EPT];
#pragma unroll
        for (int q = 0; q < EPT; q++) acc[q] = cmake<C>(0, 0);
        for (int fi = 0; fi < seg.nin; fi++) {
            const C* src = a.in + seg.in[fi] * a.fstride + base;
            const C* cf = seg.coef[0][fi];
#pragma unroll
            for (int q = 0; q < EPT; q++) {
                const int e = tid + q * NT;
                if (e < ne) {
                    const int k = e / cz;
                    const int c = e - k * cz;
                    cfma(acc[q], cf[k], src[k * a.stride + c]);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < EPT; q++) {
            const int e = tid + q * NT;
            if (e < ne) {
                const int k = e / cz;
                buf[k * a.Cz + (e - k * cz)] = acc[q];
            }
        }
        __syncthreads();
        fft_pencils<T, EPT>(buf, pg, a.ap, tid, NT);
        C* dst = a.out + seg.out[0] * a.fstride + base;
#pragma unroll
        for (int q = 0; q < EPT; q++) {
            const int e = tid + q * NT;
            if (e < ne) {
                const int i = e / cz;
                const int c = e - i * cz;
                dst[i * a.stride + c] = buf[i * a.Cz + c];
            }
        }
        __syncthreads();
    }
}

// Transpose of add_source: accumulate the gradient of one (phase, atom) term at a cell.
template <typename T>
__device__ __forceinline__ void add_adjoint(const CellIn<T>& c, const AtomPhase<T>& k, T w, const double qc[3],
                                            C_t<T> gE, C_t<T> gX, C_t<T> gY, C_t<T> gZ, T dU[3], T dP[3]) {
    double t = c.tu + k.bq[0] * (double)c.p[0] + k.bq[1] * (double)c.p[1] + k.bq[2] * (double)c.p[2];
    t -= rint(t);
    T sn, cs;
    expm2pi(t, &sn, &cs);
    const T er = w * (k.fr * cs + k.fi * sn);
    const T ei = w * (k.fi * cs - k.fr * sn);
    const T ua0 = c.u[0] + k.su[0] * c.p[0] + k.su[1] * c.p[1] + k.su[2] * c.p[2];
    const T ua1 = c.u[1] + k.su[3] * c.p[0] + k.su[4] * c.p[1] + k.su[5] * c.p[2];
    const T ua2 = c.u[2] + k.su[6] * c.p[0] + k.su[7] * c.p[1] + k.su[8] * c.p[2];
    // s = conj(G_E) + sum_d u_d conj(G_Ud);  Im(Q) = Im(e s)
    const T sr = gE.x + ua0 * gX.x + ua1 * gY.x + ua2 * gZ.x;
    const T si = gE.y + ua0 * gX.y + ua1 * gY.y + ua2 * gZ.y;
    const T imq = er * si + ei * sr;
    T h[3];
    h[0] = T(2) * (T(qc[0]) * imq + er * gX.x - ei * gX.y);
    h[1] = T(2) * (T(qc[1]) * imq + er * gY.x - ei * gY.y);
    h[2] = T(2) * (T(qc[2]) * imq + er * gZ.x - ei * gZ.y);
#pragma unroll
    for (int d = 0; d < 3; d++) dU[d] += h[d];
#pragma unroll
    for (int s = 0; s < 3; s++) dP[s] += k.su[s] * h[0] + k.su[3 + s] * h[1] + k.su[6 + s] * h[2];
}

template <typename T> struct AdjZArgs {
    ZArgs<T> z;             // inputs, tables, groups; z.out unused
    const C_t<T>* fin;      // conjugate adjoint fields after the y pass: 3 g + {0: A, 1: X, 2: Y}
    T* dU;                  // 3 planes of n
    T* dP;                  // 3 planes of n
    double qc[3];           // qC
};

template <typename T, int NT, int EPT>
__global__ void __launch_bounds__(NT) adj_zstage_kernel(AdjZArgs<T> a) {
    using C = C_t<T>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    const ZArgs<T>& z = a.z;
    const int plane = z.M * z.ps;
    AtomPhase<T>* apc = reinterpret_cast<AtomPhase<T>*>(buf + 4 * plane);
    const int tid = threadIdx.x;
    const int nap = z.in.nPhase * z.nAtom;
    for (int i = tid; i < nap; i += NT) apc[i] = z.apc[i];

    constexpr int CPT = EPT / 4;
    const long long c0 = (long long)blockIdx.x * z.M;
    const int mcols = (int)min((long long)z.M, z.ncols - c0);
    const int ncell = mcols * z.nz;
    const long long g0 = c0 * z.nz;
    const long long n = z.in.n;

    CellIn<T> cell[CPT];
    int ph[CPT];
    T wt[CPT], dU[CPT][3], dP[CPT][3];
#pragma unroll
    for (int q = 0; q < CPT; q++) {
        const int e = tid + q * NT;
        ph[q] = -1;
        wt[q] = T(0);
        for (int d = 0; d < 3; d++) dU[q][d] = dP[q][d] = T(0);
        if (e < ncell) {
            const long long g = g0 + e;
            load_cell<T>(z.in, g, z.tq, cell[q]);
            if (!z.in.wdense) {
                ph[q] = z.in.phase[g];
                wt[q] = z.in.weight ? z.in.weight[g] : T(1);
            }
        }
    }
    const Pencils pg{4 * z.M, 4 * z.M, 0, z.ps, 1};
    __syncthreads();
    for (int at = 0; at < z.nAtom; at++) {
        const int g = z.grp[at];
        const C* fa = a.fin + 3LL * g * z.fstride + g0;
        const C* ce = z.coefE + (long long)at * z.nz;
        const C* cu = z.coefUz + (long long)at * z.nz;
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            const int e = tid + q * NT;
            if (e < ncell) {
                const int m = e / z.nz;
                const int kz = e - m * z.nz;
                const int s = m * z.ps + kz;
                const C A = fa[e], X = fa[z.fstride + e], Y = fa[2 * z.fstride + e];
                const C e1 = ce[kz], u1 = cu[kz];
                buf[s] = cmul(e1, A);
                buf[plane + s] = cmul(e1, X);
                buf[2 * plane + s] = cmul(e1, Y);
                buf[3 * plane + s] = cmul(u1, A);
            }
        }
        __syncthreads();
        fft_pencils<T, EPT>(buf, pg, z.zp, tid, NT);
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            const int e = tid + q * NT;
            if (e < ncell) {
                const int m = e / z.nz;
                const int s = m * z.ps + (e - m * z.nz);
                const C gE = buf[s], gX = buf[plane + s], gY = buf[2 * plane + s], gZ = buf[3 * plane + s];
                if (z.in.wdense) {
                    for (int p = 0; p < z.in.nPhase; p++) {
                        const T w = z.in.wdense[p * n + g0 + e];
                        if (w != T(0)) add_adjoint<T>(cell[q], apc[p * z.nAtom + at], w, a.qc, gE, gX, gY, gZ, dU[q], dP[q]);
                    }
                } else if (ph[q] >= 0 && ph[q] < z.in.nPhase) {
                    add_adjoint<T>(cell[q], apc[ph[q] * z.nAtom + at], wt[q], a.qc, gE, gX, gY, gZ, dU[q], dP[q]);
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < CPT; q++) {
        const int e = tid + q * NT;
        if (e < ncell) {
            const long long g = g0 + e;
            for (int d = 0; d < 3; d++) {
                a.dU[d * n + g] = dU[q][d];
                a.dP[d * n + g] = d < z.in.nStruc ? dP[q][d] : T(0);
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// Plain schedule
// ---------------------------------------------------------------------------------------

template <typename T> struct SourceArgs {
    Inputs<T> in;
    const AtomPhase<T>* apc;
    int nAtom, at, comp;  // comp 0: fE, 1..3: fE u_a[comp - 1]
    double tq[3];
    C_t<T>* buf;
};

template <typename T> __global__ void source_kernel(SourceArgs<T> a) {
    using C = C_t<T>;
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= a.in.n) return;
    CellIn<T> c;
    load_cell<T>(a.in, g, a.tq, c);
    int ph = -1;
    T wt = T(0);
    if (!a.in.wdense) {
        ph = a.in.phase[g];
        wt = a.in.weight ? a.in.weight[g] : T(1);
    }
    C v[4];
    cell_source<T>(a.in, g, c, ph, wt, a.apc, a.nAtom, a.at, v[0], v[1], v[2], v[3]);
    a.buf[g] = v[a.comp];
}

// FFT along z of one field, in place, M columns per CTA.
template <typename T> struct FftzArgs {
    C_t<T>* buf;
    long long ncols;
    int nz, M, ps;
    AxisPlan zp;
};

template <typename T, int NT, int EPT>
__global__ void __launch_bounds__(NT) fftz_kernel(FftzArgs<T> a) {
    using C = C_t<T>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    C* sb = reinterpret_cast<C*>(smem_raw);
    const int tid = threadIdx.x;
    const long long c0 = (long long)blockIdx.x * a.M;
    const int mcols = (int)min((long long)a.M, a.ncols - c0);
    const int ncell = mcols * a.nz;
    C* g = a.buf + c0 * a.nz;
#pragma unroll
    for (int q = 0; q < EPT; q++) {
        const int e = tid + q * NT;
        if (e < ncell) {
            const int m = e / a.nz;
            sb[m * a.ps + (e - m * a.nz)] = g[e];
        }
    }
    __syncthreads();
    const Pencils pg{a.M, a.M, 0, a.ps, 1};
    fft_pencils<T, EPT>(sb, pg, a.zp, tid, NT);
#pragma unroll
    for (int q = 0; q < EPT; q++) {
        const int e = tid + q * NT;
        if (e < ncell) {
            const int m = e / a.nz;
            g[e] = sb[m * a.ps + (e - m * a.nz)];
        }
    }
}

// amp += exp(-i (k + G) . R_a) (1, or -i k_d for component d) buf; per-axis factors in double.
template <typename T> struct AccArgs {
    C_t<T>* amp;
    const C_t<T>* buf;
    const double2* ex;   // [nx] exp(-i (k_x + G_x) R_x) of this atom
    const double2* ey;
    const double2* ez;
    const double* kd;    // wavenumbers of the component's axis (null for comp 0)
    int comp;
    long long nx, ny, nz;
};

template <typename T> __global__ void accumulate_kernel(AccArgs<T> a) {
    using C = C_t<T>;
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= a.nx * a.ny * a.nz) return;
    const long long z = g % a.nz;
    const long long y = (g / a.nz) % a.ny;
    const long long x = g / (a.nz * a.ny);
    double2 ph = a.ex[x];
    const double2 py = a.ey[y], pz = a.ez[z];
    ph = cmul(ph, py);
    ph = cmul(ph, pz);
    if (a.comp > 0) {
        const long long idx = a.comp == 1 ? x : (a.comp == 2 ? y : z);
        const double k = a.kd[idx];
        ph = cmake<double2>(k * ph.y, -k * ph.x);  // -i k ph
    }
    const C b = a.buf[g];
    C v = a.amp[g];
    v.x += T(ph.x * (double)b.x - ph.y * (double)b.y);
    v.y += T(ph.x * (double)b.y + ph.y * (double)b.x);
    a.amp[g] = v;
}

template <typename T> struct IntensityArgs {
    double* I;
    const C_t<T>* amp;
    const double* S[3];
    double scale2;
    long long nx, ny, nz;
};

template <typename T> __global__ void intensity_kernel(IntensityArgs<T> a) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= a.nx * a.ny * a.nz) return;
    const long long z = g % a.nz;
    const long long y = (g / a.nz) % a.ny;
    const long long x = g / (a.nz * a.ny);
    const double S = a.S[0][x] * a.S[1][y] * a.S[2][z];
    const double re = (double)a.amp[g].x, im = (double)a.amp[g].y;
    const double v = floor_1e50(S * S * (re * re + im * im) * a.scale2);
    const long long sx = (x + a.nx / 2) % a.nx, sy = (y + a.ny / 2) % a.ny, sz = (z + a.nz / 2) % a.nz;
    a.I[(sx * a.ny + sy) * a.nz + sz] = v;
}

}  // namespace qpd
