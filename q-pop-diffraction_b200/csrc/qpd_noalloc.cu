// qpd_run_device_noalloc: the fused float32 diffraction volume without any device allocation.
//
// Some callers cannot let a library call cudaMalloc: a framework whose caching allocator already
// owns the GPU's memory and hands out buffers itself, or a real-time loop that reserves all of its
// memory at start-up because an allocation can block the host and fail mid-run.  For them this
// entry point keeps every intermediate (the folded z-stage fields, twiddles, phase tables and
// segment descriptors) in one file-scope device array, g_noalloc_scratch, of
// QPD_NOALLOC_SCRATCH_BYTES.  The caller supplies the packed inputs and the output buffer, exactly
// as for qpd_run_device.
//
// Costs and limits: every GPU that loads the library holds the array until the process exits;
// grids whose fields and tables do not fit are refused with QPD_ERR_NOMEM, and crystals with more
// atom groups than the fused passes' segments hold with QPD_ERR_UNSUPPORTED, before any launch.
// All calls share the one array and each call overwrites it: calls that may overlap on the GPU
// (other streams, other host threads) race and must be serialised by the caller.  The first call
// on a device looks up the array's device address (cudaGetSymbolAddress) and uploads the
// butterflies' unit roots to constant memory, with that device current; make that first call
// before any stream capture.  Both are cached per device ordinal for the life of the process, so a
// device reset (cudaDeviceReset) after the first call is not supported.  The per-call constants
// and segment descriptors travel as a kernel argument, so no host memory is read after the call
// returns.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "qpopdiff.h"
#include "qpd_kernels.cuh"

using namespace qpd;

// The scratch of every call on this device (see the file comment).
static __device__ __align__(256) unsigned char g_noalloc_scratch[QPD_NOALLOC_SCRATCH_BYTES];

// qpd_api.cu: records the message qpd_last_error(NULL) returns
void qpd_internal_set_error(const char* msg);

namespace {

constexpr size_t kNoAllocBytes = (size_t)QPD_NOALLOC_SCRATCH_BYTES;
constexpr int kNoAllocAtoms = 16;
constexpr int kNoAllocGroups = kNoAllocAtoms;
constexpr int kNoAllocApc = 64;                // nAtom * nPhase
constexpr int kNoAllocSegs = kMaxSegIn + 1;    // 2 G2 y-pass segments (2 G2 <= kMaxSegIn) + the x pass
constexpr int kMaxDevices = 64;

int nfail(int code, const char* msg) {
    qpd_internal_set_error(msg);
    return code;
}

#define NA_CU(call)                                                                          \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            char m_[512];                                                                    \
            std::snprintf(m_, sizeof m_, "%s: %s", #call, cudaGetErrorString(e_));           \
            return nfail(QPD_ERR_CUDA, m_);                                                  \
        }                                                                                    \
    } while (0)

// Device address of the scratch array, looked up once per device with that device current.
int scratch_address(int device, unsigned char** out) {
    static std::mutex mu;
    static unsigned char* addr[kMaxDevices] = {};
    static bool roots[kMaxDevices] = {};
    if (device < 0 || device >= kMaxDevices) return nfail(QPD_ERR_ARG, "device index outside the supported range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        void* p = nullptr;
        NA_CU(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        addr[device] = static_cast<unsigned char*>(p);
    }
    if (!roots[device]) {
        // this translation unit's copy of the butterflies' unit roots
        double2 rd[kRootsTotal];
        float2 rf[kRootsTotal];
        for (int R : kOddRadices) {
            const int off = root_offset(R);
            for (int m = 0; m < R; m++) {
                const double a = 2.0 * M_PI * (double)m / (double)R;
                rd[off + m] = make_double2(std::cos(a), -std::sin(a));
                rf[off + m] = make_float2((float)rd[off + m].x, (float)rd[off + m].y);
            }
        }
        NA_CU(cudaMemcpyToSymbol(c_roots_d, rd, sizeof rd));
        NA_CU(cudaMemcpyToSymbol(c_roots_f, rf, sizeof rf));
        roots[device] = true;
    }
    *out = addr[device];
    return QPD_OK;
}

// Radix stages into a fixed array (the same factorisation qpd_plan uses).
int radices(int64_t N, int* r) {
    int k = 0;
    int64_t m = N;
    int e2 = 0;
    while (m % 2 == 0) {
        m /= 2;
        e2++;
    }
    int n8 = e2 / 3, rem = e2 % 3;
    for (int i = 0; i < n8; i++) r[k++] = 8;
    if (rem == 2) r[k++] = 4;
    if (rem == 1) {
        if (n8 > 0) {
            r[k - 1] = 4;
            r[k++] = 4;
        } else {
            r[k++] = 2;
        }
    }
    for (int64_t p = 3; p * p <= m; p += 2)
        while (m % p == 0) {
            r[k++] = (int)p;
            m /= p;
        }
    if (m > 1) r[k++] = (int)m;
    return k;
}

// Everything the table kernel computes, with device addresses inside the scratch array.
struct TableJob {
    int64_t N[3];
    double h[3], G[3];
    int nAtom, G1, G2;
    double rz[kNoAllocAtoms];   // R_z of each atom, processing order
    double ry[kNoAllocGroups];  // R_y of each (R_x, R_y) group
    double rx[kNoAllocGroups];  // R_x of each R_x group
    float2* tw[3];              // exp(-2 pi i m / N)
    double* S[3];               // voxel shape factor per axis
    float2* coefE;              // [at][kz]
    float2* coefUz;
    float2* ytab;               // [g1][2][ny]: exp(-i (k_y + G_y) R_y), -i k_y times that
    float2* xtab;               // [g2][2][nx]
};

__device__ double wavenumber_d(int64_t i, int64_t N, double h) {
    const double val = 1.0 / ((double)N * h);
    const int64_t m = i <= (N - 1) / 2 ? i : i - N;
    return 2.0 * M_PI * ((double)m * val);
}

__global__ void noalloc_tables(TableJob j) {
    const int64_t nt = j.N[0] + j.N[1] + j.N[2];
    const int64_t nc = (int64_t)j.nAtom * j.N[2];
    const int64_t ny2 = (int64_t)j.G1 * j.N[1];
    const int64_t nx2 = (int64_t)j.G2 * j.N[0];
    const int64_t total = nt + nc + ny2 + nx2;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = i;
        if (r < nt) {
            int d = 0;
            while (r >= j.N[d]) r -= j.N[d++];
            double s, c;
            sincospi(2.0 * (double)r / (double)j.N[d], &s, &c);
            j.tw[d][r] = make_float2((float)c, (float)-s);
            const double x = wavenumber_d(r, j.N[d], j.h[d]) * j.h[d] / (2.0 * M_PI);
            const double y = M_PI * (x == 0.0 ? 1.0e-20 : x);
            j.S[d][r] = sin(y) / y;
            continue;
        }
        r -= nt;
        if (r < nc) {
            const int at = (int)(r / j.N[2]);
            const int64_t z = r % j.N[2];
            const double k = wavenumber_d(z, j.N[2], j.h[2]);
            double s, c;
            sincos((k + j.G[2]) * j.rz[at], &s, &c);
            j.coefE[r] = make_float2((float)c, (float)-s);
            j.coefUz[r] = make_float2((float)(k * -s), (float)(-k * c));
            continue;
        }
        r -= nc;
        if (r < ny2) {
            const int g = (int)(r / j.N[1]);
            const int64_t y = r % j.N[1];
            const double k = wavenumber_d(y, j.N[1], j.h[1]);
            double s, c;
            sincos((k + j.G[1]) * j.ry[g], &s, &c);
            j.ytab[(2 * g) * j.N[1] + y] = make_float2((float)c, (float)-s);
            j.ytab[(2 * g + 1) * j.N[1] + y] = make_float2((float)(k * -s), (float)(-k * c));
            continue;
        }
        r -= ny2;
        {
            const int g = (int)(r / j.N[0]);
            const int64_t x = r % j.N[0];
            const double k = wavenumber_d(x, j.N[0], j.h[0]);
            double s, c;
            sincos((k + j.G[0]) * j.rx[g], &s, &c);
            j.xtab[(2 * g) * j.N[0] + x] = make_float2((float)c, (float)-s);
            j.xtab[(2 * g + 1) * j.N[0] + x] = make_float2((float)(k * -s), (float)(-k * c));
        }
    }
}

// Per-call constants and segment descriptors: one kernel argument (under the 32 KB parameter limit),
// copied into the scratch array by noalloc_upload.
struct Upload {
    AtomPhase<float> apc[kNoAllocApc];
    Segment<float> seg[kNoAllocSegs];
    int napc, nseg;
};
static_assert(sizeof(Upload) < 32000, "the upload must fit the kernel parameter space");

__global__ void noalloc_upload(const __grid_constant__ Upload u, AtomPhase<float>* apc, Segment<float>* seg) {
    for (int i = threadIdx.x; i < u.napc; i += blockDim.x) apc[i] = u.apc[i];
    for (int i = threadIdx.x; i < u.nseg; i += blockDim.x) seg[i] = u.seg[i];
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

extern "C" int qpd_run_device_noalloc(const qpd_grid* grid, const qpd_crystal* k, const void* P, const void* U,
                                      const int8_t* phase, const void* weight, double* I_dev, void* stream) {
    if (!grid || !k || !P || !U || !phase || !I_dev) return nfail(QPD_ERR_ARG, "qpd_run_device_noalloc: NULL argument");
    const int64_t nx = grid->nx, ny = grid->ny, nz = grid->nz;
    if (nx < 1 || ny < 1 || nz < 1) return nfail(QPD_ERR_ARG, "empty grid");
    if (!(grid->dx > 0 && grid->dy > 0 && grid->dz > 0)) return nfail(QPD_ERR_ARG, "grid spacings must be positive");
    if (k->nAtom < 1 || k->nAtom > kNoAllocAtoms) return nfail(QPD_ERR_ARG, "nAtom outside 1..16 for the allocation-free call");
    if (k->nPhase < 1 || k->nPhase > kMaxPhases || k->nStruc < 0 || k->nStruc > 3)
        return nfail(QPD_ERR_ARG, "nPhase outside 1..8 or nStruc outside 0..3");
    if (k->nAtom * k->nPhase > kNoAllocApc)
        return nfail(QPD_ERR_ARG, "nAtom * nPhase above 64 for the allocation-free call");
    if (!k->R || !k->f_re || !k->f_im || (k->nStruc > 0 && !k->su)) return nfail(QPD_ERR_ARG, "crystal arrays are NULL");
    if (nz > 1024 || nx > 4096 || ny > 4096) return nfail(QPD_ERR_UNSUPPORTED, "the allocation-free call takes nz <= 1024, nx, ny <= 4096");
    const int A = k->nAtom, NP = k->nPhase, NS = k->nStruc;
    const int64_t n = nx * ny * nz;

    // atom groups: g2 by R_x, g1 by (R_x, R_y), g1 numbered in g2 order; atoms processed by g1
    const double* R = k->R;
    double rx[kNoAllocGroups], ry[kNoAllocGroups];
    int g2a[kNoAllocAtoms], g1a[kNoAllocAtoms], g2of[kNoAllocGroups], order[kNoAllocAtoms];
    int G2 = 0, G1 = 0;
    for (int a = 0; a < A; a++) {
        int f = -1;
        for (int i = 0; i < G2; i++)
            if (rx[i] == R[3 * a]) f = i;
        if (f < 0) {
            f = G2;
            rx[G2++] = R[3 * a];
        }
        g2a[a] = f;
    }
    for (int g2 = 0; g2 < G2; g2++) {
        const int first = G1;
        for (int a = 0; a < A; a++) {
            if (g2a[a] != g2) continue;
            int f = -1;
            for (int i = first; i < G1; i++)
                if (ry[i] == R[3 * a + 1]) f = i;
            if (f < 0) {
                f = G1;
                ry[G1] = R[3 * a + 1];
                g2of[G1++] = g2;
            }
            g1a[a] = f;
        }
    }
    int no = 0;
    for (int g = 0; g < G1; g++)
        for (int a = 0; a < A; a++)
            if (g1a[a] == g) order[no++] = a;
    // segment limits of the fused passes, checked before anything is launched: the x pass reads
    // 2 fields per R_x group, a y-pass segment 2 fields per (R_x, R_y) group sharing its R_x
    if (2 * G2 > kMaxSegIn) return nfail(QPD_ERR_UNSUPPORTED, "more than 12 distinct R_x for the allocation-free call");
    for (int g2 = 0; g2 < G2; g2++) {
        int cnt = 0;
        for (int g1 = 0; g1 < G1; g1++) cnt += g2of[g1] == g2;
        if (2 * cnt > kMaxSegIn)
            return nfail(QPD_ERR_UNSUPPORTED, "more than 12 distinct R_y share one R_x for the allocation-free call");
    }

    // scratch layout
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align256(off + bytes);
        return o;
    };
    const size_t o_fields = take(sizeof(float2) * 3 * G1 * n);
    size_t o_tw[3], o_S[3];
    const int64_t N[3] = {nx, ny, nz};
    for (int d = 0; d < 3; d++) o_tw[d] = take(sizeof(float2) * N[d]);
    for (int d = 0; d < 3; d++) o_S[d] = take(sizeof(double) * N[d]);
    const size_t o_ce = take(sizeof(float2) * A * nz), o_cu = take(sizeof(float2) * A * nz);
    const size_t o_y = take(sizeof(float2) * 2 * G1 * ny), o_x = take(sizeof(float2) * 2 * G2 * nx);
    const size_t o_apc = take(sizeof(AtomPhase<float>) * NP * A);
    const int nseg = 2 * G2 + 1;
    const size_t o_seg = take(sizeof(Segment<float>) * nseg);
    if (off > kNoAllocBytes)
        return nfail(QPD_ERR_NOMEM, "grid too large for the allocation-free call: its fields and tables exceed "
                                    "QPD_NOALLOC_SCRATCH_BYTES");

    int dev = 0;
    NA_CU(cudaGetDevice(&dev));
    unsigned char* base = nullptr;
    int rc = scratch_address(dev, &base);
    if (rc != QPD_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // per-axis and per-group tables, computed on the device
    TableJob tj;
    std::memset(&tj, 0, sizeof tj);
    const double h[3] = {grid->dx, grid->dy, grid->dz};
    for (int d = 0; d < 3; d++) {
        tj.N[d] = N[d];
        tj.h[d] = h[d];
        tj.G[d] = k->G[d];
        tj.tw[d] = reinterpret_cast<float2*>(base + o_tw[d]);
        tj.S[d] = reinterpret_cast<double*>(base + o_S[d]);
    }
    tj.nAtom = A;
    tj.G1 = G1;
    tj.G2 = G2;
    for (int i = 0; i < A; i++) tj.rz[i] = R[3 * order[i] + 2];
    for (int g = 0; g < G1; g++) tj.ry[g] = ry[g];
    for (int g = 0; g < G2; g++) tj.rx[g] = rx[g];
    tj.coefE = reinterpret_cast<float2*>(base + o_ce);
    tj.coefUz = reinterpret_cast<float2*>(base + o_cu);
    tj.ytab = reinterpret_cast<float2*>(base + o_y);
    tj.xtab = reinterpret_cast<float2*>(base + o_x);
    noalloc_tables<<<148, 256, 0, st>>>(tj);
    NA_CU(cudaGetLastError());

    // per (phase, atom) constants and segment descriptors, passed to the device by value
    Upload up;
    std::memset(&up, 0, sizeof up);
    AtomPhase<float>* apc = up.apc;
    for (int p = 0; p < NP; p++)
        for (int i = 0; i < A; i++) {
            const int a = order[i];
            AtomPhase<float>& e = apc[p * A + i];
            for (int s = 0; s < 3; s++) {
                double b = 0.0;
                for (int d = 0; d < 3; d++) {
                    const double su = s < NS ? k->su[((d * NS + s) * NP + p) * A + a] : 0.0;
                    e.su[d * 3 + s] = (float)su;
                    b += k->qC[d] * su;
                }
                e.bq[s] = b / (2.0 * M_PI);
            }
            e.fr = (float)k->f_re[p * A + a];
            e.fi = (float)k->f_im[p * A + a];
        }
    Segment<float>* seg = up.seg;
    const float2* ytab = tj.ytab;
    const float2* xtab = tj.xtab;
    int s = 0;
    for (int g2 = 0; g2 < G2; g2++)
        for (int out = 0; out < 2; out++, s++) {
            seg[s].nout = 1;
            seg[s].out[0] = 2 * g2 + out;
            for (int g1 = 0; g1 < G1; g1++) {
                if (g2of[g1] != g2) continue;
                if (out == 0) {
                    seg[s].in[seg[s].nin] = 3 * g1;
                    seg[s].coef[0][seg[s].nin++] = ytab + (2 * g1) * ny;
                    seg[s].in[seg[s].nin] = 3 * g1 + 2;
                    seg[s].coef[0][seg[s].nin++] = ytab + (2 * g1 + 1) * ny;
                } else {
                    seg[s].in[seg[s].nin] = 3 * g1 + 1;
                    seg[s].coef[0][seg[s].nin++] = ytab + (2 * g1) * ny;
                }
            }
        }
    seg[s].nout = 1;
    for (int g2 = 0; g2 < G2; g2++) {
        seg[s].in[seg[s].nin] = 2 * g2;
        seg[s].coef[0][seg[s].nin++] = xtab + (2 * g2) * nx;
        seg[s].in[seg[s].nin] = 2 * g2 + 1;
        seg[s].coef[0][seg[s].nin++] = xtab + (2 * g2 + 1) * nx;
    }
    up.napc = NP * A;
    up.nseg = nseg;
    noalloc_upload<<<1, 128, 0, st>>>(up, reinterpret_cast<AtomPhase<float>*>(base + o_apc),
                                      reinterpret_cast<Segment<float>*>(base + o_seg));
    NA_CU(cudaGetLastError());

    Inputs<float> in;
    in.P = static_cast<const float*>(P);
    in.U = static_cast<const float*>(U);
    in.phase = reinterpret_cast<const signed char*>(phase);
    in.weight = static_cast<const float*>(weight);
    in.wdense = nullptr;
    in.n = n;
    in.nStruc = NS;
    in.nPhase = NP;
    float2* F = reinterpret_cast<float2*>(base + o_fields);
    auto plan_of = [&](int d) {
        AxisPlan ap;
        std::memset(&ap, 0, sizeof ap);
        ap.N = (int)N[d];
        ap.nstages = N[d] > 1 ? radices(N[d], ap.radix) : 0;
        ap.tw = base + o_tw[d];
        return ap;
    };

    // z stage (generic kernel: 256 threads, tiles of up to 1024 cells, under 48 KB of shared memory)
    ZArgs<float> z;
    std::memset(&z, 0, sizeof z);
    z.in = in;
    z.ncols = nx * ny;
    z.nz = (int)nz;
    z.M = (int)std::max<int64_t>(1, std::min<int64_t>(256 * 16 / 4 / nz, z.ncols));
    z.ps = nz % 2 ? (int)nz : (int)nz + 1;
    z.nAtom = A;
    z.apc = reinterpret_cast<const AtomPhase<float>*>(base + o_apc);
    z.coefE = reinterpret_cast<const float2*>(base + o_ce);
    z.coefUz = reinterpret_cast<const float2*>(base + o_cu);
    for (int i = 0; i < A; i++) z.grp[i] = g1a[order[i]];
    z.out = F;
    z.fstride = n;
    for (int d = 0; d < 3; d++) z.tq[d] = k->qC[d] / (2.0 * M_PI);
    z.zp = plan_of(2);
    const size_t zsmem = sizeof(float2) * 4 * z.M * z.ps + sizeof(AtomPhase<float>) * NP * A + 16;
    if (zsmem > 48 * 1024) return nfail(QPD_ERR_UNSUPPORTED, "z tile too large for the allocation-free call");
    zstage_kernel<float, 256, 16><<<(unsigned)((z.ncols + z.M - 1) / z.M), 256, zsmem, st>>>(z);
    NA_CU(cudaGetLastError());

    // y pass in place, then x pass with the |S Amp|^2 + fftshift epilogue
    for (int d = 1; d >= 0; d--) {
        AxisArgs<float> ax;
        std::memset(&ax, 0, sizeof ax);
        ax.N = (int)N[d];
        ax.stride = d == 1 ? nz : ny * nz;
        ax.ostride = d == 1 ? ny * nz : nz;
        ax.nz = (int)nz;
        ax.Cz = (int)std::max<int64_t>(1, std::min<int64_t>(nz, 256 * 16 / N[d]));
        ax.nzc = (int)((nz + ax.Cz - 1) / ax.Cz);
        ax.in = F;
        ax.out = F;
        ax.fstride = n;
        ax.ap = plan_of(d);
        ax.nx = nx;
        ax.ny = ny;
        const unsigned blocks = (unsigned)((d == 1 ? nx : ny) * ax.nzc);
        const size_t smem = sizeof(float2) * ax.N * ax.Cz + 16;
        if (d == 1) {
            ax.segs = reinterpret_cast<const Segment<float>*>(base + o_seg);
            ax.nseg = 2 * G2;
            axis_kernel<float, 256, 16, false><<<blocks, 256, smem, st>>>(ax);
        } else {
            ax.segs = reinterpret_cast<const Segment<float>*>(base + o_seg) + 2 * G2;
            ax.nseg = 1;
            ax.I = I_dev;
            for (int e = 0; e < 3; e++) ax.S[e] = reinterpret_cast<const double*>(base + o_S[e]);
            const double nV = (double)n * k->V;
            ax.scale2 = 1.0 / (nV * nV);
            axis_kernel<float, 256, 16, true><<<blocks, 256, smem, st>>>(ax);
        }
        NA_CU(cudaGetLastError());
    }
    return QPD_OK;
}
