// libqpopdiff.so: the C ABI declared in include/qpopdiff.h.
//
// Host side of the B200 diffraction path: axis planning (radix factorisation, twiddle tables),
// crystal tables (atom grouping for the fused schedule, per-axis phase factors, voxel shape
// factor), workspace management under an HBM budget, and the launch sequence of both schedules.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "qpopdiff.h"
#include "qpd_fast.cuh"
#include "qpd_fields.cuh"
#include "qpd_zpfa.cuh"
#include "qpd_host.h"
#include "qpd_kernels.cuh"
#include "qpd_n4000.h"

namespace qpd {
// qpd_probe.cu: a kernel that takes the bounded-wait failure path (a barrier no copy completes)
cudaError_t launch_wait_probe(int* status, long long polls, cudaStream_t st);
}  // namespace qpd

using namespace qpd;

namespace {

thread_local std::string g_create_error;

struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct qpd_ctx {
    int device = 0;
    uint64_t budget = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    uint64_t launches = 0;
    size_t held = 0;

    // plan
    bool planned = false;
    int64_t nx = 0, ny = 0, nz = 0, n = 0;
    double h[3] = {0, 0, 0};
    int nPhase = 0, nStruc = 0, precision = QPD_FP32, schedule = QPD_SCHED_FUSED;
    std::vector<int> radix[3];
    DevMem tw[3];

    // crystal
    bool have_crystal = false;
    int nAtom = 0;
    int sched_used = QPD_SCHED_FUSED;  // fused falls back to plain when the grouping does not fit
    int ng1 = 0, ng2 = 0;
    std::vector<int> grp;              // group of each atom in processing order
    double tq[3] = {0, 0, 0};
    double scale2 = 0;
    DevMem tables;                     // complex coefficient tables, shape factors, constants, segments
    // offsets into `tables`
    size_t off_apc = 0, off_coefE = 0, off_coefUz = 0, off_S[3] = {0, 0, 0}, off_segY = 0, off_segX = 0;
    size_t off_pex = 0, off_pey = 0, off_pez = 0, off_k[3] = {0, 0, 0};
    int nsegY = 0;
    size_t off_segAX = 0, off_segAY = 0;  // adjoint passes
    int nsegAX = 0, nsegAY = 0;
    // register-resident 4000-point passes (float32 fused): their input descriptors, device addresses
    // inside `tables` (have_p4y: ny = 4000, have_p4x: nx = 4000)
    bool have_p4y = false, have_p4x = false;
    qpd::Pass4k p4y, p4x;

    // workspace
    DevMem fields;  // fused: 3 * ng1 fields; plain: buf + amp
    DevMem adjw;    // adjoint: the seed D and 2 * ng2 fields after the adjoint x pass
    DevMem packed;  // host path: P, U, phase, weight
    DevMem dense;   // host path, dense weights
    DevMem stage;   // host path, float64 staging
    DevMem Idev;    // host path, intensity
    DevMem flags;
    DevMem status;  // device status word of the bounded waits (QPD_DEVERR_*)
    // host path: packing threads and a pinned ring of chunk slots
    std::unique_ptr<qpd::Workers> workers;
    void* hring = nullptr;
    size_t hring_bytes = 0;
    cudaEvent_t ring_ev[3] = {nullptr, nullptr, nullptr};
    bool ring_busy[3] = {false, false, false};
    static constexpr int kChunkEv = 8;
    cudaEvent_t chunk_ev[kChunkEv] = {};
    bool tma = true;  // TMA-fed kernels where the layout allows (QPOP_B200_NO_TMA=1 disables)

    // compile-time specialised kernels where an instantiation covers the axis (QPOP_B200_GENERIC=1 disables)
    bool fast = true;
    // launch-shape choices among equivalent kernels: QPOP_B200_ZCFG=1 (z stage, nz = 104: 416 threads
    // reading inputs from shared memory instead of 256 holding them in registers),
    // QPOP_B200_NBUF (tile buffers of the TMA passes, 2 or 3)
    int knob_z = 0;
    int knob_nbuf = 2;
    // z stage for nz = 104 and 68: the register-fused prime-factor kernel (zstage_pfa) or the Stockham one.
    // Default (-1): fused for nz = 68 (69.8 against 89.3 ms at 4000x4000x68), Stockham for nz = 104 (1.81
    // against 1.84 ms at 512x512x104); QPOP_B200_ZPFA=0 or 1 forces one of them for both lengths.
    int knob_zpfa = -1;
    // QPOP_B200_N4000: launch shape of the 4000-point passes (0: 512 threads, out-of-place swizzled
    // stages; 1: one buffer, two CTAs per SM; 2: 1024 threads in place; 3: 512 threads in place;
    // 4: 1024 threads out of place)
    int knob_n4000 = 0;
    // QPOP_B200_YFAST=0: keep the z-fastest field layout at 4000 x 4000 x 68 (the y-fastest route writes
    // the z stage's fields with y fastest so the 4000-point y transforms read contiguous pencils)
    int knob_yfast = 1;
    int knob_bulk_nt = 256;
    // QPOP_B200_ZREGIN=0: nz = 64 and 128 z stages with 512 threads reading their inputs from shared
    // memory for every atom, instead of 256 threads holding them in registers (0.262 against 0.239 ms
    // at 256x256x64, 0.156 against 0.142 ms at 128^3)
    int knob_zregin = 1;
    // QPOP_B200_ADJ_TMA=0: the adjoint's x and y passes on the generic kernels instead of the TMA one
    int knob_adj_tma = 1;  // QPOP_B200_BULK_NT: threads of the bulk y pass (256: 72.8 ms, 512: 80.9 ms)
    // QPOP_B200_N4K=0: the 4000-point passes on the shared-memory Stockham kernels (axis_tma, axis_bulk)
    // instead of the register-resident ones of qpd_n4000.cu
    int knob_n4k = 1;
    // qpd_set_cta_tiles: at most this many tiles per CTA of the persistent z stages (0: one wave of CTAs
    // walks every tile)
    int cta_tiles = 0;
    // QPOP_B200_OOP=0: in-place stages for the 256- and 512-point TMA passes (out-of-place measured
    // 1.080 against 1.104 ms for the y pass at 512x512x104)
    int knob_oop = 1;

    // per-kernel timing
    bool timing = false;
    struct Rec {
        int kind;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
};

namespace {

int fail(qpd_ctx* c, int code, const char* fmt, ...) {
    char msg[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(msg, sizeof msg, fmt, ap);
    va_end(ap);
    if (c) c->err = msg;
    else g_create_error = msg;
    return code;
}

#define QPD_CU(ctx, call)                                                                                     \
    do {                                                                                                      \
        cudaError_t e_ = (call);                                                                              \
        if (e_ != cudaSuccess)                                                                                \
            return fail((ctx), QPD_ERR_CUDA, "%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
    } while (0)

#define QPD_TRY(expr)          \
    do {                       \
        int r_ = (expr);       \
        if (r_ != QPD_OK) return r_; \
    } while (0)

int check_status(qpd_ctx* c);
int field_map(qpd_ctx* c, CUtensorMap* m, void* base, bool fp64, int64_t nz, int64_t ny, int64_t nfx, int bz, int by,
              int bx);

int dev_free(qpd_ctx* c, DevMem& m) {
    if (m.p) {
        cudaError_t e = cudaFree(m.p);
        c->held -= m.bytes;
        m.p = nullptr;
        m.bytes = 0;
        if (e != cudaSuccess) return fail(c, QPD_ERR_CUDA, "cudaFree: %s", cudaGetErrorString(e));
    }
    return QPD_OK;
}

// Make m hold at least `bytes` (contents not kept when it grows).
int dev_reserve(qpd_ctx* c, DevMem& m, size_t bytes, const char* what) {
    if (m.p && m.bytes >= bytes) return QPD_OK;
    QPD_TRY(dev_free(c, m));
    if (bytes == 0) return QPD_OK;
    if (c->budget && c->held + bytes > c->budget)
        return fail(c, QPD_ERR_NOMEM, "%s needs %zu bytes; the context holds %zu of its %llu-byte budget", what, bytes,
                    c->held, (unsigned long long)c->budget);
    cudaError_t e = cudaMalloc(&m.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        m.p = nullptr;
        return fail(c, QPD_ERR_NOMEM, "%s: cudaMalloc of %zu bytes failed: %s", what, bytes, cudaGetErrorString(e));
    }
    m.bytes = bytes;
    c->held += bytes;
    return QPD_OK;
}

cudaEvent_t take_event(qpd_ctx* c) {
    if (!c->pool.empty()) {
        cudaEvent_t e = c->pool.back();
        c->pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

// Event before a timed launch (nullptr when timing is off).
int tstart(qpd_ctx* c, cudaStream_t st, cudaEvent_t* a) {
    *a = nullptr;
    if (!c->timing) return QPD_OK;
    *a = take_event(c);
    if (!*a) return fail(c, QPD_ERR_CUDA, "cudaEventCreate failed");
    QPD_CU(c, cudaEventRecord(*a, st));
    return QPD_OK;
}

// Event after it; the pair is kept for qpd_stage_times.
int tstop(qpd_ctx* c, int kind, cudaStream_t st, cudaEvent_t a) {
    c->launches++;
    QPD_CU(c, cudaGetLastError());
    if (!a) return QPD_OK;
    cudaEvent_t b = take_event(c);
    if (!b) return fail(c, QPD_ERR_CUDA, "cudaEventCreate failed");
    QPD_CU(c, cudaEventRecord(b, st));
    c->recs.push_back({kind, a, b});
    return QPD_OK;
}

// Radix stages of an axis: as many 8s as the power of two allows (a leftover 2 turns an 8 into
// 4 * 4), then the odd primes in increasing order.
std::vector<int> factorise(int64_t N) {
    std::vector<int> r;
    int64_t m = N;
    int e2 = 0;
    while (m % 2 == 0) {
        m /= 2;
        e2++;
    }
    int n8 = e2 / 3, rem = e2 % 3;
    for (int i = 0; i < n8; i++) r.push_back(8);
    if (rem == 2) r.push_back(4);
    if (rem == 1) {
        if (n8 > 0) {
            r.pop_back();
            r.push_back(4);
            r.push_back(4);
        } else {
            r.push_back(2);
        }
    }
    for (int64_t p = 3; p * p <= m; p += 2)
        while (m % p == 0) {
            r.push_back((int)p);
            m /= p;
        }
    if (m > 1) r.push_back((int)m);
    return r;
}

// 2 pi numpy.fft.fftfreq(N, h)[i], in numpy's operation order.
double wavenumber(int64_t i, int64_t N, double h) {
    const double val = 1.0 / ((double)N * h);
    const int64_t m = i <= (N - 1) / 2 ? i : i - N;
    return 2.0 * M_PI * ((double)m * val);
}

// numpy.sinc
double sinc_np(double x) {
    const double y = M_PI * (x == 0.0 ? 1.0e-20 : x);
    return std::sin(y) / y;
}

// exp(-i theta) as numpy evaluates exp(-1j * x * R): (cos theta, -sin theta)
double2 expmi(double theta) { return make_double2(std::cos(theta), -std::sin(theta)); }


template <typename T> C_t<T> to_c(double2 v) { return cmake<C_t<T>>((T)v.x, (T)v.y); }

AxisPlan axis_plan(const qpd_ctx* c, int d) {
    AxisPlan ap;
    std::memset(&ap, 0, sizeof ap);
    ap.N = (int)(d == 0 ? c->nx : d == 1 ? c->ny : c->nz);
    ap.nstages = (int)c->radix[d].size();
    for (int s = 0; s < ap.nstages; s++) ap.radix[s] = c->radix[d][s];
    ap.tw = c->tw[d].p;
    return ap;
}

// ------------------------------------------------------------------------------------------
// Launch configurations.  EPT * NT bounds the complex values a CTA tile holds.
// ------------------------------------------------------------------------------------------

size_t max_smem(qpd_ctx* c) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    return (size_t)v;
}

template <typename K> int set_smem(qpd_ctx* c, K kernel, size_t bytes) {
    if (bytes > 48 * 1024)
        QPD_CU(c, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return QPD_OK;
}

// weight of a chunk whose packed weights are all 0 or 1: 1 where the cell has a phase
template <typename T> __global__ void fill_weight_kernel(const int8_t* ph, T* w, long long cnt) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < cnt) w[i] = ph[i] >= 0 ? T(1) : T(0);
}

struct Cfg {
    int nt, ept;
};

// z stage / fftz: a tile of M columns (4 fields each for the z stage)
const Cfg kZCfg[] = {{256, 16}, {512, 16}, {1024, 8}, {1024, 16}};
// strided axis passes: a tile of N x Cz
const Cfg kACfg[] = {{256, 16}, {512, 16}, {1024, 8}, {1024, 16}};

int odd_stride(int nz) { return nz % 2 ? nz : nz + 1; }

template <typename T> struct Impl {
    using C = C_t<T>;

    // ---------------- tables ----------------
    static int set_crystal(qpd_ctx* c, const qpd_crystal* k) {
        const int A = k->nAtom, NP = k->nPhase, NS = k->nStruc;
        const double* R = k->R;
        // groups: g2 by R_x, g1 by (R_x, R_y), g1 numbered in g2 order
        std::vector<double> rx;
        std::vector<int> g2a(A), g1a(A);
        for (int a = 0; a < A; a++) {
            int f = -1;
            for (size_t i = 0; i < rx.size(); i++)
                if (rx[i] == R[3 * a]) f = (int)i;
            if (f < 0) {
                f = (int)rx.size();
                rx.push_back(R[3 * a]);
            }
            g2a[a] = f;
        }
        const int G2 = (int)rx.size();
        std::vector<double> ry;     // R_y of each g1
        std::vector<int> g2of;      // g2 of each g1
        for (int g2 = 0; g2 < G2; g2++) {
            const size_t first = ry.size();
            for (int a = 0; a < A; a++) {
                if (g2a[a] != g2) continue;
                int f = -1;
                for (size_t i = first; i < ry.size(); i++)
                    if (ry[i] == R[3 * a + 1]) f = (int)i;
                if (f < 0) {
                    f = (int)ry.size();
                    ry.push_back(R[3 * a + 1]);
                    g2of.push_back(g2);
                }
                g1a[a] = f;
            }
        }
        const int G1 = (int)ry.size();
        std::vector<int> order(A);
        for (int a = 0; a < A; a++) order[a] = a;
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return g1a[x] < g1a[y]; });

        int sched = c->schedule;
        if (sched == QPD_SCHED_FUSED) {
            int maxin = 0;
            for (int g2 = 0; g2 < G2; g2++) {
                int cnt = 0;
                for (int g1 = 0; g1 < G1; g1++) cnt += g2of[g1] == g2;
                maxin = std::max(maxin, 3 * cnt);
            }
            if (A > kMaxAtoms || maxin > kMaxSegIn || 2 * G2 > kMaxSegIn || 2 * G2 > kMaxSegs) sched = QPD_SCHED_PLAIN;
        }
        c->sched_used = sched;
        c->nAtom = A;
        c->ng1 = G1;
        c->ng2 = G2;
        c->grp.assign(A, 0);
        for (int i = 0; i < A; i++) c->grp[i] = g1a[order[i]];
        for (int d = 0; d < 3; d++) c->tq[d] = k->qC[d] / (2.0 * M_PI);
        const double nV = (double)c->n * k->V;
        c->scale2 = 1.0 / (nV * nV);

        const int64_t N[3] = {c->nx, c->ny, c->nz};
        std::vector<double> kd[3], S[3];
        for (int d = 0; d < 3; d++) {
            kd[d].resize(N[d]);
            S[d].resize(N[d]);
            for (int64_t i = 0; i < N[d]; i++) {
                kd[d][i] = wavenumber(i, N[d], c->h[d]);
                S[d][i] = sinc_np(kd[d][i] * c->h[d] / (2.0 * M_PI));
            }
        }

        // host images of every table, laid out in one device buffer
        std::vector<unsigned char> host;
        auto place = [&](size_t bytes) {
            size_t off = (host.size() + 255) & ~size_t(255);
            host.resize(off + bytes);
            return off;
        };
        c->off_apc = place(sizeof(AtomPhase<T>) * NP * A);
        {
            AtomPhase<T>* apc = reinterpret_cast<AtomPhase<T>*>(host.data() + c->off_apc);
            for (int p = 0; p < NP; p++)
                for (int i = 0; i < A; i++) {
                    const int a = order[i];
                    AtomPhase<T>& e = apc[p * A + i];
                    std::memset(&e, 0, sizeof e);
                    for (int s = 0; s < 3; s++) {
                        double b = 0.0;
                        for (int d = 0; d < 3; d++) {
                            const double su = s < NS ? k->su[((d * NS + s) * NP + p) * A + a] : 0.0;
                            e.su[d * 3 + s] = (T)su;
                            b += k->qC[d] * su;
                        }
                        e.bq[s] = b / (2.0 * M_PI);
                    }
                    e.fr = (T)k->f_re[p * A + a];
                    e.fi = (T)k->f_im[p * A + a];
                }
        }
        for (int d = 0; d < 3; d++) {
            c->off_S[d] = place(sizeof(double) * N[d]);
            std::memcpy(host.data() + c->off_S[d], S[d].data(), sizeof(double) * N[d]);
        }
        std::vector<Segment<T>> segY, segX, segAX, segAY;
        // inputs of the register-resident 4000-point y pass, in segment order: field, g1, -i k_y, closes a
        // segment, its output field
        size_t off4y = 0, off4x = 0;
        std::vector<int> in4y_g, in4y_ik, in4y_f, in4y_last, in4y_out;
        const bool f4y = sizeof(T) == 4 && N[1] == 4000, f4x = sizeof(T) == 4 && N[0] == 4000;
        if (sched == QPD_SCHED_FUSED) {
            c->off_coefE = place(sizeof(C) * A * N[2]);
            c->off_coefUz = place(sizeof(C) * A * N[2]);
            C* cE = reinterpret_cast<C*>(host.data() + c->off_coefE);
            C* cU = reinterpret_cast<C*>(host.data() + c->off_coefUz);
            for (int i = 0; i < A; i++) {
                const int a = order[i];
                for (int64_t z = 0; z < N[2]; z++) {
                    const double2 e = expmi((kd[2][z] + k->G[2]) * R[3 * a + 2]);
                    cE[i * N[2] + z] = to_c<T>(e);
                    cU[i * N[2] + z] = to_c<T>(make_double2(kd[2][z] * e.y, -kd[2][z] * e.x));  // -i k_z e
                }
            }
            // y tables per g1: ey, -i k_y ey; x tables per g2: ex, -i k_x ex
            std::vector<size_t> offY(G1), offX(G2);
            for (int g1 = 0; g1 < G1; g1++) {
                offY[g1] = place(sizeof(C) * 2 * N[1]);
                C* t = reinterpret_cast<C*>(host.data() + offY[g1]);
                for (int64_t y = 0; y < N[1]; y++) {
                    const double2 e = expmi((kd[1][y] + k->G[1]) * ry[g1]);
                    t[y] = to_c<T>(e);
                    t[N[1] + y] = to_c<T>(make_double2(kd[1][y] * e.y, -kd[1][y] * e.x));
                }
            }
            for (int g2 = 0; g2 < G2; g2++) {
                offX[g2] = place(sizeof(C) * 2 * N[0]);
                C* t = reinterpret_cast<C*>(host.data() + offX[g2]);
                for (int64_t x = 0; x < N[0]; x++) {
                    const double2 e = expmi((kd[0][x] + k->G[0]) * rx[g2]);
                    t[x] = to_c<T>(e);
                    t[N[0] + x] = to_c<T>(make_double2(kd[0][x] * e.y, -kd[0][x] * e.x));
                }
            }
            // fold factors of the register-resident 4000-point passes (float32): per g1 for a 4000-point y
            // axis, per g2 for a 4000-point x axis, 200 values u[t] then 20 values V[r] each (Pass4k)
            auto fold4k = [&](C* dst, int64_t Nd, double hd, double G, double Rd) {
                const double val = 1.0 / ((double)Nd * hd);
                for (int t = 0; t < 200; t++) dst[t] = to_c<T>(expmi(2.0 * M_PI * ((double)t * val) * Rd));
                for (int r = 0; r < 20; r++) {
                    const double m = 200.0 * r - (r >= 10 ? (double)Nd : 0.0);
                    dst[200 + r] = to_c<T>(expmi(2.0 * M_PI * (m * val) * Rd + G * Rd));
                }
            };
            if (f4y) {
                off4y = place(sizeof(C) * 220 * G1);
                for (int g1 = 0; g1 < G1; g1++)
                    fold4k(reinterpret_cast<C*>(host.data() + off4y) + 220 * g1, N[1], c->h[1], k->G[1], ry[g1]);
            }
            if (f4x) {
                off4x = place(sizeof(C) * 220 * G2);
                for (int g2 = 0; g2 < G2; g2++)
                    fold4k(reinterpret_cast<C*>(host.data() + off4x) + 220 * g2, N[0], c->h[0], k->G[0], rx[g2]);
            }
            // segments hold device addresses: filled in once the buffer exists
            // one output per segment: E2 <- (E1, Y1) of the g1 groups sharing R_x, then X2 <- X1.
            // Writing E2 into slot 2 g2 before X1 of the same g2 is read is safe: X1 slots are 3 g1 + 1 > 2 g2.
            for (int g2 = 0; g2 < G2; g2++) {
                for (int out = 0; out < 2; out++) {
                    Segment<T> s;
                    std::memset(&s, 0, sizeof s);
                    s.nout = 1;
                    s.out[0] = 2 * g2 + out;
                    for (int g1 = 0; g1 < G1; g1++) {
                        if (g2of[g1] != g2) continue;
                        // table offsets + 1 for now (0 = no contribution); fixed up once the buffer exists
                        const size_t e = offY[g1] + 1, mi = offY[g1] + sizeof(C) * N[1] + 1;
                        if (out == 0) {
                            s.in[s.nin] = 3 * g1 + 0;
                            s.coef[0][s.nin++] = reinterpret_cast<const C*>(e);
                            s.in[s.nin] = 3 * g1 + 2;
                            s.coef[0][s.nin++] = reinterpret_cast<const C*>(mi);
                            in4y_f.insert(in4y_f.end(), {3 * g1, 3 * g1 + 2});
                            in4y_g.insert(in4y_g.end(), {g1, g1});
                            in4y_ik.insert(in4y_ik.end(), {0, 1});
                        } else {
                            s.in[s.nin] = 3 * g1 + 1;
                            s.coef[0][s.nin++] = reinterpret_cast<const C*>(e);
                            in4y_f.push_back(3 * g1 + 1);
                            in4y_g.push_back(g1);
                            in4y_ik.push_back(0);
                        }
                    }
                    in4y_last.resize(in4y_f.size(), 0);
                    in4y_out.resize(in4y_f.size(), 0);
                    if (!in4y_f.empty()) {
                        in4y_last.back() = 1;
                        in4y_out.back() = 2 * g2 + out;
                    }
                    segY.push_back(s);
                }
            }
            Segment<T> s;
            std::memset(&s, 0, sizeof s);
            s.nout = 1;
            for (int g2 = 0; g2 < G2; g2++) {
                s.in[s.nin] = 2 * g2;
                s.coef[0][s.nin++] = reinterpret_cast<const C*>(offX[g2] + 1);
                s.in[s.nin] = 2 * g2 + 1;
                s.coef[0][s.nin++] = reinterpret_cast<const C*>(offX[g2] + sizeof(C) * N[0] + 1);
            }
            segX.push_back(s);
            c->nsegY = 2 * G2;
            c->off_segY = place(sizeof(Segment<T>) * segY.size());
            c->off_segX = place(sizeof(Segment<T>));
            // adjoint x pass: adjoint workspace slot 0 (the seed) -> slots 1 + 2 g2 (ex) and 2 + 2 g2 (-i k_x ex);
            // adjoint y pass: slot 1 + 2 g2 -> fields 3 g1 (ey) and 3 g1 + 2 (-i k_y ey), slot 2 + 2 g2 -> 3 g1 + 1 (ey)
            auto one = [](int in, size_t coef, int out) {
                Segment<T> t;
                std::memset(&t, 0, sizeof t);
                t.nin = 1;
                t.nout = 1;
                t.in[0] = in;
                t.coef[0][0] = reinterpret_cast<const C*>(coef + 1);
                t.out[0] = out;
                return t;
            };
            for (int g2 = 0; g2 < G2; g2++) {
                segAX.push_back(one(0, offX[g2], 1 + 2 * g2));
                segAX.push_back(one(0, offX[g2] + sizeof(C) * N[0], 2 + 2 * g2));
            }
            for (int g1 = 0; g1 < G1; g1++) {
                const int g2 = g2of[g1];
                segAY.push_back(one(1 + 2 * g2, offY[g1], 3 * g1));
                segAY.push_back(one(1 + 2 * g2, offY[g1] + sizeof(C) * N[1], 3 * g1 + 2));
                segAY.push_back(one(2 + 2 * g2, offY[g1], 3 * g1 + 1));
            }
            c->nsegAX = (int)segAX.size();
            c->nsegAY = (int)segAY.size();
            c->off_segAX = place(sizeof(Segment<T>) * segAX.size());
            c->off_segAY = place(sizeof(Segment<T>) * segAY.size());
        } else {
            // plain: per-atom axis factors in double and the wavenumbers
            c->off_pex = place(sizeof(double2) * A * N[0]);
            c->off_pey = place(sizeof(double2) * A * N[1]);
            c->off_pez = place(sizeof(double2) * A * N[2]);
            const size_t offs[3] = {c->off_pex, c->off_pey, c->off_pez};
            for (int d = 0; d < 3; d++) {
                double2* t = reinterpret_cast<double2*>(host.data() + offs[d]);
                for (int i = 0; i < A; i++) {
                    const int a = order[i];
                    for (int64_t m = 0; m < N[d]; m++) t[i * N[d] + m] = expmi((kd[d][m] + k->G[d]) * R[3 * a + d]);
                }
                c->off_k[d] = place(sizeof(double) * N[d]);
                std::memcpy(host.data() + c->off_k[d], kd[d].data(), sizeof(double) * N[d]);
            }
            Segment<T> s;
            std::memset(&s, 0, sizeof s);
            s.nin = 1;
            s.nout = 1;
            s.ident = 1;
            segX.push_back(s);
            c->off_segX = place(sizeof(Segment<T>));
        }
        QPD_TRY(dev_reserve(c, c->tables, host.size(), "crystal tables"));
        const uintptr_t base = reinterpret_cast<uintptr_t>(c->tables.p);
        auto fix = [&](Segment<T>& s) {
            for (int o = 0; o < 2; o++)
                for (int i = 0; i < kMaxSegIn; i++)
                    if (s.coef[o][i]) s.coef[o][i] = reinterpret_cast<const C*>(base + reinterpret_cast<uintptr_t>(s.coef[o][i]) - 1);
        };
        for (auto& s : segY) fix(s);
        c->have_p4y = c->have_p4x = false;
        if constexpr (sizeof(T) == 4) {
            if (sched == QPD_SCHED_FUSED && f4y && (int)in4y_f.size() <= kPass4kMax) {
                Pass4k& P = c->p4y;
                std::memset(&P, 0, sizeof P);
                for (size_t i = 0; i < in4y_f.size(); i++) {
                    const C* u = reinterpret_cast<const C*>(base + off4y) + 220 * in4y_g[i];
                    P.u[P.n] = u;
                    P.V[P.n] = u + 200;
                    P.field[P.n] = in4y_f[i];
                    P.out[P.n] = in4y_out[i];
                    if (in4y_ik[i]) P.ik |= 1ull << P.n;
                    if (in4y_last[i]) P.last |= 1ull << P.n;
                    P.n++;
                }
                P.kscale = (float)(2.0 * M_PI * (1.0 / ((double)c->ny * c->h[1])));
                c->have_p4y = true;
            }
            if (sched == QPD_SCHED_FUSED && f4x && 2 * G2 <= kPass4kMax) {
                Pass4k& P = c->p4x;
                std::memset(&P, 0, sizeof P);
                for (int g2 = 0; g2 < G2; g2++)
                    for (int kind = 0; kind < 2; kind++) {
                        const C* u = reinterpret_cast<const C*>(base + off4x) + 220 * g2;
                        P.u[P.n] = u;
                        P.V[P.n] = u + 200;
                        P.field[P.n] = 2 * g2 + kind;
                        if (kind) P.ik |= 1ull << P.n;
                        P.n++;
                    }
                P.last = 1ull << (P.n - 1);
                P.kscale = (float)(2.0 * M_PI * (1.0 / ((double)c->nx * c->h[0])));
                c->have_p4x = true;
            }
        }
        for (auto& s : segX) fix(s);
        for (auto& s : segAX) fix(s);
        for (auto& s : segAY) fix(s);
        if (!segY.empty()) std::memcpy(host.data() + c->off_segY, segY.data(), sizeof(Segment<T>) * segY.size());
        if (!segAX.empty()) std::memcpy(host.data() + c->off_segAX, segAX.data(), sizeof(Segment<T>) * segAX.size());
        if (!segAY.empty()) std::memcpy(host.data() + c->off_segAY, segAY.data(), sizeof(Segment<T>) * segAY.size());
        std::memcpy(host.data() + c->off_segX, segX.data(), sizeof(Segment<T>));
        QPD_CU(c, cudaMemcpyAsync(c->tables.p, host.data(), host.size(), cudaMemcpyHostToDevice, c->stream));
        QPD_CU(c, cudaStreamSynchronize(c->stream));

        const size_t fb = sched == QPD_SCHED_FUSED ? (size_t)3 * G1 * c->n * sizeof(C) : (size_t)2 * c->n * sizeof(C);
        QPD_TRY(dev_reserve(c, c->fields, fb, "field workspace"));
        return QPD_OK;
    }

    template <typename A> static A* tab(qpd_ctx* c, size_t off) {
        return reinterpret_cast<A*>(static_cast<unsigned char*>(c->tables.p) + off);
    }

    // ---------------- launches ----------------
    template <int NT, int EPT> static int launch_z(qpd_ctx* c, ZArgs<T>& a, cudaStream_t st) {
        const int cap = NT * EPT / 4;
        a.M = std::max(1, (int)std::min<int64_t>(cap / a.nz, a.ncols));
        a.ps = odd_stride(a.nz);
        const size_t smem = sizeof(C) * 4 * a.M * a.ps + sizeof(AtomPhase<T>) * a.in.nPhase * a.nAtom + 16;
        QPD_TRY(set_smem(c, zstage_kernel<T, NT, EPT>, smem));
        const int64_t grid = (a.ncols + a.M - 1) / a.M;
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        zstage_kernel<T, NT, EPT><<<(unsigned)grid, NT, smem, st>>>(a);
        return tstop(c, QPD_K_ZSTAGE, st, t0);
    }

    static int run_z(qpd_ctx* c, ZArgs<T>& a, cudaStream_t st) {
        const size_t lim = max_smem(c);
        for (const Cfg& f : kZCfg) {
            const int cap = f.nt * f.ept / 4;
            if (a.nz > cap) continue;
            const int M = std::max(1, (int)std::min<int64_t>(cap / a.nz, a.ncols));
            const size_t smem = sizeof(C) * 4 * M * odd_stride(a.nz) + sizeof(AtomPhase<T>) * a.in.nPhase * a.nAtom + 16;
            if (smem > lim) continue;
            if (f.nt == 256 && f.ept == 16) return launch_z<256, 16>(c, a, st);
            if (f.nt == 512 && f.ept == 16) return launch_z<512, 16>(c, a, st);
            if (f.nt == 1024 && f.ept == 8) return launch_z<1024, 8>(c, a, st);
            if (f.nt == 1024 && f.ept == 16) return launch_z<1024, 16>(c, a, st);
        }
        return fail(c, QPD_ERR_UNSUPPORTED, "nz = %d is too long for the z stage in this precision", a.nz);
    }

    template <int NT, int EPT> static int launch_fftz(qpd_ctx* c, FftzArgs<T>& a, cudaStream_t st) {
        a.M = std::max(1, (int)std::min<int64_t>(NT * EPT / a.nz, a.ncols));
        a.ps = odd_stride(a.nz);
        const size_t smem = sizeof(C) * a.M * a.ps + 16;
        QPD_TRY(set_smem(c, fftz_kernel<T, NT, EPT>, smem));
        const int64_t grid = (a.ncols + a.M - 1) / a.M;
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        fftz_kernel<T, NT, EPT><<<(unsigned)grid, NT, smem, st>>>(a);
        return tstop(c, QPD_K_FFTZ, st, t0);
    }

    static int run_fftz(qpd_ctx* c, FftzArgs<T>& a, cudaStream_t st) {
        const size_t lim = max_smem(c);
        for (const Cfg& f : kZCfg) {
            const int cap = f.nt * f.ept;
            if (a.nz > cap) continue;
            const int M = std::max(1, (int)std::min<int64_t>(cap / a.nz, a.ncols));
            if (sizeof(C) * M * odd_stride(a.nz) + 16 > lim) continue;
            if (f.nt == 256 && f.ept == 16) return launch_fftz<256, 16>(c, a, st);
            if (f.nt == 512 && f.ept == 16) return launch_fftz<512, 16>(c, a, st);
            if (f.nt == 1024 && f.ept == 8) return launch_fftz<1024, 8>(c, a, st);
            if (f.nt == 1024 && f.ept == 16) return launch_fftz<1024, 16>(c, a, st);
        }
        return fail(c, QPD_ERR_UNSUPPORTED, "nz = %d is too long for the z transform in this precision", a.nz);
    }

    template <int NT, int EPT, int EPI>
    static int launch_axis(qpd_ctx* c, AxisArgs<T>& a, int64_t nouter, int kind, cudaStream_t st) {
        a.Cz = std::max(1, std::min(a.nz, NT * EPT / a.N));
        a.nzc = (a.nz + a.Cz - 1) / a.Cz;
        const size_t smem = sizeof(C) * a.N * a.Cz + 16;
        QPD_TRY(set_smem(c, axis_kernel<T, NT, EPT, EPI>, smem));
        const int64_t grid = nouter * a.nzc;
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        axis_kernel<T, NT, EPT, EPI><<<(unsigned)grid, NT, smem, st>>>(a);
        return tstop(c, kind, st, t0);
    }

    template <int EPI> static int run_axis(qpd_ctx* c, AxisArgs<T>& a, int64_t nouter, int kind, cudaStream_t st) {
        const size_t lim = max_smem(c);
        int best = -1, bestCz = 0;
        for (int i = 0; i < 4; i++) {
            const Cfg& f = kACfg[i];
            const int cap = f.nt * f.ept;
            if (a.N > cap) continue;
            const int Cz = std::min(a.nz, cap / a.N);
            if (sizeof(C) * a.N * Cz + 16 > lim) continue;
            // prefer a z chunk of up to 8 (64-byte rows in float32), then fewer threads
            if (best < 0 || std::min(Cz, 8) > std::min(bestCz, 8)) {
                best = i;
                bestCz = Cz;
            }
        }
        switch (best) {
            case 0: return launch_axis<256, 16, EPI>(c, a, nouter, kind, st);
            case 1: return launch_axis<512, 16, EPI>(c, a, nouter, kind, st);
            case 2: return launch_axis<1024, 8, EPI>(c, a, nouter, kind, st);
            case 3: return launch_axis<1024, 16, EPI>(c, a, nouter, kind, st);
        }
        return fail(c, QPD_ERR_UNSUPPORTED, "an axis of length %d is too long in this precision", a.N);
    }

    // ---------------- adjoint (generic kernels) ----------------
    template <int NT, int EPT> static int launch_adj_axis(qpd_ctx* c, AxisArgs<T>& a, int64_t nouter, cudaStream_t st) {
        a.Cz = std::max(1, std::min(a.nz, NT * EPT / a.N));
        a.nzc = (a.nz + a.Cz - 1) / a.Cz;
        const size_t smem = sizeof(C) * a.N * a.Cz + 16;
        QPD_TRY(set_smem(c, adj_axis_kernel<T, NT, EPT>, smem));
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        adj_axis_kernel<T, NT, EPT><<<(unsigned)(nouter * a.nzc), NT, smem, st>>>(a);
        return tstop(c, QPD_K_ADJAXIS, st, t0);
    }

    // adjoint x / y pass on the TMA kernel (coefficients before the transform), for the lengths the
    // forward specialises; nfields_in: fields of the adjoint workspace the input lives in
    template <int N, int NT, class RAD>
    static int adj_tma_(qpd_ctx* c, AxisArgs<T>& a, int64_t nouter, bool xp, cudaStream_t st, int64_t nfields_in) {
        if (xp) return tma_axis_b<N, 8, NT, 2, false, true, RAD, 2, true, false, true>(c, a, nouter, QPD_K_ADJAXIS, st,
                                                                                   nfields_in);
        return tma_axis_b<N, 8, NT, 2, false, false, RAD, 2, true, false, true>(c, a, nouter, QPD_K_ADJAXIS, st,
                                                                             nfields_in);
    }

    static int run_adj_axis(qpd_ctx* c, AxisArgs<T>& a, int64_t nouter, cudaStream_t st, bool xp = false,
                            int64_t nfields_in = 0) {
        if constexpr (sizeof(T) == 4) {
            if (c->fast && c->tma && c->knob_adj_tma && nfields_in > 0 && a.nz % 2 == 0) {
                if (a.N == 256) return adj_tma_<256, 256, Radix<8, 8, 4>>(c, a, nouter, xp, st, nfields_in);
                if (a.N == 512) return adj_tma_<512, 512, Radix<8, 8, 8>>(c, a, nouter, xp, st, nfields_in);
            }
        }
        const size_t lim = max_smem(c);
        int best = -1, bestCz = 0;
        for (int i = 0; i < 4; i++) {
            const Cfg& f = kACfg[i];
            const int cap = f.nt * f.ept;
            if (a.N > cap) continue;
            const int Cz = std::min(a.nz, cap / a.N);
            if (sizeof(C) * a.N * Cz + 16 > lim) continue;
            if (best < 0 || std::min(Cz, 8) > std::min(bestCz, 8)) {
                best = i;
                bestCz = Cz;
            }
        }
        switch (best) {
            case 0: return launch_adj_axis<256, 16>(c, a, nouter, st);
            case 1: return launch_adj_axis<512, 16>(c, a, nouter, st);
            case 2: return launch_adj_axis<1024, 8>(c, a, nouter, st);
            case 3: return launch_adj_axis<1024, 16>(c, a, nouter, st);
        }
        return fail(c, QPD_ERR_UNSUPPORTED, "an axis of length %d is too long for the adjoint in this precision", a.N);
    }

    template <int NT, int EPT> static int launch_adj_z(qpd_ctx* c, AdjZArgs<T>& a, cudaStream_t st) {
        const int cap = NT * EPT / 4;
        a.z.M = std::max(1, (int)std::min<int64_t>(cap / a.z.nz, a.z.ncols));
        a.z.ps = odd_stride(a.z.nz);
        const size_t smem = sizeof(C) * 4 * a.z.M * a.z.ps + sizeof(AtomPhase<T>) * a.z.in.nPhase * a.z.nAtom + 16;
        QPD_TRY(set_smem(c, adj_zstage_kernel<T, NT, EPT>, smem));
        const int64_t grid = (a.z.ncols + a.z.M - 1) / a.z.M;
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        adj_zstage_kernel<T, NT, EPT><<<(unsigned)grid, NT, smem, st>>>(a);
        return tstop(c, QPD_K_ADJZ, st, t0);
    }

    template <int NZ, int M, int NT, class RAD> static int adj_z_fast_(qpd_ctx* c, AdjZArgs<T>& a, cudaStream_t st) {
        constexpr int PS = NZ % 2 ? NZ : NZ + 1;
        a.z.M = M;
        a.z.ps = PS;
        // transform buffer (4 planes), two stages of the 3 input fields, the atom table
        const size_t smem = sizeof(C) * (4 * M * PS + 6 * M * NZ) + sizeof(AtomPhase<T>) * a.z.in.nPhase * a.z.nAtom + 16;
        if (smem > max_smem(c)) return run_adj_z(c, a, st);
        QPD_TRY(set_smem(c, adj_zstage_fast<T, NZ, M, NT, RAD>, smem));
        const int64_t grid = (a.z.ncols + M - 1) / M;
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        adj_zstage_fast<T, NZ, M, NT, RAD><<<(unsigned)grid, NT, smem, st>>>(a);
        return tstop(c, QPD_K_ADJZ, st, t0);
    }

    static int run_adj_z(qpd_ctx* c, AdjZArgs<T>& a, cudaStream_t st) {
        const size_t lim = max_smem(c);
        for (const Cfg& f : kZCfg) {
            const int cap = f.nt * f.ept / 4;
            if (a.z.nz > cap) continue;
            const int M = std::max(1, (int)std::min<int64_t>(cap / a.z.nz, a.z.ncols));
            const size_t smem = sizeof(C) * 4 * M * odd_stride(a.z.nz) + sizeof(AtomPhase<T>) * a.z.in.nPhase * a.z.nAtom + 16;
            if (smem > lim) continue;
            if (f.nt == 256 && f.ept == 16) return launch_adj_z<256, 16>(c, a, st);
            if (f.nt == 512 && f.ept == 16) return launch_adj_z<512, 16>(c, a, st);
            if (f.nt == 1024 && f.ept == 8) return launch_adj_z<1024, 8>(c, a, st);
            if (f.nt == 1024 && f.ept == 16) return launch_adj_z<1024, 16>(c, a, st);
        }
        return fail(c, QPD_ERR_UNSUPPORTED, "nz = %d is too long for the adjoint z stage in this precision", a.z.nz);
    }

    // ---------------- compile-time specialised kernels ----------------
    template <int NZ, int M, int NT, class RAD> static int fast_z_(qpd_ctx* c, ZArgs<T>& a, cudaStream_t st) {
        constexpr int PS = NZ % 2 ? NZ : NZ + 1;
        a.M = M;
        a.ps = PS;
        const size_t smem = sizeof(C) * 4 * M * PS + sizeof(AtomPhase<T>) * a.in.nPhase * a.nAtom + 16;
        QPD_TRY(set_smem(c, zstage_fast<T, NZ, M, NT, RAD>, smem));
        const int64_t grid = (a.ncols + M - 1) / M;
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        zstage_fast<T, NZ, M, NT, RAD><<<(unsigned)grid, NT, smem, st>>>(a);
        return tstop(c, QPD_K_ZSTAGE, st, t0);
    }

    // CTAs of a persistent z stage (each walks tiles gridDim.x apart): one wave of per_sm CTAs per SM, or
    // with qpd_set_cta_tiles(k) enough CTAs that each takes at most k tiles, so that CTAs retire every k
    // tiles and the block scheduler can start other streams' (higher-priority) kernels in between
    static int64_t z_grid(const qpd_ctx* c, int64_t ntiles, int per_sm, int sms) {
        const int64_t wave = (int64_t)std::max(per_sm, 1) * sms;
        const int64_t grid = c->cta_tiles > 0 ? std::max(wave, (ntiles + c->cta_tiles - 1) / c->cta_tiles) : wave;
        return std::max<int64_t>(1, std::min<int64_t>(ntiles, grid));
    }

    template <int NZ, int M, int NT, class RAD, bool REGIN = false>
    static int smem_z_(qpd_ctx* c, ZArgs<T>& a, cudaStream_t st) {
        using L = ZLayout<T, NZ, M>;
        a.M = M;
        a.ps = L::PS;
        const size_t smem = L::bytes(a.in.nPhase * a.nAtom, a.nAtom);
        if (smem > max_smem(c)) return fail(c, QPD_ERR_UNSUPPORTED, "z stage tables exceed shared memory");
        QPD_TRY(set_smem(c, zstage_pipe<T, NZ, M, NT, RAD, REGIN>, smem));
        int per_sm = 0, sms = 0;
        QPD_CU(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, zstage_pipe<T, NZ, M, NT, RAD, REGIN>, NT,
                                                                smem));
        QPD_CU(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
        const int64_t ntiles = (a.ncols + M - 1) / M;
        const int64_t grid = z_grid(c, ntiles, per_sm, sms);
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        zstage_pipe<T, NZ, M, NT, RAD, REGIN><<<(unsigned)grid, NT, smem, st>>>(a);
        return tstop(c, QPD_K_ZSTAGE, st, t0);
    }

    template <int N1, int N2> static int pfa_z_(qpd_ctx* c, ZArgs<T>& a, cudaStream_t st) {
        using L = ZPfaLayout<T, N1, N2>;
        constexpr int NT = ZPfa<N1, N2>::NT;
        a.M = L::M;
        a.ps = L::PS;
        const size_t smem = L::bytes(a.in.nPhase * a.nAtom, a.nAtom);
        if (smem > max_smem(c)) return fail(c, QPD_ERR_UNSUPPORTED, "z stage tables exceed shared memory");
        QPD_TRY(set_smem(c, zstage_pfa<T, N1, N2>, smem));
        int per_sm = 0, sms = 0;
        QPD_CU(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, zstage_pfa<T, N1, N2>, NT, smem));
        QPD_CU(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
        const int64_t ntiles = (a.ncols + L::M - 1) / L::M;
        const int64_t grid = z_grid(c, ntiles, per_sm, sms);
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        zstage_pfa<T, N1, N2><<<(unsigned)grid, NT, smem, st>>>(a);
        return tstop(c, QPD_K_ZSTAGE, st, t0);
    }

    // Returns QPD_OK and sets *done when an instantiation covers nz.
    static int fast_z(qpd_ctx* c, ZArgs<T>& a, cudaStream_t st, bool* done) {
        *done = true;
        constexpr bool F = sizeof(T) == 4;
        if constexpr (F) {
            // single-phase inputs: the register-fused prime-factor z stage
            if (c->tma && !a.in.wdense && a.nAtom <= 16) {
                if (a.nz == 104 && c->knob_zpfa == 1 &&
                    ZPfaLayout<T, 8, 13>::bytes(a.in.nPhase * a.nAtom, a.nAtom) <= max_smem(c))
                    return pfa_z_<8, 13>(c, a, st);
                if (a.nz == 68 && c->knob_zpfa != 0 &&
                    ZPfaLayout<T, 4, 17>::bytes(a.in.nPhase * a.nAtom, a.nAtom) <= max_smem(c))
                    return pfa_z_<4, 17>(c, a, st);
            }
        }
        if (c->tma && ZLayout<T, 128, 8>::bytes(a.in.nPhase * a.nAtom, a.nAtom) <= max_smem(c)) {
            switch (a.nz) {
                case 32: return smem_z_<32, F ? 32 : 16, F ? 512 : 256, Radix<8, 4>>(c, a, st);
                case 64:
                    if (F && c->knob_zregin == 1) return smem_z_<64, 16, 256, Radix<8, 8>, true>(c, a, st);
                    return smem_z_<64, F ? 16 : 8, F ? 512 : 256, Radix<8, 8>>(c, a, st);
                case 68: return smem_z_<68, F ? 12 : 6, F ? 416 : 224, Pfa<4, 17>>(c, a, st);
                case 104:
                    // float: 256 threads with each thread's inputs in registers measured fastest (1.82 ms at
                    // 512x512x104 against 1.86 for 416 threads reading them from shared memory per atom)
                    if (F && c->knob_z == 1) return smem_z_<104, 8, 416, Pfa<8, 13>>(c, a, st);
                    if (F) return smem_z_<104, 8, 256, Pfa<8, 13>, true>(c, a, st);
                    return smem_z_<104, 4, 224, Pfa<8, 13>>(c, a, st);
                case 128:
                    if (F && c->knob_zregin == 1) return smem_z_<128, 8, 256, Radix<8, 4, 4>, true>(c, a, st);
                    return smem_z_<128, F ? 8 : 4, F ? 512 : 256, Radix<8, 4, 4>>(c, a, st);
            }
        }
        switch (a.nz) {
            case 32: return fast_z_<32, F ? 32 : 16, 256, Radix<8, 4>>(c, a, st);
            case 64: return fast_z_<64, F ? 16 : 8, 256, Radix<8, 8>>(c, a, st);
            case 68: return fast_z_<68, F ? 12 : 6, 256, Radix<4, 17>>(c, a, st);
            case 104: return fast_z_<104, F ? 8 : 4, 256, Radix<8, 13>>(c, a, st);
            case 128: return fast_z_<128, F ? 8 : 4, 256, Radix<8, 4, 4>>(c, a, st);
        }
        *done = false;
        return QPD_OK;
    }

    template <int N, int CZ, int NT, int VEC, bool EPI, class RAD>
    static int fast_axis_(qpd_ctx* c, AxisArgs<T>& a, int64_t nouter, int kind, cudaStream_t st) {
        a.Cz = CZ;
        a.nzc = (a.nz + CZ - 1) / CZ;
        const size_t smem = sizeof(C) * N * CZ + 16;
        QPD_TRY(set_smem(c, axis_fast<T, N, CZ, NT, VEC, EPI, RAD>, smem));
        const int64_t grid = nouter * a.nzc;
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        axis_fast<T, N, CZ, NT, VEC, EPI, RAD><<<(unsigned)grid, NT, smem, st>>>(a);
        return tstop(c, kind, st, t0);
    }

    template <int N, int CZ, int NT, int VEC, bool EPI, bool XP, class RAD>
    static int tma_axis_(qpd_ctx* c, AxisArgs<T>& a, int64_t nouter, int kind, cudaStream_t st) {
        if constexpr (sizeof(T) == 4 && (N == 512 || N == 256)) {
            if (c->knob_oop == 1) return tma_axis_b<N, CZ, NT, VEC, EPI, XP, RAD, 2, true>(c, a, nouter, kind, st);
        }
        if (c->knob_nbuf == 2) return tma_axis_b<N, CZ, NT, VEC, EPI, XP, RAD, 2>(c, a, nouter, kind, st);
        return tma_axis_b<N, CZ, NT, VEC, EPI, XP, RAD, 3>(c, a, nouter, kind, st);
    }

    // YZ: the x pass over fields laid out (x, k_z, y): a.nz is then the y extent and nouter the k_z extent
    // nfields_in: fields of the input buffer the tensor map covers (default: the forward's field workspace)
    template <int N, int CZ, int NT, int VEC, bool EPI, bool XP, class RAD, int NBUF, bool OOP = false, bool YZ = false,
              bool PRE = false, bool SEED = false>
    static int tma_axis_b(qpd_ctx* c, AxisArgs<T>& a, int64_t nouter, int kind, cudaStream_t st,
                          int64_t nfields_in = -1) {
        constexpr int BOX = tma_rows(N, CZ * (int)sizeof(C));
        a.Cz = CZ;
        a.nzc = (a.nz + CZ - 1) / CZ;
        a.nouter = (int)nouter;
        CUtensorMap map;
        const int64_t nfields = nfields_in > 0 ? nfields_in : c->sched_used == QPD_SCHED_FUSED ? 3 * c->ng1 : 2;
        QPD_TRY(field_map(c, &map, const_cast<C*>(a.in), sizeof(T) == 8, a.nz, YZ ? c->nz : c->ny, nfields * c->nx,
                          2 * CZ, XP ? 1 : BOX, XP ? BOX : 1));
        const size_t smem = sizeof(C) * N * CZ * (NBUF + (OOP ? 1 : 0)) + sizeof(C) * N + 128;
        if (smem > max_smem(c)) return fail(c, QPD_ERR_UNSUPPORTED, "axis tile exceeds shared memory");
        QPD_TRY(set_smem(c, axis_tma<T, N, CZ, NT, VEC, EPI, XP, RAD, NBUF, OOP, YZ, PRE, SEED>, smem));
        const int64_t grid = nouter * a.nzc;
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        axis_tma<T, N, CZ, NT, VEC, EPI, XP, RAD, NBUF, OOP, YZ, PRE, SEED><<<(unsigned)grid, NT, smem, st>>>(map, a);
        return tstop(c, kind, st, t0);
    }

    // y pass over fields laid out (x, k_z, y): one contiguous pencil per CTA (axis_bulk)
    template <int N, int NT, class RAD> static int bulk_axis_(qpd_ctx* c, AxisArgs<T>& a, cudaStream_t st) {
        const size_t smem = sizeof(C) * (3 * N + (N + 63) / 64 + 64) + 128;
        if (smem > max_smem(c)) return fail(c, QPD_ERR_UNSUPPORTED, "axis pencils exceed shared memory");
        QPD_TRY(set_smem(c, axis_bulk<T, N, NT, RAD>, smem));
        const int64_t grid = c->nx * c->nz;
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        axis_bulk<T, N, NT, RAD><<<(unsigned)grid, NT, smem, st>>>(a);
        return tstop(c, QPD_K_YPASS, st, t0);
    }

    // The 4000 x 4000 x 68 route: fused z stage writing y-fastest fields, bulk y pass, swapped x pass.
    static bool yfast_ok(qpd_ctx* c, const Inputs<T>& in) {
        if constexpr (sizeof(T) != 4) return false;
        return c->knob_yfast && c->fast && c->tma && c->knob_zpfa != 0 && !in.wdense && c->nAtom <= 16 &&
               c->nx == 4000 && c->ny == 4000 && c->nz == 68 &&
               ZPfaLayout<T, 4, 17>::bytes(in.nPhase * c->nAtom, c->nAtom) <= max_smem(c);
    }

    // The y-fastest route on the register-resident passes: (k_z, x, y) fields, bulk y pass, strided x pass
    // (the shared-memory Stockham passes read the (x, k_z, y) layout instead).
    static bool yfast4k(const qpd_ctx* c) { return c->knob_n4k && c->have_p4y && c->have_p4x; }

    // float: z chunks of 8 complex64 (64-byte rows), 16-byte accesses when nz is even;
    // double: chunks of 4 complex128 (64-byte rows).
    template <int N, int NT, bool EPI, class RAD>
    static int fast_axis_n(qpd_ctx* c, AxisArgs<T>& a, int64_t nouter, int kind, cudaStream_t st) {
        // TMA: the map's row strides must be multiples of 16 bytes (nz even for complex64)
        const bool tma_ok = c->tma && (sizeof(T) == 8 || a.nz % 2 == 0);
        if (tma_ok) {
            const bool xp = kind == QPD_K_XPASS || (kind == QPD_K_AXIS && a.stride != a.nz);
            if constexpr (sizeof(T) == 4) {
                if (xp) return tma_axis_<N, 8, NT, 2, EPI, true, RAD>(c, a, nouter, kind, st);
                return tma_axis_<N, 8, NT, 2, EPI, false, RAD>(c, a, nouter, kind, st);
            } else {
                if (xp) return tma_axis_<N, 4, NT, 1, EPI, true, RAD>(c, a, nouter, kind, st);
                return tma_axis_<N, 4, NT, 1, EPI, false, RAD>(c, a, nouter, kind, st);
            }
        }
        if constexpr (sizeof(T) == 4) {
            if (a.nz % 2 == 0) return fast_axis_<N, 8, NT, 2, EPI, RAD>(c, a, nouter, kind, st);
            return fast_axis_<N, 8, NT, 1, EPI, RAD>(c, a, nouter, kind, st);
        } else {
            return fast_axis_<N, 4, NT, 1, EPI, RAD>(c, a, nouter, kind, st);
        }
    }

    template <bool EPI> static int fast_axis(qpd_ctx* c, AxisArgs<T>& a, int64_t nouter, int kind, cudaStream_t st,
                                            bool* done) {
        *done = true;
        switch (a.N) {
            case 32: return fast_axis_n<32, 128, EPI, Radix<8, 4>>(c, a, nouter, kind, st);
            case 64: return fast_axis_n<64, 128, EPI, Radix<8, 8>>(c, a, nouter, kind, st);
            case 128: return fast_axis_n<128, 128, EPI, Radix<8, 4, 4>>(c, a, nouter, kind, st);
            case 256: return fast_axis_n<256, 256, EPI, Radix<8, 8, 4>>(c, a, nouter, kind, st);
            case 512: return fast_axis_n<512, 512, EPI, Radix<8, 8, 8>>(c, a, nouter, kind, st);
            case 1024: return fast_axis_n<1024, 1024, EPI, Radix<8, 8, 4, 4>>(c, a, nouter, kind, st);
            case 4000:
                if constexpr (sizeof(T) == 4) {
                    if (c->knob_n4k && c->tma && kind == QPD_K_YPASS && c->have_p4y && a.nz == 1 && !a.accumulate) {
                        // one z value: every y pencil is contiguous, so the bulk y pass reads it whole
                        cudaEvent_t t0;
                        QPD_TRY(tstart(c, st, &t0));
                        QPD_CU(c, launch_ypass4000(a, c->p4y, c->nx, st));
                        return tstop(c, kind, st, t0);
                    }
                    const bool yp = kind == QPD_K_YPASS && c->have_p4y, xp4 = kind == QPD_K_XPASS && c->have_p4x;
                    if (c->knob_n4k && c->tma && a.nz % 2 == 0 && !a.accumulate && (yp || xp4)) {
                        // register-resident passes over tiles of two neighbouring z values: rows along y for the y
                        // pass, along x for the x pass
                        CUtensorMap map;
                        const int64_t nfields = 3 * c->ng1;
                        QPD_TRY(field_map(c, &map, const_cast<C*>(a.in), false, c->nz, c->ny, nfields * c->nx, 4,
                                          yp ? 200 : 1, yp ? 1 : 200));
                        cudaEvent_t t0;
                        QPD_TRY(tstart(c, st, &t0));
                        QPD_CU(c, launch_strided4000(map, a, yp ? c->p4y : c->p4x, (int)nouter,
                                                     yp ? Strided4k::YPassZFast : Strided4k::XPassZFast, st));
                        return tstop(c, kind, st, t0);
                    }
                }
                // 4000 x 2 tiles (16-byte rows: the other half of each 32-byte sector is read by the CTA of
                // the neighbouring z chunk while it is still in L2), 200-row boxes, two buffers
                if constexpr (sizeof(T) == 4) {
                    if (c->tma && a.nz % 2 == 0) {
                        const bool xp = kind == QPD_K_XPASS || (kind == QPD_K_AXIS && a.stride != a.nz);
                        using R4000 = Radix<8, 4, 5, 5, 5>;
                        if (c->knob_n4000 == 1) {  // one tile buffer: two CTAs per SM
                            if (xp) return tma_axis_b<4000, 2, 512, 2, EPI, true, R4000, 1>(c, a, nouter, kind, st);
                            return tma_axis_b<4000, 2, 512, 2, EPI, false, R4000, 1>(c, a, nouter, kind, st);
                        }
                        if (c->knob_n4000 == 2) {  // 1024 threads, two tile buffers
                            if (xp) return tma_axis_b<4000, 2, 1024, 2, EPI, true, R4000, 2>(c, a, nouter, kind, st);
                            return tma_axis_b<4000, 2, 1024, 2, EPI, false, R4000, 2>(c, a, nouter, kind, st);
                        }
                        if (c->knob_n4000 == 4) {  // 1024 threads, out-of-place stages
                            if (xp) return tma_axis_b<4000, 2, 1024, 2, EPI, true, R4000, 2, true>(c, a, nouter, kind, st);
                            return tma_axis_b<4000, 2, 1024, 2, EPI, false, R4000, 2, true>(c, a, nouter, kind, st);
                        }
                        if (c->knob_n4000 == 3) {  // in-place stages (registers hold all butterflies of a stage)
                            if (xp) return tma_axis_b<4000, 2, 512, 2, EPI, true, R4000, 2>(c, a, nouter, kind, st);
                            return tma_axis_b<4000, 2, 512, 2, EPI, false, R4000, 2>(c, a, nouter, kind, st);
                        }
                        // out-of-place swizzled stages: 3 tiles of 64 KB + twiddles, one barrier per stage;
                        // measured at 4000x4000x68: y pass 98.2 ms with 512 threads (108.8 with 1024), x pass
                        // 53.2 ms
                        if (xp) return tma_axis_b<4000, 2, 512, 2, EPI, true, R4000, 2, true>(c, a, nouter, kind, st);
                        return tma_axis_b<4000, 2, 512, 2, EPI, false, R4000, 2, true>(c, a, nouter, kind, st);
                    }
                }
                break;
        }
        *done = false;
        return QPD_OK;
    }

    static Inputs<T> inputs(qpd_ctx* c, const void* P, const void* U, const int8_t* phase, const void* weight,
                            const void* wdense) {
        Inputs<T> in;
        in.P = static_cast<const T*>(P);
        in.U = static_cast<const T*>(U);
        in.phase = reinterpret_cast<const signed char*>(phase);
        in.weight = static_cast<const T*>(weight);
        in.wdense = static_cast<const T*>(wdense);
        in.n = c->n;
        in.nStruc = c->nStruc;
        in.nPhase = c->nPhase;
        return in;
    }

    // fused z stage (source + z transform + fold) and y pass, leaving 2 ng2 fields in c->fields
    static ZArgs<T> zargs(qpd_ctx* c, const Inputs<T>& in) {
        ZArgs<T> z;
        std::memset(&z, 0, sizeof z);
        z.in = in;
        z.ncols = c->nx * c->ny;
        z.nz = (int)c->nz;
        z.nAtom = c->nAtom;
        z.apc = tab<AtomPhase<T>>(c, c->off_apc);
        z.coefE = tab<C>(c, c->off_coefE);
        z.coefUz = tab<C>(c, c->off_coefUz);
        for (int i = 0; i < c->nAtom; i++) z.grp[i] = c->grp[i];
        z.out = static_cast<C*>(c->fields.p);
        z.fstride = c->n;
        for (int d = 0; d < 3; d++) z.tq[d] = c->tq[d];
        z.zp = axis_plan(c, 2);
        z.status = static_cast<int*>(c->status.p);
        return z;
    }

    static AxisArgs<T> xargs(qpd_ctx* c) {
        AxisArgs<T> x;
        std::memset(&x, 0, sizeof x);
        x.N = (int)c->nx;
        x.stride = c->ny * c->nz;
        x.ostride = c->nz;
        x.nz = (int)c->nz;
        x.in = static_cast<C*>(c->fields.p);
        x.fstride = c->n;
        x.segs = tab<Segment<T>>(c, c->off_segX);
        x.nseg = 1;
        x.ap = axis_plan(c, 0);
        for (int d = 0; d < 3; d++) x.S[d] = tab<double>(c, c->off_S[d]);
        x.scale2 = c->scale2;
        x.nx = c->nx;
        x.ny = c->ny;
        x.status = static_cast<int*>(c->status.p);
        return x;
    }

    // Gradient of a loss through the fused schedule: recompute the forward to the x pass, seed,
    // then the adjoint x, y and z passes (the last fused with the source transpose).
    static int adjoint(qpd_ctx* c, const Inputs<T>& in, const double* dI, T* dP, T* dU, cudaStream_t st) {
        const int64_t n = c->n;
        QPD_TRY(dev_reserve(c, c->adjw, sizeof(C) * (size_t)(1 + 2 * c->ng2) * n, "adjoint workspace"));
        C* F = static_cast<C*>(c->fields.p);
        C* W = static_cast<C*>(c->adjw.p);
        QPD_TRY(forward_zy(c, in, st));

        AxisArgs<T> x = xargs(c);
        x.out = W;
        x.gI = dI;
        bool seeded = false;
        if constexpr (sizeof(T) == 4) {
            if (c->fast && c->tma && c->knob_adj_tma && c->nz % 2 == 0) {
                using namespace qpd;
                if (c->nx == 256) {
                    QPD_TRY((tma_axis_b<256, 8, 256, 2, true, true, Radix<8, 8, 4>, 2, true, false, false, true>(
                        c, x, c->ny, QPD_K_ADJSEED, st)));
                    seeded = true;
                } else if (c->nx == 512) {
                    QPD_TRY((tma_axis_b<512, 8, 512, 2, true, true, Radix<8, 8, 8>, 2, true, false, false, true>(
                        c, x, c->ny, QPD_K_ADJSEED, st)));
                    seeded = true;
                }
            }
        }
        if (!seeded) QPD_TRY(run_axis<2>(c, x, c->ny, QPD_K_ADJSEED, st));

        AxisArgs<T> ax;
        std::memset(&ax, 0, sizeof ax);
        ax.N = (int)c->nx;
        ax.stride = c->ny * c->nz;
        ax.ostride = c->nz;
        ax.nz = (int)c->nz;
        ax.in = W;
        ax.out = W;
        ax.fstride = n;
        ax.segs = tab<Segment<T>>(c, c->off_segAX);
        ax.nseg = c->nsegAX;
        ax.ap = axis_plan(c, 0);
        ax.nx = c->nx;
        ax.ny = c->ny;
        ax.status = static_cast<int*>(c->status.p);
        QPD_TRY(run_adj_axis(c, ax, c->ny, st, true, 1 + 2 * c->ng2));

        AxisArgs<T> ay;
        std::memset(&ay, 0, sizeof ay);
        ay.N = (int)c->ny;
        ay.stride = c->nz;
        ay.ostride = c->ny * c->nz;
        ay.nz = (int)c->nz;
        ay.in = W;
        ay.out = F;
        ay.fstride = n;
        ay.segs = tab<Segment<T>>(c, c->off_segAY);
        ay.nseg = c->nsegAY;
        ay.ap = axis_plan(c, 1);
        ay.nx = c->nx;
        ay.ny = c->ny;
        ay.status = static_cast<int*>(c->status.p);
        QPD_TRY(run_adj_axis(c, ay, c->nx, st, false, 1 + 2 * c->ng2));

        AdjZArgs<T> az;
        std::memset(&az, 0, sizeof az);
        az.z = zargs(c, in);
        az.fin = F;
        az.dU = dU;
        az.dP = dP;
        for (int d = 0; d < 3; d++) az.qc[d] = 2.0 * M_PI * c->tq[d];
        if constexpr (sizeof(T) == 4) {
            if (c->fast && c->knob_adj_tma && !in.wdense) {
                if (c->nz == 64) return adj_z_fast_<64, 16, 256, Radix<8, 8>>(c, az, st);
                if (c->nz == 104) return adj_z_fast_<104, 8, 256, Pfa<8, 13>>(c, az, st);
            }
        }
        return run_adj_z(c, az, st);
    }

    static int forward_zy(qpd_ctx* c, const Inputs<T>& in, cudaStream_t st, bool yfast = false) {
        C* F = static_cast<C*>(c->fields.p);
        const int64_t n = c->n;
        {
            ZArgs<T> z = zargs(c, in);
            bool done = false;
            if constexpr (sizeof(T) == 4) {
                if (yfast) {
                    z.yfast = yfast4k(c) ? 2 : 1;
                    z.ny = c->ny;
                    QPD_TRY((pfa_z_<4, 17>(c, z, st)));
                    done = true;
                }
            }
            if (!done && c->fast) QPD_TRY(fast_z(c, z, st, &done));
            if (!done) QPD_TRY(run_z(c, z, st));

            AxisArgs<T> y;
            std::memset(&y, 0, sizeof y);
            y.N = (int)c->ny;
            y.stride = c->nz;
            y.ostride = c->ny * c->nz;
            y.nz = (int)c->nz;
            y.in = F;
            y.out = F;
            y.fstride = n;
            y.segs = tab<Segment<T>>(c, c->off_segY);
            y.nseg = c->nsegY;
            y.ap = axis_plan(c, 1);
            y.nx = c->nx;
            y.ny = c->ny;
            y.status = static_cast<int*>(c->status.p);
            if (yfast) {
                if constexpr (sizeof(T) == 4) {
                    if (yfast4k(c)) {
                        cudaEvent_t t0;
                        QPD_TRY(tstart(c, st, &t0));
                        QPD_CU(c, launch_ypass4000(y, c->p4y, c->nx * c->nz, st));
                        return tstop(c, QPD_K_YPASS, st, t0);
                    }
                    if (c->knob_bulk_nt == 512) return bulk_axis_<4000, 512, Radix<8, 4, 5, 5, 5>>(c, y, st);
                    return bulk_axis_<4000, 256, Radix<8, 4, 5, 5, 5>>(c, y, st);
                }
            }
            done = false;
            if (c->fast) QPD_TRY(fast_axis<false>(c, y, c->nx, QPD_K_YPASS, st, &done));
            if (!done) QPD_TRY(run_axis<0>(c, y, c->nx, QPD_K_YPASS, st));
        }
        return QPD_OK;
    }

    static int run_device(qpd_ctx* c, const Inputs<T>& in, double* I, cudaStream_t st) {
        C* F = static_cast<C*>(c->fields.p);
        const int64_t n = c->n;
        if (c->sched_used == QPD_SCHED_FUSED) {
            const bool yfast = yfast_ok(c, in);
            QPD_TRY(forward_zy(c, in, st, yfast));
            AxisArgs<T> x = xargs(c);
            x.I = I;
            if constexpr (sizeof(T) == 4) {
                if (yfast) {
                    x.nz = (int)c->ny;  // the contiguous axis of the y-fastest fields
                    if (yfast4k(c)) {
                        // (k_z, x, y) fields: tiles of two neighbouring k_y at one k_z, rows along x (ny values apart)
                        CUtensorMap map;
                        QPD_TRY(field_map(c, &map, const_cast<C*>(x.in), false, c->ny, c->nx, 3 * c->ng1 * c->nz, 4, 200,
                                          1));
                        // the intensity is staged as (k_z, k_y, k_x) rows in a field slot the x pass does not
                        // read (the y pass leaves its outputs in the first 2 G2 slots of 3 G1), then moved to I
                        auto read_by_x = [&](int f) {
                            for (int i = 0; i < c->p4x.n; i++)
                                if (c->p4x.field[i] == f) return true;
                            return false;
                        };
                        int slot = 0;
                        while (read_by_x(slot)) slot++;
                        if (slot >= 3 * c->ng1) return fail(c, QPD_ERR_STATE, "no free field slot for the staged intensity");
                        x.Istage = reinterpret_cast<double*>(F + (int64_t)slot * n);
                        cudaEvent_t t0;
                        QPD_TRY(tstart(c, st, &t0));
                        QPD_CU(c, launch_strided4000(map, x, c->p4x, (int)c->nz, Strided4k::XPassYFast, st));
                        QPD_CU(c, launch_unstage_intensity(x.Istage, I, c->nx, c->ny, c->nz, st));
                        return tstop(c, QPD_K_XPASS, st, t0);
                    }
                    return tma_axis_b<4000, 2, 512, 2, true, true, Radix<8, 4, 5, 5, 5>, 2, true, true>(c, x, c->nz,
                                                                                                    QPD_K_XPASS, st);
                }
            }
            bool done = false;
            if (c->fast) QPD_TRY(fast_axis<true>(c, x, c->ny, QPD_K_XPASS, st, &done));
            if (done) return QPD_OK;
            return run_axis<1>(c, x, c->ny, QPD_K_XPASS, st);
        }
        // plain schedule
        C* buf = F;
        C* amp = F + n;
        QPD_CU(c, cudaMemsetAsync(amp, 0, sizeof(C) * n, st));
        const unsigned blocks = (unsigned)((n + 255) / 256);
        for (int at = 0; at < c->nAtom; at++) {
            for (int comp = 0; comp < 4; comp++) {
                SourceArgs<T> s;
                std::memset(&s, 0, sizeof s);
                s.in = in;
                s.apc = tab<AtomPhase<T>>(c, c->off_apc);
                s.nAtom = c->nAtom;
                s.at = at;
                s.comp = comp;
                for (int d = 0; d < 3; d++) s.tq[d] = c->tq[d];
                s.buf = buf;
                cudaEvent_t t0;
                QPD_TRY(tstart(c, st, &t0));
                source_kernel<T><<<blocks, 256, 0, st>>>(s);
                QPD_TRY(tstop(c, QPD_K_SOURCE, st, t0));

                FftzArgs<T> fz;
                std::memset(&fz, 0, sizeof fz);
                fz.buf = buf;
                fz.ncols = c->nx * c->ny;
                fz.nz = (int)c->nz;
                fz.zp = axis_plan(c, 2);
                QPD_TRY(run_fftz(c, fz, st));

                for (int d = 1; d >= 0; d--) {
                    AxisArgs<T> ax;
                    std::memset(&ax, 0, sizeof ax);
                    ax.N = (int)(d == 1 ? c->ny : c->nx);
                    ax.stride = d == 1 ? c->nz : c->ny * c->nz;
                    ax.ostride = d == 1 ? c->ny * c->nz : c->nz;
                    ax.nz = (int)c->nz;
                    ax.in = buf;
                    ax.out = buf;
                    ax.fstride = n;
                    ax.segs = tab<Segment<T>>(c, c->off_segX);
                    ax.nseg = 1;
                    ax.ap = axis_plan(c, d);
                    ax.nx = c->nx;
                    ax.ny = c->ny;
                    ax.status = static_cast<int*>(c->status.p);
                    QPD_TRY(run_axis<0>(c, ax, d == 1 ? c->nx : c->ny, QPD_K_AXIS, st));
                }

                AccArgs<T> ac;
                ac.amp = amp;
                ac.buf = buf;
                ac.ex = tab<double2>(c, c->off_pex) + (int64_t)at * c->nx;
                ac.ey = tab<double2>(c, c->off_pey) + (int64_t)at * c->ny;
                ac.ez = tab<double2>(c, c->off_pez) + (int64_t)at * c->nz;
                ac.kd = comp > 0 ? tab<double>(c, c->off_k[comp - 1]) : nullptr;
                ac.comp = comp;
                ac.nx = c->nx;
                ac.ny = c->ny;
                ac.nz = c->nz;
                cudaEvent_t t1;
                QPD_TRY(tstart(c, st, &t1));
                accumulate_kernel<T><<<blocks, 256, 0, st>>>(ac);
                QPD_TRY(tstop(c, QPD_K_ACC, st, t1));
            }
        }
        IntensityArgs<T> ia;
        ia.I = I;
        ia.amp = amp;
        for (int d = 0; d < 3; d++) ia.S[d] = tab<double>(c, c->off_S[d]);
        // the plain amplitude carries the 1/V of the per-atom factors only through scale2
        ia.scale2 = c->scale2;
        ia.nx = c->nx;
        ia.ny = c->ny;
        ia.nz = c->nz;
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        intensity_kernel<T><<<blocks, 256, 0, st>>>(ia);
        return tstop(c, QPD_K_INTENSITY, st, t0);
    }

    // float64 planes -> packed inputs, cells [g0, g0 + cnt); planes point at cell g0
    static int pack(qpd_ctx* c, int64_t g0, int64_t cnt, const double* const* ost, const double* const* uu,
                    const double* const* oph, const double* region, void* P, void* U, int8_t* phase, void* weight,
                    void* wdense, uint32_t* flags, cudaStream_t st) {
        PackArgs<T> a;
        std::memset(&a, 0, sizeof a);
        a.cnt = cnt;
        a.g0 = g0;
        a.n = c->n;
        a.nStruc = c->nStruc;
        a.nPhase = c->nPhase;
        for (int k = 0; k < c->nStruc; k++) a.ost[k] = ost[k];
        for (int k = 0; k < 3; k++) a.uu[k] = uu[k];
        for (int p = 0; p < c->nPhase; p++) a.oph[p] = oph[p];
        a.region = region;
        a.P = static_cast<T*>(P);
        a.U = static_cast<T*>(U);
        a.phase = reinterpret_cast<signed char*>(phase);
        a.weight = static_cast<T*>(weight);
        a.wdense = static_cast<T*>(wdense);
        a.flags = flags;
        if (cnt <= 0) return QPD_OK;
        cudaEvent_t t0;
        QPD_TRY(tstart(c, st, &t0));
        pack_kernel<T><<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(a);
        return tstop(c, QPD_K_PACK, st, t0);
    }

    static int run_host(qpd_ctx* c, const double* oPhase, const double* oStruc, const double* u, const double* region,
                        double* I) {
        const int64_t n = c->n;
        const int NS = c->nStruc, NP = c->nPhase;
        // packed inputs (P, U, weight, phase) + intensity on the device
        const size_t pk = sizeof(T) * 7 * n + n;
        QPD_TRY(dev_reserve(c, c->packed, pk, "packed inputs"));
        QPD_TRY(dev_reserve(c, c->Idev, sizeof(double) * n, "intensity"));
        unsigned char* pb = static_cast<unsigned char*>(c->packed.p);
        T* P = reinterpret_cast<T*>(pb);
        T* U = P + 3 * n;
        T* W = U + 3 * n;
        int8_t* ph = reinterpret_cast<int8_t*>(W + n);
        cudaStream_t st = c->stream;
        if (!c->workers) {
            int nt = (int)std::min<unsigned>(16u, std::max(1u, std::thread::hardware_concurrency()));
            if (const char* e = std::getenv("QPOP_B200_HOST_THREADS")) nt = std::max(1, std::atoi(e));
            c->workers.reset(new qpd::Workers(nt - 1));  // the calling thread is the last worker
        }
        for (auto& e : c->ring_ev)
            if (!e) QPD_CU(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        const int64_t C = std::min<int64_t>(n, (int64_t)1 << 21);  // cells per chunk
        constexpr int NSLOT = 3;
        // Chunks take one of two routes that run at the same time: the host workers pack a chunk
        // (fewer bytes on the link, host memory bandwidth spent) or it crosses the link as float64
        // and pack_kernel packs it on the device.  The split balances itself: a chunk goes the device
        // way whenever no chunk waits on the copy engine, so the link never idles while
        // the host packs, and a slow host packs fewer chunks (QPOP_B200_ROUTE_DEPTH sets that queue
        // depth, default 1).  QPOP_B200_HOST_SHARE fixes the share
        // of host-packed chunks instead (0: all device, 1: all host).
        double share = -1.0;
        if (const char* e = std::getenv("QPOP_B200_HOST_SHARE")) share = std::min(1.0, std::max(0.0, std::atof(e)));
        int depth = 1;  // device route while fewer than `depth` chunks wait on the copy engine
        if (const char* e = std::getenv("QPOP_B200_ROUTE_DEPTH")) depth = std::max(1, std::atoi(e));
        const int NPL = NS + 3 + NP + (region ? 1 : 0);
        constexpr int NSTAGE = 2;  // device-route staging slots
        if (share < 1.0) QPD_TRY(dev_reserve(c, c->stage, sizeof(double) * NPL * C * NSTAGE, "float64 staging"));
        for (auto& e : c->chunk_ev)
            if (!e) QPD_CU(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        QPD_TRY(dev_reserve(c, c->flags, 256, "flags"));
        uint32_t* dflags = static_cast<uint32_t*>(c->flags.p);
        double* sg = static_cast<double*>(c->stage.p);

        // one pass over the host arrays: host chunk i is packed into ring slot i % 3 on the workers
        // while the copies of the previous chunks run; returns the OR of the pack flags
        auto pass = [&](bool dense, T* WD, uint32_t* flags_out) -> int {
            QPD_CU(c, cudaMemsetAsync(dflags, 0, sizeof(uint32_t), st));
            const size_t slot = (qpd::HostChunk<T>::bytes(C, NP, dense) + 255) & ~size_t(255);
            if (c->hring_bytes < NSLOT * slot) {
                for (int s = 0; s < NSLOT; s++)
                    if (c->ring_busy[s]) QPD_CU(c, cudaEventSynchronize(c->ring_ev[s]));
                if (c->hring) QPD_CU(c, cudaFreeHost(c->hring));
                c->hring = nullptr;
                c->hring_bytes = 0;
                QPD_CU(c, cudaHostAlloc(&c->hring, NSLOT * slot, cudaHostAllocDefault));
                c->hring_bytes = NSLOT * slot;
                for (bool& b : c->ring_busy) b = false;
            }
            uint32_t flags = 0;
            int64_t hosted = 0, staged = 0;
            // completion events of the chunks in flight, oldest first (a ring of kChunkEv)
            int64_t ev_head = 0, ev_tail = 0;
            auto pending = [&]() {
                while (ev_head < ev_tail && cudaEventQuery(c->chunk_ev[ev_head % qpd_ctx::kChunkEv]) == cudaSuccess) ev_head++;
                return ev_tail - ev_head;
            };
            auto record = [&]() -> int {
                if (ev_tail - ev_head == qpd_ctx::kChunkEv) {  // ring full: wait for the oldest
                    QPD_CU(c, cudaEventSynchronize(c->chunk_ev[ev_head % qpd_ctx::kChunkEv]));
                    ev_head++;
                }
                QPD_CU(c, cudaEventRecord(c->chunk_ev[ev_tail % qpd_ctx::kChunkEv], st));
                ev_tail++;
                return QPD_OK;
            };
            for (int64_t g0 = 0, i = 0; g0 < n; g0 += C, i++) {
                const int64_t cnt = std::min(C, n - g0);
                const bool device_route = share >= 0.0 ? (int64_t)((i + 1) * share) == (int64_t)(i * share)
                                                        : pending() < depth;
                if (device_route) {
                    const double* ost[3] = {nullptr, nullptr, nullptr};
                    const double* uu[3];
                    const double* oph[kMaxPhases];
                    double* slot = sg + (size_t)(staged++ % NSTAGE) * NPL * C;
                    int pl = 0;
                    auto put = [&](const double* src, const double** dst) -> int {
                        double* d = slot + (size_t)(pl++) * C;
                        QPD_CU(c, cudaMemcpyAsync(d, src + g0, sizeof(double) * cnt, cudaMemcpyHostToDevice, st));
                        *dst = d;
                        return QPD_OK;
                    };
                    for (int k = 0; k < NS; k++) QPD_TRY(put(oStruc + (int64_t)k * n, &ost[k]));
                    for (int k = 0; k < 3; k++) QPD_TRY(put(u + (int64_t)k * n, &uu[k]));
                    for (int p = 0; p < NP; p++) QPD_TRY(put(oPhase + (int64_t)p * n, &oph[p]));
                    const double* rg = nullptr;
                    if (region) QPD_TRY(put(region, &rg));
                    QPD_TRY(pack(c, g0, cnt, ost, uu, oph, rg, P, U, ph, W, dense ? WD : nullptr, dflags, st));
                    QPD_TRY(record());  // the staging slot is reused two device chunks later, after this pack in stream order
                    continue;
                }
                const int s = (int)(hosted++ % NSLOT);
                if (c->ring_busy[s]) QPD_CU(c, cudaEventSynchronize(c->ring_ev[s]));
                const qpd::HostChunk<T> h = qpd::HostChunk<T>::at(static_cast<unsigned char*>(c->hring) + s * slot, C);
                const int parts = (int)std::max<int64_t>(1, std::min<int64_t>(c->workers->size() + 1, cnt >> 16));
                std::atomic<uint32_t> fl{0};
                c->workers->parallel(parts, [&](int t) {
                    const int64_t i0 = cnt * t / parts, i1 = cnt * (t + 1) / parts;
                    fl.fetch_or(qpd::host_pack<T>(h, n, g0, i0, i1, NS, NP, oPhase, oStruc, u, region, dense));
                });
                const uint32_t f = fl.load();
                flags |= f;
                for (int k = 0; k < 3; k++) {
                    QPD_CU(c, cudaMemcpyAsync(P + k * n + g0, h.P + k * C, sizeof(T) * cnt, cudaMemcpyHostToDevice, st));
                    QPD_CU(c, cudaMemcpyAsync(U + k * n + g0, h.U + k * C, sizeof(T) * cnt, cudaMemcpyHostToDevice, st));
                }
                if (dense) {
                    for (int p = 0; p < NP; p++)
                        QPD_CU(c, cudaMemcpyAsync(WD + p * n + g0, h.WD + p * C, sizeof(T) * cnt, cudaMemcpyHostToDevice, st));
                } else {
                    QPD_CU(c, cudaMemcpyAsync(ph + g0, h.ph, cnt, cudaMemcpyHostToDevice, st));
                    if (f & 2u) {
                        QPD_CU(c, cudaMemcpyAsync(W + g0, h.W, sizeof(T) * cnt, cudaMemcpyHostToDevice, st));
                    } else {  // weights 0 or 1 only: rebuild them from the phase index on the device
                        fill_weight_kernel<T><<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(ph + g0, W + g0, cnt);
                        QPD_CU(c, cudaGetLastError());
                    }
                }
                QPD_CU(c, cudaEventRecord(c->ring_ev[s], st));
                c->ring_busy[s] = true;
                QPD_TRY(record());
            }
            uint32_t df = 0;
            QPD_CU(c, cudaMemcpyAsync(&df, dflags, sizeof df, cudaMemcpyDeviceToHost, st));
            QPD_CU(c, cudaStreamSynchronize(st));
            *flags_out = flags | df;
            return QPD_OK;
        };

        uint32_t f = 0;
        QPD_TRY(pass(false, nullptr, &f));
        Inputs<T> in;
        if (f & 1u) {
            QPD_TRY(dev_reserve(c, c->dense, sizeof(T) * NP * n, "dense phase weights"));
            uint32_t f2 = 0;
            QPD_TRY(pass(true, static_cast<T*>(c->dense.p), &f2));
            in = inputs(c, P, U, nullptr, nullptr, c->dense.p);
        } else {
            in = inputs(c, P, U, ph, (f & 2u) ? W : nullptr, nullptr);
        }
        double* Id = static_cast<double*>(c->Idev.p);
        QPD_TRY(run_device(c, in, Id, st));
        QPD_CU(c, cudaMemcpyAsync(I, Id, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        QPD_CU(c, cudaStreamSynchronize(st));
        for (bool& b : c->ring_busy) b = false;
        return check_status(c);
    }
};

int upload_twiddles(qpd_ctx* c, int d, int64_t N) {
    std::vector<double2> w(N);
    for (int64_t m = 0; m < N; m++) {
        const double a = 2.0 * M_PI * (double)m / (double)N;
        w[m] = make_double2(std::cos(a), -std::sin(a));
    }
    if (c->precision == QPD_FP64) {
        QPD_TRY(dev_reserve(c, c->tw[d], sizeof(double2) * N, "twiddles"));
        QPD_CU(c, cudaMemcpy(c->tw[d].p, w.data(), sizeof(double2) * N, cudaMemcpyHostToDevice));
    } else {
        std::vector<float2> f(N);
        for (int64_t m = 0; m < N; m++) f[m] = make_float2((float)w[m].x, (float)w[m].y);
        QPD_TRY(dev_reserve(c, c->tw[d], sizeof(float2) * N, "twiddles"));
        QPD_CU(c, cudaMemcpy(c->tw[d].p, f.data(), sizeof(float2) * N, cudaMemcpyHostToDevice));
    }
    return QPD_OK;
}

// The butterflies' unit roots, once per device (constant memory is per device and module).
int roots_init(qpd_ctx* c) {
    static std::mutex mu;
    static std::vector<char> done;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)done.size() <= c->device) done.resize(c->device + 1, 0);
    if (done[c->device]) return QPD_OK;
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
    QPD_CU(c, cudaMemcpyToSymbol(c_roots_d, rd, sizeof rd));
    QPD_CU(c, cudaMemcpyToSymbol(c_roots_f, rf, sizeof rf));
    done[c->device] = 1;
    return QPD_OK;
}

// Read and clear the device status word; a recorded timeout becomes QPD_ERR_CUDA.
int check_status(qpd_ctx* c) {
    int v = 0;
    QPD_CU(c, cudaMemcpy(&v, c->status.p, sizeof v, cudaMemcpyDeviceToHost));
    if (v == 0) return QPD_OK;
    QPD_CU(c, cudaMemset(c->status.p, 0, sizeof v));
    return fail(c, QPD_ERR_CUDA, "device status %d: %s", v,
                v == QPD_DEVERR_ALIGN ? "shared memory was not aligned for TMA, the kernel stopped before loading"
                                      : "a kernel gave up waiting for its tile loads");
}

int use_device(qpd_ctx* c) {
    QPD_CU(c, cudaSetDevice(c->device));
    return QPD_OK;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Tensor map over a field array viewed as (2 nz reals, ny, nfields * nx), box (bz, by, bx).
int field_map(qpd_ctx* c, CUtensorMap* m, void* base, bool fp64, int64_t nz, int64_t ny, int64_t nfx, int bz, int by,
              int bx) {
    auto fn = encode_fn();
    if (!fn) return fail(c, QPD_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t esz = fp64 ? 8 : 4;
    cuuint64_t dims[3] = {(cuuint64_t)(2 * nz), (cuuint64_t)ny, (cuuint64_t)nfx};
    cuuint64_t strides[2] = {(cuuint64_t)(2 * nz) * esz, (cuuint64_t)(2 * nz * ny) * esz};
    cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)by, (cuuint32_t)bx};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = fn(m, fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides,
                    box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(c, QPD_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return QPD_OK;
}

}  // namespace

namespace {

template <typename T>
int pack_fields_t(qpd_ctx* c, const qpd_fields* in, void* P, void* U, int8_t* phase, void* weight, void* wdense,
                  uint32_t* fd, cudaStream_t st) {
    FieldsArgs<T> a;
    std::memset(&a, 0, sizeof a);
    for (int k = 0; k < c->nStruc; k++) a.P[k] = in->P[k];
    if (in->u[0])
        for (int k = 0; k < 3; k++) a.u[k] = in->u[k];
    a.phase = in->phase;
    a.region = in->region;
    a.mat = reinterpret_cast<const signed char*>(in->material);
    a.nx = c->nx;
    a.ny = c->ny;
    a.nz = c->nz;
    a.z0 = in->z0;
    a.nStruc = c->nStruc;
    a.nPhase = c->nPhase;
    a.nMat = in->n_material;
    a.dz = in->ramp_dz;
    a.p_scale = in->p_scale;
    a.u_scale = in->u_scale;
    for (int m = 0; m < in->n_material; m++) {
        a.dc[m] = in->dc[m];
        a.phase_of[m] = (signed char)in->phase_of[m];
    }
    a.Pout = static_cast<T*>(P);
    a.Uout = static_cast<T*>(U);
    a.phase_idx = reinterpret_cast<signed char*>(phase);
    a.weight = static_cast<T*>(weight);
    a.wdense = static_cast<T*>(wdense);
    a.flags = fd;
    const int planes = c->nStruc + (in->u[0] ? 3 : 0) + (in->phase ? c->nPhase : 0) + (in->region ? 1 : 0);
    const size_t smem = fields_smem_bytes(planes);
    QPD_CU(c, cudaFuncSetAttribute(fields_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaEvent_t t0;
    QPD_TRY(tstart(c, st, &t0));
    dim3 grid((unsigned)((c->nx + kFT - 1) / kFT), (unsigned)c->ny);
    fields_kernel<T><<<grid, dim3(kFT, kFRows), smem, st>>>(a);
    return tstop(c, QPD_K_PACK, st, t0);
}

}  // namespace

extern "C" {

int qpd_create(int device, uint64_t hbm_budget_bytes, qpd_ctx** out) {
    if (!out) return fail(nullptr, QPD_ERR_ARG, "qpd_create: out is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return fail(nullptr, QPD_ERR_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    if (device < 0 || device >= count) return fail(nullptr, QPD_ERR_ARG, "device %d outside 0..%d", device, count - 1);
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(nullptr, QPD_ERR_CUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
    qpd_ctx* c = new qpd_ctx();
    c->device = device;
    c->budget = hbm_budget_bytes;
    const char* gen = std::getenv("QPOP_B200_GENERIC");
    c->fast = !(gen && gen[0] == '1');
    const char* notma = std::getenv("QPOP_B200_NO_TMA");
    c->tma = !(notma && notma[0] == '1');
    if (const char* k = std::getenv("QPOP_B200_ZCFG")) c->knob_z = std::atoi(k);
    if (const char* k = std::getenv("QPOP_B200_NBUF")) c->knob_nbuf = std::atoi(k) == 3 ? 3 : 2;
    if (const char* k = std::getenv("QPOP_B200_ZPFA")) c->knob_zpfa = std::atoi(k);
    if (const char* k = std::getenv("QPOP_B200_N4000")) c->knob_n4000 = std::atoi(k);
    if (const char* k = std::getenv("QPOP_B200_OOP")) c->knob_oop = std::atoi(k);
    if (const char* k = std::getenv("QPOP_B200_YFAST")) c->knob_yfast = std::atoi(k);
    if (const char* k = std::getenv("QPOP_B200_N4K")) c->knob_n4k = std::atoi(k);
    if (const char* k = std::getenv("QPOP_B200_ADJ_TMA")) c->knob_adj_tma = std::atoi(k);
    if (const char* k = std::getenv("QPOP_B200_ZREGIN")) c->knob_zregin = std::atoi(k);
    if (const char* k = std::getenv("QPOP_B200_BULK_NT")) c->knob_bulk_nt = std::atoi(k) == 512 ? 512 : 256;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return fail(nullptr, QPD_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
    int r = roots_init(c);
    if (r == QPD_OK) r = dev_reserve(c, c->status, 256, "status word");
    if (r == QPD_OK && cudaMemset(c->status.p, 0, 256) != cudaSuccess) r = fail(c, QPD_ERR_CUDA, "cudaMemset failed");
    if (r != QPD_OK) {
        g_create_error = c->err;
        cudaStreamDestroy(c->stream);
        delete c;
        return r;
    }
    *out = c;
    return QPD_OK;
}

int qpd_destroy(qpd_ctx* c) {
    if (!c) return QPD_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (DevMem* m : {&c->tw[0], &c->tw[1], &c->tw[2], &c->tables, &c->fields, &c->adjw, &c->packed, &c->dense,
                      &c->stage, &c->Idev, &c->flags, &c->status})
        dev_free(c, *m);
    c->workers.reset();
    if (c->hring) cudaFreeHost(c->hring);
    for (cudaEvent_t e : c->ring_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : c->chunk_ev)
        if (e) cudaEventDestroy(e);
    for (auto& r : c->recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : c->pool) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return QPD_OK;
}

const char* qpd_last_error(const qpd_ctx* c) { return c ? c->err.c_str() : g_create_error.c_str(); }

}  // extern "C"

// For qpd_noalloc.cu, which has no context: its failures read back through qpd_last_error(NULL).
void qpd_internal_set_error(const char* msg) { g_create_error = msg; }

extern "C" {

int qpd_axis_radices(int64_t N, int32_t* radices, int32_t cap) {
    if (N < 1) return QPD_ERR_ARG;
    std::vector<int> r = factorise(N);
    if (!radices || cap < (int)r.size()) return (int)r.size();
    for (size_t i = 0; i < r.size(); i++) radices[i] = r[i];
    return (int)r.size();
}

int qpd_plan(qpd_ctx* c, const qpd_grid* g, int32_t nPhase, int32_t nStruc, int32_t precision, int32_t schedule) {
    if (!c || !g) return fail(c, QPD_ERR_ARG, "qpd_plan: NULL argument");
    if (g->nx < 1 || g->ny < 1 || g->nz < 1) return fail(c, QPD_ERR_ARG, "grid %lld x %lld x %lld is empty",
                                                         (long long)g->nx, (long long)g->ny, (long long)g->nz);
    if (!(g->dx > 0 && g->dy > 0 && g->dz > 0)) return fail(c, QPD_ERR_ARG, "grid spacings must be positive");
    if (nPhase < 1 || nPhase > kMaxPhases) return fail(c, QPD_ERR_ARG, "nPhase = %d outside 1..%d", nPhase, kMaxPhases);
    if (nStruc < 0 || nStruc > 3) return fail(c, QPD_ERR_ARG, "nStruc = %d outside 0..3", nStruc);
    if (precision != QPD_FP32 && precision != QPD_FP64) return fail(c, QPD_ERR_ARG, "unknown precision %d", precision);
    if (schedule != QPD_SCHED_FUSED && schedule != QPD_SCHED_PLAIN) return fail(c, QPD_ERR_ARG, "unknown schedule %d", schedule);
    if (g->nx > 16384 || g->ny > 16384 || g->nz > 4096)
        return fail(c, QPD_ERR_UNSUPPORTED, "axis lengths above 16384 (x, y) or 4096 (z) are not supported");
    const int64_t n = g->nx * g->ny * g->nz;
    if (n > ((int64_t)1 << 40)) return fail(c, QPD_ERR_UNSUPPORTED, "grid of %lld cells is too large", (long long)n);
    QPD_TRY(use_device(c));
    c->planned = false;
    c->have_crystal = false;
    c->nx = g->nx;
    c->ny = g->ny;
    c->nz = g->nz;
    c->n = n;
    c->h[0] = g->dx;
    c->h[1] = g->dy;
    c->h[2] = g->dz;
    c->nPhase = nPhase;
    c->nStruc = nStruc;
    c->precision = precision;
    c->schedule = schedule;
    const int64_t N[3] = {g->nx, g->ny, g->nz};
    for (int d = 0; d < 3; d++) {
        c->radix[d] = N[d] > 1 ? factorise(N[d]) : std::vector<int>();
        if ((int)c->radix[d].size() > kMaxStages) return fail(c, QPD_ERR_UNSUPPORTED, "axis %d has too many stages", d);
        QPD_TRY(upload_twiddles(c, d, N[d]));
    }
    c->planned = true;
    return QPD_OK;
}

int qpd_set_crystal(qpd_ctx* c, const qpd_crystal* k) {
    if (!c || !k) return fail(c, QPD_ERR_ARG, "qpd_set_crystal: NULL argument");
    if (!c->planned) return fail(c, QPD_ERR_STATE, "qpd_set_crystal before qpd_plan");
    if (k->nAtom < 1) return fail(c, QPD_ERR_ARG, "nAtom = %d", k->nAtom);
    if (k->nPhase != c->nPhase || k->nStruc != c->nStruc)
        return fail(c, QPD_ERR_ARG, "crystal has nPhase %d, nStruc %d; the plan %d, %d", k->nPhase, k->nStruc, c->nPhase,
                    c->nStruc);
    if (!k->R || !k->f_re || !k->f_im || (k->nStruc > 0 && !k->su)) return fail(c, QPD_ERR_ARG, "crystal arrays are NULL");
    if (!(k->V != 0.0 && std::isfinite(k->V))) return fail(c, QPD_ERR_ARG, "cell volume V = %g", k->V);
    QPD_TRY(use_device(c));
    c->have_crystal = false;
    int r = c->precision == QPD_FP64 ? Impl<double>::set_crystal(c, k) : Impl<float>::set_crystal(c, k);
    if (r == QPD_OK) c->have_crystal = true;
    return r;
}

int qpd_run_host(qpd_ctx* c, const double* oPhase, const double* oStruc, const double* u, const double* region,
                 double* I) {
    if (!c) return fail(c, QPD_ERR_ARG, "qpd_run_host: ctx is NULL");
    if (!c->planned || !c->have_crystal) return fail(c, QPD_ERR_STATE, "qpd_run_host needs qpd_plan and qpd_set_crystal");
    if (!oPhase || !u || !I || (c->nStruc > 0 && !oStruc)) return fail(c, QPD_ERR_ARG, "qpd_run_host: NULL array");
    QPD_TRY(use_device(c));
    return c->precision == QPD_FP64 ? Impl<double>::run_host(c, oPhase, oStruc, u, region, I)
                                    : Impl<float>::run_host(c, oPhase, oStruc, u, region, I);
}

int qpd_pack_device(qpd_ctx* c, const double* oPhase, const double* oStruc, const double* u, const double* region,
                    void* P, void* U, int8_t* phase, void* weight, void* wdense, int32_t dense, uint32_t* flags,
                    void* stream) {
    if (!c) return fail(c, QPD_ERR_ARG, "qpd_pack_device: ctx is NULL");
    if (!c->planned) return fail(c, QPD_ERR_STATE, "qpd_pack_device before qpd_plan");
    if (!oPhase || !u || !P || !U || (c->nStruc > 0 && !oStruc)) return fail(c, QPD_ERR_ARG, "qpd_pack_device: NULL array");
    if (dense ? !wdense : (!phase || !weight)) return fail(c, QPD_ERR_ARG, "qpd_pack_device: NULL weight output");
    QPD_TRY(use_device(c));
    QPD_TRY(dev_reserve(c, c->flags, 256, "flags"));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = c->n;
    const double* ost[3] = {nullptr, nullptr, nullptr};
    const double* uu[3];
    const double* oph[kMaxPhases];
    for (int k = 0; k < c->nStruc; k++) ost[k] = oStruc + k * n;
    for (int k = 0; k < 3; k++) uu[k] = u + k * n;
    for (int p = 0; p < c->nPhase; p++) oph[p] = oPhase + p * n;
    uint32_t* fd = static_cast<uint32_t*>(c->flags.p);
    QPD_CU(c, cudaMemsetAsync(fd, 0, sizeof(uint32_t), st));
    int r = c->precision == QPD_FP64
                ? Impl<double>::pack(c, 0, n, ost, uu, oph, region, P, U, phase, weight, dense ? wdense : nullptr, fd, st)
                : Impl<float>::pack(c, 0, n, ost, uu, oph, region, P, U, phase, weight, dense ? wdense : nullptr, fd, st);
    QPD_TRY(r);
    uint32_t f = 0;
    QPD_CU(c, cudaMemcpyAsync(&f, fd, sizeof f, cudaMemcpyDeviceToHost, st));
    QPD_CU(c, cudaStreamSynchronize(st));
    if (flags) *flags = f;
    return QPD_OK;
}

int qpd_pack_fields(qpd_ctx* c, const qpd_fields* in, void* P, void* U, int8_t* phase, void* weight, void* wdense,
                    int32_t dense, uint32_t* flags, void* stream) {
    if (!c) return fail(c, QPD_ERR_ARG, "qpd_pack_fields: ctx is NULL");
    if (!c->planned) return fail(c, QPD_ERR_STATE, "qpd_pack_fields before qpd_plan");
    if (!in || !in->material || !in->dc || !in->phase_of) return fail(c, QPD_ERR_ARG, "qpd_pack_fields: NULL fields or tables");
    for (int k = 0; k < c->nStruc; k++)
        if (!in->P[k]) return fail(c, QPD_ERR_ARG, "qpd_pack_fields: P[%d] is NULL", k);
    if ((in->u[0] != nullptr) != (in->u[1] != nullptr) || (in->u[0] != nullptr) != (in->u[2] != nullptr))
        return fail(c, QPD_ERR_ARG, "qpd_pack_fields: give all three displacement components or none");
    if (!P || !U || (dense ? !wdense : (!phase || !weight))) return fail(c, QPD_ERR_ARG, "qpd_pack_fields: NULL output");
    if (in->n_material < 1 || in->n_material > kMaxMaterials)
        return fail(c, QPD_ERR_ARG, "qpd_pack_fields: n_material %d outside 1..%d", in->n_material, kMaxMaterials);
    for (int m = 0; m < in->n_material; m++)
        if (in->phase_of[m] < -1 || in->phase_of[m] >= c->nPhase)
            return fail(c, QPD_ERR_ARG, "qpd_pack_fields: phase_of[%d] = %d outside -1..%d", m, in->phase_of[m], c->nPhase - 1);
    if (c->ny > 65535) return fail(c, QPD_ERR_UNSUPPORTED, "qpd_pack_fields: ny %lld > 65535", (long long)c->ny);
    if (in->z0 < 0 || in->z0 + c->nz > in->nz_full)
        return fail(c, QPD_ERR_ARG, "qpd_pack_fields: crop z0 %lld + nz %lld outside the %lld-layer stack",
                    (long long)in->z0, (long long)c->nz, (long long)in->nz_full);
    QPD_TRY(use_device(c));
    QPD_TRY(dev_reserve(c, c->flags, 256, "flags"));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint32_t* fd = static_cast<uint32_t*>(c->flags.p);
    QPD_CU(c, cudaMemsetAsync(fd, 0, sizeof(uint32_t), st));
    int r = c->precision == QPD_FP64 ? pack_fields_t<double>(c, in, P, U, phase, weight, dense ? wdense : nullptr, fd, st)
                                     : pack_fields_t<float>(c, in, P, U, phase, weight, dense ? wdense : nullptr, fd, st);
    QPD_TRY(r);
    uint32_t f = 0;
    QPD_CU(c, cudaMemcpyAsync(&f, fd, sizeof f, cudaMemcpyDeviceToHost, st));
    QPD_CU(c, cudaStreamSynchronize(st));
    if (f & kFlagBadMaterial) return fail(c, QPD_ERR_ARG, "qpd_pack_fields: a material index lies outside the dc / phase_of tables");
    if (flags) *flags = f;
    return QPD_OK;
}

int qpd_run_device(qpd_ctx* c, const void* P, const void* U, const int8_t* phase, const void* weight,
                   const void* wdense, double* I_dev, void* stream) {
    if (!c) return fail(c, QPD_ERR_ARG, "qpd_run_device: ctx is NULL");
    if (!c->planned || !c->have_crystal) return fail(c, QPD_ERR_STATE, "qpd_run_device needs qpd_plan and qpd_set_crystal");
    if (!P || !U || !I_dev || (!wdense && !phase)) return fail(c, QPD_ERR_ARG, "qpd_run_device: NULL array");
    QPD_TRY(use_device(c));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (c->precision == QPD_FP64) {
        Inputs<double> in = Impl<double>::inputs(c, P, U, phase, weight, wdense);
        return Impl<double>::run_device(c, in, I_dev, st);
    }
    Inputs<float> in = Impl<float>::inputs(c, P, U, phase, weight, wdense);
    return Impl<float>::run_device(c, in, I_dev, st);
}

int qpd_adjoint_device(qpd_ctx* c, const void* P, const void* U, const int8_t* phase, const void* weight,
                       const void* wdense, const double* dI, void* dP, void* dU, void* stream) {
    if (!c) return fail(c, QPD_ERR_ARG, "qpd_adjoint_device: ctx is NULL");
    if (!c->planned || !c->have_crystal) return fail(c, QPD_ERR_STATE, "qpd_adjoint_device needs qpd_plan and qpd_set_crystal");
    if (!P || !U || !dI || !dP || !dU || (!wdense && !phase)) return fail(c, QPD_ERR_ARG, "qpd_adjoint_device: NULL array");
    if (c->sched_used != QPD_SCHED_FUSED)
        return fail(c, QPD_ERR_UNSUPPORTED, "qpd_adjoint_device: the adjoint runs on the fused schedule only");
    QPD_TRY(use_device(c));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (c->precision == QPD_FP64) {
        Inputs<double> in = Impl<double>::inputs(c, P, U, phase, weight, wdense);
        return Impl<double>::adjoint(c, in, dI, static_cast<double*>(dP), static_cast<double*>(dU), st);
    }
    Inputs<float> in = Impl<float>::inputs(c, P, U, phase, weight, wdense);
    return Impl<float>::adjoint(c, in, dI, static_cast<float*>(dP), static_cast<float*>(dU), st);
}

int qpd_set_cta_tiles(qpd_ctx* c, int32_t tiles) {
    if (!c) return fail(c, QPD_ERR_ARG, "qpd_set_cta_tiles: ctx is NULL");
    if (tiles < 0) return fail(c, QPD_ERR_ARG, "qpd_set_cta_tiles: tiles = %d must be >= 0", (int)tiles);
    c->cta_tiles = tiles;
    return QPD_OK;
}

int qpd_enable_timing(qpd_ctx* c, int32_t on) {
    if (!c) return fail(c, QPD_ERR_ARG, "qpd_enable_timing: ctx is NULL");
    c->timing = on != 0;
    return QPD_OK;
}

int qpd_stage_times(qpd_ctx* c, double* ms, uint64_t* counts, int32_t cap) {
    if (!c || !ms || !counts || cap < QPD_K_COUNT) return fail(c, QPD_ERR_ARG, "qpd_stage_times: bad arguments");
    QPD_TRY(use_device(c));
    for (int k = 0; k < QPD_K_COUNT; k++) {
        ms[k] = 0.0;
        counts[k] = 0;
    }
    int rc = QPD_OK;
    for (auto& r : c->recs) {
        float t = 0.0f;
        cudaError_t e = cudaEventSynchronize(r.b);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, r.a, r.b);
        if (e != cudaSuccess && rc == QPD_OK) rc = fail(c, QPD_ERR_CUDA, "event timing: %s", cudaGetErrorString(e));
        ms[r.kind] += t;
        counts[r.kind]++;
        c->pool.push_back(r.a);
        c->pool.push_back(r.b);
    }
    c->recs.clear();
    return rc;
}

int qpd_device_status(qpd_ctx* c) {
    if (!c) return fail(c, QPD_ERR_ARG, "qpd_device_status: ctx is NULL");
    QPD_TRY(use_device(c));
    return check_status(c);
}

int qpd_probe_wait_timeout(qpd_ctx* c, int64_t polls) {
    if (!c) return fail(c, QPD_ERR_ARG, "qpd_probe_wait_timeout: ctx is NULL");
    if (polls < 1 || polls > kWaitLimit) return fail(c, QPD_ERR_ARG, "polls outside 1..2^24");
    QPD_TRY(use_device(c));
    QPD_CU(c, launch_wait_probe(static_cast<int*>(c->status.p), (long long)polls, c->stream));
    QPD_CU(c, cudaStreamSynchronize(c->stream));
    return QPD_OK;
}

uint64_t qpd_workspace_bytes(const qpd_ctx* c) { return c ? c->held : 0; }
uint64_t qpd_launch_count(const qpd_ctx* c) { return c ? c->launches : 0; }

}  // extern "C"
