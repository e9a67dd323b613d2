/*
 * qpopdiff.h: C ABI of libqpopdiff.so, the B200 (sm_100a) kinematic-diffraction hot path.
 *
 * The library computes, for one snapshot and one reciprocal-lattice point G,
 *
 *     u_ap(r) = u(r) + su[:, :, p, a] . P(r)
 *     fE_a(r) = sum_p w_p(r) f_pa exp(-i qC . u_ap(r)),   fU_a(r) = fE_a(r) u_ap(r)
 *     Amp(k)  = sum_a exp(-i (k + G) . R_a) / V [FFT(fE_a)/n - i k . FFT(fU_a)/n]
 *     I       = fftshift(max(|S(k) Amp(k)|^2, 1e-50)),  S(k) = prod_d sinc(k_d h_d / 2)
 *
 * the body of the reference's standard-build diffraction() (src/python/diffraction.py:62-113)
 * and of the per-cell GPU work of its multi-GPU program (src/heffte/qpop_diffraction_mgpu.cu:166-186).
 *
 * Conventions: every entry point returns QPD_OK (0) or a negative QPD_ERR_* code and never
 * aborts or exits; qpd_last_error() then describes the failure (this replaces fail() /
 * MPI_Abort, src/heffte/util.hpp:12-16).  The caller owns every input and output buffer; the
 * context owns its device workspace.  A context belongs to one host thread at a time.
 * Fields are flat, component-major, each component (nx, ny, nz) in C order (z fastest).
 */
#ifndef QPOPDIFF_H_
#define QPOPDIFF_H_

#include <stddef.h>
#include <stdint.h>

#if defined(QPD_BUILD) && defined(__GNUC__)
#define QPD_API __attribute__((visibility("default")))
#else
#define QPD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define QPD_OK 0
#define QPD_ERR_ARG (-1)         /* invalid argument or shape */
#define QPD_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define QPD_ERR_NOMEM (-3)       /* the workspace does not fit the device or the context's budget */
#define QPD_ERR_UNSUPPORTED (-4) /* valid input outside what the kernels handle (e.g. nz > 4096) */
#define QPD_ERR_STATE (-5)       /* call out of order (no plan, no crystal) */

#define QPD_FP32 0 /* float32 fields, float64 phase reduction, float64 intensity */
#define QPD_FP64 1 /* float64 throughout */

#define QPD_SCHED_FUSED 0 /* 3 kernels per volume: source+z, y, x+epilogue */
#define QPD_SCHED_PLAIN 1 /* the reference's loop: per atom and component, source, 3-D FFT, accumulate */

typedef struct qpd_ctx qpd_ctx;

/* Grid of the (cropped) snapshot: the SizeContext fields nx, ny, nz, dx, dy, dz (nm) that
 * diffraction() reads (src/python/diffraction.py:75-86). */
typedef struct qpd_grid {
    int64_t nx, ny, nz;
    double dx, dy, dz;
} qpd_grid;

/* Crystal and reflection: G, qC from reciprocal_centre (src/python/diffraction.py:36-48),
 * V = det(aC), R = xAtom @ aC (nAtom x 3, nm), f = fAtom (nPhase x nAtom, complex as two
 * real arrays), su = stack(su1, su2, su3) (3 x nStruc x nPhase x nAtom, nm per C/m^2),
 * the same quantities qpop_diffraction_mgpu reads from _params.h5 (src/heffte/params.hpp:13-35). */
typedef struct qpd_crystal {
    int32_t nAtom, nPhase, nStruc;
    double G[3], qC[3], V;
    const double* R;
    const double* f_re;
    const double* f_im;
    const double* su;
} qpd_crystal;

/* Create a context on CUDA device `device`.  hbm_budget_bytes caps the device memory the
 * context may allocate (0: no cap).  Replaces the rank -> GPU binding of
 * src/heffte/qpop_diffraction_mgpu.cu:41-47. */
QPD_API int qpd_create(int device, uint64_t hbm_budget_bytes, qpd_ctx** out);

/* Release the context and all of its device memory. */
QPD_API int qpd_destroy(qpd_ctx* ctx);

/* Message of the last failure on ctx (or of the last failed qpd_create when ctx is NULL). */
QPD_API const char* qpd_last_error(const qpd_ctx* ctx);

/* Plan a grid: factorise each axis into FFT stages, build the twiddle tables.  nPhase and
 * nStruc fix the input layout (1 <= nPhase <= 8, 0 <= nStruc <= 3).  Replaces the HeFFTe
 * plan construction (src/heffte/qpop_diffraction_mgpu.cu:154-157). */
QPD_API int qpd_plan(qpd_ctx* ctx, const qpd_grid* grid, int32_t nPhase, int32_t nStruc, int32_t precision,
             int32_t schedule);

/* Set the crystal and reflection used by the following runs: groups the atoms, builds the
 * per-axis phase tables and allocates the workspace.  Replaces mgpuParams::read's constants
 * (src/heffte/params.hpp:66-108). */
QPD_API int qpd_set_crystal(qpd_ctx* ctx, const qpd_crystal* crystal);

/* The reference-facing call with host buffers, synchronous: oPhase (nPhase * n), oStruc
 * (nStruc * n, C/m^2), u (3 * n, nm, u_z including its reference ramp), region (n, or NULL
 * for 1), all float64 as diffraction() receives them (src/python/diffraction.py:62-74);
 * writes I (n float64, fftshifted, (nx, ny, nz) C order).  Host -> device copies, packing,
 * the transform and the device -> host copy all happen inside. */
QPD_API int qpd_run_host(qpd_ctx* ctx, const double* oPhase, const double* oStruc, const double* u, const double* region,
                 double* I);

/* Pack float64 fields already on the device (same layout as qpd_run_host's) into the kernel
 * inputs: P (3 * n) and U (3 * n) in the plan precision, and either the phase index and
 * weight (single mode: at most one phase per cell) or dense weights (nPhase * n, dense != 0).
 * *flags receives bit 0 (a cell has several phases: repack dense) and bit 1 (a weight differs
 * from 0 and 1: keep the weight array).  Replaces the scale / columns preparation of
 * src/heffte/qpop_diffraction_mgpu.cu:96,137 for data that is already on the GPU.
 * stream is a cudaStream_t (NULL: the legacy default stream); the call synchronises it. */
QPD_API int qpd_pack_device(qpd_ctx* ctx, const double* oPhase, const double* oStruc, const double* u, const double* region,
                    void* P, void* U, int8_t* phase, void* weight, void* wdense, int32_t dense, uint32_t* flags,
                    void* stream);

/* Q-POP-FerroDyn fields on the device, in their file order (nz, ny, nx) with x fastest, float32
 * as FerroDyn writes them, already cropped to the planned grid except for the material field. */
typedef struct qpd_fields {
    const float* P[3];         /* order-parameter components (nStruc of them), C/m^2 before p_scale */
    const float* u[3];         /* displacement components before u_scale (FerroDyn: metres), or all NULL */
    const float* phase;        /* nPhase planes of phase fractions, or NULL: one-hot from the material */
    const float* region;       /* scattering weight, or NULL: 1 */
    const int8_t* material;    /* (nz_full, ny, nx) material indices: the crop's columns, full stack */
    int64_t nz_full, z0;       /* layers in the material stack; the crop's first layer in it */
    int32_t n_material;        /* entries of dc and phase_of, 1 .. 64 */
    const double* dc;          /* host: c_m(T) / aC_z - 1 per material */
    const int32_t* phase_of;   /* host: phase index of each material, -1 if it does not scatter */
    double ramp_dz;            /* layer spacing of the u_z ramp, nm */
    double p_scale, u_scale;   /* 1 / OS0 and the metres -> nm factor (1e9) */
} qpd_fields;

/* Boundary-input preparation on the GPU: the packed kernel inputs (same outputs and flags as
 * qpd_pack_device) straight from FerroDyn fields.  Transposes to (x, y, z), scales P and u, sets
 * the phases one-hot over the scattering materials (or from the phase fractions), the weight
 * region = (material scatters) x region, and adds the u_z reference ramp
 * (cumsum_z dc[mat] - dc[mat] / 2) ramp_dz summed over the full material stack from layer 0 and
 * cropped at z0.  Replaces the host preparation of src/python/cli.py:174-217 and the `columns`
 * kernel of src/heffte/kernels.cuh:34-50; a material index outside the tables fails with
 * QPD_ERR_ARG.  stream is a cudaStream_t (NULL: the legacy default stream); the call
 * synchronises it. */
QPD_API int qpd_pack_fields(qpd_ctx* ctx, const qpd_fields* fields, void* P, void* U, int8_t* phase, void* weight,
                            void* wdense, int32_t dense, uint32_t* flags, void* stream);

/* The hot path on device-resident packed inputs, asynchronous on `stream` (a cudaStream_t;
 * NULL: the legacy default stream): P, U, weight, wdense in the plan precision (weight NULL: 1; wdense
 * non-NULL selects dense mode and phase/weight are ignored); I_dev receives n float64.
 * Replaces source / fft.forward / accumulate / intensity of
 * src/heffte/qpop_diffraction_mgpu.cu:169-186. */
QPD_API int qpd_run_device(qpd_ctx* ctx, const void* P, const void* U, const int8_t* phase, const void* weight,
                   const void* wdense, double* I_dev, void* stream);

/* No counterpart in the reference (differentiation through the model): the gradient of a scalar
 * loss L(I) with respect to the packed inputs.  dI holds dL/dI (n float64, the fftshifted
 * layout of I); writes dL/dP (3 * n; planes beyond nStruc are 0) and dL/dU (3 * n) in the plan
 * precision, for the same packed inputs as qpd_run_device (which need not have run: the forward is
 * recomputed pass by pass, nothing is kept between the calls).  Voxels at the 1e-50 floor pass no
 * gradient.  Fused schedule only (QPD_ERR_UNSUPPORTED otherwise); needs (1 + 2 G2) more complex
 * fields of workspace, G2 the atoms' distinct R_x.  Asynchronous on `stream` (NULL: the legacy
 * default stream). */
QPD_API int qpd_adjoint_device(qpd_ctx* ctx, const void* P, const void* U, const int8_t* phase, const void* weight,
                               const void* wdense, const double* dI, void* dP, void* dU, void* stream);

/* Wait for the device and report whether a kernel of this context gave up on a bounded wait
 * (a tile load that never completed): QPD_OK, or QPD_ERR_CUDA with the status cleared.
 * qpd_run_host checks this itself; callers of qpd_run_device call it after synchronising. */
QPD_API int qpd_device_status(qpd_ctx* ctx);

/* No counterpart in the reference (its failures abort through MPI_Abort, src/heffte/util.hpp:12-16).
 * Runs the bounded-wait failure path once, on the context's stream, and waits for it: a kernel arms a
 * shared-memory barrier for bytes that no copy ever delivers and gives up after `polls` polls
 * (1 <= polls <= 2^24), recording a timeout in the context's device status word exactly as a
 * TMA-fed kernel does when a tile load never lands.  qpd_device_status then returns QPD_ERR_CUDA and
 * clears the word.  For tests of the error path: nothing is loaded, nothing faults and the context
 * stays usable. */
QPD_API int qpd_probe_wait_timeout(qpd_ctx* ctx, int64_t polls);

/* Device bytes the context holds, and kernels it has launched since creation. */
QPD_API uint64_t qpd_workspace_bytes(const qpd_ctx* ctx);
QPD_API uint64_t qpd_launch_count(const qpd_ctx* ctx);

/* Kernel kinds reported by qpd_stage_times. */
#define QPD_K_ZSTAGE 0   /* fused: source + z transform + fold */
#define QPD_K_YPASS 1    /* fused: y transform + fold */
#define QPD_K_XPASS 2    /* fused: x transform + |S Amp|^2 + fftshift */
#define QPD_K_PACK 3     /* float64 -> packed inputs */
#define QPD_K_SOURCE 4   /* plain: one source component */
#define QPD_K_FFTZ 5     /* plain: z transform */
#define QPD_K_AXIS 6     /* plain: y or x transform */
#define QPD_K_ACC 7      /* plain: amplitude update */
#define QPD_K_INTENSITY 8 /* plain: intensity + fftshift */
#define QPD_K_ADJSEED 9  /* adjoint: x pass of the recomputed forward, seeding dL/dconj(Amp) */
#define QPD_K_ADJAXIS 10 /* adjoint: x or y pass */
#define QPD_K_ADJZ 11    /* adjoint: z transform + source transpose */
#define QPD_K_COUNT 12

/* Per-kernel timing: while on, CUDA events are recorded around every kernel the context
 * launches.  qpd_stage_times waits for them, writes the summed device milliseconds and the
 * launch count of each kind (arrays of cap >= QPD_K_COUNT) and clears the record.  Replaces
 * the MPI_Wtime splits of src/heffte/qpop_diffraction_mgpu.cu:168-178. */
QPD_API int qpd_enable_timing(qpd_ctx* ctx, int32_t on);
QPD_API int qpd_stage_times(qpd_ctx* ctx, double* ms, uint64_t* counts, int32_t cap);

/* Tiles per CTA of the persistent z stages (0, the default: one wave of CTAs walks all tiles of a
 * volume).  With k > 0 every CTA takes at most k tiles, so CTAs retire while the kernel runs and a
 * kernel on a higher-priority stream gets SMs within about k tiles' time instead of after the whole
 * z stage: the serving loop uses it so that small volumes are not held behind a large one.  Results
 * do not depend on it.  No counterpart in the reference (its z transform is a cuFFT/HeFFTe call). */
QPD_API int qpd_set_cta_tiles(qpd_ctx* ctx, int32_t tiles);

/* Reciprocal-space-map projections of a device-resident intensity I (nx, ny, nz) float64, z
 * fastest: xy[x * ny + y] = sum_z I, xz[x * nz + z] = sum_y I, yz[y * nz + z] = sum_x I (a NULL
 * output is skipped).  Deterministic: fixed summation order, no atomics.  With the tensor-product
 * q grid every map of src/python/rsm.py:88-104 (numpy.histogram2d of I over two broadcast q
 * components) is one of these projections re-binned along its two 1-D axes, which the host does
 * on the small maps.  No context: failures are described by qpd_last_error(NULL); ny <= 16384.
 * Asynchronous on `stream` (NULL: the default stream). */
QPD_API int qpd_rsm_project(const double* I, int64_t nx, int64_t ny, int64_t nz, double* xy, double* xz, double* yz,
                            void* stream);

/* Bytes of the device array behind qpd_run_device_noalloc. */
#define QPD_NOALLOC_SCRATCH_BYTES (32u << 20)

/* No counterpart in the reference: an allocation-free variant of qpd_run_device for callers
 * that must not let a library allocate device memory (a framework whose allocator owns the GPU's
 * memory, a real-time loop that reserves everything at start-up).  Same float32 fused computation
 * and the same caller-owned packed inputs (single phase mode: phase index and optional weight) and
 * output as qpd_run_device, but no context: the grid and crystal come with the call, and the
 * intermediate fields and tables live in one library-wide device array of
 * QPD_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until exit.  Grids whose
 * fields (96 bytes per cell for the perovskite cell) and tables do not fit are refused with
 * QPD_ERR_NOMEM; more than 12 distinct R_x, or more than 12 distinct R_y sharing one R_x, with
 * QPD_ERR_UNSUPPORTED; both before anything is launched.  nAtom <= 16, nz <= 1024, nx, ny <= 4096.
 * The first call on a device looks up the array's address and uploads constant tables with that
 * device current, so make it before any stream capture; a device reset after it is not supported.
 * Calls share the array: calls that can overlap on the GPU race and must be serialised by the
 * caller.  Failures are described by qpd_last_error(NULL).  Asynchronous on `stream` (NULL: the
 * default stream). */
QPD_API int qpd_run_device_noalloc(const qpd_grid* grid, const qpd_crystal* crystal, const void* P, const void* U,
                                   const int8_t* phase, const void* weight, double* I_dev, void* stream);

/* Stage plan of an axis of length N (no GPU needed): writes at most cap radices, returns
 * their count, or a negative code. */
QPD_API int qpd_axis_radices(int64_t N, int32_t* radices, int32_t cap);

#ifdef __cplusplus
}
#endif

#endif /* QPOPDIFF_H_ */
