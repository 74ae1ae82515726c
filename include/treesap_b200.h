/* treesap-b200: C ABI of the B200 single-level explicit integrator.
 *
 * Plain C types only (no CUDA, no C++ and no torch types in any signature). Every entry
 * point returns a ts_status and never throws or aborts; the text of the last failure of a
 * context is available from ts_context_last_error(). The reference (treesap, header-only
 * C++20 over AMReX) has no FFI of its own; each entry point below names the reference
 * interface it stands in for (paths relative to the reference's src/treesap/).
 *
 * Threading: one ts_context per host thread. All device work of a context is enqueued on
 * the context's CUDA stream in call order; *_sync entry points wait for it.
 *
 * HBM layout of a field (all state and stage buffers): component-major, [comp][z][y][x] with
 * x fastest, `ngrow` ghost cells on every face, the x origin shifted by `xoff` (ngrow rounded
 * up to 32 bytes) so that interior rows start on a 32-byte sector, and the row pitch padded to
 * 32 bytes:  element (i, j, k, c) is at  ((c*pz + k+ngrow)*py + j+ngrow)*px + i+xoff
 * for i in [-ngrow, n0+ngrow), j in [-ngrow, n1+ngrow), k in [-ngrow, n2+ngrow).
 */
#ifndef TREESAP_B200_H
#define TREESAP_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define TS_ABI_VERSION 2

#if defined(__GNUC__)
#define TS_API __attribute__((visibility("default")))
#else
#define TS_API
#endif

typedef enum ts_status {
    TS_OK = 0,
    TS_ERR_INVALID_ARGUMENT = 1, /* bad descriptor, size or pointer */
    TS_ERR_UNSUPPORTED = 2,      /* valid request outside the instantiated model set */
    TS_ERR_CUDA = 3,             /* a CUDA runtime call failed (text in ts_context_last_error) */
    TS_ERR_OUT_OF_MEMORY = 4,
    TS_ERR_DEVICE = 5,           /* a kernel reported an error word (bounded wait expired, bad index) */
    TS_ERR_NO_DEVICE = 6,        /* no usable sm_100 device */
    TS_ERR_NONFINITE = 7         /* ts_integrator_check_finite found a NaN or infinite state value */
} ts_status;

typedef enum ts_dtype { TS_F64 = 0, TS_F32 = 1 } ts_dtype;
typedef enum ts_model { TS_MODEL_WAVE = 0, TS_MODEL_TENSOR_WAVE = 1 } ts_model;
typedef enum ts_scheme {
    TS_EULER = 0,
    TS_RK4 = 1,
    TS_DOPRI5 = 2 /* Dormand-Prince 5(4) with step-size control (rtol, atol); FP64, one box */
} ts_scheme;
typedef enum ts_bc { TS_BC_NOOP = 0, TS_BC_DIRICHLET = 1 } ts_bc;
typedef enum ts_precision {
    TS_PRECISION_F64 = 0,      /* plain form: FP64 throughout, the reference's register scheme */
    TS_PRECISION_F32_STAGE = 1 /* FP32 stage arithmetic and storage, FP64 state and final combination */
} ts_precision;
typedef enum ts_init_kind {
    TS_INIT_STATE = 0,
    TS_INIT_GAUSSIAN = 1,
    TS_INIT_FOURIER = 2,
    TS_INIT_EXPRESSION = 3 /* ts_integrator_initialise_expressions */
} ts_init_kind;

/* ------------------------------------------------------------------ runtime */
typedef struct ts_context ts_context;

TS_API int ts_abi_version(void);
TS_API const char* ts_status_string(ts_status s);

/* One device, one stream, one device error word. */
TS_API ts_status ts_context_create(int device, ts_context** out);
TS_API ts_status ts_context_destroy(ts_context* ctx);
/* Waits for all work of the context, then reads and clears the device error word. */
TS_API ts_status ts_context_sync(ts_context* ctx);
TS_API const char* ts_context_last_error(const ts_context* ctx);
/* The context's cudaStream_t and its device error word (int*), for callers that launch
 * their own kernels (e.g. the header-only C++ front end) on the same stream. */
TS_API void* ts_context_stream(ts_context* ctx);
TS_API int* ts_context_error_word(ts_context* ctx);
TS_API int ts_context_sm_count(const ts_context* ctx);

/* Failure injection (test and diagnostic hooks; no counterpart in the reference, which aborts
 * inside AMReX on errors). Nothing here faults, traps or hangs a GPU:
 *   TS_FAULT_SKIP_COPY: in the next fused stage launch of a single-box integrator on this
 *     context, the producer warps skip the TMA copy of item plane `arg` (>= 0) and every
 *     mbarrier wait of that launch gives up after 1 ms instead of 2 s. The consumer warps that
 *     needed the plane time out, record kErrMbarTimeout in the device error word and return;
 *     the next ts_context_sync reports TS_ERR_DEVICE and clears the word. One-shot.
 *   TS_FAULT_ALLOC: the next `arg` device field allocations made on the calling host thread
 *     fail as out of memory (no cudaMalloc is made), so the entry point that allocates returns
 *     TS_ERR_OUT_OF_MEMORY. arg = 0 clears it.
 *   TS_FAULT_NONE: clears both. */
typedef enum ts_fault { TS_FAULT_NONE = 0, TS_FAULT_SKIP_COPY = 1, TS_FAULT_ALLOC = 2 } ts_fault;
TS_API ts_status ts_context_inject_fault(ts_context* ctx, int fault, long long arg);
/* Used by the header front end when it builds a stage launch: takes (and clears) the pending
 * TS_FAULT_SKIP_COPY of the context. Returns 1 with *plane and *wait_ns set when one is
 * pending, else 0. */
TS_API int ts_context_take_stage_fault(ts_context* ctx, int* plane, unsigned long long* wait_ns);

/* ------------------------------------------------------------------ field layout */
typedef struct ts_field_layout {
    int n[3];          /* valid cells per direction */
    int ngrow;         /* ghost width */
    int ncomp;
    int dtype;         /* ts_dtype */
    int xoff;          /* x index of cell i = 0 within a row, ngrow rounded up to 32 bytes */
    int reserved;
    long long px, py, pz; /* padded extents (elements): row pitch, rows per plane, planes per component */
} ts_field_layout;

/* Fills *out for the given extents (replaces the allocation rule of
 * SingleLevelIntegrator.hpp:47-49: MultiFab(ba, dm, ncomp, ngrow)). */
TS_API ts_status ts_field_layout_make(const int n[3], int ngrow, int ncomp, int dtype, ts_field_layout* out);
TS_API long long ts_field_bytes(const ts_field_layout* layout);
/* Encodes the TMA descriptor (a 128-byte CUtensorMap) used by the fused stage kernels to
 * stream a field plane by plane: a 4-d tensor (x, y, z, comp) read in boxes of
 * (box_x, box_y, 1, ncomp). `base` is a device pointer to the field. */
TS_API ts_status ts_field_tensor_map(const ts_field_layout* layout, const void* base, int box_x, int box_y,
                              void* tensor_map_out);

/* ------------------------------------------------------------------ built-in models
 * The built-in models are ordinary treesap user models (treesap_b200/cpp/rhs/) instantiated
 * in this library through the header front end:
 *   TS_MODEL_WAVE         {phi, pi}: phi_t = pi, pi_t = c(x)^2 sum_a D2_aa phi
 *   TS_MODEL_TENSOR_WAVE  {h_ij, p_ij} (2 x SymRank2Alias): h_t = p,
 *                         p_t = Lap h - 1/3 delta Lap tr h + 1/2 (d_i d_k h_kj + d_j d_k h_ki)
 * optionally wrapped in KODecorator{rhs, ko_strength} (order = ngrow) and, when
 * abl_thickness > 0, built as ABLPDEModel (absorbing layer, Dirichlet(target) ghosts).
 * TS_MODEL_TENSOR_WAVE is built for ngrow 3, ko_strength > 0, TS_BC_NOOP, TS_RK4 (FP64 or
 * FP32-stage), no absorbing layer; other tensor descriptors return TS_ERR_UNSUPPORTED. */
typedef struct ts_wave_desc {
    int n[3];
    double prob_lo[3];
    double prob_hi[3];
    int periodic[3];
    int ngrow;               /* 1..4 */
    int model;               /* ts_model */
    double ko_strength;      /* > 0: Kreiss-Oliger dissipation */
    int abl_thickness;       /* > 0: absorbing layer of this many cells */
    double abl_max_strength;
    int abl_profile;         /* 1: s, 2: s^2 */
    int bc;                  /* ts_bc, for non-periodic faces (forced to Dirichlet(target) by the layer) */
    double bc_values[12];    /* Dirichlet values / absorbing-layer targets per component */
    double dt;
    int scheme;              /* ts_scheme */
    int precision;           /* ts_precision (TS_PRECISION_F32_STAGE needs TS_RK4) */
    const double* c2;        /* TS_MODEL_WAVE only: host array of c(x)^2 per valid cell, x fastest; NULL = 1 */
    int block[3];            /* block_size (SingleLevelIntegrator.hpp:47-49): 0 < block[2] < n[2] splits the
                              * domain into z slabs of at most block[2] planes (any scheme), whose ghost
                              * planes are exchanged every stage; the result is bitwise the single box's.
                              * block[0], block[1] (and 0 = the whole domain) keep one box in x and y, which
                              * the stage kernels tile themselves. */
    double rtol, atol;       /* TS_DOPRI5: relative / absolute error tolerance (0: 1e-6 / 1e-9) */
} ts_wave_desc;

typedef struct ts_integrator ts_integrator;

/* SingleLevelRK4Integrator / SingleLevelEulerIntegrator(model, block_size)
 * (integrators/SingleLevelRK4Integrator.hpp:65-67, SingleLevelEulerIntegrator.hpp:51-52). */
TS_API ts_status ts_integrator_create(ts_context* ctx, const ts_wave_desc* desc, ts_integrator** out);
TS_API ts_status ts_integrator_destroy(ts_integrator* it);

/* One z slab of a domain shared by several processes or GPUs (no counterpart in the reference,
 * whose boxes are exchanged by AMReX's MPI FillPatch, SingleLevelIntegrator.hpp:153-163): planes
 * [zlo, zlo + nz) of the domain `desc` (TS_MODEL_WAVE with unit speed; RK4, FP32-stage RK4 or
 * Euler), with the
 * lower / upper ghost planes filled by the caller's halo exchange when lo_ex / hi_ex is set
 * (interior faces, and both end faces of a domain periodic in z), else by the ghost fill. The
 * integrator's set/get_state and initialise act on the slab's own cells ([comp][z_slab][y][x],
 * global coordinates); it steps through the calls below, all enqueued on the context stream:
 *   for each stage s < ts_slab_stages():
 *     ts_slab_prepare(s)                     (stage register step)
 *     exchange: ts_slab_send_planes(s, face) gives the ngrow boundary planes to send to the
 *       neighbour across `face` (0 lower, 1 upper; whole planes from component 0, `elems`
 *       elements of `elem_size` bytes per component (8, or 4 for the FP32 stage registers),
 *       components `comp_stride` elements apart, device memory); the planes the neighbour
 *       sends are copied into this slab's ghost planes with ts_slab_receive_planes(s, face,
 *       buf), buf holding ncomp blocks of `elems` elements (device memory)
 *     ts_slab_fill(s)                        (every other ghost cell)
 *     ts_slab_launch(s)                      (the fused stage kernel)
 *   ts_slab_finish()                         (time, step count, state swap)
 * Every process must take the same stages in the same order; the neighbour's planes for stage s
 * are those of its stage-s register after its ts_slab_prepare(s). */
TS_API ts_status ts_integrator_create_slab(ts_context* ctx, const ts_wave_desc* desc, int zlo, int nz, int lo_ex,
                                           int hi_ex, ts_integrator** out);
TS_API int ts_slab_stages(ts_integrator* it);
TS_API ts_status ts_slab_prepare(ts_integrator* it, int stage);
TS_API ts_status ts_slab_send_planes(ts_integrator* it, int stage, int face, void** ptr, long long* elems,
                                     long long* comp_stride, int* elem_size);
TS_API ts_status ts_slab_receive_planes(ts_integrator* it, int stage, int face, const void* buf);
TS_API ts_status ts_slab_fill(ts_integrator* it, int stage);
TS_API ts_status ts_slab_launch(ts_integrator* it, int stage);
TS_API ts_status ts_slab_finish(ts_integrator* it);
TS_API int ts_integrator_ncomp(const ts_integrator* it);

/* initialise() (Integrator.hpp:75-78, SingleLevelIntegrator.hpp:75-93): evaluates the
 * initial condition at cell centres lo + (i + 1/2) dx on the device. init_kind
 * TS_INIT_GAUSSIAN: nitems pulses {comp, A, w, cx, cy, cz};
 * TS_INIT_FOURIER: nitems modes {comp, A, kx, ky, kz, phase}. Resets time and step count. */
TS_API ts_status ts_integrator_initialise(ts_integrator* it, int init_kind, int nitems, const double* items);

/* initialise() with treesap::FunctionInit (init/FunctionInit.hpp:34-101): one expression of
 * x, y, z per component (count = ncomp), e.g. "exp(-(x^2 + y^2 + z^2)/0.1^2)", compiled on the
 * host and evaluated at the cell centres on the device. Operators + - * / ^ ** (right
 * associative), comparisons, and / or, functions sin cos tan asin acos atan sinh cosh tanh exp
 * log log10 sqrt abs floor ceil erf heaviside pow atan2 min max fmod if(c, a, b), constant pi.
 * Invalid text returns TS_ERR_INVALID_ARGUMENT (message in ts_context_last_error). */
TS_API ts_status ts_integrator_initialise_expressions(ts_integrator* it, int count, const char* const* exprs);

/* Host evaluation of one expression at n points (the program the device evaluates); for
 * checking expressions without a device. */
TS_API ts_status ts_expression_eval(const char* expr, int n, const double* x, const double* y, const double* z,
                                    double* out);

/* Valid-cell state, component-major [comp][z][y][x] FP64. `src`/`dst` are host pointers
 * (pageable or pinned) unless *_is_device is nonzero. set_state resets time and step count. */
TS_API ts_status ts_integrator_set_state(ts_integrator* it, const double* src, int src_is_device);
TS_API ts_status ts_integrator_get_state(ts_integrator* it, double* dst, int dst_is_device);

/* step() x nsteps (Integrator.hpp:91-106): ghost fill + computeNewState + swap per step,
 * enqueued on the context stream (returns without waiting). */
TS_API ts_status ts_integrator_step(ts_integrator* it, int nsteps);

/* End-to-end call: host state in -> nsteps steps -> host state out, synchronous. */
TS_API ts_status ts_integrator_run(ts_integrator* it, const double* host_in, int nsteps, double* host_out);

TS_API ts_status ts_integrator_time(const ts_integrator* it, double* time, long long* steps);

/* Device pointer and layout of the current FP64 state (valid after the last enqueued step). */
TS_API ts_status ts_integrator_state_field(ts_integrator* it, void** device_ptr, ts_field_layout* layout);

/* Capture one step into a CUDA graph and replay it for subsequent ts_integrator_step calls
 * (enable != 0), or go back to per-kernel launches (enable == 0). */
TS_API ts_status ts_integrator_use_graph(ts_integrator* it, int enable);
/* TS_DOPRI5 integrators: steps accepted and rejected since the last initialise / set_state, the
 * step size proposed for the next step and the scaled error norm of the last attempt. Each
 * ts_integrator_step call advances one accepted step (retrying rejected ones); the simulation
 * time (ts_integrator_time) is the sum of the accepted step sizes. */
TS_API ts_status ts_integrator_adaptive_stats(ts_integrator* it, long long* accepted, long long* rejected,
                                              double* next_dt, double* last_error);
/* Health check (no counterpart in the reference): waits for the integrator's stream and scans
 * the valid cells of the state; TS_ERR_NONFINITE when any value is NaN or infinite. */
TS_API ts_status ts_integrator_check_finite(ts_integrator* it);

/* Device time of the most recent ts_integrator_step call, measured with CUDA events on the
 * context stream (valid after ts_context_sync), and the number of kernels it launched. */
TS_API ts_status ts_integrator_last_step_timing(ts_integrator* it, double* ms, long long* launches);

/* Runs nsteps steps (like ts_integrator_step) with a CUDA event pair around every kernel
 * launch, waits, and returns per kernel class c < nclasses the number of launches and their
 * summed device time in ms. Classes: 0 ghost fill, 1 + s stage s of the step (Euler: 1).
 * (Instrumentation of Integrator.hpp:91-106 / ScopedTimer.hpp, with device clocks.) */
TS_API ts_status ts_integrator_profile(ts_integrator* it, int nsteps, int nclasses, long long* launches, double* ms);

/* Overrides the launch shape of the fused stage kernels: rows = tile height (consumer warps
 * per CTA, 0 = automatic), chunks = number of z chunks (0 = automatic). Used by the autotuner;
 * the default shape is chosen per launch from the SM count and the domain. */
TS_API ts_status ts_integrator_set_launch_shape(ts_integrator* it, int rows, int chunks);

/* ------------------------------------------------------------------ batched instances
 * No counterpart in the reference, which advances one model per integrator object: `count`
 * independent instances of TS_MODEL_WAVE (each descriptor its own extents, geometry, dt,
 * periodicity, boundary values and Kreiss-Oliger strength; all with the same ngrow (2 or 4),
 * precision, scheme TS_RK4 and either all or none with Kreiss-Oliger; no absorbing layer, no
 * c2) advanced together. Per RK4 stage ONE persistent launch of the fused stage kernel walks a
 * work list of (instance, tile, z range) items; per ghost fill one launch covers all
 * instances; with ts_batch_use_graph each step replays a captured CUDA graph. Results are
 * bitwise identical to ts_integrator_* on each instance. TS_BC_NOOP ghost cells hold 0. */
typedef struct ts_batch ts_batch;
/* A batch (like an integrator) uses its context's stream: destroy it before the context. */
TS_API ts_status ts_batch_create(ts_context* ctx, const ts_wave_desc* descs, int count, ts_batch** out);
TS_API ts_status ts_batch_destroy(ts_batch* b);
TS_API int ts_batch_size(const ts_batch* b);
/* Like ts_integrator_initialise for one instance (at most 64 items). */
TS_API ts_status ts_batch_initialise(ts_batch* b, int instance, int init_kind, int nitems, const double* items);
TS_API ts_status ts_batch_set_state(ts_batch* b, int instance, const double* src, int src_is_device);
TS_API ts_status ts_batch_get_state(ts_batch* b, int instance, double* dst, int dst_is_device);
/* nsteps RK4 steps of every instance, enqueued on the context stream. */
TS_API ts_status ts_batch_step(ts_batch* b, int nsteps);
TS_API ts_status ts_batch_use_graph(ts_batch* b, int enable);
/* Work-item shape: tile rows and z-range length in planes (0 = automatic: the largest tile,
 * whole z extents). */
TS_API ts_status ts_batch_set_launch_shape(ts_batch* b, int rows, int zchunk);
/* Times candidate shapes on the batch itself (trial_steps steps each, states restored
 * afterwards), keeps the fastest and returns it. */
TS_API ts_status ts_batch_autotune(ts_batch* b, int trial_steps, int* rows, int* zchunk);
/* Device time and kernel launches of the last ts_batch_step call (valid after ts_context_sync). */
TS_API ts_status ts_batch_last_step_timing(ts_batch* b, double* ms, long long* launches);

/* ------------------------------------------------------------------ discrete adjoint
 * No counterpart in the reference. Variable-speed scalar wave model
 *   phi_t = pi + s K phi,   pi_t = c(x)^2 sum_a D2_aa phi + s K pi
 * (D2 centred of half-width ngrow, K the Kreiss-Oliger operator of order ngrow, s =
 * ko_strength) on a periodic grid, RK4 in FP64: the same arithmetic as ts_integrator_* with
 * KO and a c2 field. desc: TS_MODEL_WAVE, ngrow 2 or 4, periodic in every direction,
 * TS_RK4, TS_PRECISION_F64, no absorbing layer; desc->c2 is ignored (the speed is an argument
 * of every call). All arrays are host arrays of the valid cells (x fastest, n0 n1 n2 values).
 * Loss J = 1/2 sum_cells (phi(T) - phi_target)^2. The reverse sweep runs RK4 with the
 * transposed operator, recomputing the forward states from checkpoints taken every
 * `checkpoint_every` steps. */
typedef struct ts_adjoint ts_adjoint;
TS_API ts_status ts_adjoint_create(ts_context* ctx, const ts_wave_desc* desc, int checkpoint_every, ts_adjoint** out);
TS_API ts_status ts_adjoint_destroy(ts_adjoint* a);
/* phi(T), pi(T) after nsteps from (phi0, pi0 (NULL = 0)) with speed c; outputs may be NULL. */
TS_API ts_status ts_adjoint_forward(ts_adjoint* a, const double* phi0, const double* pi0, const double* c, int nsteps,
                                    double* phi_T, double* pi_T);
/* J and dJ/dphi0, dJ/dpi0, dJ/dc (any output may be NULL). */
TS_API ts_status ts_adjoint_gradient(ts_adjoint* a, const double* phi0, const double* pi0, const double* c, int nsteps,
                                     const double* phi_target, double* loss, double* grad_phi0, double* grad_pi0,
                                     double* grad_c);
/* FP32-stage form of J and dJ/dphi0, dJ/dpi0, dJ/dc: forward run and reverse sweep in the
 * FP32-stage RK4 form (stencils of the stage differences in FP32, FP64 states). The state
 * gradient needs no checkpoints; the speed gradient (grad_c non-NULL) recomputes each forward
 * step's FP32-stage registers from checkpoints taken every `checkpoint_every` steps, like
 * ts_adjoint_gradient. Any output may be NULL. */
TS_API ts_status ts_adjoint_gradient_f32(ts_adjoint* a, const double* phi0, const double* pi0, const double* c,
                                         int nsteps, const double* phi_target, double* loss, double* grad_phi0,
                                         double* grad_pi0, double* grad_c);
/* Tangent-linear run: the perturbation (dphi(T), dpi(T)) caused by (dphi0, dpi0, dc) (NULL = 0). */
TS_API ts_status ts_adjoint_tangent(ts_adjoint* a, const double* phi0, const double* pi0, const double* c,
                                    const double* dphi0, const double* dpi0, const double* dc, int nsteps,
                                    double* dphi_T, double* dpi_T);

/* ------------------------------------------------------------------ allocation-free stepping
 * No counterpart in the reference. For callers that must not allocate device memory: host
 * applications that own all device memory through their own pool or arena, and loops that
 * cannot afford cudaMalloc / cudaFree because those may synchronise the device and stall the
 * caller's other streams. Advances `state` (a caller-owned device buffer in the layout of
 * ts_field_layout_make(n, 2, 2, TS_F64), ghost cells included) by nsteps RK4 steps with the
 * same fused stage kernels and ghost fills as ts_integrator_step, on `stream` (a
 * cudaStream_t, 0 = the legacy default stream), and waits for it, on errors as well: when
 * the call returns, none of its GPU work is still in flight. Supported: TS_MODEL_WAVE,
 * ngrow 2, optional Kreiss-Oliger, periodic / Dirichlet / NoOp boundaries, TS_RK4 in FP64;
 * anything else returns TS_ERR_UNSUPPORTED. Simulation time restarts at 0 on every call (the
 * supported models do not depend on time).
 * Scratch: the three RK4 stage registers and a device error word live in one static device
 * array of TS_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until exit; a
 * domain whose three padded fields do not fit (about 100^3 cells) returns
 * TS_ERR_INVALID_ARGUMENT before any work. The first call on a device looks up the array's
 * device address; make that first call before any stream capture. All calls share the array
 * (each call clears it first), so calls whose GPU work overlaps, on any streams, race. */
#define TS_NOALLOC_SCRATCH_BYTES (48ull * 1024ull * 1024ull)
TS_API ts_status ts_wave_rk4_steps_noalloc(const ts_wave_desc* desc, double* state, int nsteps, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TREESAP_B200_H */
