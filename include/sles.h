/*
 * sles.h -- C ABI of the B200 spectral-LES library (libsles_b200.so).
 *
 * The reference (a-k-sangwan/spectral-LES) is pure Python; its hot path is
 * a set of functions that mutate an ``InitializeDomain`` attribute bag.  This
 * library replaces the arithmetic of those functions; the Python package
 * ``sles`` (spectral-les_b200/sles) keeps the reference's call surface and
 * calls these entry points through ctypes.  Each declaration names the
 * reference code it replaces (path:line inside the reference repository).
 *
 * Conventions
 *  - All pointers are device pointers unless stated; fields use the layouts
 *    documented in sles_layout below.  No torch or C++ types cross the ABI.
 *  - Every call takes an explicit cudaStream_t (passed as void*), enqueues
 *    work and returns without synchronising, except where stated.
 *  - Return value: SLES_OK (0) or a positive SLES_ERR_* code; nothing throws.
 *  - No entry point allocates device memory on the hot path: intermediate
 *    fields live in a caller-provided workspace (sles_plan_workspace_bytes).
 *  - A plan is not thread-safe; use one stream per plan.
 */
#ifndef SLES_H
#define SLES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SLES_VERSION 1

enum sles_status {
  SLES_OK = 0,
  SLES_ERR_INVALID_ARG = 1,     /* null pointer, bad enum, inconsistent sizes       */
  SLES_ERR_UNSUPPORTED = 2,     /* grid size / combination without a compiled kernel */
  SLES_ERR_CUDA = 3,            /* a CUDA runtime call failed                        */
  SLES_ERR_WORKSPACE = 4,       /* workspace missing or smaller than required        */
  SLES_ERR_TIMEOUT = 5,         /* a bounded device-side wait gave up                */
  SLES_ERR_NONFINITE = 6,       /* a reduction saw NaN/Inf (reference: dt != dt)     */
  SLES_ERR_STATE = 7            /* call out of order (e.g. ETD2 step before bootstrap) */
};

enum sles_dtype { SLES_F32 = 0, SLES_F64 = 1 };
enum sles_les_model { SLES_LES_NONE = 0, SLES_LES_SMAGORINSKY = 1, SLES_LES_VREMAN = 2 };
enum sles_scheme { SLES_RK4 = 0, SLES_RK3 = 1, SLES_ETD2 = 2 };

/*
 * Plan descriptor.  Mirrors InitializeDomain(nu, dimension, No_of_gridpoint,
 * forcing, method, LES_ON, Cs, LES_model) (src/initialize_domain.py:20-33).
 * ``n`` is the computational grid (the reference divides No_of_gridpoint by 4
 * when LES is on, src/initialize_domain.py:38-40; the Python layer applies it).
 */
typedef struct sles_plan_desc {
  int dim;          /* 2 or 3 */
  int n;            /* grid points per axis: 16,24,32,48,64,96,128,256,512 (3D); up to 1024 (2D) */
  int dtype;        /* enum sles_dtype: arithmetic of the fields and transforms */
  int les_model;    /* enum sles_les_model */
  int scheme;       /* enum sles_scheme */
  int parity;       /* 1: the reference's arithmetic including its quirks; 0: corrected schemes */
  double nu;        /* kinematic viscosity */
  double cs;        /* Smagorinsky / Vreman constant */
  double forcing;   /* linear forcing coefficient (src/RK4_method.py:58-64) */
} sles_plan_desc;

typedef struct sles_plan sles_plan;

/* Field layout numbers for a plan: elements per half-complex field (complex
 * count, rows padded to nkp), per real field, and the padded row length. */
typedef struct sles_layout {
  int64_t hc_elems;     /* N*N*nkp (3D) or N*nkp (2D) complex elements */
  int64_t real_elems;   /* N^dim real elements */
  int32_t nkp;          /* padded length of a half-complex row (>= N/2+1) */
  int32_t nk;           /* N/2 + 1 */
} sles_layout;

/* Build a plan (replaces the PFFT plan + wavenumber/mask set-up,
 * src/initialize_domain.py:59-65, 76-114, 162-167).  No device allocation. */
int sles_plan_create(const sles_plan_desc* desc, sles_plan** out);
int sles_plan_destroy(sles_plan* plan);
int sles_plan_layout(const sles_plan* plan, sles_layout* out);
/*
 * Kernel variants (no counterpart in the reference): some passes are compiled
 * in several tile geometries; which one runs is a plan setting, chosen by
 * default per grid size and precision or by the autotuner (sles/autotune.py),
 * which times each.  Every variant computes the same arithmetic (results agree
 * to the last bit or, where the compiler contracts a*b+c differently, to round-off).
 *   SLES_PASS_X: the x pass (stage update); variants 0..count-1
 *   SLES_PASS_Y: the y passes (tile width 8 or 16 columns; variant 1 only for
 *                the float32 3D grids 128, 256, 512, where the count is 2)
 *   SLES_PASS_Z: the fused z pass (1 or 2 z lines per work item; idem)
 *   SLES_PASS_AX: the adjoint's x pass (sles_adjoint_stage / _prime): 0 direct
 *                loads, 1 the TMA tile ring for the Runge-Kutta schemes (the
 *                3D grids 128, 256, 512, where the count is 2 and 1 is the
 *                default; ETD2 reverse steps load directly under either)
 * sles_plan_variant_count returns 0 for an invalid pass (1: no alternative);
 * sles_plan_get_variant returns -1 for an invalid pass.
 */
enum { SLES_PASS_X = 0, SLES_PASS_Y = 1, SLES_PASS_Z = 2, SLES_PASS_AX = 3 };
int sles_plan_variant_count(const sles_plan* plan, int pass);
int sles_plan_get_variant(const sles_plan* plan, int pass);
int sles_plan_set_variant(sles_plan* plan, int pass, int variant);
/*
 * Slab decomposition of one 3D domain over P ranks (one GPU each), the
 * layout of the reference's mpi4py-fft PFFT (src/initialize_domain.py:59-65,
 * slab bounds src/utilites.py:18-24 with N divisible by P): rank r holds the
 * ky rows [r m, (r+1) m) of every spectral field, as [N kx][m ky][nkp], and the
 * x planes [r m, (r+1) m) of physical space (m = N/P <= 256).  Call
 * sles_plan_set_slab before sles_plan_set_workspace; afterwards
 * sles_plan_layout reports the slab's element counts, the whole-grid entry
 * points (sles_rhs, sles_stage, transforms, diagnostics, adjoint, static
 * workspace) return SLES_ERR_STATE, and one RHS evaluation is
 *   sles_slab_prime   (or the previous sles_slab_stage): the inverse
 *                     x-transforms of the state on this rank's ky rows, into
 *                     the n_exchange1 fields at send1
 *   exchange 1        the caller's all-to-all (NCCL): for each field f, block
 *                     q (block_elems elements) of send1[f] goes to rank q and
 *                     block r of recv1[f] on rank q comes from rank r
 *                     (src/initialize_domain.py:59-65: the PFFT global transpose)
 *   sles_slab_middle  y inverse (reading recv1 across the P blocks), the fused
 *                     z pass (u x omega, eddy viscosity, stress), y forward,
 *                     whose n_exchange2 output fields are stored at send2 as P
 *                     blocks; umax_bits (optional device word, zeroed by the
 *                     caller) receives the ordered encoding of this rank's
 *                     max u (find_max_velocity, src/SM_solver.py:245-255; the
 *                     caller all-reduces the max over ranks)
 *   exchange 2        the same all-to-all from send2 into recv2
 *   sles_slab_stage   x forward, combine, projection, the stage update
 *                     (as sles_stage; not SLES_STAGE_RECORD_F1/PRIMED, not the
 *                     reference's ETD2 with LES), and unless
 *                     SLES_STAGE_NO_PREPARE the priming of the next evaluation.
 * State fields (u_cur, u0, u1, u_out, aux) are 3 fields in the slab layout.
 * The exchange buffers live in the plan's workspace (sles_slab_buffers).
 */
typedef struct sles_slab_layout {
  int32_t nranks, rank, m;        /* P, r, rows per block (N/P) */
  int32_t n_exchange1;            /* fields of exchange 1 (6 with LES, else 5) */
  int32_t n_exchange2;            /* fields of exchange 2 (6 with LES, else 3) */
  int32_t reserved;
  int64_t block_elems;            /* complex elements per block: m*m*nkp */
  int64_t field_elems;            /* complex elements per field on this rank: N*m*nkp */
} sles_slab_layout;
int sles_plan_set_slab(sles_plan* plan, int nranks, int rank);
/*
 * Ensemble batch (no counterpart in the reference; the reference runs one
 * domain per process): the plan steps `nmembers` independent domains of its
 * grid, scheme, closure and precision together, every pass one launch over
 * the work items of all members.  Each field argument of sles_stage / sles_rhs
 * then holds the members one after another inside each component:
 * [component][member][layout of one domain] (sles_plan_layout's hc_elems
 * counts all members).  nu_dev / cs_dev: device arrays of nmembers float64
 * values (each member's viscosity and C_s; NULL: the descriptor's value for
 * all), read by the kernels, so they must stay valid while the plan runs.
 * Call before sles_plan_set_workspace (the workspace scales with nmembers);
 * not with sles_plan_set_slab.  On a batched plan only sles_stage (without
 * u_phys / curl_phys) and sles_rhs run; the other entry points return
 * SLES_ERR_STATE.
 */
int sles_plan_set_batch(sles_plan* plan, int nmembers, const double* nu_dev, const double* cs_dev);
int sles_slab_info(const sles_plan* plan, sles_slab_layout* out);
int sles_slab_buffers(sles_plan* plan, void** send1, void** recv1, void** send2, void** recv2);
int sles_slab_prime(sles_plan* plan, const void* u_state, void* stream);
int sles_slab_middle(sles_plan* plan, unsigned long long* umax_bits, void* stream);
int sles_slab_stage(sles_plan* plan, int stage, double dt, const void* u_cur, const void* u0, void* u1,
                    void* u_out, void* aux_out, int flags, void* stream);
/* Bytes of device workspace the plan needs for intermediate fields. */
size_t sles_plan_workspace_bytes(const sles_plan* plan);
/* Attach caller-owned device workspace (>= sles_plan_workspace_bytes). */
int sles_plan_set_workspace(sles_plan* plan, void* ws, size_t bytes);
/* Update run-time scalars (nu, cs, forcing) without rebuilding. */
int sles_plan_set_params(sles_plan* plan, double nu, double cs, double forcing);

/* Batched unscaled r2c over the last ``dim`` axes: PFFT.forward(normalize=False)
 * (src/math_formula.py:7-12, src/initial.py:13).  real_in: nfields real
 * fields; hc_out: nfields half-complex fields. */
int sles_fft_r2c(sles_plan* plan, const void* real_in, void* hc_out, int nfields, void* stream);
/* Batched c2r scaled by 1/N^dim: PFFT.backward(normalize=True)
 * (src/math_formula.py:18-24, src/RK4_method.py:32-34).  Uses the workspace;
 * hc_in is not modified. */
int sles_fft_c2r(sles_plan* plan, const void* hc_in, void* real_out, int nfields, void* stream);

/* Physical velocity and vorticity from U_hat: U = irfftn(U_hat) and
 * curl = irfftn(i k x U_hat) (src/RK4_method.py:28-34, src/math_formula.py:16-25).
 * curl has 3 fields in 3D, 1 in 2D.  Either output may be NULL. */
int sles_velocity_curl(sles_plan* plan, const void* u_hat, void* u_out, void* curl_out, void* stream);

/* Velocity gradient a[i][j] = d u_j / d x_i = irfftn(i K_i U_hat_j) as dim*dim
 * real fields in row-major (i, j) order (src/math_formula.py:27-62). */
int sles_velocity_gradient(sles_plan* plan, const void* u_hat, void* grad_out, void* stream);

/*
 * One right-hand-side evaluation, fused: dU = P(mask*rfftn(u x omega) + T_hat)
 * [+ f U_hat] - nu K^2 U_hat (src/RK4_method.py:38-71 == src/RK3_method.py:44-77,
 * with Smagorinsky_model / Vreman_model, src/smagorinsky.py:8-47,
 * src/vreman.py:8-123, and residue_stress, src/math_formula.py:64-127).
 * u_phys / curl_phys: optional physical fields used instead of the ones
 * implied by u_hat (the reference's stage 0 reuses the stored U and curl,
 * src/RK4_method.py:39-47); pass NULL to derive them from u_hat.
 * f1_out (optional): the projected term before the viscous term and before
 * T_hat is added back (the reference's ETD2 F1, src/RK4_method.py:65-66).
 */
int sles_rhs(sles_plan* plan, const void* u_hat, const void* u_phys, const void* curl_phys,
             void* du_out, void* f1_out, void* stream);

/*
 * One integrator stage, fused with the right-hand side it needs.
 * Replaces the bodies of RK4.solveForNextTimestep (src/RK4_method.py:20-35),
 * RK3.solveForNextTimestep (src/RK3_method.py:20-41) and
 * ETD2.solveForNextTimestep (src/ETD2_method.py:7-37).
 *   u_cur   : U_hat the RHS is evaluated at (read)
 *   u0      : U_hat at the start of the step (read; RK stages)
 *   u1      : RK4 accumulator U_hat1 (read+write); ETD2: F1 of the previous step (read)
 *   u_out   : new U_hat (write; may alias u_cur).  RK4 stage 3 writes the
 *             result to both u1 and u_out (U_hat = U_hat1, src/RK4_method.py:27)
 *   aux_out : ETD2: new F1 (write); with SLES_STAGE_RECORD_F1: recorded F1
 * stage: RK4 0..3, RK3 0..2, ETD2 0.  dt: step size.  u_phys / curl_phys as in
 * sles_rhs.  flags (bitwise OR):
 *   SLES_STAGE_RECORD_F1  record the reference's ETD2 F1 in aux_out
 *   SLES_STAGE_PRIMED     the workspace already holds the x-inverse transforms
 *                         of u_cur (written by the previous stage's call)
 *   SLES_STAGE_NO_PREPARE skip the inverse transforms of u_out that prime the
 *                         next stage
 *   SLES_STAGE_RK4        run an RK4 stage whatever the plan's scheme (ETD2's
 *                         first step, src/ETD2_method.py:8-14)
 * Stage updates use the reference's expressions (RK3: U0 + (dt/2) dU,
 * U0 - dt dU + (2 dt) dU, U0 + dt (dU/6 + 2 dU/3 + dU/6)); with parity = 0 the
 * RK3 plan runs SSP-RK3 and ETD2 the Cox-Matthews weights.
 */
enum { SLES_STAGE_RECORD_F1 = 1, SLES_STAGE_PRIMED = 2, SLES_STAGE_NO_PREPARE = 4, SLES_STAGE_RK4 = 8 };
int sles_stage(sles_plan* plan, int stage, double dt, const void* u_cur, const void* u0, void* u1,
               void* u_out, void* aux_out, const void* u_phys, const void* curl_phys, int flags,
               void* stream);

/*
 * Diagnostics from U_hat, accumulated in float64 with compensated sums:
 * out[0] = E = 1/2 <u.u>, out[1] = eps = nu <|grad u|^2>, out[2] = max_i max_x u_i
 * (signed, as find_max_velocity, src/SM_solver.py:245-255; needs u_phys),
 * out[3] = nonfinite flag.  spectrum (optional, nshell doubles): E(k) on
 * integer shells round(|k|).  out and spectrum are DEVICE pointers.
 */
int sles_diag(sles_plan* plan, const void* u_hat, const void* u_phys, double* out, double* spectrum,
              int nshell, void* stream);

/*
 * Profiling helper (no counterpart in the reference): runs the kernels of one
 * fused RHS evaluation at u_hat ``iters`` times, timing each kernel class with
 * CUDA events on ``stream``, and writes the mean milliseconds per launch to
 * ms[0..4] = {x-inverse (priming), y-inverse, z, y-forward, x-forward+combine}
 * (2D: y entries are 0).  du_scratch receives dU.  Synchronizes the stream.
 */
int sles_profile_rhs(sles_plan* plan, const void* u_hat, void* du_scratch, int iters, double* ms,
                     void* stream);

/*
 * The fused RHS evaluation of sles_rhs for callers that cannot allocate device
 * memory: code that runs where cudaMalloc is off limits (inside an allocator
 * callback, a host application that owns every device allocation through its
 * own pool, a latency-critical loop that must not hit cudaMalloc's implicit
 * synchronization).  No counterpart in the reference.  The scratch is a
 * file-scope device array of SLES_STATIC_WORKSPACE_BYTES inside the library
 * instead of the plan's workspace, so the plan needs no sles_plan_set_workspace
 * for this call; inputs and outputs are still the caller's.  Plans whose
 * workspace (sles_plan_workspace_bytes) exceeds the array are rejected with
 * SLES_ERR_WORKSPACE before anything runs (e.g. 3D LES up to N = 64 in float64,
 * N = 64 in float32; 3D without LES and 2D go further).
 * The first call on a device looks up the array's device address with that
 * device current; make that first call before any stream capture.  The
 * address is kept per device together with the CUDA context it belongs to and
 * looked up again when the current context differs (after cudaDeviceReset the
 * array's old contents are gone with the context).  Every GPU
 * that loads the library holds the array until the process exits.  All calls on
 * a device share the array and it keeps the last call's contents (each call
 * clears the part that must start at zero); calls whose work overlaps on the
 * GPU race on it and must be serialized by the caller.  No cudaMalloc, cudaFree
 * or allocating library call is made.
 */
#define SLES_STATIC_WORKSPACE_BYTES (32u << 20)
int sles_rhs_static_workspace(sles_plan* plan, const void* u_hat, const void* u_phys, const void* curl_phys,
                              void* du_out, void* f1_out, void* stream);
/*
 * Error word of the static array of the current device (no counterpart in the
 * reference): as sles_plan_check, for calls of sles_rhs_static_workspace,
 * whose bounded waits report there.  Synchronises `stream`, stores the word in
 * *flags_out (may be NULL), clears it, returns SLES_ERR_TIMEOUT /
 * SLES_ERR_NONFINITE when such a bit was set.  Check after the calls and
 * before the next one (each call clears the word when it starts).
 * sles_static_workspace_selftest_timeout makes a short bounded wait on that
 * word run out, to exercise the path.
 */
int sles_static_workspace_check(unsigned* flags_out, void* stream);
int sles_static_workspace_selftest_timeout(void* stream);

/*
 * Discrete adjoint of the RK4 step (3D; no counterpart in the reference): the
 * exact transpose of the arithmetic of sles_stage with SLES_STAGE_RK4, i.e. of
 * computeRHS (src/RK4_method.py:38-71) with u x omega (src/math_formula.py:5-13),
 * the projection and mask (:52-57), residue_stress (src/math_formula.py:64-127)
 * with Smagorinsky (src/smagorinsky.py:24-47) or Vreman (src/vreman.py:30-123,
 * gate held fixed) eddy viscosity, the viscous and forcing terms, and the RK4
 * combination (src/RK4_method.py:20-35).  Gradients use the real inner product
 * <x, y> = Re sum conj(x) y over the stored half-complex entries (torch's
 * convention for complex tensors).  The calls need their own caller-owned
 * workspace (256-byte aligned, >= sles_adjoint_workspace_bytes, header word
 * zeroed before first use); the plan's workspace is not touched.
 *
 * Reverse sweep over one step whose forward stage s evaluated the RHS at the
 * state U_s (U_0 = step input, U_1 = U_0 + dt/2 k_0, U_2 = U_0 + dt/2 k_1,
 * U_3 = U_0 + dt k_2), given ubar = gradient w.r.t. the step output:
 *   sles_adjoint_seed   acc = ubar, lam = (dt/6) ubar            (once, at the end of time)
 *   sles_adjoint_prime  prepare the workspace for the stage evaluated at u_state
 *                       with cotangent lam (needed after a seed, or after a
 *                       stage called with u_next = NULL)
 *   sles_adjoint_stage  stage = 3, 2, 1, 0: g = J(U_s)^T lam; acc += g; then
 *                       lam <- dt/3 ubar + dt g (s=3), dt/3 ubar + dt/2 g (s=2),
 *                       dt/6 ubar + dt/2 g (s=1); at s=0 ubar <- acc (the
 *                       gradient w.r.t. the step input) and lam <- (dt/6) acc,
 *                       which seeds the previous step.  u_next = the state of the
 *                       next reverse stage (U_{s-1}, or U_3 of the previous
 *                       step), NULL to skip preparing it.  cs_grad (device
 *                       double, LES plans) accumulates dL/dCs.
 * All three field arguments hold 3 half-complex fields of the plan's layout.
 *
 * Plans of the reference's RK3 (scheme SLES_RK3, parity = 1; src/RK3_method.py:20-41,
 * stages U_1 = U_0 + dt/2 k_0, U_2 = U_0 + dt k_1, output U_0 + dt k_2) use the
 * same calls with stage = 2, 1, 0: seed lam = dt ubar; g = J(U_s)^T lam;
 * acc += g; lam <- dt g (s=2), dt/2 g (s=1); at s=0 ubar <- acc and
 * lam <- dt acc.  Plans of the corrected SSP-RK3 (SLES_RK3, parity = 0;
 * U_1 = U_0 + dt k_0, U_2 = 3/4 U_0 + 1/4 (U_1 + dt k_1), output
 * 1/3 U_0 + 2/3 (U_2 + dt k_2)) run the reverse stages in Shu-Osher form:
 * seed acc = ubar/3, lam = 2/3 dt ubar; s=2: w = 2/3 ubar + g, acc += 3/4 w,
 * ubar <- w/4, lam <- dt/4 w; s=1: w = ubar + g, acc += w, lam <- dt w;
 * s=0: w = acc + g, ubar <- w (the gradient w.r.t. the step input),
 * acc <- w/3, lam <- 2/3 dt w.  Plans of the corrected ETD2 (SLES_ETD2,
 * parity = 0; U_{n+1} = E U_n + w1 F(U_n) + w0 F(U_{n-1}), F without the
 * viscous term, weights at z = dt nu k^2 as in sles_stage) take one reverse
 * step per call: seed lam = w1 ubar (acc unused); stage 0: g = J_F(U_n)^T lam,
 * w = E ubar + g, lam <- w1 w + w0 ubar, ubar <- w; stage 1 (the step after
 * the first, RK4, step): the same with lam <- w0 ubar, the cotangent of
 * F(U_0); stage 2: ubar <- ubar + J_F(u_state)^T lam (applied after the RK4
 * step's reverse on an RK4 plan).  The reference's ETD2 (parity = 1) returns
 * SLES_ERR_UNSUPPORTED.
 */
size_t sles_adjoint_workspace_bytes(const sles_plan* plan);
/* Error word of an adjoint workspace (its header, written by the reverse
 * passes' bounded waits and non-finite checks): as sles_plan_check. */
int sles_adjoint_check(sles_plan* plan, void* adj_ws, unsigned* flags_out, void* stream);
int sles_adjoint_seed(sles_plan* plan, void* adj_ws, double dt, const void* ubar, void* acc, void* lam,
                      void* stream);
int sles_adjoint_prime(sles_plan* plan, void* adj_ws, const void* u_state, const void* lam, void* stream);
int sles_adjoint_stage(sles_plan* plan, void* adj_ws, int stage, double dt, const void* u_next, void* ubar,
                       void* acc, void* lam, double* cs_grad, void* stream);
/*
 * Device-side time-step control (no host synchronisation per step): the
 * driver loop of src/SM_solver.py:18-83 with its CFL rule (compute_dt,
 * src/SM_solver.py:258-277) evaluated on the GPU.  The caller allocates this
 * struct in device memory, fills it (umax_bits, flags, paused, nsteps and
 * t_init zero) and passes it to sles_stage_ctl, which works as sles_stage with
 * dt taken from it:
 *  - stage 0's z pass reduces max_i max_x u_i of the state the step starts
 *    from into umax_bits[parity] (find_max_velocity, src/SM_solver.py:245-255);
 *  - a one-thread kernel then applies the reference's loop logic: dt =
 *    min(CFL dx/u_max, 0.1 dx^2/nu) with CFL = cfl_first before the first
 *    step and cfl after; t = dt before the first step; a step is taken only if
 *    dt is finite and >= 1e-6, t < ek_next (else SLES_DT_SNAPSHOT: the caller
 *    records E(k), raises ek_next and clears paused), and t < t_end and dt >=
 *    1e-8 (else SLES_DT_DONE); a step taken adds dt to t and counts in nsteps;
 *  - while paused, dt_step = 0 and every stage leaves the state unchanged.
 * parity: the step's index modulo 2 (the z pass of a step collects into
 * umax_bits[parity] while the kernel clears the other slot for the next step).
 */
typedef struct sles_dtctl {
  double dt_step;                /* dt applied by the current step (0 while paused) */
  double dt;                     /* last dt from the CFL rule */
  double t;                      /* time as src/SM_solver.py counts it */
  double t_end;                  /* final_time */
  double ek_next;                /* next E(k) snapshot time */
  double cfl_first, cfl;         /* CFL of the first step (0.3 in the reference) and later */
  double dx, nu;
  unsigned long long umax_bits[2];
  unsigned flags;                /* SLES_DT_* */
  unsigned paused;               /* non-zero: steps are no-ops */
  unsigned nsteps;               /* steps taken */
  unsigned t_init;               /* t was set to the first dt */
  unsigned resumed;              /* set by the caller when it clears a snapshot pause: the next
                                    step skips the snapshot test once (the reference takes at
                                    most one snapshot per loop iteration) */
  unsigned reserved;
} sles_dtctl;
enum { SLES_DT_DONE = 1, SLES_DT_SNAPSHOT = 2, SLES_DT_NAN = 4, SLES_DT_TOO_SMALL = 8 };
int sles_stage_ctl(sles_plan* plan, int stage, void* dtctl, int parity, const void* u_cur, const void* u0,
                   void* u1, void* u_out, void* aux_out, const void* u_phys, const void* curl_phys, int flags,
                   void* stream);
/*
 * Device error word of the plan's workspace (no counterpart in the reference).
 * Kernels never spin without bound: a wait that gives up (e.g. on an mbarrier
 * a TMA copy should have completed) sets a bit in the word and the kernel
 * returns.  sles_plan_check synchronises `stream`, stores the word in
 * *flags_out (may be NULL), clears it and returns SLES_ERR_TIMEOUT /
 * SLES_ERR_NONFINITE when such a bit was set, else SLES_OK.
 * sles_selftest_wait_timeout enqueues a kernel that waits on an mbarrier
 * nothing arrives at, with a short limit, to exercise that path (the CUDA
 * context stays usable).
 */
int sles_plan_check(sles_plan* plan, unsigned* flags_out, void* stream);
int sles_selftest_wait_timeout(sles_plan* plan, void* stream);
/* The same self-test against any device error word (e.g. an adjoint
 * workspace's header; 4-byte aligned device pointer). */
int sles_selftest_wait_timeout_word(void* word_dev, void* stream);
/*
 * Device copy of `height` rows of `width` bytes, rows `src_pitch` /
 * `dst_pitch` bytes apart (all three multiples of 8, both pointers 8-byte
 * aligned device memory), on `stream`: fields between the padded layout
 * (rows of nkp bins) and the reference's contiguous (..., N//2+1) layout,
 * e.g. around host copies.  No counterpart in the reference.
 */
int sles_copy_rows(void* dst, size_t dst_pitch, const void* src, size_t src_pitch, size_t width, size_t height,
                   void* stream);
/* Human-readable text for a status code (static storage). */
const char* sles_status_string(int status);
int sles_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SLES_H */
