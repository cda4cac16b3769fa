/*
 * cm_b200.h -- C ABI of the B200 elastic contact library (libcm_b200.so).
 *
 * The library implements, on one NVIDIA B200 (sm_100a), the hot path of
 * ContactEngineering/ContactMechanics v1.8.3:
 *   - the FFT Green's-function operators of PeriodicFFTElasticHalfSpace and
 *     FreeFFTElasticHalfSpace (evaluate_disp / evaluate_force, Hockney
 *     zero padding for free boundaries), and
 *   - the Polonsky-Keer constrained_conjugate_gradients loop including the
 *     plastic hardness cap used by PlasticNonSmoothContactSystem.
 *
 * Conventions
 *   - Real fields are row-major (nx, ny) arrays of double (CM_FP64) or float
 *     (CM_FP32), exactly the memory layout of a C-ordered numpy array of
 *     shape (nx, ny).  "Domain" means the computational grid: (nx, ny) for
 *     periodic substrates, (2nx, 2ny) for free ones.
 *   - All pointers named *_dev are device pointers on the current device.
 *     Pointers named *_host are host pointers.
 *   - Every entry point returns an int status: CM_OK (0) or a CM_ERR_*
 *     code; cm_status_string() describes it.  Solver outcomes that the
 *     reference reports without raising (not converged) come back in
 *     cm_ccg_result.status, not as an error.
 *   - A plan is not re-entrant: calls on one plan must be serialised by the
 *     caller (the reference substrate shares its FFT buffers the same way).
 *   - stream arguments are cudaStream_t passed as void*; NULL means the
 *     plan's own stream.
 */
#ifndef CM_B200_H
#define CM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CM_OK 0
#define CM_ERR_ARG 1          /* invalid argument (mirrors ValueError) */
#define CM_ERR_SHAPE 2        /* array shape mismatch (mirrors Substrate.Error) */
#define CM_ERR_SIZE 3         /* grid too large for the single-pass transforms */
#define CM_ERR_CUDA 4         /* CUDA runtime error */
#define CM_ERR_OOM 5          /* device allocation failed */
#define CM_ERR_NAN 6          /* NaN encountered in the solve (RuntimeError) */
#define CM_ERR_BISECT 7       /* offset bisection sign error (ValueError) */
#define CM_ERR_BISECT_CONV 8  /* offset bisection did not converge (RuntimeError) */
#define CM_ERR_TIMEOUT 9      /* a solve exceeded its host-side time budget */
#define CM_ERR_STOPPED 10     /* the per-iteration observer asked the solve to stop */

/* substrate kinds */
#define CM_PERIODIC 0
#define CM_FREE 1
#define CM_SEMI 2   /* free along some axes, periodic (summed images) along others */

/* precisions */
#define CM_FP64 0   /* everything in FP64 */
#define CM_FP32 1   /* FP32 fields and FFTs, FP64 reductions and scalars */
#define CM_MIXED 2  /* FP32 solve, then FP64 refinement of the same solve; a
                       single solve's refinement that has not converged
                       within max(1000, 4 x its FP32 iterations) restarts as
                       the FP64 solve from the caller's own start */

/* stiffness at q = 0 for periodic substrates */
#define CM_Q0_DEFAULT 0  /* mean of the two lowest non-zero stiffnesses */
#define CM_Q0_ZERO 1     /* stiffness_q0 == 0: G(0) = 0 */
#define CM_Q0_VALUE 2    /* stiffness_q0 given */

/* operators */
#define CM_OP_DISP 0   /* evaluate_disp: displacement from forces */
#define CM_OP_FORCE 1  /* evaluate_force: forces from displacement */

/* solver outcome (cm_ccg_result.status) */
#define CM_SOLVE_CONVERGED 1
#define CM_SOLVE_MAXITER 2

typedef struct cm_plan cm_plan;

typedef struct {
  int kind;            /* CM_PERIODIC or CM_FREE */
  int dim;             /* 1 or 2; a 1D periodic substrate uses ny = 1 */
  int nx, ny;          /* topography grid (nb_grid_pts) */
  double sx, sy;       /* physical_sizes */
  double young;        /* Young's modulus (contact modulus if poisson = 0) */
  double poisson;      /* periodic only */
  int q0_mode;         /* CM_Q0_* (periodic only) */
  double stiffness_q0; /* used when q0_mode == CM_Q0_VALUE */
  double thickness;    /* <= 0: infinitely deep half-space (periodic only) */
  /* CM_SEMI only (SemiPeriodicFFTElasticHalfSpace): periodicity of each axis;
     a periodic axis keeps n points and sums the periodic images
     -n_images..n_images into the kernel, a free axis has 2n - 1 points */
  int periodic_x, periodic_y;
  int n_images;
} cm_plan_desc;

/*
 * One CCG iteration as a per-iteration observer sees it (the reference's
 * callback(it, f_r, d) and logger rows, ConstrainedConjugateGradients.py
 * :436-489).
 */
typedef struct {
  int it;                /* iteration number, 1-based; the FP64 refinement of a
                            CM_MIXED solve continues the FP32 count */
  int precision;         /* CM_FP32 or CM_FP64: the phase the iteration ran in */
  int mode;              /* step kind: 1 steepest descent, 2 conjugate gradient,
                            3 mixing step (delta_str 'sd', 'cg', 'mix') */
  int done;              /* 1 if the iteration ended the phase (maximum
                            iterations or an error) */
  long long area, cg_area, plastic_area;
  long long nc_count;    /* points whose sign constraint was violated (sum(nc_r)) */
  double rms_pen, max_pen, max_pres, pad_pres, maxdu;
  double total_force, offset, tau, mixfac;
  double pentol, forcetol;
  const double* forces;  /* device: the iteration's forces on the domain
                            (nxd, nyd), FP64, valid during the call */
} cm_iteration;

/* returns 0 to continue; any other value stops the solve (CM_ERR_STOPPED) */
typedef int (*cm_iteration_fn)(void* user, const cm_iteration* info);

typedef struct {
  int precision;         /* CM_FP64, CM_FP32 or CM_MIXED */
  int load_control;      /* 1: external_force given; 0: offset given */
  double external_force;
  double offset;
  int has_hardness;
  double hardness;       /* in force units (hardness * area_per_pt) */
  double pentol;         /* <= 0: the reference's default heuristic */
  double forcetol, thermotol, mixfac, mixdecfac;
  int minmixsteps, maxiter;
  int check_every;       /* iterations per host convergence poll; <= 0: auto */
  double fp32_pentol_rel;  /* CM_MIXED: FP32 phase pentol = max(pentol, rel * height range);
                             <= 0: 2e-6 */
  double timeout_s;      /* host-side wall-clock budget; <= 0: none */
  /* cm_ccg_solve only: called on the calling thread after every iteration
     that did not converge, as the reference calls its callback; the solve
     then polls after every iteration.  iteration_forces: caller-owned
     device buffer of nxd * nyd doubles that receives the forces first.
     NULL: no observer (other entry points ignore it). */
  cm_iteration_fn on_iteration;
  void* user;
  double* iteration_forces;
} cm_ccg_params;

typedef struct {
  int status;            /* CM_SOLVE_CONVERGED or CM_SOLVE_MAXITER */
  int nit, nfev;         /* iterations / operator calls (all phases, an
                            abandoned refinement included) */
  int nit_fp32;          /* iterations run in FP32 (CM_MIXED / CM_FP32) */
  int last_step_mix;     /* 1 if the last iteration was a mixing step */
  double offset, fun;
  double rms_pen, max_pen, max_pres, pad_pres, maxdu, total_force;
  double pentol_used;
  long long area, cg_area, plastic_area;
  double ms_fp32, ms_fp64, ms_total;  /* host wall time of the phases of the call */
  int polls;                          /* host convergence polls */
} cm_ccg_result;

/* Returns the message for a status code. */
const char* cm_status_string(int status);

/* Library version string. */
const char* cm_version(void);

/*
 * Create a substrate plan: domain geometry, FFT twiddles and the
 * Green's-function tables built on the device in FP64 (with an FP32 copy).
 * Replaces PeriodicFFTElasticHalfSpace.__init__ (FFTElasticHalfSpace.py:169-306,
 * tables :445-571), FreeFFTElasticHalfSpace.__init__ (:912-964, table
 * :1033-1139) and SemiPeriodicFFTElasticHalfSpace.__init__ (:1295-1363,
 * table :1365-1500).  stream: the stream all work of this plan runs on (NULL: a new
 * non-blocking stream owned by the plan).
 */
int cm_plan_create(const cm_plan_desc* desc, void* stream, cm_plan** out);

/* Release a plan and every device buffer it owns. */
int cm_plan_destroy(cm_plan* plan);

/* Domain and half-spectrum shapes: domain (nxd, nyd); half spectrum (nxd, nyh). */
int cm_plan_shape(const cm_plan* plan, int* nxd, int* nyd, int* nyh);

/*
 * Which transform engine serves the plan's operator and single solves in
 * `precision` (CM_FP64 or CM_FP32): *engine = 1 for the register-resident
 * passes (domain sides 2^k and 3 * 2^m), 0 for the shared-memory
 * mixed-radix passes of every other size.  No counterpart in the reference
 * (numpy's FFT serves every size there).
 */
int cm_plan_engine(const cm_plan* plan, int precision, int* engine);

/*
 * Copy the unscaled FP64 Green's table G(q) (surface displacement per unit
 * pressure in Fourier space) to host memory, layout (nxd, nyh) with the half
 * spectrum along y.  The reference stores the same real values halved along
 * x (FFTElasticHalfSpace.py:445-561, 1033-1139).
 */
int cm_plan_greens_host(cm_plan* plan, double* out_host);

/*
 * Apply the operator to a device field (FFTElasticHalfSpace.py:573-611,
 * free :1141-1197).  The input occupies rows [0,in_rows) x cols [0,in_cols)
 * of the domain (leading dimension in_ld) and is zero elsewhere -- this is
 * the Hockney zero padding; the output region [0,out_rows) x [0,out_cols) is
 * written with leading dimension out_ld.  precision selects float or double
 * buffers (CM_FP64 / CM_FP32).
 */
int cm_apply(cm_plan* plan, int op, int precision, const void* in_dev, int in_rows,
             int in_cols, int in_ld, void* out_dev, int out_rows, int out_cols, int out_ld,
             void* stream);

/*
 * k-space operators (FFTElasticHalfSpace.py:613-805, 841-885).  Half spectra
 * use the reference's layout: complex FP64 values (interleaved re, im) of
 * shape (nxd / 2 + 1, nyd), halved along x, unnormalised (numpy's rfftn
 * over axes (1, 0), the muGrid FFTEngine's forward transform).
 *
 * cm_fft_forward: the half spectrum of a real FP64 field that occupies rows
 * [0,in_rows) x cols [0,in_cols) of the domain (leading dimension in_ld) and
 * is zero elsewhere -- the fftengine.fft of evaluate_k_disp, evaluate_k_force
 * and evaluate (:613-656, 862-866).
 */
int cm_fft_forward(cm_plan* plan, const double* in_dev, int in_rows, int in_cols, int in_ld,
                   double* out_dev, void* stream);

/*
 * k_out = scale * T * k_in on half spectra of the reference layout, with T
 * the Green's table G (op CM_OP_DISP) or the surface stiffness K = 1/G, 0
 * where G = 0 (op CM_OP_FORCE).  evaluate_k_disp(f) = G fft(-f) / a_pt,
 * evaluate_k_force(u) = -K fft(u) a_pt, evaluate_k_force_k(u_k) = -K u_k a_pt
 * (:613-674).  k_in and k_out may be the same array.
 */
int cm_kspace_apply(cm_plan* plan, int op, double scale, const double* k_in_dev, double* k_out_dev,
                    void* stream);

/*
 * Scalar product sum_ij a_ij b_ij of two real domain fields from their half
 * spectra (the power theorem, :686-805): sum over the half spectrum of
 * w_k Re(conj(a_k) b_k) / (nxd nyd), w = 1 on the rows without a mirror
 * (row 0 and, for even nxd, row nxd / 2), 2 on the others.  *out_host
 * receives the sum (FP64 partial sums per block added in a fixed order).
 */
int cm_kspace_dot(cm_plan* plan, const double* ka_dev, const double* kb_dev, double* out_host,
                  void* stream);

/*
 * Polonsky-Keer constrained conjugate gradients
 * (ConstrainedConjugateGradients.py:47-509) on one substrate.
 *   heights_dev      (nx, ny) FP64 topography heights
 *   init_disp_dev    domain-sized FP64 initial displacements or NULL
 *   init_force_dev   domain-sized FP64 initial forces or NULL (takes precedence)
 * Outputs (any may be NULL):
 *   x_dev            domain-sized FP64 displacements (result.x)
 *   jac_dev          (nx, ny) FP64 result.jac = -forces on the topography
 *   active_dev       (nx, ny) uint8 result.active_set on the topography
 *   plastic_dev      (nx, ny) uint8 result.plastic (hardness runs)
 * Returns CM_ERR_NAN / CM_ERR_BISECT* for the cases where the reference
 * raises; otherwise CM_OK with res->status telling converged or maxiter.
 */
int cm_ccg_solve(cm_plan* plan, const cm_ccg_params* params, const double* heights_dev,
                 const double* init_disp_dev, const double* init_force_dev, double* x_dev,
                 double* jac_dev, unsigned char* active_dev, unsigned char* plastic_dev,
                 cm_ccg_result* res);

/*
 * Same as cm_ccg_solve with every array in host memory; the host<->device
 * copies are part of the call.
 */
int cm_ccg_solve_host(cm_plan* plan, const cm_ccg_params* params, const double* heights_host,
                      const double* init_disp_host, const double* init_force_host,
                      double* x_host, double* jac_host, unsigned char* active_host,
                      unsigned char* plastic_host, cm_ccg_result* res);

/*
 * Solve n independent contact problems (each with its own plan, i.e. its own
 * grid size, substrate and tables) together: every iteration advances all
 * unfinished solves with one launch per field pass over the combined
 * (solve, tile) work list, replayed from a CUDA graph.  CM_MIXED runs the
 * FP32 phase of all solves, then the FP64 refinement of all solves.  All
 * params must share the precision.  Arrays are per solve, device pointers;
 * init_disp_dev, x_dev, jac_dev, active_dev, plastic_dev may be NULL (the
 * whole array) or hold NULL entries.  Results in res[0..n).  The batch
 * replaces n calls of constrained_conjugate_gradients
 * (ConstrainedConjugateGradients.py:47-509); each solve keeps the reference's
 * semantics, and its result does not depend on the other members of the batch.
 */
int cm_ccg_solve_batch(int n, cm_plan* const* plans, const cm_ccg_params* params,
                       const double* const* heights_dev, const double* const* init_disp_dev,
                       double* const* x_dev, double* const* jac_dev,
                       unsigned char* const* active_dev, unsigned char* const* plastic_dev,
                       cm_ccg_result* res, void* stream);

/*
 * Stepping interface for continuous batching.  A stepper owns a stream and
 * reusable staging buffers.  Each in-flight solve lives on its own plan:
 *   cm_ccg_begin     set up a solve on a free plan (FP32 phase for CM_FP32 and
 *                    CM_MIXED, FP64 phase for CM_FP64)
 *   cm_ccg_step      advance any set of in-flight solves (different sizes and
 *                    phases) by `iters` iterations each, together; done[i] tells
 *                    whether solve i has finished its current phase
 *   cm_ccg_handover  for a solve whose phase finished: CM_MIXED moves from the
 *                    FP32 phase to the FP64 refinement (*finished = 0); otherwise
 *                    *finished = 1
 *   cm_ccg_end       write the results and free the plan for the next solve
 * Together they run constrained_conjugate_gradients
 * (ConstrainedConjugateGradients.py:47-509) in pieces, so that a request loop
 * can admit and retire solves between steps; a solve's result does not depend
 * on which others share its steps.
 */
typedef struct cm_stepper cm_stepper;
int cm_stepper_create(void* stream, cm_stepper** out);
int cm_stepper_destroy(cm_stepper* stepper);
int cm_ccg_begin(cm_stepper* stepper, cm_plan* plan, const cm_ccg_params* params,
                 const double* heights_dev, const double* init_disp_dev, const double* init_force_dev);
int cm_ccg_step(cm_stepper* stepper, int n, cm_plan* const* plans, int iters, int* done);
int cm_ccg_handover(cm_stepper* stepper, cm_plan* plan, const double* heights_dev, int* finished);
int cm_ccg_end(cm_stepper* stepper, cm_plan* plan, double* x_dev, double* jac_dev,
               unsigned char* active_dev, unsigned char* plastic_dev, cm_ccg_result* res);

/*
 * The periodic operator (evaluate_disp or evaluate_force of a 2D periodic
 * half-space with the default q = 0 stiffness, FP64) for callers that must
 * not allocate device memory: code that runs where the host application
 * owns every device allocation through its own pool, or inside a loop that
 * cannot afford the device-wide synchronisation cudaMalloc may cause.  No
 * plan is needed and nothing is allocated: the Green's table, twiddles and
 * spectrum are built in a fixed 4 MiB array that the library keeps in device
 * memory (each GPU that loads the library holds it until the process exits),
 * so nx and ny are limited to 512; larger grids return CM_ERR_SIZE.  in_dev
 * and out_dev are caller-owned (nx, ny) FP64 device arrays; work is enqueued
 * on `stream` (NULL: the legacy default stream).  Every call looks up that
 * array's device address on the current device (cudaGetSymbolAddress); the
 * first lookup on a device may load the library's code there, so make the
 * first call on each device before any stream capture.  All calls share the array: calls
 * that overlap on the GPU race and corrupt each other's results.
 * This entry point has no counterpart in the reference.
 */
int cm_apply_periodic_noalloc(int nx, int ny, double sx, double sy, double young, double poisson,
                              int op, const double* in_dev, double* out_dev, void* stream);

/*
 * Self-test of the bounded grid barrier that separates the passes of the
 * solver's one-launch offset bisection (and every other wait on another
 * block inside a launch): `blocks` blocks, launched cooperatively, meet at
 * one barrier whose arrival count starts at `phantom`.  With phantom = 0 the
 * barrier completes; with phantom >= blocks the count never reaches the
 * release value (arrivals that never come), so every block waits until its
 * limit of `limit_us` microseconds of SM clock runs out, the first to give up
 * raises the barrier's abort word and the others leave.  *gave_up receives
 * the number of blocks whose wait gave up.  The launch ends by itself either
 * way and leaves the context usable.  Instrumentation; no reference
 * counterpart.
 */
int cm_selftest_grid_barrier(int blocks, int phantom, double limit_us, int* gave_up);

/*
 * Tuning of the per-pass kernels that batched solves (cm_ccg_solve_batch),
 * the stepping interface and sizes without register-resident passes (sides
 * other than 2^k and 3 * 2^m) run.
 * cm_tuning_set_tiles: transform elements per row or column tile for
 * sequences of `length` points (a row tile of a domain with ny columns holds
 * tile_elems / ny rows, a column tile up to tile_elems / nx columns), for
 * plans created afterwards; 0 restores the default (2048).
 * cm_tuning_set_batch_threads: threads per block of the batched transform
 * launches (a multiple of 32, at most 512; default 256).  cm_tuning_get
 * reports the values in force.  The package's autotuner measures them and
 * stores them as JSON.  No reference counterpart (the reference's transforms
 * are muGrid's).
 */
int cm_tuning_set_tiles(int precision, int length, int tile_elems);
int cm_tuning_set_batch_threads(int precision, int threads);
int cm_tuning_get(int precision, int length, int* tile_elems, int* batch_threads);

/*
 * With enable = 1, batches of elastic solves without a timeout run in one
 * launch of the persistent cluster kernel: each thread-block cluster takes
 * whole solves (FP32 phase, FP64 refinement, result fields) from a device
 * queue.  enable = 0 (the default) runs every batch on the lockstep per-pass
 * kernels (a graph of launches per group of iterations), measured faster on
 * a B200; plastic or timed batches always take it.  No reference
 * counterpart.
 */
int cm_tuning_set_batch_persistent(int enable);

/*
 * Number of kernels this library has launched in the process (graph nodes
 * count once per replay).  Instrumentation; no reference counterpart.
 */
unsigned long long cm_launch_count(void);

/*
 * Per-kernel timing of the solver's iteration: initialises a solve like
 * cm_ccg_solve (precision CM_FP64 or CM_FP32) and runs `iters` iterations
 * eagerly with a CUDA event between kernels on the plan's stream.  Writes
 * the average milliseconds of each of the *n_kernels kernels (launch order)
 * to ms_per_kernel (capacity >= 16) and, if names is not NULL, their names.
 * Plans that run the persistent solver kernel report it as entry 0
 * ("k_ccg_persist", event-timed milliseconds per iteration) followed by its
 * phases ("k_ccg_persist:<phase>", milliseconds per iteration from
 * in-kernel timer stamps of a second run; they sum to about entry 0).
 * Returns CM_ERR_ARG if the solve stopped before `iters` iterations.
 * Instrumentation; no reference counterpart.
 */
int cm_ccg_profile(cm_plan* plan, const cm_ccg_params* params, const double* heights_dev,
                   int iters, float* ms_per_kernel, int* n_kernels, const char** names);

#ifdef __cplusplus
}
#endif
#endif /* CM_B200_H */
