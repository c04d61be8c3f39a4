/*
 * tdgl_b200.h — C ABI of the B200 trapezoidal TDGL stepper.
 *
 * Plain C: pointers, sizes and a CUDA stream handle.  Every entry point
 * returns a tdgl_status; device pointers are owned by the caller and must
 * stay valid until the stream has passed the call.  One context is used from
 * one thread at a time; distinct contexts are independent.
 *
 * Layouts
 *   reference layout  complex128 state of tdgl3d: blocks [psi, phi_x, phi_y,
 *                     (phi_z)] of n_interior entries each, interior nodes in
 *                     the order of GridIndices.interior_to_full (k fastest)
 *                     (src/tdgl3d/core/state.py:11-97,
 *                      src/tdgl3d/mesh/indices.py:271-278).  Stored as
 *                     interleaved doubles (re, im); imaginary parts of phi
 *                     are ignored on input and written as +0.0.
 *   device layout     tdgl_state_len() doubles: component arrays psi_re,
 *                     psi_im, phi_x, phi_y, (phi_z), each of tdgl_npad()
 *                     entries, nodes numbered i fastest.  Padding entries
 *                     must be zero.
 *
 * Each compute entry point names the reference function it replaces.
 */
#ifndef TDGL_B200_H
#define TDGL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* tdgl_stream_t; /* same handle as cudaStream_t */
typedef struct tdgl_ctx tdgl_ctx;

typedef enum tdgl_status {
  TDGL_OK = 0,
  TDGL_ENOCONV = 1,     /* Newton / TGCR did not converge (reference: empty array, converged=False, RuntimeError) */
  TDGL_EDTMIN = 2,      /* adaptive dt fell below dt_min (integrators.py:190-195) */
  TDGL_EKMAX = 3,       /* more Krylov directions needed than the workspace holds */
  TDGL_ENONFINITE = 4,  /* a norm became NaN or Inf */
  TDGL_ETIMEOUT = 5,    /* a device-side wait hit its time limit; the kernel returned */
  TDGL_EINVAL = 6,      /* invalid argument (reference: ValueError) */
  TDGL_ECUDA = 7,       /* CUDA runtime error */
  TDGL_ENOMEM = 8       /* workspace allocation failed */
} tdgl_status;

typedef enum tdgl_precision {
  TDGL_FP64 = 0,        /* Krylov vectors and Jacobian products in FP64 */
  TDGL_MIXED = 1        /* Krylov vectors and analytic Jacobian products in FP32; state,
                           residuals, norms and dot products in FP64 */
} tdgl_precision;

typedef enum tdgl_jvp_mode {
  TDGL_JVP_FD = 0,       /* (f(x + eps p) - f(x)) / eps, eps = eps_mf (1 + |x|) / |p| (tgcr.py:129-133); FP64 only */
  TDGL_JVP_ANALYTIC = 1, /* exact tangent-linear RHS */
  TDGL_JVP_KRYLOV = 2    /* tdgl_jvp only: the exact product as the context's analytic-product
                            Krylov solves compute it (its Krylov precision, FP32 for TDGL_MIXED;
                            the step graph's stencil kernel on the full-grid layout) */
} tdgl_jvp_mode;

typedef enum tdgl_krylov {
  TDGL_KRYLOV_GMRES = 0, /* Arnoldi basis, one stored vector per iteration (default) */
  TDGL_KRYLOV_GCR = 1    /* the reference's GCR: (p, Ap) pairs, tgcr.py:96-156 */
} tdgl_krylov;

/* Grid and physics (SimulationParameters, src/tdgl3d/core/parameters.py:10-51). */
typedef struct tdgl_grid_desc {
  int32_t Nx, Ny, Nz;                       /* cells; Nz == 1 is the 2-D model */
  int32_t periodic_x, periodic_y, periodic_z;
  double hx, hy, hz;
  double kappa;                             /* used when kappa_full is NULL */
} tdgl_grid_desc;

/* Holes and materials, all host pointers, any may be NULL / zero-length.
 * hole_*_links: GridIndices.hole_*_bc_mask (full-grid link indices);
 * hole_*_interior: GridIndices.hole_*_bc_interior (reference interior numbering)
 * (src/tdgl3d/mesh/indices.py:136-232).  kappa_full: MaterialMap.kappa (dim_x);
 * sc_interior: MaterialMap.interior_sc_mask (n_interior); a NULL sc_interior
 * means "no material map" (bare Ginzburg-Landau term, sparse_operators.py:218-226). */
typedef struct tdgl_material_desc {
  const int64_t* hole_links[3];
  int64_t n_hole_links[3];
  const int64_t* hole_interior[3];
  int64_t n_hole_interior[3];
  const double* kappa_full;
  const double* sc_interior;
} tdgl_material_desc;

/* Applied field schedule (AppliedField, src/tdgl3d/physics/applied_field.py:14-56). */
typedef struct tdgl_field {
  double Bx, By, Bz;
  double t_on_fraction, ramp_fraction;
  double t_field_stop;                      /* the t_stop the schedule is relative to */
  int32_t ramp;
  int32_t constant;                         /* 1: (Bx,By,Bz) at every t, schedule ignored */
} tdgl_field;

/* Trapezoidal options (trapezoidal(), src/tdgl3d/solvers/integrators.py:92-118). */
typedef struct tdgl_trap_opts {
  double t_stop, dt, dt_min;
  double newton_tol_f, newton_tol_dx, tol_gcr, eps_mf;
  int32_t newton_max_iter;
  int32_t krylov_max_iter;                  /* <= 0: the reference default, len(b) (capped by the workspace) */
  int32_t adaptive;
  int32_t jvp_mode;                         /* tdgl_jvp_mode */
} tdgl_trap_opts;

/* Counters and last values of one call. */
typedef struct tdgl_stats {
  int32_t status;
  int32_t steps;                            /* accepted steps in this call */
  int32_t newton_converged, newton_iters_last, krylov_last, max_krylov;
  int64_t newton_iters, krylov_iters, rhs_evals, jvp_evals, rejections;
  int64_t krylov_sq;                        /* sum over linear solves of (iterations)^2 */
  double t, dt_cur;                         /* integrator clock after the call */
  double last_gnorm, last_dxnorm;
  int64_t kernel_launches;
} tdgl_stats;

/* ---- context ------------------------------------------------------------ */

/* Build the device description of a grid (construct_indices + material map,
 * src/tdgl3d/mesh/indices.py:239-450, src/tdgl3d/core/material.py:182-254).
 * precision: tdgl_precision.  kmax: Krylov directions the workspace holds (>= 1). */
int tdgl_ctx_create(const tdgl_grid_desc* grid, const tdgl_material_desc* material, int32_t precision,
                    int32_t kmax, tdgl_ctx** out);
int tdgl_ctx_destroy(tdgl_ctx* ctx);
/* Krylov method of the context's solves (tdgl_krylov).  Both minimise the
 * residual over the same Krylov space with the reference's stopping test
 * (tgcr.py:125, 154); GMRES stores one vector per iteration instead of two. */
int tdgl_ctx_set_krylov(tdgl_ctx* ctx, int32_t kind);
int64_t tdgl_n_interior(const tdgl_ctx* ctx);
int64_t tdgl_npad(const tdgl_ctx* ctx);
int64_t tdgl_state_len(const tdgl_ctx* ctx);        /* doubles of one device-layout state */
int64_t tdgl_workspace_bytes(const tdgl_ctx* ctx);  /* device bytes the context holds */
const char* tdgl_status_string(int status);
const char* tdgl_last_error(void);                  /* text of the last failure on this thread */

/* ---- layout -------------------------------------------------------------- */

/* Reference layout (2*n_state doubles) -> device layout. */
int tdgl_pack(tdgl_ctx* ctx, const double* x_ref, double* x_dev, tdgl_stream_t stream);
/* Device layout -> reference layout. */
int tdgl_unpack(tdgl_ctx* ctx, const double* x_dev, double* x_ref, tdgl_stream_t stream);

/* ---- operators ----------------------------------------------------------- */

/* f = dX/dt in the device layout.  Replaces eval_f (src/tdgl3d/physics/rhs.py:147-239)
 * with the applied field (Bx, By, Bz) placed as build_boundary_field_vectors does. */
int tdgl_rhs(tdgl_ctx* ctx, const double* x_dev, double* f_dev, double Bx, double By, double Bz,
             tdgl_stream_t stream);
/* Adjoint of tdgl_rhs at x (device layout, FP64, any context precision):
 * gx = J(x)^T v with J = d f / d x (device layout, overwritten);
 * gsc[d] = d(v . f)/d sc at interior node d (device order; zero without a
 * material map; may be NULL); gk2[d] = d(v . f)/d kappa(d)^2 (may be NULL);
 * gpar = d(v . f)/d(Bx, By, Bz, kappa) (4 doubles, may be NULL; the kappa
 * entry is for a uniform kappa and 0 with per-node kappa).  Adds the
 * differentiation form the reference lacks: it is the hand-derived reverse
 * pass of eval_f (src/tdgl3d/physics/rhs.py:147-239) including the
 * boundary procedure (rhs.py:54-139). */
int tdgl_vjp(tdgl_ctx* ctx, const double* x_dev, const double* v_dev, double Bx, double By, double Bz,
             double* gx_dev, double* gsc_dev, double* gk2_dev, double* gpar_dev, tdgl_stream_t stream);
/* eval_f on reference-layout device buffers (pack, RHS, unpack). */
int tdgl_eval_f(tdgl_ctx* ctx, const double* x_ref, double* f_ref, double Bx, double By, double Bz,
                tdgl_stream_t stream);
/* ap = p - dt/2 J(x) p in the device layout (the A*p of tgcr_matrix_free_trap,
 * src/tdgl3d/solvers/tgcr.py:129-133).  mode FD uses eps = eps_mf (1+|x|)/|p|.
 * mode TDGL_JVP_KRYLOV runs the stepper's own product kernel in the context's
 * Krylov precision on its stepping workspace and blocks until the stream has
 * passed it (TDGL_EINVAL while a tdgl_trap_launch is uncollected;
 * TDGL_ETIMEOUT when a bounded wait of the kernel ran out). */
int tdgl_jvp(tdgl_ctx* ctx, const double* x_dev, const double* p_dev, double* ap_dev, double dt, int32_t mode,
             double eps_mf, double Bx, double By, double Bz, tdgl_stream_t stream);
/* Observables at interior nodes in reference order (n_interior doubles each):
 * |psi|^2 (solution.py:76-78), B with boundary conditions (solution.py:94-158),
 * J_s without boundary conditions (solution.py:180-217). */
int tdgl_observables(tdgl_ctx* ctx, const double* x_dev, double Bx, double By, double Bz, double* psi2,
                     double* bx, double* by, double* bz, double* jx, double* jy, double* jz,
                     tdgl_stream_t stream);

/* ---- analysis (post-processing of one device-layout state) ---------------- */
/* Phase winding number of every elementary plaquette of every interior
 * z-slice, as count_vortices_plaquette computes it for one slice
 * (src/tdgl3d/analysis/vortex_counting.py:14-139): w_dev holds
 * max(Nz-1, 1) x (Nx-2) x (Ny-2) doubles, index (k (Nx-2) + i) (Ny-2) + j for
 * the plaquette with corners at interior nodes (i, j) .. (i+1, j+1) of slice
 * k; NaN where a corner's |psi|^2 is below mask_threshold. */
int tdgl_plaquette_winding(tdgl_ctx* ctx, const double* x_dev, double mask_threshold, double* w_dev,
                           tdgl_stream_t stream);
/* Mean |psi|^2 and mean |J_s| over the interior nodes with sc_ref > 0
 * (sc_ref: interior superconducting mask in reference order, device memory;
 * NULL: all nodes), the quantities compute_convergence_metrics compares
 * (src/tdgl3d/analysis/convergence.py:14-117).  out_dev: 3 doubles [mean
 * |psi|^2, mean |J_s|, node count].  Allocates its scratch on first use. */
int tdgl_convergence_means(tdgl_ctx* ctx, const double* x_dev, const double* sc_ref_dev, double* out_dev,
                           tdgl_stream_t stream);

/* ---- solvers (device-resident control; blocking: returns after the stream work) ---- */

/* Solve (I - dt/2 J(x_lin)) d = b.  Replaces tgcr_matrix_free_trap
 * (src/tdgl3d/solvers/tgcr.py:96-156).  Returns TDGL_ENOCONV when the relative
 * residual stays above tol (the reference returns an empty array). */
int tdgl_tgcr_trap(tdgl_ctx* ctx, const double* x_lin_dev, const double* b_dev, double* d_dev, double dt,
                   double tol, int32_t max_iter, double eps_mf, int32_t jvp_mode, double Bx, double By,
                   double Bz, tdgl_stats* stats, tdgl_stream_t stream);
/* Newton on x - dt/2 f(x) - gamma = 0 from x (updated in place).  Replaces
 * newton_gcr_trap (src/tdgl3d/solvers/newton.py:76-120); convergence is
 * reported in stats->newton_converged and iterations in stats->newton_iters_last. */
int tdgl_newton_trap(tdgl_ctx* ctx, double* x_dev, const double* gamma_dev, double dt, double tol_f,
                     double tol_dx, int32_t max_iter, double tol_gcr, double eps_mf, int32_t jvp_mode,
                     double Bx, double By, double Bz, tdgl_stats* stats, tdgl_stream_t stream);
/* Advance x (device layout, in place) through at most max_steps accepted
 * trapezoidal steps from *t with step *dt_cur (both updated).  Replaces the
 * loop of trapezoidal (src/tdgl3d/solvers/integrators.py:150-197). */
int tdgl_trap_run(tdgl_ctx* ctx, double* x_dev, double* t, double* dt_cur, int32_t max_steps,
                  const tdgl_trap_opts* opts, const tdgl_field* field, tdgl_stats* stats, tdgl_stream_t stream);
/* Adjoint trapezoidal solve (no reference counterpart): (I - h J(x)^T) mu = b
 * for the RHS with field (Bx, By, Bz), J^T applied by the adjoint kernel of
 * tdgl_vjp, by GMRES from mu = 0 to ||b - A mu|| <= tol ||b||, entirely on
 * the device (one graph launch; the host reads the outcome once).  FP64
 * contexts only; x, b, mu in the device layout.  Stops at kmax iterations
 * without restart: TDGL_ENOCONV then, with the last iterate in mu (a caller
 * can restart from it).  *iters = iterations.  Synchronises the stream. */
int tdgl_adjoint_solve(tdgl_ctx* ctx, const double* x_dev, const double* b_dev, double* mu_dev, double h,
                       double tol, double Bx, double By, double Bz, int32_t* iters, tdgl_stream_t stream);
/* tdgl_trap_run in two halves, for stepping many contexts concurrently (the
 * batched form; no reference counterpart): tdgl_trap_launch enqueues the
 * steps on the stream and returns at once (GMRES contexts only; x must stay
 * valid until the stream has passed them); tdgl_trap_collect waits for the
 * launch and returns the clock, step size, counters and status.  One
 * tdgl_trap_launch per context at a time (plus one tdgl_trap_launch_next
 * queued behind it); while a launch is pending, the
 * context's other stepping entry points (tdgl_trap_run, tdgl_newton_trap,
 * tdgl_tgcr_trap, tdgl_euler_run, tdgl_arnoldi_probe, tdgl_ctx_set_blocks,
 * tdgl_ctx_set_poly)
 * return TDGL_EINVAL, as they share its workspace. */
int tdgl_trap_launch(tdgl_ctx* ctx, double* x_dev, double t, double dt_cur, int32_t max_steps,
                     const tdgl_trap_opts* opts, const tdgl_field* field, tdgl_stream_t stream);
int tdgl_trap_collect(tdgl_ctx* ctx, double* t, double* dt_cur, tdgl_stats* stats);
/* A continuation of the context's last step-graph launch (no reference
 * counterpart; it keeps the loop of trapezoidal, integrators.py:150-197, on
 * the device across calls): enqueues up to max_steps more steps on the
 * stream, starting from the clock (t, dt_cur) and the state that the
 * previous launch leaves, so that a caller can queue the next steps before it
 * collects the previous ones (at most two launches queued per context).
 * Launches are collected in order with tdgl_trap_collect, which waits for
 * the launch it collects; a continuation whose clock has reached t_stop runs
 * no step (steps = 0). */
int tdgl_trap_launch_next(tdgl_ctx* ctx, double* x_dev, int32_t max_steps, const tdgl_trap_opts* opts,
                          const tdgl_field* field, tdgl_stream_t stream);
/* Launch shape of the step graph's grid kernels: block counts, each in
 * [1, 8 x SMs], of the grid-stride passes and of the Arnoldi streams (defaults
 * 8 and 5 blocks per SM), and whether the Arnoldi product and projections run
 * as one kernel (fused 1) or two (0; -1: the default, one kernel for FP64
 * vectors and two for FP32).  Any setting gives a correct step; reductions are
 * deterministic for a given setting.  Used by the batched form's autotuner
 * (small instances run concurrently on few blocks each); the graph is rebuilt
 * at the next launch.  No reference counterpart. */
int tdgl_ctx_set_blocks(tdgl_ctx* ctx, int32_t stream_blocks, int32_t krylov_blocks, int32_t fused);
/* Limits of the context's device-side waits and loops (no reference
 * counterpart; the reference runs on one host thread and has none):
 * wait_ns bounds every single wait inside a kernel (the persistent kernel's
 * grid barrier, the staged-copy waits of the TMA-staged stencil), after which
 * the kernel stops and the call returns TDGL_ETIMEOUT; loop_cap bounds the
 * conditional-loop iterations of one step-graph launch, after which the
 * launch stops and the call returns TDGL_ETIMEOUT.  Values <= 0 restore the
 * defaults (5 s; a cap derived from max_steps, newton_max_iter and kmax).
 * The context stays usable after either limit has run out. */
int tdgl_ctx_set_limits(tdgl_ctx* ctx, int64_t wait_ns, int64_t loop_cap);
/* Degree (0 to 12) of the polynomial right preconditioner of the GMRES solves
 * with analytic Jacobian products: GMRES runs on A p(A), A = I - dt/2 J,
 * p the Chebyshev-iteration polynomial of that degree for the interval
 * [1 - dt/2, 1 + dt/2 rho], rho a Gershgorin bound of J; the Newton
 * correction is p(A) times the Krylov combination, so the stop test and the
 * solution are those of the unpreconditioned system.  0 turns it off, -1
 * restores the default (10, or TDGL_POLY_DEGREE).  The finite-difference
 * (reference) form never uses it.  The graph is rebuilt at the next launch;
 * TDGL_EINVAL while a launch is pending.  No reference counterpart (the
 * reference's GCR is unpreconditioned). */
int tdgl_ctx_set_poly(tdgl_ctx* ctx, int32_t degree);
/* Degree in use (or that the next graph will use); -1 for a null context. */
int32_t tdgl_ctx_poly_degree(const tdgl_ctx* ctx);
/* Forward Euler: n_steps steps of min(dt, t_stop - t) from *t (updated)
 * (src/tdgl3d/solvers/integrators.py:35-89). */
int tdgl_euler_run(tdgl_ctx* ctx, double* x_dev, double* t, double t_stop, double dt, int32_t n_steps,
                   const tdgl_field* field, tdgl_stream_t stream);

/* ---- allocation-free operator ---------------------------------------------- */

/* dX/dt of one reference-layout state (device pointers x_ref, f_ref of
 * 2*n_state doubles each), like tdgl_eval_f, but without a context and
 * without allocating any memory: for callers that must not call cudaMalloc
 * when they run (a fixed device-memory budget, device memory owned by another
 * allocator, or no tolerance for the synchronisation an allocation implies).
 * Geometry flags and intermediates are built on the device in one static
 * array of this library (about 8.6 MiB per GPU that loads it, held until the
 * process exits).  Limits: 32768 interior nodes, 262144 full-grid nodes,
 * 65536 entries per hole list; larger inputs return TDGL_EINVAL before any
 * device work.  Calls share that array: calls that overlap on the GPU race.
 * The first call on a device looks the array up (cudaGetSymbolAddress) and
 * keeps its address for the life of the process: make it before any stream
 * capture, and do not call again after cudaDeviceReset.  The material
 * descriptor's arrays are host memory copied on every call; a call that has
 * any returns TDGL_EINVAL while its stream is capturing.  No counterpart in
 * the reference. */
int tdgl_eval_f_noalloc(const tdgl_grid_desc* grid, const tdgl_material_desc* material, const double* x_ref,
                        double* f_ref, double Bx, double By, double Bz, tdgl_stream_t stream);

/* ---- diagnostics --------------------------------------------------------- */

/* Kernel and phase timers (global-timer nanoseconds), recorded when the
 * environment variable TDGL_PROFILE is set before the solver workspace is
 * created.  GMRES graph executor: out[k] = summed first-block-start to
 * last-block-end time of kernel type k (0 prepare, 1 predict, 2 newton_rhs,
 * 3 stencil, 4 projections, 5 orthogonalisation, 6 update, 7 accept, 8 Arnoldi
 * product, 9 Arnoldi orthogonalisation, 10 Arnoldi projections), out[16 + k] =
 * its launch count, k < 16.  Persistent
 * executor: out[0..15] block-0 totals per phase, out[64 + 1024 s + b]
 * per-block compute totals of phase s (0: Krylov stencil, 1:
 * orthogonalisation).  No reference counterpart (the reference only times
 * whole runs, io/logging.py:284-314). */
int tdgl_profile(tdgl_ctx* ctx, uint64_t* out, int64_t n, int32_t reset);
/* `launches` back-to-back Arnoldi steps of the GMRES graph (analytic
 * products) outside the graph, forming basis vector ja from whatever the
 * workspace holds, without the Krylov bookkeeping; synchronises the stream.
 * kernels selects what runs (bit 0 orthogonalisation, bit 1 product, bit 2
 * projections, bit 3 fused product and projections, bit 4 the polynomial
 * preconditioner's steps, bits 5-7 the Newton-stage kernels: predictor,
 * Newton residual, Newton update over ja basis vectors, which overwrite the
 * iterate; 0 = the graph's own).
 * For timing and profiling the kernels alone.  No reference counterpart. */
int tdgl_arnoldi_probe(tdgl_ctx* ctx, int32_t ja, int32_t launches, int32_t kernels, tdgl_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* TDGL_B200_H */
