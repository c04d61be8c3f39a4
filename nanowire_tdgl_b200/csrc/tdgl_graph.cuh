// Graph executor of the trapezoidal stepper (GMRES inner solve).
//
// The same algorithm as the persistent stepper (src/tdgl3d/solvers/
// integrators.py:92-206, newton.py:76-120, tgcr.py:96-156 with the Krylov
// solve in its GMRES form), expressed as small kernels sequenced by one CUDA
// graph with nested conditional WHILE nodes:
//
//   STEP while { step_begin, prepare, predict, newton_rhs, newton_init,
//     NEWTON while { KRYLOV while { arn_orth, arn_apply, arn_dots },
//                    newton_solve, update_fused, newton_rhs, newton_check },
//     accept, step_end }
//
// (arn_apply and arn_dots as one kernel, arn_apply_dots, for FP64 vectors),
// with KRYLOV while { stencil, dots, fin_dots, orth, fin_orth } and update for
// finite-difference Jacobian products.  Grid kernels stream over the vectors
// and write per-block partial sums; one-block kernels (or, in arn_dots, the
// last block to finish) reduce them in a fixed order
// (repeatable sums), take every control decision on the device and set the
// conditional handles.  No kernel waits on another block, so nothing can spin;
// every loop also has a hard iteration cap that aborts the launch with a status.
//
// Boundary handling: the pass that produces a vector that a stencil will read
// (state, Newton iterate, linearisation copy, Arnoldi vector) also writes an
// "effective" copy on the full (Nx+1)(Ny+1)(Nz+1) grid, indexed like the
// reference's full-grid vectors, with the reference's boundary procedure
// already applied (src/tdgl3d/physics/rhs.py:54-139): normal links zeroed on
// planes 0 and N-1, face values from the adjacent (or, periodic, opposite)
// interior node with the applied-field offsets, edges zero, hole-boundary
// links zero.  Each face value is written by the single interior node it is
// copied from.  The stencils then read every neighbour directly, with no
// branches.
#pragma once

#include "tdgl_common.cuh"

namespace tdgl {

// GS_CAP: a loop ran past its watchdog count; GS_TIMEOUT: a bounded wait of a
// kernel ran out (TMA-staged stencil); GS_IDLE: the launch found its clock at
// t_stop and made no step (a continuation launch; reported as success).
enum GStatus : int {
  GS_OK = 0, GS_NOCONV = 1, GS_DTMIN = 2, GS_KMAX = 3, GS_NONFINITE = 4, GS_CAP = 5, GS_TIMEOUT = 6, GS_IDLE = 7
};

constexpr int kKTypes = 16;   // slots of the per-kernel timers

// Device control block of the graph executor.
constexpr int kPolyMax = 12;  // highest degree of the polynomial preconditioner

struct GDev {
  // inputs for one launch
  double t, dt_cur, t_stop, dt, dt_min, tol_f, tol_dx, tol_gcr, eps_mf;
  double Bx, By, Bz, t_on_fraction, ramp_fraction, t_field_stop;
  int ramp, field_const, newton_max_iter, krylov_max_iter, adaptive, jvp_mode, max_steps;
  // state
  double dta, czxy, cyzx, cxyz;    // current step and its face offsets
  double rho0, rho, xnorm, gnorm, dxnorm, eps;
  double tol_lin;                  // relative residual at which the current Krylov solve stops
  int steps, status, newton_k, newton_failed, accepted, j;
  long long watchdog, watchdog_cap;   // loop iterations of this launch and their hard limit
  unsigned long long wait_ns;         // limit of one bounded wait inside a kernel
  // counters
  long long newton_iters, krylov_iters, krylov_sq, rhs_evals, jvp_evals, rejections;
  int max_krylov, krylov_last;
  int ja;                          // basis vector the next Arnoldi step forms
  int arn_stop;                    // the solve stopped at this Arnoldi step's check: its products are skipped
  // polynomial preconditioner of the analytic-product Krylov solves (set per
  // step from dta): p(lambda) = sum_k poly_e[k] t^k, t = (lambda - theta) / delta
  double poly_e[kPolyMax + 1];
  double poly_theta, poly_delta;
  // per-kernel timers (diagnostics, on when prof_on): first block start to
  // last block end of each launch, summed per kernel type
  int prof_on;
  unsigned long long kt_start[kKTypes], kt_end[kKTypes], kt_total[kKTypes];
  long long kt_count[kKTypes];
};

enum KType : int { KT_PREPARE = 0, KT_PREDICT, KT_NRHS, KT_STENCIL, KT_DOTS, KT_ORTH, KT_UPDATE, KT_ACCEPT, KT_ARN_APPLY, KT_ARN_ORTH, KT_ARN_DOTS };

__device__ __forceinline__ void kt_begin(GDev* d, int k) {
  if (d->prof_on && threadIdx.x == 0) atomicMin(&d->kt_start[k], global_ns());
}
__device__ __forceinline__ void kt_end(GDev* d, int k) {
  if (d->prof_on) {
    __syncthreads();
    if (threadIdx.x == 0) atomicMax(&d->kt_end[k], global_ns());
  }
}
// Fold the last launch of kernel type k into its total (thread 0 of a one-block kernel).
__device__ __forceinline__ void kt_fold(GDev* d, int k) {
  if (d->prof_on && d->kt_end[k] > 0) {
    d->kt_total[k] += d->kt_end[k] - d->kt_start[k];
    d->kt_count[k] += 1;
    d->kt_start[k] = ~0ull;
    d->kt_end[k] = 0;
  }
}

struct TlSched;   // work-item claims of the TMA-staged stencil (tdgl_tl.cuh)

// Forcing term: the relative residual at which the first Krylov solve of a
// step stops at the latest (Eisenstat and Walker's usual starting value).
// Measured with the degree-8 preconditioner, Krylov / Newton iterations and
// steps/s: 128x128x32 film over 20 steps, 1e-3: 117 / 41 / 713.3, 1e-2:
// 117 / 41 / 713.7, 1e-1: 109 / 44 / 738.1; 256x256x64 trilayer, 1e-3:
// 341 / 60 / 45.66, 1e-2: 326 / 60 / 47.44, 1e-1: 314 / 60 / 48.98.
constexpr double kEtaFirst = 1e-1;

template <typename T>
struct GArgs {
  Grid g;
  GDev* dev;
  double* Xn;      // accepted state (raw, device layout)
  double* Xi;      // Newton iterate
  double* G;       // gamma
  double* F;       // f(iterate)
  double* En;      // effective copy of Xn (full grid, FP64)
  double* Ei;      // effective copy of Xi (FP64)
  T* XLe;          // effective linearisation copy in T (aliases Ei for T = double)
  T* VE;           // effective copy of the current Arnoldi vector
  T* V;            // basis: kmax + 1 raw vectors
  T* W;            // A v_j (raw)
  double* part_dots;   // [(kmax + 1) x nblk]
  double* part_orth;   // [nblk]
  double* part_nrhs;   // [3 x nblk]
  double* part_upd;    // [nblk]
  double* kry;         // sj[kmax+1], gam[kmax+1], cj[kmax+1], gv[kmax+1], cs[kmax], sn[kmax], H[(kmax+1) kmax]
  long L;              // ncomp * npad
  long npf;            // full-grid component stride
  int kmax, nblk;
  cudaGraphConditionalHandle h_step, h_newton, h_krylov;
  // two-kernel Arnoldi form (analytic Jacobian products): unnormalised basis U_0..U_kmax
  // and A U_j (ping-pong) on the full grid -- raw values at interior nodes, the
  // boundary procedure's face values (no field offsets) at face nodes, zero at edges
  int fused;
  T* UB;               // (kmax + 1) vectors of vs entries
  T* Zb[2];
  long vs;             // ncomp * npf
  double* part_arn;    // [(kmax + 2) x nblk_arn]
  unsigned* ticket;    // arrival counter of kg_arn_dots (the last block reduces)
  int nblk_arn;        // blocks of kg_arn_dots
  int nblk_orth;       // blocks of kg_arn_orth (<= nblk: its partials go to part_orth)
  int arn_gx, arn_gy;  // grid of kg_arn_apply: (ceil(nx / 32), ceil(ny / 8), nz), 32 x 8 nodes a block
  const uint8_t* imask;   // full grid: 1 at interior nodes
  double cxu, cyu, czu;   // uniform kappa^2 / h^2 (node_coef's values without a per-node kappa)
  int standalone;      // diagnostic launch outside the graph: no bookkeeping, no conditionals
  // product and projections in one kernel (kg_arn_apply_dots): per-tile partials
  // [(kmax + 1) x ntiles] in part_arn, group partials [(kmax + 1) x ngroups]
  int apply_dots;      // 1: kg_arn_apply_dots; 0: kg_arn_apply then kg_arn_dots
  const uint32_t* deadmask;   // per interior node: dead links among the product's neighbour reads
  const uint8_t* ldead;       // per full-grid node: bit a set = its link a reads as zero (normal link on
                              // plane N-1 of axis a, or a hole link); the rule NbM applies
  // adjoint solve (tdgl_adjoint_graph.cuh): linearisation state, right-hand
  // side, solution, J^T v scratch (device layout, L entries each)
  const double* ax;
  const double* ab;
  double* amu;
  double* aT;
  int ntiles, ngroups;
  double* gpart;
  unsigned* gticket;   // [ngroups] arrival counters
  // polynomial right preconditioner of the analytic-product solves: degree
  // (0: none), an upper bound of the spectral radius of J, the Horner buffers
  // (ping-pong), and the preconditioned basis PB_j = p(A) U_j ((kmax + 1)
  // vectors like UB), written by the last Horner step of Arnoldi step j and
  // read by its product; the Newton correction is sum_i c_i PB_i.  pstep is
  // per kernel node (the Horner step).
  int poly_deg;
  double poly_rho;
  T* PW[2];
  T* PB;
  int pstep;
  // TMA-staged stencil: the work-item claim counters (two sets; stencil
  // launches that depend programmatically on one another use alternate sets)
  // and the set of this kernel node (null: each block takes the item of its
  // block index)
  TlSched* tls;
  int tl_par;
  // forcing term of the analytic-product GMRES solves: 1 (the default) = a
  // solve also stops once its residual bounds the Newton test's (tol_lin,
  // krylov_start), 0 = tol_gcr always (the finite-difference GCR form and the
  // adjoint solves)
  int forcing;
};

template <typename T> __host__ __device__ __forceinline__ double* kry_sj(const GArgs<T>& A) { return A.kry; }
template <typename T> __host__ __device__ __forceinline__ double* kry_gam(const GArgs<T>& A) { return A.kry + (A.kmax + 1); }
template <typename T> __host__ __device__ __forceinline__ double* kry_cj(const GArgs<T>& A) { return A.kry + 2 * (A.kmax + 1); }
template <typename T> __host__ __device__ __forceinline__ double* kry_gv(const GArgs<T>& A) { return A.kry + 3 * (A.kmax + 1); }
template <typename T> __host__ __device__ __forceinline__ double* kry_cs(const GArgs<T>& A) { return A.kry + 4 * (A.kmax + 1); }
template <typename T> __host__ __device__ __forceinline__ double* kry_sn(const GArgs<T>& A) { return A.kry + 4 * (A.kmax + 1) + A.kmax; }
template <typename T> __host__ __device__ __forceinline__ double* kry_H(const GArgs<T>& A) { return A.kry + 4 * (A.kmax + 1) + 2 * A.kmax; }
__host__ __device__ __forceinline__ long kry_len(int kmax) { return 4L * (kmax + 1) + 2L * kmax + (long)(kmax + 1) * kmax; }

// ---------------------------------------------------------------------------
// Effective full-grid copies
// ---------------------------------------------------------------------------

// Full-grid accessor of an effective copy (neighbours by direct offsets).
template <typename T, typename S>
struct NbE {
  const S* E; long npf; long m; int mj, mk;
  __device__ __forceinline__ void psi(int di, int dj, int dk, T& re, T& im) const {
    long e = m + di + (long)dj * mj + (long)dk * mk;
    re = (T)E[e];
    im = (T)E[npf + e];
  }
  __device__ __forceinline__ T phi(int a, int di, int dj, int dk) const {
    return (T)E[(2 + a) * npf + m + di + (long)dj * mj + (long)dk * mk];
  }
};
// NbE through the read-only data path (ld.global.nc): for buffers that no
// thread of the launch writes (the Arnoldi product's linearisation copy).
// Neighbour offsets are 32-bit from the node's address (a component block of
// the full grid stays far below 2^31 entries / 4), so each read is one
// address computation from a loop-invariant base.
template <typename T>
struct NbEro {
  const T* __restrict__ E; long npf; long m; int mj, mk;
  __device__ __forceinline__ void psi(int di, int dj, int dk, T& re, T& im) const {
    const T* p = E + m + (di + dj * mj + dk * mk);
    re = __ldg(p);
    im = __ldg(p + (int)npf);
  }
  __device__ __forceinline__ T phi(int a, int di, int dj, int dk) const {
    return __ldg(E + m + ((2 + a) * (int)npf + di + dj * mj + dk * mk));
  }
};
// E1 + s * E2 (finite-difference point x + eps v in effective form: the boundary
// procedure is affine, so its value at x + eps v is E(x) + eps E0(v)).
template <typename S2>
struct NbE2 {
  const double* E1; const S2* E2; double s; long npf; long m; int mj, mk;
  __device__ __forceinline__ void psi(int di, int dj, int dk, double& re, double& im) const {
    long e = m + di + (long)dj * mj + (long)dk * mk;
    re = E1[e] + s * (double)E2[e];
    im = E1[npf + e] + s * (double)E2[npf + e];
  }
  __device__ __forceinline__ double phi(int a, int di, int dj, int dk) const {
    long e = (2 + a) * npf + m + di + (long)dj * mj + (long)dk * mk;
    return E1[e] + s * (double)E2[e];
  }
};

__device__ __forceinline__ long full_index(const Grid& g, int i, int j, int k) {
  return i + (long)g.mj * j + (long)g.mk * k;
}

// Write node (i, j, k)'s effective values and the face values copied from it.
// v: raw values (psi re, psi im, phi x, phi y, phi z); c*: face offsets of the
// applied field (zero for tangent vectors).
// RAW_OWN: the node itself keeps its raw values (dead links included); only
// the face copies get the boundary procedure.
template <typename T, bool D3, bool RAW_OWN = false>
__device__ __forceinline__ void write_eff(const Grid& g, T* E, long npf, int i, int j, int k, const double* v,
                                          double czxy, double cyzx, double cxyz) {
  const long m = full_index(g, i, j, k);
  const uint8_t lf = g.lflags ? g.lflags[m] : 0;
  const double tx = (i == g.Nx - 1) ? 0.0 : v[2];
  const double ty = (j == g.Ny - 1) ? 0.0 : v[3];
  const double tz = (D3 && k == g.Nz - 1) ? 0.0 : (D3 ? v[4] : 0.0);
  E[m] = (T)v[0];
  E[npf + m] = (T)v[1];
  if (RAW_OWN) {
    E[2 * npf + m] = (T)v[2];
    E[3 * npf + m] = (T)v[3];
    if (D3) E[4 * npf + m] = (T)v[4];
  } else {
    E[2 * npf + m] = (lf & LF_HX) ? T(0) : (T)tx;
    E[3 * npf + m] = (lf & LF_HY) ? T(0) : (T)ty;
    if (D3) E[4 * npf + m] = (lf & LF_HZ) ? T(0) : (T)tz;
  }
  auto ghost = [&](long mg, double fx, double fy, double fz) {
    const uint8_t lg = g.lflags ? g.lflags[mg] : 0;
    E[mg] = (T)v[0];
    E[npf + mg] = (T)v[1];
    E[2 * npf + mg] = (lg & LF_HX) ? T(0) : (T)fx;
    E[3 * npf + mg] = (lg & LF_HY) ? T(0) : (T)fy;
    if (D3) E[4 * npf + mg] = (lg & LF_HZ) ? T(0) : (T)fz;
  };
  // x faces (inner j, k)
  if (!g.px) {
    if (i == 1) ghost(m - 1, 0.0, -czxy + ty, cyzx + tz);
    if (i == g.Nx - 1) ghost(m + 1, 0.0, czxy + ty, -cyzx + tz);
  } else {
    if (i == g.Nx - 1) ghost(m - (g.Nx - 1), tx, 0.0, 0.0);
    if (i == 1) ghost(m + (g.Nx - 1), tx, 0.0, 0.0);
  }
  // y faces (inner i, k)
  if (!g.py) {
    if (j == 1) ghost(m - g.mj, czxy + tx, 0.0, -cxyz + tz);
    if (j == g.Ny - 1) ghost(m + g.mj, -czxy + tx, 0.0, cxyz + tz);
  } else {
    if (j == g.Ny - 1) ghost(m - (long)(g.Ny - 1) * g.mj, 0.0, ty, 0.0);
    if (j == 1) ghost(m + (long)(g.Ny - 1) * g.mj, 0.0, ty, 0.0);
  }
  // z faces (inner i, j)
  if (D3) {
    if (!g.pz) {
      if (k == 1) ghost(m - g.mk, -cyzx + tx, cxyz + ty, 0.0);
      if (k == g.Nz - 1) ghost(m + g.mk, cyzx + tx, -cxyz + ty, 0.0);
    } else {
      if (k == g.Nz - 1) ghost(m - (long)(g.Nz - 1) * g.mk, 0.0, 0.0, tz);
      if (k == 1) ghost(m + (long)(g.Nz - 1) * g.mk, 0.0, 0.0, tz);
    }
  }
}

// Full-grid copy in T of a device-layout FP64 vector x: the boundary
// procedure's face values with the given field offsets; RAW: the nodes keep
// their raw values (a Krylov direction), else they get the procedure too (a
// linearisation state).
template <typename T, bool D3, bool RAW>
__global__ void __launch_bounds__(kThreads) kg_to_full(Grid g, const double* __restrict__ x, T* E, long npf,
                                                       double czxy, double cyzx, double cxyz) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.n; n += gridDim.x * blockDim.x) {
    int i, j, k;
    node_ijk(g, n, i, j, k);
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) v[c] = x[(long)c * g.npad + n];
    write_eff<T, D3, RAW>(g, E, npf, i, j, k, v, czxy, cyzx, cxyz);
  }
}

// Interior entries of a full-grid vector in T into a device-layout FP64 vector
// (padding entries written as zero).
template <typename T>
__global__ void __launch_bounds__(kThreads) kg_from_full(Grid g, const T* __restrict__ E, long npf, double* x) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.npad; n += gridDim.x * blockDim.x) {
    long m = 0;
    if (n < g.n) {
      int i, j, k;
      node_ijk(g, n, i, j, k);
      m = full_index(g, i, j, k);
    }
    for (int c = 0; c < g.ncomp; ++c) x[(long)c * g.npad + n] = n < g.n ? (double)E[(long)c * npf + m] : 0.0;
  }
}

// ---------------------------------------------------------------------------
// Reduction helpers
// ---------------------------------------------------------------------------

// Block-reduce NV values (sum or max) and write them to part[s * nblk + block].
template <int NV>
__device__ __forceinline__ void block_partials(double (&v)[NV], const bool (&is_max)[NV], double* part, int nblk) {
  __shared__ double red[kWarps][NV > 0 ? NV : 1];
#pragma unroll
  for (int s = 0; s < NV; ++s) {
    v[s] = is_max[s] ? warp_max(v[s]) : warp_sum(v[s]);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][s] = v[s];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    int s = threadIdx.x;
    double a = 0.0;
    for (int w = 0; w < kWarps; ++w) a = is_max[s] ? fmax(a, red[w][s]) : a + red[w][s];
    part[(long)s * nblk + blockIdx.x] = a;
  }
}

// One-block reduction of part[s * nblk + b] over b for s < ns (fixed order).
__device__ __forceinline__ void reduce_parts(const double* part, int nblk, int ns, bool is_max, double* out_smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int s = warp; s < ns; s += kWarps) {
    double a = 0.0;
    for (int b = lane; b < nblk; b += 32) {
      double x = part[(long)s * nblk + b];
      a = is_max ? fmax(a, x) : a + x;
    }
    a = is_max ? warp_max(a) : warp_sum(a);
    if (lane == 0) out_smem[s] = a;
  }
  __syncthreads();
}

__device__ __forceinline__ double gfinite(double v) { return isfinite(v) ? v : INFINITY; }

__device__ __forceinline__ bool gdev_ok(const GDev* d) { return d->status == GS_OK; }

// Programmatic dependent launch.  grid_dep_wait: wait until the kernels this
// launch depends on have completed and their writes are visible (returns at
// once for a launch without a programmatic dependency).  grid_dep_launch: let
// the next kernel, when its launch depends on this one programmatically,
// start its part before its own grid_dep_wait; a kernel calls it only after
// its own grid_dep_wait, so that every kernel before it has completed when the
// next one starts.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Stop every loop of the graph with a status (one-block kernels only).
template <typename T>
__device__ __forceinline__ void abort_all(const GArgs<T>& A, int status) {
  if (threadIdx.x == 0) {
    if (A.dev->status == GS_OK) A.dev->status = status;
    if (A.standalone) return;      // a launch outside the graph has no conditional nodes to stop
    cudaGraphSetConditional(A.h_krylov, 0);
    cudaGraphSetConditional(A.h_newton, 0);
    cudaGraphSetConditional(A.h_step, 0);
  }
}

// Arnoldi / Krylov initialisation after a Newton residual (thread 0).
template <typename T>
__device__ __forceinline__ bool krylov_start(const GArgs<T>& A, GDev* d) {
  d->j = 0;
  d->ja = 0;
  d->arn_stop = 0;
  d->rho = d->rho0;
  kry_gv(A)[0] = d->rho0;
  kry_sj(A)[0] = d->rho0 > 0.0 ? 1.0 / d->rho0 : 0.0;
  d->eps = d->eps_mf * (1.0 + d->xnorm);       // eps_mf (1 + |x|) / |v|, |v| = 1 (tgcr.py:129)
  // The solve's stopping tolerance.  The reference's is tol_gcr relative to
  // ||r0||_2.  With the forcing term a solve also stops once its residual is
  // below 0.1 tol_f in the 2-norm, which bounds the max norm the Newton test
  // uses (||r||_inf <= ||r||_2): the last Newton iteration of a step is not
  // solved far past what the test accepts.  The first solve of a step stops
  // at kEtaFirst relative at the latest: the Newton iteration after it, which
  // the test's quadratic term requires anyway, corrects what it leaves.  The
  // test itself is unchanged.
  d->tol_lin = d->tol_gcr;
  if (A.forcing && d->rho0 > 0.0) {
    double eta = fmax(d->tol_gcr, 0.1 * d->tol_f / d->rho0);
    if (d->newton_k == 1) eta = fmax(eta, kEtaFirst);
    d->tol_lin = fmin(0.5, eta);
  }
  return d->rho0 > 0.0 && d->rho / d->rho0 > d->tol_lin && d->krylov_max_iter > 0;
}

// ---------------------------------------------------------------------------
// Grid kernels
// ---------------------------------------------------------------------------

// Effective copy of the accepted state with this step's field.
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads) kg_prepare(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  kt_begin(A.dev, KT_PREPARE);
  const Grid& g = A.g;
  const double czxy = d->czxy, cyzx = d->cyzx, cxyz = d->cxyz;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.n; n += gridDim.x * blockDim.x) {
    int i, j, k;
    node_ijk(g, n, i, j, k);
    double v[5];
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) v[c] = A.Xn[(long)c * g.npad + n];
    write_eff<double, D3>(g, A.En, A.npf, i, j, k, v, czxy, cyzx, cxyz);
  }
  kt_end(A.dev, KT_PREPARE);
}

// Tiles of the interior (3-D grids): 32 x 8 nodes of one plane, planes
// 1 .. nz, so that the grid kernels take node coordinates from the tile with
// no division per node.  Index q = tile * kThreads + thread in the tile.
struct EffTiles {
  int gx, gxy, n;
  __device__ __forceinline__ explicit EffTiles(const Grid& g)
      : gx((g.nx + 31) / 32), gxy(((g.nx + 31) / 32) * ((g.ny + 7) / 8)), n(gxy * g.nz) {}
  // node of index q: false past the grid's last column or row
  __device__ __forceinline__ bool node(const Grid& g, int q, int& i, int& j, int& k) const {
    const int t = q / kThreads, l = q - t * kThreads;
    const int z = t / gxy, r = t - z * gxy;
    const int ty = r / gx;
    k = 1 + z;
    j = 1 + 8 * ty + (l >> 5);
    i = 1 + 32 * (r - ty * gx) + (l & 31);
    return i <= g.nx && j <= g.ny;
  }
};

// node_coef<double> with the uniform kappa^2 / h^2 of the launch (no division
// per node unless kappa varies per node).
template <typename T>
__device__ __forceinline__ NodeCoef<double> node_coef_u(const GArgs<T>& A, const Grid& g, int n, uint8_t nf) {
  if (g.kappa_per_node) return node_coef<double>(g, n, nf);
  NodeCoef<double> nc;
  nc.cx = A.cxu;
  nc.cy = A.cyu;
  nc.cz = A.czu;
  nc.material = g.has_material != 0;
  if (!nc.material) nc.sc = 1.0;
  else if (nf & NF_SCFRAC) nc.sc = g.scint[n];
  else nc.sc = (nf & NF_SC0) ? 0.0 : 1.0;
  set_ih(g, nc);
  return nc;
}

// Predictor: f = rhs(Xn); Xi = Xn + dt f; G = Xn + dt/2 f (integrators.py:156-158);
// effective copies of Xi (FP64, and in T for the Jacobian products).
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads, 3) kg_predict(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  kt_begin(A.dev, KT_PREDICT);
  const Grid& g = A.g;
  const double dt = d->dta, czxy = d->czxy, cyzx = d->cyzx, cxyz = d->cxyz;
  auto node = [&](int n, int i, int j, int k, const double o[5]) {
    double xi[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) {
      long e = (long)c * g.npad + n;
      double xv = A.Xn[e];
      xi[c] = xv + dt * o[c];
      A.Xi[e] = xi[c];
      A.G[e] = xv + (dt / 2.0) * o[c];
    }
    write_eff<double, D3>(g, A.Ei, A.npf, i, j, k, xi, czxy, cyzx, cxyz);
    if ((void*)A.XLe != (void*)A.Ei) write_eff<T, D3>(g, A.XLe, A.npf, i, j, k, xi, czxy, cyzx, cxyz);
  };
  const EffTiles tl(g);
  const int nt = D3 ? tl.n * kThreads : g.n;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nt; q += gridDim.x * blockDim.x) {
    int i, j, k, n;
    if constexpr (D3) {
      if (!tl.node(g, q, i, j, k)) continue;
      n = dix(g, i, j, k);
    } else {
      n = q;
      node_ijk(g, n, i, j, k);
    }
    const uint8_t nf = g.nflags[n];
    const NodeCoef<double> nc = node_coef_u(A, g, n, nf);
    const NbEro<double> X{A.En, A.npf, full_index(g, i, j, k), g.mj, g.mk};   // En: read only in this kernel
    double o[5];
    rhs_body<double, D3>(g, X, nc, nf, o);
    node(n, i, j, k, o);
  }
  kt_end(A.dev, KT_PREDICT);
}

// Newton residual: f = rhs(Xi) into F; g = Xi - dt/2 f - G; r0 = -g into the
// first basis vector (raw) and its effective copy.  Partials: ||r0||^2, ||x||^2, max|g|.
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads, 3) kg_newton_rhs(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d) || d->newton_failed) return;
  kt_begin(A.dev, KT_NRHS);
  const Grid& g = A.g;
  const double dt = d->dta;
  double acc[3] = {0.0, 0.0, 0.0};
  auto node = [&](int n, int i, int j, int k, const double o[5]) {
    double gv[5] = {0, 0, 0, 0, 0}, r[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) {
      long e = (long)c * g.npad + n;
      double xv = A.Xi[e];
      A.F[e] = o[c];
      gv[c] = xv - (dt / 2.0) * o[c] - A.G[e];
      T rt = (T)(-gv[c]);
      if (!A.fused) A.V[e] = rt;
      r[c] = (double)rt;
      acc[0] += r[c] * r[c];
      acc[1] += xv * xv;
    }
    double m = gfinite(hypot(gv[0], gv[1]));
#pragma unroll
    for (int c = 2; c < (D3 ? 5 : 4); ++c) m = fmax(m, gfinite(fabs(gv[c])));
    acc[2] = fmax(acc[2], m);
    if (A.fused) write_eff<T, D3, true>(g, A.UB, A.npf, i, j, k, r, 0.0, 0.0, 0.0);
    else write_eff<T, D3>(g, A.VE, A.npf, i, j, k, r, 0.0, 0.0, 0.0);
  };
  const EffTiles tl(g);
  const int nt = D3 ? tl.n * kThreads : g.n;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nt; q += gridDim.x * blockDim.x) {
    int i, j, k, n;
    if constexpr (D3) {
      if (!tl.node(g, q, i, j, k)) continue;
      n = dix(g, i, j, k);
    } else {
      n = q;
      node_ijk(g, n, i, j, k);
    }
    const uint8_t nf = g.nflags[n];
    const NodeCoef<double> nc = node_coef_u(A, g, n, nf);
    const NbEro<double> X{A.Ei, A.npf, full_index(g, i, j, k), g.mj, g.mk};   // Ei: read only in this kernel
    double o[5];
    rhs_body<double, D3>(g, X, nc, nf, o);
    node(n, i, j, k, o);
  }
  const bool mx[3] = {false, false, true};
  block_partials<3>(acc, mx, A.part_nrhs, A.nblk);
  kt_end(A.dev, KT_NRHS);
}

// Arnoldi stencil: W = A v_j, v_j = s_j v~_j (basis slot j-1, effective copy VE).
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads) kg_stencil(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  kt_begin(A.dev, KT_STENCIL);
  const Grid& g = A.g;
  const int jc = d->j + 1;
  const double sj = kry_sj(A)[jc - 1];
  const double dth = d->dta / 2.0, eps = d->eps;
  const T* Vj = A.V + (long)(jc - 1) * A.L;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.n; n += gridDim.x * blockDim.x) {
    int i, j, k;
    node_ijk(g, n, i, j, k);
    const uint8_t nf = g.nflags[n];
    const long m = full_index(g, i, j, k);
    double w[5];
    if (d->jvp_mode == JVP_FD) {
      NodeCoef<double> nc = node_coef<double>(g, n, nf);
      NbE2<T> X{A.Ei, A.VE, eps * sj, A.npf, m, g.mj, g.mk};
      double o[5];
      rhs_body<double, D3>(g, X, nc, nf, o);
#pragma unroll
      for (int c = 0; c < (D3 ? 5 : 4); ++c) {
        long e = (long)c * g.npad + n;
        w[c] = sj * (double)Vj[e] - dth * ((o[c] - A.F[e]) / eps);
      }
    } else {
      NodeCoef<T> nc = node_coef<T>(g, n, nf);
      NbE<T, T> X{A.XLe, A.npf, m, g.mj, g.mk};
      NbE<T, T> P{A.VE, A.npf, m, g.mj, g.mk};
      T o[5];
      jvp_body<T, D3>(g, X, P, nc, nf, o);
#pragma unroll
      for (int c = 0; c < (D3 ? 5 : 4); ++c) w[c] = sj * ((double)Vj[(long)c * g.npad + n] - dth * (double)o[c]);
    }
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) A.W[(long)c * g.npad + n] = (T)w[c];
  }
  kt_end(A.dev, KT_STENCIL);
}

template <typename T> struct GGroup { static constexpr int JB = 8; };
template <> struct GGroup<double> { static constexpr int JB = 4; };

template <typename T> struct V4 { T a, b, c, d; };
// Sum over the 32 lanes of a warp in T (butterfly: every lane gets the sum).
template <typename T>
__device__ __forceinline__ T warp_sum_t(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ V4<float> ld4(const float* p) {
  float4 v = *reinterpret_cast<const float4*>(p);
  return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ V4<double> ld4(const double* p) {
  double2 u = reinterpret_cast<const double2*>(p)[0], v = reinterpret_cast<const double2*>(p)[1];
  return {u.x, u.y, v.x, v.y};
}
// The same through L2 only (read once by this kernel: keeps L1 for re-read data).
__device__ __forceinline__ V4<float> ld4cg(const float* p) {
  const float4 v = __ldcg(reinterpret_cast<const float4*>(p));
  return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ V4<double> ld4cg(const double* p) {
  const double2 u = __ldcg(reinterpret_cast<const double2*>(p)), v = __ldcg(reinterpret_cast<const double2*>(p) + 1);
  return {u.x, u.y, v.x, v.y};
}
__device__ __forceinline__ void st4(float* p, const double* v) {
  *reinterpret_cast<float4*>(p) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
}
__device__ __forceinline__ void st4(double* p, const double* v) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

// Projections <W, v~_i> for i < j (partials per block, one slot per i).
template <typename T>
__global__ void __launch_bounds__(kThreads) kg_dots(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  kt_begin(A.dev, KT_DOTS);
  constexpr int JB = GGroup<T>::JB;
  __shared__ double red[kWarps][JB];
  const int jc = d->j + 1;
  const long nq = A.L / 4;
  for (int i0 = 0; i0 < jc; i0 += JB) {
    double acc[JB];
#pragma unroll
    for (int t = 0; t < JB; ++t) acc[t] = 0.0;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nq; q += (long)gridDim.x * blockDim.x) {
      V4<T> w = ld4(A.W + 4 * q);
      V4<T> a[JB];
#pragma unroll
      for (int t = 0; t < JB; ++t) a[t] = (i0 + t < jc) ? ld4(A.V + (long)(i0 + t) * A.L + 4 * q) : V4<T>{0, 0, 0, 0};
#pragma unroll
      for (int t = 0; t < JB; ++t)
        acc[t] += (double)w.a * (double)a[t].a + (double)w.b * (double)a[t].b + (double)w.c * (double)a[t].c +
                  (double)w.d * (double)a[t].d;
    }
#pragma unroll
    for (int t = 0; t < JB; ++t) {
      double v = warp_sum(acc[t]);
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][t] = v;
    }
    __syncthreads();
    if (threadIdx.x < JB && i0 + (int)threadIdx.x < jc) {
      double s = 0.0;
      for (int w = 0; w < kWarps; ++w) s += red[w][threadIdx.x];
      A.part_dots[(long)(i0 + threadIdx.x) * A.nblk + blockIdx.x] = s;
    }
    __syncthreads();
  }
  kt_end(A.dev, KT_DOTS);
}

// Orthogonalisation: v~_{j+1} = W - sum_{i<j} gam_i v~_i (raw, slot j) and its
// effective copy; partial ||v~_{j+1}||^2.  Lane work: four consecutive nodes.
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads) kg_orth(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  kt_begin(A.dev, KT_ORTH);
  constexpr int JB = GGroup<T>::JB;
  constexpr int NC = D3 ? 5 : 4;
  const Grid& g = A.g;
  const int jc = d->j + 1;
  const double* gam = kry_gam(A);
  T* Vn = A.V + (long)jc * A.L;
  double acc[1] = {0.0};
  const long nq = g.npad / 4;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nq; q += (long)gridDim.x * blockDim.x) {
    const long base = 4 * q;
    double val[NC][4];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const long e = (long)c * g.npad + base;
      V4<T> w = ld4(A.W + e);
      double v[4] = {(double)w.a, (double)w.b, (double)w.c, (double)w.d};
      for (int i0 = 0; i0 < jc; i0 += JB) {
        V4<T> a[JB];
#pragma unroll
        for (int t = 0; t < JB; ++t) a[t] = (i0 + t < jc) ? ld4(A.V + (long)(i0 + t) * A.L + e) : V4<T>{0, 0, 0, 0};
#pragma unroll
        for (int t = 0; t < JB; ++t) {
          double gm = (i0 + t < jc) ? gam[i0 + t] : 0.0;
          v[0] -= gm * (double)a[t].a; v[1] -= gm * (double)a[t].b;
          v[2] -= gm * (double)a[t].c; v[3] -= gm * (double)a[t].d;
        }
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        v[t] = (double)(T)v[t];
        val[c][t] = v[t];
        acc[0] += v[t] * v[t];
      }
      st4(Vn + e, v);
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      int n = (int)(base + t);
      if (n >= g.n) break;
      int i, j, k;
      node_ijk(g, n, i, j, k);
      double v[5];
#pragma unroll
      for (int c = 0; c < NC; ++c) v[c] = val[c][t];
      write_eff<T, D3>(g, A.VE, A.npf, i, j, k, v, 0.0, 0.0, 0.0);
    }
  }
  const bool mx[1] = {false};
  block_partials<1>(acc, mx, A.part_orth, A.nblk);
  kt_end(A.dev, KT_ORTH);
}

// Newton update: x += sum_i cj_i v~_i (raw FP64), effective copies of the new
// iterate; partial max|dx| (complex modulus on psi).
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads) kg_update(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d) || d->newton_failed) return;
  kt_begin(A.dev, KT_UPDATE);
  constexpr int JB = GGroup<T>::JB;
  constexpr int NC = D3 ? 5 : 4;
  const Grid& g = A.g;
  const int nk = d->j;
  const double* cj = kry_cj(A);
  const double czxy = d->czxy, cyzx = d->cyzx, cxyz = d->cxyz;
  double acc[1] = {0.0};
  const long nq = g.npad / 4;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nq; q += (long)gridDim.x * blockDim.x) {
    const long base = 4 * q;
    double xn[NC][4], dx[NC][4];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const long e = (long)c * g.npad + base;
      double s[4] = {0, 0, 0, 0};
      for (int i0 = 0; i0 < nk; i0 += JB) {
        V4<T> a[JB];
#pragma unroll
        for (int t = 0; t < JB; ++t) a[t] = (i0 + t < nk) ? ld4(A.V + (long)(i0 + t) * A.L + e) : V4<T>{0, 0, 0, 0};
#pragma unroll
        for (int t = 0; t < JB; ++t) {
          double cc = (i0 + t < nk) ? cj[i0 + t] : 0.0;
          s[0] += cc * (double)a[t].a; s[1] += cc * (double)a[t].b;
          s[2] += cc * (double)a[t].c; s[3] += cc * (double)a[t].d;
        }
      }
      V4<double> x = ld4(A.Xi + e);
      double nx4[4] = {x.a + s[0], x.b + s[1], x.c + s[2], x.d + s[3]};
      st4(A.Xi + e, nx4);
#pragma unroll
      for (int t = 0; t < 4; ++t) { xn[c][t] = nx4[t]; dx[c][t] = s[t]; }
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      int n = (int)(base + t);
      if (n >= g.n) break;
      double m = gfinite(hypot(dx[0][t], dx[1][t]));
#pragma unroll
      for (int c = 2; c < NC; ++c) m = fmax(m, gfinite(fabs(dx[c][t])));
      acc[0] = fmax(acc[0], m);
      int i, j, k;
      node_ijk(g, n, i, j, k);
      double v[5];
#pragma unroll
      for (int c = 0; c < NC; ++c) v[c] = xn[c][t];
      write_eff<double, D3>(g, A.Ei, A.npf, i, j, k, v, czxy, cyzx, cxyz);
      if ((void*)A.XLe != (void*)A.Ei) write_eff<T, D3>(g, A.XLe, A.npf, i, j, k, v, czxy, cyzx, cxyz);
    }
  }
  const bool mx[1] = {true};
  block_partials<1>(acc, mx, A.part_upd, A.nblk);
  kt_end(A.dev, KT_UPDATE);
}

// Newton update of the analytic-product graph (basis on the full grid), one
// node per thread: x += sum c_i U_i, the update's max-norm partials and the
// effective copies.  Kept apart from kg_update so that it is not held to
// that kernel's register budget (one block per SM).
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads, 3) kg_update_fused(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d) || d->newton_failed) return;
  kt_begin(A.dev, KT_UPDATE);
  constexpr int NC = D3 ? 5 : 4;
  const Grid& g = A.g;
  // with the polynomial preconditioner the correction is p(A) sum_i c_i U_i
  // = sum_i c_i PB_i (PB_i = p(A) U_i, kept by the Arnoldi steps)
  const int nk = d->j;
  const double* cj = kry_cj(A);
  const T* UBase = A.poly_deg > 0 ? A.PB : A.UB;
  const double czxy = d->czxy, cyzx = d->cyzx, cxyz = d->cxyz;
  double acc[1] = {0.0};
  // basis on the full grid: one node per thread (3-D: tiles of 32 x 8 nodes
  // of one plane, no division per node)
  const EffTiles tl(g);
  const int nt = D3 ? tl.n * kThreads : g.n;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nt; q += gridDim.x * blockDim.x) {
    int i, j, k, n;
    if constexpr (D3) {
      if (!tl.node(g, q, i, j, k)) continue;
      n = dix(g, i, j, k);
    } else {
      n = q;
      node_ijk(g, n, i, j, k);
    }
    const long m = full_index(g, i, j, k);
    double s[NC], v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int c = 0; c < NC; ++c) s[c] = 0.0;
    int i0 = 0;
    // the basis is read only in this kernel: read-only loads
    for (; i0 + 4 <= nk; i0 += 4) {
      const T* U = UBase + (long)i0 * A.vs + m;
      const double c0 = cj[i0], c1 = cj[i0 + 1], c2 = cj[i0 + 2], c3 = cj[i0 + 3];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const long e = (long)c * A.npf;
        s[c] += c0 * (double)__ldg(U + e) + c1 * (double)__ldg(U + A.vs + e) + c2 * (double)__ldg(U + 2 * A.vs + e) +
                c3 * (double)__ldg(U + 3 * A.vs + e);
      }
    }
    for (; i0 < nk; ++i0) {
      const T* U = UBase + (long)i0 * A.vs + m;
#pragma unroll
      for (int c = 0; c < NC; ++c) s[c] += cj[i0] * (double)__ldg(U + (long)c * A.npf);
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const long e = (long)c * g.npad + n;
      v[c] = A.Xi[e] + s[c];
      A.Xi[e] = v[c];
    }
    double mm = gfinite(hypot(s[0], s[1]));
#pragma unroll
    for (int c = 2; c < NC; ++c) mm = fmax(mm, gfinite(fabs(s[c])));
    acc[0] = fmax(acc[0], mm);
    write_eff<double, D3>(g, A.Ei, A.npf, i, j, k, v, czxy, cyzx, cxyz);
    if ((void*)A.XLe != (void*)A.Ei) write_eff<T, D3>(g, A.XLe, A.npf, i, j, k, v, czxy, cyzx, cxyz);
  }
  const bool mx[1] = {true};
  block_partials<1>(acc, mx, A.part_upd, A.nblk);
  kt_end(A.dev, KT_UPDATE);
}

// Accepted step: Xn = Xi.
template <typename T>
__global__ void __launch_bounds__(kThreads) kg_accept(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d) || !d->accepted) return;
  kt_begin(A.dev, KT_ACCEPT);
  const long nq = A.L / 2;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nq; q += (long)gridDim.x * blockDim.x)
    reinterpret_cast<double2*>(A.Xn)[q] = reinterpret_cast<const double2*>(A.Xi)[q];
  kt_end(A.dev, KT_ACCEPT);
}

// ---------------------------------------------------------------------------
// Arnoldi step (analytic Jacobian products)
// ---------------------------------------------------------------------------
//
// Step ja of a Krylov solve runs
//   kg_arn_orth   U_ja = s_{ja-1} (Z_{ja-1} - sum_{i<ja} gam_i U_i)   (nothing for ja = 0:
//                 U_0 = r0, written by the Newton residual)
//   kg_arn_apply  Z_ja = U_ja - dt/2 J(x) U_ja  (A U_ja; the tangent-linear product is
//                 linear)
//   kg_arn_dots   <Z_ja, U_i> (i <= ja) over the interior entries (||U_ja||^2 comes
//                 with the orthogonalisation; kg_arn_check, between the
//                 orthogonalisation and the product, completes column ja - 1
//                 from it and stops the solve before the products when it
//                 has converged).
// The basis stays unnormalised (v_i = s_i U_i, s_i = 1 / ||U_i||): with
// gam_i = s_i^2 <Z_{ja-1}, U_i>, U_ja is the classical Gram-Schmidt remainder of
// A v_{ja-1}, so ||U_ja|| = h_{ja,ja-1} stays of the order of ||A|| (without the
// factor s_{ja-1} the norms would multiply from one vector to the next and
// leave the FP32 range within a few dozen iterations of a stiff system).
// The partials are added in a fixed order (the last block of each group of 32
// blocks sums its group, the last group sums the groups), and that last block
// stores column ja and the next coefficients.  Column ja-1 (norm, Givens
// rotation, residual estimate and the stop test of tgcr.py:125, 141-142) is
// completed earlier in the step, by kg_arn_check right after the
// orthogonalisation: a solve of m iterations stops in the check of step m,
// before that step's polynomial steps, product and projections, which then
// return at once.
//
// The vectors live on the full grid with their face values, and the boundary
// procedure is linear for directions, so kg_arn_orth combines every entry
// (faces, edges, padding) without looking at positions.  kg_arn_apply reads
// the raw values and zeroes the dead links of the stencil's neighbours (normal
// links on plane N-1, hole links) on the fly.

// Completion of Hessenberg column ja - 1 at Arnoldi step ja > 0, from
// un2 = ||U_ja||^2 (thread 0 of kg_arn_check, before the step's products):
// h_{ja, ja-1} = ||U_ja||, the Givens rotation, the residual estimate and the
// stop test of tgcr.py:125, 141-142.  When the solve stops here the Krylov
// loop ends and the step's products are marked skipped (arn_stop).
template <typename T>
__device__ void arn_complete(const GArgs<T>& A, GDev* d, int ja, double un2) {
  if (!isfinite(un2)) { abort_all(A, GS_NONFINITE); return; }
  double* sj = kry_sj(A);
  const int jc = ja;                                   // columns complete after this step
  double* gv = kry_gv(A);
  double* cs = kry_cs(A);
  double* sn = kry_sn(A);
  double* col = kry_H(A) + (long)(jc - 1) * (A.kmax + 1);
  const double un = sqrt(un2);
  const double hn = un;                                // h_{jc, jc-1} = ||A v - sum h v|| = ||U_jc||
  sj[jc] = un > 0.0 ? 1.0 / un : 0.0;
  d->jvp_evals += 1 + A.poly_deg;
  col[jc] = hn;
  for (int i = 0; i + 1 < jc; ++i) {
    double a = col[i], b = col[i + 1];
    col[i] = cs[i] * a + sn[i] * b;
    col[i + 1] = -sn[i] * a + cs[i] * b;
  }
  double a = col[jc - 1], b = col[jc];
  double r = hypot(a, b);
  double c = r > 0.0 ? a / r : 1.0, sv = r > 0.0 ? b / r : 0.0;
  cs[jc - 1] = c;
  sn[jc - 1] = sv;
  col[jc - 1] = r;
  col[jc] = 0.0;
  gv[jc] = -sv * gv[jc - 1];
  gv[jc - 1] = c * gv[jc - 1];
  d->rho = fabs(gv[jc]);
  d->j = jc;
  bool cont = hn > 0.0 && d->rho / d->rho0 > d->tol_lin && jc < d->krylov_max_iter;
  if (cont && jc + 1 > A.kmax) { abort_all(A, GS_KMAX); return; }
  if (!cont) {
    d->arn_stop = 1;
    cudaGraphSetConditional(A.h_krylov, 0);
  }
}

// Column bookkeeping of launch ja (thread 0 of the last block), after
// kg_arn_check has completed column ja - 1: S[i] = <Z_ja, U_i> gives column
// ja's projections and the next orthogonalisation coefficients.
template <typename T>
__device__ void arn_finish(const GArgs<T>& A, GDev* d, int ja, const double* S) {
  if (++d->watchdog > d->watchdog_cap) { abort_all(A, GS_CAP); return; }
  double* sj = kry_sj(A);
  double* gam = kry_gam(A);
  for (int i = 0; i <= ja; ++i)
    if (!isfinite(S[i])) { abort_all(A, GS_NONFINITE); return; }
  double* colj = kry_H(A) + (long)ja * (A.kmax + 1);
  for (int i = 0; i <= ja; ++i) {
    colj[i] = sj[ja] * sj[i] * S[i];
    gam[i] = sj[i] * sj[i] * S[i];
  }
  d->ja = ja + 1;
  cudaGraphSetConditional(A.h_krylov, 1);
}



// Neighbourhood of a direction vector stored raw at interior nodes: the
// stencil sees the normal link zeroed on plane N-1 of its axis and hole links
// zeroed.  Face entries already hold the boundary procedure's values, which
// satisfy the same rules.
template <typename T>
struct NbM {
  const T* E; long npf; long m; int mj, mk; int i, j, k; const Grid* g; const uint8_t* lflags;
  __device__ __forceinline__ void psi(int di, int dj, int dk, T& re, T& im) const {
    long e = m + di + (long)dj * mj + (long)dk * mk;
    re = E[e];
    im = E[npf + e];
  }
  // branch-free: both loads are issued before the select
  __device__ __forceinline__ T phi(int a, int di, int dj, int dk) const {
    const long e = m + di + (long)dj * mj + (long)dk * mk;
    const T v = E[(2 + a) * npf + e];
    const unsigned lf = lflags ? (unsigned)lflags[e] : 0u;
    const bool dead = (a == 0 && i + di == g->Nx - 1) || (a == 1 && j + dj == g->Ny - 1) ||
                      (a == 2 && k + dk == g->Nz - 1) || ((lf >> a) & 1u);
    return dead ? T(0) : v;
  }
};

// The 27 neighbour links (axis a, offset di, dj, dk) that the tangent-linear
// stencil reads from a direction vector; bit b of a node's dead-link mask says
// whether link dead_link(b, .) is dead (normal link on plane N-1 of its axis,
// or a hole link), the rule NbM applies on the fly.
__host__ __device__ constexpr int dead_link(int b, int c) {
  constexpr int t[27][4] = {
      {0, 0, 0, 0}, {0, -1, 0, 0}, {0, 1, 0, 0}, {0, 0, -1, 0}, {0, 0, 1, 0}, {0, -1, 1, 0}, {0, 0, 0, -1},
      {0, 0, 0, 1}, {0, -1, 0, 1}, {1, 0, 0, 0}, {1, 0, -1, 0}, {1, -1, 0, 0}, {1, 1, 0, 0}, {1, 0, 1, 0},
      {1, 1, -1, 0}, {1, 0, 0, -1}, {1, 0, 0, 1}, {1, 0, -1, 1}, {2, 0, 0, 0}, {2, 0, 0, -1}, {2, -1, 0, 0},
      {2, 1, 0, 0}, {2, 0, -1, 0}, {2, 0, 1, 0}, {2, 0, 0, 1}, {2, 1, 0, -1}, {2, 0, 1, -1}};
  return t[b][c];
}

__host__ __device__ constexpr int dead_bit(int a, int di, int dj, int dk) {
  for (int b = 0; b < 27; ++b)
    if (dead_link(b, 0) == a && dead_link(b, 1) == di && dead_link(b, 2) == dj && dead_link(b, 3) == dk) return b;
  return -1;
}

// NbM with the node's precomputed dead-link mask: one load per node instead
// of a link-flag load and plane tests per neighbour read.  The direction is
// read-only during the product, so its loads take the read-only data path.
template <typename T>
struct NbMk {
  const T* __restrict__ E; long npf; long m; int mj, mk; uint32_t dm; NbM<T> slow;
  __device__ __forceinline__ void psi(int di, int dj, int dk, T& re, T& im) const {
    const T* p = E + m + (di + dj * mj + dk * mk);
    re = __ldg(p);
    im = __ldg(p + (int)npf);
  }
  __device__ __forceinline__ T phi(int a, int di, int dj, int dk) const {
    const int b = dead_bit(a, di, dj, dk);
    if (b < 0) return slow.phi(a, di, dj, dk);
    const T v = __ldg(E + m + ((2 + a) * (int)npf + di + dj * mj + dk * mk));
    return ((dm >> b) & 1u) ? T(0) : v;
  }
};

template <typename T>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 4 : 3) kg_arn_orth(GArgs<T> A) {
  GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  const int ja = d->ja;
  if (ja == 0) return;
  kt_begin(d, KT_ARN_ORTH);
  extern __shared__ double gsm[];              // s_{ja-1} gam_0 .. s_{ja-1} gam_{ja-1}
  const double sc = kry_sj(A)[ja - 1];
  for (int t = threadIdx.x; t < ja; t += blockDim.x) gsm[t] = sc * kry_gam(A)[t];
  __syncthreads();
  const T* Zin = A.Zb[(ja + 1) & 1];
  T* Uj = A.UB + (long)ja * A.vs;
  const long vs = A.vs, npf = A.npf, nq = vs / 4;
  const long stride = (long)gridDim.x * blockDim.x;
  long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  long mo = (4 * q) % npf;                     // offset within the component (interior mask)
  double nrm = 0.0;
  for (; q < nq; q += stride) {
    const long e = 4 * q;
    const V4<T> z = ld4(Zin + e);
    double v[4] = {sc * (double)z.a, sc * (double)z.b, sc * (double)z.c, sc * (double)z.d};
    const T* U = A.UB + e;
    int i = 0;
    for (; i + 8 <= ja; i += 8) {                // eight vectors' loads in flight together
      V4<T> a[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) a[t] = ld4(U + (long)(i + t) * vs);
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const double gt = gsm[i + t];
        v[0] -= gt * (double)a[t].a;
        v[1] -= gt * (double)a[t].b;
        v[2] -= gt * (double)a[t].c;
        v[3] -= gt * (double)a[t].d;
      }
    }
    for (; i + 4 <= ja; i += 4) {
      const V4<T> a0 = ld4(U + (long)i * vs), a1 = ld4(U + (long)(i + 1) * vs);
      const V4<T> a2 = ld4(U + (long)(i + 2) * vs), a3 = ld4(U + (long)(i + 3) * vs);
      const double g0 = gsm[i], g1 = gsm[i + 1], g2 = gsm[i + 2], g3 = gsm[i + 3];
      v[0] -= g0 * (double)a0.a + g1 * (double)a1.a + g2 * (double)a2.a + g3 * (double)a3.a;
      v[1] -= g0 * (double)a0.b + g1 * (double)a1.b + g2 * (double)a2.b + g3 * (double)a3.b;
      v[2] -= g0 * (double)a0.c + g1 * (double)a1.c + g2 * (double)a2.c + g3 * (double)a3.c;
      v[3] -= g0 * (double)a0.d + g1 * (double)a1.d + g2 * (double)a2.d + g3 * (double)a3.d;
    }
    for (; i < ja; ++i) {
      const V4<T> a = ld4(U + (long)i * vs);
      const double g = gsm[i];
      v[0] -= g * (double)a.a; v[1] -= g * (double)a.b; v[2] -= g * (double)a.c; v[3] -= g * (double)a.d;
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) v[t] = (double)(T)v[t];
    st4(Uj + e, v);
    const uchar4 mk = *reinterpret_cast<const uchar4*>(A.imask + mo);
    nrm += (mk.x ? v[0] * v[0] : 0.0) + (mk.y ? v[1] * v[1] : 0.0) + (mk.z ? v[2] * v[2] : 0.0) +
           (mk.w ? v[3] * v[3] : 0.0);
    mo += 4 * stride;
    while (mo >= npf) mo -= npf;
  }
  double acc[1] = {nrm};
  const bool mx[1] = {false};
  block_partials<1>(acc, mx, A.part_orth, A.nblk_orth);
  kt_end(d, KT_ARN_ORTH);
}

template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads, 3) kg_arn_apply(GArgs<T> A) {
  GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  if (d->arn_stop && !A.standalone) return;   // the solve stopped at this step's check
  kt_begin(d, KT_ARN_APPLY);
  constexpr int NC = D3 ? 5 : 4;
  const Grid& g = A.g;
  const int ja = d->ja;
  const long npf = A.npf;
  // product input: U_ja, or p(A) U_ja from the polynomial steps
  const T* Uj = (A.poly_deg > 0 ? A.PB : A.UB) + (long)ja * A.vs;
  T* Zout = A.Zb[ja & 1];
  const double dth = d->dta / 2.0;
  const int i = 1 + blockIdx.x * 32 + (threadIdx.x & 31), j = 1 + blockIdx.y * 8 + (threadIdx.x >> 5);
  const int k = D3 ? 1 + (int)blockIdx.z : 0;
  if (i <= g.nx && j <= g.ny) {
    const int n = dix(g, i, j, k);
    const long m = full_index(g, i, j, k);
    const uint8_t nf = g.nflags[n];
    NodeCoef<T> nc;
    if (g.kappa_per_node) nc = node_coef<T>(g, n, nf);
    else {
      nc.cx = (T)A.cxu; nc.cy = (T)A.cyu; nc.cz = (T)A.czu;
      nc.material = g.has_material != 0;
      if (!nc.material) nc.sc = T(1);
      else if (nf & NF_SCFRAC) nc.sc = (T)g.scint[n];
      else nc.sc = (nf & NF_SC0) ? T(0) : T(1);
      set_ih(g, nc);
    }
    NbEro<T> X{A.XLe, npf, m, g.mj, g.mk};
    NbMk<T> P{Uj, npf, m, g.mj, g.mk, A.deadmask[n], NbM<T>{Uj, npf, m, g.mj, g.mk, i, j, k, &g, g.lflags}};
    T o[5];
    jvp_body<T, D3>(g, X, P, nc, nf, o);
    double z[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int c = 0; c < NC; ++c) z[c] = (double)Uj[c * npf + m] - dth * (double)o[c];
    write_eff<T, D3, true>(g, Zout, npf, i, j, k, z, 0.0, 0.0, 0.0);
  }
  kt_end(d, KT_ARN_APPLY);
}

// Polynomial right preconditioner of the analytic-product solves.  The
// trapezoidal operator A = I - dt/2 J(x) has its spectrum in [a, b] with
// a = 1 - dt/2 (J's eigenvalues are at most 1: the (1 - |psi|^2) psi term)
// and b = 1 + dt/2 rho, rho a Gershgorin bound of J from the stencil
// coefficients.  p is the Chebyshev-iteration polynomial of degree d for that
// interval, p(lambda) = (1 - T_{d+1}((theta - lambda) / delta) / T_{d+1}(theta / delta)) / lambda,
// theta = (a + b) / 2, delta = (b - a) / 2, so that lambda p(lambda) lies within
// 1 +- 1 / T_{d+1}(theta / delta) on [a, b]; GMRES then runs on A p(A), and the
// Newton correction is p(A) applied to the Krylov combination.  p is stored in
// the centred variable t = (lambda - theta) / delta (|t| <= 1 on [a, b]) and
// applied by Horner's rule, one stencil launch per degree.
template <typename T>
__device__ void poly_setup(const GArgs<T>& A, GDev* d) {
  const int n = A.poly_deg + 1;
  const double h = d->dta / 2.0;
  double* e = d->poly_e;
  for (int k = 0; k <= kPolyMax; ++k) e[k] = 0.0;
  const double a = 1.0 - h, b = 1.0 + h * A.poly_rho;
  if (!(a > 0.05) || !(b > a)) {                 // no usable interval: p = 1
    e[0] = 1.0;
    d->poly_theta = 1.0;
    d->poly_delta = 1.0;
    return;
  }
  const double th = 0.5 * (a + b), de = 0.5 * (b - a), x0 = th / de;
  // T_n(-t) in powers of t by the three-term recurrence, and T_n(x0)
  double tm[kPolyMax + 2] = {1.0}, tc[kPolyMax + 2] = {0.0, -1.0}, tn[kPolyMax + 2];
  double vm = 1.0, vc = x0;
  for (int m = 1; m < n; ++m) {
    for (int k = 0; k <= m + 1; ++k) tn[k] = (k > 0 ? -2.0 * tc[k - 1] : 0.0) - (k <= m - 1 ? tm[k] : 0.0);
    for (int k = 0; k <= m + 1; ++k) { tm[k] = tc[k]; tc[k] = tn[k]; }
    const double vn = 2.0 * x0 * vc - vm;
    vm = vc;
    vc = vn;
  }
  // N(t) = 1 - T_n(-t) / T_n(x0) vanishes at t0 = -x0 (lambda = 0); p = N / (delta (t - t0))
  double N[kPolyMax + 2];
  for (int k = 0; k <= n; ++k) N[k] = -tc[k] / vc;
  N[0] += 1.0;
  const double t0 = -x0;
  double q = N[n];
  e[n - 1] = q / de;
  for (int k = n - 1; k >= 1; --k) {
    q = N[k] + t0 * q;
    e[k - 1] = q / de;
  }
  d->poly_theta = th;
  d->poly_delta = de;
}

// One Horner step of the preconditioner on the full grid:
//   W_k = e_k V + beta t(W_in),  t(W) = (A W - theta W) / delta,
// V = U_ja, the Krylov direction; the first step (k = d - 1) starts from
// W_in = V with beta = e_d, the others read W_{k+1} with beta = 1, and the
// last (k = 0) writes p(A) U_ja into the preconditioned basis PB_ja.  The
// stencil is the product kernel's (dead links from the per-node mask); W_k
// is written with its face values.
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads, 3) kg_arn_poly(GArgs<T> A) {
  GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  if (d->arn_stop && !A.standalone) return;   // the solve stopped at this step's check
  kt_begin(d, KT_ARN_APPLY);
  constexpr int NC = D3 ? 5 : 4;
  const Grid& g = A.g;
  const long npf = A.npf;
  const int kst = A.pstep, deg = A.poly_deg;
  const T* V = A.UB + (long)d->ja * A.vs;
  const T* Win = kst == deg - 1 ? V : A.PW[(kst + 1) & 1];
  T* Wout = kst == 0 ? A.PB + (long)d->ja * A.vs : A.PW[kst & 1];
  const double alpha = d->poly_e[kst], beta = kst == deg - 1 ? d->poly_e[deg] : 1.0;
  const double th = d->poly_theta, ide = 1.0 / d->poly_delta, dth = d->dta / 2.0;
  const int i = 1 + blockIdx.x * 32 + (threadIdx.x & 31), j = 1 + blockIdx.y * 8 + (threadIdx.x >> 5);
  const int k = D3 ? 1 + (int)blockIdx.z : 0;
  if (i <= g.nx && j <= g.ny) {
    const int n = dix(g, i, j, k);
    const long m = full_index(g, i, j, k);
    const uint8_t nf = g.nflags[n];
    NodeCoef<T> nc;
    if (g.kappa_per_node) nc = node_coef<T>(g, n, nf);
    else {
      nc.cx = (T)A.cxu; nc.cy = (T)A.cyu; nc.cz = (T)A.czu;
      nc.material = g.has_material != 0;
      if (!nc.material) nc.sc = T(1);
      else if (nf & NF_SCFRAC) nc.sc = (T)g.scint[n];
      else nc.sc = (nf & NF_SC0) ? T(0) : T(1);
      set_ih(g, nc);
    }
    NbEro<T> X{A.XLe, npf, m, g.mj, g.mk};
    NbMk<T> P{Win, npf, m, g.mj, g.mk, A.deadmask[n], NbM<T>{Win, npf, m, g.mj, g.mk, i, j, k, &g, g.lflags}};
    T o[5];
    jvp_body<T, D3>(g, X, P, nc, nf, o);
    double z[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const double w = (double)Win[c * npf + m];
      z[c] = alpha * (double)V[c * npf + m] + beta * ((w - dth * (double)o[c]) - th * w) * ide;
    }
    write_eff<T, D3, true>(g, Wout, npf, i, j, k, z, 0.0, 0.0, 0.0);
  }
  kt_end(d, KT_ARN_APPLY);
}

// Blocks of a two-level fold: groups of kTileGroup consecutive blocks.
constexpr int kTileGroup = 32;

// Level 1 of the two-level fold of the projections (whole block, after its
// partials part[s * nb + b] for s <= ja are written): the last block of block
// b's group to arrive adds the group's partials into gpart[s * ng + group].
// Returns true in the block that, after that, is the last of all groups.
template <typename T>
__device__ bool arn_fold_groups(const GArgs<T>& A, const double* part, int nb, int b, int ja) {
  __shared__ bool last;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = b / kTileGroup, g0 = grp * kTileGroup;
  const int gs = min(kTileGroup, nb - g0);
  const int ng = (nb + kTileGroup - 1) / kTileGroup;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(A.gticket + grp, 1u) == (unsigned)gs - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
  for (int s2 = warp; s2 <= ja; s2 += kWarps) {
    double a = lane < gs ? __ldcg(part + (long)s2 * nb + g0 + lane) : 0.0;
    a = warp_sum(a);
    if (lane == 0) A.gpart[(long)s2 * ng + grp] = a;
  }
  if (threadIdx.x == 0) A.gticket[grp] = 0u;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(A.ticket, 1u) == (unsigned)ng - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
  return true;
}

// Final fold (whole block of the last group): S[s] = sum over the ng group
// partials for s <= ja, in a fixed order.
template <typename T>
__device__ void arn_fold_final(const GArgs<T>& A, int ng, int ja, double* S) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int s2 = warp; s2 <= ja; s2 += kWarps) {
    double a = 0.0;
    for (int bb = lane; bb < ng; bb += 32) a += __ldcg(A.gpart + (long)s2 * ng + bb);
    a = warp_sum(a);
    if (lane == 0) S[s2] = a;
  }
  __syncthreads();
}

// Stop test of Arnoldi step ja before its products (one block): folds
// ||U_ja||^2 from the orthogonalisation's nblk_orth partials in a fixed order
// and completes column ja - 1 (arn_complete).  A solve of m iterations runs m
// full steps and stops in the check of step m, so no product goes unused.
template <typename T>
__global__ void kg_arn_check(GArgs<T> A) {
  __shared__ double ow[kWarps];
  // the first polynomial step (or the product) may start staging the
  // linearisation copy while this one-block kernel runs
  grid_dep_launch();
  GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  const int ja = d->ja;
  if (ja == 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double o = 0.0;
  for (int bb = threadIdx.x; bb < A.nblk_orth; bb += kThreads) o += __ldcg(A.part_orth + bb);
  o = warp_sum(o);
  if (lane == 0) ow[warp] = o;
  __syncthreads();
  if (threadIdx.x != 0) return;
  double un2 = 0.0;
  for (int w = 0; w < kWarps; ++w) un2 += ow[w];
  arn_complete(A, d, ja, un2);
  if (d->arn_stop) kt_fold(d, KT_ARN_ORTH);
}

// Projections <Z_ja, U_i> (i <= ja) over the interior entries (imask): each
// block sweeps a contiguous range of entries once per group of GGroup<T>::JB
// basis vectors (whose loads are all in flight together), Z's range staying
// in L1 between the sweeps.  Threads sum their entries' products per vector in
// T (the vectors' precision); warps and blocks add those sums in double; the
// block partials are folded in two fixed-order levels with the
// orthogonalisation's ||U_ja||^2 partials, and the last block does the column
// bookkeeping.
template <typename T>
__global__ void __launch_bounds__(kThreads, 4) kg_arn_dots(GArgs<T> A) {
  GDev* d = A.dev;
  if (!gdev_ok(d)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) abort_all(A, d->status);
    return;
  }
  if (d->arn_stop && !A.standalone) return;   // the solve stopped at this step's check
  kt_begin(d, KT_ARN_DOTS);
  extern __shared__ double red[];              // [kWarps][ja + 2]
  const int ja = d->ja;
  const int nd = ja + 2;
  const T* Z = A.Zb[ja & 1];
  const long vs = A.vs, npf = A.npf, nq = vs / 4;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int DG = GGroup<T>::JB;            // vectors per pass: their loads are all in flight at once
  // The block's contiguous range of 4-entry groups, swept once per DG
  // vectors: each thread accumulates its entries' products per vector in T,
  // the warp adds its 32 sums in double once per vector, and lane 0 keeps the
  // warp's sums.  Z's range (a few tens of KB) is re-read from L1 by the later
  // passes; the basis vectors are read through L2 only.
  const long q0 = nq * blockIdx.x / gridDim.x, q1 = nq * (blockIdx.x + 1) / gridDim.x;
  const long mo0 = (4 * (q0 + threadIdx.x)) % npf;   // offset within the component (interior mask)
  const long mstep = 4L * blockDim.x;
  for (int i0 = 0; i0 <= ja; i0 += DG) {
    T acc[DG];
#pragma unroll
    for (int t = 0; t < DG; ++t) acc[t] = T(0);
    long mo = mo0;
    for (long q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
      const long e = 4 * q;
      V4<T> z = ld4(Z + e);
      const uchar4 mk = *reinterpret_cast<const uchar4*>(A.imask + mo);
      if (!mk.x) z.a = T(0);
      if (!mk.y) z.b = T(0);
      if (!mk.z) z.c = T(0);
      if (!mk.w) z.d = T(0);
      V4<T> a[DG];
#pragma unroll
      for (int t = 0; t < DG; ++t)
        a[t] = (i0 + t <= ja) ? ld4cg(A.UB + (long)(i0 + t) * vs + e) : V4<T>{0, 0, 0, 0};
#pragma unroll
      for (int t = 0; t < DG; ++t)
        acc[t] = fma(z.a, a[t].a, fma(z.b, a[t].b, fma(z.c, a[t].c, fma(z.d, a[t].d, acc[t]))));
      mo += mstep;
      while (mo >= npf) mo -= npf;
    }
#pragma unroll
    for (int t = 0; t < DG; ++t) {
      if (i0 + t > ja) break;                  // block-uniform: no sums for vectors past ja
      const double w = warp_sum((double)acc[t]);
      if (lane == 0) red[warp * nd + i0 + t] = w;
    }
  }
  __syncthreads();
  for (int s = threadIdx.x; s <= ja; s += blockDim.x) {
    double a = 0.0;
    for (int w = 0; w < kWarps; ++w) a += red[w * nd + s];
    A.part_arn[(long)s * A.nblk_arn + blockIdx.x] = a;
  }
  if (!arn_fold_groups(A, A.part_arn, A.nblk_arn, blockIdx.x, ja)) return;
  double* S = red;
  arn_fold_final(A, (A.nblk_arn + kTileGroup - 1) / kTileGroup, ja, S);
  if (threadIdx.x == 0) {
    *A.ticket = 0u;
    if (A.standalone) return;
    if (d->status != GS_OK) { abort_all(A, d->status); return; }
    kt_fold(d, KT_ARN_ORTH);
    kt_fold(d, KT_ARN_APPLY);
    arn_finish(A, d, ja, S);
    if (d->prof_on) {
      d->kt_total[KT_ARN_DOTS] += global_ns() - d->kt_start[KT_ARN_DOTS];
      d->kt_count[KT_ARN_DOTS] += 1;
      d->kt_start[KT_ARN_DOTS] = ~0ull;
    }
  }
}

// Product and projections in one kernel: each block computes Z_ja = A U_ja
// on its 32 x 8 tile of one plane (the stencil of kg_arn_apply) and, with the
// tile's Z values still in registers, the tile's share of <Z_ja, U_i> for
// i <= ja (reading U_i at the same nodes).  Blocks are scheduled in waves, so
// stencil arithmetic of some blocks overlaps the basis reads of others, and
// Z_ja is not read back.  Per tile and vector, each thread's product goes to
// shared memory and one warp sums the block's 256 products in double; the tile
// sums are folded in two fixed-order levels (groups of kTileGroup tiles, then
// the groups) by the last block of each group and the last group, which does
// the column bookkeeping (arn_finish).
template <typename T> struct ProdChunk { static constexpr int VC = 16; };   // vectors per shared-memory pass

// Dynamic shared memory of kg_arn_apply_dots: the products of one pass, and
// (last block) the kmax + 2 folded sums.
template <typename T>
__host__ __device__ inline size_t apply_dots_smem(int kmax) {
  const size_t prod = (size_t)ProdChunk<T>::VC * kThreads * sizeof(T);
  const size_t sums = (size_t)(kmax + 2) * sizeof(double);
  return prod > sums ? prod : sums;
}

template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads, 3) kg_arn_apply_dots(GArgs<T> A) {
  GDev* d = A.dev;
  if (!gdev_ok(d)) {
    if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0) abort_all(A, d->status);
    return;
  }
  if (d->arn_stop && !A.standalone) return;   // the solve stopped at this step's check
  kt_begin(d, KT_ARN_APPLY);
  constexpr int NC = D3 ? 5 : 4;
  constexpr int VC = ProdChunk<T>::VC;
  const Grid& g = A.g;
  const int ja = d->ja;
  const long npf = A.npf;
  // product input: U_ja, or p(A) U_ja from the polynomial steps
  const T* Uj = (A.poly_deg > 0 ? A.PB : A.UB) + (long)ja * A.vs;
  T* Zout = A.Zb[ja & 1];
  const double dth = d->dta / 2.0;
  const int i = 1 + blockIdx.x * 32 + (threadIdx.x & 31), j = 1 + blockIdx.y * 8 + (threadIdx.x >> 5);
  const int k = D3 ? 1 + (int)blockIdx.z : 0;
  const bool inside = i <= g.nx && j <= g.ny;
  const long m = full_index(g, i, j, k);
  T zt[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) zt[c] = T(0);
  if (inside) {
    const int n = dix(g, i, j, k);
    const uint8_t nf = g.nflags[n];
    NodeCoef<T> nc;
    if (g.kappa_per_node) nc = node_coef<T>(g, n, nf);
    else {
      nc.cx = (T)A.cxu; nc.cy = (T)A.cyu; nc.cz = (T)A.czu;
      nc.material = g.has_material != 0;
      if (!nc.material) nc.sc = T(1);
      else if (nf & NF_SCFRAC) nc.sc = (T)g.scint[n];
      else nc.sc = (nf & NF_SC0) ? T(0) : T(1);
      set_ih(g, nc);
    }
    NbEro<T> X{A.XLe, npf, m, g.mj, g.mk};
    NbMk<T> P{Uj, npf, m, g.mj, g.mk, A.deadmask[n], NbM<T>{Uj, npf, m, g.mj, g.mk, i, j, k, &g, g.lflags}};
    T o[5];
    jvp_body<T, D3>(g, X, P, nc, nf, o);
    double z[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      z[c] = (double)Uj[c * npf + m] - dth * (double)o[c];
      zt[c] = (T)z[c];
    }
    write_eff<T, D3, true>(g, Zout, npf, i, j, k, z, 0.0, 0.0, 0.0);
  }
  // projections of this tile
  extern __shared__ __align__(16) unsigned char psm[];
  T* pv = reinterpret_cast<T*>(psm);                 // [VC][kThreads] per-thread products
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tile = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  const int ntiles = A.ntiles;
  for (int c0 = 0; c0 <= ja; c0 += VC) {
    const int nv = min(VC, ja + 1 - c0);
    for (int t0 = 0; t0 < nv; t0 += 4) {
      T u[4][NC];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const T* U = A.UB + (long)(c0 + t0 + t) * A.vs + m;
        const bool ok = inside && t0 + t < nv;
#pragma unroll
        for (int c = 0; c < NC; ++c) u[t][c] = ok ? U[c * npf] : T(0);
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        T pr = T(0);
#pragma unroll
        for (int c = 0; c < NC; ++c) pr += zt[c] * u[t][c];
        if (t0 + t < nv) pv[(t0 + t) * kThreads + threadIdx.x] = pr;
      }
    }
    __syncthreads();
    for (int v = warp; v < nv; v += kWarps) {
      double a = 0.0;
#pragma unroll
      for (int r = 0; r < kThreads / 32; ++r) a += (double)pv[v * kThreads + r * 32 + lane];
      a = warp_sum(a);
      if (lane == 0) A.part_arn[(long)(c0 + v) * ntiles + tile] = a;
    }
    __syncthreads();
  }
  if (!arn_fold_groups(A, A.part_arn, ntiles, tile, ja)) {
    kt_end(d, KT_ARN_APPLY);
    return;
  }
  double* S = reinterpret_cast<double*>(psm);
  arn_fold_final(A, A.ngroups, ja, S);
  if (threadIdx.x == 0) {
    *A.ticket = 0u;
    if (A.standalone) return;
    if (d->status != GS_OK) { abort_all(A, d->status); return; }
    kt_fold(d, KT_ARN_ORTH);
    arn_finish(A, d, ja, S);
    if (d->prof_on) {
      d->kt_total[KT_ARN_APPLY] += global_ns() - d->kt_start[KT_ARN_APPLY];
      d->kt_count[KT_ARN_APPLY] += 1;
      d->kt_start[KT_ARN_APPLY] = ~0ull;
      d->kt_end[KT_ARN_APPLY] = 0;
    }
  }
}

// ---------------------------------------------------------------------------
// One-block control kernels
// ---------------------------------------------------------------------------

// Start of a step: dt, field at t (applied_field.py:42-56) and its face offsets.
template <typename T>
__global__ void kg_step_begin(GArgs<T> A) {
  if (threadIdx.x != 0) return;
  GDev* d = A.dev;
  if (d->status != GS_OK) return;
  // the loop test of integrators.py:150 before the first step of a launch
  // (a continuation launch takes its clock from the launch before it)
  if (!(d->t < d->t_stop - 1e-14) || d->steps >= d->max_steps) { abort_all(A, GS_IDLE); return; }
  if (++d->watchdog > d->watchdog_cap) { abort_all(A, GS_CAP); return; }
  d->dta = fmin(d->dt_cur, d->t_stop - d->t);
  double bx, by, bz;
  if (d->field_const) { bx = d->Bx; by = d->By; bz = d->Bz; }
  else if (d->t <= 0.0 || d->t > d->t_field_stop * d->t_on_fraction) { bx = by = bz = 0.0; }
  else {
    double s = 1.0;
    if (d->ramp) {
      double tr = d->t_field_stop * d->ramp_fraction;
      s = tr > 0.0 ? fmin(d->t / tr, 1.0) : 1.0;
    }
    bx = d->Bx * s; by = d->By * s; bz = d->Bz * s;
  }
  const Grid& g = A.g;
  d->czxy = bz * g.hx * g.hy;
  d->cyzx = by * g.hz * g.hx;
  d->cxyz = bx * g.hy * g.hz;
  d->newton_k = 1;
  d->newton_failed = 0;
  d->accepted = 0;
  d->rhs_evals += 1;     // the predictor's f(x_n)
}

// After the first Newton residual of a step.
template <typename T>
__global__ void kg_newton_init(GArgs<T> A) {
  __shared__ double s[3];
  GDev* d = A.dev;
  if (d->status != GS_OK) return;
  reduce_parts(A.part_nrhs, A.nblk, 2, false, s);
  reduce_parts(A.part_nrhs + 2L * A.nblk, A.nblk, 1, true, s + 2);
  if (threadIdx.x != 0) return;
  kt_fold(d, KT_PREPARE);
  kt_fold(d, KT_PREDICT);
  kt_fold(d, KT_NRHS);
  d->rhs_evals += 1;
  d->rho0 = sqrt(s[0]);
  d->xnorm = sqrt(s[1]);
  if (!isfinite(d->rho0) || !isfinite(d->xnorm)) { abort_all(A, GS_NONFINITE); return; }
  if (A.poly_deg > 0) poly_setup(A, d);
  bool run_newton = d->newton_max_iter >= 1;
  bool kc = run_newton && krylov_start(A, d);
  cudaGraphSetConditional(A.h_newton, run_newton ? 1 : 0);
  cudaGraphSetConditional(A.h_krylov, kc ? 1 : 0);
}

// After the projections: Hessenberg column and orthogonalisation coefficients.
template <typename T>
__global__ void kg_fin_dots(GArgs<T> A) {
  extern __shared__ double sh[];
  GDev* d = A.dev;
  if (d->status != GS_OK) return;
  const int jc = d->j + 1;
  reduce_parts(A.part_dots, A.nblk, jc, false, sh);
  if (threadIdx.x == 0) {
    kt_fold(d, KT_STENCIL);
    kt_fold(d, KT_DOTS);
  }
  double* sj = kry_sj(A);
  double* gam = kry_gam(A);
  double* col = kry_H(A) + (long)(jc - 1) * (A.kmax + 1);
  for (int i = threadIdx.x; i < jc; i += blockDim.x) {
    double h = sh[i] * sj[i];      // h_ij = <w, v_i>
    col[i] = h;
    gam[i] = h * sj[i];            // coefficient on the raw v~_i
  }
}

// After the orthogonalisation: new basis scale, Givens rotation, residual
// estimate, continue / stop (tgcr.py:125 loop test, 141-142 breakdown).
template <typename T>
__global__ void kg_fin_orth(GArgs<T> A) {
  __shared__ double s[1];
  GDev* d = A.dev;
  if (d->status != GS_OK) return;
  reduce_parts(A.part_orth, A.nblk, 1, false, s);
  if (threadIdx.x != 0) return;
  if (++d->watchdog > d->watchdog_cap) { abort_all(A, GS_CAP); return; }
  kt_fold(d, KT_ORTH);
  const int jc = d->j + 1;
  d->jvp_evals += 1;
  double hn = sqrt(s[0]);
  if (!isfinite(hn)) { abort_all(A, GS_NONFINITE); return; }
  double* sj = kry_sj(A);
  double* gv = kry_gv(A);
  double* cs = kry_cs(A);
  double* sn = kry_sn(A);
  double* col = kry_H(A) + (long)(jc - 1) * (A.kmax + 1);
  sj[jc] = hn > 0.0 ? 1.0 / hn : 0.0;
  col[jc] = hn;
  for (int i = 0; i + 1 < jc; ++i) {
    double a = col[i], b = col[i + 1];
    col[i] = cs[i] * a + sn[i] * b;
    col[i + 1] = -sn[i] * a + cs[i] * b;
  }
  double a = col[jc - 1], b = col[jc];
  double r = hypot(a, b);
  double c = r > 0.0 ? a / r : 1.0, sv = r > 0.0 ? b / r : 0.0;
  cs[jc - 1] = c;
  sn[jc - 1] = sv;
  col[jc - 1] = r;
  col[jc] = 0.0;
  gv[jc] = -sv * gv[jc - 1];
  gv[jc - 1] = c * gv[jc - 1];
  d->rho = fabs(gv[jc]);
  d->j = jc;
  bool cont = hn > 0.0 && d->rho / d->rho0 > d->tol_lin && jc < d->krylov_max_iter;
  if (cont && jc + 1 > A.kmax) { abort_all(A, GS_KMAX); return; }
  cudaGraphSetConditional(A.h_krylov, cont ? 1 : 0);
}

// End of a Krylov solve: least-squares coefficients and the reference's final
// residual test (tgcr.py:154-155; failure ends Newton, newton.py:103-106).
template <typename T>
__global__ void kg_newton_solve(GArgs<T> A) {
  if (threadIdx.x != 0) return;
  GDev* d = A.dev;
  if (d->status != GS_OK) return;
  const int j = d->j;
  d->krylov_iters += j;
  d->krylov_sq += (long long)j * j;
  d->krylov_last = j;
  if (j > d->max_krylov) d->max_krylov = j;
  bool ok = !(d->rho > d->tol_lin * d->rho0);
  if (!ok) {
    d->newton_failed = 1;
    cudaGraphSetConditional(A.h_newton, 0);
    return;
  }
  const double* H = kry_H(A);
  const double* gv = kry_gv(A);
  const double* sj = kry_sj(A);
  double* y = kry_gam(A);
  double* cj = kry_cj(A);
  for (int i = j - 1; i >= 0; --i) {
    double acc = gv[i];
    for (int l = i + 1; l < j; ++l) acc -= H[(long)l * (A.kmax + 1) + i] * y[l];
    y[i] = acc / H[(long)i * (A.kmax + 1) + i];
  }
  for (int i = 0; i < j; ++i) cj[i] = y[i] * sj[i];
}

// After the Newton residual of the updated iterate: convergence test
// (newton.py:108-118), next iteration or stop.
template <typename T>
__global__ void kg_newton_check(GArgs<T> A) {
  __shared__ double s[4];
  GDev* d = A.dev;
  if (d->status != GS_OK || d->newton_failed) return;
  reduce_parts(A.part_nrhs, A.nblk, 2, false, s);
  reduce_parts(A.part_nrhs + 2L * A.nblk, A.nblk, 1, true, s + 2);
  reduce_parts(A.part_upd, A.nblk, 1, true, s + 3);
  if (threadIdx.x != 0) return;
  if (++d->watchdog > d->watchdog_cap) { abort_all(A, GS_CAP); return; }
  kt_fold(d, KT_UPDATE);
  kt_fold(d, KT_NRHS);
  d->rhs_evals += 1;
  d->newton_iters += 1;
  d->rho0 = sqrt(s[0]);
  d->xnorm = sqrt(s[1]);
  d->gnorm = s[2];
  d->dxnorm = s[3];
  if (!isfinite(d->gnorm) || !isfinite(d->dxnorm) || !isfinite(d->rho0)) { abort_all(A, GS_NONFINITE); return; }
  if (d->gnorm <= d->tol_f && d->dxnorm <= d->tol_dx) {
    d->accepted = 1;
    cudaGraphSetConditional(A.h_newton, 0);
    return;
  }
  if (d->newton_k >= d->newton_max_iter) {
    cudaGraphSetConditional(A.h_newton, 0);
    return;
  }
  d->newton_k += 1;
  bool kc = krylov_start(A, d);
  cudaGraphSetConditional(A.h_krylov, kc ? 1 : 0);
  cudaGraphSetConditional(A.h_newton, 1);
}

// End of a step attempt: accept (t += dt) or retry with dt / 10
// (integrators.py:174-197); continue while steps remain.
template <typename T>
__global__ void kg_step_end(GArgs<T> A) {
  if (threadIdx.x != 0) return;
  GDev* d = A.dev;
  kt_fold(d, KT_ACCEPT);
  if (d->status == GS_OK) {
    if (d->accepted) {
      d->t += d->dta;
      d->steps += 1;
      d->dt_cur = d->dt;
    } else {
      d->rejections += 1;
      if (!d->adaptive) d->status = GS_NOCONV;
      else {
        d->dt_cur /= 10.0;
        if (d->dt_cur < d->dt_min) d->status = GS_DTMIN;
      }
    }
  }
  bool more = d->status == GS_OK && d->t < d->t_stop - 1e-14 && d->steps < d->max_steps;
  cudaGraphSetConditional(A.h_step, more ? 1 : 0);
}

}  // namespace tdgl
