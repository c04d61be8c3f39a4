// Persistent, cooperatively launched trapezoidal Newton-Krylov stepper.
//
// One launch advances the state through up to `max_steps` accepted
// trapezoidal steps (src/tdgl3d/solvers/integrators.py:92-206), each solved by
// Newton (src/tdgl3d/solvers/newton.py:76-120) with a GCR inner solve of
// (I - dt/2 J) d = -g (src/tdgl3d/solvers/tgcr.py:96-156).  All control
// decisions (Krylov stopping test, breakdown, Newton tests, dt/10 retries,
// dt_min) are taken on the device: every block reads the same reduced scalars
// after a grid barrier and takes the same branch, so there is no host round
// trip inside a launch.
//
// GCR as in the reference, with two changes that do not alter the iterates in
// exact arithmetic:
//   * classical instead of modified Gram-Schmidt: the projections of a new
//     direction on all stored ones come from one reduction (the stored A p_j are
//     orthonormal, so CGS and MGS agree up to rounding), accumulated in FP64;
//   * the normalisation of p_k, Ap_k is kept as a scale factor instead of a
//     rewrite, the residual update r -= alpha Ap_k is folded into the next
//     stencil pass, and the solution update x += alpha p_k is applied once at
//     the end of the solve.
// Per Krylov iteration: one stencil pass (new A r, its projections, and the
// norm of r) and one orthogonalisation pass, each ended by a grid reduction.
//
// Storage precision T (double, or float in the mixed form) applies to the
// Krylov vectors r, p_j, Ap_j and to the linearisation copy of x used by the
// analytic Jacobian product; the state, gamma, f(x), residual g and all
// reductions stay FP64.
#pragma once

#include "tdgl_kernels.cuh"

namespace tdgl {

enum RunMode : int { RUN_TRAP = 0, RUN_NEWTON = 1, RUN_TGCR = 2 };
enum JvpMode : int { JVP_FD = 0, JVP_ANALYTIC = 1 };
enum Status : int { ST_OK = 0, ST_NOCONV = 1, ST_DTMIN = 2, ST_KMAX = 3, ST_NONFINITE = 4, ST_TIMEOUT = 5 };

// Host <-> device control block (one per context).
struct Ctl {
  // inputs
  double t_stop, dt, dt_min, tol_f, tol_dx, tol_gcr, eps_mf;
  double Bx, By, Bz, t_on_fraction, ramp_fraction, t_field_stop;
  int newton_max_iter, krylov_max_iter, adaptive, jvp_mode, max_steps, ramp, field_const, run_mode;
  // inputs / outputs
  double t, dt_cur;
  int cur;                  // X buffer holding the accepted state (trapezoidal) or the iterate
  // outputs
  int status, steps, newton_converged, newton_iters_last, krylov_last;
  long long newton_iters, krylov_iters, rhs_evals, jvp_evals, rejections;
  int max_krylov;
  double last_gnorm, last_dxnorm, last_rnorm_rel;
};

template <typename T>
struct StepArgs {
  Grid g;
  Sync sy;
  Ctl* ctl;
  double* X[2];     // FP64 states (accepted / iterate)
  double* G;        // gamma
  double* F;        // f(iterate)
  double* D;        // RUN_TGCR output (FP64 solution)
  T* R[3];          // residual buffers (rotating)
  T* XL;            // linearisation copy (analytic JVP) in T, or nullptr to read X
  T* P;             // kmax slots of length L
  T* AP;            // kmax slots of length L
  int kmax;
  long L;           // ncomp * npad
};

template <typename T>
struct Shared {
  double* acc;      // [kWarps][nacc]
  double* blk;      // [nacc]
  double* red;      // [nacc]
  double* gam;      // [kmax]   projection coefficients of the current direction
  double* cj;       // [kmax]   solution coefficients alpha_j * s_j
  double* sj;       // [kmax]   normalisation scales 1/||Ap~_j||
  int nacc;
};

__device__ __forceinline__ void field_at(const Ctl& c, double t, double& bx, double& by, double& bz) {
  // src/tdgl3d/physics/applied_field.py:42-56
  if (c.field_const) { bx = c.Bx; by = c.By; bz = c.Bz; return; }
  if (t <= 0.0 || t > c.t_field_stop * c.t_on_fraction) { bx = by = bz = 0.0; return; }
  double s = 1.0;
  if (c.ramp) {
    double tr = c.t_field_stop * c.ramp_fraction;
    s = tr > 0.0 ? fmin(t / tr, 1.0) : 1.0;
  }
  bx = c.Bx * s; by = c.By * s; bz = c.Bz * s;
}

// Face offsets of the applied field in the reference's product order
// (src/tdgl3d/physics/rhs.py:92-134): Bz*hx*hy, By*hz*hx, Bx*hy*hz.
__host__ __device__ __forceinline__ BTerms<double> bterms(const Grid& g, double bx, double by, double bz) {
  return BTerms<double>{bz * g.hx * g.hy, by * g.hz * g.hx, bx * g.hy * g.hz};
}

// Zero the per-warp accumulators.
template <typename T>
__device__ __forceinline__ void acc_zero(Shared<T>& sm, int nslot) {
  for (int t = threadIdx.x; t < kWarps * sm.nacc; t += blockDim.x) sm.acc[t] = 0.0;
  __syncthreads();
  (void)nslot;
}
// Fold per-warp accumulators (fixed order) into block values.
template <typename T>
__device__ __forceinline__ void acc_fold(Shared<T>& sm, int nslot, int nsum) {
  __syncthreads();
  for (int t = threadIdx.x; t < nslot; t += blockDim.x) {
    double v = 0.0;
    for (int w = 0; w < kWarps; ++w) v = t < nsum ? v + sm.acc[w * sm.nacc + t] : fmax(v, sm.acc[w * sm.nacc + t]);
    sm.blk[t] = v;
  }
  __syncthreads();
}
// Warp-reduce v into accumulator slot `slot` (lane 0 writes; fixed order).
__device__ __forceinline__ void acc_add(double* acc, int nacc, int slot, double v) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) acc[(threadIdx.x >> 5) * nacc + slot] += v;
}
__device__ __forceinline__ void acc_max(double* acc, int nacc, int slot, double v) {
  v = warp_max(v);
  if ((threadIdx.x & 31) == 0) {
    double* p = &acc[(threadIdx.x >> 5) * nacc + slot];
    *p = fmax(*p, v);
  }
}

__device__ __forceinline__ double nonfinite_guard(double v) { return isfinite(v) ? v : INFINITY; }

// ---------------------------------------------------------------------------
// Passes.  Node loops are grid-stride loops padded to whole warps so that every
// lane of a warp takes part in the warp reductions.
// ---------------------------------------------------------------------------

// f = rhs(X); Xn = X + dt f; G = X + dt/2 f   (integrators.py:156-158)
template <typename T>
__device__ void pass_predict(const StepArgs<T>& A, const double* X, double* Xn, double dt, BTerms<double> b) {
  const Grid& g = A.g;
  SrcVec<double, double> sx{X, g.npad};
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    double o[5];
    rhs_at<double>(g, sx, b, d, o);
    for (int c = 0; c < g.ncomp; ++c) {
      long e = (long)c * g.npad + d;
      double xv = X[e];
      Xn[e] = xv + dt * o[c];
      A.G[e] = xv + (dt / 2.0) * o[c];
    }
  }
}

// f = rhs(x); g = x - dt/2 f - gamma; r0 = -g (as T); slots: 0 ||r0||^2, 1 ||x||^2, 2 max|g| (max slot)
template <typename T>
__device__ void pass_newton_rhs(const StepArgs<T>& A, Shared<T>& sm, const double* x, T* r0, double dt,
                                BTerms<double> b) {
  const Grid& g = A.g;
  SrcVec<double, double> sx{x, g.npad};
  const int nstride = gridDim.x * blockDim.x;
  const int nround = (g.n + nstride - 1) / nstride;
  for (int it = 0; it < nround; ++it) {
    int d = it * nstride + blockIdx.x * blockDim.x + threadIdx.x;
    double s_r = 0.0, s_x = 0.0, m_g = 0.0;
    if (d < g.n) {
      double o[5];
      rhs_at<double>(g, sx, b, d, o);
      double gv[5];
      for (int c = 0; c < g.ncomp; ++c) {
        long e = (long)c * g.npad + d;
        double xv = x[e];
        A.F[e] = o[c];
        gv[c] = xv - (dt / 2.0) * o[c] - A.G[e];
        T rv = (T)(-gv[c]);
        r0[e] = rv;
        if (A.XL) A.XL[e] = (T)xv;
        s_r += (double)rv * (double)rv;
        s_x += xv * xv;
      }
      m_g = nonfinite_guard(hypot(gv[0], gv[1]));
      for (int c = 2; c < g.ncomp; ++c) m_g = fmax(m_g, nonfinite_guard(fabs(gv[c])));
    }
    acc_add(sm.acc, sm.nacc, 0, s_r);
    acc_add(sm.acc, sm.nacc, 1, s_x);
    acc_max(sm.acc, sm.nacc, 2, m_g);
  }
}

// Krylov stencil pass for direction k (1-based).
//   r_{k-1} = Rin - a_prev * Ap~_{k-1}   (k > 1; written to Rout, ||r||^2 -> slot k-1)
//   w       = r - dt/2 J(x) r            (written to Ap~_k)
//   slot j-1 (j < k) <- <w, Ap~_j>
template <typename T>
__device__ void pass_krylov_stencil(const StepArgs<T>& A, Shared<T>& sm, int k, const T* Rin, T* Rout,
                                    double a_prev, const double* x, double dt, double eps, BTerms<double> b,
                                    int jvp_mode, bool norm_only) {
  const Grid& g = A.g;
  const long L = A.L;
  const T* APprev = k > 1 ? A.AP + (long)(k - 2) * L : nullptr;
  T* W = A.AP + (long)(k - 1) * L;
  const int nstride = gridDim.x * blockDim.x;
  const int nround = (g.n + nstride - 1) / nstride;
  const double dth = dt / 2.0;
  for (int it = 0; it < nround; ++it) {
    int d = it * nstride + blockIdx.x * blockDim.x + threadIdx.x;
    bool live = d < g.n;
    double rv[5] = {0, 0, 0, 0, 0}, wv[5] = {0, 0, 0, 0, 0};
    double s_r = 0.0;
    if (live) {
      for (int c = 0; c < g.ncomp; ++c) {
        long e = (long)c * g.npad + d;
        double r = (double)Rin[e];
        if (APprev) {
          T rt = (T)((T)Rin[e] - (T)a_prev * APprev[e]);
          Rout[e] = rt;
          r = (double)rt;
        }
        rv[c] = r;
        s_r += r * r;
      }
      if (!norm_only) {
        if (jvp_mode == JVP_FD) {
          // reference finite-difference product around x (FP64 only)
          SrcFD<T> sfd{x, Rin, APprev, a_prev, eps, g.npad};
          double o[5];
          rhs_at<double>(g, sfd, b, d, o);
          for (int c = 0; c < g.ncomp; ++c) {
            long e = (long)c * g.npad + d;
            wv[c] = rv[c] - dth * ((o[c] - A.F[e]) / eps);
          }
        } else {
          SrcAxpy<T, T> sp{Rin, APprev, (T)a_prev, g.npad};
          BTerms<T> bt{(T)b.czxy, (T)b.cyzx, (T)b.cxyz};
          T o[5];
          if (A.XL) {
            SrcVec<T, T> sx{A.XL, g.npad};
            jvp_at<T>(g, sx, bt, sp, d, o);
          } else {
            SrcVec<T, double> sx{x, g.npad};
            jvp_at<T>(g, sx, bt, sp, d, o);
          }
          for (int c = 0; c < g.ncomp; ++c) wv[c] = rv[c] - dth * (double)o[c];
        }
        for (int c = 0; c < g.ncomp; ++c) {
          T wt = (T)wv[c];
          W[(long)c * g.npad + d] = wt;
          wv[c] = (double)wt;
        }
      }
    }
    if (k > 1) acc_add(sm.acc, sm.nacc, k - 1, s_r);
    if (!norm_only) {
      for (int j = 1; j < k; ++j) {
        const T* APj = A.AP + (long)(j - 1) * L;
        double s = 0.0;
        if (live)
          for (int c = 0; c < g.ncomp; ++c) s += wv[c] * (double)APj[(long)c * g.npad + d];
        acc_add(sm.acc, sm.nacc, j - 1, s);
      }
    }
  }
}

// Orthogonalisation pass for direction k:
//   P~_k  = r - sum_j gam_j P~_j,  Ap~_k = w - sum_j gam_j Ap~_j
//   slot 0 <- ||Ap~_k||^2, slot 1 <- <r, Ap~_k>
template <typename T>
__device__ void pass_krylov_orth(const StepArgs<T>& A, Shared<T>& sm, int k, const T* Rk) {
  const long L = A.L;
  T* Pk = A.P + (long)(k - 1) * L;
  T* APk = A.AP + (long)(k - 1) * L;
  const int nstride = gridDim.x * blockDim.x;
  const long nround = (L + nstride - 1) / nstride;
  for (long it = 0; it < nround; ++it) {
    long e = it * nstride + blockIdx.x * blockDim.x + threadIdx.x;
    double s_q = 0.0, s_rq = 0.0;
    if (e < L) {
      double r = (double)Rk[e];
      double p = r, q = (double)APk[e];
      for (int j = 0; j < k - 1; ++j) {
        double gj = sm.gam[j];
        p -= gj * (double)A.P[(long)j * L + e];
        q -= gj * (double)A.AP[(long)j * L + e];
      }
      T pt = (T)p, qt = (T)q;
      Pk[e] = pt;
      APk[e] = qt;
      s_q = (double)qt * (double)qt;
      s_rq = r * (double)qt;
    }
    acc_add(sm.acc, sm.nacc, 0, s_q);
    acc_add(sm.acc, sm.nacc, 1, s_rq);
  }
}

// x += sum_j cj_j P~_j; slot 0 <- max |dx| (complex modulus on psi entries)
template <typename T>
__device__ void pass_update(const StepArgs<T>& A, Shared<T>& sm, double* x, int nk, double* dout) {
  const Grid& g = A.g;
  const long L = A.L;
  const int nstride = gridDim.x * blockDim.x;
  const int nround = (g.n + nstride - 1) / nstride;
  for (int it = 0; it < nround; ++it) {
    int d = it * nstride + blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0;
    if (d < g.n) {
      double dv[5];
      for (int c = 0; c < g.ncomp; ++c) {
        long e = (long)c * g.npad + d;
        double s = 0.0;
        for (int j = 0; j < nk; ++j) s += sm.cj[j] * (double)A.P[(long)j * L + e];
        dv[c] = s;
        if (x) x[e] += s;
        if (dout) dout[e] = s;
      }
      m = nonfinite_guard(hypot(dv[0], dv[1]));
      for (int c = 2; c < g.ncomp; ++c) m = fmax(m, nonfinite_guard(fabs(dv[c])));
    }
    acc_max(sm.acc, sm.nacc, 0, m);
  }
}

// rhs(x) into F; slot 0 <- ||x||^2 (used by RUN_TGCR for the FD base point)
template <typename T>
__device__ void pass_base(const StepArgs<T>& A, Shared<T>& sm, const double* x, BTerms<double> b) {
  const Grid& g = A.g;
  SrcVec<double, double> sx{x, g.npad};
  const int nstride = gridDim.x * blockDim.x;
  const int nround = (g.n + nstride - 1) / nstride;
  for (int it = 0; it < nround; ++it) {
    int d = it * nstride + blockIdx.x * blockDim.x + threadIdx.x;
    double s_x = 0.0;
    if (d < g.n) {
      double o[5];
      rhs_at<double>(g, sx, b, d, o);
      for (int c = 0; c < g.ncomp; ++c) {
        long e = (long)c * g.npad + d;
        A.F[e] = o[c];
        double xv = x[e];
        if (A.XL) A.XL[e] = (T)xv;
        s_x += xv * xv;
      }
    }
    acc_add(sm.acc, sm.nacc, 0, s_x);
  }
}

// ---------------------------------------------------------------------------
// Solvers
// ---------------------------------------------------------------------------

struct KrylovOut {
  bool ok;        // converged (reference: non-empty solution)
  int nk;         // directions in the solution
  int status;     // ST_OK, ST_NOCONV, ST_KMAX, ST_TIMEOUT
};

// GCR on (I - dt/2 J(x)) d = r0 where r0 sits in A.R[0] (||r0|| = rho0).
// The solution is sum_j sm.cj[j] * P~_j, j < nk.
template <typename T>
__device__ KrylovOut krylov(const StepArgs<T>& A, Shared<T>& sm, const double* x, double xnorm, double rho0,
                            double dt, double tol, int max_iter, double eps_mf, int jvp_mode, BTerms<double> b,
                            long long& jvp_count) {
  KrylovOut out{true, 0, ST_OK};
  if (!isfinite(rho0) || !isfinite(xnorm)) { out.ok = false; out.status = ST_NONFINITE; return out; }
  if (rho0 == 0.0) return out;                 // tgcr.py:121-122
  double rho = rho0;                           // ||r_{k-1}|| once computed
  double rho_est = rho0;                       // estimate used by the FD epsilon
  double a_prev = 0.0;
  int rin = 0;                                 // R[rin] holds the last materialised residual
  int k = 0;
  bool converged_exit = false;
  while (true) {
    if (!(rho / rho0 > tol)) { converged_exit = true; break; }
    if (k >= max_iter) break;
    if (k + 1 > A.kmax) { out.status = ST_KMAX; out.ok = false; return out; }
    ++k;
    int rout = k > 1 ? (rin + 1) % 3 : rin;
    double eps = eps_mf * (1.0 + xnorm) / rho_est;
    // stencil pass: materialise r_{k-1}, w = A r_{k-1}, projections
    acc_zero(sm, k);
    pass_krylov_stencil<T>(A, sm, k, A.R[rin], A.R[rout], a_prev, x, dt, eps, b, jvp_mode, false);
    acc_fold(sm, k, k);
    if (!grid_reduce(A.sy, sm.blk, k, k, sm.red)) { out.status = ST_TIMEOUT; out.ok = false; return out; }
    ++jvp_count;
    if (k > 1) {
      rho = sqrt(sm.red[k - 1]);
      rin = rout;
      if (!isfinite(rho)) { out.status = ST_NONFINITE; out.ok = false; return out; }
      if (!(rho / rho0 > tol)) { --k; converged_exit = true; break; }
    }
    for (int t = threadIdx.x; t < k - 1; t += blockDim.x) sm.gam[t] = sm.red[t] * sm.sj[t] * sm.sj[t];
    __syncthreads();
    // orthogonalisation pass
    acc_zero(sm, 2);
    pass_krylov_orth<T>(A, sm, k, A.R[rin]);
    acc_fold(sm, 2, 2);
    if (!grid_reduce(A.sy, sm.blk, 2, 2, sm.red)) { out.status = ST_TIMEOUT; out.ok = false; return out; }
    double nu = sqrt(sm.red[0]);
    if (!(nu >= 1e-14)) {                       // tgcr.py:141-142 (also stops on NaN)
      if (!isfinite(nu)) { out.status = ST_NONFINITE; out.ok = false; return out; }
      --k;
      break;
    }
    double s = 1.0 / nu;
    double alpha = s * sm.red[1];
    if (threadIdx.x == 0) { sm.sj[k - 1] = s; sm.cj[k - 1] = alpha * s; }
    __syncthreads();
    a_prev = alpha * s;
    double r2 = rho * rho - alpha * alpha;
    rho_est = r2 > 0.0 ? sqrt(r2) : rho * 1e-8;
    if (k >= max_iter) {
      // the reference leaves the loop here and tests the explicit residual norm
      int rout2 = (rin + 1) % 3;
      acc_zero(sm, k + 1);
      pass_krylov_stencil<T>(A, sm, k + 1, A.R[rin], A.R[rout2], a_prev, x, dt, eps, b, jvp_mode, true);
      acc_fold(sm, k + 1, k + 1);
      if (!grid_reduce(A.sy, sm.blk, k + 1, k + 1, sm.red)) { out.status = ST_TIMEOUT; out.ok = false; return out; }
      rho = sqrt(sm.red[k]);
      rin = rout2;
      break;
    }
  }
  (void)converged_exit;
  out.nk = k;
  // final test of the reference (tgcr.py:154-155)
  out.ok = !(rho > tol * rho0);
  out.status = out.ok ? ST_OK : ST_NOCONV;
  return out;
}

// Newton on g(x) = x - dt/2 f(x) - gamma from x = X[xi]; returns converged.
template <typename T>
__device__ bool newton(const StepArgs<T>& A, Shared<T>& sm, Ctl& c, double* x, double dt, BTerms<double> b,
                       int& status, int& iters) {
  // top of the first iteration: f(x), g, -g
  acc_zero(sm, 3);
  pass_newton_rhs<T>(A, sm, x, A.R[0], dt, b);
  acc_fold(sm, 3, 2);
  if (!grid_reduce(A.sy, sm.blk, 3, 2, sm.red)) { status = ST_TIMEOUT; return false; }
  c.rhs_evals += 1;
  double rho0 = sqrt(sm.red[0]), xnorm = sqrt(sm.red[1]);
  for (int k = 1; k <= c.newton_max_iter; ++k) {
    long long jv = 0;
    KrylovOut ko = krylov<T>(A, sm, x, xnorm, rho0, dt, c.tol_gcr, c.krylov_max_iter, c.eps_mf, c.jvp_mode, b, jv);
    c.jvp_evals += jv;
    c.krylov_iters += ko.nk;
    c.krylov_last = ko.nk;
    if (ko.nk > c.max_krylov) c.max_krylov = ko.nk;
    if (ko.status == ST_TIMEOUT || ko.status == ST_KMAX || ko.status == ST_NONFINITE) { status = ko.status; iters = k; return false; }
    if (!ko.ok) { status = ST_NOCONV; iters = k; return false; }   // newton.py:103-106
    acc_zero(sm, 1);
    pass_update<T>(A, sm, x, ko.nk, nullptr);
    acc_fold(sm, 1, 0);
    if (!grid_reduce(A.sy, sm.blk, 1, 0, sm.red)) { status = ST_TIMEOUT; return false; }
    double dxn = sm.red[0];
    acc_zero(sm, 3);
    pass_newton_rhs<T>(A, sm, x, A.R[0], dt, b);
    acc_fold(sm, 3, 2);
    if (!grid_reduce(A.sy, sm.blk, 3, 2, sm.red)) { status = ST_TIMEOUT; return false; }
    c.rhs_evals += 1;
    c.newton_iters += 1;
    rho0 = sqrt(sm.red[0]);
    xnorm = sqrt(sm.red[1]);
    double gn = sm.red[2];
    c.last_gnorm = gn;
    c.last_dxnorm = dxn;
    if (!isfinite(gn) || !isfinite(dxn)) { status = ST_NONFINITE; iters = k; return false; }
    if (gn <= c.tol_f && dxn <= c.tol_dx) { status = ST_OK; iters = k; return true; }
  }
  status = ST_NOCONV;
  iters = c.newton_max_iter;
  return false;
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 1) k_stepper(StepArgs<T> A) {
  extern __shared__ double smem[];
  Shared<T> sm;
  sm.nacc = A.kmax + 4;
  sm.acc = smem;
  sm.blk = sm.acc + kWarps * sm.nacc;
  sm.red = sm.blk + sm.nacc;
  sm.gam = sm.red + sm.nacc;
  sm.cj = sm.gam + A.kmax;
  sm.sj = sm.cj + A.kmax;

  Ctl c = *A.ctl;     // every block keeps an identical copy of the control state
  const Grid& g = A.g;
  int status = ST_OK;

  if (c.run_mode == RUN_TGCR) {
    // one linear solve: x_lin in X[0], b in R[0]; solution (FP64) into D
    BTerms<double> b = bterms(g, c.Bx, c.By, c.Bz);
    acc_zero(sm, 2);
    pass_base<T>(A, sm, A.X[0], b);
    {
      const int nstride = gridDim.x * blockDim.x;
      const long nround = (A.L + nstride - 1) / nstride;
      for (long it = 0; it < nround; ++it) {
        long e = it * nstride + blockIdx.x * blockDim.x + threadIdx.x;
        double v = e < A.L ? (double)A.R[0][e] : 0.0;
        acc_add(sm.acc, sm.nacc, 1, v * v);
      }
    }
    acc_fold(sm, 2, 2);
    if (!grid_reduce(A.sy, sm.blk, 2, 2, sm.red)) status = ST_TIMEOUT;
    c.rhs_evals += 1;
    if (status == ST_OK) {
      double xnorm = sqrt(sm.red[0]), rho0 = sqrt(sm.red[1]);
      long long jv = 0;
      KrylovOut ko = krylov<T>(A, sm, A.X[0], xnorm, rho0, c.dt, c.tol_gcr, c.krylov_max_iter, c.eps_mf,
                               c.jvp_mode, b, jv);
      c.jvp_evals += jv;
      c.krylov_last = ko.nk;
      c.krylov_iters += ko.nk;
      c.last_rnorm_rel = 0.0;
      status = ko.status;
      if (ko.status == ST_OK || ko.status == ST_NOCONV) {
        acc_zero(sm, 1);
        pass_update<T>(A, sm, nullptr, ko.nk, A.D);
        acc_fold(sm, 1, 0);
        if (!grid_reduce(A.sy, sm.blk, 1, 0, sm.red)) status = ST_TIMEOUT;
      }
    }
  } else if (c.run_mode == RUN_NEWTON) {
    // one Newton solve: iterate in X[c.cur], gamma in G
    BTerms<double> b = bterms(g, c.Bx, c.By, c.Bz);
    int iters = 0;
    bool ok = newton<T>(A, sm, c, A.X[c.cur], c.dt, b, status, iters);
    c.newton_converged = ok ? 1 : 0;
    c.newton_iters_last = iters;
    if (status == ST_NOCONV) status = ST_OK;   // non-convergence is reported, not an error
  } else {
    // trapezoidal steps (integrators.py:150-197)
    int steps = 0;
    while (c.t < c.t_stop - 1e-14 && steps < c.max_steps) {
      double dta = fmin(c.dt_cur, c.t_stop - c.t);
      double bx, by, bz;
      field_at(c, c.t, bx, by, bz);
      BTerms<double> b = bterms(g, bx, by, bz);
      double* Xs = A.X[c.cur];
      double* Xi = A.X[1 - c.cur];
      pass_predict<T>(A, Xs, Xi, dta, b);
      c.rhs_evals += 1;
      if (!grid_sync(A.sy, sm.blk)) { status = ST_TIMEOUT; break; }
      int st = ST_OK, iters = 0;
      bool ok = newton<T>(A, sm, c, Xi, dta, b, st, iters);
      c.newton_iters_last = iters;
      if (st == ST_TIMEOUT || st == ST_KMAX || st == ST_NONFINITE) { status = st; break; }
      if (ok) {
        c.cur = 1 - c.cur;
        c.t += dta;
        ++steps;
        c.dt_cur = c.dt;
      } else {
        c.rejections += 1;
        if (!c.adaptive) { status = ST_NOCONV; break; }
        c.dt_cur /= 10.0;
        if (c.dt_cur < c.dt_min) { status = ST_DTMIN; break; }
      }
    }
    c.steps = steps;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c.status = status;
    *A.ctl = c;
  }
}

}  // namespace tdgl
