// Persistent, cooperatively launched trapezoidal Newton-Krylov stepper.
//
// One launch advances the state through up to `max_steps` accepted
// trapezoidal steps (src/tdgl3d/solvers/integrators.py:92-206), each solved by
// Newton (src/tdgl3d/solvers/newton.py:76-120) with a Krylov solve of
// (I - dt/2 J) d = -g (src/tdgl3d/solvers/tgcr.py:96-156).  All control
// decisions (Krylov stopping test, breakdown, Newton tests, dt/10 retries,
// dt_min) are taken on the device: every block reads the same reduced scalars
// after a grid barrier and takes the same branch, so there is no host round
// trip inside a launch.
//
// Krylov methods (both minimise ||b - A d|| over the same Krylov space, so
// their iterates agree in exact arithmetic; the stopping test is the
// reference's ||r|| / ||r0|| > tol loop condition and final check):
//   KRY_GCR    the reference's GCR: direction pairs (p_k, A p_k), A p_k
//              orthonormalised against all previous ones.  Classical instead of
//              modified Gram-Schmidt (one reduction for all projections, FP64
//              accumulation); normalisation kept as a scale factor; r -= alpha
//              A p_k folded into the next stencil pass; d = sum alpha_k p_k
//              applied once at the end.  Two passes over both stored sets per
//              iteration.
//   KRY_GMRES  Arnoldi with one stored set (the orthonormal basis v_i, kept
//              unnormalised with scale factors), Givens rotations of the
//              Hessenberg column on every block, the residual norm from the
//              rotated right-hand side, and d = V y from the triangular solve
//              at the end.  Two passes over one stored set per iteration.
//
// Storage precision T (double, or float in the mixed form) applies to the
// Krylov vectors and to the linearisation copy of x used by the analytic
// Jacobian product; the state, gamma, f(x), residual g and all reductions stay
// FP64.
//
// Stencil passes give each warp 128-node regions: lanes first take the plain
// interior ("fast") nodes of the region, then the region's boundary / hole
// ("slow") nodes from a compacted list, so no warp runs both paths divergently.
#pragma once

#include "tdgl_common.cuh"

namespace tdgl {

enum RunMode : int { RUN_TRAP = 0, RUN_NEWTON = 1, RUN_TGCR = 2 };
enum KrylovKind : int { KRY_GMRES = 0, KRY_GCR = 1 };
enum Status : int { ST_OK = 0, ST_NOCONV = 1, ST_DTMIN = 2, ST_KMAX = 3, ST_NONFINITE = 4, ST_TIMEOUT = 5 };

// Host <-> device control block (one per context).
struct Ctl {
  // inputs
  double t_stop, dt, dt_min, tol_f, tol_dx, tol_gcr, eps_mf;
  double Bx, By, Bz, t_on_fraction, ramp_fraction, t_field_stop;
  int newton_max_iter, krylov_max_iter, adaptive, jvp_mode, max_steps, ramp, field_const, run_mode, krylov;
  // inputs / outputs
  double t, dt_cur;
  int cur;                  // X buffer holding the accepted state (trapezoidal) or the iterate
  // outputs
  int status, steps, newton_converged, newton_iters_last, krylov_last;
  long long newton_iters, krylov_iters, rhs_evals, jvp_evals, rejections, krylov_sq;
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
  T* R[3];          // GCR residual buffers (rotating)
  T* XL;            // linearisation copy (analytic JVP) in T, or nullptr to read X
  T* P;             // kmax + 1 slots of length L: GCR p~_k / GMRES basis v~_i
  T* AP;            // kmax slots: GCR Ap~_k / GMRES slot 0 = w
  double* hbuf;     // per-block Hessenberg / Givens scratch (GMRES)
  int kmax;
  long L;           // ncomp * npad
  unsigned long long* prof;   // phase timers (diagnostics), or nullptr
};

template <typename T>
struct Shared {
  double* acc;      // [kWarps][nacc]
  double* blk;      // [nacc]
  double* red;      // [nacc]
  double* gam;      // [kmax + 1] coefficients of the current orthogonalisation
  double* cj;       // [kmax + 1] solution coefficients
  double* sj;       // [kmax + 1] normalisation scales
  int nacc;
};

// Hessenberg scratch layout per block (GMRES): R column-major (kmax+1) x kmax,
// then g[kmax+1], cs[kmax], sn[kmax].
__host__ __device__ __forceinline__ long hbuf_stride(int kmax) {
  return (long)(kmax + 1) * kmax + (kmax + 1) + 2L * kmax;
}

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

// ---------------------------------------------------------------------------
// Block accumulators and diagnostics
// ---------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ void acc_zero(Shared<T>& sm) {
  for (int t = threadIdx.x; t < kWarps * sm.nacc; t += blockDim.x) sm.acc[t] = 0.0;
  __syncthreads();
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

// Phase timers (diagnostics, off when prof is null): thread 0 of each block
// adds the global time since its previous mark to a slot.  Slots 0..15 are
// block 0's phase totals; 64 + 1024 * s + block holds per-block totals of
// the compute phases s = 0 (Krylov stencil) and s = 1 (orthogonalisation).
enum ProfSlot : int { PF_PREDICT = 0, PF_NEWTON_RHS = 1, PF_STENCIL_A = 2, PF_STENCIL_B = 3, PF_ORTH = 4,
                      PF_UPDATE = 5, PF_BASE = 6, PF_WAIT_STENCIL = 8, PF_WAIT_ORTH = 9, PF_WAIT_OTHER = 10,
                      PF_COUNT_STENCIL = 12, PF_COUNT_ORTH = 13 };
__device__ __forceinline__ void prof_lap(unsigned long long* prof, int slot, int per_block = -1) {
  if (!prof || threadIdx.x != 0) return;
  __shared__ unsigned long long s_t;
  unsigned long long now = global_ns();
  if (slot >= 0) {
    unsigned long long dt = now - s_t;
    if (blockIdx.x == 0) prof[slot] += dt;
    if (per_block >= 0 && blockIdx.x < 1024) prof[64 + 1024 * per_block + blockIdx.x] += dt;
  }
  s_t = now;
}
__device__ __forceinline__ void prof_count(unsigned long long* prof, int slot) {
  if (prof && threadIdx.x == 0 && blockIdx.x == 0) prof[slot] += 1;
}

// ---------------------------------------------------------------------------
// Vector access: four consecutive elements (one float4, or two double2).
// Component arrays are npad long with npad a multiple of 128, so every
// 4-element chunk is 16-byte aligned.  Plain (coherent) loads: these arrays
// are written by other blocks earlier in the same launch.
// ---------------------------------------------------------------------------

template <typename T> struct Q4 { T a, b, c, d; };

__device__ __forceinline__ Q4<float> ldq(const float* p) {
  float4 v = *reinterpret_cast<const float4*>(p);
  return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ Q4<double> ldq(const double* p) {
  double2 u = reinterpret_cast<const double2*>(p)[0], v = reinterpret_cast<const double2*>(p)[1];
  return {u.x, u.y, v.x, v.y};
}
__device__ __forceinline__ void stq(float* p, const double* v) {
  *reinterpret_cast<float4*>(p) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
}
__device__ __forceinline__ void stq(double* p, const double* v) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}
template <typename T>
__device__ __forceinline__ double dot4(const Q4<T>& u, const Q4<T>& v) {
  return (double)u.a * (double)v.a + (double)u.b * (double)v.b + (double)u.c * (double)v.c +
         (double)u.d * (double)v.d;
}

// Stored vectors per group in the multi-vector loops: enough independent
// loads in flight to cover HBM latency without spilling.
template <typename T> struct Group { static constexpr int JB = 8; };
template <> struct Group<double> { static constexpr int JB = 4; };

__device__ __forceinline__ int gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int gthreads() { return gridDim.x * blockDim.x; }

// Visit every interior node once, by 128-node regions per warp: first the
// region's fast nodes (lane l: base + 32 t + l), then its slow nodes from the
// compacted list.  f(d, nf, slow).
template <class F>
__device__ __forceinline__ void for_nodes(const Grid& g, F&& f) {
  const int lane = threadIdx.x & 31;
  const int wid = blockIdx.x * kWarps + (threadIdx.x >> 5);
  const int nw = gridDim.x * kWarps;
  const int nreg = g.npad / 128;
  for (int rg = wid; rg < nreg; rg += nw) {
#pragma unroll 1
    for (int t = 0; t < 4; ++t) {
      int d = rg * 128 + t * 32 + lane;
      if (d < g.n) {
        uint8_t nf = g.nflags[d];
        if (!(nf & NF_SLOW)) f(d, nf, false);
      }
    }
    for (int s = g.slow_off[rg] + lane; s < g.slow_off[rg + 1]; s += 32) {
      int d = g.slow_idx[s];
      f(d, g.nflags[d], true);
    }
  }
}

// Projections <W, Q_j> for j < nq (slots 0..nq-1), over the regions this warp
// visited in for_nodes (so it reads back only its own writes of W).
template <typename T>
__device__ __noinline__ void region_dots(const Grid& g, Shared<T>& sm, const T* W, const T* Q, long L, int nq) {
  constexpr int JB = Group<T>::JB;
  const int lane = threadIdx.x & 31;
  const int wid = blockIdx.x * kWarps + (threadIdx.x >> 5);
  const int nw = gridDim.x * kWarps;
  const int nreg = g.npad / 128;
  __syncwarp();
  for (int j0 = 0; j0 < nq; j0 += JB) {
    double acc[JB];
#pragma unroll
    for (int jj = 0; jj < JB; ++jj) acc[jj] = 0.0;
    for (int rg = wid; rg < nreg; rg += nw) {
      const long base = (long)rg * 128 + 4 * lane;
      for (int c = 0; c < g.ncomp; ++c) {
        const long e = (long)c * g.npad + base;
        Q4<T> w4 = ldq(W + e);
        Q4<T> a4[JB];
#pragma unroll
        for (int jj = 0; jj < JB; ++jj)
          a4[jj] = (j0 + jj < nq) ? ldq(Q + (long)(j0 + jj) * L + e) : Q4<T>{0, 0, 0, 0};
#pragma unroll
        for (int jj = 0; jj < JB; ++jj) acc[jj] += dot4(w4, a4[jj]);
      }
    }
#pragma unroll
    for (int jj = 0; jj < JB; ++jj)
      if (j0 + jj < nq) acc_add(sm.acc, sm.nacc, j0 + jj, acc[jj]);
  }
}

// RHS of the FP64 state at node d through the fast or slow path.
template <bool D3>
__device__ __forceinline__ void rhs64(const Grid& g, const SrcVec<double, double>& s, const BTerms<double>& b, int d,
                                      uint8_t nf, bool slow, double o[5]) {
  if (slow) rhs_slow<double, D3>(g, s, b, d, nf, o);
  else rhs_fast<double, D3>(g, s, d, nf, o);
}

// ---------------------------------------------------------------------------
// Passes.  Each thread accumulates its partial sums in registers and reduces
// them once per pass (fixed assignment of work to threads, so sums repeat
// bitwise for a fixed grid).
// ---------------------------------------------------------------------------

// f = rhs(X); Xn = X + dt f; G = X + dt/2 f   (integrators.py:156-158)
template <typename T, bool D3>
__device__ __noinline__ void pass_predict(const StepArgs<T>& A, const double* X, double* Xn, double dt, BTerms<double> b) {
  const Grid& g = A.g;
  SrcVec<double, double> sx{X, g.npad};
  for_nodes(g, [&](int d, uint8_t nf, bool slow) {
    double o[5];
    rhs64<D3>(g, sx, b, d, nf, slow, o);
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) {
      long e = (long)c * g.npad + d;
      double xv = X[e];
      Xn[e] = xv + dt * o[c];
      A.G[e] = xv + (dt / 2.0) * o[c];
    }
  });
}

// f = rhs(x); g = x - dt/2 f - gamma; r0 = -g (as T);
// slots: 0 ||r0||^2, 1 ||x||^2, 2 max|g| (max slot)
template <typename T, bool D3>
__device__ __noinline__ void pass_newton_rhs(const StepArgs<T>& A, Shared<T>& sm, const double* x, T* r0, double dt,
                                BTerms<double> b) {
  const Grid& g = A.g;
  SrcVec<double, double> sx{x, g.npad};
  double s_r = 0.0, s_x = 0.0, m_g = 0.0;
  for_nodes(g, [&](int d, uint8_t nf, bool slow) {
    double o[5];
    rhs64<D3>(g, sx, b, d, nf, slow, o);
    double gv[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) {
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
    double m = nonfinite_guard(hypot(gv[0], gv[1]));
#pragma unroll
    for (int c = 2; c < (D3 ? 5 : 4); ++c) m = fmax(m, nonfinite_guard(fabs(gv[c])));
    m_g = fmax(m_g, m);
  });
  acc_add(sm.acc, sm.nacc, 0, s_r);
  acc_add(sm.acc, sm.nacc, 1, s_x);
  acc_max(sm.acc, sm.nacc, 2, m_g);
}

// w = A v at node d, v given by source sp (T) and, for the finite-difference
// product, by sfd = x + eps_eff * v (FP64).  scale multiplies the whole
// result (GMRES applies the basis scale here).
template <typename T, bool D3, class SP, class SFD>
__device__ __forceinline__ void apply_A(const StepArgs<T>& A, const SP& sp, const SFD& sfd, double scale,
                                        const double* x, double dth, double eps, BTerms<double> b, int jvp_mode,
                                        int d, uint8_t nf, bool slow, double w[5]) {
  const Grid& g = A.g;
  double v[5];
#pragma unroll
  for (int c = 0; c < (D3 ? 5 : 4); ++c) v[c] = (double)sp(c, d);
  if (jvp_mode == JVP_FD) {
    double o[5];
    if (slow) rhs_slow<double, D3>(g, sfd, b, d, nf, o);
    else rhs_fast<double, D3>(g, sfd, d, nf, o);
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) w[c] = scale * v[c] - dth * ((o[c] - A.F[(long)c * g.npad + d]) / eps);
  } else {
    BTerms<T> bt{(T)b.czxy, (T)b.cyzx, (T)b.cxyz};
    T o[5];
    if (A.XL) {
      SrcVec<T, T> sxl{A.XL, g.npad};
      if (slow) jvp_slow<T, D3>(g, sxl, bt, sp, d, nf, o);
      else jvp_fast<T, D3>(g, sxl, sp, d, nf, o);
    } else {
      SrcVec<T, double> sxd{x, g.npad};
      if (slow) jvp_slow<T, D3>(g, sxd, bt, sp, d, nf, o);
      else jvp_fast<T, D3>(g, sxd, sp, d, nf, o);
    }
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) w[c] = scale * (v[c] - dth * (double)o[c]);
  }
}

// GCR stencil pass for direction k (1-based).
//   r_{k-1} = Rin - a_prev * Ap~_{k-1}   (k > 1; written to Rout, ||r||^2 -> slot k-1)
//   w       = r - dt/2 J(x) r            (written to Ap~_k)
//   slot j-1 (j < k) <- <w, Ap~_j>
template <typename T, bool D3>
__device__ __noinline__ void pass_gcr_stencil(const StepArgs<T>& A, Shared<T>& sm, int k, const T* Rin, T* Rout, double a_prev,
                                 const double* x, double dt, double eps, BTerms<double> b, int jvp_mode,
                                 bool norm_only) {
  const Grid& g = A.g;
  const long L = A.L;
  const T* APprev = k > 1 ? A.AP + (long)(k - 2) * L : nullptr;
  T* W = A.AP + (long)(k - 1) * L;
  const double dth = dt / 2.0;
  const T ta = (T)a_prev;
  double s_r = 0.0;
  SrcAxpy<T, T> sp{Rin, APprev, ta, g.npad};
  SrcFD<T> sfd{x, Rin, APprev, a_prev, eps, g.npad};
  for_nodes(g, [&](int d, uint8_t nf, bool slow) {
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) {
      long e = (long)c * g.npad + d;
      T rt = sp(c, d);
      if (APprev) Rout[e] = rt;
      s_r += (double)rt * (double)rt;
    }
    if (norm_only) return;
    double w[5];
    apply_A<T, D3>(A, sp, sfd, 1.0, x, dth, eps, b, jvp_mode, d, nf, slow, w);
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) W[(long)c * g.npad + d] = (T)w[c];
  });
  if (k > 1) acc_add(sm.acc, sm.nacc, k - 1, s_r);
  if (norm_only) return;
  if (A.prof) {
    __syncthreads();
    prof_lap(A.prof, PF_STENCIL_A);
  }
  region_dots<T>(g, sm, W, A.AP, L, k - 1);
}

// GCR orthogonalisation pass for direction k:
//   P~_k  = r - sum_j gam_j P~_j,  Ap~_k = w - sum_j gam_j Ap~_j
//   slot 0 <- ||Ap~_k||^2, slot 1 <- <r, Ap~_k>
template <typename T>
__device__ __noinline__ void pass_gcr_orth(const StepArgs<T>& A, Shared<T>& sm, int k, const T* Rk) {
  const long L = A.L;
  T* Pk = A.P + (long)(k - 1) * L;
  T* APk = A.AP + (long)(k - 1) * L;
  constexpr int JB = Group<T>::JB;
  const long nq = L / 4;
  double s_q = 0.0, s_rq = 0.0;
  for (long q = gtid(); q < nq; q += gthreads()) {
    const long e = 4 * q;
    Q4<T> r4 = ldq(Rk + e), w4 = ldq(APk + e);
    double p[4] = {(double)r4.a, (double)r4.b, (double)r4.c, (double)r4.d};
    double v[4] = {(double)w4.a, (double)w4.b, (double)w4.c, (double)w4.d};
    for (int j0 = 0; j0 < k - 1; j0 += JB) {
      Q4<T> pj[JB], aj[JB];
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) {
        bool on = j0 + jj < k - 1;
        pj[jj] = on ? ldq(A.P + (long)(j0 + jj) * L + e) : Q4<T>{0, 0, 0, 0};
        aj[jj] = on ? ldq(A.AP + (long)(j0 + jj) * L + e) : Q4<T>{0, 0, 0, 0};
      }
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) {
        double gm = (j0 + jj < k - 1) ? sm.gam[j0 + jj] : 0.0;
        p[0] -= gm * (double)pj[jj].a; p[1] -= gm * (double)pj[jj].b;
        p[2] -= gm * (double)pj[jj].c; p[3] -= gm * (double)pj[jj].d;
        v[0] -= gm * (double)aj[jj].a; v[1] -= gm * (double)aj[jj].b;
        v[2] -= gm * (double)aj[jj].c; v[3] -= gm * (double)aj[jj].d;
      }
    }
    double vr[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) vr[t] = (double)(T)v[t];
    stq(Pk + e, p);
    stq(APk + e, vr);
    s_q += vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2] + vr[3] * vr[3];
    s_rq += (double)r4.a * vr[0] + (double)r4.b * vr[1] + (double)r4.c * vr[2] + (double)r4.d * vr[3];
  }
  acc_add(sm.acc, sm.nacc, 0, s_q);
  acc_add(sm.acc, sm.nacc, 1, s_rq);
}

// Arnoldi stencil pass for basis vector j (1-based): w = A v_j with
// v_j = s_j v~_j (w stored in AP slot 0), then slots i-1 <- <w, v~_i>, i <= j.
template <typename T, bool D3>
__device__ __noinline__ void pass_arnoldi_stencil(const StepArgs<T>& A, Shared<T>& sm, int j, const double* x, double dt,
                                     double eps, BTerms<double> b, int jvp_mode) {
  const Grid& g = A.g;
  const long L = A.L;
  const T* V = A.P + (long)(j - 1) * L;
  T* W = A.AP;
  const double sj = sm.sj[j - 1];
  const double dth = dt / 2.0;
  SrcVec<T, T> sp{V, g.npad};
  SrcFD<T> sfd{x, V, nullptr, 0.0, eps * sj, g.npad};
  for_nodes(g, [&](int d, uint8_t nf, bool slow) {
    double w[5];
    apply_A<T, D3>(A, sp, sfd, sj, x, dth, eps, b, jvp_mode, d, nf, slow, w);
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) W[(long)c * g.npad + d] = (T)w[c];
  });
  if (A.prof) {
    __syncthreads();
    prof_lap(A.prof, PF_STENCIL_A);
  }
  region_dots<T>(g, sm, W, A.P, L, j);
}

// Arnoldi orthogonalisation: v~_{j+1} = w - sum_{i<=j} gam_i v~_i; slot 0 <- ||v~_{j+1}||^2
template <typename T>
__device__ __noinline__ void pass_arnoldi_orth(const StepArgs<T>& A, Shared<T>& sm, int j) {
  const long L = A.L;
  const T* W = A.AP;
  T* Vn = A.P + (long)j * L;
  constexpr int JB = Group<T>::JB;
  const long nq = L / 4;
  double s_q = 0.0;
  for (long q = gtid(); q < nq; q += gthreads()) {
    const long e = 4 * q;
    Q4<T> w4 = ldq(W + e);
    double v[4] = {(double)w4.a, (double)w4.b, (double)w4.c, (double)w4.d};
    for (int i0 = 0; i0 < j; i0 += JB) {
      Q4<T> vi[JB];
#pragma unroll
      for (int ii = 0; ii < JB; ++ii) vi[ii] = (i0 + ii < j) ? ldq(A.P + (long)(i0 + ii) * L + e) : Q4<T>{0, 0, 0, 0};
#pragma unroll
      for (int ii = 0; ii < JB; ++ii) {
        double gm = (i0 + ii < j) ? sm.gam[i0 + ii] : 0.0;
        v[0] -= gm * (double)vi[ii].a; v[1] -= gm * (double)vi[ii].b;
        v[2] -= gm * (double)vi[ii].c; v[3] -= gm * (double)vi[ii].d;
      }
    }
    double vr[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) vr[t] = (double)(T)v[t];
    stq(Vn + e, vr);
    s_q += vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2] + vr[3] * vr[3];
  }
  acc_add(sm.acc, sm.nacc, 0, s_q);
}

// dx = sum_j cj_j Q_j; x += dx (if x) and/or dout = dx; slot 0 <- max |dx|
// (complex modulus on psi entries).  Lane work: four consecutive nodes.
template <typename T>
__device__ __noinline__ void pass_update(const StepArgs<T>& A, Shared<T>& sm, const T* Q, double* x, int nk, double* dout) {
  const Grid& g = A.g;
  const long L = A.L;
  constexpr int JB = Group<T>::JB;
  const long nq = g.npad / 4;
  double m = 0.0;
  for (long q = gtid(); q < nq; q += gthreads()) {
    const long base = 4 * q;
    double dre[4] = {0, 0, 0, 0};
    for (int c = 0; c < g.ncomp; ++c) {
      const long e = (long)c * g.npad + base;
      double dl[4] = {0, 0, 0, 0};
      for (int j0 = 0; j0 < nk; j0 += JB) {
        Q4<T> pj[JB];
#pragma unroll
        for (int jj = 0; jj < JB; ++jj)
          pj[jj] = (j0 + jj < nk) ? ldq(Q + (long)(j0 + jj) * L + e) : Q4<T>{0, 0, 0, 0};
#pragma unroll
        for (int jj = 0; jj < JB; ++jj) {
          double cj = (j0 + jj < nk) ? sm.cj[j0 + jj] : 0.0;
          dl[0] += cj * (double)pj[jj].a; dl[1] += cj * (double)pj[jj].b;
          dl[2] += cj * (double)pj[jj].c; dl[3] += cj * (double)pj[jj].d;
        }
      }
      if (x) {
        Q4<double> x4 = ldq(x + e);
        double xn[4] = {x4.a + dl[0], x4.b + dl[1], x4.c + dl[2], x4.d + dl[3]};
        stq(x + e, xn);
      }
      if (dout) stq(dout + e, dl);
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        if (c == 0) dre[t] = dl[t];
        else if (c == 1) m = fmax(m, nonfinite_guard(hypot(dre[t], dl[t])));
        else m = fmax(m, nonfinite_guard(fabs(dl[t])));
      }
    }
  }
  acc_max(sm.acc, sm.nacc, 0, m);
}

// rhs(x) into F (and the linearisation copy); slot 0 <- ||x||^2
template <typename T, bool D3>
__device__ __noinline__ void pass_base(const StepArgs<T>& A, Shared<T>& sm, const double* x, BTerms<double> b) {
  const Grid& g = A.g;
  SrcVec<double, double> sx{x, g.npad};
  double s_x = 0.0;
  for_nodes(g, [&](int d, uint8_t nf, bool slow) {
    double o[5];
    rhs64<D3>(g, sx, b, d, nf, slow, o);
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) {
      long e = (long)c * g.npad + d;
      A.F[e] = o[c];
      double xv = x[e];
      if (A.XL) A.XL[e] = (T)xv;
      s_x += xv * xv;
    }
  });
  acc_add(sm.acc, sm.nacc, 0, s_x);
}

// ---------------------------------------------------------------------------
// Solvers
// ---------------------------------------------------------------------------

struct KrylovOut {
  bool ok;        // converged (reference: non-empty solution)
  int nk;         // directions in the solution
  int status;     // ST_OK, ST_NOCONV, ST_KMAX, ST_TIMEOUT, ST_NONFINITE
};

// Reduce `nslot` accumulators of this block across the grid (slots >= nsum: max).
#define TDGL_REDUCE(nslot, nsum, on_fail)                                       \
  do {                                                                          \
    acc_fold(sm, (nslot), (nsum));                                              \
    if (!grid_reduce(A.sy, sm.blk, (nslot), (nsum), sm.red)) { on_fail; }       \
  } while (0)

// GCR on (I - dt/2 J(x)) d = r0, r0 in A.R[0] (||r0|| = rho0); solution
// sum_j sm.cj[j] P~_j, j < nk.
template <typename T, bool D3>
__device__ KrylovOut krylov_gcr(const StepArgs<T>& A, Shared<T>& sm, const double* x, double xnorm, double rho0,
                                double dt, double tol, int max_iter, double eps_mf, int jvp_mode, BTerms<double> b,
                                long long& jvp_count) {
  KrylovOut out{true, 0, ST_OK};
  if (!isfinite(rho0) || !isfinite(xnorm)) return KrylovOut{false, 0, ST_NONFINITE};
  if (rho0 == 0.0) return out;                 // tgcr.py:121-122
  double rho = rho0, rho_est = rho0, a_prev = 0.0;
  int rin = 0, k = 0;
  while (true) {
    if (!(rho / rho0 > tol)) break;
    if (k >= max_iter) break;
    if (k + 1 > A.kmax) return KrylovOut{false, k, ST_KMAX};
    ++k;
    int rout = k > 1 ? (rin + 1) % 3 : rin;
    double eps = eps_mf * (1.0 + xnorm) / rho_est;
    acc_zero(sm);
    pass_gcr_stencil<T, D3>(A, sm, k, A.R[rin], A.R[rout], a_prev, x, dt, eps, b, jvp_mode, false);
    prof_lap(A.prof, PF_STENCIL_B, 0);
    TDGL_REDUCE(k, k, return (KrylovOut{false, k, ST_TIMEOUT}));
    prof_lap(A.prof, PF_WAIT_STENCIL);
    prof_count(A.prof, PF_COUNT_STENCIL);
    ++jvp_count;
    if (k > 1) {
      rho = sqrt(sm.red[k - 1]);
      rin = rout;
      if (!isfinite(rho)) return KrylovOut{false, k, ST_NONFINITE};
      if (!(rho / rho0 > tol)) { --k; break; }
    }
    for (int t = threadIdx.x; t < k - 1; t += blockDim.x) sm.gam[t] = sm.red[t] * sm.sj[t] * sm.sj[t];
    __syncthreads();
    acc_zero(sm);
    pass_gcr_orth<T>(A, sm, k, A.R[rin]);
    prof_lap(A.prof, PF_ORTH, 1);
    TDGL_REDUCE(2, 2, return (KrylovOut{false, k, ST_TIMEOUT}));
    prof_lap(A.prof, PF_WAIT_ORTH);
    prof_count(A.prof, PF_COUNT_ORTH);
    double nu = sqrt(sm.red[0]);
    if (!(nu >= 1e-14)) {                       // tgcr.py:141-142 (also stops on NaN)
      if (!isfinite(nu)) return KrylovOut{false, k, ST_NONFINITE};
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
      acc_zero(sm);
      pass_gcr_stencil<T, D3>(A, sm, k + 1, A.R[rin], A.R[rout2], a_prev, x, dt, eps, b, jvp_mode, true);
      TDGL_REDUCE(k + 1, k + 1, return (KrylovOut{false, k, ST_TIMEOUT}));
      rho = sqrt(sm.red[k]);
      rin = rout2;
      break;
    }
  }
  out.nk = k;
  out.ok = !(rho > tol * rho0);               // tgcr.py:154-155
  out.status = out.ok ? ST_OK : ST_NOCONV;
  return out;
}

// GMRES on the same system: basis v~_1 = r0 in A.P slot 0 (scale 1/rho0).
// Solution sum_i sm.cj[i] v~_{i+1}, i < nk.
template <typename T, bool D3>
__device__ KrylovOut krylov_gmres(const StepArgs<T>& A, Shared<T>& sm, const double* x, double xnorm, double rho0,
                                  double dt, double tol, int max_iter, double eps_mf, int jvp_mode,
                                  BTerms<double> b, long long& jvp_count) {
  if (!isfinite(rho0) || !isfinite(xnorm)) return KrylovOut{false, 0, ST_NONFINITE};
  if (rho0 == 0.0) return KrylovOut{true, 0, ST_OK};
  __shared__ double s_rho;
  const int km = A.kmax;
  double* H = A.hbuf + (long)blockIdx.x * hbuf_stride(km);   // R column-major, ld = km + 1
  double* gv = H + (long)(km + 1) * km;
  double* cs = gv + (km + 1);
  double* sn = cs + km;
  if (threadIdx.x == 0) {
    sm.sj[0] = 1.0 / rho0;
    gv[0] = rho0;
  }
  __syncthreads();
  double rho = rho0;
  // eps = eps_mf (1 + |x|) / |v|, |v| = 1 (tgcr.py:129)
  const double eps = eps_mf * (1.0 + xnorm);
  int j = 0;
  while (true) {
    if (!(rho / rho0 > tol)) break;
    if (j >= max_iter) break;
    if (j + 1 > km) return KrylovOut{false, j, ST_KMAX};
    ++j;
    acc_zero(sm);
    pass_arnoldi_stencil<T, D3>(A, sm, j, x, dt, eps, b, jvp_mode);
    prof_lap(A.prof, PF_STENCIL_B, 0);
    TDGL_REDUCE(j, j, return (KrylovOut{false, j, ST_TIMEOUT}));
    prof_lap(A.prof, PF_WAIT_STENCIL);
    prof_count(A.prof, PF_COUNT_STENCIL);
    ++jvp_count;
    double* col = H + (long)(j - 1) * (km + 1);
    for (int i = threadIdx.x; i < j; i += blockDim.x) {
      double h = sm.red[i] * sm.sj[i];       // h_ij = <w, v_i>
      sm.gam[i] = h * sm.sj[i];              // coefficient on v~_i
      col[i] = h;
    }
    __syncthreads();
    acc_zero(sm);
    pass_arnoldi_orth<T>(A, sm, j);
    prof_lap(A.prof, PF_ORTH, 1);
    TDGL_REDUCE(1, 1, return (KrylovOut{false, j, ST_TIMEOUT}));
    prof_lap(A.prof, PF_WAIT_ORTH);
    prof_count(A.prof, PF_COUNT_ORTH);
    double hn = sqrt(sm.red[0]);
    if (!isfinite(hn)) return KrylovOut{false, j, ST_NONFINITE};
    if (threadIdx.x == 0) {
      sm.sj[j] = hn > 0.0 ? 1.0 / hn : 0.0;
      col[j] = hn;
      for (int i = 0; i + 1 < j; ++i) {          // earlier rotations
        double a = col[i], c2 = col[i + 1];
        col[i] = cs[i] * a + sn[i] * c2;
        col[i + 1] = -sn[i] * a + cs[i] * c2;
      }
      double a = col[j - 1], c2 = col[j];
      double r = hypot(a, c2);
      double c = r > 0.0 ? a / r : 1.0, s = r > 0.0 ? c2 / r : 0.0;
      cs[j - 1] = c;
      sn[j - 1] = s;
      col[j - 1] = r;
      col[j] = 0.0;
      gv[j] = -s * gv[j - 1];
      gv[j - 1] = c * gv[j - 1];
      s_rho = fabs(gv[j]);
    }
    __syncthreads();
    rho = s_rho;
    if (!(hn > 0.0)) break;                       // exact solution in the current space
  }
  // d = V y with R y = g (back substitution on thread 0)
  if (threadIdx.x == 0) {
    for (int i = j - 1; i >= 0; --i) {
      double acc = gv[i];
      for (int l = i + 1; l < j; ++l) acc -= H[(long)l * (km + 1) + i] * sm.gam[l];
      sm.gam[i] = acc / H[(long)i * (km + 1) + i];
    }
    for (int i = 0; i < j; ++i) sm.cj[i] = sm.gam[i] * sm.sj[i];
  }
  __syncthreads();
  KrylovOut out{true, j, ST_OK};
  out.ok = !(rho > tol * rho0);
  out.status = out.ok ? ST_OK : ST_NOCONV;
  return out;
}

template <typename T, bool D3>
__device__ KrylovOut krylov(const StepArgs<T>& A, Shared<T>& sm, int kind, const double* x, double xnorm,
                            double rho0, double dt, double tol, int max_iter, double eps_mf, int jvp_mode,
                            BTerms<double> b, long long& jvp_count) {
  if (kind == KRY_GCR)
    return krylov_gcr<T, D3>(A, sm, x, xnorm, rho0, dt, tol, max_iter, eps_mf, jvp_mode, b, jvp_count);
  return krylov_gmres<T, D3>(A, sm, x, xnorm, rho0, dt, tol, max_iter, eps_mf, jvp_mode, b, jvp_count);
}

// First vector of the Krylov solve: GCR keeps r0 in R[0], GMRES in basis slot 0.
// The solution is a combination of P slots in both cases.
template <typename T>
__device__ __forceinline__ T* r0_buffer(const StepArgs<T>& A, int kind) {
  return kind == KRY_GCR ? A.R[0] : A.P;
}

// Newton on g(x) = x - dt/2 f(x) - gamma from x; returns converged.
template <typename T, bool D3>
__device__ bool newton(const StepArgs<T>& A, Shared<T>& sm, Ctl& c, double* x, double dt, BTerms<double> b,
                       int& status, int& iters) {
  T* r0 = r0_buffer(A, c.krylov);
  acc_zero(sm);
  prof_lap(A.prof, -1);
  pass_newton_rhs<T, D3>(A, sm, x, r0, dt, b);
  prof_lap(A.prof, PF_NEWTON_RHS);
  TDGL_REDUCE(3, 2, { status = ST_TIMEOUT; return false; });
  prof_lap(A.prof, PF_WAIT_OTHER);
  c.rhs_evals += 1;
  double rho0 = sqrt(sm.red[0]), xnorm = sqrt(sm.red[1]);
  for (int k = 1; k <= c.newton_max_iter; ++k) {
    long long jv = 0;
    KrylovOut ko = krylov<T, D3>(A, sm, c.krylov, x, xnorm, rho0, dt, c.tol_gcr, c.krylov_max_iter, c.eps_mf,
                                 c.jvp_mode, b, jv);
    c.jvp_evals += jv;
    c.krylov_iters += ko.nk;
    c.krylov_sq += (long long)ko.nk * ko.nk;
    c.krylov_last = ko.nk;
    if (ko.nk > c.max_krylov) c.max_krylov = ko.nk;
    if (ko.status == ST_TIMEOUT || ko.status == ST_KMAX || ko.status == ST_NONFINITE) {
      status = ko.status;
      iters = k;
      return false;
    }
    if (!ko.ok) { status = ST_NOCONV; iters = k; return false; }   // newton.py:103-106
    acc_zero(sm);
    pass_update<T>(A, sm, A.P, x, ko.nk, nullptr);
    prof_lap(A.prof, PF_UPDATE);
    TDGL_REDUCE(1, 0, { status = ST_TIMEOUT; return false; });
    prof_lap(A.prof, PF_WAIT_OTHER);
    double dxn = sm.red[0];
    acc_zero(sm);
    pass_newton_rhs<T, D3>(A, sm, x, r0, dt, b);
    prof_lap(A.prof, PF_NEWTON_RHS);
    TDGL_REDUCE(3, 2, { status = ST_TIMEOUT; return false; });
    prof_lap(A.prof, PF_WAIT_OTHER);
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

template <typename T, bool D3>
__device__ void stepper_body(const StepArgs<T>& A, Shared<T>& sm, Ctl& c, int& status) {
  const Grid& g = A.g;
  if (c.run_mode == RUN_TGCR) {
    // one linear solve: x_lin in X[0], b in the first Krylov vector; solution (FP64) into D
    BTerms<double> b = bterms(g, c.Bx, c.By, c.Bz);
    const T* r0 = r0_buffer(A, c.krylov);
    acc_zero(sm);
    pass_base<T, D3>(A, sm, A.X[0], b);
    double sb = 0.0;
    for (long e = gtid(); e < A.L; e += gthreads()) {
      double v = (double)r0[e];
      sb += v * v;
    }
    acc_add(sm.acc, sm.nacc, 1, sb);
    TDGL_REDUCE(2, 2, { status = ST_TIMEOUT; return; });
    c.rhs_evals += 1;
    double xnorm = sqrt(sm.red[0]), rho0 = sqrt(sm.red[1]);
    long long jv = 0;
    KrylovOut ko = krylov<T, D3>(A, sm, c.krylov, A.X[0], xnorm, rho0, c.dt, c.tol_gcr, c.krylov_max_iter,
                                 c.eps_mf, c.jvp_mode, b, jv);
    c.jvp_evals += jv;
    c.krylov_last = ko.nk;
    c.krylov_iters += ko.nk;
    c.krylov_sq += (long long)ko.nk * ko.nk;
    status = ko.status;
    if (ko.status == ST_OK || ko.status == ST_NOCONV) {
      acc_zero(sm);
      pass_update<T>(A, sm, A.P, nullptr, ko.nk, A.D);
      TDGL_REDUCE(1, 0, { status = ST_TIMEOUT; return; });
    }
  } else if (c.run_mode == RUN_NEWTON) {
    // one Newton solve: iterate in X[c.cur], gamma in G
    BTerms<double> b = bterms(g, c.Bx, c.By, c.Bz);
    int iters = 0;
    bool ok = newton<T, D3>(A, sm, c, A.X[c.cur], c.dt, b, status, iters);
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
      prof_lap(A.prof, -1);
      pass_predict<T, D3>(A, Xs, Xi, dta, b);
      prof_lap(A.prof, PF_PREDICT);
      c.rhs_evals += 1;
      if (!grid_sync(A.sy, sm.blk)) { status = ST_TIMEOUT; break; }
      int st = ST_OK, iters = 0;
      bool ok = newton<T, D3>(A, sm, c, Xi, dta, b, st, iters);
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
  sm.cj = sm.gam + (A.kmax + 1);
  sm.sj = sm.cj + (A.kmax + 1);
  Ctl c = *A.ctl;     // every block keeps an identical copy of the control state
  int status = ST_OK;
  if (A.g.is3d) stepper_body<T, true>(A, sm, c, status);
  else stepper_body<T, false>(A, sm, c, status);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c.status = status;
    *A.ctl = c;
  }
}

// Dynamic shared memory of k_stepper in bytes.
inline size_t stepper_smem(int kmax) {
  int nacc = kmax + 4;
  return (size_t)(kWarps * nacc + 2 * nacc + 3 * (kmax + 1)) * sizeof(double);
}

}  // namespace tdgl
