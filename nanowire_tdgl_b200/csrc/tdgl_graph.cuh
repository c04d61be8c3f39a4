// Graph executor of the trapezoidal stepper (GMRES inner solve).
//
// The same algorithm as the persistent stepper (src/tdgl3d/solvers/
// integrators.py:92-206, newton.py:76-120, tgcr.py:96-156 with the Krylov
// solve in its GMRES form), expressed as small kernels sequenced by one CUDA
// graph with nested conditional WHILE nodes:
//
//   STEP while { step_begin, prepare, predict, newton_rhs, newton_init,
//     NEWTON while { KRYLOV while { stencil, dots, fin_dots, orth, fin_orth },
//                    newton_solve, update, newton_rhs, newton_check },
//     accept, step_end }
//
// Grid kernels stream over the vectors and write per-block partial sums;
// one-block kernels reduce them in a fixed order (repeatable sums), take every
// control decision on the device and set the conditional handles.  No kernel
// waits on another block, so nothing can spin; every loop also has a hard
// iteration cap that aborts the launch with a status.
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

enum GStatus : int { GS_OK = 0, GS_NOCONV = 1, GS_DTMIN = 2, GS_KMAX = 3, GS_NONFINITE = 4, GS_CAP = 5 };

// Device control block of the graph executor.
struct GDev {
  // inputs for one launch
  double t, dt_cur, t_stop, dt, dt_min, tol_f, tol_dx, tol_gcr, eps_mf;
  double Bx, By, Bz, t_on_fraction, ramp_fraction, t_field_stop;
  int ramp, field_const, newton_max_iter, krylov_max_iter, adaptive, jvp_mode, max_steps;
  // state
  double dta, czxy, cyzx, cxyz;    // current step and its face offsets
  double rho0, rho, xnorm, gnorm, dxnorm, eps;
  int steps, status, newton_k, newton_failed, accepted, j;
  long long watchdog, watchdog_cap;   // loop iterations of this launch and their hard limit
  // counters
  long long newton_iters, krylov_iters, krylov_sq, rhs_evals, jvp_evals, rejections;
  int max_krylov, krylov_last;
};

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
template <typename T, bool D3>
__device__ __forceinline__ void write_eff(const Grid& g, T* E, long npf, int i, int j, int k, const double* v,
                                          double czxy, double cyzx, double cxyz) {
  const long m = full_index(g, i, j, k);
  const uint8_t lf = g.lflags ? g.lflags[m] : 0;
  const double tx = (i == g.Nx - 1) ? 0.0 : v[2];
  const double ty = (j == g.Ny - 1) ? 0.0 : v[3];
  const double tz = (D3 && k == g.Nz - 1) ? 0.0 : (D3 ? v[4] : 0.0);
  E[m] = (T)v[0];
  E[npf + m] = (T)v[1];
  E[2 * npf + m] = (lf & LF_HX) ? T(0) : (T)tx;
  E[3 * npf + m] = (lf & LF_HY) ? T(0) : (T)ty;
  if (D3) E[4 * npf + m] = (lf & LF_HZ) ? T(0) : (T)tz;
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

// Stop every loop of the graph with a status (one-block kernels only).
template <typename T>
__device__ __forceinline__ void abort_all(const GArgs<T>& A, int status) {
  if (threadIdx.x == 0) {
    if (A.dev->status == GS_OK) A.dev->status = status;
    cudaGraphSetConditional(A.h_krylov, 0);
    cudaGraphSetConditional(A.h_newton, 0);
    cudaGraphSetConditional(A.h_step, 0);
  }
}

// Arnoldi / Krylov initialisation after a Newton residual (thread 0).
template <typename T>
__device__ __forceinline__ bool krylov_start(const GArgs<T>& A, GDev* d) {
  d->j = 0;
  d->rho = d->rho0;
  kry_gv(A)[0] = d->rho0;
  kry_sj(A)[0] = d->rho0 > 0.0 ? 1.0 / d->rho0 : 0.0;
  d->eps = d->eps_mf * (1.0 + d->xnorm);       // eps_mf (1 + |x|) / |v|, |v| = 1 (tgcr.py:129)
  return d->rho0 > 0.0 && d->rho / d->rho0 > d->tol_gcr && d->krylov_max_iter > 0;
}

// ---------------------------------------------------------------------------
// Grid kernels
// ---------------------------------------------------------------------------

// Effective copy of the accepted state with this step's field.
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads) kg_prepare(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
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
}

// Predictor: f = rhs(Xn); Xi = Xn + dt f; G = Xn + dt/2 f (integrators.py:156-158);
// effective copies of Xi (FP64, and in T for the Jacobian products).
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads) kg_predict(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  const Grid& g = A.g;
  const double dt = d->dta, czxy = d->czxy, cyzx = d->cyzx, cxyz = d->cxyz;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.n; n += gridDim.x * blockDim.x) {
    int i, j, k;
    node_ijk(g, n, i, j, k);
    const uint8_t nf = g.nflags[n];
    NodeCoef<double> nc = node_coef<double>(g, n, nf);
    NbE<double, double> X{A.En, A.npf, full_index(g, i, j, k), g.mj, g.mk};
    double o[5];
    rhs_body<double, D3>(g, X, nc, nf, o);
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
  }
}

// Newton residual: f = rhs(Xi) into F; g = Xi - dt/2 f - G; r0 = -g into the
// first basis vector (raw) and its effective copy.  Partials: ||r0||^2, ||x||^2, max|g|.
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads) kg_newton_rhs(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d) || d->newton_failed) return;
  const Grid& g = A.g;
  const double dt = d->dta;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.n; n += gridDim.x * blockDim.x) {
    int i, j, k;
    node_ijk(g, n, i, j, k);
    const uint8_t nf = g.nflags[n];
    NodeCoef<double> nc = node_coef<double>(g, n, nf);
    NbE<double, double> X{A.Ei, A.npf, full_index(g, i, j, k), g.mj, g.mk};
    double o[5];
    rhs_body<double, D3>(g, X, nc, nf, o);
    double gv[5] = {0, 0, 0, 0, 0}, r[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) {
      long e = (long)c * g.npad + n;
      double xv = A.Xi[e];
      A.F[e] = o[c];
      gv[c] = xv - (dt / 2.0) * o[c] - A.G[e];
      T rt = (T)(-gv[c]);
      A.V[e] = rt;
      r[c] = (double)rt;
      acc[0] += r[c] * r[c];
      acc[1] += xv * xv;
    }
    double m = gfinite(hypot(gv[0], gv[1]));
#pragma unroll
    for (int c = 2; c < (D3 ? 5 : 4); ++c) m = fmax(m, gfinite(fabs(gv[c])));
    acc[2] = fmax(acc[2], m);
    write_eff<T, D3>(g, A.VE, A.npf, i, j, k, r, 0.0, 0.0, 0.0);
  }
  const bool mx[3] = {false, false, true};
  block_partials<3>(acc, mx, A.part_nrhs, A.nblk);
}

// Arnoldi stencil: W = A v_j, v_j = s_j v~_j (basis slot j-1, effective copy VE).
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads) kg_stencil(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
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
}

template <typename T> struct GGroup { static constexpr int JB = 8; };
template <> struct GGroup<double> { static constexpr int JB = 4; };

template <typename T> struct V4 { T a, b, c, d; };
__device__ __forceinline__ V4<float> ld4(const float* p) {
  float4 v = *reinterpret_cast<const float4*>(p);
  return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ V4<double> ld4(const double* p) {
  double2 u = reinterpret_cast<const double2*>(p)[0], v = reinterpret_cast<const double2*>(p)[1];
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
}

// Orthogonalisation: v~_{j+1} = W - sum_{i<j} gam_i v~_i (raw, slot j) and its
// effective copy; partial ||v~_{j+1}||^2.  Lane work: four consecutive nodes.
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads) kg_orth(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
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
}

// Newton update: x += sum_i cj_i v~_i (raw FP64), effective copies of the new
// iterate; partial max|dx| (complex modulus on psi).
template <typename T, bool D3>
__global__ void __launch_bounds__(kThreads) kg_update(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d) || d->newton_failed) return;
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
}

// Accepted step: Xn = Xi.
template <typename T>
__global__ void __launch_bounds__(kThreads) kg_accept(GArgs<T> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d) || !d->accepted) return;
  const long nq = A.L / 2;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nq; q += (long)gridDim.x * blockDim.x)
    reinterpret_cast<double2*>(A.Xn)[q] = reinterpret_cast<const double2*>(A.Xi)[q];
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
  d->rhs_evals += 1;
  d->rho0 = sqrt(s[0]);
  d->xnorm = sqrt(s[1]);
  if (!isfinite(d->rho0) || !isfinite(d->xnorm)) { abort_all(A, GS_NONFINITE); return; }
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
  bool cont = hn > 0.0 && d->rho / d->rho0 > d->tol_gcr && jc < d->krylov_max_iter;
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
  bool ok = !(d->rho > d->tol_gcr * d->rho0);
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
