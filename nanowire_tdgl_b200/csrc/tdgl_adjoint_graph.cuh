// Device-resident solve of the adjoint trapezoidal system
//   (I - h J(x)^T) mu = b       (FP64, device layout)
// by GMRES from mu = 0: one CUDA graph with a conditional WHILE node, whose
// body applies the operator with the adjoint kernel (J^T v scattered with
// FP64 atomics, as tdgl_vjp does) and then runs the projection,
// orthogonalisation and Givens kernels of the finite-difference stepper graph
// on the raw basis.  Control decisions stay on the device; the host reads the
// outcome once, after the solve.
//
//   ONCE while { init, init_fin, KRYLOV while { zero, vjp, combine, dots,
//   fin_dots, orth, fin_orth }, solve, update, end }
//
// (the outer loop runs once; its handle also stands for the Newton handle
// that the shared kernels clear when they abort, so every handle of the
// graph drives a conditional node)
//
// The solve stops at the GMRES tolerance or at kmax iterations (no restart);
// the caller restarts on the host from the returned iterate if needed.
#pragma once

#include "tdgl_adjoint.cuh"
#include "tdgl_graph_build.cuh"

namespace tdgl {

// V_0 = b; ||b||^2 block partials.
__global__ void __launch_bounds__(kThreads) kg_adj_init(GArgs<double> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  double acc[1] = {0.0};
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < A.L; e += (long)gridDim.x * blockDim.x) {
    const double v = A.ab[e];
    A.V[e] = v;
    acc[0] += v * v;
  }
  const bool mx[1] = {false};
  block_partials<1>(acc, mx, A.part_orth, A.nblk);
}

// rho0 = ||b||, the first basis scale, and whether to iterate.
__global__ void kg_adj_init_fin(GArgs<double> A) {
  __shared__ double s[1];
  GDev* d = A.dev;
  if (d->status != GS_OK) return;
  reduce_parts(A.part_orth, A.nblk, 1, false, s);
  if (threadIdx.x != 0) return;
  d->rho0 = sqrt(s[0]);
  if (!isfinite(d->rho0)) { abort_all(A, GS_NONFINITE); return; }
  d->j = 0;
  d->rho = d->rho0;
  d->tol_lin = d->tol_gcr;         // the adjoint solves stop at tol_gcr relative
  kry_gv(A)[0] = d->rho0;
  kry_sj(A)[0] = d->rho0 > 0.0 ? 1.0 / d->rho0 : 0.0;
  cudaGraphSetConditional(A.h_krylov, d->rho0 > 0.0 ? 1 : 0);
}

// T = 0 before the scatter.
__global__ void __launch_bounds__(kThreads) kg_adj_zero(GArgs<double> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < A.L; e += (long)gridDim.x * blockDim.x)
    A.aT[e] = 0.0;
}

// T = J(x)^T v~_j (raw basis vector j), the adjoint kernel's loop with the
// state gradient only.
template <bool D3>
__global__ void __launch_bounds__(kThreads) kg_adj_vjp(GArgs<double> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  const Grid& g = A.g;
  const double* v = A.V + (long)d->j * A.L;
  const BTerms<double> b = bterms(g, d->Bx, d->By, d->Bz);
  AdjSink S{&g, 0, 0, 0, A.aT, g.hx * g.hy, g.hz * g.hx, g.hy * g.hz, {0.0, 0.0, 0.0}};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.n; n += gridDim.x * blockDim.x) {
    int i, j, k;
    node_ijk(g, n, i, j, k);
    S.i = i; S.j = j; S.k = k;
    const uint8_t nf = g.nflags[n];
    NodeCoef<double> nc = node_coef<double>(g, n, nf);
    double vv[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) vv[c] = v[(long)c * g.npad + n];
    if (nf & NF_HOLEX) vv[AX] = 0.0;
    if (nf & NF_HOLEY) vv[AY] = 0.0;
    if (D3 && (nf & NF_HOLEZ)) vv[AZ] = 0.0;
    NbSlow<double, SrcVec<double, double>> X{Ext<double, SrcVec<double, double>>{&g, SrcVec<double, double>{A.ax, g.npad}, b},
                                            i, j, k};
    double sc_bar, k2_bar;
    rhs_adjoint<D3>(g, X, nc, vv, S, sc_bar, k2_bar);
  }
}

// W = s_j (v~_j - h T): the operator applied to the normalised basis vector.
__global__ void __launch_bounds__(kThreads) kg_adj_combine(GArgs<double> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  const double sj = kry_sj(A)[d->j], h = d->dta / 2.0;
  const double* v = A.V + (long)d->j * A.L;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < A.L; e += (long)gridDim.x * blockDim.x)
    A.W[e] = sj * (v[e] - h * A.aT[e]);
}

// Least-squares coefficients of the iterate and the convergence verdict.
__global__ void kg_adj_solve(GArgs<double> A) {
  if (threadIdx.x != 0) return;
  GDev* d = A.dev;
  if (d->status != GS_OK) return;
  const int j = d->j;
  d->krylov_iters = j;
  d->accepted = !(d->rho > d->tol_gcr * d->rho0);
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

// End of the single pass of the outer loop.
__global__ void kg_adj_end(GArgs<double> A) {
  if (threadIdx.x == 0) cudaGraphSetConditional(A.h_step, 0);
}

// mu = sum_i c_i v~_i.
__global__ void __launch_bounds__(kThreads) kg_adj_update(GArgs<double> A) {
  const GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  const int j = d->j;
  const double* cj = kry_cj(A);
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < A.L; e += (long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < j; ++i) s += cj[i] * A.V[(long)i * A.L + e];
    A.amu[e] = s;
  }
}

template <bool D3>
cudaError_t build_adjoint_graph(GArgs<double> A, cudaGraph_t* out_graph, cudaGraphExec_t* out_exec) {
  cudaGraph_t G;
  TDGL_GCK(cudaGraphCreate(&G, 0));
  *out_graph = G;
  TDGL_GCK(cudaGraphConditionalHandleCreate(&A.h_step, G, 1, cudaGraphCondAssignDefault));
  A.h_newton = A.h_step;
  TDGL_GCK(cudaGraphConditionalHandleCreate(&A.h_krylov, G, 0, 0));
  const int nb = A.nblk;
  const size_t fin_smem = (size_t)(A.kmax + 1) * sizeof(double);
  Chain top{G};
  cudaGraph_t once, body;
  TDGL_GCK(top.loop(A.h_step, &once));
  Chain co{once};
  TDGL_GCK(co.kernel((const void*)kg_adj_init, nb, kThreads, 0, A));
  TDGL_GCK(co.kernel((const void*)kg_adj_init_fin, 1, kThreads, 0, A));
  TDGL_GCK(co.loop(A.h_krylov, &body));
  Chain ck{body};
  TDGL_GCK(ck.kernel((const void*)kg_adj_zero, nb, kThreads, 0, A));
  TDGL_GCK(ck.kernel((const void*)kg_adj_vjp<D3>, nb, kThreads, 0, A));
  TDGL_GCK(ck.kernel((const void*)kg_adj_combine, nb, kThreads, 0, A));
  TDGL_GCK(ck.kernel((const void*)kg_dots<double>, nb, kThreads, 0, A));
  TDGL_GCK(ck.kernel((const void*)kg_fin_dots<double>, 1, kThreads, fin_smem, A));
  TDGL_GCK(ck.kernel((const void*)kg_orth<double, D3>, nb, kThreads, 0, A));
  TDGL_GCK(ck.kernel((const void*)kg_fin_orth<double>, 1, kThreads, 0, A));
  TDGL_GCK(co.kernel((const void*)kg_adj_solve, 1, kThreads, 0, A));
  TDGL_GCK(co.kernel((const void*)kg_adj_update, nb, kThreads, 0, A));
  TDGL_GCK(co.kernel((const void*)kg_adj_end, 1, kThreads, 0, A));
  TDGL_GCK(cudaGraphInstantiate(out_exec, G, 0));
  return cudaSuccess;
}

}  // namespace tdgl
