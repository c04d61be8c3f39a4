// Trapezoidal-stepper graph for double Krylov storage (one translation unit per
// precision, so the two compile in parallel).
#include "tdgl_graph_build.cuh"

namespace tdgl {

cudaError_t graph_build_f64(const GArgs<double>& A, cudaGraph_t* graph, cudaGraphExec_t* exec) {
  if (A.g.is3d) return build_trap_graph<double, true>(A, nullptr, 0, graph, exec);
  return build_trap_graph<double, false>(A, nullptr, 0, graph, exec);
}

// The Arnoldi product alone (the standalone Krylov-precision Jacobian product).
cudaError_t product_f64(const GArgs<double>& A, cudaStream_t s) {
  const dim3 grid(A.arn_gx, A.arn_gy, A.g.is3d ? A.g.nz : 1);
  if (A.g.is3d) kg_arn_apply<double, true><<<grid, kThreads, 0, s>>>(A);
  else kg_arn_apply<double, false><<<grid, kThreads, 0, s>>>(A);
  return cudaGetLastError();
}

// Diagnostic: `launches` standalone Arnoldi steps.  kernels: bit 0 the
// orthogonalisation, bit 1 the product, bit 2 the projections, bit 3 the fused
// product and projections, bit 4 the polynomial preconditioner's steps (its
// degree, before the product); 0 = the kernels of this context's graph.
cudaError_t arnoldi_probe_f64(const GArgs<double>& A, int launches, int kernels, cudaStream_t s) {
  const size_t smo = (size_t)(A.kmax + 1) * sizeof(double);
  const size_t smd = (size_t)kWarps * (A.kmax + 2) * sizeof(double);
  const size_t smp = apply_dots_smem<double>(A.kmax);
  if (kernels == 0) kernels = 1 | (A.poly_deg > 0 ? 16 : 0) | (A.apply_dots ? 8 : 2 | 4);
  cudaError_t e = cudaFuncSetAttribute((const void*)kg_arn_orth<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smo);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)kg_arn_dots<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smd);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)kg_arn_apply_dots<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smp);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)kg_arn_apply_dots<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smp);
  const dim3 grid(A.arn_gx, A.arn_gy, A.g.is3d ? A.g.nz : 1);
  for (int r = 0; r < launches && e == cudaSuccess; ++r) {
    if (kernels & 1) kg_arn_orth<double><<<A.nblk_orth, kThreads, smo, s>>>(A);
    for (int k = (kernels & 16) ? A.poly_deg - 1 : -1; k >= 0; --k) {
      GArgs<double> P = A;
      P.pstep = k;
      if (A.g.is3d) kg_arn_poly<double, true><<<grid, kThreads, 0, s>>>(P);
      else kg_arn_poly<double, false><<<grid, kThreads, 0, s>>>(P);
    }
    if (kernels & 2) {
      if (A.g.is3d) kg_arn_apply<double, true><<<grid, kThreads, 0, s>>>(A);
      else kg_arn_apply<double, false><<<grid, kThreads, 0, s>>>(A);
    }
    if (kernels & 4) kg_arn_dots<double><<<A.nblk_arn, kThreads, smd, s>>>(A);
    if (kernels & 32) {
      if (A.g.is3d) kg_predict<double, true><<<A.nblk, kThreads, 0, s>>>(A);
      else kg_predict<double, false><<<A.nblk, kThreads, 0, s>>>(A);
    }
    if (kernels & 64) {
      if (A.g.is3d) kg_newton_rhs<double, true><<<A.nblk, kThreads, 0, s>>>(A);
      else kg_newton_rhs<double, false><<<A.nblk, kThreads, 0, s>>>(A);
    }
    if (kernels & 128) {
      if (A.g.is3d) kg_update_fused<double, true><<<A.nblk, kThreads, 0, s>>>(A);
      else kg_update_fused<double, false><<<A.nblk, kThreads, 0, s>>>(A);
    }
    if (kernels & 8) {
      if (A.g.is3d) kg_arn_apply_dots<double, true><<<grid, kThreads, smp, s>>>(A);
      else kg_arn_apply_dots<double, false><<<grid, kThreads, smp, s>>>(A);
    }
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace tdgl
