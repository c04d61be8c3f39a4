// Trapezoidal-stepper graph for float Krylov storage (one translation unit per
// precision, so the two compile in parallel).
#include "tdgl_graph_build.cuh"

namespace tdgl {

cudaError_t graph_build_f32(const GArgs<float>& A, const TlMaps* tm, int chunks, cudaGraph_t* graph,
                            cudaGraphExec_t* exec) {
  if (A.g.is3d) return build_trap_graph<float, true>(A, tm, chunks, graph, exec);
  return build_trap_graph<float, false>(A, nullptr, 0, graph, exec);
}

// One tangent-linear stencil launch outside the graph (Horner step when poly,
// else the product): the TMA-staged kernel when tm is given, else the kernel
// that reads global memory.
static cudaError_t launch_tl(const GArgs<float>& A, const TlMaps* tm, int chunks, bool poly, cudaStream_t s) {
  if (A.g.is3d && tm) {
    const void* fn = tm->nx == 2 ? (poly ? (const void*)kg_tl<true, 2> : (const void*)kg_tl<false, 2>)
                                 : (poly ? (const void*)kg_tl<true, 1> : (const void*)kg_tl<false, 1>);
    const size_t smem = tl_smem_bytes(tm->nx);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid(tl_grid_x(A.g.nx, tm->nx), A.arn_gy, chunks);
    void* args[] = {const_cast<TlMaps*>(tm), const_cast<GArgs<float>*>(&A)};
    return cudaLaunchKernel(fn, grid, dim3(kThreads), args, smem, s);
  }
  const dim3 grid(A.arn_gx, A.arn_gy, A.g.is3d ? A.g.nz : 1);
  if (poly) {
    if (A.g.is3d) kg_arn_poly<float, true><<<grid, kThreads, 0, s>>>(A);
    else kg_arn_poly<float, false><<<grid, kThreads, 0, s>>>(A);
  } else {
    if (A.g.is3d) kg_arn_apply<float, true><<<grid, kThreads, 0, s>>>(A);
    else kg_arn_apply<float, false><<<grid, kThreads, 0, s>>>(A);
  }
  return cudaGetLastError();
}

// The Arnoldi product alone (the standalone Krylov-precision Jacobian product).
cudaError_t product_f32(const GArgs<float>& A, const TlMaps* tm, int chunks, cudaStream_t s) {
  return launch_tl(A, tm, chunks, false, s);
}

// Diagnostic: `launches` standalone Arnoldi steps.  kernels: bit 0 the
// orthogonalisation, bit 1 the product, bit 2 the projections, bit 3 the fused
// product and projections, bit 4 the polynomial preconditioner's steps (its
// degree, before the product); 0 = the kernels of this context's graph.
cudaError_t arnoldi_probe_f32(const GArgs<float>& A, const TlMaps* tm, int chunks, int launches, int kernels,
                              cudaStream_t s) {
  const size_t smo = (size_t)(A.kmax + 1) * sizeof(double);
  const size_t smd = (size_t)kWarps * (A.kmax + 2) * sizeof(double);
  const size_t smp = apply_dots_smem<float>(A.kmax);
  if (kernels == 0) kernels = 1 | (A.poly_deg > 0 ? 16 : 0) | (A.apply_dots ? 8 : 2 | 4);
  cudaError_t e = cudaFuncSetAttribute((const void*)kg_arn_orth<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smo);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)kg_arn_dots<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smd);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)kg_arn_apply_dots<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smp);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)kg_arn_apply_dots<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smp);
  const dim3 grid(A.arn_gx, A.arn_gy, A.g.is3d ? A.g.nz : 1);
  for (int r = 0; r < launches && e == cudaSuccess; ++r) {
    if (kernels & 1) kg_arn_orth<float><<<A.nblk_orth, kThreads, smo, s>>>(A);
    for (int k = (kernels & 16) ? A.poly_deg - 1 : -1; k >= 0 && e == cudaSuccess; --k) {
      GArgs<float> P = A;
      P.pstep = k;
      e = launch_tl(P, tm, chunks, true, s);
    }
    if ((kernels & 2) && e == cudaSuccess) e = launch_tl(A, tm, chunks, false, s);
    if (e != cudaSuccess) break;
    if (kernels & 4) kg_arn_dots<float><<<A.nblk_arn, kThreads, smd, s>>>(A);
    if (kernels & 8) {
      if (A.g.is3d) kg_arn_apply_dots<float, true><<<grid, kThreads, smp, s>>>(A);
      else kg_arn_apply_dots<float, false><<<grid, kThreads, smp, s>>>(A);
    }
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace tdgl
