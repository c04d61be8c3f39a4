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
// pdl: the launch may start before the previous kernel in the stream
// completes (only where that kernel writes no linearisation copy: the
// probe's repeated Arnoldi-step kernels, as in the step graph).
static cudaError_t launch_tl(const GArgs<float>& A, const TlMaps* tm, int chunks, bool poly, cudaStream_t s,
                             bool pdl = false) {
  if (A.g.is3d && tm) {
    const void* fn = tl_kernel(tm->nx, poly, A.g.kappa_per_node != 0);
    const size_t smem = tl_smem_bytes(tm->nx);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid(tl_grid_x(A.g.nx, tm->nx), A.arn_gy, chunks);
    void* args[] = {const_cast<TlMaps*>(tm), const_cast<GArgs<float>*>(&A)};
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelExC(&cfg, fn, args);
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
// degree, before the product), bits 5-7 the Newton-stage kernels (predictor,
// Newton residual, Newton update over ja basis vectors; they overwrite the
// iterate); 0 = the kernels of this context's graph.
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
  int par = 0;                  // claim-counter set: alternates along the launches of the stencil
  for (int r = 0; r < launches && e == cudaSuccess; ++r) {
    if (kernels & 1) kg_arn_orth<float><<<A.nblk_orth, kThreads, smo, s>>>(A);
    for (int k = (kernels & 16) ? A.poly_deg - 1 : -1; k >= 0 && e == cudaSuccess; --k) {
      GArgs<float> P = A;
      P.pstep = k;
      P.tl_par = par ^= 1;
      e = launch_tl(P, tm, chunks, true, s, tm && tm->pdl);
    }
    if ((kernels & 2) && e == cudaSuccess) {
      GArgs<float> P = A;
      P.tl_par = par ^= 1;
      e = launch_tl(P, tm, chunks, false, s, tm && tm->pdl);
    }
    if (e != cudaSuccess) break;
    if (kernels & 4) kg_arn_dots<float><<<A.nblk_arn, kThreads, smd, s>>>(A);
    if (kernels & 8) {
      if (A.g.is3d) kg_arn_apply_dots<float, true><<<grid, kThreads, smp, s>>>(A);
      else kg_arn_apply_dots<float, false><<<grid, kThreads, smp, s>>>(A);
    }
    if (kernels & 32) {
      if (A.g.is3d) kg_predict<float, true><<<A.nblk, kThreads, 0, s>>>(A);
      else kg_predict<float, false><<<A.nblk, kThreads, 0, s>>>(A);
    }
    if (kernels & 64) {
      if (A.g.is3d) kg_newton_rhs<float, true><<<A.nblk, kThreads, 0, s>>>(A);
      else kg_newton_rhs<float, false><<<A.nblk, kThreads, 0, s>>>(A);
    }
    if (kernels & 128) {
      if (A.g.is3d) kg_update_fused<float, true><<<A.nblk, kThreads, 0, s>>>(A);
      else kg_update_fused<float, false><<<A.nblk, kThreads, 0, s>>>(A);
    }
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace tdgl
