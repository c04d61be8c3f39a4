// Construction of the trapezoidal-stepper graph (see tdgl_graph.cuh): kernel
// nodes chained linearly inside three nested conditional WHILE bodies.  The
// Krylov body is the three-kernel Arnoldi step for analytic Jacobian products, or
// stencil / projection / orthogonalisation kernels with one-block reductions
// for finite-difference products.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "tdgl_graph.cuh"
#include "tdgl_tl.cuh"

namespace tdgl {

struct Chain {
  cudaGraph_t g;
  cudaGraphNode_t last = nullptr;
  template <class Args>
  cudaError_t kernel(const void* fn, dim3 grid, int block, size_t smem, Args& args) {
    cudaKernelNodeParams p{};
    p.func = const_cast<void*>(fn);
    p.gridDim = grid;
    p.blockDim = dim3(block);
    p.sharedMemBytes = (unsigned)smem;
    void* a[] = {&args};
    p.kernelParams = a;
    cudaGraphNode_t n;
    cudaError_t e = cudaGraphAddKernelNode(&n, g, last ? &last : nullptr, last ? 1 : 0, &p);
    if (e == cudaSuccess) last = n;
    return e;
  }
  // kernel with a __grid_constant__ first parameter (the tensor maps) and the
  // arguments; pdl: a programmatic dependency on the previous kernel node (the
  // kernel may start before that one completes and waits for it with
  // grid_dep_wait)
  template <class M, class Args>
  cudaError_t kernel2(const void* fn, dim3 grid, int block, size_t smem, const M& m, Args& args, bool pdl = false) {
    cudaKernelNodeParams p{};
    p.func = const_cast<void*>(fn);
    p.gridDim = grid;
    p.blockDim = dim3(block);
    p.sharedMemBytes = (unsigned)smem;
    void* a[] = {const_cast<M*>(&m), &args};
    p.kernelParams = a;
    cudaGraphNode_t n;
    if (pdl && last) {
      cudaError_t e = cudaGraphAddKernelNode(&n, g, nullptr, 0, &p);
      if (e != cudaSuccess) return e;
      cudaGraphEdgeData ed{};
      ed.from_port = cudaGraphKernelNodePortProgrammatic;
      ed.type = cudaGraphDependencyTypeProgrammatic;
      e = cudaGraphAddDependencies_v2(g, &last, &n, &ed, 1);
      if (e == cudaSuccess) last = n;
      return e;
    }
    cudaError_t e = cudaGraphAddKernelNode(&n, g, last ? &last : nullptr, last ? 1 : 0, &p);
    if (e == cudaSuccess) last = n;
    return e;
  }
  cudaError_t loop(cudaGraphConditionalHandle h, cudaGraph_t* body) {
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t n;
    cudaError_t e = cudaGraphAddNode(&n, g, last ? &last : nullptr, last ? 1 : 0, &p);
    if (e == cudaSuccess) {
      last = n;
      *body = p.conditional.phGraph_out[0];
    }
    return e;
  }
};

#define TDGL_GCK(x)                      \
  do {                                   \
    cudaError_t e_ = (x);                \
    if (e_ != cudaSuccess) return e_;    \
  } while (0)

// Tangent-linear stencil node (Horner step when poly, else the Arnoldi
// product): the TMA-staged kernel when tensor maps are given (FP32 vectors,
// 3-D grids; `chunks` z-chunks; a programmatic dependency on the kernel node
// before it when tm->pdl), else the kernel that reads global memory.
template <typename T, bool D3>
cudaError_t add_tl(Chain& ch, const GArgs<T>& A, const TlMaps* tm, int chunks, bool poly, int par) {
  GArgs<T> a = A;
  a.tl_par = par;
  if constexpr (std::is_same<T, float>::value && D3) {
    if (tm) {
      const void* fn = tl_kernel(tm->nx, poly, A.g.kappa_per_node != 0);
      const size_t smem = tl_smem_bytes(tm->nx);
      TDGL_GCK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      return ch.kernel2(fn, dim3(tl_grid_x(A.g.nx, tm->nx), A.arn_gy, chunks), kThreads, smem, *tm, a,
                        tm->pdl != 0);
    }
  }
  const dim3 tiles(A.arn_gx, A.arn_gy, D3 ? A.g.nz : 1);
  return ch.kernel(poly ? (const void*)kg_arn_poly<T, D3> : (const void*)kg_arn_apply<T, D3>, tiles, kThreads, 0,
                   a);
}

template <typename T, bool D3>
cudaError_t build_trap_graph(GArgs<T> A, const TlMaps* tm, int chunks, cudaGraph_t* out_graph,
                             cudaGraphExec_t* out_exec) {
  cudaGraph_t G;
  TDGL_GCK(cudaGraphCreate(&G, 0));
  *out_graph = G;
  TDGL_GCK(cudaGraphConditionalHandleCreate(&A.h_step, G, 1, cudaGraphCondAssignDefault));
  TDGL_GCK(cudaGraphConditionalHandleCreate(&A.h_newton, G, 0, 0));
  TDGL_GCK(cudaGraphConditionalHandleCreate(&A.h_krylov, G, 0, 0));
  const int nb = A.nblk;
  const size_t fin_smem = (size_t)(A.kmax + 1) * sizeof(double);
  Chain top{G};
  cudaGraph_t step_body, newton_body, krylov_body;
  TDGL_GCK(top.loop(A.h_step, &step_body));
  Chain cs{step_body};
  TDGL_GCK(cs.kernel((const void*)kg_step_begin<T>, 1, kThreads, 0, A));
  TDGL_GCK(cs.kernel((const void*)kg_prepare<T, D3>, nb, kThreads, 0, A));
  TDGL_GCK(cs.kernel((const void*)kg_predict<T, D3>, nb, kThreads, 0, A));
  TDGL_GCK(cs.kernel((const void*)kg_newton_rhs<T, D3>, nb, kThreads, 0, A));
  TDGL_GCK(cs.kernel((const void*)kg_newton_init<T>, 1, kThreads, 0, A));
  TDGL_GCK(cs.loop(A.h_newton, &newton_body));
  TDGL_GCK(cs.kernel((const void*)kg_accept<T>, nb, kThreads, 0, A));
  TDGL_GCK(cs.kernel((const void*)kg_step_end<T>, 1, kThreads, 0, A));
  Chain cn{newton_body};
  TDGL_GCK(cn.loop(A.h_krylov, &krylov_body));
  TDGL_GCK(cn.kernel((const void*)kg_newton_solve<T>, 1, kThreads, 0, A));
  const dim3 tiles(A.arn_gx, A.arn_gy, D3 ? A.g.nz : 1);
  if (A.fused) {                    // x += sum_i c_i U_i, or sum_i c_i p(A) U_i with the preconditioner
    TDGL_GCK(cn.kernel((const void*)kg_update_fused<T, D3>, nb, kThreads, 0, A));
  } else {
    TDGL_GCK(cn.kernel((const void*)kg_update<T, D3>, nb, kThreads, 0, A));
  }
  TDGL_GCK(cn.kernel((const void*)kg_newton_rhs<T, D3>, nb, kThreads, 0, A));
  TDGL_GCK(cn.kernel((const void*)kg_newton_check<T>, 1, kThreads, 0, A));
  Chain ck{krylov_body};
  if (A.fused) {
    const size_t smo = (size_t)(A.kmax + 1) * sizeof(double);
    const size_t smd = (size_t)kWarps * (A.kmax + 2) * sizeof(double);
    TDGL_GCK(cudaFuncSetAttribute((const void*)kg_arn_orth<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smo));
    TDGL_GCK(cudaFuncSetAttribute((const void*)kg_arn_dots<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smd));
    TDGL_GCK(ck.kernel((const void*)kg_arn_orth<T>, A.nblk_orth, kThreads, smo, A));
    TDGL_GCK(ck.kernel((const void*)kg_arn_check<T>, 1, kThreads, 0, A));
    for (int k = A.poly_deg - 1; k >= 0; --k) {   // p(A) U_ja into PB_ja
      GArgs<T> P = A;
      P.pstep = k;
      TDGL_GCK((add_tl<T, D3>(ck, P, tm, chunks, true, (A.poly_deg - 1 - k) & 1)));
    }
    if (A.apply_dots) {
      const size_t smp = apply_dots_smem<T>(A.kmax);
      TDGL_GCK(cudaFuncSetAttribute((const void*)kg_arn_apply_dots<T, D3>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp));
      TDGL_GCK(ck.kernel((const void*)kg_arn_apply_dots<T, D3>, tiles, kThreads, smp, A));
    } else {
      TDGL_GCK((add_tl<T, D3>(ck, A, tm, chunks, false, A.poly_deg & 1)));
      TDGL_GCK(ck.kernel((const void*)kg_arn_dots<T>, A.nblk_arn, kThreads, smd, A));
    }
  } else {
    TDGL_GCK(ck.kernel((const void*)kg_stencil<T, D3>, nb, kThreads, 0, A));
    TDGL_GCK(ck.kernel((const void*)kg_dots<T>, nb, kThreads, 0, A));
    TDGL_GCK(ck.kernel((const void*)kg_fin_dots<T>, 1, kThreads, fin_smem, A));
    TDGL_GCK(ck.kernel((const void*)kg_orth<T, D3>, nb, kThreads, 0, A));
    TDGL_GCK(ck.kernel((const void*)kg_fin_orth<T>, 1, kThreads, 0, A));
  }
  TDGL_GCK(cudaGraphInstantiate(out_exec, G, 0));
  return cudaSuccess;
}

}  // namespace tdgl
