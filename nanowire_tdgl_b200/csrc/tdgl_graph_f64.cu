// Trapezoidal-stepper graph for double Krylov storage (one translation unit per
// precision, so the two compile in parallel).
#include "tdgl_graph_build.cuh"

namespace tdgl {

cudaError_t graph_build_f64(const GArgs<double>& A, cudaGraph_t* graph, cudaGraphExec_t* exec) {
  if (A.g.is3d) return build_trap_graph<double, true>(A, graph, exec);
  return build_trap_graph<double, false>(A, graph, exec);
}

}  // namespace tdgl
