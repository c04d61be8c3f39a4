// Instantiation of the persistent stepper for float Krylov storage (one
// translation unit per precision, so the two compile in parallel).
#include <cuda_runtime.h>

#include "tdgl_stepper.cuh"

namespace tdgl {

cudaError_t stepper_occupancy_f32(size_t smem, int* occ) {
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_stepper<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k_stepper<float>, kThreads, smem);
}

cudaError_t stepper_launch_f32(StepArgs<float> A, int blocks, size_t smem, cudaStream_t s) {
  void* args[] = {&A};
  return cudaLaunchCooperativeKernel((void*)k_stepper<float>, blocks, kThreads, args, smem, s);
}

}  // namespace tdgl
