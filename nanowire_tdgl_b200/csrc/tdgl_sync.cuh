// Grid-wide barrier with a deterministic reduction, for the persistent
// (cooperatively launched) stepper kernel.
//
// Every block writes its partial values for `nslot` slots; the last block to
// arrive reduces them in a fixed order (the same order on every call, so runs
// are bitwise repeatable for a fixed grid), publishes the results and releases
// the others.  Every wait is bounded: a waiter gives up after `timeout_ns` of
// global time, raises the shared error word, and all blocks leave at their
// next barrier.  No wait can outlive the kernel's own bound.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tdgl {

constexpr int kErrTimeout = 5;     // == TDGL_ETIMEOUT

struct Sync {
  double* partials;      // [nslot_max][gridDim.x], slot-major
  double* results;       // [nslot_max]
  unsigned* bar;         // [0] arrivals, [1] generation
  int* err;              // first error status raised by any block (0 = none)
  int nslot_max;
  unsigned long long timeout_ns;
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_volatile(const unsigned* p) { return *(volatile const unsigned*)p; }
__device__ __forceinline__ int ld_volatile(const int* p) { return *(volatile const int*)p; }

__device__ __forceinline__ void raise_error(const Sync& s, int code) { atomicCAS(s.err, 0, code); }

// Block-level partials live in shared memory `blk[0..nslot)`; slots whose
// index is >= nsum are max-reductions (inputs >= 0), the others are sums.
// Returns false when an error was raised anywhere (all threads agree).
__device__ inline bool grid_reduce(const Sync& s, const double* blk, int nslot, int nsum, double* out_smem) {
  __shared__ int s_last;
  __shared__ unsigned s_gen;
  const int G = gridDim.x;
  for (int t = threadIdx.x; t < nslot; t += blockDim.x) s.partials[(long)t * G + blockIdx.x] = blk[t];
  __syncthreads();
  if (threadIdx.x == 0) {
    s_gen = ld_volatile(s.bar + 1);
    __threadfence();
    unsigned arrived = atomicAdd(s.bar, 1u);
    s_last = (arrived == (unsigned)G - 1u);
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    // each warp reduces whole slots; lanes stride over blocks, then a fixed shuffle tree
    for (int t0 = warp; t0 < nslot; t0 += 2 * nw) {
      int t1 = t0 + nw;
      bool mx0 = t0 >= nsum, mx1 = t1 >= nsum;
      double a0 = 0.0, a1 = 0.0;
      for (int b = lane; b < G; b += 32) {
        double v0 = __ldcg(&s.partials[(long)t0 * G + b]);
        double v1 = t1 < nslot ? __ldcg(&s.partials[(long)t1 * G + b]) : 0.0;
        a0 = mx0 ? fmax(a0, v0) : a0 + v0;
        a1 = mx1 ? fmax(a1, v1) : a1 + v1;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        double u0 = __shfl_down_sync(0xffffffffu, a0, o);
        double u1 = __shfl_down_sync(0xffffffffu, a1, o);
        a0 = mx0 ? fmax(a0, u0) : a0 + u0;
        a1 = mx1 ? fmax(a1, u1) : a1 + u1;
      }
      if (lane == 0) {
        s.results[t0] = a0;
        if (t1 < nslot) s.results[t1] = a1;
      }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      s.bar[0] = 0u;
      __threadfence();
      atomicAdd(s.bar + 1, 1u);
    }
  } else if (threadIdx.x == 0) {
    unsigned long long t0 = global_ns();
    unsigned spins = 0;
    while (ld_volatile(s.bar + 1) == s_gen) {
      if (ld_volatile(s.err)) break;
      if ((++spins & 63u) == 0u && global_ns() - t0 > s.timeout_ns) {
        raise_error(s, kErrTimeout);
        break;
      }
      __nanosleep(40);
    }
    __threadfence();
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nslot; t += blockDim.x) out_smem[t] = __ldcg(&s.results[t]);
  __syncthreads();
  return ld_volatile(s.err) == 0;
}

// Plain barrier (no values).
__device__ inline bool grid_sync(const Sync& s, double* scratch_smem) {
  return grid_reduce(s, scratch_smem, 0, 0, scratch_smem);
}

// Warp-level sum / max (fixed tree).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace tdgl
