// Launch constants shared by the standalone kernels and the persistent stepper.
#pragma once

#include "tdgl_stencil.cuh"
#include "tdgl_sync.cuh"

namespace tdgl {

constexpr int kThreads = 256;          // threads per block of every kernel
constexpr int kWarps = kThreads / 32;

// Jacobian-vector product of the Krylov solves.
enum JvpMode : int { JVP_FD = 0, JVP_ANALYTIC = 1 };

}  // namespace tdgl
