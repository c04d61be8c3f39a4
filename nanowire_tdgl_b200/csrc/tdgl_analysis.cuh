// Post-processing kernels on device-layout states: plaquette phase winding
// (vortex counting) and the masked means of the steady-state check.
#pragma once

#include "tdgl_common.cuh"

namespace tdgl {

// Phase winding around every elementary plaquette of every interior z-slice
// (src/tdgl3d/analysis/vortex_counting.py:14-139).  Plaquette (i, j) of slice
// k joins interior nodes (i, j), (i+1, j), (i+1, j+1), (i, j+1) (0-based
// interior indices); the winding is the sum of the four phase differences
// around it, each wrapped to [-pi, pi] as atan2(sin d, cos d), divided by 2 pi.
// A plaquette with any corner |psi|^2 below mask_thr is marked NaN.  Output
// w[(k * (nx - 1) + i) * (ny - 1) + j]: per slice, i-major like the
// reference's scan.
__global__ void k_plaquette(Grid g, const double* __restrict__ x, double mask_thr, double* __restrict__ w) {
  const int px = g.nx - 1, py = g.ny - 1, ns = g.is3d ? g.nz : 1;
  const long total = (long)ns * px * py;
  const double two_pi = 6.283185307179586;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int j = (int)(t % py);
    const long r = t / py;
    const int i = (int)(r % px);
    const int k = (int)(r / px);
    const long d0 = i + (long)g.nx * (j + (long)g.ny * k);
    const long dd[4] = {d0, d0 + 1, d0 + 1 + g.nx, d0 + g.nx};
    double ph[4];
    bool masked = false;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double re = x[dd[c]], im = x[g.npad + dd[c]];
      const double a = hypot(re, im);
      if (a * a < mask_thr) masked = true;
      ph[c] = atan2(im, re);
    }
    if (masked) {
      w[t] = nan("");
      continue;
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double dphi = ph[(c + 1) & 3] - ph[c];
      double sn, cs;
      sincos(dphi, &sn, &cs);
      s += atan2(sn, cs);
    }
    w[t] = s / two_pi;
  }
}

// Means over the superconducting interior nodes (sc > 0; all nodes without
// sc) of |psi|^2 and |J_s| = sqrt(Jx^2 + Jy^2 + Jz^2), from observables in
// reference order (src/tdgl3d/analysis/convergence.py:14-117).  One block of
// exactly kThreads threads (the reduction buffer holds kWarps warps):
// strided per-thread sums, then a fixed-order block reduction.
// out: [mean |psi|^2, mean |J_s|, node count].
__global__ void k_conv_means(long n, const double* __restrict__ psi2, const double* __restrict__ jx,
                             const double* __restrict__ jy, const double* __restrict__ jz,
                             const double* __restrict__ sc, double* __restrict__ out) {
  __shared__ double red[3][kWarps];
  if (blockDim.x != kThreads) return;
  double a = 0.0, b = 0.0, c = 0.0;
  for (long r = threadIdx.x; r < n; r += blockDim.x) {
    if (sc && !(sc[r] > 0.0)) continue;
    a += psi2[r];
    const double j2 = jx[r] * jx[r] + jy[r] * jy[r] + (jz ? jz[r] * jz[r] : 0.0);
    b += sqrt(j2);
    c += 1.0;
  }
  a = warp_sum(a);
  b = warp_sum(b);
  c = warp_sum(c);
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][warp] = a;
    red[1][warp] = b;
    red[2][warp] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int w = 0; w < kWarps; ++w) {
      s0 += red[0][w];
      s1 += red[1][w];
      s2 += red[2][w];
    }
    out[0] = s2 > 0.0 ? s0 / s2 : nan("");
    out[1] = s2 > 0.0 ? s1 / s2 : nan("");
    out[2] = s2;
  }
}

}  // namespace tdgl
