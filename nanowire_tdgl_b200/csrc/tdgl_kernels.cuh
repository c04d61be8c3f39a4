// Standalone kernels: layout conversion, RHS / Jacobian products, observables,
// forward Euler.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "tdgl_common.cuh"

namespace tdgl {

// ---------------------------------------------------------------------------
// Layout conversion between the reference state (complex128, interior nodes in
// the k-fastest order of src/tdgl3d/mesh/indices.py:271-278, blocks
// [psi, phi_x, phi_y, (phi_z)] as in src/tdgl3d/core/state.py:11-97) and the
// device layout (component arrays, i fastest, phi stored real).
// ---------------------------------------------------------------------------

__device__ __forceinline__ int ref_index(const Grid& g, int d) {
  int i, j, k;
  node_ijk(g, d, i, j, k);
  int kk = g.is3d ? k - 1 : 0;
  return ((i - 1) * g.ny + (j - 1)) * g.nz + kk;
}

__global__ void k_pack(Grid g, const double2* __restrict__ xref, double* __restrict__ xdev) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    int r = ref_index(g, d);
    double2 p = xref[r];
    xdev[d] = p.x;
    xdev[(long)g.npad + d] = p.y;
    for (int a = 0; a < g.ncomp - 2; ++a) xdev[(long)(2 + a) * g.npad + d] = xref[(long)(a + 1) * g.n + r].x;
  }
}

__global__ void k_unpack(Grid g, const double* __restrict__ xdev, double2* __restrict__ xref) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    int r = ref_index(g, d);
    xref[r] = make_double2(xdev[d], xdev[(long)g.npad + d]);
    for (int a = 0; a < g.ncomp - 2; ++a) xref[(long)(a + 1) * g.n + r] = make_double2(xdev[(long)(2 + a) * g.npad + d], 0.0);
  }
}

// f = rhs(x) in the device layout, FP64.
__global__ void k_rhs(Grid g, const double* __restrict__ x, double* __restrict__ f, BTerms<double> b) {
  SrcVec<double, double> sx{x, g.npad};
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    double o[5];
    rhs_at<double>(g, sx, b, d, o);
    for (int c = 0; c < g.ncomp; ++c) f[(long)c * g.npad + d] = o[c];
  }
}

// ap = p - dth * J(x) p, analytic tangent (T = float or double storage of p/ap)
template <typename T>
__global__ void k_jvp_analytic(Grid g, const double* __restrict__ x, const T* __restrict__ p, T* __restrict__ ap,
                               double dth, BTerms<double> b) {
  SrcVec<T, double> sx{x, g.npad};
  SrcVec<T, T> sp{p, g.npad};
  BTerms<T> bt{(T)b.czxy, (T)b.cyzx, (T)b.cxyz};
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    T o[5];
    jvp_at<T>(g, sx, bt, sp, d, o);
    for (int c = 0; c < g.ncomp; ++c) {
      long e = (long)c * g.npad + d;
      ap[e] = (T)((double)p[e] - dth * (double)o[c]);
    }
  }
}

// ap = p - dth * (f(x + eps p) - fx) / eps, the reference's finite-difference
// product (src/tdgl3d/solvers/tgcr.py:129-133), FP64.
__global__ void k_jvp_fd(Grid g, const double* __restrict__ x, const double* __restrict__ fx,
                         const double* __restrict__ p, double* __restrict__ ap, double dth, double eps,
                         BTerms<double> b) {
  SrcFD<double> s{x, p, nullptr, 0.0, eps, g.npad};
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    double o[5];
    rhs_at<double>(g, s, b, d, o);
    for (int c = 0; c < g.ncomp; ++c) {
      long e = (long)c * g.npad + d;
      ap[e] = p[e] - dth * ((o[c] - fx[e]) / eps);
    }
  }
}

// Observables at interior nodes, reference order: |psi|^2, B (with boundary
// conditions), J_s (zero-extended state, no boundary conditions).
__global__ void k_observables(Grid g, const double* __restrict__ x, BTerms<double> b, double ihxhy, double ihyhz,
                              double ihzhx, double* __restrict__ psi2, double* __restrict__ Bx,
                              double* __restrict__ By, double* __restrict__ Bz, double* __restrict__ Jx,
                              double* __restrict__ Jy, double* __restrict__ Jz) {
  SrcVec<double, double> s{x, g.npad};
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    int i, j, k;
    node_ijk(g, d, i, j, k);
    int r = ref_index(g, d);
    Ext<double, SrcVec<double, double>> E{&g, s, b};
    double cr = s(PR, d), ci = s(PI, d);
    psi2[r] = cr * cr + ci * ci;
    // B = curl(phi) with the boundary-extended links (src/tdgl3d/physics/bfield.py:12-78)
    double fx0 = E.phi(0, i, j, k), fy0 = E.phi(1, i, j, k);
    Bz[r] = (fx0 - E.phi(0, i, j + 1, k) - fy0 + E.phi(1, i + 1, j, k)) * ihxhy;
    if (g.is3d) {
      double fz0 = E.phi(2, i, j, k);
      Bx[r] = (fy0 - E.phi(1, i, j, k + 1) - fz0 + E.phi(2, i, j + 1, k)) * ihyhz;
      By[r] = (fz0 - E.phi(2, i + 1, j, k) - fx0 + E.phi(0, i, j, k + 1)) * ihzhx;
    } else {
      Bx[r] = 0.0;
      By[r] = 0.0;
    }
    // J_s,a = Im[conj(psi) e^{-i phi_a} psi(m+a)] on the zero-extended raw state
    // (src/tdgl3d/physics/current_density.py:14-72)
    double J[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < (g.is3d ? 3 : 2); ++a) {
      int ii = i + (a == 0), jj = j + (a == 1), kk = k + (a == 2);
      bool inside = ii <= g.Nx - 1 && jj <= g.Ny - 1 && (!g.is3d || kk <= g.Nz - 1);
      double pr = 0.0, pi = 0.0;
      if (inside) {
        int e = dix(g, ii, jj, kk);
        pr = s(PR, e);
        pi = s(PI, e);
      }
      double ph = s(AX + a, d), sn, cs;
      sincos(ph, &sn, &cs);
      // conj(c) * e^{-i ph} = (cr - i ci)(cs - i sn)
      double ur = cr * cs - ci * sn, ui = -(cr * sn + ci * cs);
      J[a] = ur * pi + ui * pr;
    }
    Jx[r] = J[0];
    Jy[r] = J[1];
    Jz[r] = J[2];
  }
}

// x <- x + dt * rhs(x), one forward-Euler step into xn (src/tdgl3d/solvers/integrators.py:79-83)
__global__ void k_euler(Grid g, const double* __restrict__ x, double* __restrict__ xn, double dt, BTerms<double> b) {
  SrcVec<double, double> sx{x, g.npad};
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    double o[5];
    rhs_at<double>(g, sx, b, d, o);
    for (int c = 0; c < g.ncomp; ++c) {
      long e = (long)c * g.npad + d;
      xn[e] = x[e] + dt * o[c];
    }
  }
}

}  // namespace tdgl
