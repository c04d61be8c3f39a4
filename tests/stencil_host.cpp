// CPU build of the device stencil code, for the CPU test suite only.
//
// The RHS and Jacobian-product node functions of tdgl_stencil.cuh are plain
// arithmetic; compiled here for the host they let tests/test_stencil_host.py
// compare the kernels' index and boundary logic with the oracle without a GPU.
// This file is not part of the library.
#include <cstring>
#include <string>

#include "tdgl_b200.h"
#include "tdgl_geometry.h"
#include "tdgl_stencil.cuh"

using namespace tdgl;

static thread_local std::string g_err;

static int setup(const tdgl_grid_desc* gd, const tdgl_material_desc* md, HostGeometry& hg) {
  int rc = build_geometry(gd, md, hg, g_err);
  if (rc) return rc;
  hg.g.nflags = hg.nflags.data();
  hg.g.lflags = hg.lflags.empty() ? nullptr : hg.lflags.data();
  hg.g.k2int = hg.k2.empty() ? nullptr : hg.k2.data();
  hg.g.scint = hg.sc.empty() ? nullptr : hg.sc.data();
  return 0;
}

extern "C" const char* host_last_error() { return g_err.c_str(); }

extern "C" int host_layout(const tdgl_grid_desc* gd, int64_t* n, int64_t* npad, int64_t* ncomp) {
  HostGeometry hg;
  int rc = setup(gd, nullptr, hg);
  if (rc) return rc;
  *n = hg.g.n; *npad = hg.g.npad; *ncomp = hg.g.ncomp;
  return 0;
}

extern "C" int host_nflags(const tdgl_grid_desc* gd, const tdgl_material_desc* md, uint8_t* out) {
  HostGeometry hg;
  int rc = setup(gd, md, hg);
  if (rc) return rc;
  std::memcpy(out, hg.nflags.data(), hg.nflags.size());
  return 0;
}

// f = rhs(x), device layout
extern "C" int host_rhs(const tdgl_grid_desc* gd, const tdgl_material_desc* md, const double* x, double* f,
                        double Bx, double By, double Bz) {
  HostGeometry hg;
  int rc = setup(gd, md, hg);
  if (rc) return rc;
  const Grid& g = hg.g;
  BTerms<double> b{Bz * g.hx * g.hy, By * g.hz * g.hx, Bx * g.hy * g.hz};
  SrcVec<double, double> s{x, g.npad};
  for (int d = 0; d < g.n; ++d) {
    double o[5];
    rhs_at<double>(g, s, b, d, o);
    for (int c = 0; c < g.ncomp; ++c) f[(long)c * g.npad + d] = o[c];
  }
  return 0;
}

// jp = J(x) p (analytic), device layout; as_float: evaluate in single precision
extern "C" int host_jvp(const tdgl_grid_desc* gd, const tdgl_material_desc* md, const double* x, const double* p,
                        double* jp, double Bx, double By, double Bz, int as_float) {
  HostGeometry hg;
  int rc = setup(gd, md, hg);
  if (rc) return rc;
  const Grid& g = hg.g;
  BTerms<double> b{Bz * g.hx * g.hy, By * g.hz * g.hx, Bx * g.hy * g.hz};
  for (int d = 0; d < g.n; ++d) {
    if (as_float) {
      SrcVec<float, double> sx{x, g.npad};
      SrcVec<float, double> sp{p, g.npad};
      BTerms<float> bf{(float)b.czxy, (float)b.cyzx, (float)b.cxyz};
      float o[5];
      jvp_at<float>(g, sx, bf, sp, d, o);
      for (int c = 0; c < g.ncomp; ++c) jp[(long)c * g.npad + d] = o[c];
    } else {
      SrcVec<double, double> sx{x, g.npad};
      SrcVec<double, double> sp{p, g.npad};
      double o[5];
      jvp_at<double>(g, sx, b, sp, d, o);
      for (int c = 0; c < g.ncomp; ++c) jp[(long)c * g.npad + d] = o[c];
    }
  }
  return 0;
}
