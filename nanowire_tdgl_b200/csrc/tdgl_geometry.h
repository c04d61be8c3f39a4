// Host-side derivation of the device grid description: node flags, link
// flags and per-node coefficients from the reference's index maps and
// material map (src/tdgl3d/mesh/indices.py:136-232, src/tdgl3d/core/material.py).
// Plain C++ (no CUDA), shared by tdgl_ctx_create and the CPU stencil test.
#pragma once

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "tdgl_b200.h"
#include "tdgl_stencil.cuh"

namespace tdgl {

struct HostGeometry {
  Grid g{};                       // pointers left null; the caller points them at its copies
  std::vector<uint8_t> lflags;    // full grid (empty when there are no holes)
  std::vector<uint8_t> nflags;    // interior, device order
  std::vector<double> k2;         // interior kappa^2 (empty when uniform)
  std::vector<double> sc;         // interior sc (empty unless fractional values occur)
  std::vector<int> slow_off;      // per 128-node region offsets into slow_idx
  std::vector<int> slow_idx;      // slow nodes grouped by region
};

inline long round_up_l(long v, long m) { return (v + m - 1) / m * m; }

// Returns TDGL_OK or TDGL_EINVAL with a message.
inline int build_geometry(const tdgl_grid_desc* gd, const tdgl_material_desc* md, HostGeometry& out,
                          std::string& err) {
  if (gd->Nx < 2 || gd->Ny < 2) { err = "Nx and Ny must each be >= 2."; return TDGL_EINVAL; }
  if (gd->Nz < 1) { err = "Nz must be >= 1."; return TDGL_EINVAL; }
  const long Nx = gd->Nx, Ny = gd->Ny, Nz = gd->Nz;
  const bool d3 = Nz > 1;
  const long nx = Nx - 1, ny = Ny - 1, nz = d3 ? Nz - 1 : 1;
  const long n = nx * ny * nz;
  // Full-grid strides: the reference's (mjr, mkr: the index of its full-grid
  // arrays, m = i + (Nx+1) j + (Nx+1)(Ny+1) k, src/tdgl3d/mesh/indices.py:46-55)
  // for the input arrays, and the device's (mj, mk), whose rows are padded to a
  // multiple of 4 entries so that every row of an FP32 full-grid vector starts
  // on a 16-byte boundary (the row pitch a TMA tensor map requires).
  const long mjr = Nx + 1, mkr = (Nx + 1) * (Ny + 1);
  const long dimx_ref = d3 ? mkr * (Nz + 1) : mkr;
  const long mj = round_up_l(Nx + 1, 4), mk = mj * (Ny + 1);
  const long dimx = d3 ? mk * (Nz + 1) : mk;
  if (n > (1L << 30) || dimx > (1L << 31) - 1) { err = "grid too large for 32-bit node indices"; return TDGL_EINVAL; }
  Grid& g = out.g;
  g.Nx = (int)Nx; g.Ny = (int)Ny; g.Nz = (int)Nz;
  g.nx = (int)nx; g.ny = (int)ny; g.nz = (int)nz;
  g.is3d = d3;
  g.px = gd->periodic_x != 0; g.py = gd->periodic_y != 0; g.pz = gd->periodic_z != 0;
  g.n = (int)n;
  g.npad = (int)round_up_l(n, 128);
  g.ncomp = d3 ? 5 : 4;
  g.mj = (int)mj; g.mk = (int)mk;
  g.hx = gd->hx; g.hy = gd->hy; g.hz = gd->hz;
  g.ihx2 = 1.0 / (gd->hx * gd->hx);
  g.ihy2 = 1.0 / (gd->hy * gd->hy);
  g.ihz2 = 1.0 / (gd->hz * gd->hz);
  g.hx2 = gd->hx * gd->hx; g.hy2 = gd->hy * gd->hy; g.hz2 = gd->hz * gd->hz;

  auto dev_of = [&](long i, long j, long k) { return (i - 1) + nx * ((j - 1) + ny * (d3 ? (k - 1) : 0)); };
  auto ref_to_dev = [&](long r) {
    long kk = r % nz, q = r / nz;
    long j = q % ny + 1, i = q / ny + 1;
    return dev_of(i, j, d3 ? kk + 1 : 0);
  };
  std::vector<uint8_t> lf(dimx, 0), nf(n, 0);
  bool any_hole = false;
  for (int a = 0; a < 3; ++a) {
    if (a == 2 && !d3) continue;
    const int64_t* hl = md ? md->hole_links[a] : nullptr;
    int64_t nh = md ? md->n_hole_links[a] : 0;
    for (int64_t t = 0; t < nh; ++t) {
      int64_t m = hl[t];
      if (m < 0 || m >= dimx_ref) { err = "hole link index out of range"; return TDGL_EINVAL; }
      const long i = m % mjr, q = m / mjr;
      lf[i + mj * (q % (Ny + 1)) + mk * (q / (Ny + 1))] |= (uint8_t)(1u << a);
      any_hole = true;
    }
    const int64_t* hi = md ? md->hole_interior[a] : nullptr;
    int64_t ni = md ? md->n_hole_interior[a] : 0;
    for (int64_t t = 0; t < ni; ++t) {
      int64_t r = hi[t];
      if (r < 0 || r >= n) { err = "hole interior index out of range"; return TDGL_EINVAL; }
      nf[ref_to_dev(r)] |= (uint8_t)(NF_HOLEX << a);
    }
  }
  // kappa at interior nodes: one scalar when uniform, else per node
  double kap0 = gd->kappa;
  std::vector<double> k2;
  bool kappa_uniform = true;
  if (md && md->kappa_full) {
    k2.assign(n, 0.0);
    kap0 = md->kappa_full[1 + mjr + (d3 ? mkr : 0)];
    for (long k = (d3 ? 1 : 0); k <= (d3 ? Nz - 1 : 0); ++k)
      for (long j = 1; j <= ny; ++j)
        for (long i = 1; i <= nx; ++i) {
          double kv = md->kappa_full[i + mjr * j + mkr * k];
          k2[dev_of(i, j, k)] = kv * kv;
          if (kv != kap0) kappa_uniform = false;
        }
  }
  g.kappa2 = kap0 * kap0;
  g.kappa_per_node = !kappa_uniform;
  if (kappa_uniform) k2.clear();
  // superconducting fraction: flags for 0 and 1, an array only for other values
  std::vector<double> scv;
  bool sc_frac = false;
  g.has_material = (md && md->sc_interior) ? 1 : 0;
  if (g.has_material) {
    scv.assign(n, 1.0);
    for (long r = 0; r < n; ++r) {
      double s = md->sc_interior[r];
      long d = ref_to_dev(r);
      scv[d] = s;
      if (s == 0.0) nf[d] |= NF_SC0;
      else if (s != 1.0) { nf[d] |= NF_SCFRAC; sc_frac = true; }
    }
    if (!sc_frac) scv.clear();
  }
  // slow path: a neighbour (3x3x3) is a face or edge node, sits on a zeroed
  // plane (i = Nx-1, j = Ny-1, k = Nz-1) or carries a hole link
  for (long k = (d3 ? 1 : 0); k <= (d3 ? Nz - 1 : 0); ++k)
    for (long j = 1; j <= Ny - 1; ++j)
      for (long i = 1; i <= Nx - 1; ++i) {
        bool slow = i < 2 || i > Nx - 3 || j < 2 || j > Ny - 3 || (d3 && (k < 2 || k > Nz - 3));
        if (!slow && any_hole) {
          for (int dk = (d3 ? -1 : 0); dk <= (d3 ? 1 : 0) && !slow; ++dk)
            for (int dj = -1; dj <= 1 && !slow; ++dj)
              for (int di = -1; di <= 1 && !slow; ++di)
                if (lf[(i + di) + mj * (j + dj) + mk * (k + dk)]) slow = true;
        }
        if (slow) nf[dev_of(i, j, k)] |= NF_SLOW;
      }
  // face copies (the ghost node across each face that a face node writes):
  // NF_GHOSTLF where such a ghost carries hole links, so that the copies read
  // the link flags only at those nodes
  if (any_hole) {
    for (long k = (d3 ? 1 : 0); k <= (d3 ? Nz - 1 : 0); ++k)
      for (long j = 1; j <= Ny - 1; ++j)
        for (long i = 1; i <= Nx - 1; ++i) {
          bool h = false;
          auto ghost = [&](long gi, long gj, long gk) { h = h || lf[gi + mj * gj + mk * gk] != 0; };
          if (i == 1) ghost(g.px ? Nx : 0, j, k);
          if (i == Nx - 1) ghost(g.px ? 0 : Nx, j, k);
          if (j == 1) ghost(i, g.py ? Ny : 0, k);
          if (j == Ny - 1) ghost(i, g.py ? 0 : Ny, k);
          if (d3 && k == 1) ghost(i, j, g.pz ? Nz : 0);
          if (d3 && k == Nz - 1) ghost(i, j, g.pz ? 0 : Nz);
          if (h) nf[dev_of(i, j, k)] |= NF_GHOSTLF;
        }
  }
  // slow nodes grouped by 128-node region (the unit of work of one warp)
  const long nreg = g.npad / 128;
  out.slow_off.assign(nreg + 1, 0);
  out.slow_idx.clear();
  for (long r = 0; r < nreg; ++r) {
    out.slow_off[r] = (int)out.slow_idx.size();
    for (long d = r * 128; d < std::min(n, (r + 1) * 128); ++d)
      if (nf[d] & NF_SLOW) out.slow_idx.push_back((int)d);
  }
  out.slow_off[nreg] = (int)out.slow_idx.size();
  if (!any_hole) lf.clear();
  out.lflags.swap(lf);
  out.nflags.swap(nf);
  out.k2.swap(k2);
  out.sc.swap(scv);
  return TDGL_OK;
}

}  // namespace tdgl
