// Adjoint (vector-Jacobian product) of the TDGL right-hand side.
//
// For a direction v in the device layout, one thread per interior node m
// recomputes the forward intermediates of rhs_body at m, runs the reverse
// pass of its arithmetic, and scatters the adjoint of every value it read back
// to where that value came from.  A read goes through the boundary procedure
// (src/tdgl3d/physics/rhs.py:54-139), so its adjoint is sent through the same
// rules in reverse: to the interior node a face value copies (the opposite
// side when periodic), nowhere for edges, dead normal links and hole links,
// and, for a tangential face link, also to the applied field through its
// +-B h h offset.  Outputs:
//   gx      d(v . f)/dx   (device layout, accumulated with FP64 atomics)
//   gsc     d(v . f)/d sc per interior node (device order; with a material)
//   gk2     d(v . f)/d kappa^2 per interior node (device order)
//   gB      d(v . f)/d(Bx, By, Bz) (block partials, then atomics)
// All in FP64.
#pragma once

#include "tdgl_common.cuh"

namespace tdgl {

// Scatter target of the reverse pass at node (i, j, k).
struct AdjSink {
  const Grid* g;
  int i, j, k;
  double* gx;
  double hxy, hzx, hyz;        // d offset / dB: hx hy (Bz), hz hx (By), hy hz (Bx)
  double gB[3];                // Bx, By, Bz

  __device__ __forceinline__ bool face(int& ii, int& jj, int& kk, int& ox, int& oy, int& oz) const {
    ox = ii <= 0 ? -1 : (ii >= g->Nx ? 1 : 0);
    oy = jj <= 0 ? -1 : (jj >= g->Ny ? 1 : 0);
    oz = g->is3d ? (kk <= 0 ? -1 : (kk >= g->Nz ? 1 : 0)) : 0;
    return (ox != 0) + (oy != 0) + (oz != 0) <= 1;
  }
  __device__ __forceinline__ void add(int c, int ii, int jj, int kk, double v) const {
    atomicAdd(&gx[(long)c * g->npad + dix(*g, ii, jj, kk)], v);
  }
  // psi read at (i + di, j + dj, k + dk): face values copy an interior psi
  __device__ __forceinline__ void psi(int di, int dj, int dk, double br, double bi) {
    int ii = i + di, jj = j + dj, kk = k + dk, ox, oy, oz;
    if (!face(ii, jj, kk, ox, oy, oz)) return;              // edge: zero
    if (ox) ii = g->px ? (ox < 0 ? g->Nx - 1 : 1) : (ox < 0 ? 1 : g->Nx - 1);
    else if (oy) jj = g->py ? (oy < 0 ? g->Ny - 1 : 1) : (oy < 0 ? 1 : g->Ny - 1);
    else if (oz) kk = g->pz ? (oz < 0 ? g->Nz - 1 : 1) : (oz < 0 ? 1 : g->Nz - 1);
    add(PR, ii, jj, kk, br);
    add(PI, ii, jj, kk, bi);
  }
  __device__ __forceinline__ bool dead(int a, int ii, int jj, int kk) const {
    return (a == 0 && ii == g->Nx - 1) || (a == 1 && jj == g->Ny - 1) || (a == 2 && kk == g->Nz - 1);
  }
  __device__ __forceinline__ bool hole(int a, int ii, int jj, int kk) const {
    return g->lflags && ((g->lflags[ii + g->mj * jj + g->mk * kk] >> a) & 1u);
  }
  // link a read at (i + di, j + dj, k + dk)
  __device__ __forceinline__ void phi(int a, int di, int dj, int dk, double b) {
    int ii = i + di, jj = j + dj, kk = k + dk, ox, oy, oz;
    if (!face(ii, jj, kk, ox, oy, oz)) return;
    if (hole(a, ii, jj, kk)) return;
    const int nb = (ox != 0) + (oy != 0) + (oz != 0);
    if (nb == 0) {
      if (!dead(a, ii, jj, kk)) add(AX + a, ii, jj, kk, b);
      return;
    }
    const int f = ox ? 0 : (oy ? 1 : 2);
    const int side = ox ? ox : (oy ? oy : oz);
    const int per = f == 0 ? g->px : (f == 1 ? g->py : g->pz);
    if (per) {
      if (a != f || side < 0) return;
      if (f == 0) ii = 1; else if (f == 1) jj = 1; else kk = 1;
      if (!dead(a, ii, jj, kk)) add(AX + a, ii, jj, kk, b);
      return;
    }
    if (a == f) return;
    // offset c = s * B * h h with the forward's signs (Ext::phi)
    double sgn;
    int which;                 // 0: Bx, 1: By, 2: Bz
    double hh;
    if (f == 0) { if (a == 1) { sgn = -1; which = 2; hh = hxy; } else { sgn = 1; which = 1; hh = hzx; } }
    else if (f == 1) { if (a == 0) { sgn = 1; which = 2; hh = hxy; } else { sgn = -1; which = 0; hh = hyz; } }
    else { if (a == 0) { sgn = -1; which = 1; hh = hzx; } else { sgn = 1; which = 0; hh = hyz; } }
    if (side > 0) sgn = -sgn;
    gB[which] += sgn * hh * b;
    if (f == 0) ii = side < 0 ? 1 : g->Nx - 1;
    else if (f == 1) jj = side < 0 ? 1 : g->Ny - 1;
    else kk = side < 0 ? 1 : g->Nz - 1;
    if (!dead(a, ii, jj, kk)) add(AX + a, ii, jj, kk, b);
  }
};

// Reverse pass of rhs_body at one node.  v: the node's adjoint seed (five
// components, links already masked where the forward output is masked).
// Returns d(v . f)/d sc and d(v . f)/d kappa^2 of the node.
template <bool D3, class XAcc>
__device__ void rhs_adjoint(const Grid& g, const XAcc& X, const NodeCoef<double>& nc, const double v[5], AdjSink& S,
                            double& sc_bar, double& k2_bar) {
  const double bre = v[PR], bim = v[PI];
  const double bf[3] = {v[AX], v[AY], D3 ? v[AZ] : 0.0};
  double cr, ci;
  X.psi(0, 0, 0, cr, ci);
  double cr_bar = 0.0, ci_bar = 0.0;
#pragma unroll
  for (int a = 0; a < (D3 ? 3 : 2); ++a) {
    const int ex = a == 0, ey = a == 1, ez = a == 2;
    double pmr, pmi, ppr, ppi;
    X.psi(-ex, -ey, -ez, pmr, pmi);
    X.psi(ex, ey, ez, ppr, ppi);
    const double am = X.phi(a, -ex, -ey, -ez), a0 = X.phi(a, 0, 0, 0);
    double sm, cm, s0, c0;
    sincos(am, &sm, &cm);
    sincos(a0, &s0, &c0);
    const double ih = a == 0 ? g.ihx2 : (a == 1 ? g.ihy2 : g.ihz2);
    const double Lr = bre * ih, Li = bim * ih, sb = bf[a];
    const double ur = c0 * cr - s0 * ci, ui = -(s0 * cr + c0 * ci);
    S.psi(-ex, -ey, -ez, Lr * cm - Li * sm, Lr * sm + Li * cm);
    S.psi(ex, ey, ez, Lr * c0 + Li * s0 + sb * ui, -Lr * s0 + Li * c0 + sb * ur);
    cr_bar += -2.0 * Lr;
    ci_bar += -2.0 * Li;
    const double cm_bar = Lr * pmr + Li * pmi, sm_bar = Lr * pmi - Li * pmr;
    double c0_bar = Lr * ppr + Li * ppi, s0_bar = -Lr * ppi + Li * ppr;
    const double ur_bar = sb * ppi, ui_bar = sb * ppr;
    c0_bar += ur_bar * cr - ui_bar * ci;
    s0_bar += -ur_bar * ci - ui_bar * cr;
    cr_bar += ur_bar * c0 - ui_bar * s0;
    ci_bar += -ur_bar * s0 - ui_bar * c0;
    S.phi(a, -ex, -ey, -ez, -sm * cm_bar + cm * sm_bar);
    S.phi(a, 0, 0, 0, -s0 * c0_bar + c0 * s0_bar);
  }
  // Ginzburg-Landau / relaxation term
  const double m2 = cr * cr + ci * ci;
  const double sc = nc.material ? (double)nc.sc : 1.0;
  const double lin = nc.material ? sc * (1.0 - m2) - (1.0 - sc) / kTauRelax : (1.0 - m2);
  cr_bar += bre * lin;
  ci_bar += bim * lin;
  const double m2_bar = -sc * (bre * cr + bim * ci);
  cr_bar += 2.0 * cr * m2_bar;
  ci_bar += 2.0 * ci * m2_bar;
  sc_bar = nc.material ? bre * ((1.0 - m2) * cr + cr / kTauRelax) + bim * ((1.0 - m2) * ci + ci / kTauRelax) : 0.0;
  S.psi(0, 0, 0, cr_bar, ci_bar);

  // links: every term is coefficient x link
  const double cx = nc.cx, cy = nc.cy, cz = nc.cz;
  const double bx = bf[0], by = bf[1], bz = bf[2];
  // reads (names as in rhs_body)
  const double fx0 = X.phi(0, 0, 0, 0), fxxm = X.phi(0, -1, 0, 0), fxxp = X.phi(0, 1, 0, 0);
  const double fxym = X.phi(0, 0, -1, 0), fxyp = X.phi(0, 0, 1, 0);
  const double fy0 = X.phi(1, 0, 0, 0), fyxm = X.phi(1, -1, 0, 0), fyxp = X.phi(1, 1, 0, 0);
  const double fyym = X.phi(1, 0, -1, 0), fyyp = X.phi(1, 0, 1, 0);
  const double fxypxm = X.phi(0, -1, 1, 0), fyxpym = X.phi(1, 1, -1, 0);
  // d(dfx), d(dfy) wrt the coefficients, for the kappa^2 gradient
  double dcx = bx * (-4.0 * fx0 + 2.0 * (fxxm + fxxp)) + by * (-2.0 * fy0 + (fyxm + fyxp) + (-fxyp + fx0 + fxypxm - fxxm));
  double dcy = bx * (-2.0 * fx0 + (fxym + fxyp) + (-fyxp + fy0 + fyxpym - fyym)) + by * (-4.0 * fy0 + 2.0 * (fyym + fyyp));
  double dcz = 0.0;
  // dfx terms
  S.phi(0, 0, 0, 0, -2.0 * (2.0 * cx + cy + cz) * bx + cx * by);
  S.phi(0, -1, 0, 0, 2.0 * cx * bx - cx * by);
  S.phi(0, 1, 0, 0, 2.0 * cx * bx);
  S.phi(0, 0, -1, 0, cy * bx);
  S.phi(0, 0, 1, 0, cy * bx - cx * by);
  S.phi(1, 1, 0, 0, -cy * bx + cx * by);
  S.phi(1, 0, 0, 0, cy * bx - 2.0 * (cx + 2.0 * cy + cz) * by);
  S.phi(1, 1, -1, 0, cy * bx);
  S.phi(1, 0, -1, 0, -cy * bx + 2.0 * cy * by);
  // dfy terms not yet sent
  S.phi(1, -1, 0, 0, cx * by);
  S.phi(1, 0, 1, 0, 2.0 * cy * by);
  S.phi(0, -1, 1, 0, cx * by);
  if constexpr (D3) {
    const double fxzm = X.phi(0, 0, 0, -1), fxzp = X.phi(0, 0, 0, 1);
    const double fyzm = X.phi(1, 0, 0, -1), fyzp = X.phi(1, 0, 0, 1);
    const double fz0 = X.phi(2, 0, 0, 0), fzxm = X.phi(2, -1, 0, 0), fzxp = X.phi(2, 1, 0, 0);
    const double fzym = X.phi(2, 0, -1, 0), fzyp = X.phi(2, 0, 1, 0);
    const double fzzm = X.phi(2, 0, 0, -1), fzzp = X.phi(2, 0, 0, 1);
    const double fzxpzm = X.phi(2, 1, 0, -1), fzypzm = X.phi(2, 0, 1, -1);
    const double fxzpxm = X.phi(0, -1, 0, 1), fyzpym = X.phi(1, 0, -1, 1);
    dcx += bz * (-2.0 * fz0 + (fzxm + fzxp) + (-fxzp + fx0 + fxzpxm - fxxm));
    dcy += bz * (-2.0 * fz0 + (fzym + fzyp) + (-fyzp + fy0 + fyzpym - fyym));
    dcz = bx * (-2.0 * fx0 + (fxzm + fxzp) + (-fzxp + fz0 + fzxpzm - fzzm)) +
          by * (-2.0 * fy0 + (fyzm + fyzp) + (-fzyp + fz0 + fzypzm - fzzm)) +
          bz * (-4.0 * fz0 + 2.0 * (fzzm + fzzp));
    // dfx: + cz (fxzm + fxzp) + cz (-fzxp + fz0 + fzxpzm - fzzm)
    S.phi(0, 0, 0, -1, cz * bx);
    S.phi(0, 0, 0, 1, cz * bx - cx * bz);
    S.phi(2, 1, 0, 0, -cz * bx + cx * bz);
    S.phi(2, 0, 0, 0, cz * bx + cz * by - 2.0 * (cx + cy + 2.0 * cz) * bz);
    S.phi(2, 1, 0, -1, cz * bx);
    S.phi(2, 0, 0, -1, -cz * bx - cz * by + 2.0 * cz * bz);
    // dfy: + cz (fyzm + fyzp) + cz (-fzyp + fz0 + fzypzm - fzzm)
    S.phi(1, 0, 0, -1, cz * by);
    S.phi(1, 0, 0, 1, cz * by - cy * bz);
    S.phi(2, 0, 1, 0, -cz * by + cy * bz);
    S.phi(2, 0, 1, -1, cz * by);
    // dfz: cx (fzxm + fzxp) + cy (fzym + fzyp) + 2cz fzzp
    //      + cx (-fxzp + fx0 + fxzpxm - fxxm) + cy (-fyzp + fy0 + fyzpym - fyym)
    S.phi(2, -1, 0, 0, cx * bz);
    S.phi(2, 0, -1, 0, cy * bz);
    S.phi(2, 0, 0, 1, 2.0 * cz * bz);
    S.phi(0, 0, 0, 0, cx * bz);
    S.phi(0, -1, 0, 1, cx * bz);
    S.phi(0, -1, 0, 0, -cx * bz);
    S.phi(1, 0, 0, 0, cy * bz);
    S.phi(1, 0, -1, 1, cy * bz);
    S.phi(1, 0, -1, 0, -cy * bz);
  }
  k2_bar = dcx / g.hx2 + dcy / g.hy2 + (D3 ? dcz / g.hz2 : 0.0);
}

// gx += J(x)^T v, gsc / gk2 per node, gB partials (one slot per block, 3 values).
template <bool D3>
__global__ void __launch_bounds__(kThreads) k_vjp(Grid g, const double* x, const double* v, BTerms<double> b,
                                                  double* gx, double* gsc, double* gk2, double* gB_part) {
  __shared__ double red[kWarps][3];
  AdjSink S{&g, 0, 0, 0, gx, g.hx * g.hy, g.hz * g.hx, g.hy * g.hz, {0.0, 0.0, 0.0}};
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    int i, j, k;
    node_ijk(g, d, i, j, k);
    S.i = i; S.j = j; S.k = k;
    const uint8_t nf = g.nflags[d];
    NodeCoef<double> nc = node_coef<double>(g, d, nf);
    double vv[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int c = 0; c < (D3 ? 5 : 4); ++c) vv[c] = v[(long)c * g.npad + d];
    if (nf & NF_HOLEX) vv[AX] = 0.0;
    if (nf & NF_HOLEY) vv[AY] = 0.0;
    if (D3 && (nf & NF_HOLEZ)) vv[AZ] = 0.0;
    NbSlow<double, SrcVec<double, double>> X{Ext<double, SrcVec<double, double>>{&g, SrcVec<double, double>{x, g.npad}, b},
                                            i, j, k};
    double sc_bar, k2_bar;
    rhs_adjoint<D3>(g, X, nc, vv, S, sc_bar, k2_bar);
    if (gsc) gsc[d] = sc_bar;
    if (gk2) gk2[d] = k2_bar;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    double a = warp_sum(S.gB[s]);
    if (lane == 0) red[warp][s] = a;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double a = 0.0;
    for (int w = 0; w < kWarps; ++w) a += red[w][threadIdx.x];
    gB_part[(long)threadIdx.x * gridDim.x + blockIdx.x] = a;
  }
}

}  // namespace tdgl
