// Boundary-extended stencils of the TDGL right-hand side and its Jacobian.
//
// The reference evaluates dX/dt by scattering the interior state into a full
// (Nx+1)(Ny+1)(Nz+1) grid, writing boundary values, building scipy CSR
// operators and multiplying (src/tdgl3d/physics/rhs.py:147-239,
// src/tdgl3d/operators/sparse_operators.py:35-317).  Here every output node
// reads its 3x3x3 neighbourhood directly; a neighbour that is not a plain
// interior value is produced on the fly by the same boundary rules
// (src/tdgl3d/physics/rhs.py:54-139):
//
//   * the normal link is zero on planes 0 and N-1 of its own axis;
//   * on a face (one index at 0 or N, the other two inner):
//       psi    = psi of the adjacent interior node (zero-current; the Peierls
//                factor there is e^{0} = 1 because the link it uses is zeroed),
//                or of the opposite side when that axis is periodic;
//       normal link = 0 (periodic: the wrapped link, zero on the low face);
//       tangential links = +-B h h offset + adjacent interior link
//                (zero when the face's axis is periodic);
//   * edges and corners are zero;
//   * hole-boundary links are zero after all of the above; the values written
//     on faces still read the adjacent link before that zeroing.
//
// All functions are plain arithmetic on (i, j, k) and compile for the host as
// well, so the CPU test suite can check the index logic against the oracle.
#pragma once

#include <cstdint>
#include <cmath>

#ifdef __CUDACC__
#define TDGL_HD __host__ __device__ __forceinline__
#else
#define TDGL_HD inline
#endif

namespace tdgl {

// Device state layout: component-major arrays of length npad, interior nodes
// numbered d = (i-1) + nx*((j-1) + ny*(k-1)) (i fastest).
enum Comp : int { PR = 0, PI = 1, AX = 2, AY = 3, AZ = 4 };

// Per-interior-node flags (device order).
enum : uint8_t {
  NF_SLOW = 1u << 0,    // neighbourhood reaches a face, a zeroed link or a hole link
  NF_HOLEX = 1u << 1,   // d(phi_x)/dt := 0 (hole-boundary link, rhs.py:229-234)
  NF_HOLEY = 1u << 2,
  NF_HOLEZ = 1u << 3,
  NF_SC0 = 1u << 4,     // sc == 0: pure relaxation -psi/tau
  NF_SCFRAC = 1u << 5,  // sc not in {0, 1}: read the sc array
  NF_GHOSTLF = 1u << 6, // a face copy of this node lands on a ghost with hole links
};
// Per-full-grid-node link flags.
enum : uint8_t { LF_HX = 1u, LF_HY = 2u, LF_HZ = 4u };

constexpr double kTauRelax = 0.1;   // src/tdgl3d/operators/sparse_operators.py:223

// v / tau_relax.  FP64 divides, as the reference does; FP32 (the Jacobian
// products of the mixed form) multiplies by the reciprocal 10, which agrees
// with the FP32 quotient to within one rounding and avoids a division
// sequence per node.
template <typename T> TDGL_HD T over_tau(T v) { return v / (T)kTauRelax; }
template <> TDGL_HD float over_tau<float>(float v) { return v * 10.0f; }

struct Grid {
  int Nx, Ny, Nz;          // cells
  int nx, ny, nz;          // interior extents (nz = 1 in 2-D)
  int is3d;
  int px, py, pz;          // periodic flags
  int n, npad, ncomp;      // interior nodes, component stride, components (4 or 5)
  int mj, mk;              // full-grid strides
  double hx, hy, hz;
  double ihx2, ihy2, ihz2; // 1/h^2 (psi Laplacian)
  double hx2, hy2, hz2;    // h^2 (kappa^2 / h^2 of the link Laplacians)
  double kappa2;           // uniform kappa^2
  int has_material;        // FPSI uses sc (else the bare GL term)
  int kappa_per_node;
  const uint8_t* lflags;   // full grid link flags, or nullptr when there are no holes
  const uint8_t* nflags;   // interior node flags, device order
  const double* k2int;     // kappa^2 per interior node (device order) or nullptr
  const double* scint;     // sc per interior node (device order) or nullptr
  const int* slow_off;     // per 128-node region: offsets into slow_idx (nregions + 1)
  const int* slow_idx;     // nodes with NF_SLOW, grouped by region, ascending
};

// Applied-field offsets of the tangential face links, in the reference's
// product order: Bz*hx*hy, By*hz*hx, Bx*hy*hz.
template <typename T>
struct BTerms {
  T czxy, cyzx, cxyz;
};

template <typename T> TDGL_HD void sincos_t(T a, T* s, T* c);
template <> TDGL_HD void sincos_t<double>(double a, double* s, double* c) {
#ifdef __CUDA_ARCH__
  sincos(a, s, c);
#else
  *s = std::sin(a); *c = std::cos(a);
#endif
}
// Single precision only carries Jacobian products of the mixed form (Krylov
// directions); the hardware approximation (abs. error < 2^-21 on [-pi, pi])
// is below the float rounding those products already have.
template <> TDGL_HD void sincos_t<float>(float a, float* s, float* c) {
#ifdef __CUDA_ARCH__
  __sincosf(a, s, c);
#else
  *s = std::sin(a); *c = std::cos(a);
#endif
}

TDGL_HD int dix(const Grid& g, int i, int j, int k) {
  return (i - 1) + g.nx * ((j - 1) + g.ny * (g.is3d ? (k - 1) : 0));
}

// ---------------------------------------------------------------------------
// Sources: interior values of one device-layout vector by (component, node).
// ---------------------------------------------------------------------------

template <typename T, typename S>
struct SrcVec {                       // v
  const S* v; int npad;
  TDGL_HD T operator()(int c, int d) const { return (T)v[(long)c * npad + d]; }
};

template <typename T, typename S>
struct SrcAxpy {                      // a - beta * b
  const S* a; const S* b; T beta; int npad;
  TDGL_HD T operator()(int c, int d) const {
    long e = (long)c * npad + d;
    T av = (T)a[e];
    return b ? av - beta * (T)b[e] : av;
  }
};

template <typename S>
struct SrcFD {                        // x + eps * (r - beta * b)   (finite-difference point)
  const double* x; const S* r; const S* b; double beta; double eps; int npad;
  TDGL_HD double operator()(int c, int d) const {
    long e = (long)c * npad + d;
    double p = (double)r[e];
    if (b) p = p - beta * (double)b[e];
    return x[e] + eps * p;
  }
};

// ---------------------------------------------------------------------------
// Boundary-extended full-grid values.
// ---------------------------------------------------------------------------

template <typename T, class Src>
struct Ext {
  const Grid* g; Src s; BTerms<T> b;

  TDGL_HD bool hole(int a, int i, int j, int k) const {
    if (!g->lflags) return false;
    return (g->lflags[i + g->mj * j + g->mk * k] >> a) & 1u;
  }
  // interior link after the normal-plane zeroing, before hole zeroing
  TDGL_HD T phit(int a, int i, int j, int k) const {
    if ((a == 0 && i == g->Nx - 1) || (a == 1 && j == g->Ny - 1) || (a == 2 && k == g->Nz - 1)) return T(0);
    return s(AX + a, dix(*g, i, j, k));
  }
  TDGL_HD void face(int i, int j, int k, int& ox, int& oy, int& oz) const {
    ox = i <= 0 ? -1 : (i >= g->Nx ? 1 : 0);
    oy = j <= 0 ? -1 : (j >= g->Ny ? 1 : 0);
    oz = g->is3d ? (k <= 0 ? -1 : (k >= g->Nz ? 1 : 0)) : 0;
  }
  TDGL_HD void psi(int i, int j, int k, T& re, T& im) const {
    int ox, oy, oz;
    face(i, j, k, ox, oy, oz);
    int nb = (ox != 0) + (oy != 0) + (oz != 0);
    if (nb > 1) { re = T(0); im = T(0); return; }
    if (ox) i = g->px ? (ox < 0 ? g->Nx - 1 : 1) : (ox < 0 ? 1 : g->Nx - 1);
    else if (oy) j = g->py ? (oy < 0 ? g->Ny - 1 : 1) : (oy < 0 ? 1 : g->Ny - 1);
    else if (oz) k = g->pz ? (oz < 0 ? g->Nz - 1 : 1) : (oz < 0 ? 1 : g->Nz - 1);
    int d = dix(*g, i, j, k);
    re = s(PR, d);
    im = s(PI, d);
  }
  TDGL_HD T phi(int a, int i, int j, int k) const {
    int ox, oy, oz;
    face(i, j, k, ox, oy, oz);
    int nb = (ox != 0) + (oy != 0) + (oz != 0);
    if (nb > 1) return T(0);
    if (hole(a, i, j, k)) return T(0);
    if (nb == 0) return phit(a, i, j, k);
    int f = ox ? 0 : (oy ? 1 : 2);
    int side = ox ? ox : (oy ? oy : oz);
    int per = f == 0 ? g->px : (f == 1 ? g->py : g->pz);
    if (per) {
      if (a != f || side < 0) return T(0);
      if (f == 0) i = 1; else if (f == 1) j = 1; else k = 1;
      return phit(a, i, j, k);
    }
    if (a == f) return T(0);
    T c;
    if (f == 0) c = (a == 1) ? -b.czxy : b.cyzx;
    else if (f == 1) c = (a == 0) ? b.czxy : -b.cxyz;
    else c = (a == 0) ? -b.cyzx : b.cxyz;
    if (side > 0) c = -c;
    if (f == 0) i = side < 0 ? 1 : g->Nx - 1;
    else if (f == 1) j = side < 0 ? 1 : g->Ny - 1;
    else k = side < 0 ? 1 : g->Nz - 1;
    return c + phit(a, i, j, k);
  }
};

// Neighbourhood accessors relative to the output node: a fast one for nodes
// whose whole 3x3x3 neighbourhood is plain interior data, and the general one.
template <typename T, class Src>
struct NbFast {
  Src s; int d, sy, sz;
  TDGL_HD void psi(int di, int dj, int dk, T& re, T& im) const {
    int e = d + di + dj * sy + dk * sz;
    re = s(PR, e);
    im = s(PI, e);
  }
  TDGL_HD T phi(int a, int di, int dj, int dk) const { return s(AX + a, d + di + dj * sy + dk * sz); }
};

template <typename T, class Src>
struct NbSlow {
  Ext<T, Src> e; int i, j, k;
  TDGL_HD void psi(int di, int dj, int dk, T& re, T& im) const { e.psi(i + di, j + dj, k + dk, re, im); }
  TDGL_HD T phi(int a, int di, int dj, int dk) const { return e.phi(a, i + di, j + dj, k + dk); }
};

// Per-node material coefficients.
template <typename T>
struct NodeCoef {
  T cx, cy, cz;     // kappa(m)^2 / h^2 (cz = 0 in 2-D)
  T sc;             // superconducting fraction (1 without material)
  bool material;
  T ihx, ihy, ihz;  // 1 / h^2 of the psi Laplacian
};

template <typename T>
TDGL_HD void set_ih(const Grid& g, NodeCoef<T>& nc) {
  nc.ihx = (T)g.ihx2;
  nc.ihy = (T)g.ihy2;
  nc.ihz = (T)g.ihz2;
}

template <typename T>
TDGL_HD NodeCoef<T> node_coef(const Grid& g, int d, uint8_t nf) {
  NodeCoef<T> nc;
  double k2 = g.kappa_per_node ? g.k2int[d] : g.kappa2;
  nc.cx = (T)(k2 / g.hx2);
  nc.cy = (T)(k2 / g.hy2);
  nc.cz = g.is3d ? (T)(k2 / g.hz2) : T(0);
  nc.material = g.has_material != 0;
  if (!nc.material) nc.sc = T(1);
  else if (nf & NF_SCFRAC) nc.sc = (T)g.scint[d];
  else nc.sc = (nf & NF_SC0) ? T(0) : T(1);
  set_ih(g, nc);
  return nc;
}

// ---------------------------------------------------------------------------
// RHS at one interior node: out[PR..AZ] = dX/dt.
// ---------------------------------------------------------------------------

template <typename T, bool D3, class A>
TDGL_HD void rhs_body(const Grid& g, const A& X, const NodeCoef<T>& nc, uint8_t nf, T out[5]) {
  T cr, ci;
  X.psi(0, 0, 0, cr, ci);
  T sup[3] = {T(0), T(0), T(0)};
  T dre = T(0), dim = T(0);
  // gauge-covariant psi Laplacian and the supercurrent along each axis
#pragma unroll
  for (int a = 0; a < (D3 ? 3 : 2); ++a) {
    int ex = a == 0, ey = a == 1, ez = a == 2;
    T pmr, pmi, ppr, ppi;
    X.psi(-ex, -ey, -ez, pmr, pmi);
    X.psi(ex, ey, ez, ppr, ppi);
    T am = X.phi(a, -ex, -ey, -ez), a0 = X.phi(a, 0, 0, 0);
    T sm, cm, s0, c0;
    sincos_t<T>(am, &sm, &cm);
    sincos_t<T>(a0, &s0, &c0);
    T Lr = (cm * pmr + sm * pmi) - T(2) * cr + (c0 * ppr - s0 * ppi);
    T Li = (cm * pmi - sm * pmr) - T(2) * ci + (c0 * ppi + s0 * ppr);
    T ih = (T)(a == 0 ? g.ihx2 : (a == 1 ? g.ihy2 : g.ihz2));
    dre += Lr * ih;
    dim += Li * ih;
    // Im[e^{-i a0} conj(psi) psi(m+a)]
    T ur = c0 * cr - s0 * ci, ui = -(s0 * cr + c0 * ci);
    sup[a] = ur * ppi + ui * ppr;
  }
  T m2 = cr * cr + ci * ci;
  T glr = (T(1) - m2) * cr, gli = (T(1) - m2) * ci;
  if (nc.material) {
    dre += nc.sc * glr - over_tau<T>((T(1) - nc.sc) * cr);
    dim += nc.sc * gli - over_tau<T>((T(1) - nc.sc) * ci);
  } else {
    dre += glr;
    dim += gli;
  }
  out[PR] = dre;
  out[PI] = dim;

  const T cx = nc.cx, cy = nc.cy, cz = nc.cz;
  // links (names: f<comp><offsets>)
  T fx0 = X.phi(0, 0, 0, 0), fxxm = X.phi(0, -1, 0, 0), fxxp = X.phi(0, 1, 0, 0);
  T fxym = X.phi(0, 0, -1, 0), fxyp = X.phi(0, 0, 1, 0);
  T fy0 = X.phi(1, 0, 0, 0), fyxm = X.phi(1, -1, 0, 0), fyxp = X.phi(1, 1, 0, 0);
  T fyym = X.phi(1, 0, -1, 0), fyyp = X.phi(1, 0, 1, 0);
  T fxypxm = X.phi(0, -1, 1, 0);     // phi_x(m + y - x)
  T fyxpym = X.phi(1, 1, -1, 0);     // phi_y(m + x - y)
  T dfx = T(-2) * (T(2) * cx + cy + cz) * fx0 + T(2) * cx * (fxxm + fxxp) + cy * (fxym + fxyp)
          + sup[0] + cy * (-fyxp + fy0 + fyxpym - fyym);
  T dfy = T(-2) * (cx + T(2) * cy + cz) * fy0 + cx * (fyxm + fyxp) + T(2) * cy * (fyym + fyyp)
          + sup[1] + cx * (-fxyp + fx0 + fxypxm - fxxm);
  T dfz = T(0);
  if constexpr (D3) {
    T fxzm = X.phi(0, 0, 0, -1), fxzp = X.phi(0, 0, 0, 1);
    T fyzm = X.phi(1, 0, 0, -1), fyzp = X.phi(1, 0, 0, 1);
    T fz0 = X.phi(2, 0, 0, 0), fzxm = X.phi(2, -1, 0, 0), fzxp = X.phi(2, 1, 0, 0);
    T fzym = X.phi(2, 0, -1, 0), fzyp = X.phi(2, 0, 1, 0);
    T fzzm = X.phi(2, 0, 0, -1), fzzp = X.phi(2, 0, 0, 1);
    T fzxpzm = X.phi(2, 1, 0, -1);   // phi_z(m + x - z)
    T fzypzm = X.phi(2, 0, 1, -1);   // phi_z(m + y - z)
    T fxzpxm = X.phi(0, -1, 0, 1);   // phi_x(m + z - x)
    T fyzpym = X.phi(1, 0, -1, 1);   // phi_y(m + z - y)
    dfx += cz * (fxzm + fxzp) + cz * (-fzxp + fz0 + fzxpzm - fzzm);
    dfy += cz * (fyzm + fyzp) + cz * (-fzyp + fz0 + fzypzm - fzzm);
    dfz = T(-2) * (cx + cy + T(2) * cz) * fz0 + cx * (fzxm + fzxp) + cy * (fzym + fzyp)
          + T(2) * cz * (fzzm + fzzp) + sup[2]
          + cx * (-fxzp + fx0 + fxzpxm - fxxm) + cy * (-fyzp + fy0 + fyzpym - fyym);
  }
  out[AX] = (nf & NF_HOLEX) ? T(0) : dfx;
  out[AY] = (nf & NF_HOLEY) ? T(0) : dfy;
  out[AZ] = (nf & NF_HOLEZ) ? T(0) : dfz;
}

// ---------------------------------------------------------------------------
// Tangent-linear RHS at one node: out = J(x) p, with X the boundary-extended
// state (applied field) and P the boundary-extended direction (no field: the
// boundary maps are affine, so their tangent drops the field offsets).
// ---------------------------------------------------------------------------

template <typename T, bool D3, class AXs, class APs>
TDGL_HD void jvp_body(const Grid& g, const AXs& X, const APs& P, const NodeCoef<T>& nc, uint8_t nf, T out[5]) {
  T cr, ci, dcr, dci;
  X.psi(0, 0, 0, cr, ci);
  P.psi(0, 0, 0, dcr, dci);
  T dsup[3] = {T(0), T(0), T(0)};
  T dre = T(0), dim = T(0);
#pragma unroll
  for (int a = 0; a < (D3 ? 3 : 2); ++a) {
    int ex = a == 0, ey = a == 1, ez = a == 2;
    T pmr, pmi, ppr, ppi, qmr, qmi, qpr, qpi;
    X.psi(-ex, -ey, -ez, pmr, pmi);
    X.psi(ex, ey, ez, ppr, ppi);
    P.psi(-ex, -ey, -ez, qmr, qmi);
    P.psi(ex, ey, ez, qpr, qpi);
    T am = X.phi(a, -ex, -ey, -ez), a0 = X.phi(a, 0, 0, 0);
    T dam = P.phi(a, -ex, -ey, -ez), da0 = P.phi(a, 0, 0, 0);
    T sm, cm, s0, c0;
    sincos_t<T>(am, &sm, &cm);
    sincos_t<T>(a0, &s0, &c0);
    // d[e^{-i am} pm] = e^{-i am} (dpm - i dam pm)
    T vr = qmr + dam * pmi, vi = qmi - dam * pmr;
    T lmr = cm * vr + sm * vi, lmi = cm * vi - sm * vr;
    // d[e^{i a0} pp] = e^{i a0} (dpp + i da0 pp)
    T wr = qpr - da0 * ppi, wi = qpi + da0 * ppr;
    T lpr = c0 * wr - s0 * wi, lpi = c0 * wi + s0 * wr;
    const T ih = a == 0 ? nc.ihx : (a == 1 ? nc.ihy : nc.ihz);
    dre += (lmr - T(2) * dcr + lpr) * ih;
    dim += (lmi - T(2) * dci + lpi) * ih;
    // d Im[e^{-i a0} conj(psi) psi1]
    T ur = c0 * cr - s0 * ci, ui = -(s0 * cr + c0 * ci);        // e^{-i a0} conj(psi)
    T u1r = c0 * dcr - s0 * dci, u1i = -(s0 * dcr + c0 * dci);  // e^{-i a0} conj(dpsi)
    dsup[a] = (u1r * ppi + u1i * ppr) + (ur * qpi + ui * qpr) - da0 * (ur * ppr - ui * ppi);
  }
  T m2 = cr * cr + ci * ci;
  T pr = cr * dcr + ci * dci;
  T dglr = (T(1) - m2) * dcr - T(2) * pr * cr;
  T dgli = (T(1) - m2) * dci - T(2) * pr * ci;
  if (nc.material) {
    dre += nc.sc * dglr - over_tau<T>((T(1) - nc.sc) * dcr);
    dim += nc.sc * dgli - over_tau<T>((T(1) - nc.sc) * dci);
  } else {
    dre += dglr;
    dim += dgli;
  }
  out[PR] = dre;
  out[PI] = dim;

  const T cx = nc.cx, cy = nc.cy, cz = nc.cz;
  T fx0 = P.phi(0, 0, 0, 0), fxxm = P.phi(0, -1, 0, 0), fxxp = P.phi(0, 1, 0, 0);
  T fxym = P.phi(0, 0, -1, 0), fxyp = P.phi(0, 0, 1, 0);
  T fy0 = P.phi(1, 0, 0, 0), fyxm = P.phi(1, -1, 0, 0), fyxp = P.phi(1, 1, 0, 0);
  T fyym = P.phi(1, 0, -1, 0), fyyp = P.phi(1, 0, 1, 0);
  T fxypxm = P.phi(0, -1, 1, 0);
  T fyxpym = P.phi(1, 1, -1, 0);
  T dfx = T(-2) * (T(2) * cx + cy + cz) * fx0 + T(2) * cx * (fxxm + fxxp) + cy * (fxym + fxyp)
          + dsup[0] + cy * (-fyxp + fy0 + fyxpym - fyym);
  T dfy = T(-2) * (cx + T(2) * cy + cz) * fy0 + cx * (fyxm + fyxp) + T(2) * cy * (fyym + fyyp)
          + dsup[1] + cx * (-fxyp + fx0 + fxypxm - fxxm);
  T dfz = T(0);
  if constexpr (D3) {
    T fxzm = P.phi(0, 0, 0, -1), fxzp = P.phi(0, 0, 0, 1);
    T fyzm = P.phi(1, 0, 0, -1), fyzp = P.phi(1, 0, 0, 1);
    T fz0 = P.phi(2, 0, 0, 0), fzxm = P.phi(2, -1, 0, 0), fzxp = P.phi(2, 1, 0, 0);
    T fzym = P.phi(2, 0, -1, 0), fzyp = P.phi(2, 0, 1, 0);
    T fzzm = P.phi(2, 0, 0, -1), fzzp = P.phi(2, 0, 0, 1);
    T fzxpzm = P.phi(2, 1, 0, -1);
    T fzypzm = P.phi(2, 0, 1, -1);
    T fxzpxm = P.phi(0, -1, 0, 1);
    T fyzpym = P.phi(1, 0, -1, 1);
    dfx += cz * (fxzm + fxzp) + cz * (-fzxp + fz0 + fzxpzm - fzzm);
    dfy += cz * (fyzm + fyzp) + cz * (-fzyp + fz0 + fzypzm - fzzm);
    dfz = T(-2) * (cx + cy + T(2) * cz) * fz0 + cx * (fzxm + fzxp) + cy * (fzym + fzyp)
          + T(2) * cz * (fzzm + fzzp) + dsup[2]
          + cx * (-fxzp + fx0 + fxzpxm - fxxm) + cy * (-fyzp + fy0 + fyzpym - fyym);
  }
  out[AX] = (nf & NF_HOLEX) ? T(0) : dfx;
  out[AY] = (nf & NF_HOLEY) ? T(0) : dfy;
  out[AZ] = (nf & NF_HOLEZ) ? T(0) : dfz;
}

// Node coordinates of device index d.
TDGL_HD void node_ijk(const Grid& g, int d, int& i, int& j, int& k) {
  int q = d / g.nx;
  i = d - q * g.nx + 1;
  if (g.is3d) {
    int r = q / g.ny;
    j = q - r * g.ny + 1;
    k = r + 1;
  } else {
    j = q + 1;
    k = 0;
  }
}

// RHS at node d from source s.  _fast: every neighbour is plain interior data
// (node flag NF_SLOW clear); _slow: neighbours through the boundary rules.
template <typename T, bool D3, class Src>
TDGL_HD void rhs_fast(const Grid& g, const Src& s, int d, uint8_t nf, T out[5]) {
  NodeCoef<T> nc = node_coef<T>(g, d, nf);
  NbFast<T, Src> A{s, d, g.nx, g.nx * g.ny};
  rhs_body<T, D3>(g, A, nc, nf, out);
}
template <typename T, bool D3, class Src>
TDGL_HD void rhs_slow(const Grid& g, const Src& s, const BTerms<T>& b, int d, uint8_t nf, T out[5]) {
  NodeCoef<T> nc = node_coef<T>(g, d, nf);
  int i, j, k;
  node_ijk(g, d, i, j, k);
  NbSlow<T, Src> A{Ext<T, Src>{&g, s, b}, i, j, k};
  rhs_body<T, D3>(g, A, nc, nf, out);
}
template <typename T, class Src>
TDGL_HD void rhs_at(const Grid& g, const Src& s, const BTerms<T>& b, int d, T out[5]) {
  uint8_t nf = g.nflags[d];
  if (g.is3d) {
    if (nf & NF_SLOW) rhs_slow<T, true>(g, s, b, d, nf, out);
    else rhs_fast<T, true>(g, s, d, nf, out);
  } else {
    if (nf & NF_SLOW) rhs_slow<T, false>(g, s, b, d, nf, out);
    else rhs_fast<T, false>(g, s, d, nf, out);
  }
}

// Tangent RHS at node d: out = J(x) p.
template <typename T, bool D3, class SrcX, class SrcP>
TDGL_HD void jvp_fast(const Grid& g, const SrcX& sx, const SrcP& sp, int d, uint8_t nf, T out[5]) {
  NodeCoef<T> nc = node_coef<T>(g, d, nf);
  NbFast<T, SrcX> AX_{sx, d, g.nx, g.nx * g.ny};
  NbFast<T, SrcP> AP_{sp, d, g.nx, g.nx * g.ny};
  jvp_body<T, D3>(g, AX_, AP_, nc, nf, out);
}
template <typename T, bool D3, class SrcX, class SrcP>
TDGL_HD void jvp_slow(const Grid& g, const SrcX& sx, const BTerms<T>& b, const SrcP& sp, int d, uint8_t nf,
                      T out[5]) {
  NodeCoef<T> nc = node_coef<T>(g, d, nf);
  int i, j, k;
  node_ijk(g, d, i, j, k);
  BTerms<T> zero{T(0), T(0), T(0)};
  NbSlow<T, SrcX> AX_{Ext<T, SrcX>{&g, sx, b}, i, j, k};
  NbSlow<T, SrcP> AP_{Ext<T, SrcP>{&g, sp, zero}, i, j, k};
  jvp_body<T, D3>(g, AX_, AP_, nc, nf, out);
}
template <typename T, class SrcX, class SrcP>
TDGL_HD void jvp_at(const Grid& g, const SrcX& sx, const BTerms<T>& b, const SrcP& sp, int d, T out[5]) {
  uint8_t nf = g.nflags[d];
  if (g.is3d) {
    if (nf & NF_SLOW) jvp_slow<T, true>(g, sx, b, sp, d, nf, out);
    else jvp_fast<T, true>(g, sx, sp, d, nf, out);
  } else {
    if (nf & NF_SLOW) jvp_slow<T, false>(g, sx, b, sp, d, nf, out);
    else jvp_fast<T, false>(g, sx, sp, d, nf, out);
  }
}

}  // namespace tdgl
