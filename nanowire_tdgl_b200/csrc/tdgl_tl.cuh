// Tangent-linear stencil of the FP32 Krylov solves, staged through shared
// memory by TMA (3-D grids, FP32 vectors).
//
// The operator is the tangent-linear RHS of eval_f (src/tdgl3d/physics/
// rhs.py:147-239; the operators of src/tdgl3d/operators/sparse_operators.py:
// 35-317), applied as in kg_arn_apply / kg_arn_poly: the Arnoldi product
// Z = W - dt/2 J(x) W, or one Horner step of the polynomial preconditioner,
// W_k = e_k V + beta ((W_in - dt/2 J W_in) - theta W_in) / delta.
//
// Each block owns a (32 NX) x 8 tile of interior nodes (NX nodes per thread,
// 32 apart in x; NX = 1 or 2) and marches through a range of z-planes.  For
// every plane it stages a (32 NX + 4) x 10 box of the linearisation copy and
// of the direction vector (all components; the box starts one node before
// the tile in x and y, so the tile's x- and y-neighbours are in it) into a
// ring of shared-memory slots with cp.async.bulk.tensor, one elected thread
// issuing the copies, each slot guarded by an mbarrier that the copies
// complete.  Once a plane has landed, the threads zero the direction's dead
// links in it (normal links on plane N - 1 of their axis, hole links; each
// thread its own positions and one position of the ring around the tile),
// keeping their own raw values; a node then reads its 3 x 3 x 3
// neighbourhood from the slots of planes k - 1, k and k + 1 with constant
// offsets and no selects.  The planes after k + 1 are in flight while plane
// k is computed.
//
// Layout requirements (met by the context): full-grid rows padded to a
// multiple of 4 entries (16 bytes of FP32), component and vector strides
// multiples of 4 entries; the box's x origin 32 b is a multiple of 4 entries,
// the 16-byte alignment every tiled copy needs.  Out-of-range box entries
// (past the grid's last row or column) are filled with zeros by the copy and
// never read.  The tensor maps cover this GPU's own buffers only and the
// copies carry no multicast.
//
// Every wait is bounded: a thread whose mbarrier wait outlasts the context's
// wait limit flags the block; the block then stops, its issuing thread waits
// (bounded again) for the copies still in flight into its shared memory, the
// status GS_TIMEOUT is recorded in the device control block, and every later
// kernel of the graph returns at once.
#pragma once

#include <cuda.h>

#include "tdgl_graph.cuh"

namespace tdgl {

constexpr int kTlTy = 8;                              // tile rows (threads per column of the block)
constexpr int kTlBoxY = kTlTy + 2;                    // staged y extent: j0 - 1 .. j0 + 8
constexpr int kTlComp = 5;                            // components of a 3-D vector
constexpr unsigned long long kTlDrainNs = 2000000000ull;   // bound of the wait for copies in flight

// Shapes of the kernel with NX nodes per thread.
template <int NX>
struct TlShape {
  static constexpr int kTx = 32 * NX;                        // tile width
  static constexpr int kBoxX = kTx + 4;                      // staged x extent: i0 - 1 .. i0 + kTx + 2 (16-byte multiple)
  static constexpr int kPlane = kBoxX * kTlBoxY;             // entries per component and plane
  static constexpr unsigned kBytes = kTlComp * kPlane * 4;   // bytes of one staged box
  static constexpr int kSlotF = (kTlComp * kPlane + 31) / 32 * 32;   // floats per box, rounded up to 128 bytes
  static constexpr int kSlots = NX == 1 ? 5 : 4;             // ring of staged planes
  static constexpr int kAhead = kSlots - 2;                  // planes issued ahead of the one being waited for
  static constexpr size_t kSmem = (size_t)kSlots * 2 * kSlotF * sizeof(float);
  static constexpr int kRing = 2 * (kTx + 2) + 2 * kTlTy;    // positions around the tile that are read
  static constexpr int kMinBlocks = NX == 1 ? 3 : 2;         // resident blocks per SM (shared memory)
  static_assert((kSlotF * 4) % 128 == 0 && kRing <= 256 && (kBoxX * 4) % 16 == 0, "staged box shape");
};

// Tensor maps of the staged vectors: 0 linearisation copy, 1 the basis, 2 and
// 3 the Horner buffers, 4 the preconditioned basis (the bases are 5-D: the
// fifth coordinate is the basis vector).
enum TlMap : int { TM_X = 0, TM_UB = 1, TM_PW0 = 2, TM_PW1 = 3, TM_PB = 4 };
struct alignas(64) TlMaps {
  CUtensorMap m[5];
  int nx;        // nodes per thread along x of the kernel the maps' boxes are shaped for (1 or 2)
};

// Launch shape of kg_tl<.., NX>: grid width and dynamic shared memory.
__host__ __device__ inline int tl_grid_x(int nx, int NX) { return (nx + 32 * NX - 1) / (32 * NX); }
inline size_t tl_smem_bytes(int NX);


__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Order this thread's generic-proxy shared-memory writes before later
// async-proxy (TMA) writes to the same slots.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test_wait(uint64_t* b, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase of parity `parity` of b to complete; false when that takes
// longer than limit_ns.  Non-blocking polls with a short back-off, the clock
// read between polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity, unsigned long long limit_ns) {
  if (mbar_test_wait(b, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_test_wait(b, parity)) {
    if (global_ns() - t0 > limit_ns) return false;
    __nanosleep(20);
  }
  return true;
}
// Tiled tensor copies global -> shared, completing on mbarrier b.
__device__ __forceinline__ void tma_load4(float* dst, const CUtensorMap* m, int c0, int c1, int c2, int c3,
                                          uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(b))
      : "memory");
}
__device__ __forceinline__ void tma_load5(float* dst, const CUtensorMap* m, int c0, int c1, int c2, int c3, int c4,
                                          uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_addr(b))
      : "memory");
}

// Dynamic shared memory of kg_tl: [slots][2][kSlotF] floats (per slot the
// linearisation's box, then the direction's).
extern __shared__ __align__(128) float tl_smem[];

// Neighbourhood of a node in the staged boxes of planes k - 1, k, k + 1:
// entry offsets (in floats) of the node's position in the three boxes; the
// neighbour reads are the offsets plus constants (component blocks of kPlane
// entries, rows of kBoxX).  Dead links of the direction were zeroed in the
// staged boxes, so every read is a plain shared-memory load.
template <int NX>
struct TlNb {
  using S = TlShape<NX>;
  int lo, mid, hi;
  __device__ __forceinline__ int at(int di, int dj, int dk) const {
    return (dk < 0 ? lo : (dk > 0 ? hi : mid)) + di + dj * S::kBoxX;
  }
  __device__ __forceinline__ void psi(int di, int dj, int dk, float& re, float& im) const {
    const int e = at(di, dj, dk);
    re = tl_smem[e];
    im = tl_smem[e + S::kPlane];
  }
  __device__ __forceinline__ float phi(int a, int di, int dj, int dk) const {
    return tl_smem[at(di, dj, dk) + (2 + a) * S::kPlane];
  }
};

// Output node (i, j, k) of a tangent vector on the full grid: its raw values
// and the face values copied from it (write_eff with RAW_OWN and no field
// offsets, in float).
__device__ __forceinline__ void tl_store(const Grid& g, float* E, long npf, long m, int i, int j, int k, bool face,
                                         const float* v) {
  float* e = E + m;
#pragma unroll
  for (int c = 0; c < kTlComp; ++c, e += npf) *e = v[c];
  if (!face) return;
  const float tx = (i == g.Nx - 1) ? 0.0f : v[2];
  const float ty = (j == g.Ny - 1) ? 0.0f : v[3];
  const float tz = (k == g.Nz - 1) ? 0.0f : v[4];
  auto ghost = [&](long mg, float fx, float fy, float fz) {
    const uint8_t lg = g.lflags ? g.lflags[mg] : 0;
    E[mg] = v[0];
    E[npf + mg] = v[1];
    E[2 * npf + mg] = (lg & LF_HX) ? 0.0f : fx;
    E[3 * npf + mg] = (lg & LF_HY) ? 0.0f : fy;
    E[4 * npf + mg] = (lg & LF_HZ) ? 0.0f : fz;
  };
  if (!g.px) {
    if (i == 1) ghost(m - 1, 0.0f, ty, tz);
    if (i == g.Nx - 1) ghost(m + 1, 0.0f, ty, tz);
  } else {
    if (i == g.Nx - 1) ghost(m - (g.Nx - 1), tx, 0.0f, 0.0f);
    if (i == 1) ghost(m + (g.Nx - 1), tx, 0.0f, 0.0f);
  }
  if (!g.py) {
    if (j == 1) ghost(m - g.mj, tx, 0.0f, tz);
    if (j == g.Ny - 1) ghost(m + g.mj, tx, 0.0f, tz);
  } else {
    if (j == g.Ny - 1) ghost(m - (long)(g.Ny - 1) * g.mj, 0.0f, ty, 0.0f);
    if (j == 1) ghost(m + (long)(g.Ny - 1) * g.mj, 0.0f, ty, 0.0f);
  }
  if (!g.pz) {
    if (k == 1) ghost(m - g.mk, tx, ty, 0.0f);
    if (k == g.Nz - 1) ghost(m + g.mk, tx, ty, 0.0f);
  } else {
    if (k == g.Nz - 1) ghost(m - (long)(g.Nz - 1) * g.mk, 0.0f, 0.0f, tz);
    if (k == 1) ghost(m + (long)(g.Nz - 1) * g.mk, 0.0f, 0.0f, tz);
  }
}

// Zero the dead links (bits b) at entry offset o of a staged direction box of
// kPlane entries per component; raw (may be null) receives the three raw link
// values first.
template <int PLANE>
__device__ __forceinline__ void tl_fix(float* P, int o, uint32_t b, float* raw) {
  if (raw) {
    raw[0] = P[2 * PLANE + o];
    raw[1] = P[3 * PLANE + o];
    raw[2] = P[4 * PLANE + o];
  }
  if (b & 1u) P[2 * PLANE + o] = 0.0f;
  if (b & 2u) P[3 * PLANE + o] = 0.0f;
  if (b & 4u) P[4 * PLANE + o] = 0.0f;
}

// Product (POLY false) or Horner step (POLY true) over a (32 NX) x 8 tile and
// the planes of chunk blockIdx.z.  Grid: (ceil(nx / (32 NX)), ceil(ny / 8),
// chunks), chunks <= nz; kThreads threads; TlShape<NX>::kSmem bytes of
// dynamic shared memory.
//
// Staged plane q (z = k0 - 1 + q) goes to slot q % kSlots.  Iteration p
// (plane k = k0 - 1 + p) waits for staged plane p + 1, zeroes its dead links,
// passes the block barrier, lets thread 0 issue staged plane p + kAhead into
// the slot of plane p - 2 (every thread is past iteration p - 1, the last
// reader of that slot), and computes plane k from the slots of p - 1, p, p + 1.
template <bool POLY, int NX>
__global__ void __launch_bounds__(kThreads, TlShape<NX>::kMinBlocks)
    kg_tl(const __grid_constant__ TlMaps M, GArgs<float> A) {
  using S = TlShape<NX>;
  constexpr int SL = S::kSlots, SF = S::kSlotF, PL = S::kPlane, BX = S::kBoxX;
  float* const tsm = tl_smem;
  __shared__ __align__(8) uint64_t bar[SL];
  GDev* d = A.dev;
  if (!gdev_ok(d)) return;
  if (d->arn_stop && !A.standalone) return;       // the solve stopped at this step's check
  kt_begin(d, KT_ARN_APPLY);
  const Grid& g = A.g;
  const long npf = A.npf;
  const int ja = d->ja;
  // the stenciled vector (its tensor map and, for the basis, its index), the
  // output and the coefficients of the output: z = cv V + cw W + cr (J W)
  int pm = TM_UB;
  float* out;
  const float* Vg = nullptr;     // Horner steps after the first: the vector of the e_k term
  float cv = 0.0f, cw = 1.0f, cr;
  {
    const double dth = d->dta / 2.0;
    if (POLY) {
      const int kst = A.pstep, deg = A.poly_deg;
      const bool first = kst == deg - 1;           // W_in is V itself
      if (first) {
        pm = TM_UB;
      } else {
        pm = ((kst + 1) & 1) ? TM_PW1 : TM_PW0;
        Vg = A.UB + (long)ja * A.vs;
      }
      out = kst == 0 ? A.PB + (long)ja * A.vs : A.PW[kst & 1];   // the last step: PB_ja = p(A) U_ja
      const double beta = first ? d->poly_e[deg] : 1.0, ide = 1.0 / d->poly_delta;
      const double e = d->poly_e[kst];
      // z = e V + beta ((W - dth J W) - theta W) / delta
      cw = (float)(beta * (1.0 - d->poly_theta) * ide + (first ? e : 0.0));
      cv = first ? 0.0f : (float)e;
      cr = (float)(-beta * dth * ide);
    } else {
      if (A.poly_deg > 0) pm = TM_PB;
      out = A.Zb[ja & 1];
      cr = (float)(-dth);                           // z = W - dth J W
    }
  }
  const unsigned long long wait_ns = d->wait_ns;
  // z-planes of this chunk (interior k0..k1) and the staged planes k0 - 1 .. k1 + 1
  const int nch = gridDim.z;
  const int k0 = 1 + (int)(((long)blockIdx.z * g.nz) / nch);
  const int k1 = (int)(((long)(blockIdx.z + 1) * g.nz) / nch);
  const int nq = k1 - k0 + 3;
  const int bx = blockIdx.x * S::kTx, by = blockIdx.y * kTlTy;   // box origin: (i0 - 1, j0 - 1)
  const CUtensorMap* mx = &M.m[TM_X];
  const CUtensorMap* mp = &M.m[pm];
  const bool p5 = pm == TM_UB || pm == TM_PB;
  int issued = 0;                                  // thread 0: staged planes issued so far
  auto issue = [&](int q) {                        // staged plane q into slot q % SL
    const int s = q % SL;
    float* dx = tsm + (size_t)s * 2 * SF;
    const int z = k0 - 1 + q;
    fence_proxy_async_smem();                      // the block's earlier writes to this slot come first
    mbar_expect_tx(&bar[s], 2 * S::kBytes);
    tma_load4(dx, mx, bx, by, z, 0, &bar[s]);
    if (p5) tma_load5(dx + SF, mp, bx, by, z, 0, ja, &bar[s]);
    else tma_load4(dx + SF, mp, bx, by, z, 0, &bar[s]);
    ++issued;
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < SL; ++s) mbar_init(&bar[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int q = 0; q <= S::kAhead && q < nq; ++q) issue(q);
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int j = 1 + by + ty;
  int iu[NX], ou[NX];
  bool act[NX], own_in[NX];
  long om[NX];
#pragma unroll
  for (int u = 0; u < NX; ++u) {
    iu[u] = 1 + bx + tx + 32 * u;
    act[u] = iu[u] <= g.nx && j <= g.ny;
    own_in[u] = iu[u] <= g.Nx && j <= g.Ny;      // on the full grid: its dead links are zeroed
    ou[u] = (ty + 1) * BX + (tx + 1 + 32 * u);
    om[u] = (long)iu[u] + (long)g.mj * j;        // full-grid index in plane 0
  }
  // one position of the ring around the tile (threads 0 .. kRing - 1)
  int ho = -1;
  long hm = 0;
  {
    const int t = threadIdx.x, w = S::kTx + 2;
    int hx = -1, hy = -1;
    if (t < w) hx = t, hy = 0;
    else if (t < 2 * w) hx = t - w, hy = kTlBoxY - 1;
    else if (t < 2 * w + kTlTy) hx = 0, hy = 1 + (t - 2 * w);
    else if (t < S::kRing) hx = S::kTx + 1, hy = 1 + (t - 2 * w - kTlTy);
    if (hx >= 0 && bx + hx <= g.Nx && by + hy <= g.Ny) {
      ho = hy * BX + hx;
      hm = (long)(bx + hx) + (long)g.mj * (by + hy);
    }
  }
  auto dead_bits = [&](int q) -> uint32_t {        // own bits << 4 u | ring bits << 16 of staged plane q
    const long zb = (long)g.mk * (k0 - 1 + q);
    uint32_t b = 0u;
#pragma unroll
    for (int u = 0; u < NX; ++u)
      if (own_in[u]) b |= (uint32_t)__ldg(A.ldead + zb + om[u]) << (4 * u);
    if (ho >= 0) b |= (uint32_t)__ldg(A.ldead + zb + hm) << 16;
    return b;
  };
  auto fix = [&](int q, uint32_t b, float (*raw)[3]) {
    float* P = tsm + (size_t)(q % SL) * 2 * SF + SF;
#pragma unroll
    for (int u = 0; u < NX; ++u)
      if (own_in[u]) tl_fix<PL>(P, ou[u], b >> (4 * u), raw ? raw[u] : nullptr);
    if (ho >= 0) tl_fix<PL>(P, ho, b >> 16, nullptr);
  };
  auto aborted = [&](bool ok) -> bool {            // block-wide: a wait ran out
    if (!__syncthreads_or(!ok)) return false;
    // wait (bounded) for every copy still in flight into this block's shared
    // memory, record the status, stop
    if (threadIdx.x == 0) {
      for (int q = issued > SL ? issued - SL : 0; q < issued; ++q)
        mbar_wait(&bar[q % SL], (unsigned)((q / SL) & 1), kTlDrainNs);
      atomicCAS(&d->status, GS_OK, GS_TIMEOUT);
    }
    return true;
  };
  // staged planes 0 and 1 (k0 - 1, k0) before the loop
  float raw[NX][3], raw_next[NX][3];
#pragma unroll
  for (int u = 0; u < NX; ++u) raw[u][0] = raw[u][1] = raw[u][2] = 0.0f;
  bool ok = mbar_wait(&bar[0], 0u, wait_ns);
  if (ok) fix(0, dead_bits(0), nullptr);
  ok = ok && mbar_wait(&bar[1], 0u, wait_ns);
  if (ok) fix(1, dead_bits(1), raw);
  uint32_t db_next = dead_bits(2);
  // per-node data of the plane (flags, the Horner step's V) are loaded one
  // plane ahead, so that no warp waits on them after the plane's barrier.
  // Threads past the grid's last row or column compute on the first node's
  // data and store nothing.
  const int dn = g.nx * g.ny;
  const long dmk = g.mk;
  int n[NX];
  long m[NX];
  bool face_ij[NX];
  uint8_t nf[NX];
  float v[NX][5];
#pragma unroll
  for (int u = 0; u < NX; ++u) {
    n[u] = act[u] ? dix(g, iu[u], j, k0) : 0;
    m[u] = act[u] ? full_index(g, iu[u], j, k0) : full_index(g, 1, 1, k0);
    face_ij[u] = iu[u] == 1 || iu[u] == g.Nx - 1 || j == 1 || j == g.Ny - 1;
    nf[u] = g.nflags[n[u]];
#pragma unroll
    for (int c = 0; c < kTlComp; ++c) v[u][c] = (POLY && Vg) ? __ldg(Vg + c * npf + m[u]) : 0.0f;
  }
  const float cx = (float)A.cxu, cy = (float)A.cyu, cz = (float)A.czu;
  const float ihx = (float)g.ihx2, ihy = (float)g.ihy2, ihz = (float)g.ihz2;
  const bool material = g.has_material != 0;
  for (int k = k0; k <= k1; ++k) {
    const int p = k - k0 + 1;                      // staged index of plane k
    ok = ok && mbar_wait(&bar[(p + 1) % SL], (unsigned)(((p + 1) / SL) & 1), wait_ns);
    if (ok) fix(p + 1, db_next, raw_next);
    if (aborted(ok)) return;
    if (threadIdx.x == 0 && p + S::kAhead < nq) issue(p + S::kAhead);
    if (p + 2 < nq) db_next = dead_bits(p + 2);
    const bool more = k < k1;
    uint8_t nf_next[NX];
    float v_next[NX][5];
#pragma unroll
    for (int u = 0; u < NX; ++u) {
      nf_next[u] = more ? g.nflags[n[u] + dn] : (uint8_t)0;
#pragma unroll
      for (int c = 0; c < kTlComp; ++c)
        v_next[u][c] = (POLY && Vg && more) ? __ldg(Vg + c * npf + m[u] + dmk) : 0.0f;
    }
    const int s0 = (p % SL) * 2 * SF, sm = ((p - 1) % SL) * 2 * SF, sp = ((p + 1) % SL) * 2 * SF;
#pragma unroll
    for (int u = 0; u < NX; ++u) {
      NodeCoef<float> nc;
      if (g.kappa_per_node) {
        nc = node_coef<float>(g, n[u], nf[u]);
      } else {
        nc.cx = cx; nc.cy = cy; nc.cz = cz;
        nc.material = material;
        nc.sc = (material && (nf[u] & NF_SCFRAC)) ? (float)g.scint[n[u]]
                                                  : ((material && (nf[u] & NF_SC0)) ? 0.0f : 1.0f);
        nc.ihx = ihx; nc.ihy = ihy; nc.ihz = ihz;
      }
      const int b0 = s0 + ou[u], bm = sm + ou[u], bp = sp + ou[u];
      const TlNb<NX> X{bm, b0, bp};
      const TlNb<NX> P{bm + SF, b0 + SF, bp + SF};
      float r[5];
      jvp_body<float, true>(g, X, P, nc, nf[u], r);
      // the direction's raw values at the node: psi from the box, links saved before zeroing
      const float w[5] = {tl_smem[b0 + SF], tl_smem[b0 + SF + PL], raw[u][0], raw[u][1], raw[u][2]};
      float z[5];
#pragma unroll
      for (int c = 0; c < kTlComp; ++c) z[c] = fmaf(cr, r[c], fmaf(cw, w[c], cv * v[u][c]));
      if (act[u]) tl_store(g, out, npf, m[u], iu[u], j, k, face_ij[u] || k == 1 || k == g.Nz - 1, z);
    }
#pragma unroll
    for (int u = 0; u < NX; ++u) {
#pragma unroll
      for (int c = 0; c < 3; ++c) raw[u][c] = raw_next[u][c];
      nf[u] = nf_next[u];
#pragma unroll
      for (int c = 0; c < kTlComp; ++c) v[u][c] = v_next[u][c];
      if (act[u]) {
        n[u] += dn;
        m[u] += dmk;
      }
    }
  }
  kt_end(d, KT_ARN_APPLY);
}

}  // namespace tdgl

namespace tdgl {
inline size_t tl_smem_bytes(int NX) { return NX == 2 ? TlShape<2>::kSmem : TlShape<1>::kSmem; }
}  // namespace tdgl
