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
// The graph launches the kernel with a programmatic dependency on the kernel
// before it: until grid_dep_wait a block reads only its parameters, the
// static grid arrays and the linearisation copy (which no kernel of the
// Krylov solve writes), so it sets up its barriers and indices and stages the
// linearisation's first planes while the previous kernel's last blocks run;
// the direction's planes, the device control block and the coefficients
// come after the wait.
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
// Pair coefficients of the two-nodes-per-thread kernel with a uniform kappa
// (both entries the same value): kappa^2 / h^2 per axis, twice those, the
// centre coefficients of the link Laplacians, 1 / h^2 of the psi Laplacian.
enum TlK : int { K_CX, K_CY, K_CZ, K_C2X, K_C2Y, K_C2Z, K_D0X, K_D0Y, K_D0Z, K_IHX, K_IHY, K_IHZ, K_N };
struct alignas(64) TlMaps {
  CUtensorMap m[5];
  int nx;        // nodes per thread along x of the kernel the maps' boxes are shaped for (1 or 2)
  int pdl;       // graph and probe launches depend programmatically on the kernel before them
  float2 k2[K_N];
};
// The pair coefficients from kappa^2 / h^2 per axis (float arithmetic, as the
// kernel's own for a per-node kappa).
__host__ __device__ inline void tl_pair_coef(float2* k, float2 cx, float2 cy, float2 cz) {
  auto add = [](float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); };
  auto m2 = [](float2 a) { return make_float2(-2.0f * a.x, -2.0f * a.y); };
  k[K_CX] = cx; k[K_CY] = cy; k[K_CZ] = cz;
  k[K_C2X] = add(cx, cx); k[K_C2Y] = add(cy, cy); k[K_C2Z] = add(cz, cz);
  k[K_D0X] = m2(add(add(k[K_C2X], cy), cz));
  k[K_D0Y] = m2(add(add(cx, k[K_C2Y]), cz));
  k[K_D0Z] = m2(add(add(cx, cy), k[K_C2Z]));
}

// Work items of one kg_tl launch: the (tile, z-chunk) pairs, numbered
// chunk-major with the longer chunks (nz % chunks of them, one plane more)
// first.  Blocks claim them as they start: the first block to arrive on an SM
// takes the next item from the front of the list, a later one the next from
// the back, so that two blocks sharing an SM (and its issue slots) get a long
// and a short chunk whatever the hardware's placement.  Every block claims
// exactly once, so the two ends meet without a check.  The last block of the
// launch to finish clears the counters for a later launch that uses the same
// set.
constexpr int kTlMaxSms = 256;
struct TlSched {
  unsigned arr[kTlMaxSms];       // blocks arrived per SM
  unsigned front, back, done, pad;
};

// Work item of this block (its thread 0).  A claim outside the list (counters
// not cleared by an earlier launch) falls back to the block index, so that no
// block addresses planes past the grid.
__device__ __forceinline__ int tl_claim(TlSched* s, int total) {
  const int own = (int)(blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z));
  if (!s) return own;
  unsigned sm;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
  const unsigned r = atomicAdd(&s->arr[sm % kTlMaxSms], 1u);
  const int item = r == 0 ? (int)atomicAdd(&s->front, 1u) : total - 1 - (int)atomicAdd(&s->back, 1u);
  return (item >= 0 && item < total) ? item : own;
}
// A block has finished (its thread 0, once, on every exit path).
__device__ __forceinline__ void tl_release(TlSched* s, int total) {
  if (!s) return;
  if (atomicAdd(&s->done, 1u) != (unsigned)(total - 1)) return;
  for (int i = 0; i < kTlMaxSms; ++i) s->arr[i] = 0u;
  s->front = 0u;
  s->back = 0u;
  s->done = 0u;
}

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
// Raise the transaction count of the current phase without arriving (copies
// issued before the phase's one arrival).
__device__ __forceinline__ void mbar_add_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
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

// ---------------------------------------------------------------------------
// Two nodes per thread (NX = 2): the nodes sit 32 entries apart along x in the
// same staged boxes, so the second node's reads are the first node's plus a
// constant, and their arithmetic is identical: jvp_body's operations run on
// the pair at once (x: the first node, y: the second) with the packed FP32
// instructions of sm_100 (one instruction for both nodes).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2s(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2neg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 tl_ld2(int e) { return make_float2(tl_smem[e], tl_smem[e + 32]); }

// jvp_body<float, true> for the pair: out = J(x) p at both nodes.  kc: the
// pair coefficients (TlK); sc, rx: the superconducting fraction and the
// relaxation coefficient -(1 - sc) / tau_relax of each node (material only).
template <int NX>
__device__ __forceinline__ void jvp_body_x2(const TlNb<NX>& X, const TlNb<NX>& P, const float2* kc, bool material,
                                            float2 sc, float2 rx, uint8_t nf0, uint8_t nf1, float2 out[5]) {
  constexpr int PL = TlShape<NX>::kPlane;
  auto psi = [](const TlNb<NX>& B, int di, int dj, int dk, float2& re, float2& im) {
    const int e = B.at(di, dj, dk);
    re = tl_ld2(e);
    im = tl_ld2(e + PL);
  };
  auto phi = [](const TlNb<NX>& B, int a, int di, int dj, int dk) { return tl_ld2(B.at(di, dj, dk) + (2 + a) * PL); };
  float2 cr, ci, dcr, dci;
  psi(X, 0, 0, 0, cr, ci);
  psi(P, 0, 0, 0, dcr, dci);
  float2 dsup[3];
  float2 dre = f2s(0.0f), dim = f2s(0.0f);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int ex = a == 0, ey = a == 1, ez = a == 2;
    float2 pmr, pmi, ppr, ppi, qmr, qmi, qpr, qpi;
    psi(X, -ex, -ey, -ez, pmr, pmi);
    psi(X, ex, ey, ez, ppr, ppi);
    psi(P, -ex, -ey, -ez, qmr, qmi);
    psi(P, ex, ey, ez, qpr, qpi);
    const float2 am = phi(X, a, -ex, -ey, -ez), a0 = phi(X, a, 0, 0, 0);
    const float2 dam = phi(P, a, -ex, -ey, -ez), da0 = phi(P, a, 0, 0, 0);
    float2 sm, cm, s0, c0;
    sincos_t<float>(am.x, &sm.x, &cm.x);
    sincos_t<float>(am.y, &sm.y, &cm.y);
    sincos_t<float>(a0.x, &s0.x, &c0.x);
    sincos_t<float>(a0.y, &s0.y, &c0.y);
    // d[e^{-i am} pm] = e^{-i am} (dpm - i dam pm)
    const float2 vr = f2fma(dam, pmi, qmr), vi = f2fma(f2neg(dam), pmr, qmi);
    const float2 lmr = f2fma(cm, vr, f2mul(sm, vi)), lmi = f2fma(cm, vi, f2mul(f2neg(sm), vr));
    // d[e^{i a0} pp] = e^{i a0} (dpp + i da0 pp)
    const float2 wr = f2fma(f2neg(da0), ppi, qpr), wi = f2fma(da0, ppr, qpi);
    const float2 lpr = f2fma(c0, wr, f2mul(f2neg(s0), wi)), lpi = f2fma(c0, wi, f2mul(s0, wr));
    const float2 ih = kc[K_IHX + a];
    dre = f2fma(f2add(f2fma(f2s(-2.0f), dcr, lmr), lpr), ih, dre);
    dim = f2fma(f2add(f2fma(f2s(-2.0f), dci, lmi), lpi), ih, dim);
    // d Im[e^{-i a0} conj(psi) psi1]; e^{-i a0} conj(psi) = (ur, -nu), likewise (u1r, -nu1) for dpsi
    const float2 ur = f2fma(c0, cr, f2mul(f2neg(s0), ci)), nu = f2fma(s0, cr, f2mul(c0, ci));
    const float2 u1r = f2fma(c0, dcr, f2mul(f2neg(s0), dci)), nu1 = f2fma(s0, dcr, f2mul(c0, dci));
    const float2 t1 = f2fma(u1r, ppi, f2mul(f2neg(nu1), ppr));     // u1r ppi + u1i ppr
    const float2 t2 = f2fma(ur, qpi, f2mul(f2neg(nu), qpr));       // ur qpi + ui qpr
    const float2 t3 = f2fma(ur, ppr, f2mul(nu, ppi));              // ur ppr - ui ppi
    dsup[a] = f2fma(f2neg(da0), t3, f2add(t1, t2));
  }
  const float2 m2 = f2fma(cr, cr, f2mul(ci, ci));
  const float2 pr = f2fma(cr, dcr, f2mul(ci, dci));
  const float2 om2 = f2sub(f2s(1.0f), m2);
  const float2 m2pr = f2mul(f2s(-2.0f), pr);
  const float2 dglr = f2fma(om2, dcr, f2mul(m2pr, cr));
  const float2 dgli = f2fma(om2, dci, f2mul(m2pr, ci));
  if (material) {
    dre = f2fma(sc, dglr, f2fma(rx, dcr, dre));
    dim = f2fma(sc, dgli, f2fma(rx, dci, dim));
  } else {
    dre = f2add(dre, dglr);
    dim = f2add(dim, dgli);
  }
  out[PR] = dre;
  out[PI] = dim;
  const float2 fx0 = phi(P, 0, 0, 0, 0), fxxm = phi(P, 0, -1, 0, 0), fxxp = phi(P, 0, 1, 0, 0);
  const float2 fxym = phi(P, 0, 0, -1, 0), fxyp = phi(P, 0, 0, 1, 0);
  const float2 fy0 = phi(P, 1, 0, 0, 0), fyxm = phi(P, 1, -1, 0, 0), fyxp = phi(P, 1, 1, 0, 0);
  const float2 fyym = phi(P, 1, 0, -1, 0), fyyp = phi(P, 1, 0, 1, 0);
  const float2 fxypxm = phi(P, 0, -1, 1, 0), fyxpym = phi(P, 1, 1, -1, 0);
  const float2 fxzm = phi(P, 0, 0, 0, -1), fxzp = phi(P, 0, 0, 0, 1);
  const float2 fyzm = phi(P, 1, 0, 0, -1), fyzp = phi(P, 1, 0, 0, 1);
  const float2 fz0 = phi(P, 2, 0, 0, 0), fzxm = phi(P, 2, -1, 0, 0), fzxp = phi(P, 2, 1, 0, 0);
  const float2 fzym = phi(P, 2, 0, -1, 0), fzyp = phi(P, 2, 0, 1, 0);
  const float2 fzzm = phi(P, 2, 0, 0, -1), fzzp = phi(P, 2, 0, 0, 1);
  const float2 fzxpzm = phi(P, 2, 1, 0, -1), fzypzm = phi(P, 2, 0, 1, -1);
  const float2 fxzpxm = phi(P, 0, -1, 0, 1), fyzpym = phi(P, 1, 0, -1, 1);
  // the curl-curl terms: centre minus lower neighbour of each component, shared
  const float2 gx = f2sub(fx0, fxxm), gy = f2sub(fy0, fyym), gz = f2sub(fz0, fzzm);
  float2 dfx = f2fma(kc[K_D0X], fx0, dsup[0]);
  dfx = f2fma(kc[K_C2X], f2add(fxxm, fxxp), dfx);
  dfx = f2fma(kc[K_CY], f2add(f2add(fxym, fxyp), f2add(gy, f2sub(fyxpym, fyxp))), dfx);
  dfx = f2fma(kc[K_CZ], f2add(f2add(fxzm, fxzp), f2add(gz, f2sub(fzxpzm, fzxp))), dfx);
  float2 dfy = f2fma(kc[K_D0Y], fy0, dsup[1]);
  dfy = f2fma(kc[K_C2Y], f2add(fyym, fyyp), dfy);
  dfy = f2fma(kc[K_CX], f2add(f2add(fyxm, fyxp), f2add(gx, f2sub(fxypxm, fxyp))), dfy);
  dfy = f2fma(kc[K_CZ], f2add(f2add(fyzm, fyzp), f2add(gz, f2sub(fzypzm, fzyp))), dfy);
  float2 dfz = f2fma(kc[K_D0Z], fz0, dsup[2]);
  dfz = f2fma(kc[K_C2Z], f2add(fzzm, fzzp), dfz);
  dfz = f2fma(kc[K_CX], f2add(f2add(fzxm, fzxp), f2add(gx, f2sub(fxzpxm, fxzp))), dfz);
  dfz = f2fma(kc[K_CY], f2add(f2add(fzym, fzyp), f2add(gy, f2sub(fyzpym, fyzp))), dfz);
  out[AX] = make_float2((nf0 & NF_HOLEX) ? 0.0f : dfx.x, (nf1 & NF_HOLEX) ? 0.0f : dfx.y);
  out[AY] = make_float2((nf0 & NF_HOLEY) ? 0.0f : dfy.x, (nf1 & NF_HOLEY) ? 0.0f : dfy.y);
  out[AZ] = make_float2((nf0 & NF_HOLEZ) ? 0.0f : dfz.x, (nf1 & NF_HOLEZ) ? 0.0f : dfz.y);
}

// Output node (i, j, k) of a tangent vector on the full grid: its raw values
// and the face values copied from it (write_eff with RAW_OWN and no field
// offsets, in float).  The ghosts' link flags are read only for nodes flagged
// NF_GHOSTLF (every other ghost has none), so the copies of the x faces, which
// fall in every warp, wait on no load.
__device__ __forceinline__ void tl_store(const Grid& g, float* E, long npf, long m, int i, int j, int k, bool face,
                                         uint8_t nf, const float* v) {
  float* e = E + m;
#pragma unroll
  for (int c = 0; c < kTlComp; ++c, e += npf) *e = v[c];
  if (!face) return;
  const float tx = (i == g.Nx - 1) ? 0.0f : v[2];
  const float ty = (j == g.Ny - 1) ? 0.0f : v[3];
  const float tz = (k == g.Nz - 1) ? 0.0f : v[4];
  auto ghost = [&](long mg, float fx, float fy, float fz) {
    const uint8_t lg = (nf & NF_GHOSTLF) ? g.lflags[mg] : 0;
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
// the planes of one z-chunk (the block's work item).  Grid: (ceil(nx / (32
// NX)), ceil(ny / 8), chunks), chunks <= nz; kThreads threads;
// TlShape<NX>::kSmem bytes of dynamic shared memory.
//
// Staged plane q (z = k0 - 1 + q) goes to slot q % kSlots.  Iteration p
// (plane k = k0 - 1 + p) waits for staged plane p + 1, zeroes its dead links,
// passes the block barrier, lets thread 0 issue staged plane p + kAhead into
// the slot of plane p - 2 (every thread is past iteration p - 1, the last
// reader of that slot), and computes plane k from the slots of p - 1, p, p + 1.
template <bool POLY, int NX, bool KPN>
__global__ void __launch_bounds__(kThreads, TlShape<NX>::kMinBlocks)
    kg_tl(const __grid_constant__ TlMaps M, GArgs<float> A) {
  using S = TlShape<NX>;
  constexpr int SL = S::kSlots, SF = S::kSlotF, PL = S::kPlane, BX = S::kBoxX;
  float* const tsm = tl_smem;
  __shared__ __align__(8) uint64_t bar[SL];
  __shared__ int s_item;
  GDev* d = A.dev;
  const Grid& g = A.g;
  const long npf = A.npf;
  const int tiles = gridDim.x * gridDim.y, total = tiles * gridDim.z;
  TlSched* const sch = A.tls ? A.tls + (A.tl_par & 1) : nullptr;
  if (threadIdx.x == 0) {
    for (int s = 0; s < SL; ++s) mbar_init(&bar[s], 1);
    mbar_fence_init();
    s_item = tl_claim(sch, total);
  }
  __syncthreads();
  // the block's tile and z-chunk: interior planes k0..k1, staged planes
  // k0 - 1 .. k1 + 1 (chunk `rank` of nch, the nz % nch longer ones first)
  const int item = s_item, tile = item % tiles, rank = item / tiles;
  const int nch = gridDim.z, qz = g.nz / nch, rz = g.nz % nch;
  const int k0 = 1 + rank * qz + (rank < rz ? rank : rz);
  const int k1 = k0 + qz - (rank < rz ? 0 : 1);
  const int nq = k1 - k0 + 3;
  const int bx = (tile % gridDim.x) * S::kTx, by = (tile / gridDim.x) * kTlTy;   // box origin: (i0 - 1, j0 - 1)
  const CUtensorMap* mx = &M.m[TM_X];
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
  // Before the grid dependency wait: the linearisation's boxes of the first
  // staged planes (their slots' single arrival comes with the direction's
  // copies), the dead-link bits and the node data of the first plane.
  const int npre = nq < S::kAhead + 1 ? nq : S::kAhead + 1;
  if (threadIdx.x == 0)
    for (int q = 0; q < npre; ++q) {
      fence_proxy_async_smem();
      mbar_add_tx(&bar[q], S::kBytes);
      tma_load4(tsm + (size_t)q * 2 * SF, mx, bx, by, k0 - 1 + q, 0, &bar[q]);
    }
  const uint32_t db0 = dead_bits(0), db1 = dead_bits(1);
  uint32_t db_next = dead_bits(2);
  const int dn = g.nx * g.ny;
  const long dmk = g.mk;
  int n[NX];
  long m[NX];
  bool face_ij[NX];
  uint8_t nf[NX];
#pragma unroll
  for (int u = 0; u < NX; ++u) {
    n[u] = act[u] ? dix(g, iu[u], j, k0) : 0;
    m[u] = act[u] ? full_index(g, iu[u], j, k0) : full_index(g, 1, 1, k0);
    face_ij[u] = iu[u] == 1 || iu[u] == g.Nx - 1 || j == 1 || j == g.Ny - 1;
    nf[u] = g.nflags[n[u]];
  }
  grid_dep_wait();
  grid_dep_launch();
  if (!gdev_ok(d) || (d->arn_stop && !A.standalone)) {   // stopped (or the solve stopped at this step's check)
    if (threadIdx.x == 0) {                    // complete the staged slots' phases and wait for their copies
      for (int q = 0; q < npre; ++q) mbar_arrive(&bar[q]);
      for (int q = 0; q < npre; ++q) mbar_wait(&bar[q], 0u, kTlDrainNs);
      tl_release(sch, total);
    }
    return;
  }
  kt_begin(d, KT_ARN_APPLY);
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
  const CUtensorMap* mp = &M.m[pm];
  const bool p5 = pm == TM_UB || pm == TM_PB;
  auto load_dir = [&](int q, float* dx, uint64_t* b) {   // the direction's box of staged plane q
    const int z = k0 - 1 + q;
    if (p5) tma_load5(dx + SF, mp, bx, by, z, 0, ja, b);
    else tma_load4(dx + SF, mp, bx, by, z, 0, b);
  };
  int issued = npre;                               // thread 0: staged planes issued so far
  auto issue = [&](int q) {                        // staged plane q into slot q % SL
    const int s = q % SL;
    float* dx = tsm + (size_t)s * 2 * SF;
    fence_proxy_async_smem();                      // the block's earlier writes to this slot come first
    mbar_expect_tx(&bar[s], 2 * S::kBytes);
    tma_load4(dx, mx, bx, by, k0 - 1 + q, 0, &bar[s]);
    load_dir(q, dx, &bar[s]);
    ++issued;
  };
  if (threadIdx.x == 0)
    for (int q = 0; q < npre; ++q) {               // the direction's boxes of the first planes: the slots' arrival
      mbar_expect_tx(&bar[q], S::kBytes);
      load_dir(q, tsm + (size_t)q * 2 * SF, &bar[q]);
    }
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
      tl_release(sch, total);
    }
    return true;
  };
  // staged planes 0 and 1 (k0 - 1, k0) before the loop
  float raw[NX][3], raw_next[NX][3];
#pragma unroll
  for (int u = 0; u < NX; ++u) raw[u][0] = raw[u][1] = raw[u][2] = 0.0f;
  bool ok = mbar_wait(&bar[0], 0u, wait_ns);
  if (ok) fix(0, db0, nullptr);
  ok = ok && mbar_wait(&bar[1], 0u, wait_ns);
  if (ok) fix(1, db1, raw);
  // per-node data of the plane (flags, the Horner step's V) are loaded one
  // plane ahead, so that no warp waits on them after the plane's barrier.
  // Threads past the grid's last row or column compute on the first node's
  // data and store nothing.
  float v[NX][5];
#pragma unroll
  for (int u = 0; u < NX; ++u) {
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
    if constexpr (NX == 2) {
      // both nodes at once (ou[1] = ou[0] + 32)
      // coefficients: the parameter table (uniform kappa, KPN false) or the
      // nodes' own (a kappa per node)
      float sc[2];
      float2 kl[K_N];
      const float2* kc = M.k2;
      if constexpr (KPN) {
        const NodeCoef<float> a = node_coef<float>(g, n[0], nf[0]), b = node_coef<float>(g, n[1], nf[1]);
        tl_pair_coef(kl, make_float2(a.cx, b.cx), make_float2(a.cy, b.cy), make_float2(a.cz, b.cz));
        kl[K_IHX] = M.k2[K_IHX]; kl[K_IHY] = M.k2[K_IHY]; kl[K_IHZ] = M.k2[K_IHZ];
        kc = kl;
        sc[0] = a.sc;
        sc[1] = b.sc;
      } else {
#pragma unroll
        for (int u = 0; u < 2; ++u)
          sc[u] = (material && (nf[u] & NF_SCFRAC)) ? (float)g.scint[n[u]]
                                                    : ((material && (nf[u] & NF_SC0)) ? 0.0f : 1.0f);
      }
      const float2 scp = make_float2(sc[0], sc[1]);
      const float2 rxp = make_float2(-10.0f * (1.0f - sc[0]), -10.0f * (1.0f - sc[1]));   // tau_relax = 0.1
      const int b0 = s0 + ou[0], bm = sm + ou[0], bp = sp + ou[0];
      const TlNb<NX> X{bm, b0, bp};
      const TlNb<NX> P{bm + SF, b0 + SF, bp + SF};
      float2 r[5];
      jvp_body_x2<NX>(X, P, kc, material, scp, rxp, nf[0], nf[1], r);
      // the direction's raw values at the nodes: psi from the box, links saved before zeroing
      const float2 w[5] = {tl_ld2(b0 + SF), tl_ld2(b0 + SF + PL), make_float2(raw[0][0], raw[1][0]),
                           make_float2(raw[0][1], raw[1][1]), make_float2(raw[0][2], raw[1][2])};
      float2 z[5];
#pragma unroll
      for (int c = 0; c < kTlComp; ++c) {
        const float2 zw = f2mul(f2s(cw), w[c]);
        z[c] = f2fma(f2s(cr), r[c], POLY ? f2fma(f2s(cv), make_float2(v[0][c], v[1][c]), zw) : zw);
      }
      const bool kface = k == 1 || k == g.Nz - 1;
      float z0[5], z1[5];
#pragma unroll
      for (int c = 0; c < kTlComp; ++c) z0[c] = z[c].x, z1[c] = z[c].y;
      if (act[0]) tl_store(g, out, npf, m[0], iu[0], j, k, face_ij[0] || kface, nf[0], z0);
      if (act[1]) tl_store(g, out, npf, m[1], iu[1], j, k, face_ij[1] || kface, nf[1], z1);
    } else {
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
      if (act[u]) tl_store(g, out, npf, m[u], iu[u], j, k, face_ij[u] || k == 1 || k == g.Nz - 1, nf[u], z);
    }
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
  if (threadIdx.x == 0) tl_release(sch, total);
  kt_end(d, KT_ARN_APPLY);
}

}  // namespace tdgl

namespace tdgl {
inline size_t tl_smem_bytes(int NX) { return NX == 2 ? TlShape<2>::kSmem : TlShape<1>::kSmem; }

// The kernel for NX nodes per thread, a Horner step or the product, and a
// kappa per node (two-nodes-per-thread kernel only).
inline const void* tl_kernel(int nx, bool poly, bool kpn) {
  if (nx == 2) {
    if (poly) return kpn ? (const void*)kg_tl<true, 2, true> : (const void*)kg_tl<true, 2, false>;
    return kpn ? (const void*)kg_tl<false, 2, true> : (const void*)kg_tl<false, 2, false>;
  }
  return poly ? (const void*)kg_tl<true, 1, false> : (const void*)kg_tl<false, 1, false>;
}
}  // namespace tdgl
