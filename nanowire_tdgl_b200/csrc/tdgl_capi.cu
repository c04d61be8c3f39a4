// C ABI of the B200 TDGL stepper (include/tdgl_b200.h): context set-up,
// workspace, launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "tdgl_b200.h"
#include "tdgl_geometry.h"
#include "tdgl_kernels.cuh"
#include "tdgl_stepper.cuh"
#include "tdgl_graph.cuh"
#include "tdgl_adjoint.cuh"
#include "tdgl_analysis.cuh"
#include "tdgl_adjoint_graph.cuh"
#include "tdgl_tl.cuh"

#include <cudaTypedefs.h>

using namespace tdgl;

namespace tdgl {
cudaError_t stepper_occupancy_f32(size_t smem, int* occ);
cudaError_t stepper_occupancy_f64(size_t smem, int* occ);
cudaError_t stepper_launch_f32(StepArgs<float> A, int blocks, size_t smem, cudaStream_t s);
cudaError_t stepper_launch_f64(StepArgs<double> A, int blocks, size_t smem, cudaStream_t s);
cudaError_t graph_build_f32(const GArgs<float>& A, const TlMaps* tm, int chunks, cudaGraph_t* graph,
                            cudaGraphExec_t* exec);
cudaError_t graph_build_f64(const GArgs<double>& A, cudaGraph_t* graph, cudaGraphExec_t* exec);
cudaError_t arnoldi_probe_f32(const GArgs<float>& A, const TlMaps* tm, int chunks, int launches, int kernels,
                              cudaStream_t s);
cudaError_t product_f32(const GArgs<float>& A, const TlMaps* tm, int chunks, cudaStream_t s);
cudaError_t product_f64(const GArgs<double>& A, cudaStream_t s);
cudaError_t arnoldi_probe_f64(const GArgs<double>& A, int launches, int kernels, cudaStream_t s);
}  // namespace tdgl

static constexpr long kProfLen = 64 + 2 * 1024;
// upper bound of the step graph's blocks per SM (its partial-sum buffers are sized for it)
static constexpr int kMaxBlocksPerSm = 8;
// default degree of the polynomial preconditioner (analytic-product GMRES):
// on the 128x128x32 film with the forcing term degrees 3-8 gave 604.7, 640.7,
// 671.3, 685.4, 694.4, 706.5 steps/s, and on the final stencil build degrees
// 8, 10, 12 gave 737.0, 809.1, 733.1; on the 256x256x64 trilayer degrees 8,
// 10, 12 gave 48.74, 51.41, 52.13 steps/s
static constexpr int kPolyDefault = 10;
// default limit of one bounded device wait (grid barrier, staged-copy mbarrier)
static constexpr unsigned long long kWaitDefaultNs = 5000000000ull;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define TDGL_CUDA(call)                                                                 \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(TDGL_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)


}  // namespace

struct tdgl_ctx {
  Grid g{};
  int precision = TDGL_FP64;
  int kmax = 0;
  int device = 0;
  int num_sms = 0;
  long L = 0;           // doubles (or floats) of one device-layout vector
  size_t bytes = 0;
  // geometry
  uint8_t* lflags = nullptr;
  uint8_t* nflags = nullptr;
  double* k2 = nullptr;
  double* sc = nullptr;
  int* slow_off = nullptr;
  int* slow_idx = nullptr;
  // scratch for the reference-layout operators
  double* s_x = nullptr;
  double* s_f = nullptr;
  double* s_red = nullptr;
  // solver workspace (allocated on first use)
  bool ws_ready = false;
  double* X1 = nullptr;
  double* G = nullptr;
  double* F = nullptr;
  void* R[3] = {nullptr, nullptr, nullptr};
  void* XL = nullptr;
  void* P = nullptr;
  void* AP = nullptr;
  double* hbuf = nullptr;
  double* partials = nullptr;
  int krylov = KRY_GMRES;
  double* results = nullptr;
  unsigned* bar = nullptr;
  int* err = nullptr;
  Ctl* ctl_dev = nullptr;
  Ctl* ctl_host = nullptr;
  unsigned long long* prof = nullptr;   // phase timers when TDGL_PROFILE is set
  int blocks = 0;
  size_t smem = 0;
  // graph executor (GMRES trapezoidal steps)
  bool gws_ready = false;
  long npf = 0;             // full-grid component stride of the effective copies
  int gblocks = 0;          // blocks of its grid kernels
  double* Xn = nullptr;
  double* En = nullptr;
  double* Ei = nullptr;
  void* XLe = nullptr;
  void* VE = nullptr;
  double* part_dots = nullptr;
  double* part_orth = nullptr;
  double* part_nrhs = nullptr;
  double* part_upd = nullptr;
  double* kry = nullptr;
  GDev* gdev = nullptr;
  GDev* gdev_host = nullptr;
  cudaGraph_t graph[2] = {nullptr, nullptr};        // [0]: finite-difference Krylov body, [1]: analytic
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  bool gprof = false;                               // per-kernel timers of the graph (TDGL_PROFILE)
  unsigned long long gk_total[kKTypes] = {};
  long long gk_count[kKTypes] = {};
  // Arnoldi workspace of the analytic-product graph (allocated with it)
  void* UB = nullptr;
  void* Zb[2] = {nullptr, nullptr};
  double* part_arn = nullptr;
  unsigned* ticket = nullptr;
  int ntiles = 0, ngroups = 0;   // tiles of the product-and-projections kernel, groups of 32 tiles
  int ngroups_cap = 0;           // group-partial slots: groups of tiles or of projection blocks
  double* gpart = nullptr;
  unsigned* gticket = nullptr;
  int apply_dots = 0;            // product and projections in one kernel (FP64 default; TDGL_ARN_APPLY_DOTS)
  int apply_dots_req = -1;       // set by tdgl_ctx_set_blocks (-1: the default)
  int nblk_arn = 0, nblk_orth = 0, arn_gx = 0, arn_gy = 0;
  int blk_stream = 0, blk_krylov = 0;   // blocks of the graph's grid kernels (0: defaults)
  // polynomial preconditioner of the analytic-product solves: requested degree
  // (-1: the default), the degree in use, the largest kappa^2 of the grid, and
  // the Horner buffers / Newton correction (full-grid vectors)
  int poly_req = -1, poly_deg = 0;
  double k2max = 0.0;
  void* PW[2] = {nullptr, nullptr};
  void* PB = nullptr;     // preconditioned basis p(A) U_j ((kmax + 1) vectors)
  // queued step-graph launches (tdgl_trap_launch / tdgl_trap_launch_next):
  // per launch slot a pinned input and output control block and a completion
  // event; up to two launches queued, collected in order
  GDev* gin[2] = {nullptr, nullptr};
  GDev* gout[2] = {nullptr, nullptr};
  cudaEvent_t gev[2] = {nullptr, nullptr};
  double* gclk = nullptr;         // device: the clock (t, dt_cur) carried into a continuation
  int npend = 0, pend_head = 0, next_slot = 0;
  bool pend_noop[2] = {false, false};
  bool has_clock = false;         // a launch has left its clock in the device control block
  uint8_t* imask = nullptr;
  uint32_t* deadmask = nullptr;   // per interior node: dead links read by the Arnoldi product
  uint8_t* ldead = nullptr;       // per full-grid node: its dead links (TMA-staged stencil)
  TlSched* tls = nullptr;         // the TMA-staged stencil's two sets of work-item claim counters
  int forcing = 1;                // forcing term of the analytic-product GMRES solves (TDGL_FORCING=0: off)
  // TMA-staged tangent-linear stencil (FP32 vectors, 3-D grids): tensor maps of
  // the staged vectors and the z-chunks per tile column
  TlMaps tlm{};
  bool tl_on = false;
  int tl_chunks = 0;
  // limits of the device's bounded waits and of the graph's loop iterations
  // (tdgl_ctx_set_limits; 0: the defaults)
  unsigned long long wait_ns = kWaitDefaultNs;
  long long watchdog_req = 0;
  // adjoint scratch (allocated on first use)
  double* vjp_part = nullptr;   // 3 x vjp blocks
  double* vjp_k2 = nullptr;     // n
  double* obs = nullptr;        // 7 x n observables scratch of tdgl_convergence_means
  // device-resident adjoint solve (tdgl_adjoint_solve): x, b, mu, T (L each) and its graph
  double* adj = nullptr;
  cudaGraph_t adj_graph = nullptr;
  cudaGraphExec_t adj_exec = nullptr;
  std::vector<void*> owned;
  bool unsettled = false;       // initialisation memsets / copies not yet known complete
};

// Zero-filled device buffer owned by the context.  The fill (and the pageable
// host copies of initial contents) run on the legacy default stream, which
// work on a non-blocking stream does not wait for: settle() ends every
// function that allocates, before work on the caller's stream may use it.
static int ctx_alloc(tdgl_ctx* c, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) return fail(TDGL_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  c->owned.push_back(*p);
  c->bytes += bytes;
  c->unsettled = true;
  e = cudaMemset(*p, 0, bytes);
  if (e != cudaSuccess) return fail(TDGL_ECUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
  return TDGL_OK;
}

static int settle(tdgl_ctx* c) {
  if (!c->unsettled) return TDGL_OK;
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return fail(TDGL_ECUDA, std::string("initialising buffers: ") + cudaGetErrorString(e));
  c->unsettled = false;
  return TDGL_OK;
}

extern "C" const char* tdgl_status_string(int s) {
  switch (s) {
    case TDGL_OK: return "ok";
    case TDGL_ENOCONV: return "did not converge";
    case TDGL_EDTMIN: return "dt reduced below dt_min";
    case TDGL_EKMAX: return "Krylov workspace exhausted";
    case TDGL_ENONFINITE: return "non-finite value";
    case TDGL_ETIMEOUT: return "device wait timed out";
    case TDGL_EINVAL: return "invalid argument";
    case TDGL_ECUDA: return "CUDA error";
    case TDGL_ENOMEM: return "out of device memory";
    default: return "unknown status";
  }
}

extern "C" const char* tdgl_last_error(void) { return g_last_error.c_str(); }

namespace tdgl {
// Lets the other translation units of the library report through tdgl_last_error().
int report_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace tdgl

extern "C" int tdgl_ctx_create(const tdgl_grid_desc* gd, const tdgl_material_desc* md, int32_t precision,
                               int32_t kmax, tdgl_ctx** out) {
  if (!gd || !out) return fail(TDGL_EINVAL, "null argument");
  *out = nullptr;
  if (precision != TDGL_FP64 && precision != TDGL_MIXED) return fail(TDGL_EINVAL, "unknown precision");
  if (kmax < 1) return fail(TDGL_EINVAL, "kmax must be >= 1");
  HostGeometry hg;
  std::string msg;
  int rc = build_geometry(gd, md, hg, msg);
  if (rc) return fail(rc, msg);
  tdgl_ctx* c = new tdgl_ctx();
  c->precision = precision;
  c->kmax = kmax;
  cudaGetDevice(&c->device);
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
  c->g = hg.g;
  Grid& g = c->g;
  c->L = (long)g.ncomp * g.npad;
  const long n = g.n;
  if ((rc = ctx_alloc(c, (void**)&c->nflags, n))) { tdgl_ctx_destroy(c); return rc; }
  TDGL_CUDA(cudaMemcpy(c->nflags, hg.nflags.data(), n, cudaMemcpyHostToDevice));
  g.nflags = c->nflags;
  if (!hg.lflags.empty()) {
    if ((rc = ctx_alloc(c, (void**)&c->lflags, hg.lflags.size()))) { tdgl_ctx_destroy(c); return rc; }
    TDGL_CUDA(cudaMemcpy(c->lflags, hg.lflags.data(), hg.lflags.size(), cudaMemcpyHostToDevice));
  }
  g.lflags = c->lflags;
  if (!hg.k2.empty()) {
    if ((rc = ctx_alloc(c, (void**)&c->k2, n * sizeof(double)))) { tdgl_ctx_destroy(c); return rc; }
    TDGL_CUDA(cudaMemcpy(c->k2, hg.k2.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  }
  g.k2int = c->k2;
  c->k2max = g.kappa2;
  if (!hg.k2.empty()) c->k2max = *std::max_element(hg.k2.begin(), hg.k2.end());
  if (!hg.sc.empty()) {
    if ((rc = ctx_alloc(c, (void**)&c->sc, n * sizeof(double)))) { tdgl_ctx_destroy(c); return rc; }
    TDGL_CUDA(cudaMemcpy(c->sc, hg.sc.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  }
  g.scint = c->sc;
  if ((rc = ctx_alloc(c, (void**)&c->slow_off, hg.slow_off.size() * sizeof(int)))) { tdgl_ctx_destroy(c); return rc; }
  TDGL_CUDA(cudaMemcpy(c->slow_off, hg.slow_off.data(), hg.slow_off.size() * sizeof(int), cudaMemcpyHostToDevice));
  g.slow_off = c->slow_off;
  if (!hg.slow_idx.empty()) {
    if ((rc = ctx_alloc(c, (void**)&c->slow_idx, hg.slow_idx.size() * sizeof(int)))) { tdgl_ctx_destroy(c); return rc; }
    TDGL_CUDA(cudaMemcpy(c->slow_idx, hg.slow_idx.data(), hg.slow_idx.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  g.slow_idx = c->slow_idx;
  const size_t vbytes = (size_t)c->L * sizeof(double);
  if ((rc = ctx_alloc(c, (void**)&c->s_x, vbytes))) { tdgl_ctx_destroy(c); return rc; }
  if ((rc = ctx_alloc(c, (void**)&c->s_f, vbytes))) { tdgl_ctx_destroy(c); return rc; }
  if ((rc = ctx_alloc(c, (void**)&c->s_red, 64 * sizeof(double)))) { tdgl_ctx_destroy(c); return rc; }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { tdgl_ctx_destroy(c); return fail(TDGL_ECUDA, cudaGetErrorString(e)); }
  if ((rc = settle(c))) { tdgl_ctx_destroy(c); return rc; }
  *out = c;
  return TDGL_OK;
}

extern "C" int tdgl_ctx_destroy(tdgl_ctx* c) {
  if (!c) return TDGL_OK;
  // work of this context may still be in flight on the caller's streams (an
  // uncollected tdgl_trap_launch): let it finish before its buffers go
  cudaDeviceSynchronize();
  for (int v = 0; v < 2; ++v) {
    if (c->gexec[v]) cudaGraphExecDestroy(c->gexec[v]);
    if (c->graph[v]) cudaGraphDestroy(c->graph[v]);
  }
  if (c->adj_exec) cudaGraphExecDestroy(c->adj_exec);
  if (c->adj_graph) cudaGraphDestroy(c->adj_graph);
  for (void* p : c->owned) cudaFree(p);
  if (c->ctl_host) cudaFreeHost(c->ctl_host);
  if (c->gdev_host) cudaFreeHost(c->gdev_host);
  if (c->gin[1]) cudaFreeHost(c->gin[1]);
  for (int k = 0; k < 2; ++k) {
    if (c->gout[k]) cudaFreeHost(c->gout[k]);
    if (c->gev[k]) cudaEventDestroy(c->gev[k]);
  }
  delete c;
  return TDGL_OK;
}

extern "C" int64_t tdgl_n_interior(const tdgl_ctx* c) { return c ? c->g.n : -1; }
extern "C" int64_t tdgl_npad(const tdgl_ctx* c) { return c ? c->g.npad : -1; }
extern "C" int64_t tdgl_state_len(const tdgl_ctx* c) { return c ? c->L : -1; }
extern "C" int64_t tdgl_workspace_bytes(const tdgl_ctx* c) { return c ? (int64_t)c->bytes : -1; }

static int grid_1d(const tdgl_ctx* c, long work) {
  long b = (work + kThreads - 1) / kThreads;
  long cap = (long)c->num_sms * 4;
  return (int)std::max(1L, std::min(b, cap));
}

extern "C" int tdgl_pack(tdgl_ctx* c, const double* x_ref, double* x_dev, tdgl_stream_t s) {
  if (!c || !x_ref || !x_dev) return fail(TDGL_EINVAL, "null argument");
  k_pack<<<grid_1d(c, c->g.n), kThreads, 0, s>>>(c->g, (const double2*)x_ref, x_dev);
  TDGL_CUDA(cudaGetLastError());
  return TDGL_OK;
}

extern "C" int tdgl_unpack(tdgl_ctx* c, const double* x_dev, double* x_ref, tdgl_stream_t s) {
  if (!c || !x_ref || !x_dev) return fail(TDGL_EINVAL, "null argument");
  k_unpack<<<grid_1d(c, c->g.n), kThreads, 0, s>>>(c->g, x_dev, (double2*)x_ref);
  TDGL_CUDA(cudaGetLastError());
  return TDGL_OK;
}

extern "C" int tdgl_rhs(tdgl_ctx* c, const double* x, double* f, double Bx, double By, double Bz, tdgl_stream_t s) {
  if (!c || !x || !f) return fail(TDGL_EINVAL, "null argument");
  k_rhs<<<grid_1d(c, c->g.n), kThreads, 0, s>>>(c->g, x, f, bterms(c->g, Bx, By, Bz));
  TDGL_CUDA(cudaGetLastError());
  return TDGL_OK;
}

namespace {
// Sum of the per-block field partials and the uniform-kappa gradient
// (d/dkappa = 2 kappa sum_m d/dkappa^2(m)), fixed order, one block.
__global__ void k_vjp_finish(const double* part, int nblk, const double* gk2, int n, double kappa, double* out) {
  __shared__ double s[4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = warp; q < 4; q += kWarps) {
    double a = 0.0;
    if (q < 3) {
      for (int b = lane; b < nblk; b += 32) a += part[(long)q * nblk + b];
    } else {
      for (int d = lane; d < n; d += 32) a += gk2[d];
    }
    a = warp_sum(a);
    if (lane == 0) s[q] = a;
  }
  __syncthreads();
  if (threadIdx.x < 3) out[threadIdx.x] = s[threadIdx.x];
  if (threadIdx.x == 3) out[3] = 2.0 * kappa * s[3];
}
}  // namespace

extern "C" int tdgl_vjp(tdgl_ctx* c, const double* x, const double* v, double Bx, double By, double Bz, double* gx,
                        double* gsc, double* gk2, double* gpar, tdgl_stream_t s) {
  if (!c || !x || !v || !gx) return fail(TDGL_EINVAL, "null argument");
  const Grid& g = c->g;
  const int nb = grid_1d(c, g.n);
  int rc;
  if (!c->vjp_part) {
    if ((rc = ctx_alloc(c, (void**)&c->vjp_part, sizeof(double) * 3 * (size_t)nb))) return rc;
    if ((rc = ctx_alloc(c, (void**)&c->vjp_k2, sizeof(double) * (size_t)g.n))) return rc;
    if ((rc = settle(c))) return rc;
  }
  double* k2 = gk2 ? gk2 : c->vjp_k2;
  TDGL_CUDA(cudaMemsetAsync(gx, 0, sizeof(double) * c->L, s));
  if (gsc && !g.has_material) TDGL_CUDA(cudaMemsetAsync(gsc, 0, sizeof(double) * g.n, s));
  const BTerms<double> b = bterms(g, Bx, By, Bz);
  if (g.is3d) k_vjp<true><<<nb, kThreads, 0, s>>>(g, x, v, b, gx, g.has_material ? gsc : nullptr, k2, c->vjp_part);
  else k_vjp<false><<<nb, kThreads, 0, s>>>(g, x, v, b, gx, g.has_material ? gsc : nullptr, k2, c->vjp_part);
  TDGL_CUDA(cudaGetLastError());
  if (gpar) {
    const double kappa = g.kappa_per_node ? 0.0 : std::sqrt(g.kappa2);
    k_vjp_finish<<<1, kThreads, 0, s>>>(c->vjp_part, nb, k2, g.n, kappa, gpar);
    TDGL_CUDA(cudaGetLastError());
  }
  return TDGL_OK;
}

extern "C" int tdgl_eval_f(tdgl_ctx* c, const double* x_ref, double* f_ref, double Bx, double By, double Bz,
                           tdgl_stream_t s) {
  int rc;
  if ((rc = tdgl_pack(c, x_ref, c->s_x, s))) return rc;
  if ((rc = tdgl_rhs(c, c->s_x, c->s_f, Bx, By, Bz, s))) return rc;
  return tdgl_unpack(c, c->s_f, f_ref, s);
}

// sum of squares of a device-layout FP64 vector (single block, deterministic)
__global__ void k_norm2(const double* __restrict__ v, long L, double* out) {
  double s = 0.0;
  for (long e = threadIdx.x; e < L; e += blockDim.x) s += v[e] * v[e];
  s = warp_sum(s);
  __shared__ double w[kWarps];
  if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < kWarps; ++i) t += w[i];
    *out = t;
  }
}

static int krylov_product(tdgl_ctx* c, const double* x, const double* p, double* ap, double dt, double Bx,
                          double By, double Bz, tdgl_stream_t s);

extern "C" int tdgl_jvp(tdgl_ctx* c, const double* x, const double* p, double* ap, double dt, int32_t mode,
                        double eps_mf, double Bx, double By, double Bz, tdgl_stream_t s) {
  if (!c || !x || !p || !ap) return fail(TDGL_EINVAL, "null argument");
  if (mode == TDGL_JVP_KRYLOV) return krylov_product(c, x, p, ap, dt, Bx, By, Bz, s);
  BTerms<double> b = bterms(c->g, Bx, By, Bz);
  if (mode == TDGL_JVP_ANALYTIC) {
    k_jvp_analytic<double><<<grid_1d(c, c->g.n), kThreads, 0, s>>>(c->g, x, p, ap, dt / 2.0, b);
    TDGL_CUDA(cudaGetLastError());
    return TDGL_OK;
  }
  if (mode != TDGL_JVP_FD) return fail(TDGL_EINVAL, "unknown jvp mode");
  k_rhs<<<grid_1d(c, c->g.n), kThreads, 0, s>>>(c->g, x, c->s_f, b);
  k_norm2<<<1, kThreads, 0, s>>>(x, c->L, c->s_red);
  k_norm2<<<1, kThreads, 0, s>>>(p, c->L, c->s_red + 1);
  double h[2];
  TDGL_CUDA(cudaMemcpyAsync(h, c->s_red, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  TDGL_CUDA(cudaStreamSynchronize(s));
  double pn = std::sqrt(h[1]);
  if (pn == 0.0) return fail(TDGL_EINVAL, "zero direction");
  double eps = eps_mf * (1.0 + std::sqrt(h[0])) / pn;
  k_jvp_fd<<<grid_1d(c, c->g.n), kThreads, 0, s>>>(c->g, x, c->s_f, p, ap, dt / 2.0, eps, b);
  TDGL_CUDA(cudaGetLastError());
  return TDGL_OK;
}

extern "C" int tdgl_observables(tdgl_ctx* c, const double* x, double Bx, double By, double Bz, double* psi2,
                                double* bx, double* by, double* bz, double* jx, double* jy, double* jz,
                                tdgl_stream_t s) {
  if (!c || !x || !psi2 || !bx || !by || !bz || !jx || !jy || !jz) return fail(TDGL_EINVAL, "null argument");
  const Grid& g = c->g;
  k_observables<<<grid_1d(c, g.n), kThreads, 0, s>>>(g, x, bterms(g, Bx, By, Bz), 1.0 / (g.hx * g.hy),
                                                      1.0 / (g.hy * g.hz), 1.0 / (g.hz * g.hx), psi2, bx, by, bz,
                                                      jx, jy, jz);
  TDGL_CUDA(cudaGetLastError());
  return TDGL_OK;
}

extern "C" int tdgl_plaquette_winding(tdgl_ctx* c, const double* x, double mask_threshold, double* w,
                                      tdgl_stream_t s) {
  if (!c) return fail(TDGL_EINVAL, "null argument");
  const Grid& g = c->g;
  const long total = (long)(g.is3d ? g.nz : 1) * (g.nx - 1) * (g.ny - 1);
  if (total <= 0) return TDGL_OK;        // no plaquettes (Nx or Ny = 2): nothing to write
  if (!x || !w) return fail(TDGL_EINVAL, "null argument");
  const int blocks = (int)std::min<long>((total + kThreads - 1) / kThreads, (long)c->num_sms * 8);
  k_plaquette<<<blocks, kThreads, 0, s>>>(g, x, mask_threshold, w);
  TDGL_CUDA(cudaGetLastError());
  return TDGL_OK;
}

extern "C" int tdgl_convergence_means(tdgl_ctx* c, const double* x, const double* sc_ref, double* out,
                                      tdgl_stream_t s) {
  if (!c || !x || !out) return fail(TDGL_EINVAL, "null argument");
  const Grid& g = c->g;
  const long n = g.n;
  int rc;
  if (!c->obs) {
    if ((rc = ctx_alloc(c, (void**)&c->obs, sizeof(double) * 7 * (size_t)n))) return rc;
    if ((rc = settle(c))) return rc;
  }
  double* o = c->obs;
  if ((rc = tdgl_observables(c, x, 0.0, 0.0, 0.0, o, o + n, o + 2 * n, o + 3 * n, o + 4 * n, o + 5 * n, o + 6 * n,
                             s)))
    return rc;
  k_conv_means<<<1, kThreads, 0, s>>>(n, o, o + 4 * n, o + 5 * n, g.is3d ? o + 6 * n : nullptr, sc_ref, out);
  TDGL_CUDA(cudaGetLastError());
  return TDGL_OK;
}

// ---------------------------------------------------------------------------
// Solver workspace and the persistent launch
// ---------------------------------------------------------------------------

static int setup_launch(tdgl_ctx* c) {
  c->smem = stepper_smem(c->kmax);
  int occ = 0;
  TDGL_CUDA(c->precision == TDGL_MIXED ? stepper_occupancy_f32(c->smem, &occ) : stepper_occupancy_f64(c->smem, &occ));
  if (occ < 1) return fail(TDGL_ECUDA, "stepper kernel does not fit on an SM");
  c->blocks = c->num_sms * std::min(occ, 1);
  return TDGL_OK;
}

static int ensure_workspace(tdgl_ctx* c) {
  if (c->ws_ready) return TDGL_OK;
  const size_t vb = (size_t)c->L * sizeof(double);
  const size_t tb = (size_t)c->L * (c->precision == TDGL_MIXED ? sizeof(float) : sizeof(double));
  int rc;
  if ((rc = ctx_alloc(c, (void**)&c->X1, vb))) return rc;
  if ((rc = ctx_alloc(c, (void**)&c->G, vb))) return rc;
  if ((rc = ctx_alloc(c, (void**)&c->F, vb))) return rc;
  for (int i = 0; i < 3; ++i)
    if ((rc = ctx_alloc(c, &c->R[i], tb))) return rc;
  if (c->precision == TDGL_MIXED)
    if ((rc = ctx_alloc(c, &c->XL, tb))) return rc;
  if ((rc = ctx_alloc(c, &c->P, tb * (c->kmax + 1)))) return rc;
  if ((rc = ctx_alloc(c, &c->AP, tb * c->kmax))) return rc;
  rc = setup_launch(c);
  if (rc) return rc;
  if ((rc = ctx_alloc(c, (void**)&c->hbuf, sizeof(double) * hbuf_stride(c->kmax) * (size_t)c->blocks))) return rc;
  int nslot = c->kmax + 4;
  if ((rc = ctx_alloc(c, (void**)&c->partials, sizeof(double) * nslot * (size_t)c->blocks))) return rc;
  if ((rc = ctx_alloc(c, (void**)&c->results, sizeof(double) * nslot))) return rc;
  if ((rc = ctx_alloc(c, (void**)&c->bar, 4 * sizeof(unsigned)))) return rc;
  if ((rc = ctx_alloc(c, (void**)&c->err, 4 * sizeof(int)))) return rc;
  if ((rc = ctx_alloc(c, (void**)&c->ctl_dev, sizeof(Ctl)))) return rc;
  const char* pe = std::getenv("TDGL_PROFILE");
  if (pe && pe[0] && pe[0] != '0')
    if ((rc = ctx_alloc(c, (void**)&c->prof, kProfLen * sizeof(unsigned long long)))) return rc;
  TDGL_CUDA(cudaMallocHost((void**)&c->ctl_host, sizeof(Ctl)));
  c->ws_ready = true;
  return settle(c);
}

template <typename T>
static StepArgs<T> make_args(tdgl_ctx* c, double* x0, double* x1, double* G, double* D) {
  StepArgs<T> A{};
  A.g = c->g;
  A.sy.partials = c->partials;
  A.sy.results = c->results;
  A.sy.bar = c->bar;
  A.sy.err = c->err;
  A.sy.nslot_max = c->kmax + 4;
  A.sy.timeout_ns = c->wait_ns;
  A.ctl = c->ctl_dev;
  A.X[0] = x0;
  A.X[1] = x1;
  A.G = G;
  A.F = c->F;
  A.D = D;
  for (int i = 0; i < 3; ++i) A.R[i] = (T*)c->R[i];
  A.XL = (T*)c->XL;
  A.P = (T*)c->P;
  A.AP = (T*)c->AP;
  A.hbuf = c->hbuf;
  A.kmax = c->kmax;
  A.L = c->L;
  A.prof = c->prof;
  return A;
}

// Launch the persistent kernel with the control block in c->ctl_host; on
// return c->ctl_host holds the outputs.
static int run_stepper(tdgl_ctx* c, double* x0, double* x1, double* G, double* D, tdgl_stream_t s) {
  TDGL_CUDA(cudaMemsetAsync(c->bar, 0, 4 * sizeof(unsigned), s));
  TDGL_CUDA(cudaMemsetAsync(c->err, 0, 4 * sizeof(int), s));
  TDGL_CUDA(cudaMemcpyAsync(c->ctl_dev, c->ctl_host, sizeof(Ctl), cudaMemcpyHostToDevice, s));
  if (c->precision == TDGL_MIXED)
    TDGL_CUDA(stepper_launch_f32(make_args<float>(c, x0, x1, G, D), c->blocks, c->smem, s));
  else
    TDGL_CUDA(stepper_launch_f64(make_args<double>(c, x0, x1, G, D), c->blocks, c->smem, s));
  int herr = 0;
  TDGL_CUDA(cudaMemcpyAsync(c->ctl_host, c->ctl_dev, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
  TDGL_CUDA(cudaMemcpyAsync(&herr, c->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  TDGL_CUDA(cudaStreamSynchronize(s));
  if (herr) c->ctl_host->status = herr;
  return TDGL_OK;
}

static void fill_stats(const tdgl_ctx* c, tdgl_stats* st) {
  if (!st) return;
  const Ctl& k = *c->ctl_host;
  st->status = k.status;
  st->steps = k.steps;
  st->newton_converged = k.newton_converged;
  st->newton_iters_last = k.newton_iters_last;
  st->krylov_last = k.krylov_last;
  st->max_krylov = k.max_krylov;
  st->newton_iters = k.newton_iters;
  st->krylov_iters = k.krylov_iters;
  st->rhs_evals = k.rhs_evals;
  st->jvp_evals = k.jvp_evals;
  st->rejections = k.rejections;
  st->krylov_sq = k.krylov_sq;
  st->t = k.t;
  st->dt_cur = k.dt_cur;
  st->last_gnorm = k.last_gnorm;
  st->last_dxnorm = k.last_dxnorm;
  st->kernel_launches = 1;
}

static void ctl_reset(tdgl_ctx* c) {
  std::memset(c->ctl_host, 0, sizeof(Ctl));
  c->ctl_host->field_const = 1;
  c->ctl_host->krylov = c->krylov;
}

extern "C" int tdgl_ctx_set_krylov(tdgl_ctx* c, int32_t kind) {
  if (!c) return fail(TDGL_EINVAL, "null argument");
  if (kind != TDGL_KRYLOV_GMRES && kind != TDGL_KRYLOV_GCR) return fail(TDGL_EINVAL, "unknown Krylov method");
  c->krylov = kind;
  return TDGL_OK;
}

static int krylov_cap(const tdgl_ctx* c, int32_t max_iter) {
  // the reference default is len(b) = n_state; the workspace bound is enforced on the device
  long ref = (long)(c->g.ncomp - 1) * c->g.n;
  return max_iter > 0 ? max_iter : (int)std::min(ref, (long)1 << 30);
}

template <typename T>
__global__ void k_to_t(const double* __restrict__ a, T* __restrict__ b, long L) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < L; e += (long)gridDim.x * blockDim.x) b[e] = (T)a[e];
}

extern "C" int tdgl_tgcr_trap(tdgl_ctx* c, const double* x_lin, const double* bvec, double* dvec, double dt,
                              double tol, int32_t max_iter, double eps_mf, int32_t jvp_mode, double Bx, double By,
                              double Bz, tdgl_stats* st, tdgl_stream_t s) {
  if (!c || !x_lin || !bvec || !dvec) return fail(TDGL_EINVAL, "null argument");
  if (c->npend) return fail(TDGL_EINVAL, "a launch of this context has not been collected");
  if (jvp_mode == TDGL_JVP_FD && c->precision == TDGL_MIXED)
    return fail(TDGL_EINVAL, "the finite-difference product needs the FP64 context");
  int rc;
  if ((rc = ensure_workspace(c))) return rc;
  // the first Krylov vector: GCR keeps it in R[0], GMRES in basis slot 0
  void* r0 = c->krylov == KRY_GCR ? c->R[0] : c->P;
  if (c->precision == TDGL_MIXED) k_to_t<float><<<grid_1d(c, c->L), kThreads, 0, s>>>(bvec, (float*)r0, c->L);
  else TDGL_CUDA(cudaMemcpyAsync(r0, bvec, c->L * sizeof(double), cudaMemcpyDeviceToDevice, s));
  ctl_reset(c);
  Ctl& k = *c->ctl_host;
  k.run_mode = RUN_TGCR;
  k.dt = dt;
  k.tol_gcr = tol;
  k.krylov_max_iter = krylov_cap(c, max_iter);
  k.eps_mf = eps_mf;
  k.jvp_mode = jvp_mode;
  k.Bx = Bx; k.By = By; k.Bz = Bz;
  if ((rc = run_stepper(c, const_cast<double*>(x_lin), c->X1, c->G, dvec, s))) return rc;
  fill_stats(c, st);
  return c->ctl_host->status;
}

extern "C" int tdgl_newton_trap(tdgl_ctx* c, double* x, const double* gamma, double dt, double tol_f,
                                double tol_dx, int32_t max_iter, double tol_gcr, double eps_mf, int32_t jvp_mode,
                                double Bx, double By, double Bz, tdgl_stats* st, tdgl_stream_t s) {
  if (!c || !x || !gamma) return fail(TDGL_EINVAL, "null argument");
  if (c->npend) return fail(TDGL_EINVAL, "a launch of this context has not been collected");
  if (jvp_mode == TDGL_JVP_FD && c->precision == TDGL_MIXED)
    return fail(TDGL_EINVAL, "the finite-difference product needs the FP64 context");
  int rc;
  if ((rc = ensure_workspace(c))) return rc;
  ctl_reset(c);
  Ctl& k = *c->ctl_host;
  k.run_mode = RUN_NEWTON;
  k.dt = dt;
  k.tol_f = tol_f;
  k.tol_dx = tol_dx;
  k.newton_max_iter = max_iter;
  k.tol_gcr = tol_gcr;
  k.krylov_max_iter = krylov_cap(c, 0);
  k.eps_mf = eps_mf;
  k.jvp_mode = jvp_mode;
  k.Bx = Bx; k.By = By; k.Bz = Bz;
  k.cur = 0;
  if ((rc = run_stepper(c, x, c->X1, const_cast<double*>(gamma), nullptr, s))) return rc;
  fill_stats(c, st);
  return c->ctl_host->status;
}

// ---------------------------------------------------------------------------
// Graph executor (GMRES): workspace, graph, launch
// ---------------------------------------------------------------------------

// Degree of the polynomial preconditioner: tdgl_ctx_set_poly, else
// TDGL_POLY_DEGREE, else the default.
static int poly_setting(const tdgl_ctx* c) {
  int d = kPolyDefault;
  if (c->poly_req >= 0) d = c->poly_req;
  else if (const char* e = std::getenv("TDGL_POLY_DEGREE")) {
    if (e[0]) d = std::atoi(e);
  }
  return std::min(std::max(d, 0), kPolyMax);
}

// Upper bound of the spectral radius of J (Gershgorin, from the stencil
// coefficients): the vector-potential rows sum to at most 8 kappa^2 sum_a 1/h_a^2
// plus the supercurrent terms (|psi|^2 of order 1), the order-parameter rows
// to (2 + 2 sqrt 2) sum_a 1/h_a^2 plus the nonlinear and relaxation terms.
static double poly_rho_bound(const tdgl_ctx* c) {
  const Grid& g = c->g;
  const double s2 = 1.0 / g.hx2 + 1.0 / g.hy2 + (g.is3d ? 1.0 / g.hz2 : 0.0);
  const double field = 8.0 * c->k2max * s2 + 6.0;
  const double order = (2.0 + 2.0 * std::sqrt(2.0)) * s2 + 4.0 + (g.has_material ? 1.0 / kTauRelax : 0.0);
  return 1.02 * std::max(field, order);
}

template <typename T>
static GArgs<T> make_gargs(tdgl_ctx* c) {
  GArgs<T> A{};
  A.g = c->g;
  A.dev = c->gdev;
  A.Xn = c->Xn;
  A.Xi = c->X1;
  A.G = c->G;
  A.F = c->F;
  A.En = c->En;
  A.Ei = c->Ei;
  A.XLe = (T*)c->XLe;
  A.VE = (T*)c->VE;
  A.V = (T*)c->P;
  A.W = (T*)c->AP;
  A.part_dots = c->part_dots;
  A.part_orth = c->part_orth;
  A.part_nrhs = c->part_nrhs;
  A.part_upd = c->part_upd;
  A.kry = c->kry;
  A.L = c->L;
  A.npf = c->npf;
  A.kmax = c->kmax;
  A.nblk = c->gblocks;
  A.UB = (T*)c->UB;
  A.Zb[0] = (T*)c->Zb[0];
  A.Zb[1] = (T*)c->Zb[1];
  A.vs = (long)c->g.ncomp * c->npf;
  A.part_arn = c->part_arn;
  A.ticket = c->ticket;
  A.nblk_arn = c->nblk_arn;
  A.nblk_orth = c->nblk_orth;
  A.arn_gx = c->arn_gx;
  A.arn_gy = c->arn_gy;
  A.apply_dots = c->apply_dots;
  A.deadmask = c->deadmask;
  A.ldead = c->ldead;
  A.tls = c->tl_on ? c->tls : nullptr;
  A.tl_par = 0;
  A.forcing = c->forcing;
  A.ntiles = c->ntiles;
  A.ngroups = c->ngroups;
  A.gpart = c->gpart;
  A.gticket = c->gticket;
  A.imask = c->imask;
  A.cxu = c->g.kappa2 / c->g.hx2;
  A.cyu = c->g.kappa2 / c->g.hy2;
  A.czu = c->g.is3d ? c->g.kappa2 / c->g.hz2 : 0.0;
  A.poly_deg = c->UB ? c->poly_deg : 0;
  A.poly_rho = poly_rho_bound(c);
  A.PW[0] = (T*)c->PW[0];
  A.PW[1] = (T*)c->PW[1];
  A.PB = (T*)c->PB;
  return A;
}

// Dead-link masks of the interior nodes (device order), from the same rule as
// NbM::phi; links that leave the grid (the z offsets of a 2-D grid) stay clear.
static __global__ void k_deadmask(Grid g, uint32_t* __restrict__ mask) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    int i, j, k;
    node_ijk(g, d, i, j, k);
    const long m = i + (long)g.mj * j + (long)g.mk * k;
    uint32_t w = 0u;
#pragma unroll
    for (int b = 0; b < 27; ++b) {
      const int a = dead_link(b, 0), di = dead_link(b, 1), dj = dead_link(b, 2), dk = dead_link(b, 3);
      if (!g.is3d && (a == 2 || dk != 0)) continue;
      const long e = m + di + (long)dj * g.mj + (long)dk * g.mk;
      const unsigned lf = g.lflags ? (unsigned)g.lflags[e] : 0u;
      const bool dead = (a == 0 && i + di == g.Nx - 1) || (a == 1 && j + dj == g.Ny - 1) ||
                        (a == 2 && k + dk == g.Nz - 1) || ((lf >> a) & 1u);
      if (dead) w |= 1u << b;
    }
    mask[d] = w;
  }
}

// Dead links of every full-grid node (the rule of NbM::phi, stated per link
// instead of per reading node): bit a when link a of the node is the normal
// link on plane N-1 of axis a or a hole link.
static __global__ void k_ldead(Grid g, long npf, uint8_t* __restrict__ out) {
  const long dimx = g.is3d ? (long)g.mk * (g.Nz + 1) : (long)g.mk;
  for (long m = blockIdx.x * (long)blockDim.x + threadIdx.x; m < npf; m += (long)gridDim.x * blockDim.x) {
    uint8_t b = 0;
    if (m < dimx) {
      const int k = (int)(m / g.mk), r = (int)(m - (long)k * g.mk), j = r / g.mj, i = r - j * g.mj;
      if (i <= g.Nx) {
        b = g.lflags ? g.lflags[m] : (uint8_t)0;
        if (i == g.Nx - 1) b |= 1u;
        if (j == g.Ny - 1) b |= 2u;
        if (g.is3d && k == g.Nz - 1) b |= 4u;
      }
    }
    out[m] = b;
  }
}

// Product and projections as one kernel or two: as set by tdgl_ctx_set_blocks,
// else TDGL_ARN_APPLY_DOTS, else one kernel for FP64 vectors (the stencil's
// arithmetic then hides more of the basis reads) and two for FP32 ones.
static int apply_dots_setting(const tdgl_ctx* c) {
  if (c->apply_dots_req >= 0) return c->apply_dots_req;
  const char* e = std::getenv("TDGL_ARN_APPLY_DOTS");
  if (e && e[0]) return e[0] != '0';
  return c->precision == TDGL_FP64;
}

// Tensor maps of the TMA-staged stencil over the context's FP32 full-grid
// vectors (3-D grids; TDGL_TMA=0 keeps the stencil that reads global memory):
// dimensions (x, y, z, component[, vector]) with the padded row pitch, boxes
// of (32 NX + 4) x 10 x 1 x 5 entries for the kernel with NX nodes per thread
// (TDGL_TL_NX, default 2).  z-chunks per tile column: TDGL_TL_CHUNKS, else as
// many as keep every block of the launch resident at once.  The stencil nodes
// of the step graph depend programmatically on the node before them unless
// TDGL_PDL=0.
static int setup_tl(tdgl_ctx* c) {
  c->tl_on = false;
  const Grid& g = c->g;
  if (c->precision != TDGL_MIXED || !g.is3d) return TDGL_OK;
  if (const char* e = std::getenv("TDGL_TMA"))
    if (e[0] == '0') return TDGL_OK;
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    cudaError_t e = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
      return fail(TDGL_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  const cuuint64_t fs = sizeof(float);
  const cuuint64_t dims[5] = {(cuuint64_t)g.mj, (cuuint64_t)g.Ny + 1, (cuuint64_t)g.Nz + 1, (cuuint64_t)kTlComp,
                              (cuuint64_t)c->kmax + 1};
  const cuuint64_t strides[4] = {(cuuint64_t)g.mj * fs, (cuuint64_t)g.mk * fs, (cuuint64_t)c->npf * fs,
                                 (cuuint64_t)kTlComp * (cuuint64_t)c->npf * fs};
  // nodes per thread along x: TDGL_TL_NX (1 or 2), else 2
  int tnx = 2;
  if (const char* e = std::getenv("TDGL_TL_NX"))
    if (std::atoi(e) == 1 || std::atoi(e) == 2) tnx = std::atoi(e);
  c->tlm.nx = tnx;
  // programmatic dependent launches of the stencil nodes: TDGL_PDL=0 turns them off
  c->tlm.pdl = 1;
  // pair coefficients of the two-nodes-per-thread kernel (uniform kappa; the
  // 1 / h^2 entries serve a per-node kappa too)
  tl_pair_coef(c->tlm.k2, make_float2((float)(g.kappa2 / g.hx2), (float)(g.kappa2 / g.hx2)),
               make_float2((float)(g.kappa2 / g.hy2), (float)(g.kappa2 / g.hy2)),
               make_float2((float)(g.kappa2 / g.hz2), (float)(g.kappa2 / g.hz2)));
  c->tlm.k2[K_IHX] = make_float2((float)g.ihx2, (float)g.ihx2);
  c->tlm.k2[K_IHY] = make_float2((float)g.ihy2, (float)g.ihy2);
  c->tlm.k2[K_IHZ] = make_float2((float)g.ihz2, (float)g.ihz2);
  if (const char* e = std::getenv("TDGL_PDL"))
    if (e[0] == '0') c->tlm.pdl = 0;
  const cuuint32_t box[5] = {(cuuint32_t)(32 * tnx + 4), (cuuint32_t)kTlBoxY, 1u, (cuuint32_t)kTlComp, 1u};
  const cuuint32_t es[5] = {1u, 1u, 1u, 1u, 1u};
  if (g.ncomp != kTlComp || g.mj % 4 || c->npf % 4) return fail(TDGL_ECUDA, "full-grid layout not TMA-aligned");
  void* base[5] = {c->XLe, c->UB, c->PW[0], c->PW[1], c->PB};
  for (int t = 0; t < 5; ++t) {
    const cuuint32_t rank = (t == TM_UB || t == TM_PB) ? 5u : 4u;
    CUresult r = encode(&c->tlm.m[t], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, base[t], dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(TDGL_ECUDA, "cuTensorMapEncodeTiled failed (code " + std::to_string((int)r) + ")");
  }
  const int tiles = tl_grid_x(g.nx, tnx) * c->arn_gy;
  const int resident = tnx == 2 ? TlShape<2>::kMinBlocks : TlShape<1>::kMinBlocks;
  int ch = std::max(1, (c->num_sms * resident) / std::max(tiles, 1));
  if (const char* e = std::getenv("TDGL_TL_CHUNKS"))
    if (std::atoi(e) > 0) ch = std::atoi(e);
  c->tl_chunks = std::min(std::max(ch, 1), g.nz);
  if (!c->tls) {
    int rc = ctx_alloc(c, (void**)&c->tls, 2 * sizeof(TlSched));   // zeroed
    if (rc) return rc;
  }
  c->tl_on = true;
  return TDGL_OK;
}

// Buffers of the three-kernel Arnoldi step (analytic products).
static int ensure_arnoldi_ws(tdgl_ctx* c) {
  if (c->UB) return TDGL_OK;
  const Grid& g = c->g;
  const size_t tsz = c->precision == TDGL_MIXED ? sizeof(float) : sizeof(double);
  const size_t vb = (size_t)g.ncomp * c->npf * tsz;
  c->arn_gx = (g.nx + 31) / 32;
  c->arn_gy = (g.ny + 7) / 8;
  c->ntiles = c->arn_gx * c->arn_gy * (g.is3d ? g.nz : 1);
  c->ngroups = (c->ntiles + 31) / 32;
  c->ngroups_cap = std::max(c->ngroups, (c->num_sms * kMaxBlocksPerSm + 31) / 32);
  c->apply_dots = apply_dots_setting(c);
  int rc;
  if ((rc = ctx_alloc(c, &c->UB, vb * (c->kmax + 1)))) return rc;
  if ((rc = ctx_alloc(c, &c->Zb[0], vb))) return rc;
  if ((rc = ctx_alloc(c, &c->Zb[1], vb))) return rc;
  if ((rc = ctx_alloc(c, &c->PW[0], vb))) return rc;
  if ((rc = ctx_alloc(c, &c->PW[1], vb))) return rc;
  if ((rc = ctx_alloc(c, &c->PB, vb * (c->kmax + 1)))) return rc;
  c->poly_deg = poly_setting(c);
  const size_t nparts = std::max((size_t)c->num_sms * kMaxBlocksPerSm, (size_t)c->ntiles);
  if ((rc = ctx_alloc(c, (void**)&c->part_arn, sizeof(double) * (c->kmax + 2) * nparts))) return rc;
  if ((rc = ctx_alloc(c, (void**)&c->gpart, sizeof(double) * (c->kmax + 2) * (size_t)c->ngroups_cap))) return rc;
  if ((rc = ctx_alloc(c, (void**)&c->gticket, sizeof(unsigned) * (size_t)c->ngroups_cap))) return rc;
  if ((rc = ctx_alloc(c, (void**)&c->ticket, sizeof(unsigned)))) return rc;
  // interior mask of the full grid (projections run over interior entries only)
  std::vector<uint8_t> im((size_t)c->npf, 0);
  for (int k = g.is3d ? 1 : 0; k <= (g.is3d ? g.nz : 0); ++k)
    for (int j = 1; j <= g.ny; ++j)
      for (int i = 1; i <= g.nx; ++i) im[(size_t)i + (size_t)g.mj * j + (size_t)g.mk * k] = 1;
  if ((rc = ctx_alloc(c, (void**)&c->imask, (size_t)c->npf))) return rc;
  TDGL_CUDA(cudaMemcpy(c->imask, im.data(), (size_t)c->npf, cudaMemcpyHostToDevice));
  if ((rc = ctx_alloc(c, (void**)&c->deadmask, sizeof(uint32_t) * (size_t)g.n))) return rc;
  k_deadmask<<<grid_1d(c, g.n), kThreads>>>(g, c->deadmask);
  TDGL_CUDA(cudaGetLastError());
  if ((rc = ctx_alloc(c, (void**)&c->ldead, (size_t)c->npf))) return rc;
  k_ldead<<<grid_1d(c, c->npf), kThreads>>>(g, c->npf, c->ldead);
  TDGL_CUDA(cudaGetLastError());
  return setup_tl(c);
}

// Block counts of the graph's grid kernels from the stream and Krylov settings:
// the orthogonalisation and the projections run on 4/5 of the Krylov count
// (4 blocks per SM by default, their register budgets).
static void set_arnoldi_blocks(tdgl_ctx* c) {
  c->gblocks = c->blk_stream;
  c->nblk_arn = std::max(1, c->blk_krylov * 4 / 5);
  c->nblk_orth = std::min(c->gblocks, c->nblk_arn);
}

// Graph variant v: 0 = finite-difference Krylov body, 1 = three-kernel Arnoldi step.
static int ensure_graph(tdgl_ctx* c, int v) {
  if (c->gexec[v]) return TDGL_OK;
  int rc;
  if ((rc = ensure_workspace(c))) return rc;
  if (!c->gws_ready) {
    const Grid& g = c->g;
    long dimx = g.is3d ? (long)g.mk * (g.Nz + 1) : (long)g.mk;
    c->npf = (dimx + 127) / 128 * 128;
    // grid kernels of the step: 8 blocks per SM for the one-node-per-thread
    // passes, 5 for the Arnoldi streams (their register budgets), unless set by
    // tdgl_ctx_set_blocks or TDGL_STREAM_BLOCKS_PER_SM / TDGL_KRYLOV_BLOCKS_PER_SM
    auto env_bps = [](const char* name, int dflt) {
      const char* e = std::getenv(name);
      const int v = e ? std::atoi(e) : 0;
      return (v >= 1 && v <= kMaxBlocksPerSm) ? v : dflt;
    };
    if (!c->blk_stream) c->blk_stream = c->num_sms * env_bps("TDGL_STREAM_BLOCKS_PER_SM", 8);
    if (!c->blk_krylov) c->blk_krylov = c->num_sms * env_bps("TDGL_KRYLOV_BLOCKS_PER_SM", 5);
    set_arnoldi_blocks(c);
    const size_t tsz = c->precision == TDGL_MIXED ? sizeof(float) : sizeof(double);
    const size_t full64 = (size_t)g.ncomp * c->npf * sizeof(double);
    const size_t fullT = (size_t)g.ncomp * c->npf * tsz;
    const size_t nb = (size_t)c->num_sms * kMaxBlocksPerSm;
    if ((rc = ctx_alloc(c, (void**)&c->Xn, c->L * sizeof(double)))) return rc;
    if ((rc = ctx_alloc(c, (void**)&c->En, full64))) return rc;
    if ((rc = ctx_alloc(c, (void**)&c->Ei, full64))) return rc;
    if (c->precision == TDGL_MIXED) {
      if ((rc = ctx_alloc(c, &c->XLe, fullT))) return rc;
    } else {
      c->XLe = c->Ei;
    }
    if ((rc = ctx_alloc(c, &c->VE, fullT))) return rc;
    if ((rc = ctx_alloc(c, (void**)&c->part_dots, sizeof(double) * (c->kmax + 1) * nb))) return rc;
    if ((rc = ctx_alloc(c, (void**)&c->part_orth, sizeof(double) * nb))) return rc;
    if ((rc = ctx_alloc(c, (void**)&c->part_nrhs, sizeof(double) * 3 * nb))) return rc;
    if ((rc = ctx_alloc(c, (void**)&c->part_upd, sizeof(double) * nb))) return rc;
    if ((rc = ctx_alloc(c, (void**)&c->kry, sizeof(double) * kry_len(c->kmax)))) return rc;
    if ((rc = ctx_alloc(c, (void**)&c->gdev, sizeof(GDev)))) return rc;
    TDGL_CUDA(cudaMallocHost((void**)&c->gdev_host, sizeof(GDev)));
    c->gin[0] = c->gdev_host;
    TDGL_CUDA(cudaMallocHost((void**)&c->gin[1], sizeof(GDev)));
    TDGL_CUDA(cudaMallocHost((void**)&c->gout[0], sizeof(GDev)));
    TDGL_CUDA(cudaMallocHost((void**)&c->gout[1], sizeof(GDev)));
    for (int k = 0; k < 2; ++k) TDGL_CUDA(cudaEventCreateWithFlags(&c->gev[k], cudaEventDisableTiming));
    if ((rc = ctx_alloc(c, (void**)&c->gclk, 2 * sizeof(double)))) return rc;
    const char* pe = std::getenv("TDGL_PROFILE");
    c->gprof = pe && pe[0] && pe[0] != '0';
    // forcing term of the analytic-product GMRES solves (on; TDGL_FORCING=0
    // keeps every solve at tol_gcr)
    if (const char* e = std::getenv("TDGL_FORCING")) c->forcing = e[0] == '0' ? 0 : 1;
    c->gws_ready = true;
  }
  if (v == 1 && (rc = ensure_arnoldi_ws(c))) return rc;
  cudaError_t e;
  if (c->precision == TDGL_MIXED) {
    GArgs<float> A = make_gargs<float>(c);
    A.fused = v;
    if (!v) A.poly_deg = 0;
    if (!v) A.forcing = 0;
    e = graph_build_f32(A, (v && c->tl_on) ? &c->tlm : nullptr, c->tl_chunks, &c->graph[v], &c->gexec[v]);
  } else {
    GArgs<double> A = make_gargs<double>(c);
    A.fused = v;
    if (!v) A.poly_deg = 0;
    if (!v) A.forcing = 0;
    e = graph_build_f64(A, &c->graph[v], &c->gexec[v]);
  }
  if (e != cudaSuccess) {
    if (c->graph[v]) cudaGraphDestroy(c->graph[v]);
    c->graph[v] = nullptr;
    c->gexec[v] = nullptr;
    return fail(TDGL_ECUDA, std::string("building the stepper graph: ") + cudaGetErrorString(e));
  }
  return settle(c);
}

static int graph_status(int gs) {
  switch (gs) {
    case GS_OK: return TDGL_OK;
    case GS_IDLE: return TDGL_OK;
    case GS_NOCONV: return TDGL_ENOCONV;
    case GS_DTMIN: return TDGL_EDTMIN;
    case GS_KMAX: return TDGL_EKMAX;
    case GS_NONFINITE: return TDGL_ENONFINITE;
    default: return TDGL_ETIMEOUT;
  }
}

// Enqueue one graph launch for up to max_steps steps on stream s (no
// synchronisation) with the control blocks of launch slot `slot`; *noop is
// set when nothing needs to run.  cont: a continuation, which starts from the
// clock (t, dt_cur) the previous launch left in the device control block
// instead of (t0, cur0); the device's own step loop test decides whether it
// runs any step.  The slot's event is recorded after the launch's outputs.
static int graph_launch(tdgl_ctx* c, double* x, double t0, double cur0, int32_t max_steps, const tdgl_trap_opts* o,
                        const tdgl_field* f, tdgl_stream_t s, bool* noop, int slot = 0, bool cont = false) {
  int rc;
  const int v = o->jvp_mode == TDGL_JVP_ANALYTIC ? 1 : 0;
  if ((rc = ensure_graph(c, v))) return rc;
  GDev& h = *c->gin[slot];
  std::memset(&h, 0, sizeof(GDev));
  h.t = t0;
  h.dt_cur = cur0;
  h.t_stop = o->t_stop;
  h.dt = o->dt;
  h.dt_min = o->dt_min;
  h.tol_f = o->newton_tol_f;
  h.tol_dx = o->newton_tol_dx;
  h.tol_gcr = o->tol_gcr;
  h.eps_mf = o->eps_mf;
  h.Bx = f->Bx; h.By = f->By; h.Bz = f->Bz;
  h.t_on_fraction = f->t_on_fraction;
  h.ramp_fraction = f->ramp_fraction;
  h.t_field_stop = f->t_field_stop;
  h.ramp = f->ramp;
  h.field_const = f->constant;
  h.newton_max_iter = o->newton_max_iter;
  h.krylov_max_iter = krylov_cap(c, o->krylov_max_iter);
  h.adaptive = o->adaptive;
  h.jvp_mode = o->jvp_mode;
  h.max_steps = max_steps;
  // hard limit on loop iterations: every step may be retried down to dt_min
  // (at most ~12 cuts of dt/10 in double range) with full Newton / Krylov loops
  h.watchdog_cap = (long long)(max_steps + 1) * 40 * (o->newton_max_iter + 2) * (c->kmax + 3) + 1000;
  if (c->watchdog_req > 0) h.watchdog_cap = c->watchdog_req;
  h.wait_ns = c->wait_ns;
  h.prof_on = c->gprof ? 1 : 0;
  for (int k = 0; k < kKTypes; ++k) h.kt_start[k] = ~0ull;
  *noop = max_steps <= 0 || (!cont && !(h.t < h.t_stop - 1e-14));
  if (*noop) return TDGL_OK;
  static_assert(offsetof(GDev, dt_cur) == offsetof(GDev, t) + sizeof(double), "clock layout");
  char* clk = (char*)c->gdev + offsetof(GDev, t);
  TDGL_CUDA(cudaMemcpyAsync(c->Xn, x, c->L * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if (cont) TDGL_CUDA(cudaMemcpyAsync(c->gclk, clk, 2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  TDGL_CUDA(cudaMemcpyAsync(c->gdev, &h, sizeof(GDev), cudaMemcpyHostToDevice, s));
  if (cont) TDGL_CUDA(cudaMemcpyAsync(clk, c->gclk, 2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if (c->ticket) TDGL_CUDA(cudaMemsetAsync(c->ticket, 0, sizeof(unsigned), s));
  if (c->gticket) TDGL_CUDA(cudaMemsetAsync(c->gticket, 0, sizeof(unsigned) * (size_t)c->ngroups_cap, s));
  TDGL_CUDA(cudaGraphLaunch(c->gexec[v], s));
  TDGL_CUDA(cudaMemcpyAsync(c->gout[slot], c->gdev, sizeof(GDev), cudaMemcpyDeviceToHost, s));
  TDGL_CUDA(cudaMemcpyAsync(x, c->Xn, c->L * sizeof(double), cudaMemcpyDeviceToDevice, s));
  TDGL_CUDA(cudaEventRecord(c->gev[slot], s));
  c->has_clock = true;
  return TDGL_OK;
}

// Results of the graph_launch of slot `slot` (waits for its event).
static int graph_collect(tdgl_ctx* c, bool noop, double* t, double* dt_cur, tdgl_stats* st, int slot = 0) {
  if (!noop) TDGL_CUDA(cudaEventSynchronize(c->gev[slot]));
  GDev& h = noop ? *c->gin[slot] : *c->gout[slot];
  if (tdgl_stats* z = st) std::memset(z, 0, sizeof(*z));
  *t = h.t;
  *dt_cur = h.dt_cur;
  if (noop) {
    if (st) { st->t = h.t; st->dt_cur = h.dt_cur; }
    return TDGL_OK;
  }
  for (int k = 0; k < kKTypes; ++k) {
    c->gk_total[k] += h.kt_total[k];
    c->gk_count[k] += h.kt_count[k];
  }
  if (st) {
    st->status = graph_status(h.status);
    st->steps = h.steps;
    st->newton_converged = h.accepted;
    st->newton_iters_last = h.newton_k;
    st->krylov_last = h.krylov_last;
    st->max_krylov = h.max_krylov;
    st->newton_iters = h.newton_iters;
    st->krylov_iters = h.krylov_iters;
    st->krylov_sq = h.krylov_sq;
    st->rhs_evals = h.rhs_evals;
    st->jvp_evals = h.jvp_evals;
    st->rejections = h.rejections;
    st->t = h.t;
    st->dt_cur = h.dt_cur;
    st->last_gnorm = h.gnorm;
    st->last_dxnorm = h.dxnorm;
    st->kernel_launches = 1;
  }
  return graph_status(h.status);
}

static int run_graph(tdgl_ctx* c, double* x, double* t, double* dt_cur, int32_t max_steps, const tdgl_trap_opts* o,
                     const tdgl_field* f, tdgl_stats* st, tdgl_stream_t s) {
  bool noop = false;
  int rc = graph_launch(c, x, *t, *dt_cur, max_steps, o, f, s, &noop);
  if (rc) return rc;
  if (!noop) TDGL_CUDA(cudaStreamSynchronize(s));
  return graph_collect(c, noop, t, dt_cur, st);
}

extern "C" int tdgl_adjoint_solve(tdgl_ctx* c, const double* x, const double* b, double* mu, double h, double tol,
                                  double Bx, double By, double Bz, int32_t* iters, tdgl_stream_t s) {
  if (!c || !x || !b || !mu) return fail(TDGL_EINVAL, "null argument");
  if (c->npend) return fail(TDGL_EINVAL, "a launch of this context has not been collected");
  if (c->precision != TDGL_FP64) return fail(TDGL_EINVAL, "the adjoint solve needs an FP64 context");
  int rc;
  if ((rc = ensure_graph(c, 0))) return rc;            // the stepper workspace the solve shares
  const size_t L = (size_t)c->L;
  if (!c->adj) {
    if ((rc = ctx_alloc(c, (void**)&c->adj, sizeof(double) * 4 * L))) return rc;
    if ((rc = settle(c))) return rc;
  }
  if (!c->adj_exec) {
    GArgs<double> A = make_gargs<double>(c);
    A.forcing = 0;
    A.ax = c->adj;
    A.ab = c->adj + L;
    A.amu = c->adj + 2 * L;
    A.aT = c->adj + 3 * L;
    cudaError_t e = c->g.is3d ? build_adjoint_graph<true>(A, &c->adj_graph, &c->adj_exec)
                              : build_adjoint_graph<false>(A, &c->adj_graph, &c->adj_exec);
    if (e != cudaSuccess) {
      if (c->adj_graph) cudaGraphDestroy(c->adj_graph);
      c->adj_graph = nullptr;
      c->adj_exec = nullptr;
      return fail(TDGL_ECUDA, std::string("building the adjoint graph: ") + cudaGetErrorString(e));
    }
  }
  c->has_clock = false;                          // the device control block is reused below
  GDev& hd = *c->gdev_host;
  std::memset(&hd, 0, sizeof(GDev));
  hd.dta = 2.0 * h;
  hd.tol_gcr = tol;
  hd.krylov_max_iter = c->kmax;
  hd.watchdog_cap = (long long)c->kmax + 100;
  hd.Bx = Bx; hd.By = By; hd.Bz = Bz;
  for (int k = 0; k < kKTypes; ++k) hd.kt_start[k] = ~0ull;
  TDGL_CUDA(cudaMemcpyAsync(c->adj, x, L * sizeof(double), cudaMemcpyDeviceToDevice, s));
  TDGL_CUDA(cudaMemcpyAsync(c->adj + L, b, L * sizeof(double), cudaMemcpyDeviceToDevice, s));
  TDGL_CUDA(cudaMemcpyAsync(c->gdev, &hd, sizeof(GDev), cudaMemcpyHostToDevice, s));
  TDGL_CUDA(cudaGraphLaunch(c->adj_exec, s));
  TDGL_CUDA(cudaMemcpyAsync(&hd, c->gdev, sizeof(GDev), cudaMemcpyDeviceToHost, s));
  TDGL_CUDA(cudaMemcpyAsync(mu, c->adj + 2 * L, L * sizeof(double), cudaMemcpyDeviceToDevice, s));
  TDGL_CUDA(cudaStreamSynchronize(s));
  if (iters) *iters = hd.j;
  if (hd.status != GS_OK) return graph_status(hd.status);
  return hd.accepted ? TDGL_OK : TDGL_ENOCONV;
}

extern "C" int tdgl_trap_launch(tdgl_ctx* c, double* x, double t, double dt_cur, int32_t max_steps,
                                const tdgl_trap_opts* o, const tdgl_field* f, tdgl_stream_t s) {
  if (!c || !x || !o || !f) return fail(TDGL_EINVAL, "null argument");
  if (o->jvp_mode == TDGL_JVP_FD && c->precision == TDGL_MIXED)
    return fail(TDGL_EINVAL, "the finite-difference product needs the FP64 context");
  if (c->krylov != KRY_GMRES) return fail(TDGL_EINVAL, "asynchronous stepping needs the GMRES graph executor");
  if (c->npend) return fail(TDGL_EINVAL, "a launch of this context has not been collected");
  const int slot = c->next_slot;
  int rc = graph_launch(c, x, t, dt_cur, max_steps, o, f, s, &c->pend_noop[slot], slot, false);
  if (rc == TDGL_OK) {
    c->pend_head = slot;
    c->npend = 1;
    c->next_slot = slot ^ 1;
  }
  return rc;
}

extern "C" int tdgl_trap_launch_next(tdgl_ctx* c, double* x, int32_t max_steps, const tdgl_trap_opts* o,
                                     const tdgl_field* f, tdgl_stream_t s) {
  if (!c || !x || !o || !f) return fail(TDGL_EINVAL, "null argument");
  if (o->jvp_mode == TDGL_JVP_FD && c->precision == TDGL_MIXED)
    return fail(TDGL_EINVAL, "the finite-difference product needs the FP64 context");
  if (c->krylov != KRY_GMRES) return fail(TDGL_EINVAL, "asynchronous stepping needs the GMRES graph executor");
  if (c->npend > 1) return fail(TDGL_EINVAL, "two launches of this context are already queued");
  if (!c->has_clock) return fail(TDGL_EINVAL, "no earlier launch of this context to continue");
  const int slot = c->next_slot;
  int rc = graph_launch(c, x, 0.0, 0.0, max_steps, o, f, s, &c->pend_noop[slot], slot, true);
  if (rc == TDGL_OK) {
    if (c->npend == 0) c->pend_head = slot;
    ++c->npend;
    c->next_slot = slot ^ 1;
  }
  return rc;
}

extern "C" int tdgl_trap_collect(tdgl_ctx* c, double* t, double* dt_cur, tdgl_stats* st) {
  if (!c || !t || !dt_cur) return fail(TDGL_EINVAL, "null argument");
  if (!c->npend) return fail(TDGL_EINVAL, "no launch to collect");
  const int slot = c->pend_head;
  c->pend_head ^= 1;
  --c->npend;
  return graph_collect(c, c->pend_noop[slot], t, dt_cur, st, slot);
}

extern "C" int tdgl_ctx_set_blocks(tdgl_ctx* c, int32_t stream_blocks, int32_t krylov_blocks, int32_t fused) {
  if (!c) return fail(TDGL_EINVAL, "null argument");
  const int cap = c->num_sms * kMaxBlocksPerSm;
  if (stream_blocks < 1 || stream_blocks > cap || krylov_blocks < 1 || krylov_blocks > cap)
    return fail(TDGL_EINVAL, "block counts must lie in [1, 8 x SMs]");
  if (c->npend) return fail(TDGL_EINVAL, "a launch of this context has not been collected");
  c->blk_stream = stream_blocks;
  c->blk_krylov = krylov_blocks;
  c->apply_dots_req = fused < 0 ? -1 : (fused ? 1 : 0);
  if (c->UB) c->apply_dots = apply_dots_setting(c);
  if (c->gws_ready) set_arnoldi_blocks(c);
  for (int v = 0; v < 2; ++v) {           // rebuilt with the new shapes at the next launch
    if (c->gexec[v]) cudaGraphExecDestroy(c->gexec[v]);
    if (c->graph[v]) cudaGraphDestroy(c->graph[v]);
    c->gexec[v] = nullptr;
    c->graph[v] = nullptr;
  }
  return TDGL_OK;
}

extern "C" int tdgl_ctx_set_poly(tdgl_ctx* c, int32_t degree) {
  if (!c) return fail(TDGL_EINVAL, "null argument");
  if (degree < -1 || degree > kPolyMax) return fail(TDGL_EINVAL, "polynomial degree must lie in [-1, 12]");
  if (c->npend) return fail(TDGL_EINVAL, "a launch of this context has not been collected");
  c->poly_req = degree;
  if (c->UB) c->poly_deg = poly_setting(c);
  if (c->gexec[1]) cudaGraphExecDestroy(c->gexec[1]);   // the analytic-product graph is rebuilt at the next launch
  if (c->graph[1]) cudaGraphDestroy(c->graph[1]);
  c->gexec[1] = nullptr;
  c->graph[1] = nullptr;
  return TDGL_OK;
}

extern "C" int32_t tdgl_ctx_poly_degree(const tdgl_ctx* c) {
  if (!c) return -1;
  return c->UB ? c->poly_deg : poly_setting(c);
}

extern "C" int tdgl_trap_run(tdgl_ctx* c, double* x, double* t, double* dt_cur, int32_t max_steps,
                             const tdgl_trap_opts* o, const tdgl_field* f, tdgl_stats* st, tdgl_stream_t s) {
  if (!c || !x || !t || !dt_cur || !o || !f) return fail(TDGL_EINVAL, "null argument");
  if (c->npend) return fail(TDGL_EINVAL, "a launch of this context has not been collected");
  if (o->jvp_mode == TDGL_JVP_FD && c->precision == TDGL_MIXED)
    return fail(TDGL_EINVAL, "the finite-difference product needs the FP64 context");
  if (c->krylov == KRY_GMRES) return run_graph(c, x, t, dt_cur, max_steps, o, f, st, s);
  int rc;
  if ((rc = ensure_workspace(c))) return rc;
  ctl_reset(c);
  Ctl& k = *c->ctl_host;
  k.run_mode = RUN_TRAP;
  k.t_stop = o->t_stop;
  k.dt = o->dt;
  k.dt_min = o->dt_min;
  k.tol_f = o->newton_tol_f;
  k.tol_dx = o->newton_tol_dx;
  k.tol_gcr = o->tol_gcr;
  k.eps_mf = o->eps_mf;
  k.newton_max_iter = o->newton_max_iter;
  k.krylov_max_iter = krylov_cap(c, o->krylov_max_iter);
  k.adaptive = o->adaptive;
  k.jvp_mode = o->jvp_mode;
  k.max_steps = max_steps;
  k.Bx = f->Bx; k.By = f->By; k.Bz = f->Bz;
  k.t_on_fraction = f->t_on_fraction;
  k.ramp_fraction = f->ramp_fraction;
  k.t_field_stop = f->t_field_stop;
  k.ramp = f->ramp;
  k.field_const = f->constant;
  k.t = *t;
  k.dt_cur = *dt_cur;
  k.cur = 0;
  if ((rc = run_stepper(c, x, c->X1, c->G, nullptr, s))) return rc;
  if (c->ctl_host->cur == 1) {
    TDGL_CUDA(cudaMemcpyAsync(x, c->X1, c->L * sizeof(double), cudaMemcpyDeviceToDevice, s));
    TDGL_CUDA(cudaStreamSynchronize(s));
  }
  *t = c->ctl_host->t;
  *dt_cur = c->ctl_host->dt_cur;
  fill_stats(c, st);
  return c->ctl_host->status;
}

static void host_field(const tdgl_field* f, double t, double& bx, double& by, double& bz) {
  if (f->constant) { bx = f->Bx; by = f->By; bz = f->Bz; return; }
  if (t <= 0.0 || t > f->t_field_stop * f->t_on_fraction) { bx = by = bz = 0.0; return; }
  double sc = 1.0;
  if (f->ramp) {
    double tr = f->t_field_stop * f->ramp_fraction;
    sc = tr > 0.0 ? std::min(t / tr, 1.0) : 1.0;
  }
  bx = f->Bx * sc; by = f->By * sc; bz = f->Bz * sc;
}

extern "C" int tdgl_euler_run(tdgl_ctx* c, double* x, double* t, double t_stop, double dt, int32_t n_steps,
                              const tdgl_field* f, tdgl_stream_t s) {
  if (!c || !x || !t || !f) return fail(TDGL_EINVAL, "null argument");
  if (c->npend) return fail(TDGL_EINVAL, "a launch of this context has not been collected");
  double* a = x;
  double* b = c->s_x;
  for (int i = 0; i < n_steps; ++i) {
    double dta = std::min(dt, t_stop - *t);
    double bx, by, bz;
    host_field(f, *t, bx, by, bz);
    k_euler<<<grid_1d(c, c->g.n), kThreads, 0, s>>>(c->g, a, b, dta, bterms(c->g, bx, by, bz));
    TDGL_CUDA(cudaGetLastError());
    std::swap(a, b);
    *t += dta;
  }
  if (a != x) TDGL_CUDA(cudaMemcpyAsync(x, a, c->L * sizeof(double), cudaMemcpyDeviceToDevice, s));
  return TDGL_OK;
}

// ap = p - dt/2 J(x) p as the analytic-product Krylov solves compute it: x
// staged as the linearisation copy (with the field's face offsets) and p as
// basis vector 0, both on the full grid in the context's Krylov precision,
// then the graph's product kernel (the TMA-staged one for FP32 3-D contexts)
// and the interior entries back into the device layout.  Uses the stepping
// workspace; blocks until the stream has passed the product, to report a
// bounded wait that ran out.
static int krylov_product(tdgl_ctx* c, const double* x, const double* p, double* ap, double dt, double Bx,
                          double By, double Bz, tdgl_stream_t s) {
  if (c->npend) return fail(TDGL_EINVAL, "a launch of this context has not been collected");
  int rc;
  if ((rc = ensure_graph(c, 1))) return rc;
  const Grid& g = c->g;
  const BTerms<double> b = bterms(g, Bx, By, Bz);
  c->has_clock = false;                          // the device control block is reused below
  GDev& h = *c->gdev_host;
  std::memset(&h, 0, sizeof(GDev));
  h.dta = dt;
  h.wait_ns = c->wait_ns;
  for (int k = 0; k < kKTypes; ++k) h.kt_start[k] = ~0ull;
  TDGL_CUDA(cudaMemcpyAsync(c->gdev, &h, sizeof(GDev), cudaMemcpyHostToDevice, s));
  const int nb = grid_1d(c, g.n), nbp = grid_1d(c, g.npad);
  cudaError_t e;
  if (c->precision == TDGL_MIXED) {
    GArgs<float> A = make_gargs<float>(c);
    A.fused = 1;
    A.standalone = 1;
    A.poly_deg = 0;
    if (g.is3d) {
      kg_to_full<float, true, false><<<nb, kThreads, 0, s>>>(g, x, A.XLe, A.npf, b.czxy, b.cyzx, b.cxyz);
      kg_to_full<float, true, true><<<nb, kThreads, 0, s>>>(g, p, A.UB, A.npf, 0.0, 0.0, 0.0);
    } else {
      kg_to_full<float, false, false><<<nb, kThreads, 0, s>>>(g, x, A.XLe, A.npf, b.czxy, b.cyzx, b.cxyz);
      kg_to_full<float, false, true><<<nb, kThreads, 0, s>>>(g, p, A.UB, A.npf, 0.0, 0.0, 0.0);
    }
    e = product_f32(A, c->tl_on ? &c->tlm : nullptr, c->tl_chunks, s);
    if (e == cudaSuccess) kg_from_full<float><<<nbp, kThreads, 0, s>>>(g, A.Zb[0], A.npf, ap);
  } else {
    GArgs<double> A = make_gargs<double>(c);
    A.fused = 1;
    A.standalone = 1;
    A.poly_deg = 0;
    if (g.is3d) {
      kg_to_full<double, true, false><<<nb, kThreads, 0, s>>>(g, x, A.XLe, A.npf, b.czxy, b.cyzx, b.cxyz);
      kg_to_full<double, true, true><<<nb, kThreads, 0, s>>>(g, p, A.UB, A.npf, 0.0, 0.0, 0.0);
    } else {
      kg_to_full<double, false, false><<<nb, kThreads, 0, s>>>(g, x, A.XLe, A.npf, b.czxy, b.cyzx, b.cxyz);
      kg_to_full<double, false, true><<<nb, kThreads, 0, s>>>(g, p, A.UB, A.npf, 0.0, 0.0, 0.0);
    }
    e = product_f64(A, s);
    if (e == cudaSuccess) kg_from_full<double><<<nbp, kThreads, 0, s>>>(g, A.Zb[0], A.npf, ap);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail(TDGL_ECUDA, std::string("Krylov product launch: ") + cudaGetErrorString(e));
  TDGL_CUDA(cudaMemcpyAsync(&h.status, &c->gdev->status, sizeof(int), cudaMemcpyDeviceToHost, s));
  TDGL_CUDA(cudaStreamSynchronize(s));
  return graph_status(h.status);
}

extern "C" int tdgl_ctx_set_limits(tdgl_ctx* c, int64_t wait_ns, int64_t loop_cap) {
  if (!c) return fail(TDGL_EINVAL, "null context");
  if (c->npend) return fail(TDGL_EINVAL, "a launch of this context has not been collected");
  c->wait_ns = wait_ns > 0 ? (unsigned long long)wait_ns : kWaitDefaultNs;
  c->watchdog_req = loop_cap > 0 ? loop_cap : 0;
  return TDGL_OK;
}

extern "C" int tdgl_arnoldi_probe(tdgl_ctx* c, int32_t ja, int32_t launches, int32_t kernels, tdgl_stream_t s) {
  if (!c || launches < 0) return fail(TDGL_EINVAL, "invalid argument");
  if (c->npend) return fail(TDGL_EINVAL, "a launch of this context has not been collected");
  int rc;
  if ((rc = ensure_graph(c, 1))) return rc;
  if (ja < 0 || ja > c->kmax) return fail(TDGL_EINVAL, "ja must lie in [0, kmax]");
  c->has_clock = false;
  TDGL_CUDA(cudaMemcpyAsync(&c->gdev->ja, &ja, sizeof(int), cudaMemcpyHostToDevice, s));
  // the limit of the device-side waits (a graph launch writes it; the probe
  // may be the context's first launch)
  TDGL_CUDA(cudaMemcpyAsync(&c->gdev->wait_ns, &c->wait_ns, sizeof(c->wait_ns), cudaMemcpyHostToDevice, s));
  if (kernels & 128)                // the Newton update combines ja basis vectors
    TDGL_CUDA(cudaMemcpyAsync(&c->gdev->j, &ja, sizeof(int), cudaMemcpyHostToDevice, s));
  cudaError_t e;
  if (c->precision == TDGL_MIXED) {
    GArgs<float> A = make_gargs<float>(c);
    A.fused = 1;
    A.standalone = 1;
    e = arnoldi_probe_f32(A, c->tl_on ? &c->tlm : nullptr, c->tl_chunks, launches, kernels, s);
  } else {
    GArgs<double> A = make_gargs<double>(c);
    A.fused = 1;
    A.standalone = 1;
    e = arnoldi_probe_f64(A, launches, kernels, s);
  }
  if (e != cudaSuccess) return fail(TDGL_ECUDA, std::string("Arnoldi step launch: ") + cudaGetErrorString(e));
  TDGL_CUDA(cudaStreamSynchronize(s));
  return TDGL_OK;
}

extern "C" int tdgl_profile(tdgl_ctx* c, uint64_t* out, int64_t n, int32_t reset) {
  if (c && c->gprof) {
    for (int64_t k = 0; out && k < std::min<int64_t>(n, 2 * kKTypes); ++k)
      out[k] = k < kKTypes ? c->gk_total[k] : (uint64_t)c->gk_count[k - kKTypes];
    if (reset)
      for (int k = 0; k < kKTypes; ++k) c->gk_total[k] = 0, c->gk_count[k] = 0;
    return TDGL_OK;
  }
  if (!c || !c->prof) return fail(TDGL_EINVAL, "phase timers are off (set TDGL_PROFILE=1 before creating the context)");
  int64_t m = std::min<int64_t>(n, kProfLen);
  if (out && m > 0) TDGL_CUDA(cudaMemcpy(out, c->prof, m * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  if (reset) TDGL_CUDA(cudaMemset(c->prof, 0, kProfLen * sizeof(uint64_t)));
  return TDGL_OK;
}
