// tdgl_eval_f_noalloc: the right-hand side of a grid, computed without
// allocating memory.
//
// Who needs this: code that must not allocate device memory when it runs --
// for example a loop with a fixed device-memory budget, a process whose
// device memory is owned entirely by another allocator, or a caller that
// cannot afford the implicit synchronisation of cudaMalloc / cudaFree.  A
// tdgl_ctx allocates its geometry and scratch at creation; this entry point
// takes the same descriptors as tdgl_ctx_create, derives everything on the
// device, and keeps every intermediate in one fixed static device array.
//
// The scratch array (kNoallocBytes, about 8.6 MiB) lives in this library's
// module: every GPU that loads the library holds it until the process exits.
// Limits: at most kMaxNodes interior nodes, kMaxFull full-grid nodes and
// kMaxLinks entries per hole list; larger inputs are rejected with
// TDGL_EINVAL before any device work.  Calls share the array and each call
// overwrites what it uses, so calls that overlap on the GPU (different
// streams, or different host threads) race and must be serialised by the
// caller.  The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) and keeps it for the life of the process; make that
// first call before any stream capture, and do not call the entry point again
// after cudaDeviceReset (the kept address would be stale).  The material
// descriptor's arrays are host memory copied on every call, so a call that
// has any is refused while its stream is capturing.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "tdgl_b200.h"
#include "tdgl_common.cuh"

namespace tdgl {
int report_error(int code, const std::string& msg);   // tdgl_capi.cu: sets tdgl_last_error()

namespace {

constexpr long kMaxNodes = 32768;              // interior nodes
constexpr long kMaxFull = 262144;              // full-grid nodes
constexpr long kMaxLinks = 65536;              // entries of each hole list
// byte offsets of the regions of the scratch array
constexpr size_t kOffX = 0;                                            // device-layout state, 5 x kMaxNodes doubles
constexpr size_t kOffF = kOffX + 5 * kMaxNodes * sizeof(double);       // device-layout RHS
constexpr size_t kOffK2 = kOffF + 5 * kMaxNodes * sizeof(double);      // kappa^2 per interior node
constexpr size_t kOffSc = kOffK2 + kMaxNodes * sizeof(double);         // sc per interior node (reference order)
constexpr size_t kOffScD = kOffSc + kMaxNodes * sizeof(double);        // sc per interior node (device order)
constexpr size_t kOffKf = kOffScD + kMaxNodes * sizeof(double);        // kappa on the full grid
constexpr size_t kOffHl = kOffKf + kMaxFull * sizeof(double);          // hole link lists, 3 x kMaxLinks int64
constexpr size_t kOffHi = kOffHl + 3 * kMaxLinks * sizeof(int64_t);    // hole interior lists, 3 x kMaxLinks int64
constexpr size_t kOffNf = kOffHi + 3 * kMaxLinks * sizeof(int64_t);    // node flags
constexpr size_t kOffLf = kOffNf + kMaxNodes;                          // link flags
constexpr size_t kNoallocBytes = kOffLf + kMaxFull;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

constexpr int kMaxDevices = 128;
std::mutex g_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// failures are reported through tdgl_last_error()
int err(int code, const std::string& m) { return report_error(code, m); }

// Device address of the scratch array on the current device (looked up once per device).
int scratch_address(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return err(TDGL_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return err(TDGL_EINVAL, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return err(TDGL_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_ptr[dev];
  return TDGL_OK;
}

__device__ __forceinline__ int nref_index(const Grid& g, int d) {
  int i, j, k;
  node_ijk(g, d, i, j, k);
  return ((i - 1) * g.ny + (j - 1)) * g.nz + (g.is3d ? k - 1 : 0);
}

__global__ void kn_zero_bytes(unsigned char* p, long n) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) p[t] = 0;
}

// Hole-boundary links of one axis (all writes of one launch set the same bit).
__global__ void kn_mark_links(unsigned char* lf, const int64_t* links, long count, unsigned char bit) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < count; t += (long)gridDim.x * blockDim.x)
    lf[links[t]] |= bit;
}

// Node flags: slow-path neighbourhood, superconducting fraction class; per-node
// kappa^2 and sc in device order.
__global__ void kn_node_flags(Grid g, const unsigned char* lf, unsigned char* nf, const double* kappa_full,
                              double* k2, const double* sc_ref, double* sc_dev) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    int i, j, k;
    node_ijk(g, d, i, j, k);
    const bool d3 = g.is3d;
    bool slow = i < 2 || i > g.Nx - 3 || j < 2 || j > g.Ny - 3 || (d3 && (k < 2 || k > g.Nz - 3));
    if (!slow && lf) {
      for (int dk = (d3 ? -1 : 0); dk <= (d3 ? 1 : 0) && !slow; ++dk)
        for (int dj = -1; dj <= 1 && !slow; ++dj)
          for (int di = -1; di <= 1 && !slow; ++di)
            if (lf[(i + di) + (long)g.mj * (j + dj) + (long)g.mk * (k + dk)]) slow = true;
    }
    unsigned char f = slow ? NF_SLOW : 0;
    if (sc_ref) {
      double s = sc_ref[nref_index(g, d)];
      sc_dev[d] = s;
      if (s == 0.0) f |= NF_SC0;
      else if (s != 1.0) f |= NF_SCFRAC;
    }
    if (kappa_full) {
      double kv = kappa_full[i + (long)g.mj * j + (long)g.mk * k];
      k2[d] = kv * kv;
    }
    nf[d] = f;
  }
}

// d(phi)/dt := 0 flags of one axis from its interior list (reference numbering).
__global__ void kn_mark_interior(Grid g, unsigned char* nf, const int64_t* idx, long count, unsigned char bit) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < count; t += (long)gridDim.x * blockDim.x) {
    long r = idx[t];
    long kk = r % g.nz, q = r / g.nz;
    long jj = q % g.ny + 1, ii = q / g.ny + 1;
    long d = (ii - 1) + (long)g.nx * ((jj - 1) + (long)g.ny * (g.is3d ? kk : 0));
    nf[d] |= bit;
  }
}

__global__ void kn_pack(Grid g, const double2* __restrict__ xref, double* xdev) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    int r = nref_index(g, d);
    double2 p = xref[r];
    xdev[d] = p.x;
    xdev[(long)g.npad + d] = p.y;
    for (int a = 0; a < g.ncomp - 2; ++a) xdev[(long)(2 + a) * g.npad + d] = xref[(long)(a + 1) * g.n + r].x;
  }
}

__global__ void kn_rhs(Grid g, const double* x, double* f, BTerms<double> b) {
  SrcVec<double, double> sx{x, g.npad};
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    double o[5];
    rhs_at<double>(g, sx, b, d, o);
    for (int c = 0; c < g.ncomp; ++c) f[(long)c * g.npad + d] = o[c];
  }
}

__global__ void kn_unpack(Grid g, const double* fdev, double2* __restrict__ fref) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < g.n; d += gridDim.x * blockDim.x) {
    int r = nref_index(g, d);
    fref[r] = make_double2(fdev[d], fdev[(long)g.npad + d]);
    for (int a = 0; a < g.ncomp - 2; ++a)
      fref[(long)(a + 1) * g.n + r] = make_double2(fdev[(long)(2 + a) * g.npad + d], 0.0);
  }
}

}  // namespace
}  // namespace tdgl

using namespace tdgl;

extern "C" int tdgl_eval_f_noalloc(const tdgl_grid_desc* gd, const tdgl_material_desc* md, const double* x_ref,
                                   double* f_ref, double Bx, double By, double Bz, tdgl_stream_t stream) {
  if (!gd || !x_ref || !f_ref) return err(TDGL_EINVAL, "null argument");
  if (gd->Nx < 2 || gd->Ny < 2) return err(TDGL_EINVAL, "Nx and Ny must each be >= 2.");
  if (gd->Nz < 1) return err(TDGL_EINVAL, "Nz must be >= 1.");
  const long Nx = gd->Nx, Ny = gd->Ny, Nz = gd->Nz;
  const bool d3 = Nz > 1;
  const long nx = Nx - 1, ny = Ny - 1, nz = d3 ? Nz - 1 : 1;
  const long n = nx * ny * nz;
  const long mj = Nx + 1, mk = (Nx + 1) * (Ny + 1);
  const long dimx = d3 ? mk * (Nz + 1) : mk;
  if (n > kMaxNodes)
    return err(TDGL_EINVAL, "tdgl_eval_f_noalloc handles at most " + std::to_string(kMaxNodes) +
                                " interior nodes; this grid has " + std::to_string(n));
  if (dimx > kMaxFull)
    return err(TDGL_EINVAL, "tdgl_eval_f_noalloc handles at most " + std::to_string(kMaxFull) +
                                " full-grid nodes; this grid has " + std::to_string(dimx));
  for (int a = 0; a < (d3 ? 3 : 2); ++a) {      // the axes build_geometry reads (z only in 3-D)
    if (!md) break;
    if (md->n_hole_links[a] > kMaxLinks || md->n_hole_interior[a] > kMaxLinks)
      return err(TDGL_EINVAL, "tdgl_eval_f_noalloc takes at most " + std::to_string(kMaxLinks) +
                                  " entries per hole list");
    for (int64_t t = 0; t < md->n_hole_links[a]; ++t)
      if (md->hole_links[a][t] < 0 || md->hole_links[a][t] >= dimx) return err(TDGL_EINVAL, "hole link index out of range");
    for (int64_t t = 0; t < md->n_hole_interior[a]; ++t)
      if (md->hole_interior[a][t] < 0 || md->hole_interior[a][t] >= n)
        return err(TDGL_EINVAL, "hole interior index out of range");
  }
  bool host_arrays = md && (md->kappa_full || md->sc_interior);
  for (int a = 0; md && a < (d3 ? 3 : 2); ++a)
    host_arrays = host_arrays || md->n_hole_links[a] > 0 || md->n_hole_interior[a] > 0;
  if (host_arrays) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t ce = cudaStreamIsCapturing(stream, &cs);
    if (ce != cudaSuccess) return err(TDGL_ECUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(ce));
    if (cs != cudaStreamCaptureStatusNone)
      return err(TDGL_EINVAL, "tdgl_eval_f_noalloc copies the material descriptor's host arrays on every call; "
                              "such a call cannot be made while the stream is capturing");
  }
  unsigned char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;

  Grid g{};
  g.Nx = (int)Nx; g.Ny = (int)Ny; g.Nz = (int)Nz;
  g.nx = (int)nx; g.ny = (int)ny; g.nz = (int)nz;
  g.is3d = d3;
  g.px = gd->periodic_x != 0; g.py = gd->periodic_y != 0; g.pz = gd->periodic_z != 0;
  g.n = (int)n;
  g.npad = (int)((n + 127) / 128 * 128);
  g.ncomp = d3 ? 5 : 4;
  g.mj = (int)mj; g.mk = (int)mk;
  g.hx = gd->hx; g.hy = gd->hy; g.hz = gd->hz;
  g.ihx2 = 1.0 / (gd->hx * gd->hx);
  g.ihy2 = 1.0 / (gd->hy * gd->hy);
  g.ihz2 = 1.0 / (gd->hz * gd->hz);
  g.hx2 = gd->hx * gd->hx; g.hy2 = gd->hy * gd->hy; g.hz2 = gd->hz * gd->hz;
  g.kappa2 = gd->kappa * gd->kappa;

  cudaStream_t s = stream;
  double* X = reinterpret_cast<double*>(base + kOffX);
  double* F = reinterpret_cast<double*>(base + kOffF);
  double* K2 = reinterpret_cast<double*>(base + kOffK2);
  double* SC = reinterpret_cast<double*>(base + kOffSc);
  double* SCD = reinterpret_cast<double*>(base + kOffScD);
  double* KF = reinterpret_cast<double*>(base + kOffKf);
  int64_t* HL = reinterpret_cast<int64_t*>(base + kOffHl);
  int64_t* HI = reinterpret_cast<int64_t*>(base + kOffHi);
  unsigned char* NF = base + kOffNf;
  unsigned char* LF = base + kOffLf;
  const int threads = kThreads;
  auto blocks = [&](long work) { return (int)std::max(1L, std::min((work + threads - 1) / threads, 4096L)); };
#define TDGL_NCK(call)                                                                        \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return err(TDGL_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

  // link flags: cleared every call (the array keeps the previous call's contents)
  bool any_hole = false;
  if (md) {
    for (int a = 0; a < (d3 ? 3 : 2); ++a) any_hole = any_hole || md->n_hole_links[a] > 0;
  }
  if (any_hole) {
    kn_zero_bytes<<<blocks(dimx), threads, 0, s>>>(LF, dimx);
    for (int a = 0; a < (d3 ? 3 : 2); ++a) {
      long cnt = md->n_hole_links[a];
      if (cnt <= 0) continue;
      TDGL_NCK(cudaMemcpyAsync(HL + (long)a * kMaxLinks, md->hole_links[a], cnt * sizeof(int64_t),
                               cudaMemcpyHostToDevice, s));
      kn_mark_links<<<blocks(cnt), threads, 0, s>>>(LF, HL + (long)a * kMaxLinks, cnt, (unsigned char)(1u << a));
    }
  }
  const bool has_kappa = md && md->kappa_full;
  const bool has_sc = md && md->sc_interior;
  if (has_kappa) TDGL_NCK(cudaMemcpyAsync(KF, md->kappa_full, dimx * sizeof(double), cudaMemcpyHostToDevice, s));
  if (has_sc) TDGL_NCK(cudaMemcpyAsync(SC, md->sc_interior, n * sizeof(double), cudaMemcpyHostToDevice, s));
  kn_node_flags<<<blocks(n), threads, 0, s>>>(g, any_hole ? LF : nullptr, NF, has_kappa ? KF : nullptr, K2,
                                              has_sc ? SC : nullptr, SCD);
  if (md) {
    for (int a = 0; a < (d3 ? 3 : 2); ++a) {
      long cnt = md->n_hole_interior[a];
      if (cnt <= 0) continue;
      TDGL_NCK(cudaMemcpyAsync(HI + (long)a * kMaxLinks, md->hole_interior[a], cnt * sizeof(int64_t),
                               cudaMemcpyHostToDevice, s));
      kn_mark_interior<<<blocks(cnt), threads, 0, s>>>(g, NF, HI + (long)a * kMaxLinks, cnt,
                                                       (unsigned char)(NF_HOLEX << a));
    }
  }
  g.nflags = NF;
  g.lflags = any_hole ? LF : nullptr;
  g.kappa_per_node = has_kappa ? 1 : 0;
  g.k2int = has_kappa ? K2 : nullptr;
  g.has_material = has_sc ? 1 : 0;
  g.scint = has_sc ? SCD : nullptr;
  BTerms<double> b{Bz * g.hx * g.hy, By * g.hz * g.hx, Bx * g.hy * g.hz};
  kn_pack<<<blocks(n), threads, 0, s>>>(g, reinterpret_cast<const double2*>(x_ref), X);
  kn_rhs<<<blocks(n), threads, 0, s>>>(g, X, F, b);
  kn_unpack<<<blocks(n), threads, 0, s>>>(g, F, reinterpret_cast<double2*>(f_ref));
  TDGL_NCK(cudaGetLastError());
#undef TDGL_NCK
  return TDGL_OK;
}

