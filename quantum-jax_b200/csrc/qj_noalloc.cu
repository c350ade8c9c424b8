// get_potential in single precision without any device allocation.
//
// Some callers cannot let a library call cudaMalloc: a JAX / XLA FFI handler
// runs inside XLA's memory manager (XLA reserves most of the device memory up
// front, so a private cudaMalloc can fail, and cudaMalloc / cudaFree also
// synchronise the device in the middle of XLA's asynchronous schedule), and
// hosts with a fixed memory budget allocate everything once at start-up.
// qj_get_potential_f32_noalloc serves them: its scratch (the complex work
// field, the twiddle and k tables) lives in one file-scope __device__ array of
// fixed size, reserved on every GPU that loads libqj until the process exits.
//
// Limits: each axis 16, 32 or 64 cells, nz a multiple of 16, at most 64^3
// cells.  All calls on a device share the array, so two calls that overlap on
// the GPU (different streams, no ordering between them) race and give wrong
// results; calls on one stream are ordered and safe.  Nothing in the array
// needs to start at zero: every call rewrites the tables and every cell of
// the work field before reading them.
#include <cmath>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "../../include/qj.h"
#include "qj_internal.h"

namespace qj {

namespace {

constexpr int kMaxAxis = QJ_NOALLOC_MAX_AXIS;
constexpr long long kMaxCells = QJ_NOALLOC_MAX_CELLS;
// layout: work field | twiddles[3][kMaxAxis] | k[3][kMaxAxis]
constexpr size_t kWorkBytes = (size_t)kMaxCells * sizeof(float2);
constexpr size_t kTwBytes = 3 * kMaxAxis * sizeof(float2);
constexpr size_t kKBytes = 3 * kMaxAxis * sizeof(float);
constexpr size_t kScratchBytes = kWorkBytes + kTwBytes + kKBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of the scratch array on each device, looked up on the first
// call with that device current and cached with the id of the context it
// belongs to.  A later call in another context of the same device (after
// cudaDeviceReset, which unloads the module and frees the array) looks the
// address up again instead of handing out the old one.
struct ScratchAddr {
  unsigned long long ctx_id = 0;
  void *addr = nullptr;
};
std::mutex g_mu;
ScratchAddr g_addr[kMaxDevices];

// cuCtxGetCurrent and cuCtxGetId from the driver, looked up once.
struct CtxFns {
  PFN_cuCtxGetCurrent_v4000 current = nullptr;
  PFN_cuCtxGetId_v12000 id = nullptr;
};
const CtxFns &ctx_fns() {
  static CtxFns f;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      f.current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      f.id = reinterpret_cast<PFN_cuCtxGetId_v12000>(p);
  });
  return f;
}

// Id of the calling thread's current context, 0 if none or unknown.
unsigned long long current_ctx_id() {
  const CtxFns &f = ctx_fns();
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (f.current && f.id && f.current(&c) == CUDA_SUCCESS && c && f.id(c, &id) == CUDA_SUCCESS)
    return id;
  return 0;
}

int scratch_address(void **out) {
  int dev = 0;
  QJ_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("qj_get_potential_f32_noalloc: device ordinal %d out of range", dev);
    return QJ_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  ScratchAddr &s = g_addr[dev];
  const unsigned long long id = current_ctx_id();
  if (!s.addr || id == 0 || id != s.ctx_id) {
    void *p = nullptr;
    QJ_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    s.addr = p;
    s.ctx_id = current_ctx_id();  // the lookup made the device's context current
  }
  *out = s.addr;
  return 0;
}

// twiddles w[m] = exp(-2 pi i m / n) and k[i] = 2 pi / L * (i < n/2 ? i : i - n)
__global__ void k_noalloc_tables(float2 *tw, float *k, int nx, int ny, int nz, double Lx,
                                 double Ly, double Lz) {
  const int i = threadIdx.x;
  const int n[3] = {nx, ny, nz};
  const double L[3] = {Lx, Ly, Lz};
  for (int a = 0; a < 3; ++a) {
    if (i < n[a]) {
      double s, c;
      sincospi(-2.0 * i / n[a], &s, &c);
      tw[a * kMaxAxis + i] = float2{(float)c, (float)s};
      const int m = i < n[a] / 2 ? i : i - n[a];
      k[a * kMaxAxis + i] = (float)(2.0 * M_PI / L[a] * m);
    }
  }
}

}  // namespace
}  // namespace qj

using namespace qj;

extern "C" int qj_get_potential_f32_noalloc(const qj_grid *grid, const qj_phys *phys,
                                            const float *rho, float *V, int self_interaction,
                                            void *stream) {
  if (!grid || !phys || !rho || !V) {
    set_error("qj_get_potential_f32_noalloc: null argument");
    return QJ_ERR_ARG;
  }
  const int n[3] = {grid->nx, grid->ny, grid->nz};
  for (int a = 0; a < 3; ++a) {
    if (n[a] != 16 && n[a] != 32 && n[a] != 64) {
      set_error("qj_get_potential_f32_noalloc: axis %d length %d; this entry point supports "
                "16, 32 or 64 cells per axis (at most %lld cells)", a, n[a], (long long)kMaxCells);
      return QJ_ERR_ARG;
    }
  }
  if (!(grid->Lx > 0 && grid->Ly > 0 && grid->Lz > 0)) {
    set_error("qj_get_potential_f32_noalloc: box lengths must be positive");
    return QJ_ERR_ARG;
  }
  const long long ncell = (long long)n[0] * n[1] * n[2];
  cudaStream_t st = (cudaStream_t)stream;
  void *base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  unsigned char *b = (unsigned char *)base;
  float2 *work = (float2 *)b;
  float2 *tw = (float2 *)(b + kWorkBytes);
  float *k = (float *)(b + kWorkBytes + kTwBytes);

  k_noalloc_tables<<<1, kMaxAxis, 0, st>>>(tw, k, n[0], n[1], n[2], grid->Lx, grid->Ly, grid->Lz);
  QJ_CK_LAUNCH();
  // cbuf = 4 pi G (rho - rho_bar), then fftn, -1 / (k^2 + [k^2 == 0]), ifftn,
  // real part (+ b_coeff rho): quantum-stars.py:189-193.
  if ((rc = launch_build_rho(false, nullptr, nullptr, nullptr, rho, 4.0 * M_PI * phys->G,
                             phys->rho_bar, nullptr, work, ncell, st)))
    return rc;
  for (int dir = -1; dir <= 1; dir += 2) {
    for (int axis = 2; axis >= 0; --axis) {
      FftArgs a;
      a.nx = n[0];
      a.ny = n[1];
      a.nz = n[2];
      a.axis = axis;
      a.stride = axis == 0 ? (long long)n[1] * n[2] : (axis == 1 ? n[2] : 1);
      a.outer_stride = axis == 0 ? n[2] : (long long)n[1] * n[2];
      a.ztiles = n[2] / 16;
      a.data = work;
      a.tw = tw + axis * kMaxAxis;
      a.scale = dir > 0 ? 1.0 / n[axis] : 1.0;
      if ((rc = launch_fft(false, n[axis], dir, a, st))) return rc;
    }
    if (dir < 0) {
      KTabs kt;
      for (int d = 0; d < 3; ++d) {
        kt.k[d] = k + d * kMaxAxis;
        kt.n[d] = n[d];
      }
      if ((rc = launch_poisson_div(false, work, kt, ncell, st))) return rc;
    }
  }
  return launch_real_part(false, work, 1.0, self_interaction ? rho : nullptr, phys->b_coeff,
                          nullptr, V, ncell, st);
}
