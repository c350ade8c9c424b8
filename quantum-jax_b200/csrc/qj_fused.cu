// Instantiations and launchers of the fused single-precision pencil passes.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <mutex>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "../../include/qj.h"
#include "qj_internal.h"

namespace qj {

bool fft_length_supported(int n) {
  return n == 16 || n == 32 || n == 64 || n == 96 || n == 128 || n == 256 || n == 512;
}

template <int N, bool CONTIG>
static int grid_of(const FusedArgs &a) {
  using SH = PassShape<N, CONTIG>;
  if (CONTIG) {
    // a reduced range (half spectrum) rounds up to whole tiles, within the
    // grid; the rows past it are pencils the pass does not store
    const int full = ((a.full_nx > 0 ? a.full_nx : a.nx) * a.ny) / SH::TP;
    return std::min(full, (a.nx * a.ny + SH::TP - 1) / SH::TP);
  }
  return (a.axis == 0 ? a.ny : a.nx) * a.ztiles;
}

// Stage twiddle table of length n (see stage_tw_off), long double, rounded once.
template <int N> static std::vector<float2> stage_table() {
  std::vector<float2> t(stage_tw_size<N>() > 0 ? stage_tw_size<N>() : 1);
  for (int s = 1; s < FftPlan<N>::NS; ++s) {
    const int ns = stage_ns<N>(s), r = FftPlan<N>::radix(s);
    for (int q = 1; q < r; ++q)
      for (int jm = 0; jm < ns; ++jm) {
        const long long m = (long long)jm * q * (N / (ns * r));
        const long double th = -2.0L * 3.14159265358979323846264338327950288L * m / N;
        t[stage_tw_off<N>(s) + jm * tw_row<N>(s) + (q - 1)] = float2{(float)cosl(th), (float)sinl(th)};
      }
  }
  return t;
}

std::vector<float2> stage_twiddles(int n) {
  switch (n) {
    case 16: return stage_table<16>();
    case 32: return stage_table<32>();
    case 64: return stage_table<64>();
    case 96: return stage_table<96>();
    case 128: return stage_table<128>();
    case 256: return stage_table<256>();
    case 512: return stage_table<512>();
  }
  return {};
}

// Tiles (pencil groups of one CTA) of a pass along `axis` of length n_axis.
int pass_blocks(int n_axis, int axis, int nx, int ny, int nz) {
  if (axis == 2) {
    int tp = 1;
    switch (n_axis) {
      case 16: tp = PassShape<16, true>::TP; break;
      case 32: tp = PassShape<32, true>::TP; break;
      case 64: tp = PassShape<64, true>::TP; break;
      case 96: tp = PassShape<96, true>::TP; break;
      case 128: tp = PassShape<128, true>::TP; break;
      case 256: tp = PassShape<256, true>::TP; break;
      case 512: tp = PassShape<512, true>::TP; break;
    }
    return (nx * ny) / tp;
  }
  return (axis == 0 ? ny : nx) * (nz / 16);
}

// CTA slots a persistent pass leaves free for concurrent work on other
// streams, such as the star update and bucket sort that run beside the y
// drift pass (QJ_PERSIST_RESERVE, default 2).
static int reserve_ctas() {
  static int r = -1;
  if (r < 0) {
    const char *env = getenv("QJ_PERSIST_RESERVE");
    r = env ? std::max(0, atoi(env)) : 2;
  }
  return r;
}

// cuTensorMapEncodeTiled from the driver, looked up once.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Tensor maps of a strided pass' streamed fields (see TileMaps).
template <int N, int MODE>
static int strided_maps(const FusedArgs &a, TileMaps &maps) {
  auto enc = tensor_map_encoder();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return QJ_ERR_CUDA;
  }
  const int nbox = a.nbox > 1 ? a.nbox : 1;
  const cuuint64_t dims[4] = {(cuuint64_t)a.nz, (cuuint64_t)a.ny, (cuuint64_t)a.nx, (cuuint64_t)nbox};
  const cuuint64_t strides[3] = {(cuuint64_t)a.nz * 8, (cuuint64_t)a.ny * a.nz * 8,
                                 (cuuint64_t)a.box_cells * 8};
  const cuuint32_t rows = (cuuint32_t)std::min(N, 256);
  const cuuint32_t box[4] = {16, a.axis == 0 ? 1u : rows, a.axis == 0 ? rows : 1u, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  for (int f = 0; f < stream_count<MODE>(); ++f) {
    const CUresult r = enc(&maps.m[f], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
                           const_cast<float2 *>(stream_field<MODE>(a, f)), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      set_error("cuTensorMapEncodeTiled failed (%d) for a %dx%dx%d pass along axis %d", (int)r, a.nx,
                a.ny, a.nz, a.axis);
      return QJ_ERR_CUDA;
    }
  }
  return 0;
}

// Resident CTAs per SM of a pass (occupancy) and the SM count, queried once
// per device (the shared-memory attribute belongs to that device's context).
struct Occupancy {
  cudaError_t err = cudaSuccess;
  int per_sm = 1, sms = 1;
};
template <int N, bool CONTIG, int MODE>
static cudaError_t fused_occupancy(int &per_sm, int &sms) {
  using SH = PassShape<N, CONTIG>;
  static PerDevice<Occupancy> cache;
  const Occupancy *o = nullptr;
  const cudaError_t e = per_device(cache, o, [](Occupancy &r) {
    const size_t smem = fused_smem_bytes<N, CONTIG, MODE>();
    r.err = cudaFuncSetAttribute(k_fused<N, CONTIG, MODE>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int dev = 0, n_sm = 0, p = 0;
    if (r.err == cudaSuccess) r.err = cudaGetDevice(&dev);
    if (r.err == cudaSuccess) r.err = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (r.err == cudaSuccess)
      r.err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, k_fused<N, CONTIG, MODE>, SH::THREADS,
                                                            smem);
    r.per_sm = std::max(1, p);
    r.sms = std::max(1, n_sm);
  });
  if (e != cudaSuccess) return e;
  per_sm = o->per_sm;
  sms = o->sms;
  return o->err;
}

template <int N, bool CONTIG, int MODE>
static int run_fused(const FusedArgs &a, cudaStream_t st) {
  using SH = PassShape<N, CONTIG>;
  const size_t smem = fused_smem_bytes<N, CONTIG, MODE>();
  // persistent grid: the CTAs resident at once (occupancy x SMs), shared
  // between the boxes of a batched launch
  int per_sm = 0, sms = 0;
  const cudaError_t occ = fused_occupancy<N, CONTIG, MODE>(per_sm, sms);
  QJ_CK(occ);
  const int want = a.tune ? a.tune[MODE] : 0;
  const int resident = (want > 0 ? std::min(want, per_sm) : per_sm) * sms;
  const int reserve = (a.tune && a.tune[8] >= 0) ? a.tune[8] : reserve_ctas();
  // the bulk tile copies need 16-byte aligned fields
  const void *fields[4] = {a.psi, a.R, a.S1, a.S2};
  for (const void *f : fields)
    if ((reinterpret_cast<uintptr_t>(f) & 15) != 0) {
      set_error("fields of the fused passes must be 16-byte aligned");
      return QJ_ERR_ARG;
    }
  FusedArgs b = a;
  b.ntiles = grid_of<N, CONTIG>(a);
  // y passes walk backwards: each follows (and precedes) a pass that walks
  // forwards over the same slow index x
  b.rev = (!CONTIG && a.axis == 1) ? 1 : 0;
  TileMaps maps;
  std::memset(&maps, 0, sizeof(maps));
  if (!CONTIG && stream_count<MODE>() > 0) {
    const int rc = strided_maps<N, MODE>(b, maps);
    if (rc) return rc;
  }
  const int nbox = a.nbox > 1 ? a.nbox : 1;
  const int gx = std::max(1, std::min(b.ntiles, (resident - reserve) / nbox));
  const dim3 grid(gx, nbox);
  k_fused<N, CONTIG, MODE><<<grid, SH::THREADS, smem, st>>>(b, maps);
  QJ_CK_LAUNCH();
  return 0;
}

// The y-only transforms are instantiated strided; the others for both the
// strided x or y pass and the contiguous z pass (the plain drift runs along
// every axis in the adjoint's reverse sweep).
template <int MODE>
static int dispatch_mode(int n, const FusedArgs &a, cudaStream_t st) {
  constexpr bool ONLY_Y = (MODE == M_FFT_FWD || MODE == M_IFFT2);
  const bool contig = a.axis == 2;
  if (ONLY_Y && contig) {
    set_error("internal: pass mode %d requested along z", MODE);
    return 1;
  }
#define QJ_CASE(NN)                                                    \
  case NN:                                                             \
    if constexpr (ONLY_Y) return run_fused<NN, false, MODE>(a, st);    \
    else return contig ? run_fused<NN, true, MODE>(a, st) : run_fused<NN, false, MODE>(a, st);
  switch (n) {
    QJ_CASE(16)
    QJ_CASE(32)
    QJ_CASE(64)
    QJ_CASE(96)
    QJ_CASE(128)
    QJ_CASE(256)
    QJ_CASE(512)
  }
#undef QJ_CASE
  set_error("unsupported FFT length %d", n);
  return 1;
}

// The dense deposit runs along z only.
static int dispatch_deposit(int n, const FusedArgs &a, cudaStream_t st) {
  if (a.axis != 2) {
    set_error("internal: deposit pass must run along z");
    return 1;
  }
  switch (n) {
    case 16: return run_fused<16, true, M_DEPOSIT>(a, st);
    case 32: return run_fused<32, true, M_DEPOSIT>(a, st);
    case 64: return run_fused<64, true, M_DEPOSIT>(a, st);
    case 96: return run_fused<96, true, M_DEPOSIT>(a, st);
    case 128: return run_fused<128, true, M_DEPOSIT>(a, st);
    case 256: return run_fused<256, true, M_DEPOSIT>(a, st);
    case 512: return run_fused<512, true, M_DEPOSIT>(a, st);
  }
  set_error("unsupported FFT length %d", n);
  return 1;
}

static int launch_fused_impl(int mode, int n, const FusedArgs &a, cudaStream_t st) {
  switch (mode) {
    case M_DENSITY: return dispatch_mode<M_DENSITY>(n, a, st);
    case M_FFT_FWD: return dispatch_mode<M_FFT_FWD>(n, a, st);
    case M_POISSON: return dispatch_mode<M_POISSON>(n, a, st);
    case M_IFFT2: return dispatch_mode<M_IFFT2>(n, a, st);
    case M_KICK: return dispatch_mode<M_KICK>(n, a, st);
    case M_DRIFT: return dispatch_mode<M_DRIFT>(n, a, st);
    case M_DRIFT_DENSITY: return dispatch_mode<M_DRIFT_DENSITY>(n, a, st);
    case M_DEPOSIT: return dispatch_deposit(n, a, st);
  }
  set_error("internal: bad pass mode %d", mode);
  return 1;
}

template <int MODE> static int occupancy_of(int n, bool contig) {
  int per_sm = 0, sms = 0;
  cudaError_t e = cudaSuccess;
  constexpr bool ONLY_Y = (MODE == M_FFT_FWD || MODE == M_IFFT2);
  constexpr bool ONLY_Z = (MODE == M_DEPOSIT);
#define QJ_OCC(NN)                                                                          \
  case NN:                                                                                  \
    if constexpr (ONLY_Y) e = fused_occupancy<NN, false, MODE>(per_sm, sms);                \
    else if constexpr (ONLY_Z) e = fused_occupancy<NN, true, MODE>(per_sm, sms);            \
    else e = contig ? fused_occupancy<NN, true, MODE>(per_sm, sms)                          \
                    : fused_occupancy<NN, false, MODE>(per_sm, sms);                        \
    break;
  switch (n) {
    QJ_OCC(16)
    QJ_OCC(32)
    QJ_OCC(64)
    QJ_OCC(96)
    QJ_OCC(128)
    QJ_OCC(256)
    QJ_OCC(512)
    default: return 0;
  }
#undef QJ_OCC
  return e == cudaSuccess ? per_sm : 0;
}

int fused_max_ctas_per_sm(int mode, int n, bool contig) {
  switch (mode) {
    case M_DENSITY: return occupancy_of<M_DENSITY>(n, contig);
    case M_FFT_FWD: return occupancy_of<M_FFT_FWD>(n, contig);
    case M_POISSON: return occupancy_of<M_POISSON>(n, contig);
    case M_IFFT2: return occupancy_of<M_IFFT2>(n, contig);
    case M_KICK: return occupancy_of<M_KICK>(n, contig);
    case M_DRIFT: return occupancy_of<M_DRIFT>(n, contig);
    case M_DRIFT_DENSITY: return occupancy_of<M_DRIFT_DENSITY>(n, contig);
    case M_DEPOSIT: return occupancy_of<M_DEPOSIT>(n, contig);
  }
  return 0;
}

// Self-test of the bounded wait and its error report: one warp arms an
// mbarrier for 16 bytes that no copy brings, waits for it with the fused
// passes' bounded wait (limit_ns) and, when the wait gives up, sets bit 2 of
// the error word.  No copy is in flight, so giving up is safe.
__global__ void k_selftest_wait(unsigned *err, unsigned long long limit_ns) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_expect_tx(&bar, 16);
  }
  __syncthreads();
  const bool ok = __syncthreads_and(mbar_wait_bounded(&bar, 0, limit_ns));
  if (!ok && threadIdx.x == 0) atomicOr(err, 2u);
}

int launch_selftest_wait(unsigned *err, long long limit_ns, cudaStream_t st) {
  k_selftest_wait<<<1, 32, 0, st>>>(err, (unsigned long long)limit_ns);
  QJ_CK_LAUNCH();
  return 0;
}

// The kick pass's sin / cos of a float64 phase, one value per thread, for a
// direct accuracy test of sincos_reduced.
__global__ void k_selftest_sincos(const double *theta, float2 *out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    float s, c;
    sincos_reduced(theta[i], s, c);
    out[i] = float2{s, c};
  }
}

int launch_selftest_sincos(const double *theta, float2 *out, int n, cudaStream_t st) {
  k_selftest_sincos<<<(n + 255) / 256, 256, 0, st>>>(theta, out, n);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_fused(int mode, int n, const FusedArgs &a, cudaStream_t st) {
  const bool prof = prof_on();
  if (prof) prof_mark_begin(st);
  const int rc = launch_fused_impl(mode, n, a, st);
  if (prof && rc == 0) prof_mark_end(mode, st);
  return rc;
}

}  // namespace qj
