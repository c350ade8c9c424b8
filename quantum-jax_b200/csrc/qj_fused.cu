// Instantiations and launchers of the fused single-precision pencil passes.
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "qj_internal.h"

namespace qj {

bool fft_length_supported(int n) {
  return n == 16 || n == 32 || n == 64 || n == 96 || n == 128 || n == 256 || n == 512;
}

template <int N, bool CONTIG>
static int grid_of(const FusedArgs &a) {
  using SH = PassShape<N, CONTIG>;
  if (CONTIG) return (a.nx * a.ny) / SH::TP;
  return (a.axis == 0 ? a.ny : a.nx) * (a.nz / 16);
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
        t[stage_tw_off<N>(s) + (q - 1) * ns + jm] = float2{(float)cosl(th), (float)sinl(th)};
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

int pass_blocks(int n_axis, int axis, int nx, int ny, int nz) {
  if (axis == 2) {
    const int E = (n_axis == 32 || n_axis == 64) ? 8 : (n_axis == 96 ? 12 : 16);
    const int P = n_axis / E;
    const int TP = P >= 256 ? 1 : 256 / P;
    return (nx * ny) / TP;
  }
  return (axis == 0 ? ny : nx) * (nz / 16);
}

template <int N, bool CONTIG, int MODE>
static int run_fused(const FusedArgs &a, cudaStream_t st) {
  using SH = PassShape<N, CONTIG>;
  const size_t smem = fused_smem_bytes<N, CONTIG, MODE>();
  static std::once_flag once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(once, [&] {
    attr_err = cudaFuncSetAttribute(k_fused<N, CONTIG, MODE>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  QJ_CK(attr_err);
  // L2 prefetch distance: the CTAs resident at once (occupancy x SMs) times
  // QJ_L2_PREFETCH_WAVES (default 0 = off).
  static int ahead = -1;
  if (ahead < 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused<N, CONTIG, MODE>, SH::THREADS, smem);
    const char *env = getenv("QJ_L2_PREFETCH_WAVES");
    const int waves = env ? atoi(env) : 0;
    ahead = waves > 0 ? waves * sms * (per_sm > 0 ? per_sm : 1) : 0;
  }
  FusedArgs b = a;
  b.ahead = ahead;
  const dim3 grid(grid_of<N, CONTIG>(a), a.nbox > 1 ? a.nbox : 1);
  k_fused<N, CONTIG, MODE><<<grid, SH::THREADS, smem, st>>>(b);
  QJ_CK_LAUNCH();
  return 0;
}

// Modes used along y (axis 1) are only instantiated strided; the others for
// both the strided x pass and the contiguous z pass.
template <int MODE>
static int dispatch_mode(int n, const FusedArgs &a, cudaStream_t st) {
  constexpr bool ONLY_Y = (MODE == M_FFT_FWD || MODE == M_IFFT2 || MODE == M_DRIFT);
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

int launch_fused(int mode, int n, const FusedArgs &a, cudaStream_t st) {
  const bool prof = prof_on();
  if (prof) prof_mark_begin(st);
  const int rc = launch_fused_impl(mode, n, a, st);
  if (prof && rc == 0) prof_mark_end(mode, st);
  return rc;
}

}  // namespace qj
