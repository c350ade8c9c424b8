// Instantiations and launchers of the fused single-precision pencil passes
// (default shapes of every length; the shape variants of n = 128 and 256 are
// instantiated by qj_fused_v{1,2,3}.cu).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "qj_fused_run.cuh"

namespace qj {

bool fft_length_supported(int n) {
  return n == 16 || n == 32 || n == 64 || n == 96 || n == 128 || n == 256 || n == 512;
}

// Stage twiddle table of length n and radix plan RV (see stage_tw_off), long
// double, rounded once.
template <int N, int RV> static std::vector<float2> stage_table() {
  using PL = FftPlan<N, RV>;
  std::vector<float2> t(stage_tw_size<N, RV>() > 0 ? stage_tw_size<N, RV>() : 1);
  for (int s = 1; s < PL::NS; ++s) {
    const int ns = stage_ns<N, RV>(s), r = PL::radix(s);
    for (int q = 1; q < r; ++q)
      for (int jm = 0; jm < ns; ++jm) {
        const long long m = (long long)jm * q * (N / (ns * r));
        const long double th = -2.0L * 3.14159265358979323846264338327950288L * m / N;
        t[stage_tw_off<N, RV>(s) + jm * tw_row<N, RV>(s) + (q - 1)] =
            float2{(float)cosl(th), (float)sinl(th)};
      }
  }
  return t;
}

std::vector<float2> stage_twiddles(int n, int rv) {
  if (rv) {
    switch (n) {
      case 128: return stage_table<128, 1>();
      case 256: return stage_table<256, 1>();
    }
    return {};
  }
  switch (n) {
    case 16: return stage_table<16, 0>();
    case 32: return stage_table<32, 0>();
    case 64: return stage_table<64, 0>();
    case 96: return stage_table<96, 0>();
    case 128: return stage_table<128, 0>();
    case 256: return stage_table<256, 0>();
    case 512: return stage_table<512, 0>();
  }
  return {};
}

template <int N, int V> static int contig_tp() { return PassShape<N, true, V>::TP; }

int strided_tile_width(int v) {
  return (v & 2) ? PassShape<256, false, 2>::TP : PassShape<256, false, 0>::TP;
}

// Tiles (pencil groups of one CTA) of a pass along `axis` of length n_axis in
// shape variant v (0 for lengths without variants).
int pass_blocks(int n_axis, int axis, int nx, int ny, int nz, int v) {
  if (axis == 2) {
    int tp = 1;
    switch (n_axis) {
      case 16: tp = contig_tp<16, 0>(); break;
      case 32: tp = contig_tp<32, 0>(); break;
      case 64: tp = contig_tp<64, 0>(); break;
      case 96: tp = contig_tp<96, 0>(); break;
      case 128: tp = v == 1 ? contig_tp<128, 1>() : v == 2 ? contig_tp<128, 2>()
                   : v == 3 ? contig_tp<128, 3>() : contig_tp<128, 0>(); break;
      case 256: tp = v == 1 ? contig_tp<256, 1>() : v == 2 ? contig_tp<256, 2>()
                   : v == 3 ? contig_tp<256, 3>() : contig_tp<256, 0>(); break;
      case 512: tp = contig_tp<512, 0>(); break;
    }
    return (nx * ny) / tp;
  }
  return (axis == 0 ? ny : nx) * (nz / (has_radix_variant(n_axis) ? strided_tile_width(v) : 16));
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
  if (a.shape != 0 && has_radix_variant(n)) {
    switch (a.shape) {
      case 1: return run_shape_variant<1>(MODE, n, a, st);
      case 2: return run_shape_variant<2>(MODE, n, a, st);
      case 3: return run_shape_variant<3>(MODE, n, a, st);
    }
    set_error("internal: pass shape variant %d", a.shape);
    return 1;
  }
#define QJ_CASE(NN)                                                          \
  case NN:                                                                   \
    if constexpr (ONLY_Y) return run_fused<NN, false, MODE, 0>(a, st);       \
    else return contig ? run_fused<NN, true, MODE, 0>(a, st) : run_fused<NN, false, MODE, 0>(a, st);
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

// The dense deposit and the adjoint passes run along z only, in the default
// shape.
template <int MODE>
static int dispatch_z_only(int n, const FusedArgs &a, cudaStream_t st) {
  if (a.axis != 2) {
    set_error("internal: pass mode %d must run along z", MODE);
    return 1;
  }
  switch (n) {
    case 16: return run_fused<16, true, MODE, 0>(a, st);
    case 32: return run_fused<32, true, MODE, 0>(a, st);
    case 64: return run_fused<64, true, MODE, 0>(a, st);
    case 96: return run_fused<96, true, MODE, 0>(a, st);
    case 128: return run_fused<128, true, MODE, 0>(a, st);
    case 256: return run_fused<256, true, MODE, 0>(a, st);
    case 512: return run_fused<512, true, MODE, 0>(a, st);
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
    case M_DEPOSIT: return dispatch_z_only<M_DEPOSIT>(n, a, st);
    case M_ADJ_SOURCE: return dispatch_z_only<M_ADJ_SOURCE>(n, a, st);
    case M_ADJ_UPDATE: return dispatch_z_only<M_ADJ_UPDATE>(n, a, st);
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
    if constexpr (ONLY_Y) e = fused_occupancy<NN, false, MODE, 0>(per_sm, sms);             \
    else if constexpr (ONLY_Z) e = fused_occupancy<NN, true, MODE, 0>(per_sm, sms);         \
    else e = contig ? fused_occupancy<NN, true, MODE, 0>(per_sm, sms)                       \
                    : fused_occupancy<NN, false, MODE, 0>(per_sm, sms);                     \
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

int fused_max_ctas_per_sm(int mode, int n, bool contig, int shape) {
  if (shape != 0 && has_radix_variant(n) && mode != M_DEPOSIT) {
    switch (shape) {
      case 1: return shape_variant_ctas_per_sm<1>(mode, n, contig);
      case 2: return shape_variant_ctas_per_sm<2>(mode, n, contig);
      case 3: return shape_variant_ctas_per_sm<3>(mode, n, contig);
    }
    return 0;
  }
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
  // buckets 0..7 are the passes of the step; the adjoint's passes count as
  // other kernels (8)
  if (prof && rc == 0)
    prof_mark_end((mode <= M_DEPOSIT ? mode : 8) + (prof_split() && a.axis == 2 ? kProfZ : 0), st);
  return rc;
}

}  // namespace qj
