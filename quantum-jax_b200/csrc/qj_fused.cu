// Instantiations and launchers of the fused single-precision pencil passes.
#include <mutex>

#include "qj_internal.h"

namespace qj {

bool fft_length_supported(int n) {
  return n == 16 || n == 32 || n == 64 || n == 128 || n == 256 || n == 512;
}

template <int N, bool CONTIG>
static int grid_of(const FusedArgs &a) {
  using SH = PassShape<N, CONTIG>;
  if (CONTIG) return (a.nx * a.ny) / SH::TP;
  return (a.axis == 0 ? a.ny : a.nx) * (a.nz / 16);
}

int pass_blocks(int n_axis, int axis, int nx, int ny, int nz) {
  if (axis == 2) {
    const int E = (n_axis == 32 || n_axis == 64) ? 8 : 16;
    const int P = n_axis / E;
    const int TP = P >= 256 ? 1 : 256 / P;
    return (nx * ny) / TP;
  }
  return (axis == 0 ? ny : nx) * (nz / 16);
}

template <int N, bool CONTIG, int MODE>
static int run_fused(const FusedArgs &a, cudaStream_t st) {
  using SH = PassShape<N, CONTIG>;
  const size_t smem = SH::template smem_bytes<float2>();
  static std::once_flag once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(once, [&] {
    attr_err = cudaFuncSetAttribute(k_fused<N, CONTIG, MODE>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  QJ_CK(attr_err);
  k_fused<N, CONTIG, MODE><<<grid_of<N, CONTIG>(a), SH::THREADS, smem, st>>>(a);
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
