// Instantiations and launcher of the generic in-place FFT pass (float2 and
// double2), used by the plain path, the standalone operators and qj_fft3d.
#include <mutex>

#include "qj_internal.h"

namespace qj {

template <typename R, int N, bool CONTIG, int DIR>
static int run_fft(const FftArgs &a, cudaStream_t st) {
  using SH = PassShape<N, CONTIG>;
  const size_t smem = SH::template smem_bytes<cplx<R>>();
  // the attribute belongs to the current device's context: set once per device
  static PerDevice<cudaError_t> attr;
  const cudaError_t *attr_err = nullptr;
  QJ_CK(per_device(attr, attr_err, [&](cudaError_t &r) {
    r = cudaFuncSetAttribute(k_fft<R, N, CONTIG, DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
  }));
  QJ_CK(*attr_err);
  const int grid = CONTIG ? (a.nx * a.ny) / SH::TP : (a.axis == 0 ? a.ny : a.nx) * (a.nz / 16);
  k_fft<R, N, CONTIG, DIR><<<grid, SH::THREADS, smem, st>>>(a);
  QJ_CK_LAUNCH();
  return 0;
}

template <typename R, int DIR>
static int dispatch(int n, const FftArgs &a, cudaStream_t st) {
  const bool contig = a.axis == 2;
#define QJ_CASE(NN) \
  case NN: return contig ? run_fft<R, NN, true, DIR>(a, st) : run_fft<R, NN, false, DIR>(a, st);
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

int launch_fft(bool dbl, int n, int dir, const FftArgs &a, cudaStream_t st) {
  if (dbl) return dir < 0 ? dispatch<double, -1>(n, a, st) : dispatch<double, +1>(n, a, st);
  return dir < 0 ? dispatch<float, -1>(n, a, st) : dispatch<float, +1>(n, a, st);
}

}  // namespace qj
