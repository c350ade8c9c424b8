// Launchers of the fused single-precision pencil passes, shared by the
// translation units that instantiate them: qj_fused.cu (every length, the
// default shape) and qj_fused_v{1,2,3}.cu (the shape variants of n = 128 and
// 256, compiled in parallel).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "../../include/qj.h"
#include "qj_internal.h"

namespace qj {

template <int N, bool CONTIG, int V>
int grid_of(const FusedArgs &a) {
  using SH = PassShape<N, CONTIG, V>;
  if (CONTIG) {
    // a reduced range (half spectrum) rounds up to whole tiles, within the
    // grid; the rows past it are pencils the pass does not store
    const int full = ((a.full_nx > 0 ? a.full_nx : a.nx) * a.ny) / SH::TP;
    return std::min(full, (a.nx * a.ny + SH::TP - 1) / SH::TP);
  }
  return (a.axis == 0 ? a.ny : a.nx) * a.ztiles;
}

// CTA slots a persistent pass leaves free for concurrent work on other
// streams, such as the star update and bucket sort that run beside the y
// drift pass (QJ_PERSIST_RESERVE, default 2).
inline int reserve_ctas() {
  static int r = -1;
  if (r < 0) {
    const char *env = getenv("QJ_PERSIST_RESERVE");
    r = env ? std::max(0, atoi(env)) : 2;
  }
  return r;
}

// cuTensorMapEncodeTiled from the driver, looked up once.
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
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

// Tensor maps of a strided pass' streamed fields (see TileMaps): a box of the
// tile's TP z columns (TP x 8 bytes, a multiple of 16; tiles start at z
// multiples of TP) by up to 256 rows along the pass axis.
template <int N, int MODE, int V>
int strided_maps(const FusedArgs &a, TileMaps &maps) {
  auto enc = tensor_map_encoder();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return QJ_ERR_CUDA;
  }
  constexpr int TP = PassShape<N, false, V>::TP;
  static_assert((TP * 8) % 16 == 0, "a tensor-map box row must be a multiple of 16 bytes");
  const int nbox = a.nbox > 1 ? a.nbox : 1;
  const cuuint64_t dims[4] = {(cuuint64_t)a.nz, (cuuint64_t)a.ny, (cuuint64_t)a.nx, (cuuint64_t)nbox};
  const cuuint64_t strides[3] = {(cuuint64_t)a.nz * 8, (cuuint64_t)a.ny * a.nz * 8,
                                 (cuuint64_t)a.box_cells * 8};
  const cuuint32_t rows = (cuuint32_t)std::min(N, 256);
  const cuuint32_t box[4] = {(cuuint32_t)TP, a.axis == 0 ? 1u : rows, a.axis == 0 ? rows : 1u, 1};
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
template <int N, bool CONTIG, int MODE, int V>
cudaError_t fused_occupancy(int &per_sm, int &sms) {
  using SH = PassShape<N, CONTIG, V>;
  static PerDevice<Occupancy> cache;
  const Occupancy *o = nullptr;
  const cudaError_t e = per_device(cache, o, [](Occupancy &r) {
    const size_t smem = fused_smem_bytes<N, CONTIG, MODE, V>();
    r.err = cudaFuncSetAttribute(k_fused<N, CONTIG, MODE, V>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int dev = 0, n_sm = 0, p = 0;
    if (r.err == cudaSuccess) r.err = cudaGetDevice(&dev);
    if (r.err == cudaSuccess) r.err = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (r.err == cudaSuccess)
      r.err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, k_fused<N, CONTIG, MODE, V>,
                                                            SH::THREADS, smem);
    r.per_sm = std::max(1, p);
    r.sms = std::max(1, n_sm);
  });
  if (e != cudaSuccess) return e;
  per_sm = o->per_sm;
  sms = o->sms;
  return o->err;
}

template <int N, bool CONTIG, int MODE, int V>
int run_fused(const FusedArgs &a, cudaStream_t st) {
  using SH = PassShape<N, CONTIG, V>;
  const size_t smem = fused_smem_bytes<N, CONTIG, MODE, V>();
  // persistent grid: the CTAs resident at once (occupancy x SMs), shared
  // between the boxes of a batched launch
  int per_sm = 0, sms = 0;
  const cudaError_t occ = fused_occupancy<N, CONTIG, MODE, V>(per_sm, sms);
  QJ_CK(occ);
  const int want = (a.tune && MODE <= M_DEPOSIT) ? a.tune[MODE] : 0;  // [0..7]: passes
  const int resident = (want > 0 ? std::min(want, per_sm) : per_sm) * sms;
  const int reserve = (a.tune && a.tune[8] >= 0) ? a.tune[8] : reserve_ctas();
  // the bulk tile copies need 16-byte aligned fields
  const void *fields[4] = {a.psi, a.R, a.S1, a.S2};
  for (const void *f : fields)
    if ((reinterpret_cast<uintptr_t>(f) & 15) != 0) {
      set_error("fields of the fused passes must be 16-byte aligned");
      return QJ_ERR_ARG;
    }
  if (!CONTIG && a.nz % SH::TP != 0) {
    set_error("internal: nz = %d is not a multiple of the %d-wide z tiles", a.nz, SH::TP);
    return QJ_ERR_ARG;
  }
  FusedArgs b = a;
  b.ntiles = grid_of<N, CONTIG, V>(a);
  // y passes walk backwards: each follows (and precedes) a pass that walks
  // forwards over the same slow index x
  b.rev = (!CONTIG && a.axis == 1) ? 1 : 0;
  TileMaps maps;
  std::memset(&maps, 0, sizeof(maps));
  if (!CONTIG && stream_count<MODE>() > 0) {
    const int rc = strided_maps<N, MODE, V>(b, maps);
    if (rc) return rc;
  }
  const int nbox = a.nbox > 1 ? a.nbox : 1;
  const int gx = std::max(1, std::min(b.ntiles, (resident - reserve) / nbox));
  cudaLaunchConfig_t cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3(gx, nbox);
  cfg.blockDim = dim3(SH::THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  // programmatic dependent launch: the CTAs may start during the previous
  // pass's last tiles and wait for it (griddepcontrol.wait) before reading
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = a.pdl ? 1 : 0;
  QJ_CK(cudaLaunchKernelEx(&cfg, k_fused<N, CONTIG, MODE, V>, b, maps));
  QJ_CK_LAUNCH();
  return 0;
}

// Transforming passes of one shape variant V (> 0) over the lengths that have
// variants (n = 128, 256); instantiated by qj_fused_v<V>.cu.  The y-only
// transforms are instantiated strided, the others for both orientations.
template <int V> int run_shape_variant(int mode, int n, const FusedArgs &a, cudaStream_t st);
template <int V> int shape_variant_ctas_per_sm(int mode, int n, bool contig);
template <> int run_shape_variant<1>(int mode, int n, const FusedArgs &a, cudaStream_t st);
template <> int run_shape_variant<2>(int mode, int n, const FusedArgs &a, cudaStream_t st);
template <> int run_shape_variant<3>(int mode, int n, const FusedArgs &a, cudaStream_t st);
template <> int shape_variant_ctas_per_sm<1>(int mode, int n, bool contig);
template <> int shape_variant_ctas_per_sm<2>(int mode, int n, bool contig);
template <> int shape_variant_ctas_per_sm<3>(int mode, int n, bool contig);

#define QJ_VARIANT_MODE(MODE, NN, VV)                                                    \
  case MODE:                                                                             \
    if constexpr (MODE == M_FFT_FWD || MODE == M_IFFT2) return run_fused<NN, false, MODE, VV>(a, st); \
    else return contig ? run_fused<NN, true, MODE, VV>(a, st) : run_fused<NN, false, MODE, VV>(a, st);

#define QJ_VARIANT_OCC(MODE, NN, VV)                                                          \
  case MODE:                                                                                  \
    if constexpr (MODE == M_FFT_FWD || MODE == M_IFFT2) e = fused_occupancy<NN, false, MODE, VV>(per_sm, sms); \
    else e = contig ? fused_occupancy<NN, true, MODE, VV>(per_sm, sms)                        \
                    : fused_occupancy<NN, false, MODE, VV>(per_sm, sms);                      \
    break;

// Body of qj_fused_v<VV>.cu.
#define QJ_DEFINE_SHAPE_VARIANT(VV)                                                        \
  template <int NN>                                                                        \
  static int run_variant_n(int mode, const FusedArgs &a, cudaStream_t st) {                \
    const bool contig = a.axis == 2;                                                       \
    if ((mode == M_FFT_FWD || mode == M_IFFT2) && contig) {                                \
      set_error("internal: pass mode %d requested along z", mode);                        \
      return 1;                                                                            \
    }                                                                                      \
    switch (mode) {                                                                        \
      QJ_VARIANT_MODE(M_DENSITY, NN, VV)                                                   \
      QJ_VARIANT_MODE(M_FFT_FWD, NN, VV)                                                   \
      QJ_VARIANT_MODE(M_POISSON, NN, VV)                                                   \
      QJ_VARIANT_MODE(M_IFFT2, NN, VV)                                                     \
      QJ_VARIANT_MODE(M_KICK, NN, VV)                                                      \
      QJ_VARIANT_MODE(M_DRIFT, NN, VV)                                                     \
      QJ_VARIANT_MODE(M_DRIFT_DENSITY, NN, VV)                                             \
    }                                                                                      \
    set_error("internal: pass mode %d has no shape variants", mode);                      \
    return 1;                                                                              \
  }                                                                                        \
  template <int NN>                                                                        \
  static int occ_variant_n(int mode, bool contig) {                                        \
    int per_sm = 0, sms = 0;                                                               \
    cudaError_t e = cudaSuccess;                                                           \
    switch (mode) {                                                                        \
      QJ_VARIANT_OCC(M_DENSITY, NN, VV)                                                    \
      QJ_VARIANT_OCC(M_FFT_FWD, NN, VV)                                                    \
      QJ_VARIANT_OCC(M_POISSON, NN, VV)                                                    \
      QJ_VARIANT_OCC(M_IFFT2, NN, VV)                                                      \
      QJ_VARIANT_OCC(M_KICK, NN, VV)                                                       \
      QJ_VARIANT_OCC(M_DRIFT, NN, VV)                                                      \
      QJ_VARIANT_OCC(M_DRIFT_DENSITY, NN, VV)                                              \
      default: return 0;                                                                   \
    }                                                                                      \
    return e == cudaSuccess ? per_sm : 0;                                                  \
  }                                                                                        \
  template <>                                                                              \
  int run_shape_variant<VV>(int mode, int n, const FusedArgs &a, cudaStream_t st) {        \
    if (n == 128) return run_variant_n<128>(mode, a, st);                                  \
    if (n == 256) return run_variant_n<256>(mode, a, st);                                  \
    set_error("internal: length %d has no shape variants", n);                            \
    return 1;                                                                              \
  }                                                                                        \
  template <>                                                                              \
  int shape_variant_ctas_per_sm<VV>(int mode, int n, bool contig) {                        \
    if (n == 128) return occ_variant_n<128>(mode, contig);                                 \
    if (n == 256) return occ_variant_n<256>(mode, contig);                                 \
    return 0;                                                                              \
  }

}  // namespace qj
