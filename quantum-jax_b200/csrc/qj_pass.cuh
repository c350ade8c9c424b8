// Pencil-pass kernels.
//
// One CTA owns TP pencils along one axis; each pencil is held by P threads
// (see qj_fft.cuh).  A pass reads each of its input fields once from HBM,
// transforms along its axis in registers / shared memory, applies the fused
// pointwise work and writes each output field once.
//
// Fused single-precision step (a 3-D transform is one pass per axis; the
// axis order alternates between kicks so the kick, drift and density build
// share passes):
//   DENSITY        psi -> rho = |psi|^2 + rho_stars (+ rho_gas) -> FFT_q -> R
//   FFT_FWD        R -> FFT_y -> R
//   POISSON        R -> FFT_r, V^ = -4 pi G rho^ / k^2 (k=0 from the float64
//                  mean), S1 = V^(1 + k_r), S2 = V^(k_y - i k_q) -> IFFT_r
//   IFFT2          S1, S2 -> IFFT_y -> S1, S2
//   KICK           S1, S2 -> IFFT_q -> V + i a_r, a_q + i a_y; psi *= exp(-i c V);
//                  a_max; accelerations at deposit cells; optional gas kick;
//                  optional drift along q: psi <- IFFT_q(P_q FFT_q psi)
//   DRIFT          psi -> IFFT_y(P_y FFT_y psi)
//   DRIFT_DENSITY  DRIFT along r, then DENSITY along r
#pragma once

#include "qj_fft.cuh"

namespace qj {

enum PassMode : int {
  M_DENSITY = 0,
  M_FFT_FWD = 1,
  M_POISSON = 2,
  M_IFFT2 = 3,
  M_KICK = 4,
  M_DRIFT = 5,
  M_DRIFT_DENSITY = 6,
};

struct FusedArgs {
  int nx, ny, nz;
  int axis;                // 0, 1, 2
  long long stride;        // element stride along the axis
  long long outer_stride;  // strided passes: stride of the outer index
  int ztiles;              // strided passes: nz / 16
  float2 *psi;
  float2 *R;
  float2 *S1;
  float2 *S2;
  const float2 *tw;    // twiddles of this axis' length
  const float2 *prop;  // drift propagator of this axis, already scaled by 1/n
  const float *k[3];   // k value per index, per axis (Nyquist negative)
  const float *kt[3];  // k with the Nyquist entry set to 0 (odd derivatives)
  // deposit / gather list in this pass' orientation
  const int *pstart;
  const unsigned *ukey;
  const float *uval;
  float *A;  // [n_unique][3] accelerations at the deposit cells (x, y, z)
  // float64 density partial sums
  double *part;
  const double *part_in;
  int n_part;
  // scalars
  double fourpiG;
  double rho_bar;
  double inv_ncell;
  double kick_coef;  // phase = kick_coef * V
  float b_coeff;     // self-interaction coefficient (0 = off)
  const float *v_ext;
  unsigned *amax_bits;
  int do_drift;
  // isothermal gas
  const float *grho;
  float *gv[3];
  float gas_dt;
};

// Per-thread position of a pencil in the grid.
struct PencilPos {
  long long base;  // linear index of element 0 of the pencil
  int pid;         // pencil id in this axis' orientation
  int c[3];        // coordinates (the axis' own entry is unused)
};

template <bool CONTIG>
__device__ __forceinline__ PencilPos pencil_pos(const FusedArgs &a, int p, int TP) {
  PencilPos pp;
  if (CONTIG) {  // axis 2: rows x * ny + y
    const int row = blockIdx.x * TP + p;
    pp.pid = row;
    pp.base = (long long)row * a.nz;
    pp.c[0] = row / a.ny;
    pp.c[1] = row % a.ny;
    pp.c[2] = 0;
  } else {
    const int o = blockIdx.x / a.ztiles;
    const int z = (blockIdx.x % a.ztiles) * 16 + p;
    pp.base = (long long)o * a.outer_stride + z;
    pp.c[2] = z;
    if (a.axis == 0) {  // o = y
      pp.c[0] = 0;
      pp.c[1] = o;
      pp.pid = o * a.nz + z;
    } else {  // axis 1, o = x
      pp.c[0] = o;
      pp.c[1] = 0;
      pp.pid = o * a.nz + z;
    }
  }
  return pp;
}

template <int E, typename C>
__device__ __forceinline__ void load_pencil(C (&v)[E], const C *__restrict__ f, long long base,
                                            long long stride, int t, int P) {
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = f[base + (long long)(t + P * e) * stride];
}
template <int E, typename C>
__device__ __forceinline__ void store_pencil(const C (&v)[E], C *__restrict__ f, long long base,
                                             long long stride, int t, int P) {
#pragma unroll
  for (int e = 0; e < E; ++e) f[base + (long long)(t + P * e) * stride] = v[e];
}

// Register select with a runtime index (unrolled compare, no local memory).
template <int E>
__device__ __forceinline__ void reg_add(float2 (&v)[E], int e, float add) {
#pragma unroll
  for (int q = 0; q < E; ++q)
    if (q == e) v[q].x = v[q].x + add;
}
template <int E>
__device__ __forceinline__ float2 reg_get(const float2 (&v)[E], int e) {
  float2 r = v[0];
#pragma unroll
  for (int q = 1; q < E; ++q)
    if (q == e) r = v[q];
  return r;
}

// Deterministic block sum of one double per thread (fixed order).
template <int THREADS>
__device__ __forceinline__ double block_sum(double x, double *sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  __syncthreads();
  if (lane == 0) sh[w] = x;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (THREADS + 31) / 32; ++i) s += sh[i];
    sh[0] = s;
  }
  __syncthreads();
  s = sh[0];
  __syncthreads();
  return s;
}

// rho = |psi|^2 + rho_stars (+ rho_gas), element by element (float32 order
// of quantum-stars.py:299 / quantum-gas-bh.py:542).  Adds the pencil's
// deposit entries.  Returns the thread's float64 partial sum of rho.
template <int N, int E>
__device__ __forceinline__ double build_density(float2 (&v)[E], const FusedArgs &a,
                                                const PencilPos &pp, int t, int P) {
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = float2{v[e].x * v[e].x + v[e].y * v[e].y, 0.0f};
  if (a.pstart) {
    const int lo = a.pstart[pp.pid], hi = a.pstart[pp.pid + 1];
    const unsigned kbase = (unsigned)pp.pid * (unsigned)N;
    for (int k = lo; k < hi; ++k) {
      const int i = (int)(a.ukey[k] - kbase);
      if (i % P == t) reg_add<E>(v, i / P, a.uval[k]);
    }
  }
  if (a.grho) {
#pragma unroll
    for (int e = 0; e < E; ++e)
      v[e].x = v[e].x + a.grho[pp.base + (long long)(t + P * e) * a.stride];
  }
  double s = 0.0;
#pragma unroll
  for (int e = 0; e < E; ++e) s += (double)v[e].x;
  return s;
}

__device__ __forceinline__ float2 phase_rotate(float2 z, double theta) {
  // exp(-i theta) * z with theta reduced modulo 2 pi in float64 first.
  const double twopi = 6.283185307179586476925286766559;
  const double tr = theta - twopi * rint(theta * (1.0 / twopi));
  float s, c;
  sincosf((float)tr, &s, &c);
  return float2{z.x * c + z.y * s, z.y * c - z.x * s};
}

template <int N, bool CONTIG, int MODE>
__global__ void __launch_bounds__(PassShape<N, CONTIG>::THREADS)
    k_fused(FusedArgs a) {
  using SH = PassShape<N, CONTIG>;
  constexpr int E = SH::E, P = SH::P, TP = SH::TP, THREADS = SH::THREADS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2 *sm = reinterpret_cast<float2 *>(smem_raw);
  __shared__ double red[(THREADS + 31) / 32 + 1];

  const int tid = threadIdx.x;
  int p, t;
  if (CONTIG) {
    t = tid % P;
    p = tid / P;
  } else {
    p = tid % TP;
    t = tid / TP;
  }
  const PencilPos pp = pencil_pos<CONTIG>(a, p, TP);
  const long long base = pp.base, st = a.stride;
  using SMV = typename std::conditional<CONTIG, SmemContig<float2>, SmemStrided<float2, TP>>::type;
  SMV smv;
  if constexpr (CONTIG)
    smv.row = sm + p * SH::ROW;
  else
    smv.base = sm + p;
  const float2 *tw = a.tw;

  if constexpr (MODE == M_DENSITY) {
    float2 v[E];
    load_pencil<E>(v, a.psi, base, st, t, P);
    double s = build_density<N, E>(v, a, pp, t, P);
    s = block_sum<THREADS>(s, red);
    if (tid == 0) a.part[blockIdx.x] = s;
    fft_pencil<N, -1>(v, t, smv, tw);
    store_pencil<E>(v, a.R, base, st, t, P);
  } else if constexpr (MODE == M_FFT_FWD) {
    float2 v[E];
    load_pencil<E>(v, a.R, base, st, t, P);
    fft_pencil<N, -1>(v, t, smv, tw);
    store_pencil<E>(v, a.R, base, st, t, P);
  } else if constexpr (MODE == M_POISSON) {
    float2 v[E];
    load_pencil<E>(v, a.R, base, st, t, P);
    // Mean density in float64 for the k = 0 mode (pencil 0 of CTA 0 only).
    double mean = 0.0;
    if (blockIdx.x == 0) {
      double s = 0.0;
      for (int i = tid; i < a.n_part; i += THREADS) s += a.part_in[i];
      mean = block_sum<THREADS>(s, red) * a.inv_ncell;
    }
    fft_pencil<N, -1>(v, t, smv, tw);
    const int ax = a.axis;            // r: 0 or 2
    const int aq = 2 - ax;            // the other non-y axis
    const float kq2 = a.k[aq][pp.c[aq]] * a.k[aq][pp.c[aq]];
    const float ky = a.k[1][pp.c[1]];
    const float kperp2 = kq2 + ky * ky;
    const float ktq = a.kt[aq][pp.c[aq]], kty = a.kt[1][pp.c[1]];
    const float g0 = (float)(-a.fourpiG * a.inv_ncell);
    float2 w[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int i = t + P * e;
      const float kr = a.k[ax][i];
      const float k2 = kperp2 + kr * kr;
      float2 vh;
      if (k2 == 0.0f) {
        // V^(0) = -4 pi G (sum rho - ncell rho_bar) / 1, scaled by 1/ncell
        vh = float2{(float)(-a.fourpiG * (mean - a.rho_bar)), 0.0f};
      } else {
        const float g = g0 / k2;
        vh = float2{v[e].x * g, v[e].y * g};
      }
      const float f1 = 1.0f + a.kt[ax][i];
      v[e] = float2{vh.x * f1, vh.y * f1};
      // (kty - i ktq) * vh
      w[e] = float2{kty * vh.x + ktq * vh.y, kty * vh.y - ktq * vh.x};
    }
    fft_pencil<N, +1>(v, t, smv, tw);
    store_pencil<E>(v, a.S1, base, st, t, P);
    fft_pencil<N, +1>(w, t, smv, tw);
    store_pencil<E>(w, a.S2, base, st, t, P);
  } else if constexpr (MODE == M_IFFT2) {
    float2 v[E];
    load_pencil<E>(v, a.S1, base, st, t, P);
    fft_pencil<N, +1>(v, t, smv, tw);
    store_pencil<E>(v, a.S1, base, st, t, P);
    load_pencil<E>(v, a.S2, base, st, t, P);
    fft_pencil<N, +1>(v, t, smv, tw);
    store_pencil<E>(v, a.S2, base, st, t, P);
  } else if constexpr (MODE == M_KICK) {
    float2 v1[E], v2[E], ps[E];
    load_pencil<E>(v1, a.S1, base, st, t, P);
    load_pencil<E>(v2, a.S2, base, st, t, P);
    load_pencil<E>(ps, a.psi, base, st, t, P);
    fft_pencil<N, +1>(v1, t, smv, tw);  // V + i a_r
    fft_pencil<N, +1>(v2, t, smv, tw);  // a_q + i a_y
    const int aq = a.axis, ar = 2 - a.axis;
    // a_max over the three components
    float am = 0.0f;
#pragma unroll
    for (int e = 0; e < E; ++e)
      am = fmaxf(am, fmaxf(fabsf(v1[e].y), fmaxf(fabsf(v2[e].x), fabsf(v2[e].y))));
    // self-interaction needs rho = |psi|^2 + rho_stars at the kick
    float rs[E];
    if (a.b_coeff != 0.0f) {
#pragma unroll
      for (int e = 0; e < E; ++e) rs[e] = ps[e].x * ps[e].x + ps[e].y * ps[e].y;
    }
    // accelerations at the deposit cells of these pencils
    if (a.pstart) {
      const int lo = a.pstart[pp.pid], hi = a.pstart[pp.pid + 1];
      const unsigned kbase = (unsigned)pp.pid * (unsigned)N;
      for (int k = lo; k < hi; ++k) {
        const int i = (int)(a.ukey[k] - kbase);
        if (i % P == t) {
          const int e = i / P;
          const float2 s1 = reg_get<E>(v1, e), s2 = reg_get<E>(v2, e);
          float acc[3];
          acc[ar] = s1.y;
          acc[aq] = s2.x;
          acc[1] = s2.y;
          a.A[3 * k + 0] = acc[0];
          a.A[3 * k + 1] = acc[1];
          a.A[3 * k + 2] = acc[2];
          if (a.b_coeff != 0.0f) {
#pragma unroll
            for (int q = 0; q < E; ++q)
              if (q == e) rs[q] = rs[q] + a.uval[k];
          }
        }
      }
    }
    // gas half kick with the grid accelerations (quantum-gas-bh.py:255-266)
    if (a.gv[0]) {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const long long idx = base + (long long)(t + P * e) * st;
        float acc[3];
        acc[ar] = v1[e].y;
        acc[aq] = v2[e].x;
        acc[1] = v2[e].y;
#pragma unroll
        for (int d = 0; d < 3; ++d) a.gv[d][idx] = a.gv[d][idx] + acc[d] * a.gas_dt;
      }
    }
    // kick: psi <- exp(-i c V) psi, V = Poisson + b rho + V_ext
#pragma unroll
    for (int e = 0; e < E; ++e) {
      float V = v1[e].x;
      if (a.b_coeff != 0.0f) V = V + a.b_coeff * rs[e];
      if (a.v_ext) V = V + a.v_ext[base + (long long)(t + P * e) * st];
      ps[e] = phase_rotate(ps[e], a.kick_coef * (double)V);
    }
    if (a.do_drift) {
      fft_pencil<N, -1>(ps, t, smv, tw);
#pragma unroll
      for (int e = 0; e < E; ++e) ps[e] = cmul(ps[e], __ldg(&a.prop[t + P * e]));
      fft_pencil<N, +1>(ps, t, smv, tw);
    }
    store_pencil<E>(ps, a.psi, base, st, t, P);
    // block max -> one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) am = fmaxf(am, __shfl_xor_sync(0xffffffffu, am, o));
    if ((tid & 31) == 0) atomic_max_nonneg(a.amax_bits, am);
  } else if constexpr (MODE == M_DRIFT || MODE == M_DRIFT_DENSITY) {
    float2 v[E];
    load_pencil<E>(v, a.psi, base, st, t, P);
    fft_pencil<N, -1>(v, t, smv, tw);
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = cmul(v[e], __ldg(&a.prop[t + P * e]));
    fft_pencil<N, +1>(v, t, smv, tw);
    store_pencil<E>(v, a.psi, base, st, t, P);
    if constexpr (MODE == M_DRIFT_DENSITY) {
      double s = build_density<N, E>(v, a, pp, t, P);
      s = block_sum<THREADS>(s, red);
      if (tid == 0) a.part[blockIdx.x] = s;
      fft_pencil<N, -1>(v, t, smv, tw);
      store_pencil<E>(v, a.R, base, st, t, P);
    }
  }
}

// Generic in-place FFT pass over a complex field (plain path and qj_fft3d).
// scale multiplies the output (1/n for a normalised inverse).
struct FftArgs {
  int nx, ny, nz;
  int axis;
  long long stride, outer_stride;
  int ztiles;
  void *data;
  const void *tw;
  double scale;
};

template <typename R, int N, bool CONTIG, int DIR>
__global__ void __launch_bounds__(PassShape<N, CONTIG>::THREADS) k_fft(FftArgs a) {
  using C = cplx<R>;
  using SH = PassShape<N, CONTIG>;
  constexpr int E = SH::E, P = SH::P, TP = SH::TP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *sm = reinterpret_cast<C *>(smem_raw);
  const int tid = threadIdx.x;
  int p, t;
  if (CONTIG) {
    t = tid % P;
    p = tid / P;
  } else {
    p = tid % TP;
    t = tid / TP;
  }
  long long base;
  if (CONTIG) {
    base = (long long)(blockIdx.x * TP + p) * a.nz;
  } else {
    const int o = blockIdx.x / a.ztiles;
    const int z = (blockIdx.x % a.ztiles) * 16 + p;
    base = (long long)o * a.outer_stride + z;
  }
  using SMV = typename std::conditional<CONTIG, SmemContig<C>, SmemStrided<C, TP>>::type;
  SMV smv;
  if constexpr (CONTIG)
    smv.row = sm + p * SH::ROW;
  else
    smv.base = sm + p;
  C *f = reinterpret_cast<C *>(a.data);
  C v[E];
  load_pencil<E>(v, f, base, a.stride, t, P);
  fft_pencil<N, DIR>(v, t, smv, reinterpret_cast<const C *>(a.tw));
  if (a.scale != 1.0) {
    const R s = (R)a.scale;
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = C{v[e].x * s, v[e].y * s};
  }
  store_pencil<E>(v, f, base, a.stride, t, P);
}

}  // namespace qj
