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
  M_DEPOSIT = 7,  // dense star density along z (bin_stars), no transform
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
  const float2 *tw;    // stage twiddle table of this axis' length (stage_tw_off)
  const float2 *prop;  // drift propagator of this axis minus one (see drift_pencil)
  float *v_out;        // KICK: optional copy of the kick potential V (adjoint)
  const float *k[3];   // k value per index, per axis (Nyquist negative)
  const float *kt[3];  // k with the Nyquist entry set to 0 (odd derivatives)
  // stars filed by the pencil of their lower CIC corner (this pass' axis)
  int has_stars;
  const int4 *sidx;
  const float4 *sw0;
  const float4 *sw1;
  const unsigned *perm;
  const int *bstart;
  float *A;  // [8 n][3] accelerations at the 8 corners of each star (x, y, z)
  float *rho_out;  // M_DEPOSIT: dense star density
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
  // L2 prefetch distance in CTAs (0 = off): each CTA prefetches the input
  // tile of CTA blockIdx.x + ahead, one resident wave later
  int ahead;
  // batched boxes (blockIdx.y = box): per-box strides of the fields (cells),
  // stars, bucket starts, partial sums; a_max is per box
  int nbox;  // launch grid.y (0 or 1 = one box)
  long long box_cells;
  int box_stars;
  int box_bstart;
  int box_part;
};

// Offset a pass' pointers to box blockIdx.y of a batched plan.
__device__ __forceinline__ void select_box(FusedArgs &a) {
  const int b = blockIdx.y;
  if (b == 0) return;
  const long long c = (long long)b * a.box_cells;
  if (a.psi) a.psi += c;
  if (a.R) a.R += c;
  if (a.S1) a.S1 += c;
  if (a.S2) a.S2 += c;
  if (a.part) a.part += (long long)b * a.box_part;
  if (a.part_in) a.part_in += (long long)b * a.box_part;
  if (a.amax_bits) a.amax_bits += b;
  const long long s = (long long)b * a.box_stars;
  if (a.sidx) a.sidx += s;
  if (a.sw0) a.sw0 += s;
  if (a.sw1) a.sw1 += s;
  if (a.perm) a.perm += s;
  if (a.A) a.A += 24 * s;
  if (a.bstart) a.bstart += (long long)b * a.box_bstart;
}

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

// Element e of a thread's pencil sits at base + (t + P e) * stride; grids
// hold at most 512^3 = 2^27 cells, so 32-bit offsets are exact.
template <int E, typename C>
__device__ __forceinline__ void load_pencil(C (&v)[E], const C *__restrict__ f, long long base,
                                            long long stride, int t, int P) {
  const unsigned b = (unsigned)base + (unsigned)t * (unsigned)stride;
  const unsigned s = (unsigned)P * (unsigned)stride;
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = __ldcs(&f[b + (unsigned)e * s]);  // read once: evict first
}
template <int E, typename C>
__device__ __forceinline__ void store_pencil(const C (&v)[E], C *__restrict__ f, long long base,
                                             long long stride, int t, int P) {
  const unsigned b = (unsigned)base + (unsigned)t * (unsigned)stride;
  const unsigned s = (unsigned)P * (unsigned)stride;
#pragma unroll
  for (int e = 0; e < E; ++e) f[b + (unsigned)e * s] = v[e];
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

// corner number (reference order) of the corner with ip1 bits b = bx + 2 by + 4 bz
__device__ __forceinline__ int c_corner_of_bits_dev(int b) {
  return b == 3 ? 4 : (b == 4 ? 3 : b);
}

__device__ __forceinline__ int sel3(int a, int b, int c, int i) { return i == 0 ? a : (i == 1 ? b : c); }
__device__ __forceinline__ float sel3f(float a, float b, float c, int i) {
  return i == 0 ? a : (i == 1 ? b : c);
}

// The four star buckets whose stars touch this pencil: lower corners at
// (cu, cv), (cu-1, cv), (cu, cv-1), (cu-1, cv-1) in the cross-plane axes
// (u, v) of the pass axis q.
struct StarRanges {
  int lo[4], hi[4];
  int u, v, cu, cv;
};
__device__ __forceinline__ StarRanges star_ranges(const FusedArgs &a, const PencilPos &pp) {
  StarRanges r;
  const int q = a.axis;
  r.u = q == 1 ? 0 : (q == 2 ? 0 : 1);
  r.v = q == 2 ? 1 : 2;
  const int nu = r.u == 0 ? a.nx : a.ny, nv = r.v == 1 ? a.ny : a.nz;
  r.cu = pp.c[r.u];
  r.cv = pp.c[r.v];
  const int cum = r.cu == 0 ? nu - 1 : r.cu - 1, cvm = r.cv == 0 ? nv - 1 : r.cv - 1;
  const int b[4] = {r.cu * nv + r.cv, cum * nv + r.cv, r.cu * nv + cvm, cum * nv + cvm};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    r.lo[k] = a.bstart[b[k]];
    r.hi[k] = a.bstart[b[k] + 1];
  }
  return r;
}

// Visit the stars touching this pencil; with ORDERED, in increasing star
// index (a 4-way merge of the buckets, each already in star order).  For each
// star and each of its two corners on the pencil (positions i0_q and
// i0_q + 1), f(s, corner, m, wx, wy, wz, fac) is called on the thread that
// owns position m.
template <int N, bool ORDERED, class F>
__device__ __forceinline__ void for_star_corners(const FusedArgs &a, StarRanges r, int t, int P, F &&f) {
  const int q = a.axis;
  while (true) {
    int kb = -1;
    unsigned s = 0xffffffffu;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (r.lo[k] < r.hi[k]) {
        const unsigned sk = a.perm[r.lo[k]];
        if (!ORDERED) {
          if (kb < 0) {
            kb = k;
            s = sk;
          }
        } else if (sk < s) {
          s = sk;
          kb = k;
        }
      }
    }
    if (kb < 0) break;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k == kb) r.lo[k]++;
    const int4 id = a.sidx[s];
    const float4 w0 = a.sw0[s], w1 = a.sw1[s];
    const int bu = (r.cu == sel3(id.x, id.y, id.z, r.u)) ? 0 : 1;
    const int bv = (r.cv == sel3(id.x, id.y, id.z, r.v)) ? 0 : 1;
    const int q0 = sel3(id.x, id.y, id.z, q);
#pragma unroll
    for (int cq = 0; cq < 2; ++cq) {
      int m = q0 + cq;
      if (m >= N) m -= N;
      if (m % P == t) {
        const int bx = q == 0 ? cq : (r.u == 0 ? bu : bv);
        const int by = q == 1 ? cq : (r.u == 1 ? bu : bv);
        const int bz = q == 2 ? cq : bv;
        f(s, bx + 2 * by + 4 * bz, m, bx ? w1.x : w0.x, by ? w1.y : w0.y, bz ? w1.z : w0.z, w0.w);
      }
    }
  }
}

// rho = |psi|^2 + rho_stars (+ rho_gas), element by element (float32 order
// of quantum-stars.py:299 / quantum-gas-bh.py:542).  The star density of a
// cell is summed from zero in star order in the (still zero) imaginary slot,
// then added: the order of the reference's sequential bin_stars.  Returns
// the thread's float64 partial sum of rho.
template <int N, int E>
__device__ __forceinline__ double build_density(float2 (&v)[E], const FusedArgs &a,
                                                const PencilPos &pp, int t, int P) {
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = float2{v[e].x * v[e].x + v[e].y * v[e].y, 0.0f};
  if (a.has_stars) {
    for_star_corners<N, true>(a, star_ranges(a, pp), t, P,
                              [&](unsigned, int, int m, float wx, float wy, float wz, float fac) {
                                const float val = fmul_rn(fmul_rn(fmul_rn(wx, wy), wz), fac);
                                const int e = m / P;
#pragma unroll
                                for (int qq = 0; qq < E; ++qq)
                                  if (qq == e) v[qq].y = fadd_rn(v[qq].y, val);
                              });
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = float2{v[e].x + v[e].y, 0.0f};
  }
  if (a.grho) {
#pragma unroll
    for (int e = 0; e < E; ++e)
      v[e].x = v[e].x + a.grho[(unsigned)pp.base + (unsigned)(t + P * e) * (unsigned)a.stride];
  }
  double s = 0.0;
#pragma unroll
  for (int e = 0; e < E; ++e) s += (double)v[e].x;
  return s;
}

// sin and cos of theta (float64) for the kick phase.  theta is reduced in
// float64 to r in [-pi/4, pi/4] with quadrant n = rint(2 theta / pi) and a
// two-part pi/2 (Cody-Waite); sin r and cos r are their Taylor series to
// degree 9 and 10 (truncation below 2e-10 for |r| <= pi/4), evaluated in
// float32 by Horner's rule.
__device__ __forceinline__ void sincos_reduced(double theta, float &sn, float &cs) {
  const double n = rint(theta * 0.63661977236758134308);
  const double r = (theta - n * 1.5707963267948965580e+00) - n * 6.1232339957367660359e-17;
  const float x = (float)r, x2 = x * x;
  const float s = x * (1.0f + x2 * (-1.6666667163e-01f +
                            x2 * (8.3333337680e-03f + x2 * (-1.9841270114e-04f +
                                                         x2 * 2.7557318845e-06f))));
  const float c = 1.0f + x2 * (-0.5f + x2 * (4.1666667908e-02f +
                                    x2 * (-1.3888889225e-03f + x2 * (2.4801587642e-05f +
                                                                   x2 * -2.7557318845e-07f))));
  const int q = (int)((long long)n & 3);
  sn = q == 0 ? s : (q == 1 ? c : (q == 2 ? -s : -c));
  cs = q == 0 ? c : (q == 1 ? -s : (q == 2 ? -c : s));
}

__device__ __forceinline__ float2 cmulf(float2 z, float2 d) {
  return float2{fmaf(z.x, d.x, -(z.y * d.y)), fmaf(z.x, d.y, z.y * d.x)};
}

// s + w / n (the 1/n of the inverse transform): exact scaling for powers of
// two, a correctly rounded division otherwise, so no bias builds up over steps.
template <int N>
__device__ __forceinline__ float2 add_scaled(float2 s, float2 w) {
  if constexpr ((N & (N - 1)) == 0) {
    constexpr float r = 1.0f / N;
    return float2{fmaf(w.x, r, s.x), fmaf(w.y, r, s.y)};
  } else {
    return float2{s.x + __fdiv_rn(w.x, (float)N), s.y + __fdiv_rn(w.y, (float)N)};
  }
}

// Kinetic drift of one pencil along its axis, psi <- IFFT(prop FFT(psi)),
// evaluated in increment form
//   psi <- psi + IFFT(d FFT(psi - c)),  d = prop - 1,  c = the pencil's first element.
// d(k=0) = 0 removes c exactly.  The float32 rounding of the two transforms
// then scales with |d (psi - c)| instead of |psi|: for the slowly turning
// low-k modes, whose per-step rounding would otherwise repeat step after step
// and add up linearly, it is smaller by the phase d.  The pre-transform values
// wait in the thread's own slots of `save` (no barrier needed).
template <int N, int E, int P, int THREADS, class SMV>
__device__ __forceinline__ void drift_pencil(float2 (&v)[E], float2 c, const float2 *__restrict__ prop,
                                             int t, SMV &smv, const float2 *tw, float2 *save) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    save[e * THREADS + tid] = v[e];
    v[e] = float2{v[e].x - c.x, v[e].y - c.y};
  }
  fft_pencil<N, -1, true>(v, t, smv, tw);
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = cmulf(v[e], __ldg(&prop[t + P * e]));
  fft_pencil<N, +1, true>(v, t, smv, tw);
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = add_scaled<N>(save[e * THREADS + tid], v[e]);
}

// Dynamic shared memory of a fused pass: the exchange rows, the stage twiddle
// table and, for the drift passes, THREADS x E save slots.
template <int N, bool CONTIG, int MODE>
__host__ __device__ constexpr size_t fused_smem_bytes() {
  using SH = PassShape<N, CONTIG>;
  return SH::template smem_bytes<float2>() + stage_tw_size<N>() * sizeof(float2) +
         ((MODE == M_KICK || MODE == M_DRIFT || MODE == M_DRIFT_DENSITY)
              ? (size_t)SH::THREADS * SH::E * sizeof(float2)
              : 0);
}

// exp(-i theta) * z
__device__ __forceinline__ float2 phase_rotate(float2 z, double theta) {
  float s, c;
  sincos_reduced(theta, s, c);
  return float2{z.x * c + z.y * s, z.y * c - z.x * s};
}

// Bring the tile of CTA `blk` of field f into L2 (cp.async.bulk.prefetch.L2:
// no registers, no shared memory, no completion to wait for).  Strided tiles
// are N rows of 16 complex64 (128 B); contiguous tiles are TP rows of N.
template <int N, bool CONTIG>
__device__ __forceinline__ void prefetch_tile(const float2 *f, const FusedArgs &a, int blk) {
  using SH = PassShape<N, CONTIG>;
  const int tid = threadIdx.x;
  if (CONTIG) {
    if (tid < SH::TP) {
      const float2 *row = f + (long long)(blk * SH::TP + tid) * a.nz;
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(row), "r"(N * 8) : "memory");
    }
  } else {
    for (int i = tid; i < N; i += SH::THREADS) {
      const int o = blk / a.ztiles;
      const float2 *row = f + (long long)o * a.outer_stride + (blk % a.ztiles) * 16 + (long long)i * a.stride;
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], 128;" ::"l"(row) : "memory");
    }
  }
}

template <int N, bool CONTIG, int MODE>
__global__ void __launch_bounds__(PassShape<N, CONTIG>::THREADS, PassShape<N, CONTIG>::MINB)
    k_fused(FusedArgs a) {
  select_box(a);
  if (a.ahead > 0 && (int)blockIdx.x + a.ahead < (int)gridDim.x) {
    const int nb = blockIdx.x + a.ahead;
    if constexpr (MODE == M_DENSITY || MODE == M_DRIFT || MODE == M_DRIFT_DENSITY) {
      prefetch_tile<N, CONTIG>(a.psi, a, nb);
    } else if constexpr (MODE == M_FFT_FWD || MODE == M_POISSON) {
      prefetch_tile<N, CONTIG>(a.R, a, nb);
    } else if constexpr (MODE == M_IFFT2) {
      prefetch_tile<N, CONTIG>(a.S1, a, nb);
      prefetch_tile<N, CONTIG>(a.S2, a, nb);
    } else if constexpr (MODE == M_KICK) {
      prefetch_tile<N, CONTIG>(a.S1, a, nb);
      prefetch_tile<N, CONTIG>(a.S2, a, nb);
      prefetch_tile<N, CONTIG>(a.psi, a, nb);
    }
  }
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
  // the stage twiddle table of this axis, staged after the exchange rows
  float2 *tw_s = sm + SH::template smem_bytes<float2>() / sizeof(float2);
  for (int i = tid; i < stage_tw_size<N>(); i += THREADS) tw_s[i] = a.tw[i];
  __syncthreads();
  const float2 *tw = tw_s;
  float2 *save = tw_s + stage_tw_size<N>();  // drift passes: per-thread slots

  if constexpr (MODE == M_DENSITY) {
    float2 v[E];
    load_pencil<E>(v, a.psi, base, st, t, P);
    double s = build_density<N, E>(v, a, pp, t, P);
    s = block_sum<THREADS>(s, red);
    if (tid == 0) a.part[blockIdx.x] = s;
    fft_pencil<N, -1, true>(v, t, smv, tw);
    store_pencil<E>(v, a.R, base, st, t, P);
  } else if constexpr (MODE == M_FFT_FWD) {
    float2 v[E];
    load_pencil<E>(v, a.R, base, st, t, P);
    fft_pencil<N, -1, true>(v, t, smv, tw);
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
    fft_pencil<N, -1, true>(v, t, smv, tw);
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
    fft_pencil<N, +1, true>(v, t, smv, tw);
    store_pencil<E>(v, a.S1, base, st, t, P);
    fft_pencil<N, +1, true>(w, t, smv, tw);
    store_pencil<E>(w, a.S2, base, st, t, P);
  } else if constexpr (MODE == M_IFFT2) {
    float2 v[E];
    load_pencil<E>(v, a.S1, base, st, t, P);
    fft_pencil<N, +1, true>(v, t, smv, tw);
    store_pencil<E>(v, a.S1, base, st, t, P);
    load_pencil<E>(v, a.S2, base, st, t, P);
    fft_pencil<N, +1, true>(v, t, smv, tw);
    store_pencil<E>(v, a.S2, base, st, t, P);
  } else if constexpr (MODE == M_KICK) {
    const int aq = a.axis;  // the kick axis; ar = 2 - aq is the Poisson axis
    const unsigned gb = (unsigned)base + (unsigned)t * (unsigned)st, gs = (unsigned)P * (unsigned)st;
    float am = 0.0f;
    float V[E];
    {
      // phase 1: S1 -> V + i a_r
      float2 v1[E];
      load_pencil<E>(v1, a.S1, base, st, t, P);
      fft_pencil<N, +1, true>(v1, t, smv, tw);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        V[e] = v1[e].x;
        am = fmaxf(am, fabsf(v1[e].y));
      }
      if (a.has_stars)
        for_star_corners<N, false>(a, star_ranges(a, pp), t, P,
                                   [&](unsigned s, int cbits, int m, float, float, float, float) {
                                     const float ar_ = reg_get<E>(v1, m / P).y;
                                     a.A[3 * (8 * s + c_corner_of_bits_dev(cbits)) + (aq == 0 ? 2 : 0)] = ar_;
                                   });
      if (a.gv[0]) {  // gas half kick, quantum-gas-bh.py:255-266
        float *g = a.gv[aq == 0 ? 2 : 0];
#pragma unroll
        for (int e = 0; e < E; ++e) g[gb + e * gs] = g[gb + e * gs] + v1[e].y * a.gas_dt;
      }
    }
    {
      // phase 2: S2 -> a_q + i a_y
      float2 v2[E];
      load_pencil<E>(v2, a.S2, base, st, t, P);
      fft_pencil<N, +1, true>(v2, t, smv, tw);
#pragma unroll
      for (int e = 0; e < E; ++e) am = fmaxf(am, fmaxf(fabsf(v2[e].x), fabsf(v2[e].y)));
      if (a.has_stars)
        for_star_corners<N, false>(a, star_ranges(a, pp), t, P,
                                   [&](unsigned s, int cbits, int m, float, float, float, float) {
                                     const float2 w = reg_get<E>(v2, m / P);
                                     float *dst = a.A + 3 * (8 * s + c_corner_of_bits_dev(cbits));
                                     dst[aq] = w.x;
                                     dst[1] = w.y;
                                   });
      if (a.gv[0]) {
        float *gq = a.gv[aq], *gy = a.gv[1];
#pragma unroll
        for (int e = 0; e < E; ++e) {
          gq[gb + e * gs] = gq[gb + e * gs] + v2[e].x * a.gas_dt;
          gy[gb + e * gs] = gy[gb + e * gs] + v2[e].y * a.gas_dt;
        }
      }
    }
    // phase 3: psi <- exp(-i c V) psi with V = Poisson + b rho + V_ext, then
    // the drift along this axis
    float2 ps[E];
    load_pencil<E>(ps, a.psi, base, st, t, P);
    if (a.b_coeff != 0.0f) {
      // rho = |psi|^2 + rho_stars, the argument of get_potential (quantum-stars.py:193)
      float rs[E];
#pragma unroll
      for (int e = 0; e < E; ++e) rs[e] = 0.0f;
      if (a.has_stars)
        for_star_corners<N, true>(a, star_ranges(a, pp), t, P,
                                  [&](unsigned, int, int m, float wx, float wy, float wz, float fac) {
                                    const float val = fmul_rn(fmul_rn(fmul_rn(wx, wy), wz), fac);
                                    const int e = m / P;
#pragma unroll
                                    for (int qq = 0; qq < E; ++qq)
                                      if (qq == e) rs[qq] = fadd_rn(rs[qq], val);
                                  });
#pragma unroll
      for (int e = 0; e < E; ++e)
        V[e] = V[e] + a.b_coeff * (ps[e].x * ps[e].x + ps[e].y * ps[e].y + rs[e]);
    }
    if (a.v_ext) {
#pragma unroll
      for (int e = 0; e < E; ++e) V[e] = V[e] + a.v_ext[gb + e * gs];
    }
#pragma unroll
    for (int e = 0; e < E; ++e) ps[e] = phase_rotate(ps[e], a.kick_coef * (double)V[e]);
    if (a.v_out) {
#pragma unroll
      for (int e = 0; e < E; ++e) a.v_out[gb + e * gs] = V[e];
    }
    if (a.do_drift) {
      // read before any thread of this pencil stores (the FFT's barriers order it)
      const float2 c0 = a.psi[base];
      drift_pencil<N, E, P, THREADS>(ps, c0, a.prop, t, smv, tw, save);
    }
    store_pencil<E>(ps, a.psi, base, st, t, P);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) am = fmaxf(am, __shfl_xor_sync(0xffffffffu, am, o));
    if ((tid & 31) == 0) atomic_max_nonneg(a.amax_bits, am);
  } else if constexpr (MODE == M_DEPOSIT) {
    // bin_stars (quantum-stars.py:212-247): every cell sums its star
    // contributions from zero in star order
    float acc[E];
#pragma unroll
    for (int e = 0; e < E; ++e) acc[e] = 0.0f;
    if (a.has_stars)
      for_star_corners<N, true>(a, star_ranges(a, pp), t, P,
                                [&](unsigned, int, int m, float wx, float wy, float wz, float fac) {
                                  const float val = fmul_rn(fmul_rn(fmul_rn(wx, wy), wz), fac);
                                  const int e = m / P;
#pragma unroll
                                  for (int qq = 0; qq < E; ++qq)
                                    if (qq == e) acc[qq] = fadd_rn(acc[qq], val);
                                });
    const unsigned gb = (unsigned)base + (unsigned)t * (unsigned)st, gs = (unsigned)P * (unsigned)st;
#pragma unroll
    for (int e = 0; e < E; ++e) a.rho_out[gb + e * gs] = acc[e];
    (void)smv;
    (void)tw;
  } else if constexpr (MODE == M_DRIFT || MODE == M_DRIFT_DENSITY) {
    float2 v[E];
    load_pencil<E>(v, a.psi, base, st, t, P);
    // read before any thread of this pencil stores (the FFT's barriers order it)
    const float2 c0 = a.psi[base];
    drift_pencil<N, E, P, THREADS>(v, c0, a.prop, t, smv, tw, save);
    store_pencil<E>(v, a.psi, base, st, t, P);
    if constexpr (MODE == M_DRIFT_DENSITY) {
      double s = build_density<N, E>(v, a, pp, t, P);
      s = block_sum<THREADS>(s, red);
      if (tid == 0) a.part[blockIdx.x] = s;
      fft_pencil<N, -1, true>(v, t, smv, tw);
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
