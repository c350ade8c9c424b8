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
// Adjoint of the kick (reverse sweep), along z, around FFT_FWD / POISSON /
// IFFT2 of the same source:
//   ADJ_SOURCE     g, psi, V -> mu = c Im(conj(g) e^{-icV} psi) -> FFT_z -> R
//   ADJ_UPDATE     S1 -> IFFT_z -> W; g <- e^{icV} g + 2 (W + b mu) psi; the
//                  drift adjoint along z (the propagator of -dt)
#pragma once

#include <cuda.h>

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
  M_ADJ_SOURCE = 8,
  M_ADJ_UPDATE = 9,
};

struct FusedArgs {
  int nx, ny, nz;
  int axis;                // 0, 1, 2
  long long stride;        // element stride along the axis
  long long outer_stride;  // strided passes: stride of the outer index
  int ztiles;              // strided passes: nz / (z columns of a tile)
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
  const unsigned *pmask;  // bit per pencil: some star touches it (clear for most)
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
  // Uniform part of the potential (the k = 0 offset -4 pi G (mean rho - rho_bar)),
  // kept out of the float32 kicks: POISSON adds phi_coef * V0 to *phi (float64,
  // per box) instead of putting V0 into V; the call's last KICK (phi_final)
  // adds *phi to its phase.  A uniform V only turns the global phase, which
  // float32 cannot follow in sub-ulp steps (it biases |psi|).
  double *phi;
  double phi_coef;
  int phi_final;
  // a fixed density added to |psi|^2 in every density build and in the
  // self-interaction term (single box; the star density as a given source)
  const float *rho_src;
  // adjoint passes: the state before the kick (psi is the adjoint g), the
  // kick's potential, and mu (written by ADJ_SOURCE, read by ADJ_UPDATE;
  // only with self-interaction)
  const float2 *adj_pre;
  const float *adj_V;
  float *adj_mu;
  // isothermal gas
  const float *grho;
  float *gv[3];
  float gas_dt;
  // tiles of this pass per box (the persistent CTAs stride over them)
  int ntiles;
  // shape variant of the pass (PassShape's V: radix plan, tile width); set
  // with the fields that follow from it (tw, ztiles)
  int shape;
  // host side only: launch the pass as a programmatic dependent of the kernel
  // before it on the stream (that kernel must be a fused pass of this step)
  int pdl;
  // forward y / Poisson passes over half of the real density's spectrum (the
  // other non-y axis to n/2); the Poisson pass then also writes the mirrors
  int half;
  int hq;       // the half axis q (0 or 2)
  int full_nx;  // nx of the grid (nx itself may hold a pass's reduced range)
  // walk the tiles from the last: a pass then first reads what the previous
  // pass wrote last, which is still in L2
  int rev;
  // host side only: the plan's launch tuning (QJ_TUNE_* of include/qj.h)
  const int *tune;
  // set to nonzero when a pass gave up waiting for a tile copy
  unsigned *err;
  // batched boxes (the CTA's box()): per-box strides of the fields (cells),
  // stars, bucket starts, partial sums; a_max is per box
  int nbox;  // launch grid.y (0 or 1 = one box)
  long long box_cells;
  int box_stars;
  int box_bstart;
  int box_part;
};

// A CTA's place in its pass: box box(), slot bx() of the gx() persistent
// CTAs that stride over that box's tiles.  k_fused reads them from its grid
// (GridCta: blockIdx.y, blockIdx.x, gridDim.x, re-read where used, as the
// special registers they are); an ensemble launch's CTAs claim tiles instead
// (DynCta).
struct GridCta {
  static constexpr bool DYN = false;
  __device__ __forceinline__ int bx() const { return (int)blockIdx.x; }
  __device__ __forceinline__ int box() const { return (int)blockIdx.y; }
  __device__ __forceinline__ int gx() const { return (int)gridDim.x; }
};
// A CTA of an ensemble launch that claims the tiles of box box() one at a
// time from that box's counter (zeroed before the launch): every CTA of the
// launch that works on the box takes its next tile from the same counter, so
// the box's tiles are shared out as the CTAs finish their previous ones.
// Thread 0 claims (one atomicAdd) one tile ahead of the one it starts to
// copy, so the claim's round trip overlaps a tile's work, and publishes the
// tile to start in a shared-memory word; a claim of ntiles or more means the
// box has no tiles left (and every later claim of the CTA is past it too).
struct DynCta {
  static constexpr bool DYN = true;
  int box_;
  unsigned *ctr;
  int *slot;
  __device__ __forceinline__ int box() const { return box_; }
  __device__ __forceinline__ int claim() const { return (int)atomicAdd(ctr, 1u); }
  __device__ __forceinline__ void publish(int tile) const { *(volatile int *)slot = tile; }
  __device__ __forceinline__ int claimed() const { return *(volatile int *)slot; }
};

// Offset a pass' pointers to box b of a batched plan.
__device__ __forceinline__ void select_box(FusedArgs &a, int b) {
  if (b == 0) return;
  const long long c = (long long)b * a.box_cells;
  if (a.psi) a.psi += c;
  if (a.R) a.R += c;
  if (a.S1) a.S1 += c;
  if (a.S2) a.S2 += c;
  if (a.part) a.part += (long long)b * a.box_part;
  if (a.part_in) a.part_in += (long long)b * a.box_part;
  if (a.amax_bits) a.amax_bits += b;
  if (a.phi) a.phi += b;
  const long long s = (long long)b * a.box_stars;
  if (a.sidx) a.sidx += s;
  if (a.sw0) a.sw0 += s;
  if (a.sw1) a.sw1 += s;
  if (a.perm) a.perm += s;
  if (a.A) a.A += 24 * s;
  if (a.bstart) a.bstart += (long long)b * a.box_bstart;
  if (a.pmask) a.pmask += (long long)b * ((a.box_bstart + 31) / 32);
}

// Whether any star touches pencil pid (one bit of the pencil mask).
__device__ __forceinline__ bool pencil_has_stars(const FusedArgs &a, int pid) {
  return (a.pmask[pid >> 5] >> (pid & 31)) & 1u;
}

// Per-thread position of a pencil in the grid.
struct PencilPos {
  long long base;  // linear index of element 0 of the pencil
  int pid;         // pencil id in this axis' orientation
  int c[3];        // coordinates (the axis' own entry is unused)
};

template <bool CONTIG>
__device__ __forceinline__ PencilPos pencil_pos(const FusedArgs &a, int tile, int p, int TP) {
  PencilPos pp;
  if (CONTIG) {  // axis 2: rows x * ny + y
    const int row = tile * TP + p;
    pp.pid = row;
    pp.base = (long long)row * a.nz;
    pp.c[0] = row / a.ny;
    pp.c[1] = row % a.ny;
    pp.c[2] = 0;
  } else {
    const int o = tile / a.ztiles;
    const int z = (tile % a.ztiles) * TP + p;
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
// Store a thread's E elements t + P e of a pencil.  WIDE: one base pointer
// plus a 64-bit constant multiple of the element step per store; otherwise a
// 32-bit element index per store.  The two compile to different code; each
// pass uses the one measured faster for it.
template <int E, bool WIDE = true, typename C>
__device__ __forceinline__ void store_pencil(const C (&v)[E], C *__restrict__ f, long long base,
                                             long long stride, int t, int P) {
  const unsigned b = (unsigned)base + (unsigned)t * (unsigned)stride;
  const unsigned s = (unsigned)P * (unsigned)stride;
  if constexpr (WIDE) {
    C *__restrict__ q = f + b;
#pragma unroll
    for (int e = 0; e < E; ++e) q[(unsigned long long)s * (unsigned)e] = v[e];
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e) f[b + (unsigned)e * s] = v[e];
  }
}

// store_pencil of the elements t + P e <= N / 2 only: the half of a real
// field's spectrum the passes after it read.
template <int N, int E, typename C>
__device__ __forceinline__ void store_pencil_half(const C (&v)[E], C *__restrict__ f, long long base,
                                                  long long stride, int t, int P) {
  C *__restrict__ q = f + ((unsigned)base + (unsigned)t * (unsigned)stride);
  const unsigned s = (unsigned)P * (unsigned)stride;
#pragma unroll
  for (int e = 0; e < E; ++e)
    if (2 * (t + P * e) <= N) q[(unsigned long long)s * (unsigned)e] = v[e];
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
__device__ __forceinline__ void star_buckets(const FusedArgs &a, const PencilPos &pp, StarRanges &r,
                                             int (&b)[4]) {
  const int q = a.axis;
  r.u = q == 1 ? 0 : (q == 2 ? 0 : 1);
  r.v = q == 2 ? 1 : 2;
  const int nu = r.u == 0 ? a.nx : a.ny, nv = r.v == 1 ? a.ny : a.nz;
  r.cu = r.u == 0 ? pp.c[0] : pp.c[1];
  r.cv = r.v == 1 ? pp.c[1] : pp.c[2];
  const int cum = r.cu == 0 ? nu - 1 : r.cu - 1, cvm = r.cv == 0 ? nv - 1 : r.cv - 1;
  b[0] = r.cu * nv + r.cv;
  b[1] = cum * nv + r.cv;
  b[2] = r.cu * nv + cvm;
  b[3] = cum * nv + cvm;
}
__device__ __forceinline__ StarRanges star_ranges(const FusedArgs &a, const PencilPos &pp) {
  StarRanges r;
  int b[4];
  star_buckets(a, pp, r, b);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    r.lo[k] = a.bstart[b[k]];
    r.hi[k] = a.bstart[b[k] + 1];
  }
  return r;
}
// Empty ranges: for_star_corners visits nothing.
__device__ __forceinline__ StarRanges no_star_ranges() {
  StarRanges r;
#pragma unroll
  for (int k = 0; k < 4; ++k) r.lo[k] = r.hi[k] = 0;
  r.u = r.v = r.cu = r.cv = 0;
  return r;
}

// Visit the stars touching this pencil; with ORDERED, in increasing star
// index (a 4-way merge of the buckets, each already in star order), else
// bucket by bucket.  For each star and each of its two corners on the pencil
// (positions i0_q and i0_q + 1), f(s, corner, m, wx, wy, wz, fac) is called on
// the thread that owns position m.
template <int N, bool ORDERED, class F>
__device__ __forceinline__ void for_star_corners(const FusedArgs &a, StarRanges r, int t, int P, F &&f) {
  const int q = a.axis;
  while (true) {
    int kb = -1;
    unsigned s = 0xffffffffu;
    if constexpr (ORDERED) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (r.lo[k] < r.hi[k]) {
          const unsigned sk = a.perm[r.lo[k]];
          if (sk < s) {
            s = sk;
            kb = k;
          }
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (kb < 0 && r.lo[k] < r.hi[k]) kb = k;
    }
    if (kb < 0) break;
    int j = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k == kb) j = r.lo[k]++;
    if constexpr (!ORDERED) s = a.perm[j];
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

// The kick's star corners: f(s, corner, slot, m) for each corner of each
// star on this pencil, at element m of the pencil, where slot indexes the
// save slots ([E][THREADS], written by the corners' owners) at that cell.  The writes f makes do not
// depend on their order (each star corner and axis has one writer).  Along z
// (CONTIG) a pencil's P threads sit in one warp and split its stars between
// them, one lookup per star instead of one per thread; the caller syncs the
// pencil's lanes around the call (pencil_lanes).  Along x / y the pencil's
// threads span several warps, and each corner's owner visits it.
__device__ __forceinline__ unsigned pencil_lanes(int P) {
  const int lane = threadIdx.x & 31;
  return P >= 32 ? 0xffffffffu : (((1u << P) - 1u) << ((lane / P) * P));
}
template <int N, bool CONTIG, int THREADS, class F>
__device__ __forceinline__ void kick_star_corners(const FusedArgs &a, const StarRanges &r, int t,
                                                  int P, F &&f) {
  const int tid = threadIdx.x;
  if constexpr (!CONTIG) {
    for_star_corners<N, false>(a, r, t, P, [&](unsigned s, int cbits, int m, float, float, float, float) {
      f(s, cbits, (m / P) * THREADS + tid, m);
    });
  } else {
    const int q = a.axis, base = tid - t;
    const int n0 = r.hi[0] - r.lo[0], n1 = r.hi[1] - r.lo[1], n2 = r.hi[2] - r.lo[2];
    const int total = n0 + n1 + n2 + (r.hi[3] - r.lo[3]);
    for (int j = t; j < total; j += P) {
      const int idx = j < n0               ? r.lo[0] + j
                      : j < n0 + n1        ? r.lo[1] + (j - n0)
                      : j < n0 + n1 + n2   ? r.lo[2] + (j - n0 - n1)
                                           : r.lo[3] + (j - n0 - n1 - n2);
      const unsigned s = a.perm[idx];
      const int4 id = a.sidx[s];
      const int bu = (r.cu == sel3(id.x, id.y, id.z, r.u)) ? 0 : 1;
      const int bv = (r.cv == sel3(id.x, id.y, id.z, r.v)) ? 0 : 1;
      const int q0 = sel3(id.x, id.y, id.z, q);
#pragma unroll
      for (int cq = 0; cq < 2; ++cq) {
        int m = q0 + cq;
        if (m >= N) m -= N;
        const int bx = q == 0 ? cq : (r.u == 0 ? bu : bv);
        const int by = q == 1 ? cq : (r.u == 1 ? bu : bv);
        const int bz = q == 2 ? cq : bv;
        f(s, bx + 2 * by + 4 * bz, (m / P) * THREADS + base + (m % P), m);
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
                                                const PencilPos &pp, const StarRanges &sr, int t,
                                                int P) {
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = float2{v[e].x * v[e].x + v[e].y * v[e].y, 0.0f};
  if (a.has_stars) {
    for_star_corners<N, true>(a, sr, t, P,
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
  if (a.rho_src) {
#pragma unroll
    for (int e = 0; e < E; ++e)
      v[e].x = v[e].x + a.rho_src[(unsigned)pp.base + (unsigned)(t + P * e) * (unsigned)a.stride];
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
// float32 by Horner's rule.  For |theta| < 2^-10 (the kick phase of most cells
// at small dt) no reduction is needed: theta - theta^3/6 and 1 - theta^2/2
// leave out terms below 2^-46 relative, far under a float32 ulp.
__device__ __forceinline__ void sincos_reduced(double theta, float &sn, float &cs) {
  if (fabs(theta) < 0x1p-10) {
    const float x = (float)theta, x2 = x * x;
    sn = x * fmaf(x2, -1.6666667163e-01f, 1.0f);
    cs = fmaf(x2, -0.5f, 1.0f);
    return;
  }
  // n = the integer nearest 2 theta / pi, by adding 1.5 * 2^52 (|2 theta / pi|
  // < 2^51): the sum's low word is n in two's complement, so the quadrant
  // needs no conversion.  (A product within an ulp of a half-integer may round
  // the other way than rint of the rounded product; r then lies a hair beyond
  // pi/4, where the series is still accurate.)
  const double nm = fma(theta, 0.63661977236758134308, 6755399441055744.0);
  const int qn = __double2loint(nm);
  const double n = nm - 6755399441055744.0;
  const double r = (theta - n * 1.5707963267948965580e+00) - n * 6.1232339957367660359e-17;
  const float x = (float)r, x2 = x * x;
  const float s = x * (1.0f + x2 * (-1.6666667163e-01f +
                            x2 * (8.3333337680e-03f + x2 * (-1.9841270114e-04f +
                                                         x2 * 2.7557318845e-06f))));
  const float c = 1.0f + x2 * (-0.5f + x2 * (4.1666667908e-02f +
                                    x2 * (-1.3888889225e-03f + x2 * (2.4801587642e-05f +
                                                                   x2 * -2.7557318845e-07f))));
  const int q = qn & 3;
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
__device__ __forceinline__ void drift_pencil(float2 (&v)[E], float2 c, const float2 *prop,
                                             int t, SMV &smv, const float2 *tw, float2 *save) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    save[e * THREADS + tid] = v[e];
    v[e] = float2{v[e].x - c.x, v[e].y - c.y};
  }
  fft_pencil<N, -1, true>(v, t, smv, tw);
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = cmulf(v[e], prop[t + P * e]);
  fft_pencil<N, +1, true>(v, t, smv, tw);
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = add_scaled<N>(save[e * THREADS + tid], v[e]);
}

// exp(-i theta) * z
__device__ __forceinline__ float2 phase_rotate(float2 z, double theta) {
  float s, c;
  sincos_reduced(theta, s, c);
  return float2{z.x * c + z.y * s, z.y * c - z.x * s};
}

// ---------------------------------------------------------------------------
// Streaming tiles through shared memory.
//
// The CTAs of a pass are persistent (tile = bx + k gx, see GridCta).  A
// pass reads its input fields tile by tile through one landing buffer: while
// the CTA transforms one field of one tile, bulk copies (cp.async.bulk into
// this CTA's own shared memory, completion counted in bytes on an mbarrier)
// bring in the next one, i.e. the next field of the same tile or the first
// field of the CTA's next tile.  HBM reads thus overlap the in-register
// transforms instead of alternating with them.

// Landing buffer of one tile.  Contiguous tiles (z pencils) land as one row
// per pencil, padded by P elements when P < 16 so that the lanes of the
// different pencils in a warp read different banks; strided tiles land as N
// rows of the TP pencils' elements (TP x 8 B each: 128 B, or 64 B for the
// narrow tile variant), the dense box of a tensor-map copy.  Every copy is a
// multiple of 16 bytes and starts on a 16-byte boundary.
template <int N, bool CONTIG, int V = 0> struct Landing {
  using SH = PassShape<N, CONTIG, V>;
  static constexpr int PAD = CONTIG ? (SH::P >= 16 ? 0 : (SH::P >= 2 ? SH::P : 2)) : 0;
  static constexpr int ROWS = CONTIG ? SH::TP : N;       // bulk copies per tile
  static constexpr int ROW_ELEMS = CONTIG ? N : SH::TP;  // complex64 per copy
  static constexpr int ROW_STRIDE = CONTIG ? N + PAD : SH::TP;
  static constexpr size_t BYTES = (size_t)ROWS * ROW_STRIDE * sizeof(float2);
  static constexpr unsigned TX = (unsigned)ROWS * ROW_ELEMS * (unsigned)sizeof(float2);
  static_assert((ROW_STRIDE * sizeof(float2)) % 16 == 0, "landing rows must stay 16-byte aligned");
  static_assert(TX < (1u << 20), "tile larger than an mbarrier transaction count");
  __device__ static __forceinline__ int idx(int p, int i) {
    return CONTIG ? p * ROW_STRIDE + i : i * SH::TP + p;
  }
};

// Dynamic shared memory of a fused pass: the exchange rows, the stage twiddle
// table, the pass axis' own tables, THREADS x E per-thread save slots (drift
// and Poisson passes) and the landing buffer.
template <int N, bool CONTIG, int MODE, int V = 0> struct FusedSmem {
  using SH = PassShape<N, CONTIG, V>;
  static constexpr bool DRIFTS =
      MODE == M_KICK || MODE == M_DRIFT || MODE == M_DRIFT_DENSITY || MODE == M_ADJ_UPDATE;
  static constexpr bool LANDS = MODE != M_DEPOSIT;
  static constexpr bool SAVES = DRIFTS || MODE == M_POISSON || MODE == M_IFFT2;
  static constexpr size_t a16(size_t x) { return (x + 15) & ~(size_t)15; }
  // per-axis tables: the drift propagator (N complex) or k and k~ (2 N floats)
  static constexpr size_t TAB_BYTES = DRIFTS ? N * sizeof(float2)
                                      : (MODE == M_POISSON ? 2 * N * sizeof(float)
                                                           : (MODE == M_IFFT2 ? N * sizeof(float) : 0));
  static constexpr size_t TW = a16(SH::template smem_bytes<float2>());
  static constexpr size_t TAB = a16(TW + (size_t)stage_tw_size<N, SH::RV>() * sizeof(float2));
  static constexpr size_t SAVE = a16(TAB + TAB_BYTES);
  static constexpr size_t LAND =
      a16(SAVE + (SAVES ? (size_t)SH::THREADS * SH::E * sizeof(float2) : 0));
  // + slack to round the landing buffer up to a 128-byte boundary (tensor copies)
  static constexpr size_t TOTAL = LAND + (LANDS ? Landing<N, CONTIG, V>::BYTES + 128 : 0);
};
template <int N, bool CONTIG, int MODE, int V = 0>
__host__ __device__ constexpr size_t fused_smem_bytes() {
  return FusedSmem<N, CONTIG, MODE, V>::TOTAL;
}

// The input fields a pass streams, in order of use.
template <int MODE> __host__ __device__ constexpr int stream_count() {
  return (MODE == M_KICK || MODE == M_ADJ_UPDATE) ? 3
         : (MODE == M_IFFT2 || MODE == M_ADJ_SOURCE) ? 2
         : (MODE == M_DEPOSIT ? 0 : 1);
}
template <int MODE>
__host__ __device__ __forceinline__ const float2 *stream_field(const FusedArgs &a, int f) {
  if constexpr (MODE == M_KICK) return f == 0 ? a.S2 : (f == 1 ? a.S1 : a.psi);
  if constexpr (MODE == M_ADJ_SOURCE) return f == 0 ? a.psi : a.adj_pre;
  if constexpr (MODE == M_ADJ_UPDATE) return f == 0 ? a.S1 : (f == 1 ? a.psi : a.adj_pre);
  if constexpr (MODE == M_IFFT2) return f == 0 ? a.S1 : a.S2;
  if constexpr (MODE == M_FFT_FWD || MODE == M_POISSON) return a.R;
  return a.psi;
}

// Strided passes: one tiled tensor map per streamed field, over the
// (z, y, x, box) array of complex64 (8-byte elements), whose box is the
// tile's z columns (16, or 8) by up to 256 rows along the pass axis.  One copy
// instruction then brings a whole tile (two for n = 512).
struct TileMaps {
  CUtensorMap m[3];
};

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait for phase `parity` of the landing barrier: gives up after
// limit_ns (2 s by default) or 2^24 polls and returns false, so a copy that
// never completes cannot hang the GPU.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity,
                                                  unsigned long long limit_ns = 2000000000ull) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned i = 0; i < (1u << 24); ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > limit_ns) break;
  }
  return false;
}

template <bool CONTIG>
__device__ __forceinline__ long long tile_origin(const FusedArgs &a, int tile, int TP) {
  if (CONTIG) return (long long)tile * TP * a.nz;
  return (long long)(tile / a.ztiles) * a.outer_stride + (long long)(tile % a.ztiles) * TP;
}

// Start the copies of streamed field f's tile into the landing buffer (warp
// 0 only).  Contiguous tiles: one bulk copy per pencil row.  Strided tiles:
// the field's tensor map, coordinates (z0, y, x, box) with the pass axis
// starting at row h.
template <int N, bool CONTIG, int MODE, int V>
__device__ __forceinline__ void issue_tile(const FusedArgs &a, const TileMaps &maps, int f, int tile,
                                           int box, float2 *land, unsigned long long *bar) {
  using L = Landing<N, CONTIG, V>;
  constexpr int T = PassShape<N, CONTIG, V>::THREADS, TP = PassShape<N, CONTIG, V>::TP;
  constexpr unsigned MASK = T >= 32 ? 0xffffffffu : ((1u << T) - 1u);
  const int lane = threadIdx.x & 31;
  if (lane == 0) {
    // order the buffer's earlier generic-proxy reads before the async writes
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, L::TX);
  }
  if constexpr (CONTIG) {
    __syncwarp(MASK);
    const float2 *fld = stream_field<MODE>(a, f);
    const long long o = tile_origin<CONTIG>(a, tile, TP);
    for (int r = lane; r < L::ROWS; r += 32) {
      const float2 *src = fld + o + (long long)r * a.nz;
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_addr(land + r * L::ROW_STRIDE)),
          "l"(src), "r"((unsigned)(L::ROW_ELEMS * sizeof(float2))), "r"(smem_addr(bar))
          : "memory");
    }
  } else {
    if (lane == 0) {
      const int z0 = (tile % a.ztiles) * TP, o = tile / a.ztiles;
      const unsigned long long map = reinterpret_cast<unsigned long long>(&maps.m[f]);
#pragma unroll
      for (int h = 0; h < N; h += 256) {
        const int cy = a.axis == 0 ? o : h, cx = a.axis == 0 ? h : o;
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(land + h * TP)),
            "l"(map), "r"(z0), "r"(cy), "r"(cx), "r"(box), "r"(smem_addr(bar))
            : "memory");
      }
    }
  }
}

// Take the current field's tile from the landing buffer: wait for it, copy
// this thread's elements (and element 0 of its pencil, c0), release the
// buffer to the next copy and start that copy.  Returns false on every
// thread of the CTA if the wait gave up (the error word is set).
template <int N, bool CONTIG, int MODE, int V, int E, class CTA>
__device__ __forceinline__ bool take_tile(float2 (&v)[E], float2 &c0, const FusedArgs &a,
                                          const TileMaps &maps, float2 *land,
                                          unsigned long long *bar, unsigned &parity, int &f, int tile,
                                          int p, int t, const CTA &cta, int &ahead) {
  using L = Landing<N, CONTIG, V>;
  constexpr int P = N / E, NF = stream_count<MODE>();
  bool ok = mbar_wait_bounded(bar, parity);
  if (ok) {
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = land[L::idx(p, t + P * e)];
    c0 = land[L::idx(p, 0)];
  }
  ok = __syncthreads_and(ok);
  parity ^= 1u;
  if (!ok) {
    if (threadIdx.x == 0) {
      if (a.err) atomicOr(a.err, 1u);
      // a copy still in flight would land in this CTA's shared memory: give
      // it one more bounded wait before the CTA (kept alive by this thread)
      // leaves
      mbar_wait_bounded(bar, parity ^ 1u, 1000000000ull);
    }
    return false;
  }
  // tile here is the loop index; the copy goes to its logical tile
  int nf = f + 1, nt = tile;
  if (nf == NF) {
    nf = 0;
    if constexpr (CTA::DYN) {
      // the CTA's next tile is the one thread 0 claimed ahead: published for
      // warp 0's copy and for every thread after the tile (next_tile); the
      // claim after it goes out now and is waited for at the next tile
      nt = a.ntiles;
      if (threadIdx.x < 32) {
        if (threadIdx.x == 0) {
          cta.publish(ahead);
          ahead = cta.claim();
        }
        __syncwarp();
        nt = cta.claimed();
      }
    } else {
      nt = tile + cta.gx();
    }
  }
  f = nf;
  if (nt < a.ntiles && threadIdx.x < 32)
    issue_tile<N, CONTIG, MODE, V>(a, maps, nf, a.rev ? a.ntiles - 1 - nt : nt, cta.box(), land, bar);
  return true;
}

// The loop index of a CTA's next tile.  A claiming CTA reads the claim its
// thread 0 made when it started the next tile's first copy (in the tile's
// last take_tile); the barrier makes it visible, and no thread can reach the
// next claim before every thread has read this one (take_tile's barrier).
template <class CTA> __device__ __forceinline__ int next_tile(int it, const CTA &cta) {
  if constexpr (CTA::DYN) {
    __syncthreads();
    return cta.claimed();
  } else {
    return it + cta.gx();
  }
}

// The body of a fused pass for one CTA: k_fused runs it with the CTA's own
// grid position; an ensemble launch runs the body of each CTA's size class.
// maps must live in parameter space (__grid_constant__) or global memory:
// the tile copies take its address.
template <int N, bool CONTIG, int MODE, int SV, class CTA>
__device__ __forceinline__ void fused_body(FusedArgs &a, const TileMaps &maps, const CTA cta) {
  select_box(a, cta.box());
  using SH = PassShape<N, CONTIG, SV>;
  using LAY = FusedSmem<N, CONTIG, MODE, SV>;
  constexpr int E = SH::E, P = SH::P, TP = SH::TP, THREADS = SH::THREADS;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float2 *sm = reinterpret_cast<float2 *>(smem_raw);
  float2 *tw_s = reinterpret_cast<float2 *>(smem_raw + LAY::TW);
  float2 *save = reinterpret_cast<float2 *>(smem_raw + LAY::SAVE);  // per-thread slots
  // the drift propagator, staged once per CTA: read from shared memory by
  // every pencil (from global memory, through L1 beside the spill traffic, it
  // cost the kick 6 us and the y drift 4.5 us at 256^3)
  float2 *tab2 = reinterpret_cast<float2 *>(smem_raw + LAY::TAB);
  float *tabk = reinterpret_cast<float *>(smem_raw + LAY::TAB);    // Poisson: k, then k~
  float2 *land = reinterpret_cast<float2 *>(
      smem_raw + ((LAY::LAND + smem_addr(smem_raw) + 127) & ~(size_t)127) - smem_addr(smem_raw));
  __shared__ double red[(THREADS + 31) / 32 + 1];
  __shared__ __align__(8) unsigned long long lbar;

  const int tid = threadIdx.x;
  int p, t;
  if (CONTIG) {
    t = tid % P;
    p = tid / P;
  } else {
    p = tid % TP;
    t = tid / TP;
  }
  using SMV = typename std::conditional<CONTIG, SmemContig<float2>, SmemStrided<float2, TP>>::type;
  SMV smv;
  if constexpr (CONTIG)
    smv.row = sm + p * SH::ROW;
  else
    smv.base = sm + p;
  // the stage twiddle table of this axis, staged after the exchange rows
  for (int i = tid; i < stage_tw_size<N, SH::RV>(); i += THREADS) tw_s[i] = a.tw[i];
  if constexpr (LAY::DRIFTS) {
    for (int i = tid; i < N; i += THREADS) tab2[i] = a.prop[i];
  } else if constexpr (MODE == M_IFFT2) {
    for (int i = tid; i < N; i += THREADS) tabk[i] = a.kt[1][i];  // kt along y
  } else if constexpr (MODE == M_POISSON) {
    for (int i = tid; i < N; i += THREADS) {
      tabk[i] = (a.axis == 0 ? a.k[0] : (a.axis == 1 ? a.k[1] : a.k[2]))[i];
      tabk[N + i] = (a.axis == 0 ? a.kt[0] : (a.axis == 1 ? a.kt[1] : a.kt[2]))[i];
    }
  }
  static_assert(!CTA::DYN || LAY::LANDS, "claimed tiles need the landing pipeline");
  int ahead = 0;  // claiming CTAs: thread 0's claim after the published tile
  if (tid == 0) {
    mbar_init(&lbar, 1);
    if constexpr (CTA::DYN) {
      cta.publish(cta.claim());  // the CTA's first tile
      ahead = cta.claim();
    }
  }
  __syncthreads();
  // The tables above are the plan's own; the previous pass's results are read
  // from here on.  Launched as a programmatic dependent of that pass, this
  // CTA may have started (and staged its tables) during the pass's last
  // tiles: wait until it has completed.  A no-op for a plain launch.
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const float2 *tw = tw_s;
  unsigned parity = 0;
  int fld = 0;
  int first;
  if constexpr (CTA::DYN)
    first = cta.claimed();
  else
    first = cta.bx();
  if constexpr (LAY::LANDS)
    if (first < a.ntiles && tid < 32)
      issue_tile<N, CONTIG, MODE, SV>(a, maps, 0, a.rev ? a.ntiles - 1 - first : first, cta.box(),
                                      land, &lbar);

  for (int it = first; it < a.ntiles; it = next_tile(it, cta)) {
    // this CTA's last tile: a next pass launched as a programmatic dependent
    // may start its CTAs in the slots that free up from now on
    if constexpr (!CTA::DYN)
      if (it + cta.gx() >= a.ntiles) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int tile = a.rev ? a.ntiles - 1 - it : it;  // logical tile
    const PencilPos pp = pencil_pos<CONTIG>(a, tile, p, TP);
    const long long base = pp.base, st = a.stride;
    // the density passes load the pencil's star buckets before the transforms
    // they would otherwise wait behind (in the kick the extra live registers
    // cost more than the latency they hide)
    StarRanges sr = no_star_ranges();
    if constexpr (MODE == M_DENSITY || MODE == M_DRIFT_DENSITY)
      if (a.has_stars) sr = star_ranges(a, pp);
    float2 c0;
#define QJ_TAKE(v) \
  if (!take_tile<N, CONTIG, MODE, SV, E, CTA>(v, c0, a, maps, land, &lbar, parity, fld, it, p, t, cta, \
                                              ahead))                                                 \
  return

    if constexpr (MODE == M_DENSITY) {
      float2 v[E];
      QJ_TAKE(v);
      double s = build_density<N, E>(v, a, pp, sr, t, P);
      s = block_sum<THREADS>(s, red);
      if (tid == 0) a.part[tile] = s;
      fft_pencil<N, -1, true>(v, t, smv, tw);
      if (a.half)
        store_pencil_half<N, E>(v, a.R, base, st, t, P);
      else
        store_pencil<E>(v, a.R, base, st, t, P);
    } else if constexpr (MODE == M_FFT_FWD) {
      float2 v[E];
      QJ_TAKE(v);
      fft_pencil<N, -1, true>(v, t, smv, tw);
      store_pencil<E>(v, a.R, base, st, t, P);
    } else if constexpr (MODE == M_POISSON) {
      float2 v[E];
      QJ_TAKE(v);
      // Mean density in float64 for the k = 0 mode (tile 0 only).
      double mean = 0.0;
      if (tile == 0) {
        double s = 0.0;
        for (int i = tid; i < a.n_part; i += THREADS) s += a.part_in[i];
        mean = block_sum<THREADS>(s, red) * a.inv_ncell;
      }
      fft_pencil<N, -1, true>(v, t, smv, tw);
      const int ax = a.axis;  // r: 0 or 2
      const int aq = 2 - ax;  // the other non-y axis
      // (selects, not runtime indices: small arrays indexed at run time live in local memory)
      const int cq = aq == 0 ? pp.c[0] : pp.c[2];
      const float kqv = aq == 0 ? a.k[0][cq] : a.k[2][cq];
      const float kq2 = kqv * kqv;
      const float ky = a.k[1][pp.c[1]];
      const float kperp2 = kq2 + ky * ky;
      const float ktq = aq == 0 ? a.kt[0][cq] : a.kt[2][cq], kty = a.kt[1][pp.c[1]];
      const float g0 = (float)(-a.fourpiG * a.inv_ncell);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int i = t + P * e;
        const float kr = tabk[i];
        const float k2 = kperp2 + kr * kr;
        const float g = __fdividef(g0, k2);  // (k = 0 is replaced below)
        const float2 vh = float2{v[e].x * g, v[e].y * g};
        v[e] = vh;  // A = IFFT(V^)
        const float kb = tabk[N + i];
        save[e * THREADS + tid] = float2{vh.x * kb, vh.y * kb};  // B = IFFT(kt_r V^), later
      }
      if (t == 0 && kperp2 == 0.0f) {
        // element 0 of the pencil with k_perp = 0 is k = 0:
        // V^(0) = -4 pi G (sum rho - ncell rho_bar) / 1, scaled by 1/ncell
        const double v0 = -a.fourpiG * (mean - a.rho_bar);
        float2 vh;
        if (a.phi) {
          *a.phi += a.phi_coef * v0;  // the one k = 0 element of the grid
          vh = float2{0.0f, 0.0f};
        } else {
          vh = float2{(float)v0, 0.0f};
        }
        v[0] = vh;
        save[tid] = float2{vh.x * tabk[N], vh.y * tabk[N]};
      }
      // S1 = IFFT((1 + kt_r) V^) = A + B and S2 = IFFT((kty - i ktq) V^) =
      // (kty - i ktq) A (the factor is constant along the pencil).
      // With a.half the pass covers k_q <= n_q / 2 of the real density's
      // Hermitian spectrum (q = the other non-y axis), and pencil (k_q, k_y)
      // also writes its mirror (-k_q, -k_y), whose V^ is conj(V^(-k)): for a
      // spectrum m(k) V^_mirror(k) the inverse is conj(IFFT[conj(m(-k)) V^](n)),
      // so S1' = conj(A - B) and S2' = conj((-kty - i ktq) A).  Pencils past
      // n_q / 2 (padding of a z tile) write nothing; k_q = 0 and n_q / 2 are
      // their own mirrors' partners and write only themselves.
      const int nq = aq == 0 ? a.full_nx : a.nz;
      const bool own = !a.half || 2 * cq <= nq;
      const bool mirror = a.half && cq >= 1 && 2 * cq < nq;
      const int m0 = ax == 0 ? 0 : (a.full_nx - pp.c[0]) % a.full_nx;
      const int m1 = (a.ny - pp.c[1]) % a.ny;
      const int m2 = ax == 2 ? 0 : (a.nz - pp.c[2]) % a.nz;
      const unsigned es = (unsigned)P * (unsigned)st;  // element step of a thread
      float2 *__restrict__ o1 = a.S1 + ((unsigned)base + (unsigned)t * (unsigned)st);
      float2 *__restrict__ o2 = a.S2 + ((unsigned)base + (unsigned)t * (unsigned)st);
      const long long mb = ((long long)m0 * a.ny + m1) * a.nz + m2;
      float2 *__restrict__ q1 = a.S1 + ((unsigned)mb + (unsigned)t * (unsigned)st);
      float2 *__restrict__ q2 = a.S2 + ((unsigned)mb + (unsigned)t * (unsigned)st);
      fft_pencil<N, +1, true>(v, t, smv, tw);  // A
      if (a.half) {
        // A~ and B~ of this half pencil go to S1 and S2 as they are; the
        // inverse y pass forms S1, S2 and their mirrors from them
        if (own) store_pencil<E>(v, a.S1, base, st, t, P);
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = save[e * THREADS + tid];
        fft_pencil<N, +1, true>(v, t, smv, tw);  // B
        if (own) store_pencil<E>(v, a.S2, base, st, t, P);
        continue;
      }
      if (own) {
#pragma unroll
        for (int e = 0; e < E; ++e)
          o2[(unsigned long long)es * (unsigned)e] =
              float2{kty * v[e].x + ktq * v[e].y, kty * v[e].y - ktq * v[e].x};
      }
      if (mirror) {
#pragma unroll
        for (int e = 0; e < E; ++e)
          q2[(unsigned long long)es * (unsigned)e] =
              float2{-kty * v[e].x + ktq * v[e].y, kty * v[e].y + ktq * v[e].x};
      }
      // A waits in the save slots while B is transformed
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const float2 b = save[e * THREADS + tid];
        save[e * THREADS + tid] = v[e];
        v[e] = b;
      }
      fft_pencil<N, +1, true>(v, t, smv, tw);  // B
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const float2 A = save[e * THREADS + tid];
        if (own) o1[(unsigned long long)es * (unsigned)e] = float2{A.x + v[e].x, A.y + v[e].y};
        if (mirror) q1[(unsigned long long)es * (unsigned)e] = float2{A.x - v[e].x, v[e].y - A.y};
      }
    } else if constexpr (MODE == M_IFFT2) {
      float2 v[E];
      QJ_TAKE(v);
      if (a.half) {
        // y pencils (k_q <= n_q / 2, n_r) of A~ = IFFT_r V^ and B~ = IFFT_r kt_r V^
        // (in S1, S2).  Their mirrors (-k_q, -k_y) are conj(A~) and -conj(B~), so
        // along y: S1 = A~ + B~, S2 = (kt_y - i kt_q) A~, and the mirror y pencil
        // (-k_q, n_r) is conj(IFFT_y[A~ - B~]), conj(IFFT_y[(-kt_y - i kt_q) A~]).
        const int cq = a.hq == 0 ? pp.c[0] : pp.c[2];
        const int nq = a.hq == 0 ? a.full_nx : a.nz;
        const bool own = 2 * cq <= nq, mirror = cq >= 1 && 2 * cq < nq;
        const float ktq = a.hq == 0 ? a.kt[0][cq] : a.kt[2][cq];
        const long long mb = a.hq == 0
                                 ? (long long)((a.full_nx - cq) % a.full_nx) * a.ny * a.nz + pp.c[2]
                                 : (long long)pp.c[0] * a.ny * a.nz + (a.nz - cq) % a.nz;
        float2 w[E];
#pragma unroll
        for (int e = 0; e < E; ++e) save[e * THREADS + tid] = v[e];  // A~
        QJ_TAKE(w);                                                 // B~
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = float2{v[e].x + w[e].x, v[e].y + w[e].y};
        fft_pencil<N, +1, true>(v, t, smv, tw);
        if (own) store_pencil<E, false>(v, a.S1, base, st, t, P);
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const float2 A = save[e * THREADS + tid];
          v[e] = float2{A.x - w[e].x, A.y - w[e].y};
        }
        fft_pencil<N, +1, true>(v, t, smv, tw);
        if (mirror) {
#pragma unroll
          for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
          store_pencil<E, false>(v, a.S1, mb, st, t, P);
        }
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const float2 A = save[e * THREADS + tid];
          const float ky = tabk[t + P * e];
          v[e] = float2{ky * A.x + ktq * A.y, ky * A.y - ktq * A.x};
        }
        fft_pencil<N, +1, true>(v, t, smv, tw);
        if (own) store_pencil<E, false>(v, a.S2, base, st, t, P);
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const float2 A = save[e * THREADS + tid];
          const float ky = tabk[t + P * e];
          v[e] = float2{-ky * A.x + ktq * A.y, -ky * A.y - ktq * A.x};
        }
        fft_pencil<N, +1, true>(v, t, smv, tw);
        if (mirror) {
#pragma unroll
          for (int e = 0; e < E; ++e) v[e].y = -v[e].y;
          store_pencil<E, false>(v, a.S2, mb, st, t, P);
        }
        continue;
      }
      fft_pencil<N, +1, true>(v, t, smv, tw);
      store_pencil<E, false>(v, a.S1, base, st, t, P);
      QJ_TAKE(v);
      fft_pencil<N, +1, true>(v, t, smv, tw);
      store_pencil<E, false>(v, a.S2, base, st, t, P);
    } else if constexpr (MODE == M_KICK) {
      const int aq = a.axis;  // the kick axis; ar = 2 - aq is the Poisson axis
      const unsigned gb = (unsigned)base + (unsigned)t * (unsigned)st, gs = (unsigned)P * (unsigned)st;
      float am = 0.0f;
      float V[E];
      // stars touching this pencil (most pencils have none and skip the lookups)
      const bool pstars = a.has_stars && pencil_has_stars(a, pp.pid);
      {
        // phase 1: S2 -> a_q + i a_y
        float2 v2[E];
        QJ_TAKE(v2);
        fft_pencil<N, +1, true>(v2, t, smv, tw);
#pragma unroll
        for (int e = 0; e < E; ++e) am = fmaxf(am, fmaxf(fabsf(v2[e].x), fabsf(v2[e].y)));
        // a_q + i a_y wait in the thread's save slots (free until the drift)
        // for the star corners, looked up once after phase 2
        if (pstars) {
#pragma unroll
          for (int e = 0; e < E; ++e) save[e * THREADS + tid] = v2[e];
        }
        if (a.gv[0]) {
          // v += a dt/2 as fire-and-forget adds at L2: each element has one
          // writer, so this is the same single rounding as load-add-store, but
          // nothing waits on it (a load-add-store could not move the next load
          // above the store: the compiler cannot tell the elements apart)
          float *gq = aq == 0 ? a.gv[0] : a.gv[2], *gy = a.gv[1];
#pragma unroll
          for (int e = 0; e < E; ++e) {
            atomicAdd(gq + (gb + e * gs), v2[e].x * a.gas_dt);
            atomicAdd(gy + (gb + e * gs), v2[e].y * a.gas_dt);
          }
        }
      }
      {
        // phase 2: S1 -> V + i a_r (V right before the kick that uses it)
        float2 v1[E];
        QJ_TAKE(v1);
        fft_pencil<N, +1, true>(v1, t, smv, tw);
#pragma unroll
        for (int e = 0; e < E; ++e) {
          V[e] = v1[e].x;
          am = fmaxf(am, fabsf(v1[e].y));
        }
        if (pstars) {
          // a_r into the pencil's exchange row, free until the drift's first
          // exchange: in a transform's last stage each thread reads only the
          // elements of its own residue t mod P, so no thread still reads the
          // ones this thread writes
#pragma unroll
          for (int e = 0; e < E; ++e) smv.st(t + P * e, float2{v1[e].y, 0.0f});
          if constexpr (CONTIG) __syncwarp(pencil_lanes(P));
          kick_star_corners<N, CONTIG, THREADS>(a, star_ranges(a, pp), t, P,
                                                [&](unsigned s, int cbits, int slot, int m) {
                                                  const float2 w = save[slot];
                                                  float *dst = a.A + 3 * (8 * s + c_corner_of_bits_dev(cbits));
                                                  dst[aq] = w.x;
                                                  dst[1] = w.y;
                                                  dst[aq == 0 ? 2 : 0] = smv.ld(m).x;
                                                });
          if constexpr (CONTIG) __syncwarp(pencil_lanes(P));
        }
        if (a.gv[0]) {  // gas half kick, quantum-gas-bh.py:255-266 (adds as above)
          float *g = aq == 0 ? a.gv[2] : a.gv[0];
#pragma unroll
          for (int e = 0; e < E; ++e) atomicAdd(g + (gb + e * gs), v1[e].y * a.gas_dt);
        }
      }
      // phase 3: psi <- exp(-i c V) psi with V = Poisson + b rho + V_ext, then
      // the drift along this axis
      float2 ps[E];
      QJ_TAKE(ps);
      if (a.b_coeff != 0.0f) {
        // rho = |psi|^2 + rho_stars, the argument of get_potential (quantum-stars.py:193);
        // the star density of a cell is summed from zero in star order in the
        // thread's save slots
        float *rs = reinterpret_cast<float *>(save);
#pragma unroll
        for (int e = 0; e < E; ++e) rs[2 * (e * THREADS + tid)] = 0.0f;
        if (pstars)
          for_star_corners<N, true>(a, star_ranges(a, pp), t, P,
                                    [&](unsigned, int, int m, float wx, float wy, float wz, float fac) {
                                      const float val = fmul_rn(fmul_rn(fmul_rn(wx, wy), wz), fac);
                                      float &r = rs[2 * ((m / P) * THREADS + tid)];
                                      r = fadd_rn(r, val);
                                    });
        if (a.rho_src) {
#pragma unroll
          for (int e = 0; e < E; ++e) rs[2 * (e * THREADS + tid)] += a.rho_src[gb + e * gs];
        }
#pragma unroll
        for (int e = 0; e < E; ++e)
          V[e] = V[e] + a.b_coeff * (ps[e].x * ps[e].x + ps[e].y * ps[e].y + rs[2 * (e * THREADS + tid)]);
      }
      if (a.v_ext) {
#pragma unroll
        for (int e = 0; e < E; ++e) V[e] = V[e] + a.v_ext[gb + e * gs];
      }
      const double phi = (a.phi_final && a.phi) ? *a.phi : 0.0;
#pragma unroll
      for (int e = 0; e < E; ++e) ps[e] = phase_rotate(ps[e], a.kick_coef * (double)V[e] + phi);
      if (a.v_out) {
#pragma unroll
        for (int e = 0; e < E; ++e) a.v_out[gb + e * gs] = V[e];
      }
      if (a.do_drift) drift_pencil<N, E, P, THREADS>(ps, c0, tab2, t, smv, tw, save);
      store_pencil<E>(ps, a.psi, base, st, t, P);
      if constexpr (THREADS >= 32) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) am = fmaxf(am, __shfl_xor_sync(0xffffffffu, am, o));
        if ((tid & 31) == 0) atomic_max_nonneg(a.amax_bits, am);
      } else {
        atomic_max_nonneg(a.amax_bits, am);
      }
    } else if constexpr (MODE == M_ADJ_SOURCE) {
      // mu = c Im(conj(g) psi') with psi' = e^{-icV} psi (the kick adjoint's
      // Poisson source, quantum-stars.py:300 differentiated), its float64
      // partial sum, and its forward transform along z (half of R)
      const unsigned gb = (unsigned)base + (unsigned)t * (unsigned)st, gs = (unsigned)P * (unsigned)st;
      float2 v[E];
      QJ_TAKE(v);  // g
      {
        float2 z[E];
        QJ_TAKE(z);  // psi before the kick
#pragma unroll
        for (int e = 0; e < E; ++e) {
          float sn, cs;
          sincos_reduced(a.kick_coef * (double)a.adj_V[gb + e * gs], sn, cs);
          const float2 zp = float2{z[e].x * cs + z[e].y * sn, z[e].y * cs - z[e].x * sn};
          const float m = (float)a.kick_coef * (v[e].x * zp.y - v[e].y * zp.x);
          if (a.adj_mu) a.adj_mu[gb + e * gs] = m;
          v[e] = float2{m, 0.0f};
        }
      }
      double sm = 0.0;
#pragma unroll
      for (int e = 0; e < E; ++e) sm += (double)v[e].x;
      sm = block_sum<THREADS>(sm, red);
      if (tid == 0) a.part[tile] = sm;
      fft_pencil<N, -1, true>(v, t, smv, tw);
      store_pencil_half<N, E>(v, a.R, base, st, t, P);
    } else if constexpr (MODE == M_ADJ_UPDATE) {
      // W = L mu along z from S1 (its real part), then
      // g <- e^{icV} g + 2 (W + b mu) psi and the drift adjoint along z
      const unsigned gb = (unsigned)base + (unsigned)t * (unsigned)st, gs = (unsigned)P * (unsigned)st;
      float W[E];
      {
        float2 v1[E];
        QJ_TAKE(v1);
        fft_pencil<N, +1, true>(v1, t, smv, tw);
#pragma unroll
        for (int e = 0; e < E; ++e) W[e] = v1[e].x;
      }
      float2 g[E];
      QJ_TAKE(g);
      const float2 gc = c0;  // the drift's increment constant: g's element 0
      {
        float2 z[E];
        QJ_TAKE(z);  // psi before the kick
#pragma unroll
        for (int e = 0; e < E; ++e) {
          float w = W[e];
          if (a.adj_mu) w = w + a.b_coeff * a.adj_mu[gb + e * gs];
          float sn, cs;
          sincos_reduced(a.kick_coef * (double)a.adj_V[gb + e * gs], sn, cs);
          const float two_w = 2.0f * w;
          g[e] = float2{g[e].x * cs - g[e].y * sn + two_w * z[e].x,
                        g[e].y * cs + g[e].x * sn + two_w * z[e].y};
        }
      }
      if (a.do_drift) drift_pencil<N, E, P, THREADS>(g, gc, tab2, t, smv, tw, save);
      store_pencil<E>(g, a.psi, base, st, t, P);
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
      (void)c0;
    } else if constexpr (MODE == M_DRIFT || MODE == M_DRIFT_DENSITY) {
      float2 v[E];
      QJ_TAKE(v);
      drift_pencil<N, E, P, THREADS>(v, c0, tab2, t, smv, tw, save);
      store_pencil<E>(v, a.psi, base, st, t, P);
      if constexpr (MODE == M_DRIFT_DENSITY) {
        double s = build_density<N, E>(v, a, pp, sr, t, P);
        s = block_sum<THREADS>(s, red);
        if (tid == 0) a.part[tile] = s;
        fft_pencil<N, -1, true>(v, t, smv, tw);
        if (a.half)
          store_pencil_half<N, E>(v, a.R, base, st, t, P);
        else
          store_pencil<E>(v, a.R, base, st, t, P);
      }
    }
#undef QJ_TAKE
  }
  if constexpr (CTA::DYN) {
    // no copy is in flight (the last claim found no tile): retire the
    // landing barrier, so that this CTA's body for its next box can
    // initialise one in the same place
    __syncthreads();
    if (tid == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&lbar)) : "memory");
    __syncthreads();
  }
}

template <int N, bool CONTIG, int MODE, int SV = 0>
__global__ void __launch_bounds__(PassShape<N, CONTIG, SV>::THREADS, PassShape<N, CONTIG, SV>::MINB)
    k_fused(FusedArgs a, const __grid_constant__ TileMaps maps) {
  fused_body<N, CONTIG, MODE, SV>(a, maps, GridCta{});
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
  extern __shared__ __align__(128) unsigned char smem_raw[];
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
    const int z = (blockIdx.x % a.ztiles) * TP + p;
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
