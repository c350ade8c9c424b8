// Particle kernels: cloud-in-cell deposit and gather, leapfrog update.
//
// The deposit is deterministic without floating-point atomics: every particle
// emits its 8 corner contributions (key = cell in the pass orientation,
// value = w_x w_y w_z m / vol), a single-CTA stable LSD radix sort orders them
// by cell while keeping (particle, corner) order inside a cell, and the head
// of each run sums the run sequentially from zero.  That is exactly the order
// of the reference's sequential fori_loop over stars with 8 fixed-order
// scatter-adds each (quantum-stars.py:212-247), so the float32 result matches
// a float32 evaluation of the reference bit for bit.
#include <cstdio>
#include <mutex>

#include "../../include/qj.h"
#include "qj_internal.h"

namespace qj {

// Corner visit order of quantum-stars.py:220-243 and :264-287
// (bit d set = ip1 along axis d).
__constant__ int c_corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                                   {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};

template <typename R> struct CicGeom {
  int n[3];
  R d[3];
  R L[3];
  R vol;
};

template <typename R> static CicGeom<R> cast_geom(const CicGeomD &g) {
  CicGeom<R> o;
  for (int i = 0; i < 3; ++i) {
    o.n[i] = g.n[i];
    o.d[i] = (R)g.d[i];
    o.L[i] = (R)g.L[i];
  }
  o.vol = (R)g.vol;
  return o;
}

// quantum-stars.py:200-209 for one axis, every operation rounded in the
// written order:  i = floor((x - 0.5 dx) / dx);  w_i = ((i + 1 + 0.5) dx - x) / dx;
// w_ip1 = (x - (i + 0.5) dx) / dx;  indices wrapped with jnp.mod.
template <typename R>
__device__ __forceinline__ void cic_axis(R x, R dx, int n, int &i0, int &i1, R &w0, R &w1) {
  const R half = (R)0.5;
  const R i = floor(fdiv_rn(fsub_rn(x, fmul_rn(half, dx)), dx));
  const R ip1 = fadd_rn(i, (R)1);
  w0 = fdiv_rn(fsub_rn(fmul_rn(fadd_rn(ip1, half), dx), x), dx);
  w1 = fdiv_rn(fsub_rn(x, fmul_rn(fadd_rn(i, half), dx)), dx);
  R m0 = ref_mod(i, (R)n), m1 = ref_mod(ip1, (R)n);
  // non-finite positions map to cell 0 (the state is reported non-finite
  // by the caller's checks); keeps every index in bounds.
  i0 = (m0 >= (R)0 && m0 < (R)n) ? (int)m0 : 0;
  i1 = (m1 >= (R)0 && m1 < (R)n) ? (int)m1 : 0;
}

__device__ __forceinline__ unsigned cell_key(int cx, int cy, int cz, int q, int nx, int ny,
                                             int nz) {
  if (q == 2) return ((unsigned)cx * (unsigned)ny + (unsigned)cy) * (unsigned)nz + (unsigned)cz;
  if (q == 0) return ((unsigned)cy * (unsigned)nz + (unsigned)cz) * (unsigned)nx + (unsigned)cx;
  return ((unsigned)cx * (unsigned)nz + (unsigned)cz) * (unsigned)ny + (unsigned)cy;
}

template <typename R>
__device__ __forceinline__ void cic_emit(const R *pos, int s, const CicGeom<R> &g, R fac, int q,
                                         unsigned *keys, R *vals) {
  int i0[3], i1[3];
  R w0[3], w1[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) cic_axis<R>(pos[3 * s + d], g.d[d], g.n[d], i0[d], i1[d], w0[d], w1[d]);
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int bx = c_corner[c][0], by = c_corner[c][1], bz = c_corner[c][2];
    const R v = fmul_rn(fmul_rn(fmul_rn(bx ? w1[0] : w0[0], by ? w1[1] : w0[1]), bz ? w1[2] : w0[2]), fac);
    keys[8 * s + c] = cell_key(bx ? i1[0] : i0[0], by ? i1[1] : i0[1], bz ? i1[2] : i0[2], q, g.n[0],
                               g.n[1], g.n[2]);
    vals[8 * s + c] = v;
  }
}

// fac: m_s / (dx dy dz) evaluated in float64 and rounded (bin_stars,
// quantum-stars.py:219), or masses[s] / vol rounded per operation
// (bin_particles, quantum-gas-bh.py:421).
template <typename R>
__device__ __forceinline__ R cic_fac(const R *masses, int s, R fac_all, R vol) {
  return masses ? fdiv_rn(masses[s], vol) : fac_all;
}

template <typename R>
__global__ void k_cic_prepare(const R *pos, int n, const R *masses, R fac_all, CicGeom<R> g, int q,
                              unsigned *keys, R *vals) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  cic_emit<R>(pos, s, g, cic_fac<R>(masses, s, fac_all, g.vol), q, keys, vals);
}

unsigned cell_bits(long long ncell) {
  unsigned b = 0;
  while ((1ll << b) < ncell) ++b;
  return b;
}

int launch_cic_prepare(bool dbl, const void *pos, int n, const void *masses, double m_s,
                       const CicGeomD &g, int q, unsigned *keys, void *vals, cudaStream_t st) {
  if (n <= 0) return 0;
  const int T = 128, B = (n + T - 1) / T;
  const double fac = m_s / (g.d[0] * g.d[1] * g.d[2]);
  if (dbl)
    k_cic_prepare<double><<<B, T, 0, st>>>((const double *)pos, n, (const double *)masses, fac,
                                           cast_geom<double>(g), q, keys, (double *)vals);
  else
    k_cic_prepare<float><<<B, T, 0, st>>>((const float *)pos, n, (const float *)masses, (float)fac,
                                          cast_geom<float>(g), q, keys, (float *)vals);
  QJ_CK_LAUNCH();
  return 0;
}

// Single-CTA stable LSD radix sort (8-bit digits) of (key, index) pairs,
// then run-length reduction in sorted order.  32 warps each own a
// contiguous chunk; within a digit pass a warp scatters its chunk in order
// with __match_any_sync ranks, so equal keys keep their input order.
template <typename R>
__global__ void __launch_bounds__(1024)
    k_sort_unique(const unsigned *keys_in, const R *vals, int n, unsigned nbits, unsigned *kA,
                  unsigned *iA, unsigned *kB, unsigned *iB, unsigned *ukey, R *uval,
                  unsigned *cell_u, int *n_unique, R *dts_reset) {
  __shared__ unsigned hist[32 * 256];
  __shared__ unsigned dbase[256];
  __shared__ unsigned wsum[32];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid == 0 && dts_reset) *dts_reset = (R)INFINITY;
  const int chunk = (n + 31) / 32;
  const int beg = min(n, w * chunk), end = min(n, beg + chunk);
  const unsigned *kin = keys_in;
  const unsigned *iin = nullptr;
  unsigned *kout = kA, *iout = iA;
  for (unsigned shift = 0; shift < nbits; shift += 8) {
    for (int i = tid; i < 32 * 256; i += 1024) hist[i] = 0;
    __syncthreads();
    for (int i = beg + lane; i < end; i += 32) atomicAdd(&hist[w * 256 + ((kin[i] >> shift) & 255u)], 1u);
    __syncthreads();
    if (tid < 256) {
      unsigned s = 0;
      for (int ww = 0; ww < 32; ++ww) {
        const unsigned c = hist[ww * 256 + tid];
        hist[ww * 256 + tid] = s;
        s += c;
      }
      dbase[tid] = s;
    }
    __syncthreads();
    if (w == 0) {  // exclusive scan of the 256 digit totals
      unsigned v[8], loc = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        v[j] = dbase[lane * 8 + j];
        loc += v[j];
      }
      unsigned incl = loc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      unsigned run = incl - loc;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const unsigned c = v[j];
        dbase[lane * 8 + j] = run;
        run += c;
      }
    }
    __syncthreads();
    if (tid < 256)
      for (int ww = 0; ww < 32; ++ww) hist[ww * 256 + tid] += dbase[tid];
    __syncthreads();
    for (int i0 = beg; i0 < end; i0 += 32) {
      const int i = i0 + lane;
      const bool ok = i < end;
      unsigned k = 0, id = 0, d = 256u + (unsigned)lane;
      if (ok) {
        k = kin[i];
        id = iin ? iin[i] : (unsigned)i;
        d = (k >> shift) & 255u;
      }
      const unsigned peers = __match_any_sync(0xffffffffu, d);
      const unsigned rank = __popc(peers & ((1u << lane) - 1u));
      if (ok) {
        const unsigned p = hist[w * 256 + d] + rank;
        kout[p] = k;
        iout[p] = id;
      }
      __syncwarp();
      if (ok && rank == 0) hist[w * 256 + d] += __popc(peers);
      __syncwarp();
    }
    __syncthreads();
    kin = kout;
    iin = iout;
    kout = (kout == kA) ? kB : kA;
    iout = (iout == iA) ? iB : iA;
  }
  // run heads and ordered per-cell sums
  const int c2 = (n + 1023) / 1024;
  const int b2 = min(n, tid * c2), e2 = min(n, b2 + c2);
  unsigned cnt = 0;
  for (int i = b2; i < e2; ++i) cnt += (i == 0 || kin[i] != kin[i - 1]) ? 1u : 0u;
  unsigned incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    unsigned x = wsum[lane], xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += y;
    }
    wsum[lane] = xi - x;  // exclusive
  }
  __syncthreads();
  unsigned u = wsum[w] + incl - cnt;
  for (int i = b2; i < e2; ++i) {
    const unsigned k = kin[i];
    if (i == 0 || k != kin[i - 1]) {
      R s = (R)0;
      int j = i;
      do {
        s = fadd_rn(s, vals[iin ? iin[j] : (unsigned)j]);
        ++j;
      } while (j < n && kin[j] == k);
      ukey[u] = k;
      uval[u] = s;
      ++u;
    }
    cell_u[iin ? iin[i] : (unsigned)i] = u - 1;
  }
  if (tid == 1023) *n_unique = (int)(wsum[w] + incl);
}

int launch_sort_unique(bool dbl, const unsigned *keys, const void *vals, int n, unsigned nbits,
                       unsigned *kA, unsigned *iA, unsigned *kB, unsigned *iB, unsigned *ukey,
                       void *uval, unsigned *cell_u, int *n_unique, void *dts_reset,
                       cudaStream_t st) {
  if (n <= 0) return 0;
  if (dbl)
    k_sort_unique<double><<<1, 1024, 0, st>>>(keys, (const double *)vals, n, nbits, kA, iA, kB, iB,
                                              ukey, (double *)uval, cell_u, n_unique,
                                              (double *)dts_reset);
  else
    k_sort_unique<float><<<1, 1024, 0, st>>>(keys, (const float *)vals, n, nbits, kA, iA, kB, iB,
                                             ukey, (float *)uval, cell_u, n_unique,
                                             (float *)dts_reset);
  QJ_CK_LAUNCH();
  return 0;
}

__global__ void k_pencil_starts(const unsigned *ukey, const int *n_unique, int n_pencils,
                                unsigned nq, int *start) {
  const int pid = blockIdx.x * blockDim.x + threadIdx.x;
  if (pid > n_pencils) return;
  const unsigned long long target = (unsigned long long)pid * nq;
  int lo = 0, hi = *n_unique;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if ((unsigned long long)ukey[mid] < target)
      lo = mid + 1;
    else
      hi = mid;
  }
  start[pid] = lo;
}

int launch_pencil_starts(const unsigned *ukey, const int *n_unique, int n_pencils, unsigned nq,
                         int *start, cudaStream_t st) {
  const int T = 256, B = (n_pencils + 1 + T - 1) / T;
  k_pencil_starts<<<B, T, 0, st>>>(ukey, n_unique, n_pencils, nq, start);
  QJ_CK_LAUNCH();
  return 0;
}

template <typename R>
__global__ void k_scatter_unique(const unsigned *ukey, const R *uval, const int *n_unique, R *grid) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u < *n_unique) grid[ukey[u]] = uval[u];
}

int launch_scatter_unique(bool dbl, const unsigned *ukey, const void *uval, const int *n_unique,
                          int max_unique, void *grid, cudaStream_t st) {
  if (max_unique <= 0) return 0;
  const int T = 256, B = (max_unique + T - 1) / T;
  if (dbl)
    k_scatter_unique<double><<<B, T, 0, st>>>(ukey, (const double *)uval, n_unique, (double *)grid);
  else
    k_scatter_unique<float><<<B, T, 0, st>>>(ukey, (const float *)uval, n_unique, (float *)grid);
  QJ_CK_LAUNCH();
  return 0;
}

// quantum-stars.py:262-287: acc = sum over corners, in order, of
// (w_x w_y w_z) * a(corner), starting from zero.
template <typename R, bool DENSE>
__global__ void k_gather(const R *pos, int n, CicGeom<R> g, const R *A, const unsigned *cell_u,
                         const R *ax, const R *ay, const R *az, R *acc) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int i0[3], i1[3];
  R w0[3], w1[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) cic_axis<R>(pos[3 * s + d], g.d[d], g.n[d], i0[d], i1[d], w0[d], w1[d]);
  R a0 = (R)0, a1 = (R)0, a2 = (R)0;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int bx = c_corner[c][0], by = c_corner[c][1], bz = c_corner[c][2];
    const R wp = fmul_rn(fmul_rn(bx ? w1[0] : w0[0], by ? w1[1] : w0[1]), bz ? w1[2] : w0[2]);
    R gx, gy, gz;
    if (DENSE) {
      const long long cell = ((long long)(bx ? i1[0] : i0[0]) * g.n[1] + (by ? i1[1] : i0[1])) * g.n[2] +
                             (bz ? i1[2] : i0[2]);
      gx = ax[cell];
      gy = ay[cell];
      gz = az[cell];
    } else {
      const unsigned u = cell_u[8 * s + c];
      gx = A[3 * u + 0];
      gy = A[3 * u + 1];
      gz = A[3 * u + 2];
    }
    a0 = fadd_rn(a0, fmul_rn(wp, gx));
    a1 = fadd_rn(a1, fmul_rn(wp, gy));
    a2 = fadd_rn(a2, fmul_rn(wp, gz));
  }
  acc[3 * s + 0] = a0;
  acc[3 * s + 1] = a1;
  acc[3 * s + 2] = a2;
}

int launch_gather_unique(bool dbl, const void *pos, int n, const CicGeomD &g, const void *A,
                         const unsigned *cell_u, void *acc, cudaStream_t st) {
  if (n <= 0) return 0;
  const int T = 128, B = (n + T - 1) / T;
  if (dbl)
    k_gather<double, false><<<B, T, 0, st>>>((const double *)pos, n, cast_geom<double>(g),
                                             (const double *)A, cell_u, nullptr, nullptr, nullptr,
                                             (double *)acc);
  else
    k_gather<float, false><<<B, T, 0, st>>>((const float *)pos, n, cast_geom<float>(g),
                                            (const float *)A, cell_u, nullptr, nullptr, nullptr,
                                            (float *)acc);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_gather_dense(bool dbl, const void *pos, int n, const CicGeomD &g, const void *ax,
                        const void *ay, const void *az, void *acc, cudaStream_t st) {
  if (n <= 0) return 0;
  const int T = 128, B = (n + T - 1) / T;
  if (dbl)
    k_gather<double, true><<<B, T, 0, st>>>((const double *)pos, n, cast_geom<double>(g), nullptr,
                                            nullptr, (const double *)ax, (const double *)ay,
                                            (const double *)az, (double *)acc);
  else
    k_gather<float, true><<<B, T, 0, st>>>((const float *)pos, n, cast_geom<float>(g), nullptr,
                                           nullptr, (const float *)ax, (const float *)ay,
                                           (const float *)az, (float *)acc);
  QJ_CK_LAUNCH();
  return 0;
}

// vel = vel + acc * dt / 2.0 (quantum-stars.py:304,321); dt_s = min |dx / vel|
// (:328, dx for every component); pos = mod(pos + vel * dt, L) (:311-312).
template <typename R>
__global__ void k_particles_update(R *pos, R *vel, const R *acc, int n, CicGeom<R> g, R dt, int k2,
                                   int k1, int drift, R *dts, int q_next, unsigned *keys, R *vals,
                                   const R *masses, R fac_all) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  R v[3], x[3];
  float dmin = INFINITY;
  double dmind = INFINITY;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    v[d] = vel[3 * s + d];
    const R h = fdiv_rn(fmul_rn(acc[3 * s + d], dt), (R)2);
    if (k2) {
      v[d] = fadd_rn(v[d], h);
      const R r = fabs(fdiv_rn(g.d[0], v[d]));
      if constexpr (sizeof(R) == 4)
        dmin = fminf(dmin, (float)r);
      else
        dmind = fmin(dmind, (double)r);
    }
    if (k1) v[d] = fadd_rn(v[d], h);
    vel[3 * s + d] = v[d];
  }
  if (k2) {
    if constexpr (sizeof(R) == 4)
      atomic_min_nonneg((unsigned int *)dts, dmin);
    else
      atomic_min_nonneg((unsigned long long *)dts, dmind);
  }
  if (drift) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      x[d] = ref_mod(fadd_rn(pos[3 * s + d], fmul_rn(v[d], dt)), g.L[d]);
      pos[3 * s + d] = x[d];
    }
    if (keys) cic_emit<R>(pos, s, g, cic_fac<R>(masses, s, fac_all, g.vol), q_next, keys, vals);
  }
}

int launch_particles_update(bool dbl, void *pos, void *vel, const void *acc, const CicGeomD &g,
                            const UpdateArgs &u, cudaStream_t st) {
  if (u.n <= 0) return 0;
  const int T = 128, B = (u.n + T - 1) / T;
  const double fac = u.m_s / (g.d[0] * g.d[1] * g.d[2]);
  if (dbl)
    k_particles_update<double><<<B, T, 0, st>>>(
        (double *)pos, (double *)vel, (const double *)acc, u.n, cast_geom<double>(g), u.dt, u.k2,
        u.k1, u.drift, (double *)u.dts_bits, u.q_next, u.keys, (double *)u.vals,
        (const double *)u.masses, fac);
  else
    k_particles_update<float><<<B, T, 0, st>>>(
        (float *)pos, (float *)vel, (const float *)acc, u.n, cast_geom<float>(g), (float)u.dt,
        u.k2, u.k1, u.drift, (float *)u.dts_bits, u.q_next, u.keys, (float *)u.vals,
        (const float *)u.masses, (float)fac);
  QJ_CK_LAUNCH();
  return 0;
}

// ----- pencil-bucket deposit for the fused passes -----
//
// Each star is filed under the pencil (in the pass orientation q) that holds
// its lower CIC corner.  A pencil pass then finds every star touching its
// pencil in the four neighbouring buckets, and visits them in star order so
// each cell still sums its contributions in the reference's order.

// Corner number (reference order, quantum-stars.py:220-243) of the corner
// with ip1 bits (bx, by, bz): index bx + 2 by + 4 bz.
__constant__ int c_corner_of_bits[8] = {0, 1, 2, 4, 3, 5, 6, 7};

__device__ __forceinline__ unsigned bucket_of(int ix, int iy, int iz, int q, const int n[3]) {
  if (q == 2) return (unsigned)ix * (unsigned)n[1] + (unsigned)iy;
  if (q == 0) return (unsigned)iy * (unsigned)n[2] + (unsigned)iz;
  return (unsigned)ix * (unsigned)n[2] + (unsigned)iz;
}

// Per-star CIC data: lower corner (wrapped), weights w_i / w_ip1 per axis and
// the deposit factor m / vol, all in the reference's float32 order.
__device__ __forceinline__ void star_prepare(const float *pos, int s, const CicGeom<float> &g,
                                             float fac, int q, int4 *sidx, float4 *sw0,
                                             float4 *sw1, unsigned *bkey) {
  int i0[3], i1[3];
  float w0[3], w1[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) cic_axis<float>(pos[3 * s + d], g.d[d], g.n[d], i0[d], i1[d], w0[d], w1[d]);
  sidx[s] = int4{i0[0], i0[1], i0[2], 0};
  sw0[s] = float4{w0[0], w0[1], w0[2], fac};
  sw1[s] = float4{w1[0], w1[1], w1[2], 0.0f};
  bkey[s] = bucket_of(i0[0], i0[1], i0[2], q, g.n);
}

__global__ void k_stars_prepare(const float *pos, int n, const float *masses, float fac_all,
                                CicGeom<float> g, int q, int4 *sidx, float4 *sw0, float4 *sw1,
                                unsigned *bkey) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  star_prepare(pos, s, g, cic_fac<float>(masses, s, fac_all, g.vol), q, sidx, sw0, sw1, bkey);
}

int launch_stars_prepare(const void *pos, int n, const void *masses, double m_s,
                         const CicGeomD &g, int q, const StarBufs &b, cudaStream_t st) {
  if (n <= 0) return 0;
  const int T = 128, B = (n + T - 1) / T;
  const double fac = m_s / (g.d[0] * g.d[1] * g.d[2]);
  k_stars_prepare<<<B, T, 0, st>>>((const float *)pos, n, (const float *)masses, (float)fac,
                                   cast_geom<float>(g), q, b.sidx, b.sw0, b.sw1, b.bkey);
  QJ_CK_LAUNCH();
  return 0;
}

// A few particles (n <= 32: black holes): star_prepare, the sort by (bucket,
// index) and the bucket starts in one launch.  Every block works out the n
// keys; block 0 also stores the particle data, the permutation and the sorted
// keys (each particle's rank by counting, the order of the stable sort); every
// block fills its share of the bucket runs and the bucket mask, as
// k_bucket_sort leaves them.
constexpr int kSmallStars = 32;
__global__ void __launch_bounds__(256)
    k_stars_small(const float *pos, int n, const float *masses, float fac_all, CicGeom<float> g,
                  int q, int4 *sidx, float4 *sw0, float4 *sw1, unsigned *bkey, unsigned *perm,
                  unsigned *skey, int *bstart, unsigned *pmask, int n_buckets) {
  __shared__ unsigned keys[kSmallStars];
  const int s = threadIdx.x;
  if (s < kSmallStars) {
    unsigned key = 0xffffffffu;
    if (s < n) {
      if (blockIdx.x == 0) {
        star_prepare(pos, s, g, cic_fac<float>(masses, s, fac_all, g.vol), q, sidx, sw0, sw1, bkey);
        key = bkey[s];
      } else {
        int i0[3], i1[3];
        float w0[3], w1[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
          cic_axis<float>(pos[3 * s + d], g.d[d], g.n[d], i0[d], i1[d], w0[d], w1[d]);
        key = bucket_of(i0[0], i0[1], i0[2], q, g.n);
      }
    }
    keys[s] = key;
  }
  __syncthreads();
  if (blockIdx.x == 0 && s < n) {
    const unsigned key = keys[s];
    int rank = 0;
    for (int j = 0; j < n; ++j) rank += (keys[j] < key || (keys[j] == key && j < s)) ? 1 : 0;
    perm[rank] = (unsigned)s;
    skey[rank] = key;
  }
  // bstart[b] = the keys below b (the lower bound k_bucket_starts finds), and
  // the pencil mask
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= n_buckets; b += gridDim.x * blockDim.x) {
    int c = 0;
    for (int j = 0; j < n; ++j) c += keys[j] < (unsigned)b ? 1 : 0;
    bstart[b] = c;
    if (b == n_buckets) continue;
    // pencil b has particles when any of its four touching buckets does
    const int nv = q == 2 ? g.n[1] : g.n[2], nu = n_buckets / nv;
    const int cu = b / nv, cv = b - cu * nv;
    const int cum = cu == 0 ? nu - 1 : cu - 1, cvm = cv == 0 ? nv - 1 : cv - 1;
    const unsigned nb[4] = {(unsigned)b, (unsigned)(cum * nv + cv), (unsigned)(cu * nv + cvm),
                            (unsigned)(cum * nv + cvm)};
    int touch = 0;
    for (int j = 0; j < n; ++j)
      touch |= (keys[j] == nb[0]) | (keys[j] == nb[1]) | (keys[j] == nb[2]) | (keys[j] == nb[3]);
    const unsigned pword = __ballot_sync(__activemask(), touch != 0);
    if ((b & 31) == 0) pmask[b >> 5] = pword;
  }
}

int launch_stars_small(const void *pos, int n, const void *masses, double m_s, const CicGeomD &g,
                       int q, int n_buckets, const StarBufs &b, cudaStream_t st) {
  if (n <= 0 || n > kSmallStars) {
    set_error("internal: launch_stars_small with %d particles", n);
    return QJ_ERR_ARG;
  }
  const double fac = m_s / (g.d[0] * g.d[1] * g.d[2]);
  const int T = 256, B = (n_buckets + 1 + T - 1) / T;
  k_stars_small<<<B, T, 0, st>>>((const float *)pos, n, (const float *)masses, (float)fac,
                                 cast_geom<float>(g), q, b.sidx, b.sw0, b.sw1, b.bkey, b.perm, b.skey,
                                 b.bstart, b.pmask, n_buckets);
  QJ_CK_LAUNCH();
  return 0;
}

// Single-CTA stable LSD radix sort (8-bit digits) of the stars by bucket;
// buffers in shared memory up to kSortSmemMax stars, else in global scratch.
constexpr int kSortSmemMax = 8192;

__global__ void __launch_bounds__(1024)
    k_bucket_sort(const unsigned *bkey, int n, unsigned nbits, unsigned *gbuf, int use_smem,
                  unsigned *perm, unsigned *skey, int n_buckets, int nv, unsigned *pmask,
                  int mstride) {
  // dynamic shared memory: the mask of non-empty buckets (one bit per
  // bucket), then the sort buffers when they fit
  extern __shared__ unsigned dyn[];
  __shared__ unsigned hist[32 * 256];
  __shared__ unsigned dbase[256];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int mwords = (n_buckets + 31) / 32;
  unsigned *mask = dyn;
  {  // one CTA per box of a batched plan
    const long long box = blockIdx.x;
    bkey += box * n;
    gbuf += box * 4 * n;
    perm += box * n;
    skey += box * n;
    pmask += box * mstride;
  }
  for (int i = tid; i < mwords; i += 1024) mask[i] = 0u;  // (the passes below sync)
  unsigned *buf = use_smem ? dyn + mwords : gbuf;
  unsigned *kA = buf, *iA = buf + n, *kB = buf + 2 * n, *iB = buf + 3 * n;
  const int chunk = (n + 31) / 32;
  const int beg = min(n, w * chunk), end = min(n, beg + chunk);
  const unsigned *kin = bkey;
  const unsigned *iin = nullptr;
  unsigned *kout = kA, *iout = iA;
  for (unsigned shift = 0; shift < nbits; shift += 8) {
    for (int i = tid; i < 32 * 256; i += 1024) hist[i] = 0;
    __syncthreads();
    for (int i = beg + lane; i < end; i += 32) atomicAdd(&hist[w * 256 + ((kin[i] >> shift) & 255u)], 1u);
    __syncthreads();
    if (tid < 256) {
      unsigned sum = 0;
      for (int ww = 0; ww < 32; ++ww) {
        const unsigned c = hist[ww * 256 + tid];
        hist[ww * 256 + tid] = sum;
        sum += c;
      }
      dbase[tid] = sum;
    }
    __syncthreads();
    if (w == 0) {
      unsigned v[8], loc = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        v[j] = dbase[lane * 8 + j];
        loc += v[j];
      }
      unsigned incl = loc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      unsigned run = incl - loc;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const unsigned c = v[j];
        dbase[lane * 8 + j] = run;
        run += c;
      }
    }
    __syncthreads();
    if (tid < 256)
      for (int ww = 0; ww < 32; ++ww) hist[ww * 256 + tid] += dbase[tid];
    __syncthreads();
    for (int i0 = beg; i0 < end; i0 += 32) {
      const int i = i0 + lane;
      const bool ok = i < end;
      unsigned k = 0, id = 0, d = 256u + (unsigned)lane;
      if (ok) {
        k = kin[i];
        id = iin ? iin[i] : (unsigned)i;
        d = (k >> shift) & 255u;
      }
      const unsigned peers = __match_any_sync(0xffffffffu, d);
      const unsigned rank = __popc(peers & ((1u << lane) - 1u));
      if (ok) {
        const unsigned p = hist[w * 256 + d] + rank;
        kout[p] = k;
        iout[p] = id;
      }
      __syncwarp();
      if (ok && rank == 0) hist[w * 256 + d] += __popc(peers);
      __syncwarp();
    }
    __syncthreads();
    kin = kout;
    iin = iout;
    kout = (kout == kA) ? kB : kA;
    iout = (iout == iA) ? iB : iA;
  }
  // the permutation, the sorted keys and the mask of non-empty buckets (in
  // shared memory)
  for (int i = tid; i < n; i += 1024) {
    const unsigned k = kin[i];
    perm[i] = iin ? iin[i] : (unsigned)i;
    skey[i] = k;
    if (i == 0 || kin[i - 1] != k) atomicOr(&mask[k >> 5], 1u << (k & 31));
  }
  __syncthreads();
  // pencil mask: pencil (u, v) has stars when any of the buckets (u, v),
  // (u, v - 1), (u - 1, v), (u - 1, v - 1) (wrapped) does.  With rows of a
  // whole number of words this is word arithmetic: the bucket mask, its
  // one-bit shift along v within each row, and the same of the row above.
  const int nu = n_buckets / nv;
  if (nv % 32 == 0) {
    const int rw = nv / 32;  // words per row
    auto vshift = [&](int wd) {  // bits of (u, v - 1) for the pencils of word wd
      const int row0 = wd - wd % rw;
      const int prev = wd == row0 ? row0 + rw - 1 : wd - 1;
      return (mask[wd] << 1) | (mask[prev] >> 31);
    };
    for (int i = tid; i < mwords; i += 1024) {
      const int up = i >= rw ? i - rw : i + (nu - 1) * rw;
      pmask[i] = mask[i] | vshift(i) | mask[up] | vshift(up);
    }
  } else {
    for (int i = tid; i < mwords; i += 1024) {
      unsigned word = 0u;
      for (int j = 0; j < 32; ++j) {
        const int p = 32 * i + j;
        if (p >= n_buckets) break;
        const int cu = p / nv, cv = p - cu * nv;
        const int cum = cu == 0 ? nu - 1 : cu - 1, cvm = cv == 0 ? nv - 1 : cv - 1;
        const int nb[4] = {p, cum * nv + cv, cu * nv + cvm, cum * nv + cvm};
        unsigned on = 0u;
#pragma unroll
        for (int k = 0; k < 4; ++k) on |= (mask[nb[k] >> 5] >> (nb[k] & 31)) & 1u;
        word |= on << j;
      }
      pmask[i] = word;
    }
  }
}

// bstart[b] = first sorted position with bucket >= b, b = 0..n_buckets.
__global__ void k_bucket_starts(const unsigned *skey, int n, int n_buckets, int *bstart,
                                int bstride) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b > n_buckets) return;
  skey += (long long)blockIdx.y * n;
  bstart += (long long)blockIdx.y * bstride;
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (skey[mid] < (unsigned)b)
      lo = mid + 1;
    else
      hi = mid;
  }
  bstart[b] = lo;
}

// Largest bucket mask of a sort (512 x 512 pencils), in 32-bit words.
constexpr int kMaskWordsMax = 512 * 512 / 32;

int launch_bucket_sort(int n, int n_buckets, int nv, const StarBufs &b, cudaStream_t st, int nbox,
                       int bstride) {
  if (n <= 0) return 0;
  const int mwords = (n_buckets + 31) / 32;
  if (mwords > kMaskWordsMax || nv <= 0 || n_buckets % nv != 0) {
    set_error("internal: %d star buckets (rows of %d) do not fit the bucket mask", n_buckets, nv);
    return QJ_ERR_ARG;
  }
  const unsigned nbits = cell_bits(n_buckets);
  const int use_smem = n <= kSortSmemMax;
  const size_t smem = (size_t)4 * mwords + (use_smem ? (size_t)16 * n : 0);
  // the attribute belongs to the current device's context: set once per device
  static PerDevice<cudaError_t> attr;
  const cudaError_t *attr_err = nullptr;
  QJ_CK(per_device(attr, attr_err, [](cudaError_t &r) {
    r = cudaFuncSetAttribute(k_bucket_sort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             16 * kSortSmemMax + 4 * kMaskWordsMax);
  }));
  QJ_CK(*attr_err);
  k_bucket_sort<<<nbox, 1024, smem, st>>>(b.bkey, n, nbits < 8 ? 8 : nbits, b.sortbuf, use_smem,
                                          b.perm, b.skey, n_buckets, nv, b.pmask, b.mstride);
  QJ_CK_LAUNCH();
  const int T = 256, B = (n_buckets + 1 + T - 1) / T;
  k_bucket_starts<<<dim3(B, nbox), T, 0, st>>>(b.skey, n, n_buckets, b.bstart, bstride);
  QJ_CK_LAUNCH();
  return 0;
}

// Leapfrog update of the fused path.  acc = sum over the 8 corners, in the
// order of quantum-stars.py:264-287, of (w_x w_y w_z) * a(corner), with the
// corner accelerations A[8 s + c] written by the kick pass; then the half
// kicks, dt_s, drift and (optionally) the CIC data of the new positions.
__global__ void k_update_fused(float *pos, float *vel, const float *A, int n, CicGeom<float> g,
                               float dt, int k2, int k1, int drift, float *dts, int q_next,
                               const float *masses, float fac_all, int4 *sidx, float4 *sw0,
                               float4 *sw1, unsigned *bkey, int box_stars) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  dts += s / box_stars;  // dt_s of this star's box
  const float4 w0 = sw0[s], w1 = sw1[s];
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int bx = c_corner[c][0], by = c_corner[c][1], bz = c_corner[c][2];
    const float wp = fmul_rn(fmul_rn(bx ? w1.x : w0.x, by ? w1.y : w0.y), bz ? w1.z : w0.z);
    const float *ac = A + 3 * (8 * s + c);
    a0 = fadd_rn(a0, fmul_rn(wp, ac[0]));
    a1 = fadd_rn(a1, fmul_rn(wp, ac[1]));
    a2 = fadd_rn(a2, fmul_rn(wp, ac[2]));
  }
  const float acc[3] = {a0, a1, a2};
  float v[3];
  float dmin = INFINITY;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    v[d] = vel[3 * s + d];
    const float h = fdiv_rn(fmul_rn(acc[d], dt), 2.0f);
    if (k2) {
      v[d] = fadd_rn(v[d], h);
      dmin = fminf(dmin, fabsf(fdiv_rn(g.d[0], v[d])));
    }
    if (k1) v[d] = fadd_rn(v[d], h);
    vel[3 * s + d] = v[d];
  }
  if (k2) atomic_min_nonneg((unsigned int *)dts, dmin);
  if (drift) {
#pragma unroll
    for (int d = 0; d < 3; ++d) pos[3 * s + d] = ref_mod(fadd_rn(pos[3 * s + d], fmul_rn(v[d], dt)), g.L[d]);
    if (q_next >= 0)
      star_prepare(pos, s, g, cic_fac<float>(masses, s, fac_all, g.vol), q_next, sidx, sw0, sw1, bkey);
  }
}

int launch_update_fused(void *pos, void *vel, const CicGeomD &g, const UpdateArgs &u,
                        const StarBufs &b, cudaStream_t st) {
  if (u.n <= 0) return 0;
  const int T = 128, B = (u.n + T - 1) / T;
  const double fac = u.m_s / (g.d[0] * g.d[1] * g.d[2]);
  k_update_fused<<<B, T, 0, st>>>((float *)pos, (float *)vel, b.A, u.n, cast_geom<float>(g),
                                  (float)u.dt, u.k2, u.k1, u.drift, (float *)u.dts_bits, u.q_next,
                                  (const float *)u.masses, (float)fac, b.sidx, b.sw0, b.sw1, b.bkey,
                                  u.box_stars > 0 ? u.box_stars : u.n);
  QJ_CK_LAUNCH();
  return 0;
}

// ----- scalar state kernels -----
// amax / dt_s are kept as the real type's bit pattern (non-negative values,
// ordered like unsigned integers) so atomicMax / atomicMin are exact.
template <typename R> __global__ void k_diag_load(const double *diag, R *amax, int nbox) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nbox) amax[b] = (R)diag[3 * b + 1];
}
template <typename R>
__global__ void k_diag_store(double *diag, const R *amax, const R *dts, int has_particles,
                             double t_add, int nbox) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbox) return;
  diag[3 * b + 0] += t_add;
  diag[3 * b + 1] = (double)amax[b];
  diag[3 * b + 2] = has_particles ? (double)dts[b] : (double)INFINITY;
}
template <typename R> __global__ void k_set_scalar(R *dst, double v, int count) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < count) dst[b] = (R)v;
}
template <typename R> __global__ void k_to_double(const R *src, double *out) { *out = (double)*src; }

int launch_diag_load(bool dbl, const void *diag, void *amax_bits, cudaStream_t st, int nbox) {
  const int B = (nbox + 127) / 128;
  if (dbl)
    k_diag_load<double><<<B, 128, 0, st>>>((const double *)diag, (double *)amax_bits, nbox);
  else
    k_diag_load<float><<<B, 128, 0, st>>>((const double *)diag, (float *)amax_bits, nbox);
  QJ_CK_LAUNCH();
  return 0;
}
int launch_diag_store(bool dbl, void *diag, const void *amax_bits, const void *dts_bits,
                      int has_particles, double t_add, cudaStream_t st, int nbox) {
  const int B = (nbox + 127) / 128;
  if (dbl)
    k_diag_store<double><<<B, 128, 0, st>>>((double *)diag, (const double *)amax_bits,
                                            (const double *)dts_bits, has_particles, t_add, nbox);
  else
    k_diag_store<float><<<B, 128, 0, st>>>((double *)diag, (const float *)amax_bits,
                                           (const float *)dts_bits, has_particles, t_add, nbox);
  QJ_CK_LAUNCH();
  return 0;
}
int launch_set_scalar(bool dbl, void *dst, double v, cudaStream_t st, int count) {
  const int B = (count + 127) / 128;
  if (dbl)
    k_set_scalar<double><<<B, 128, 0, st>>>((double *)dst, v, count);
  else
    k_set_scalar<float><<<B, 128, 0, st>>>((float *)dst, v, count);
  QJ_CK_LAUNCH();
  return 0;
}
int launch_bits_to_double(bool dbl, const void *bits, double *out, cudaStream_t st) {
  if (dbl)
    k_to_double<double><<<1, 1, 0, st>>>((const double *)bits, out);
  else
    k_to_double<float><<<1, 1, 0, st>>>((const float *)bits, out);
  QJ_CK_LAUNCH();
  return 0;
}

}  // namespace qj
