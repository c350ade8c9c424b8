// Plain (unfused) elementwise kernels.  Each one is one line of the
// reference's step functions, in the reference's operation order; the plain
// float64 step strings them together with full 3-D FFTs exactly as
// quantum-stars.py:295-330 does.
#include "qj_internal.h"

namespace qj {

template <typename R> struct KT {
  const R *k[3];
  int n[3];
};
template <typename R> static KT<R> cast_k(const KTabs &k) {
  KT<R> o;
  for (int i = 0; i < 3; ++i) {
    o.k[i] = (const R *)k.k[i];
    o.n[i] = k.n[i];
  }
  return o;
}
template <typename R>
__device__ __forceinline__ void cell_k(const KT<R> &k, long long idx, R &kx, R &ky, R &kz) {
  const int iz = (int)(idx % k.n[2]);
  const long long r = idx / k.n[2];
  const int iy = (int)(r % k.n[1]);
  const int ix = (int)(r / k.n[1]);
  kx = k.k[0][ix];
  ky = k.k[1][iy];
  kz = k.k[2][iz];
}

#define GRID_LOOP(i, n) \
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

static int grid_blocks(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

// rho_tot = |psi|^2 + rho_s + rho_gas (quantum-stars.py:299, gas-bh :542), or
// rho_in; cbuf = 4 pi G (rho_tot - rho_bar) as a complex field (the argument
// of fftn in get_potential, :191).
template <typename R>
__global__ void k_build_rho(const cplx<R> *psi, const R *rho_s, const R *rho_gas, const R *rho_in,
                            R fourpiG, R rho_bar, R *rho_tot, cplx<R> *cbuf, long long n) {
  GRID_LOOP(i, n) {
    R r;
    if (rho_in) {
      r = rho_in[i];
    } else {
      const R a = hypot(psi[i].x, psi[i].y);
      r = a * a;
      if (rho_s) r = r + rho_s[i];
      if (rho_gas) r = r + rho_gas[i];
    }
    if (rho_tot) rho_tot[i] = r;
    cbuf[i] = cplx<R>{fourpiG * (r - rho_bar), (R)0};
  }
}

// V^ = -F / (k^2 + [k^2 == 0])  (quantum-stars.py:191)
template <typename R> __global__ void k_poisson_div(cplx<R> *c, KT<R> k, long long n) {
  GRID_LOOP(i, n) {
    R kx, ky, kz;
    cell_k(k, i, kx, ky, kz);
    const R k2 = kx * kx + ky * ky + kz * kz;
    const R den = k2 + (k2 == (R)0 ? (R)1 : (R)0);
    c[i] = cplx<R>{-c[i].x / den, -c[i].y / den};
  }
}

// out = 1j * k_d * V^  (quantum-stars.py:256-258)
template <typename R>
__global__ void k_mul_ik(const cplx<R> *vh, int d, KT<R> k, cplx<R> *out, long long n) {
  GRID_LOOP(i, n) {
    R kk[3];
    cell_k(k, i, kk[0], kk[1], kk[2]);
    const R kd = kk[d];
    out[i] = cplx<R>{-kd * vh[i].y, kd * vh[i].x};
  }
}

// out = sign * Re(c) (+ b * rho) (+ v_ext)
template <typename R>
__global__ void k_real_part(const cplx<R> *c, R sign, const R *rho, R b, const R *vext, R *out,
                            long long n) {
  GRID_LOOP(i, n) {
    R v = sign * c[i].x;
    if (rho) v = v + b * rho[i];
    if (vext) v = v + vext[i];
    out[i] = v;
  }
}

// psi = exp(-1j * coef * V) * psi, coef = m_per_hbar * dt / 2 (:301)
template <typename R> __global__ void k_kick_plain(cplx<R> *psi, const R *V, R coef, long long n) {
  GRID_LOOP(i, n) {
    R s, c;
    const R th = -coef * V[i];
    if constexpr (sizeof(R) == 8)
      sincos((double)th, (double *)&s, (double *)&c);
    else
      sincosf((float)th, (float *)&s, (float *)&c);
    const cplx<R> z = psi[i];
    psi[i] = cplx<R>{c * z.x - s * z.y, c * z.y + s * z.x};
  }
}

// psi_hat *= exp(dt * (-1j * k_sq / m_per_hbar / 2))  (:308)
template <typename R>
__global__ void k_drift_mul(cplx<R> *c, KT<R> k, R dt, R mph, long long n) {
  GRID_LOOP(i, n) {
    R kx, ky, kz;
    cell_k(k, i, kx, ky, kz);
    const R k2 = kx * kx + ky * ky + kz * kz;
    const R th = dt * (-(k2 / mph / (R)2));
    R s, cc;
    if constexpr (sizeof(R) == 8)
      sincos((double)th, (double *)&s, (double *)&cc);
    else
      sincosf((float)th, (float *)&s, (float *)&cc);
    const cplx<R> z = c[i];
    c[i] = cplx<R>{cc * z.x - s * z.y, cc * z.y + s * z.x};
  }
}

// a_max = max |a_grid| over the three components (:260)
template <typename R>
__global__ void k_amax3(const R *ax, const R *ay, const R *az, long long n, R *out) {
  R m = (R)0;
  GRID_LOOP(i, n) {
    m = fmax(m, fabs(ax[i]));
    m = fmax(m, fabs(ay[i]));
    m = fmax(m, fabs(az[i]));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) {
    if constexpr (sizeof(R) == 4)
      atomic_max_nonneg((unsigned int *)out, (float)m);
    else
      atomic_max_nonneg((unsigned long long *)out, (double)m);
  }
}

// v += a * dt (quantum-gas-bh.py:262-264)
template <typename R>
__global__ void k_gas_kick(R *vx, R *vy, R *vz, const R *ax, const R *ay, const R *az, R dt,
                           long long n) {
  GRID_LOOP(i, n) {
    vx[i] = vx[i] + ax[i] * dt;
    vy[i] = vy[i] + ay[i] * dt;
    vz[i] = vz[i] + az[i] * dt;
  }
}

// ----- adjoint of the kick psi' = exp(-i c V[|psi|^2]) psi -----
// (real adjoint with the gradient convention g = dL/dRe + i dL/dIm)
template <typename R> __device__ __forceinline__ void phase_sc(double th, R &s, R &c) {
  if constexpr (sizeof(R) == 8) {
    sincos(th, &s, &c);
  } else {
    float sf, cf;
    sincos_reduced(th, sf, cf);
    s = sf;
    c = cf;
  }
}

// mu = c Im(conj(g) psi'), psi' = exp(-i c V) psi
template <typename R>
__global__ void k_adj_mu(const cplx<R> *g, const cplx<R> *psi, const R *V, double coef, R *mu,
                         R fourpiG, cplx<R> *cbuf, long long n) {
  GRID_LOOP(i, n) {
    R s, c;
    phase_sc<R>(coef * (double)V[i], s, c);
    const cplx<R> z = psi[i];
    const cplx<R> zp = cplx<R>{z.x * c + z.y * s, z.y * c - z.x * s};
    const cplx<R> w = g[i];
    const R m = (R)coef * (w.x * zp.y - w.y * zp.x);
    if (mu) mu[i] = m;
    cbuf[i] = cplx<R>{fourpiG * m, (R)0};  // the source of L mu
  }
}

// g <- exp(+i c V) g + 2 W psi with W = Re(cbuf) (+ b mu)
template <typename R>
__global__ void k_adj_update(cplx<R> *g, const cplx<R> *psi, const R *V, const cplx<R> *cbuf,
                             const R *mu, R b, double coef, long long n) {
  GRID_LOOP(i, n) {
    R s, c;
    phase_sc<R>(coef * (double)V[i], s, c);
    R W = cbuf[i].x;
    if (mu) W = W + b * mu[i];
    const cplx<R> w = g[i];
    const R two_w = (R)2 * W;
    g[i] = cplx<R>{w.x * c - w.y * s + two_w * psi[i].x, w.y * c + w.x * s + two_w * psi[i].y};
  }
}

int launch_adj_mu(bool dbl, const void *g, const void *psi, const void *V, double coef, void *mu,
                  double fourpiG, void *cbuf, long long ncell, cudaStream_t st) {
  if (dbl)
    k_adj_mu<double><<<grid_blocks(ncell), 256, 0, st>>>(
        (const double2 *)g, (const double2 *)psi, (const double *)V, coef, (double *)mu, fourpiG,
        (double2 *)cbuf, ncell);
  else
    k_adj_mu<float><<<grid_blocks(ncell), 256, 0, st>>>(
        (const float2 *)g, (const float2 *)psi, (const float *)V, coef, (float *)mu, (float)fourpiG,
        (float2 *)cbuf, ncell);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_adj_update(bool dbl, void *g, const void *psi, const void *V, const void *cbuf,
                      const void *mu, double b, double coef, long long ncell, cudaStream_t st) {
  if (dbl)
    k_adj_update<double><<<grid_blocks(ncell), 256, 0, st>>>(
        (double2 *)g, (const double2 *)psi, (const double *)V, (const double2 *)cbuf,
        (const double *)mu, b, coef, ncell);
  else
    k_adj_update<float><<<grid_blocks(ncell), 256, 0, st>>>(
        (float2 *)g, (const float2 *)psi, (const float *)V, (const float2 *)cbuf, (const float *)mu,
        (float)b, coef, ncell);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_build_rho(bool dbl, const void *psi, const void *rho_s, const void *rho_gas,
                     const void *rho_in, double fourpiG, double rho_bar, void *rho_tot,
                     void *cbuf, long long ncell, cudaStream_t st) {
  if (dbl)
    k_build_rho<double><<<grid_blocks(ncell), 256, 0, st>>>(
        (const double2 *)psi, (const double *)rho_s, (const double *)rho_gas,
        (const double *)rho_in, fourpiG, rho_bar, (double *)rho_tot, (double2 *)cbuf, ncell);
  else
    k_build_rho<float><<<grid_blocks(ncell), 256, 0, st>>>(
        (const float2 *)psi, (const float *)rho_s, (const float *)rho_gas, (const float *)rho_in,
        (float)fourpiG, (float)rho_bar, (float *)rho_tot, (float2 *)cbuf, ncell);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_poisson_div(bool dbl, void *cbuf, const KTabs &k, long long ncell, cudaStream_t st) {
  if (dbl)
    k_poisson_div<double><<<grid_blocks(ncell), 256, 0, st>>>((double2 *)cbuf, cast_k<double>(k), ncell);
  else
    k_poisson_div<float><<<grid_blocks(ncell), 256, 0, st>>>((float2 *)cbuf, cast_k<float>(k), ncell);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_mul_ik(bool dbl, const void *vh, int d, const KTabs &k, void *out, long long ncell,
                  cudaStream_t st) {
  if (dbl)
    k_mul_ik<double><<<grid_blocks(ncell), 256, 0, st>>>((const double2 *)vh, d, cast_k<double>(k),
                                                         (double2 *)out, ncell);
  else
    k_mul_ik<float><<<grid_blocks(ncell), 256, 0, st>>>((const float2 *)vh, d, cast_k<float>(k),
                                                        (float2 *)out, ncell);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_real_part(bool dbl, const void *c, double sign, const void *rho, double b,
                     const void *vext, void *out, long long ncell, cudaStream_t st) {
  if (dbl)
    k_real_part<double><<<grid_blocks(ncell), 256, 0, st>>>(
        (const double2 *)c, sign, (const double *)rho, b, (const double *)vext, (double *)out, ncell);
  else
    k_real_part<float><<<grid_blocks(ncell), 256, 0, st>>>(
        (const float2 *)c, (float)sign, (const float *)rho, (float)b, (const float *)vext,
        (float *)out, ncell);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_kick_plain(bool dbl, void *psi, const void *V, double coef, long long ncell,
                      cudaStream_t st) {
  if (dbl)
    k_kick_plain<double><<<grid_blocks(ncell), 256, 0, st>>>((double2 *)psi, (const double *)V, coef, ncell);
  else
    k_kick_plain<float><<<grid_blocks(ncell), 256, 0, st>>>((float2 *)psi, (const float *)V, (float)coef, ncell);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_drift_mul(bool dbl, void *cbuf, const KTabs &k, double dt_kin, double m_per_hbar,
                     long long ncell, cudaStream_t st) {
  if (dbl)
    k_drift_mul<double><<<grid_blocks(ncell), 256, 0, st>>>((double2 *)cbuf, cast_k<double>(k), dt_kin,
                                                            m_per_hbar, ncell);
  else
    k_drift_mul<float><<<grid_blocks(ncell), 256, 0, st>>>((float2 *)cbuf, cast_k<float>(k),
                                                           (float)dt_kin, (float)m_per_hbar, ncell);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_amax3(bool dbl, const void *ax, const void *ay, const void *az, long long ncell,
                 void *bits, cudaStream_t st) {
  if (dbl)
    k_amax3<double><<<grid_blocks(ncell), 256, 0, st>>>((const double *)ax, (const double *)ay,
                                                        (const double *)az, ncell, (double *)bits);
  else
    k_amax3<float><<<grid_blocks(ncell), 256, 0, st>>>((const float *)ax, (const float *)ay,
                                                       (const float *)az, ncell, (float *)bits);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_gas_kick(bool dbl, void *vx, void *vy, void *vz, const void *ax, const void *ay,
                    const void *az, double dt, long long ncell, cudaStream_t st) {
  if (dbl)
    k_gas_kick<double><<<grid_blocks(ncell), 256, 0, st>>>(
        (double *)vx, (double *)vy, (double *)vz, (const double *)ax, (const double *)ay,
        (const double *)az, dt, ncell);
  else
    k_gas_kick<float><<<grid_blocks(ncell), 256, 0, st>>>(
        (float *)vx, (float *)vy, (float *)vz, (const float *)ax, (const float *)ay,
        (const float *)az, (float)dt, ncell);
  QJ_CK_LAUNCH();
  return 0;
}

}  // namespace qj

// ---------------------------------------------------------------------------
// Pieces of the quantum-fluid-accretion step (quantum-fluid-accretion.py)
// ---------------------------------------------------------------------------
namespace qj {
namespace {

// c *= exp(-(k^2 / (p + 1e-30))^4)   (kind 0: the low-pass LP, p = k_cut^2, :143-145)
// c *= exp((-0.5 p) k^2)             (kind 1: Gaussian smoothing, p = r^2, :731-733, 849)
template <typename R>
__global__ void k_kfilter(cplx<R> *c, KT<R> k, int kind, R p, long long n) {
  GRID_LOOP(i, n) {
    R kx, ky, kz;
    cell_k(k, i, kx, ky, kz);
    const R k2 = kx * kx + ky * ky + kz * kz;
    const R f = kind == 0 ? exp(-pow(k2 / (p + (R)1e-30), (R)4)) : exp(((R)-0.5 * p) * k2);
    c[i] = cplx<R>{c[i].x * f, c[i].y * f};
  }
}

// CIC cells and weights of a point, the corner order of bh_cic_density (:388-417)
template <typename R>
__device__ void point_cic(const double *x, int n, double dx, long long cells[8], R w[8]) {
  double f[3];
  long long i0[3];
  for (int d = 0; d < 3; ++d) {
    const double xi = x[d] / dx - 0.5;
    const double fl = floor(xi);
    i0[d] = (long long)fl;
    f[d] = xi - fl;
  }
  const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                         {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
  for (int c = 0; c < 8; ++c) {
    long long id[3];
    for (int d = 0; d < 3; ++d) id[d] = (((i0[d] + off[c][d]) % n) + n) % n;
    cells[c] = (id[0] * n + id[1]) * n + id[2];
    const double a = off[c][0] ? f[0] : 1.0 - f[0];
    const double b = off[c][1] ? f[1] : 1.0 - f[1];
    const double e = off[c][2] ? f[2] : 1.0 - f[2];
    w[c] = (R)(a * b * e);
  }
}

// grid[cell] += w M / dx^3 in corner order (bh_cic_density), one thread
template <typename R>
__global__ void k_cic_point(R *grid, int n, double x0, double x1, double x2, double dx, double M) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double x[3] = {x0, x1, x2};
  long long cells[8];
  R w[8];
  point_cic<R>(x, n, dx, cells, w);
  for (int c = 0; c < 8; ++c) grid[cells[c]] = grid[cells[c]] + w[c] * (R)(M / (dx * dx * dx));
}

// sum_c w_c f[cell_c] for three fields (_sample_cic, :419-437), one thread
template <typename R>
__global__ void k_cic_sample3(const R *f0, const R *f1, const R *f2, int n, double x0, double x1,
                              double x2, double dx, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double x[3] = {x0, x1, x2};
  long long cells[8];
  R w[8];
  point_cic<R>(x, n, dx, cells, w);
  const R *f[3] = {f0, f1, f2};
  for (int d = 0; d < 3; ++d) {
    double s = 0.0;
    for (int c = 0; c < 8; ++c) s += (double)(w[c] * f[d][cells[c]]);
    out[d] = s;
  }
}

// per-block float64 sums of |psi|^2 and rho
template <typename R>
__global__ void k_sum_dm_gas(const cplx<R> *psi, const R *rho, long long n, double *part) {
  __shared__ double red[2][256];
  double a = 0.0, b = 0.0;
  GRID_LOOP(i, n) {
    const double m = hypot((double)psi[i].x, (double)psi[i].y);
    a += m * m;
    b += (double)rho[i];
  }
  red[0][threadIdx.x] = a;
  red[1][threadIdx.x] = b;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      red[0][threadIdx.x] += red[0][threadIdx.x + s];
      red[1][threadIdx.x] += red[1][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = red[0][0];
    part[2 * blockIdx.x + 1] = red[1][0];
  }
}
__global__ void k_mean_final(const double *part, int nb, long long n, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double a = 0.0, b = 0.0;
  for (int i = 0; i < nb; ++i) {
    a += part[2 * i];
    b += part[2 * i + 1];
  }
  out[0] = a / (double)n;
  out[1] = b / (double)n;
}

// first index of the maximum (jnp.argmax), per block then final
template <typename R>
__global__ void k_argmax_part(const R *f, long long n, double *pv, long long *pi) {
  __shared__ double sv[256];
  __shared__ long long si[256];
  double bv = -INFINITY;
  long long bi = n;
  GRID_LOOP(i, n) {
    const double v = (double)f[i];
    if (v > bv || (v == bv && i < bi)) {
      bv = v;
      bi = i;
    }
  }
  sv[threadIdx.x] = bv;
  si[threadIdx.x] = bi;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      const double v = sv[threadIdx.x + s];
      const long long j = si[threadIdx.x + s];
      if (v > sv[threadIdx.x] || (v == sv[threadIdx.x] && j < si[threadIdx.x])) {
        sv[threadIdx.x] = v;
        si[threadIdx.x] = j;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    pv[blockIdx.x] = sv[0];
    pi[blockIdx.x] = si[0];
  }
}
__global__ void k_argmax_final(const double *pv, const long long *pi, int nb, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double bv = -INFINITY;
  long long bi = -1;
  for (int b = 0; b < nb; ++b)
    if (pv[b] > bv || (pv[b] == bv && pi[b] < bi)) {
      bv = pv[b];
      bi = pi[b];
    }
  out[0] = (double)bi;
}

}  // namespace

int launch_kfilter(bool dbl, void *c, const KTabs &k, int kind, double p, long long ncell,
                   cudaStream_t st) {
  if (dbl)
    k_kfilter<double><<<grid_blocks(ncell), 256, 0, st>>>((double2 *)c, cast_k<double>(k), kind, p, ncell);
  else
    k_kfilter<float><<<grid_blocks(ncell), 256, 0, st>>>((float2 *)c, cast_k<float>(k), kind, (float)p, ncell);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_cic_point(bool dbl, void *grid, int n, const double x[3], double dx, double M,
                     cudaStream_t st) {
  if (dbl)
    k_cic_point<double><<<1, 32, 0, st>>>((double *)grid, n, x[0], x[1], x[2], dx, M);
  else
    k_cic_point<float><<<1, 32, 0, st>>>((float *)grid, n, x[0], x[1], x[2], dx, M);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_cic_sample3(bool dbl, const void *f0, const void *f1, const void *f2, int n,
                       const double x[3], double dx, double *out, cudaStream_t st) {
  if (dbl)
    k_cic_sample3<double><<<1, 32, 0, st>>>((const double *)f0, (const double *)f1,
                                            (const double *)f2, n, x[0], x[1], x[2], dx, out);
  else
    k_cic_sample3<float><<<1, 32, 0, st>>>((const float *)f0, (const float *)f1,
                                           (const float *)f2, n, x[0], x[1], x[2], dx, out);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_mean_dm_gas(bool dbl, const void *psi, const void *rho, long long ncell, double *part,
                       int nb, double *out, cudaStream_t st) {
  if (dbl)
    k_sum_dm_gas<double><<<nb, 256, 0, st>>>((const double2 *)psi, (const double *)rho, ncell, part);
  else
    k_sum_dm_gas<float><<<nb, 256, 0, st>>>((const float2 *)psi, (const float *)rho, ncell, part);
  QJ_CK_LAUNCH();
  k_mean_final<<<1, 32, 0, st>>>(part, nb, ncell, out);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_argmax(bool dbl, const void *f, long long ncell, double *pv, long long *pi, int nb,
                  double *out, cudaStream_t st) {
  if (dbl)
    k_argmax_part<double><<<nb, 256, 0, st>>>((const double *)f, ncell, pv, pi);
  else
    k_argmax_part<float><<<nb, 256, 0, st>>>((const float *)f, ncell, pv, pi);
  QJ_CK_LAUNCH();
  k_argmax_final<<<1, 32, 0, st>>>(pv, pi, nb, out);
  QJ_CK_LAUNCH();
  return 0;
}

}  // namespace qj
