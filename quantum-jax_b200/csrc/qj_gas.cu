// Isothermal gas and black-hole kernels (quantum-gas-bh.py, quantum-bh.py,
// quantum-fluid-accretion-test.py), templated on the real type.
//
// One MUSCL-Hancock update of solve_hydro (quantum-gas-bh.py:269-337) is two
// kernels, like the reference's whole-grid arrays: k_hydro_prim stores every
// cell's limited gradients and half-step primitives (16 values per cell,
// structure of arrays); k_hydro_update reads its cell's and its six face
// neighbours' records, forms the fluxes through its six faces and applies the
// flux-form update in place, in the same floating-point order as the
// reference.  The grid is cubic with spacing dx, as in the reference.
#include <algorithm>
#include <cmath>

#include "../../include/qj.h"
#include "qj_internal.h"

namespace qj {

namespace {

template <typename R> struct Prim {
  R f[4];      // predicted primitives rho', vx', vy', vz'
  R g[4][3];   // limited gradients of rho, vx, vy, vz along x, y, z
};

// Periodic index of a cell at most one cell outside [0, n) on each axis.
struct Idx3 {
  int n;
  __device__ __forceinline__ static int wrap1(int x, int n) {
    return x < 0 ? x + n : (x >= n ? x - n : x);
  }
  __device__ __forceinline__ long long at(int x, int y, int z) const {
    return ((long long)wrap1(x, n) * n + wrap1(y, n)) * n + wrap1(z, n);
  }
};

// Coordinates of linear cell index i of an n^3 box; 32-bit divisions (the
// hydro grids hold fewer than 2^32 cells, checked on the host)
__device__ __forceinline__ void cell_xyz(long long i, int n, int &x, int &y, int &z) {
  const unsigned u = (unsigned)i, un = (unsigned)n, q = u / un;
  z = (int)(u - q * un);
  x = (int)(q / un);
  y = (int)(q - (unsigned)x * un);
}

// Linear index of cell (x, y, z) of an n^3 periodic box and of its six face
// neighbours: up[d] / dn[d] = the next / previous cell along x, y, z.
struct Nbr {
  long long c, up[3], dn[3];
  __device__ __forceinline__ Nbr(int n, int x, int y, int z) {
    const long long n1 = n, n2 = n1 * n1;
    c = ((long long)x * n1 + y) * n1 + z;
    up[0] = x == n - 1 ? c - (n1 - 1) * n2 : c + n2;
    dn[0] = x == 0 ? c + (n1 - 1) * n2 : c - n2;
    up[1] = y == n - 1 ? c - (n1 - 1) * n1 : c + n1;
    dn[1] = y == 0 ? c + (n1 - 1) * n1 : c - n1;
    up[2] = z == n - 1 ? c - (n1 - 1) : c + 1;
    dn[2] = z == 0 ? c + (n1 - 1) : c - 1;
  }
};

// a / b in the hydro stencils: correctly rounded in float64 (the path pinned
// to the reference at 1e-10); the fast divide (within 2 ulp) in float32,
// whose stencils are bound by their divisions
template <typename R> __device__ __forceinline__ R hdiv(R a, R b) {
  if constexpr (sizeof(R) == 4) {
    return __fdividef(a, b);
  } else {
    return a / b;
  }
}

// quantum-gas-bh.py:353-357
template <typename R> __device__ __forceinline__ R adjust_denominator(R d) {
  const R eps = (R)1.0e-12;
  return d > (R)0 ? d + eps : (d < (R)0 ? d - eps : eps);
}
template <typename R> __device__ __forceinline__ R clamp01(R x) {
  return fmax((R)0, fmin((R)1, x));
}

// Limited gradients and half-step primitives of cell (x, y, z):
// get_gradient (:188-193), slope_limiter (:340-395), predictor (:283-299).
// FACC: solve_hydro of quantum-fluid-accretion.py:273-317 -- the velocity
// predictor uses the limited gradient of P = rho c^2 divided by (rho + eps)
// instead of c^2 grad(rho) / rho.
template <typename R, bool FACC = false>
__device__ Prim<R> cell_prim(const R *const F[4], const Idx3 &I, int x, int y, int z, R dx, R dt,
                             R cs) {
  Prim<R> P;
  R c[4];
  const Nbr nb(I.n, x, y, z);
  for (int v = 0; v < 4; ++v) c[v] = F[v][nb.c];
  for (int v = 0; v < 4; ++v) {
    for (int d = 0; d < 3; ++d) {
      const R fp = F[v][nb.up[d]];
      const R fm = F[v][nb.dn[d]];
      R g = hdiv(fp - fm, (R)2 * dx);
      const R denom = adjust_denominator(g);
      g = clamp01(hdiv(hdiv(c[v] - fm, dx), denom)) * g;
      g = clamp01(hdiv(hdiv(-(c[v] - fp), dx), denom)) * g;
      P.g[v][d] = g;
    }
  }
  const R rho = c[0], vx = c[1], vy = c[2], vz = c[3];
  const R h = (R)0.5 * dt;
  P.f[0] = rho - h * (vx * P.g[0][0] + rho * P.g[1][0] + vy * P.g[0][1] + rho * P.g[2][1] +
                      vz * P.g[0][2] + rho * P.g[3][2]);
  if constexpr (FACC) {
    const R c2 = cs * cs;
    const R Pc = c[0] * c2;
    R gP[3];
    for (int d = 0; d < 3; ++d) {
      const R fp = F[0][nb.up[d]] * c2;
      const R fm = F[0][nb.dn[d]] * c2;
      R g = hdiv(fp - fm, (R)2 * dx);
      const R denom = adjust_denominator(g);
      g = clamp01(hdiv(hdiv(Pc - fm, dx), denom)) * g;
      g = clamp01(hdiv(hdiv(-(Pc - fp), dx), denom)) * g;
      gP[d] = g;
    }
    for (int v = 1; v < 4; ++v)
      P.f[v] = c[v] - h * (vx * P.g[v][0] + vy * P.g[v][1] + vz * P.g[v][2] +
                           hdiv(gP[v - 1], rho + (R)1e-30));
  } else {
    for (int v = 1; v < 4; ++v)
      P.f[v] = c[v] - h * (vx * P.g[v][0] + vy * P.g[v][1] + vz * P.g[v][2] +
                           hdiv((R)1, rho) * P.g[0][v - 1] * cs * cs);
  }
  return P;
}

// get_flux (:226-252) with the rotated variable order of :316-324.  u = the
// velocity component normal to the face; w1, w2 the tangential ones.
// FACC: get_flux_axis of quantum-fluid-accretion.py:252-271 (face-averaged
// c^2, eps-guarded divisions, C = sqrt(c^2) + |u|).
template <typename R, bool FACC = false>
__device__ __forceinline__ void rusanov(R rL, R uL, R aL, R bL, R rR, R uR, R aR, R bR, R cs,
                                        R out[4]) {
  const R rho_star = (R)0.5 * (rL + rR);
  const R mu = (R)0.5 * (rL * uL + rR * uR);
  const R ma = (R)0.5 * (rL * aL + rR * aR);
  const R mb = (R)0.5 * (rL * bL + rR * bR);
  R fM, fU, fA, fB, C;
  if constexpr (FACC) {
    const R c2 = cs * cs;
    const R P_star = rho_star * ((R)0.5 * (c2 + c2));
    const R eps = (R)1e-30;
    fM = mu;
    fU = hdiv(mu * mu, rho_star + eps) + P_star;
    fA = hdiv(mu * ma, rho_star + eps);
    fB = hdiv(mu * mb, rho_star + eps);
    C = fmax(sqrt(c2) + fabs(uL), sqrt(c2) + fabs(uR));
  } else {
    const R P_star = rho_star * cs * cs;
    fM = mu;
    fU = hdiv(mu * mu, rho_star) + P_star;
    fA = hdiv(mu * ma, rho_star);
    fB = hdiv(mu * mb, rho_star);
    C = fmax(cs + fabs(uL), cs + fabs(uR));
  }
  fM = fM - C * (R)0.5 * (rR - rL);
  fU = fU - C * (R)0.5 * (rR * uR - rL * uL);
  fA = fA - C * (R)0.5 * (rR * aR - rL * aL);
  fB = fB - C * (R)0.5 * (rR * bR - rL * bL);
  out[0] = fM;
  out[1] = fU;
  out[2] = fA;
  out[3] = fB;
}

// Flux through the face between cell L and its +d neighbour R, returned in
// conserved order (Mass, Momx, Momy, Momz).  Face states: extrap_to_face
// (:196-209).
template <typename R, bool FACC = false>
__device__ void face_flux(const Prim<R> &L, const Prim<R> &Rt, int d, R dx, R cs, R out[4]) {
  R fl[4], fr[4];
  for (int v = 0; v < 4; ++v) {
    fl[v] = L.f[v] + (R)0.5 * L.g[v][d] * dx;
    fr[v] = Rt.f[v] - (R)0.5 * Rt.g[v][d] * dx;
  }
  R o[4];
  if (d == 0) {
    rusanov<R, FACC>(fl[0], fl[1], fl[2], fl[3], fr[0], fr[1], fr[2], fr[3], cs, o);
    out[0] = o[0]; out[1] = o[1]; out[2] = o[2]; out[3] = o[3];
  } else if (d == 1) {  // (rho, vy, vz, vx) -> (Mass, Momy, Momz, Momx)
    rusanov<R, FACC>(fl[0], fl[2], fl[3], fl[1], fr[0], fr[2], fr[3], fr[1], cs, o);
    out[0] = o[0]; out[2] = o[1]; out[3] = o[2]; out[1] = o[3];
  } else {  // (rho, vz, vx, vy) -> (Mass, Momz, Momx, Momy)
    rusanov<R, FACC>(fl[0], fl[3], fl[1], fl[2], fr[0], fr[3], fr[1], fr[2], cs, o);
    out[0] = o[0]; out[3] = o[1]; out[1] = o[2]; out[2] = o[3];
  }
}

// Four values of one cell's record, stored together (16-byte loads and
// stores in float32, two per group in float64).
template <typename R> struct alignas(4 * sizeof(R)) Quad {
  R a, b, c, e;
};

// Record of one cell, four quads: Q[i] = the predicted primitives f[0..3],
// Q[(1 + d) ncell + i] = the gradients g[0..3][d] along axis d -- so a face
// along d reads two quads of each neighbour.
template <typename R, bool FACC>
__global__ void __launch_bounds__(256)
    k_hydro_prim(const R *rho, const R *vx, const R *vy, const R *vz, R *P, int n, R dx, R dt, R cs) {
  const long long ncell = (long long)n * n * n;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= ncell) return;
  int x, y, z;
  cell_xyz(i, n, x, y, z);
  const R *const F[4] = {rho, vx, vy, vz};
  const Prim<R> C = cell_prim<R, FACC>(F, Idx3{n}, x, y, z, dx, dt, cs);
  Quad<R> *Q = reinterpret_cast<Quad<R> *>(P);
  Q[i] = Quad<R>{C.f[0], C.f[1], C.f[2], C.f[3]};
#pragma unroll
  for (int d = 0; d < 3; ++d) Q[(1 + d) * ncell + i] = Quad<R>{C.g[0][d], C.g[1][d], C.g[2][d], C.g[3][d]};
}

// the primitives and the axis-d gradients of cell j (what face_flux uses)
template <typename R>
__device__ __forceinline__ void load_face_prim(const R *P, long long ncell, long long j, int d,
                                               Prim<R> &q) {
  const Quad<R> *Q = reinterpret_cast<const Quad<R> *>(P);
  const Quad<R> f = Q[j], g = Q[(1 + d) * ncell + j];
  q.f[0] = f.a;
  q.f[1] = f.b;
  q.f[2] = f.c;
  q.f[3] = f.e;
  q.g[0][d] = g.a;
  q.g[1][d] = g.b;
  q.g[2][d] = g.c;
  q.g[3][d] = g.e;
}

template <typename R, bool FACC>
__global__ void __launch_bounds__(256)
    k_hydro_update(R *rho, R *vx, R *vy, R *vz, const R *P, int n, R dx, R cs, R vol, R fac,
                   int clamp_rho) {
  const long long ncell = (long long)n * n * n;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= ncell) return;
  int x, y, z;
  cell_xyz(i, n, x, y, z);
  Prim<R> C;
#pragma unroll
  for (int d = 0; d < 3; ++d) load_face_prim(P, ncell, i, d, C);
  // conserved (:170-176); this thread's cell only, so the update is in place
  R U[4];
  U[0] = rho[i] * vol;
  U[1] = rho[i] * vx[i] * vol;
  U[2] = rho[i] * vy[i] * vol;
  U[3] = rho[i] * vz[i] * vol;
  // apply_fluxes (:212-223): per axis, F += -fac * flux(+face); F += fac * flux(-face)
  R up[3][4], dn[3][4];
  const Nbr nb(n, x, y, z);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    Prim<R> Pp, Pm;
    load_face_prim(P, ncell, nb.up[d], d, Pp);
    load_face_prim(P, ncell, nb.dn[d], d, Pm);
    face_flux<R, FACC>(C, Pp, d, dx, cs, up[d]);
    face_flux<R, FACC>(Pm, C, d, dx, cs, dn[d]);
  }
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    R u = U[v];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      u = u + -fac * up[d][v];
      u = u + fac * dn[d][v];
    }
    U[v] = u;
  }
  // get_primitive (:179-185; quantum-fluid-accretion.py:200-206 with eps)
  R r = hdiv(U[0], vol);
  if (clamp_rho) r = fmax((R)0, r);
  rho[i] = r;
  const R den = FACC ? U[0] + (R)1e-30 : U[0];
  vx[i] = hdiv(U[1], den);
  vy[i] = hdiv(U[2], den);
  vz[i] = hdiv(U[3], den);
}

// do_accretion (quantum-gas-bh.py:497-530; quantum-bh.py:306-339 with sigma)
template <typename R>
__global__ void k_accrete(cplx<R> *psi, const R *pos, const R *vel, R *m_bh, int n, R dx, R vol,
                          R sigma_v, R G, R m_per_hbar, R c_light, R dt) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int idx[3];
  for (int d = 0; d < 3; ++d) {
    const R i = floor((pos[d] - (R)0.5 * dx) / dx);
    R m = ref_mod(i, (R)n);
    idx[d] = (m >= (R)0 && m < (R)n) ? (int)m : 0;
  }
  const long long c = ((long long)idx[0] * n + idx[1]) * n + idx[2];
  const cplx<R> p = psi[c];
  const R amp = hypot(p.x, p.y);
  const R theta = atan2(p.y, p.x);
  const R v = sqrt(sigma_v * sigma_v + vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
  const R pi = (R)3.14159265358979323846;
  const R xi = (R)2 * pi * G * m_bh[0] * m_per_hbar / v;
  const R GM = G * m_bh[0];
  const R dM_dt = (R)32 * pi * pi * (GM * GM * GM) * m_per_hbar * amp * amp /
                  (c_light * c_light * c_light * v * ((R)1 - exp(-xi)));
  const R new_amp = fabs(amp) - sqrt(dM_dt * dt / vol);
  psi[c] = cplx<R>{new_amp * cos(theta), new_amp * sin(theta)};
  m_bh[0] = m_bh[0] + dM_dt * dt;
}

// bh_bondi_step_no_vrel (quantum-fluid-accretion-test.py:454-494): Gaussian
// kernel inside r_acc = r_acc_mult dx around the black hole, ambient density,
// isothermal Bondi rate, capped removal.  Only cells with R^2 <= r_acc^2
// contribute to the reference's sums, so one CTA covers the neighbourhood
// (K = ceil(r_acc / dx) + 1 cells each way) with fixed-order reductions.
template <typename R>
__global__ void __launch_bounds__(256)
    k_bondi(R *rho, const R *pos, R *m_bh, int n, R dx, R L, R cs, R G, R dt, R r_acc_mult,
            R lam, R fmax_frac, int K) {
  __shared__ double red[3][256];
  const int w = 2 * K + 1;
  const int tot = w * w * w;
  const R M = m_bh[0];
  const R r_B = G * M / (cs * cs);
  const R r_acc = r_acc_mult * dx;
  const R rK = fmin(fmax(r_B, (R)0.25 * dx), (R)0.5 * r_acc);
  int cidx[3];
  for (int d = 0; d < 3; ++d) cidx[d] = (int)floor(pos[d] / dx);
  double sW = 0, sWr = 0, sM = 0;
  for (int j = threadIdx.x; j < tot; j += blockDim.x) {
    const int o0 = j / (w * w) - K, o1 = (j / w) % w - K, o2 = j % w - K;
    const int ii[3] = {((cidx[0] + o0) % n + n) % n, ((cidx[1] + o1) % n + n) % n,
                       ((cidx[2] + o2) % n + n) % n};
    R R2 = 0;
    for (int d = 0; d < 3; ++d) {
      const R xs = ((R)ii[d] + (R)0.5) * dx;
      const R dd = fabs(xs - pos[d]);
      const R pd = fmin(dd, L - dd);
      R2 = R2 + pd * pd;
    }
    if (R2 <= r_acc * r_acc) {
      const long long c = ((long long)ii[0] * n + ii[1]) * n + ii[2];
      const R W = exp((R)-0.5 * R2 / (rK * rK));
      sW += (double)W;
      sWr += (double)(W * rho[c]);
      sM += (double)rho[c];
    }
  }
  red[0][threadIdx.x] = sW;
  red[1][threadIdx.x] = sWr;
  red[2][threadIdx.x] = sM;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int k = 0; k < 3; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  const double sumW = red[0][0] + 1e-30;
  const double sumWRho = red[1][0] + 1e-30;
  const double rho_inf = red[1][0] / sumW;
  const double GMd = (double)G * (double)M;
  const double dMdt = 4.0 * 3.14159265358979323846 * (double)lam * GMd * GMd * rho_inf /
                      ((double)cs * cs * cs);
  const double dM = dMdt * (double)dt;
  const double M_avail = red[2][0] * (double)dx * dx * dx;
  const double dM_cap = fmin(dM, (double)fmax_frac * M_avail);
  __syncthreads();
  for (int j = threadIdx.x; j < tot; j += blockDim.x) {
    const int o0 = j / (w * w) - K, o1 = (j / w) % w - K, o2 = j % w - K;
    const int ii[3] = {((cidx[0] + o0) % n + n) % n, ((cidx[1] + o1) % n + n) % n,
                       ((cidx[2] + o2) % n + n) % n};
    R R2 = 0;
    for (int d = 0; d < 3; ++d) {
      const R xs = ((R)ii[d] + (R)0.5) * dx;
      const R dd = fabs(xs - pos[d]);
      const R pd = fmin(dd, L - dd);
      R2 = R2 + pd * pd;
    }
    if (R2 <= r_acc * r_acc) {
      const long long c = ((long long)ii[0] * n + ii[1]) * n + ii[2];
      const R W = exp((R)-0.5 * R2 / (rK * rK));
      const double phi = (double)(W * rho[c]) / sumWRho;
      rho[c] = (R)fmax(0.0, (double)rho[c] - dM_cap / ((double)dx * dx * dx) * phi);
    }
  }
  if (threadIdx.x == 0) m_bh[0] = (R)((double)M + dM_cap);
}

// Fixed-grid sink with the ambient density sampled in a shell outside r_acc
// (bh_bondi_step_ambient, quantum-fluid-accretion.py:440-510), one CTA over
// the (2K+1)^3 cells around the black hole; float64 sums in a fixed order.
// out[7] = dMdt_target, rho_inf, rB, dM_cap, r_acc, M_avail, dM_uncl.
template <typename R>
__global__ void __launch_bounds__(256)
    k_bondi_ambient(R *rho, const R *vx, const R *vy, const R *vz, int n, double dx, double L,
                    double x0, double x1, double x2, double vb0, double vb1, double vb2,
                    double M, double cs, double G, double dt, double r_acc_mult, double lam,
                    double cap_frac, double ann_lo, double ann_hi, int K, double *out) {
  __shared__ double red[8][256];
  const double xb[3] = {x0, x1, x2};
  const double rB = G * M / (cs * cs + 1e-30);
  const double r_acc = r_acc_mult * dx;
  const double rK = fmin(0.5 * r_acc, fmax(0.5 * dx, rB));
  const double r_lo = fmax(ann_lo * r_acc, r_acc + 0.25 * dx);
  const double r_hi = fmax(ann_hi * r_acc, r_lo + 0.5 * dx);
  const bool bhl = vx != nullptr;
  const int w = 2 * K + 1, tot = w * w * w;
  int cidx[3];
  for (int d = 0; d < 3; ++d) cidx[d] = (int)floor(xb[d] / dx);
  // this thread's cells: index, distance R and kernel weight W (sink) / shell flag
  auto cell = [&](int j, long long &c, double &Rd) {
    const int o[3] = {j / (w * w) - K, (j / w) % w - K, j % w - K};
    int ii[3];
    double R2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      ii[d] = ((cidx[d] + o[d]) % n + n) % n;
      const double xs = ((double)ii[d] + 0.5) * dx;
      const double dd = fabs(xs - xb[d]);
      const double pd = fmin(dd, L - dd);
      R2 += pd * pd;
    }
    Rd = sqrt(R2);
    c = ((long long)ii[0] * n + ii[1]) * n + ii[2];
  };
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // sumWRho, M_sink, n_shell, rho_shell, v_shell[3]
  for (int j = threadIdx.x; j < tot; j += blockDim.x) {
    long long c;
    double Rd;
    cell(j, c, Rd);
    const double r = (double)rho[c];
    if (Rd <= r_acc) {
      const double q = Rd / (rK + 1e-30);
      acc[0] += exp(-0.5 * q * q) * r;
      acc[1] += r;
    }
    if (Rd >= r_lo && Rd <= r_hi) {
      acc[2] += 1.0;
      acc[3] += r;
      if (bhl) {
        acc[4] += (double)vx[c];
        acc[5] += (double)vy[c];
        acc[6] += (double)vz[c];
      }
    }
  }
  for (int k = 0; k < 8; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int k = 0; k < 8; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + st];
    __syncthreads();
  }
  const double n_sh = red[2][0] + 1e-30;
  const double rho_inf = red[3][0] / n_sh;
  double denom = cs * cs * cs;
  if (bhl) {
    const double v_inf[3] = {red[4][0] / n_sh, red[5][0] / n_sh, red[6][0] / n_sh};
    const double vb[3] = {vb0, vb1, vb2};
    double v_rel2 = 0.0;
    for (int d = 0; d < 3; ++d) v_rel2 += (vb[d] - v_inf[d]) * (vb[d] - v_inf[d]);
    denom = pow(cs * cs + v_rel2, 1.5);
  }
  const double GM = G * M;
  const double dMdt = 4.0 * 3.14159265358979323846 * lam * GM * GM * rho_inf / (denom + 1e-30);
  const double dM_uncl = dMdt * dt;
  const double sumWRho = red[0][0] + 1e-30;
  const double vol = dx * dx * dx;
  const double M_avail = red[1][0] * vol;
  const double dM_cap = cap_frac > 0.0 ? fmin(dM_uncl, cap_frac * M_avail) : fmin(dM_uncl, M_avail);
  __syncthreads();
  for (int j = threadIdx.x; j < tot; j += blockDim.x) {
    long long c;
    double Rd;
    cell(j, c, Rd);
    if (Rd <= r_acc) {
      const double q = Rd / (rK + 1e-30);
      const double phi = exp(-0.5 * q * q) * (double)rho[c] / sumWRho;
      rho[c] = (R)fmax(0.0, (double)rho[c] - (dM_cap / vol) * phi);
    }
  }
  if (threadIdx.x == 0) {
    out[0] = dMdt;
    out[1] = rho_inf;
    out[2] = rB;
    out[3] = dM_cap;
    out[4] = r_acc;
    out[5] = M_avail;
    out[6] = dM_uncl;
  }
}

// max over cells of c + |v| (c constant), per-block partial maxima
template <typename R>
__global__ void k_cfl_partial(const R *vx, const R *vy, const R *vz, long long ncell, double c,
                              double *part) {
  __shared__ double red[256];
  double m = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ncell;
       i += (long long)gridDim.x * blockDim.x) {
    const double a = vx[i], b = vy[i], d = vz[i];
    m = fmax(m, c + sqrt(a * a + b * b + d * d));
  }
  red[threadIdx.x] = m;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + st]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}
__global__ void k_cfl_final(const double *part, int nb, double dx, double cfl, double dt,
                            double *dt_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double m = 0.0;
  for (int b = 0; b < nb; ++b) m = fmax(m, part[b]);
  *dt_out = fmin(dt, cfl * dx / (m + 1e-30));
}

}  // namespace

int launch_bondi_ambient(bool dbl, void *rho, const void *vx, const void *vy, const void *vz,
                         int n, double dx, double L, const double x_bh[3], const double v_bh[3],
                         double M, double cs, double G, double dt, double r_acc_mult, double lam,
                         double fmax, double ann_lo, double ann_hi, double *out, cudaStream_t st) {
  const double r_acc = r_acc_mult * dx;
  const double r_lo = std::max(ann_lo * r_acc, r_acc + 0.25 * dx);
  const double r_hi = std::max(ann_hi * r_acc, r_lo + 0.5 * dx);
  const int K = (int)std::ceil(r_hi / dx) + 1;
  if (2 * K + 1 > n) {
    set_error("ambient Bondi sink: sampling shell radius %g cells is too large for a %d^3 grid",
              r_hi / dx, n);
    return QJ_ERR_ARG;
  }
  if (dbl)
    k_bondi_ambient<double><<<1, 256, 0, st>>>(
        (double *)rho, (const double *)vx, (const double *)vy, (const double *)vz, n, dx, L,
        x_bh[0], x_bh[1], x_bh[2], v_bh[0], v_bh[1], v_bh[2], M, cs, G, dt, r_acc_mult, lam, fmax,
        ann_lo, ann_hi, K, out);
  else
    k_bondi_ambient<float><<<1, 256, 0, st>>>(
        (float *)rho, (const float *)vx, (const float *)vy, (const float *)vz, n, dx, L, x_bh[0],
        x_bh[1], x_bh[2], v_bh[0], v_bh[1], v_bh[2], M, cs, G, dt, r_acc_mult, lam, fmax, ann_lo,
        ann_hi, K, out);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_cfl_dt(bool dbl, const void *vx, const void *vy, const void *vz, long long ncell,
                  double cs, double dx, double cfl, double dt, double *part, int nb, double *dt_out,
                  cudaStream_t st) {
  if (dbl)
    k_cfl_partial<double><<<nb, 256, 0, st>>>((const double *)vx, (const double *)vy,
                                              (const double *)vz, ncell, cs, part);
  else
    k_cfl_partial<float><<<nb, 256, 0, st>>>((const float *)vx, (const float *)vy,
                                             (const float *)vz, ncell, cs, part);
  QJ_CK_LAUNCH();
  k_cfl_final<<<1, 32, 0, st>>>(part, nb, dx, cfl, dt, dt_out);
  QJ_CK_LAUNCH();
  return 0;
}

template <bool FACC>
static int hydro_impl(bool dbl, void *rho, void *vx, void *vy, void *vz, void *prim, int n,
                      double dx, double dt, double cs, int clamp_rho, cudaStream_t st, int block) {
  const long long ncell = (long long)n * n * n;
  if (ncell >= (1LL << 32)) {
    set_error("hydro: %d^3 cells exceed 2^32", n);
    return QJ_ERR_ARG;
  }
  const int T = (block == 64 || block == 128 || block == 256) ? block : 256;
  const int B = (int)((ncell + T - 1) / T);
  const double vol = dx * dx * dx, fac = dt * dx * dx;
  if (dbl) {
    k_hydro_prim<double, FACC><<<B, T, 0, st>>>((const double *)rho, (const double *)vx,
                                                (const double *)vy, (const double *)vz,
                                                (double *)prim, n, dx, dt, cs);
    QJ_CK_LAUNCH();
    k_hydro_update<double, FACC><<<B, T, 0, st>>>((double *)rho, (double *)vx, (double *)vy,
                                                  (double *)vz, (const double *)prim, n, dx, cs,
                                                  vol, fac, clamp_rho);
  } else {
    k_hydro_prim<float, FACC><<<B, T, 0, st>>>((const float *)rho, (const float *)vx,
                                               (const float *)vy, (const float *)vz,
                                               (float *)prim, n, (float)dx, (float)dt, (float)cs);
    QJ_CK_LAUNCH();
    k_hydro_update<float, FACC><<<B, T, 0, st>>>((float *)rho, (float *)vx, (float *)vy,
                                                 (float *)vz, (const float *)prim, n, (float)dx,
                                                 (float)cs, (float)vol, (float)fac, clamp_rho);
  }
  QJ_CK_LAUNCH();
  return 0;
}

int launch_hydro(bool dbl, void *rho, void *vx, void *vy, void *vz, void *prim, int n, double dx,
                 double dt, double cs, int clamp_rho, cudaStream_t st, int block, bool facc) {
  return facc ? hydro_impl<true>(dbl, rho, vx, vy, vz, prim, n, dx, dt, cs, clamp_rho, st, block)
              : hydro_impl<false>(dbl, rho, vx, vy, vz, prim, n, dx, dt, cs, clamp_rho, st, block);
}

int launch_accrete(bool dbl, void *psi, const void *pos, const void *vel, void *m_bh, int n,
                   double dx, double sigma_v, double G, double m_per_hbar, double c_light,
                   double dt, cudaStream_t st) {
  const double vol = dx * dx * dx;
  if (dbl)
    k_accrete<double><<<1, 32, 0, st>>>((double2 *)psi, (const double *)pos, (const double *)vel,
                                        (double *)m_bh, n, dx, vol, sigma_v, G, m_per_hbar,
                                        c_light, dt);
  else
    k_accrete<float><<<1, 32, 0, st>>>((float2 *)psi, (const float *)pos, (const float *)vel,
                                       (float *)m_bh, n, (float)dx, (float)vol, (float)sigma_v,
                                       (float)G, (float)m_per_hbar, (float)c_light, (float)dt);
  QJ_CK_LAUNCH();
  return 0;
}

int launch_bondi(bool dbl, void *rho, const void *pos, void *m_bh, int n, double dx, double L,
                 double cs, double G, double dt, double r_acc_mult, cudaStream_t st) {
  const int K = (int)std::ceil(r_acc_mult) + 1;
  if (2 * K + 1 > n) {
    set_error("Bondi sink: accretion radius %g cells is too large for a %d^3 grid", r_acc_mult, n);
    return QJ_ERR_ARG;
  }
  const double lam = std::exp(1.5) / 4.0, fmaxf_ = 0.25;
  if (dbl)
    k_bondi<double><<<1, 256, 0, st>>>((double *)rho, (const double *)pos, (double *)m_bh, n, dx, L,
                                       cs, G, dt, r_acc_mult, lam, fmaxf_, K);
  else
    k_bondi<float><<<1, 256, 0, st>>>((float *)rho, (const float *)pos, (float *)m_bh, n, (float)dx,
                                      (float)L, (float)cs, (float)G, (float)dt,
                                      (float)r_acc_mult, (float)lam, (float)fmaxf_, K);
  QJ_CK_LAUNCH();
  return 0;
}

}  // namespace qj
