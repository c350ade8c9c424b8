// Host-side declarations shared by the libqj translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <vector>

#include "../../include/qj.h"
#include "qj_pass.cuh"

namespace qj {

// Set-up that belongs to one device's context (a kernel's shared-memory
// attribute, occupancy, the SM count), done once per device ordinal: the
// first call with device d current runs init(value of d); later calls on d
// reuse it.  A process that drives several GPUs gets each one's own set-up.
constexpr int kMaxDevices = 64;
template <class T> struct PerDevice {
  std::once_flag once[kMaxDevices];
  T val[kMaxDevices];
};
template <class T, class F>
cudaError_t per_device(PerDevice<T> &pd, const T *&out, F &&init) {
  int dev = 0;
  const cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::call_once(pd.once[dev], [&] { init(pd.val[dev]); });
  out = &pd.val[dev];
  return cudaSuccess;
}

// ----- error state (qj_api.cu) -----
void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define QJ_CK(call)                                                      \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) return ::qj::cuda_fail(e_, #call, __FILE__, __LINE__); \
  } while (0)
// Every kernel launch in libqj is followed by QJ_CK_LAUNCH(), which also
// counts it (qj_launch_count).
extern std::atomic<long long> g_launches;
#define QJ_CK_LAUNCH()                      \
  do {                                      \
    ::qj::g_launches.fetch_add(1, std::memory_order_relaxed); \
    QJ_CK(cudaGetLastError());              \
  } while (0)

// Optional per-pass timing with CUDA events on the launching stream
// (qj_profile_enable / qj_profile_read).  Bucket = pass mode (0..6), 7 = the
// deposit sort, 8 = other particle kernels.
constexpr int kProfBuckets = 9;
bool prof_on();
void prof_mark_begin(cudaStream_t st);
void prof_mark_end(int bucket, cudaStream_t st);
// The autotuner's pass timing: while set, a fused pass along z counts in
// bucket kProfZ + mode instead of mode.
constexpr int kProfZ = 16;
bool prof_split();

bool fft_length_supported(int n);
// Stage twiddle table of the fused passes for length n and radix plan rv
// (host, float2; rv = 1 only for has_radix_variant(n)).
std::vector<float2> stage_twiddles(int n, int rv = 0);

// Launch-shape variant (PassShape's V) of a plan's pass of `mode` along an
// axis of length n, contiguous (z) or strided (x, y): bit b of
// tune[QJ_TUNE_RADIX] gives V's bit 0 (radix plan 1), bit b of
// tune[QJ_TUNE_TILE] its bit 1 (half tile), b = mode for a strided pass and
// 8 + mode for a contiguous one.  The first density build takes the drift +
// density pass's bits of its orientation, so that both write the same number
// of partial sums; the deposit and lengths without variants always take 0.
inline int shape_of(int n, const int *tune, int mode, bool contig) {
  if (!tune || !has_radix_variant(n) || mode == M_DEPOSIT) return 0;
  const int b = (mode == M_DENSITY ? M_DRIFT_DENSITY : mode) + (contig ? 8 : 0);
  return ((tune[QJ_TUNE_RADIX] >> b) & 1) | (((tune[QJ_TUNE_TILE] >> b) & 1) << 1);
}
// z columns of a strided tile in shape variant v (16, or 8 for bit 1).
int strided_tile_width(int v);

// ----- pencil passes (qj_fused.cu, qj_fftpass.cu) -----
// Launch one fused single-precision pass of `mode` along `a.axis` (length n).
int launch_selftest_wait(unsigned *err, long long limit_ns, cudaStream_t st);
// out[i] = (sin, cos) of theta[i] by the kick pass's own sincos_reduced.
int launch_selftest_sincos(const double *theta, float2 *out, int n, cudaStream_t st);
int launch_fused(int mode, int n, const FusedArgs &a, cudaStream_t st);
// Number of tiles of a pass along `axis` in shape variant v (= the partial
// sums a density pass writes).
int pass_blocks(int n_axis, int axis, int nx, int ny, int nz, int v = 0);
// Ensemble launch of pass `mode` for np <= kEnsClasses plans of distinct
// sizes n[i] in {64, 96, 128} (their axis lengths along a[i].axis, the same
// axis for all, shape variant 0): one persistent launch whose CTAs claim the
// tiles of every plan's boxes; `reserve` CTA slots stay free.  ctr holds
// nctr >= (boxes of all plans) tile counters, zeroed before the launch and
// used by it alone.  Bit-identical to one launch_fused per plan.
constexpr int kEnsClasses = 3;
int ens_slot(int n);  // the size class of length n, -1 if none
int launch_fused_ens(int mode, int np, const FusedArgs *a, const int *n, int reserve,
                     unsigned *ctr, int nctr, cudaStream_t st);
// Generic in-place FFT pass over a complex field (float2 if dbl == 0, else
// double2) along a.axis.
int launch_fft(bool dbl, int n, int dir, const FftArgs &a, cudaStream_t st);

// ----- particles (qj_particles.cu) -----
struct CicGeomD {
  int n[3];
  double d[3];
  double L[3];
  double vol;
};
unsigned cell_bits(long long ncell);
// keys / vals of the 8 CIC corner deposits of n particles, in orientation q.
int launch_cic_prepare(bool dbl, const void *pos, int n, const void *masses, double m_s,
                       const CicGeomD &g, int q, unsigned *keys, void *vals, cudaStream_t st);
// Stable sort of (key, index) + per-cell ordered sums.  Outputs ukey[u],
// uval[u], cell_u[original index] = u, *n_unique.  dts_reset (optional) is
// set to +inf bits.
int launch_sort_unique(bool dbl, const unsigned *keys, const void *vals, int n, unsigned nbits,
                       unsigned *kA, unsigned *iA, unsigned *kB, unsigned *iB, unsigned *ukey,
                       void *uval, unsigned *cell_u, int *n_unique, void *dts_reset,
                       cudaStream_t st);
int launch_pencil_starts(const unsigned *ukey, const int *n_unique, int n_pencils, unsigned nq,
                         int *start, cudaStream_t st);
int launch_scatter_unique(bool dbl, const unsigned *ukey, const void *uval, const int *n_unique,
                          int max_unique, void *grid, cudaStream_t st);
// acc[s] = sum_c w_c A[cell_u[8 s + c]] (deposit-cell accelerations).
int launch_gather_unique(bool dbl, const void *pos, int n, const CicGeomD &g, const void *A,
                         const unsigned *cell_u, void *acc, cudaStream_t st);
// acc[s] = sum_c w_c (ax, ay, az)[cell_c] from dense grids.
int launch_gather_dense(bool dbl, const void *pos, int n, const CicGeomD &g, const void *ax,
                        const void *ay, const void *az, void *acc, cudaStream_t st);
// Leapfrog update: optional second half kick (K2, end of a step; updates
// dt_s), optional first half kick (K1), optional drift + CIC keys of the new
// positions in orientation q_next.
struct UpdateArgs {
  int n;
  double dt;
  int k2, k1, drift;
  void *dts_bits;  // unsigned (float) / unsigned long long (double)
  int q_next;
  unsigned *keys;
  void *vals;
  const void *masses;
  double m_s;
  int box_stars;  // stars per box of a batched plan (0 = n)
};
int launch_particles_update(bool dbl, void *pos, void *vel, const void *acc, const CicGeomD &g,
                            const UpdateArgs &u, cudaStream_t st);

// ----- pencil-bucket star data of the fused path -----
struct StarBufs {
  int4 *sidx;        // [n] lower CIC corner (wrapped)
  float4 *sw0;       // [n] (w_i x, y, z, m / vol)
  float4 *sw1;       // [n] (w_ip1 x, y, z, 0)
  unsigned *bkey;    // [n] bucket = pencil of the lower corner (pass orientation)
  unsigned *perm;    // [n] stars sorted by (bucket, star)
  unsigned *skey;    // [n] sorted bucket keys
  int *bstart;       // [n_buckets + 1]
  // pencil mask, [ceil(n_buckets / 32)] words per box at stride mstride: bit
  // p is set when some star's corners lie on pencil p; the kick skips the
  // star lookups of the other pencils
  unsigned *pmask;
  int mstride;
  unsigned *sortbuf; // [4 n] global sort scratch (large n)
  float *A;          // [8 n][3] accelerations at the 8 corners of each star
};
int launch_stars_prepare(const void *pos, int n, const void *masses, double m_s,
                         const CicGeomD &g, int q, const StarBufs &b, cudaStream_t st);
// n stars per box, nbox boxes (one sort CTA each): permutation, sorted keys,
// pencil mask, and bucket starts per box at stride bstride; buckets form
// rows of nv (the extent of the faster cross axis of the orientation).
int launch_bucket_sort(int n, int n_buckets, int nv, const StarBufs &b, cudaStream_t st,
                       int nbox = 1, int bstride = 0);
// n <= 32 particles, one box: launch_stars_prepare + launch_bucket_sort in one launch
int launch_stars_small(const void *pos, int n, const void *masses, double m_s, const CicGeomD &g,
                       int q, int n_buckets, const StarBufs &b, cudaStream_t st);
int launch_update_fused(void *pos, void *vel, const CicGeomD &g, const UpdateArgs &u,
                        const StarBufs &b, cudaStream_t st);

// ----- plain elementwise kernels (qj_plain.cu), R = float or double -----
struct KTabs {
  const void *k[3];  // per-axis k tables of the real type
  int n[3];
};
int launch_build_rho(bool dbl, const void *psi, const void *rho_s, const void *rho_gas,
                     const void *rho_in, double fourpiG, double rho_bar, void *rho_tot,
                     void *cbuf, long long ncell, cudaStream_t st);
int launch_poisson_div(bool dbl, void *cbuf, const KTabs &k, long long ncell, cudaStream_t st);
int launch_mul_ik(bool dbl, const void *vh, int d, const KTabs &k, void *out, long long ncell,
                  cudaStream_t st);
int launch_real_part(bool dbl, const void *c, double sign, const void *rho, double b,
                     const void *vext, void *out, long long ncell, cudaStream_t st);
int launch_kick_plain(bool dbl, void *psi, const void *V, double coef, long long ncell,
                      cudaStream_t st);
int launch_drift_mul(bool dbl, void *cbuf, const KTabs &k, double dt_kin, double m_per_hbar,
                     long long ncell, cudaStream_t st);
int launch_amax3(bool dbl, const void *ax, const void *ay, const void *az, long long ncell,
                 void *bits, cudaStream_t st);
int launch_gas_kick(bool dbl, void *vx, void *vy, void *vz, const void *ax, const void *ay,
                    const void *az, double dt, long long ncell, cudaStream_t st);

// quantum-fluid-accretion pieces (qj_plain.cu)
int launch_kfilter(bool dbl, void *c, const KTabs &k, int kind, double p, long long ncell,
                   cudaStream_t st);
int launch_cic_point(bool dbl, void *grid, int n, const double x[3], double dx, double M,
                     cudaStream_t st);
int launch_cic_sample3(bool dbl, const void *f0, const void *f1, const void *f2, int n,
                       const double x[3], double dx, double *out, cudaStream_t st);
int launch_mean_dm_gas(bool dbl, const void *psi, const void *rho, long long ncell, double *part,
                       int nb, double *out, cudaStream_t st);
int launch_argmax(bool dbl, const void *f, long long ncell, double *pv, long long *pi, int nb,
                  double *out, cudaStream_t st);

// adjoint kick: mu = coef Im(conj(g) psi') (stored when mu is non-null) and the
// Poisson source fourpiG mu in cbuf; then g <- exp(+i coef V) g + 2 W psi with
// W = Re(cbuf) (+ b mu when mu is non-null)
int launch_adj_mu(bool dbl, const void *g, const void *psi, const void *V, double coef, void *mu,
                  double fourpiG, void *cbuf, long long ncell, cudaStream_t st);
int launch_adj_update(bool dbl, void *g, const void *psi, const void *V, const void *cbuf,
                      const void *mu, double b, double coef, long long ncell, cudaStream_t st);

// ----- gas and black hole (qj_gas.cu) -----
// CTAs of a fused pass in shape variant `shape` that fit one SM (occupancy),
// 0 if unknown.
int fused_max_ctas_per_sm(int mode, int n, bool contig, int shape = 0);

int launch_hydro(bool dbl, void *rho, void *vx, void *vy, void *vz, void *prim, int n, double dx,
                 double dt, double cs, int clamp_rho, cudaStream_t st, int block = 256,
                 bool facc = false);
int launch_bondi_ambient(bool dbl, void *rho, const void *vx, const void *vy, const void *vz,
                         int n, double dx, double L, const double x_bh[3], const double v_bh[3],
                         double M, double cs, double G, double dt, double r_acc_mult, double lam,
                         double fmax, double ann_lo, double ann_hi, double *out, cudaStream_t st);
int launch_cfl_dt(bool dbl, const void *vx, const void *vy, const void *vz, long long ncell,
                  double cs, double dx, double cfl, double dt, double *part, int nb, double *dt_out,
                  cudaStream_t st);
int launch_accrete(bool dbl, void *psi, const void *pos, const void *vel, void *m_bh, int n,
                   double dx, double sigma_v, double G, double m_per_hbar, double c_light,
                   double dt, cudaStream_t st);
int launch_bondi(bool dbl, void *rho, const void *pos, void *m_bh, int n, double dx, double L,
                 double cs, double G, double dt, double r_acc_mult, cudaStream_t st);

// ----- small scalar kernels (qj_particles.cu) -----
// diag: nbox records (t, a_max, dt_s); amax / dts: nbox scalars
int launch_diag_load(bool dbl, const void *diag, void *amax_bits, cudaStream_t st, int nbox = 1);
int launch_diag_store(bool dbl, void *diag, const void *amax_bits, const void *dts_bits,
                      int has_particles, double t_add, cudaStream_t st, int nbox = 1);
int launch_set_scalar(bool dbl, void *dst, double v, cudaStream_t st, int count = 1);
int launch_bits_to_double(bool dbl, const void *bits, double *out, cudaStream_t st);

}  // namespace qj
