// libqj C ABI: plans, the kick-drift-kick step (fused float32 and plain
// float64 forms) and the standalone operators.  See include/qj.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/qj.h"
#include "qj_internal.h"

namespace qj {

static thread_local std::string g_err;

void set_error(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}

std::atomic<long long> g_launches{0};

// ----- per-pass event timing -----
namespace {
struct Prof {
  std::mutex mu;
  bool on = false;
  bool split = false;  // the autotuner's pass timing (prof_split)
  std::vector<cudaEvent_t> pool;
  struct Mark {
    int bucket;
    cudaEvent_t a, b;
  };
  std::vector<Mark> marks;
  cudaEvent_t pending = nullptr;
  cudaEvent_t get() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
};
Prof &prof() {
  static Prof p;
  return p;
}
}  // namespace

bool prof_on() { return prof().on; }
bool prof_split() { return prof().split; }
void prof_mark_begin(cudaStream_t st) {
  Prof &p = prof();
  std::lock_guard<std::mutex> g(p.mu);
  p.pending = p.get();
  cudaEventRecord(p.pending, st);
}
void prof_mark_end(int bucket, cudaStream_t st) {
  Prof &p = prof();
  std::lock_guard<std::mutex> g(p.mu);
  cudaEvent_t b = p.get();
  cudaEventRecord(b, st);
  p.marks.push_back({bucket, p.pending, b});
  p.pending = nullptr;
}

namespace {
// The autotuner's pass timing: clears the marks and turns the split timing
// on (on = true) or everything off.
void prof_session(bool on) {
  Prof &p = prof();
  std::lock_guard<std::mutex> g(p.mu);
  for (auto &m : p.marks) {
    p.pool.push_back(m.a);
    p.pool.push_back(m.b);
  }
  p.marks.clear();
  p.on = on;
  p.split = on;
}
// Mean duration of bucket b's marks (their work complete); +inf without any.
int prof_bucket_mean(int b, float &ms) {
  Prof &p = prof();
  std::lock_guard<std::mutex> g(p.mu);
  double sum = 0.0;
  int n = 0;
  for (auto &m : p.marks) {
    if (m.bucket != b) continue;
    float t = 0.f;
    const cudaError_t e = cudaEventElapsedTime(&t, m.a, m.b);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventElapsedTime", __FILE__, __LINE__);
    sum += t;
    ++n;
  }
  ms = n ? (float)(sum / n) : INFINITY;
  return 0;
}
}  // namespace

int cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
  set_error("CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file, line);
  return e == cudaErrorMemoryAllocation ? QJ_ERR_ALLOC : QJ_ERR_CUDA;
}

// Drift propagator of each axis minus one, float64 phase, rounded once:
// prop_a[i] = exp(-1j * dt_kin * k_a[i]^2 / (2 m_per_hbar)) - 1
// (the separable factor of quantum-stars.py:308).
__global__ void k_prop_tables(float2 *p0, float2 *p1, float2 *p2, const double *k0,
                              const double *k1, const double *k2, int n0, int n1, int n2,
                              double dtk, double mph) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float2 *P[3] = {p0, p1, p2};
  const double *K[3] = {k0, k1, k2};
  const int N[3] = {n0, n1, n2};
  for (int a = 0; a < 3; ++a) {
    if (i < N[a]) {
      // stored as d = exp(i th) - 1 = (-2 sin^2(th/2), sin th): the pass adds
      // IFFT(d FFT(psi)) to psi, so small phases keep full relative precision
      // (the 1/n of ifftn is applied after the transform)
      const double th = -dtk * K[a][i] * K[a][i] / (2.0 * mph);
      const double sh = sin(0.5 * th);
      P[a][i] = float2{(float)(-2.0 * sh * sh), (float)sin(th)};
    }
  }
}

}  // namespace qj

using namespace qj;

struct qj_plan {
  qj_grid g;
  qj_phys ph;
  int prec;
  bool dbl;
  int max_particles;
  int nbox = 1;  // boxes of a batched plan (fused single precision only)
  int part_stride = 0, bstart_stride = 0;
  int cur_stars = 0;  // stars per box of the running step
  int n[3];
  long long ncell;
  size_t rsz, csz;  // bytes of one real / complex element
  std::vector<void *> allocs;
  int64_t ws_bytes = 0;
  // tables
  void *tw[3] = {nullptr, nullptr, nullptr};  // float2 / double2
  float2 *tws[3] = {nullptr, nullptr, nullptr};  // stage twiddle tables (fused passes)
  float2 *tws_alt[3] = {nullptr, nullptr, nullptr};  // the same for radix plan 1 (n = 128, 256)
  double *kd[3] = {nullptr, nullptr, nullptr};
  float *kf[3] = {nullptr, nullptr, nullptr};
  float *ktf[3] = {nullptr, nullptr, nullptr};
  void *kr[3] = {nullptr, nullptr, nullptr};  // k tables of the real type
  float2 *prop[3] = {nullptr, nullptr, nullptr};
  double prop_dtk = NAN;
  // fused workspace
  float2 *R = nullptr, *S1 = nullptr, *S2 = nullptr;
  double *part = nullptr;
  // plain / standalone workspace (lazy for fused plans)
  void *c0 = nullptr, *c1 = nullptr;
  void *rho_tot = nullptr, *V = nullptr, *ax = nullptr, *ay = nullptr, *az = nullptr,
       *rho_s = nullptr;
  // particles
  unsigned *keys = nullptr, *kA = nullptr, *iA = nullptr, *kB = nullptr, *iB = nullptr,
           *ukey = nullptr, *cell_u = nullptr;
  void *vals = nullptr, *uval = nullptr, *A = nullptr, *acc = nullptr;
  int *pstart = nullptr;
  int *n_unique = nullptr;
  StarBufs sb{};  // fused path star data
  // side stream for the star pipeline (overlaps the y drift pass)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_kick = nullptr, ev_parts = nullptr;
  void *amax = nullptr, *dts = nullptr;  // real type scalars
  unsigned *err = nullptr;  // set by a fused pass whose bounded tile wait gave up
  double *phi = nullptr;    // fused: per-box phase of the uniform potential (float64)
  double *cfl_part = nullptr;  // per-block maxima of the CFL reduction
  // fluid-accretion step: softened black-hole density, small scalars, partials
  void *facc_bh = nullptr;
  double *facc_scal = nullptr, *facc_part = nullptr;
  long long *facc_pi = nullptr;
  int tune[QJ_TUNE_N] = {0, 0, 0, 0, 0, 0, 0, 0, -1, 0, 0, 0};  // launch tuning (include/qj.h)
  void *tmp_scalar = nullptr;
  void *tmp_diag = nullptr;
  void *gas_prim = nullptr;  // hydro: 16 values per cell as 4 quads (predicted primitives, gradients by axis)
  // adjoint: recomputed chunk states
  void *adj_psi = nullptr, *adj_states = nullptr, *adj_V = nullptr;
  int adj_cap = 0;
};

namespace {

int dev_alloc(qj_plan *P, void **p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
  }
  P->allocs.push_back(*p);
  P->ws_bytes += (int64_t)bytes;
  return 0;
}

template <typename T> int dev_alloc_t(qj_plan *P, T **p, size_t count) {
  return dev_alloc(P, (void **)p, count * sizeof(T));
}

#define QJ_TRY(x)             \
  do {                        \
    int rc_ = (x);            \
    if (rc_) return rc_;      \
  } while (0)

CicGeomD geom(const qj_plan *P) {
  CicGeomD g;
  g.n[0] = P->g.nx;
  g.n[1] = P->g.ny;
  g.n[2] = P->g.nz;
  g.d[0] = P->g.Lx / P->g.nx;
  g.d[1] = P->g.Ly / P->g.ny;
  g.d[2] = P->g.Lz / P->g.nz;
  g.L[0] = P->g.Lx;
  g.L[1] = P->g.Ly;
  g.L[2] = P->g.Lz;
  g.vol = g.d[0] * g.d[1] * g.d[2];
  return g;
}

KTabs ktabs(const qj_plan *P) {
  KTabs k;
  for (int a = 0; a < 3; ++a) {
    k.k[a] = P->kr[a];
    k.n[a] = P->n[a];
  }
  return k;
}

int ensure_plain_ws(qj_plan *P) {
  if (P->c0) return 0;
  QJ_TRY(dev_alloc(P, &P->c0, P->ncell * P->csz));
  QJ_TRY(dev_alloc(P, &P->c1, P->ncell * P->csz));
  for (void **f : {&P->rho_tot, &P->V, &P->ax, &P->ay, &P->az, &P->rho_s})
    QJ_TRY(dev_alloc(P, f, P->ncell * P->rsz));
  return 0;
}

FftArgs fft_args(const qj_plan *P, int axis, void *data, double scale) {
  FftArgs a;
  a.nx = P->n[0];
  a.ny = P->n[1];
  a.nz = P->n[2];
  a.axis = axis;
  a.stride = axis == 0 ? (long long)P->n[1] * P->n[2] : (axis == 1 ? P->n[2] : 1);
  a.outer_stride = axis == 0 ? P->n[2] : (long long)P->n[1] * P->n[2];
  a.ztiles = P->n[2] / 16;
  a.data = data;
  a.tw = P->tw[axis];
  a.scale = scale;
  return a;
}

// jnp.fft.fftn (dir -1) / ifftn (dir +1) in place, axes z, y, x.
int fft3d(qj_plan *P, void *data, int dir, cudaStream_t st) {
  for (int axis = 2; axis >= 0; --axis) {
    const double scale = dir > 0 ? 1.0 / P->n[axis] : 1.0;
    QJ_TRY(launch_fft(P->dbl, P->n[axis], dir, fft_args(P, axis, data, scale), st));
  }
  return 0;
}

// Arguments of a pass of `mode` along `axis`, in the plan's shape variant of
// that pass (qj.h QJ_TUNE_RADIX / QJ_TUNE_TILE).
FusedArgs fused_args(const qj_plan *P, int axis, int mode) {
  FusedArgs a;
  std::memset(&a, 0, sizeof(a));
  a.nx = P->n[0];
  a.ny = P->n[1];
  a.nz = P->n[2];
  a.axis = axis;
  a.stride = axis == 0 ? (long long)P->n[1] * P->n[2] : (axis == 1 ? P->n[2] : 1);
  a.outer_stride = axis == 0 ? P->n[2] : (long long)P->n[1] * P->n[2];
  a.shape = shape_of(P->n[axis], P->tune, mode, axis == 2);
  a.ztiles = P->n[2] / strided_tile_width(a.shape);
  a.full_nx = P->n[0];
  a.R = P->R;
  a.S1 = P->S1;
  a.S2 = P->S2;
  a.tw = (a.shape & 1) ? P->tws_alt[axis] : P->tws[axis];
  a.prop = P->prop[axis];
  for (int d = 0; d < 3; ++d) {
    a.k[d] = P->kf[d];
    a.kt[d] = P->ktf[d];
  }
  a.part = P->part;
  a.fourpiG = 4.0 * M_PI * P->ph.G;
  a.rho_bar = P->ph.rho_bar;
  a.inv_ncell = 1.0 / (double)P->ncell;
  a.amax_bits = (unsigned *)P->amax;
  a.err = P->err;
  a.tune = P->tune;
  a.nbox = P->nbox;
  a.box_cells = P->ncell;
  a.box_stars = P->cur_stars;
  a.box_bstart = P->bstart_stride;
  a.box_part = P->part_stride;
  return a;
}

void set_stars(FusedArgs &a, const qj_plan *P) {
  a.has_stars = 1;
  a.sidx = P->sb.sidx;
  a.sw0 = P->sb.sw0;
  a.sw1 = P->sb.sw1;
  a.perm = P->sb.perm;
  a.bstart = P->sb.bstart;
  a.pmask = P->sb.pmask;
  a.A = P->sb.A;
}

// The forward y and Poisson passes over half of the density's spectrum along
// axis q (0 or 2), the axis its first forward transform ran along: the density
// is real, so k_q > n_q / 2 follows from k_q < n_q / 2 (the Poisson pass writes
// those as mirrors).  x: the first n/2 + 1 planes; z: the 16-wide tiles that
// hold k_z <= n/2 (16 or, in the narrow tile variant, 8 wide).
void half_spectrum(FusedArgs &a, const qj_plan *P, int q) {
  a.hq = q;
  if (q == 0) {
    a.nx = P->n[0] / 2 + 1;
  } else {
    const int w = strided_tile_width(a.shape);
    a.ztiles = (P->n[2] / 2 + 1 + w - 1) / w;
  }
}
// Partial sums the density pass along q wrote (one per tile).
int density_parts(const qj_plan *P, int q) {
  return pass_blocks(P->n[q], q, P->n[0], P->n[1], P->n[2], shape_of(P->n[q], P->tune, M_DRIFT_DENSITY, q == 2));
}

int ensure_prop(qj_plan *P, double dtk, cudaStream_t st) {
  if (P->prop_dtk == dtk) return 0;
  const int m = std::max(P->n[0], std::max(P->n[1], P->n[2]));
  k_prop_tables<<<(m + 127) / 128, 128, 0, st>>>(P->prop[0], P->prop[1], P->prop[2], P->kd[0],
                                                  P->kd[1], P->kd[2], P->n[0], P->n[1], P->n[2], dtk,
                                                  P->ph.m_per_hbar);
  QJ_CK_LAUNCH();
  P->prop_dtk = dtk;
  return 0;
}

int n_pencils(const qj_plan *P, int q) { return (int)(P->ncell / P->n[q]); }
// Star buckets of orientation q form rows of bucket_nv pencils (b = cu nv + cv):
// v is y for z pencils, z otherwise.
int bucket_nv(const qj_plan *P, int q) { return q == 2 ? P->n[1] : P->n[2]; }

// Particle data of a single box, sorted by bucket (pencil of the lower corner
// along q): one launch for a few particles (black holes), else prepare + sort.
int stars_prepare_sort(qj_plan *P, const void *pos, int n, const void *masses, double m_s, int q,
                       cudaStream_t st) {
  if (n <= 32) return launch_stars_small(pos, n, masses, m_s, geom(P), q, n_pencils(P, q), P->sb, st);
  QJ_TRY(launch_stars_prepare(pos, n, masses, m_s, geom(P), q, P->sb, st));
  return launch_bucket_sort(n, n_pencils(P, q), bucket_nv(P, q), P->sb, st);
}


// CIC deposit list of `pos` in orientation q: sorted unique cells + starts.
int deposit_list(qj_plan *P, const void *pos, int n, double m_s, const void *masses, int q,
                 bool keys_ready, void *dts_reset, cudaStream_t st) {
  if (!keys_ready)
    QJ_TRY(launch_cic_prepare(P->dbl, pos, n, masses, m_s, geom(P), q, P->keys, P->vals, st));
  QJ_TRY(launch_sort_unique(P->dbl, P->keys, P->vals, 8 * n, cell_bits(P->ncell), P->kA, P->iA,
                            P->kB, P->iB, P->ukey, P->uval, P->cell_u, P->n_unique, dts_reset, st));
  return launch_pencil_starts(P->ukey, P->n_unique, n_pencils(P, q), (unsigned)P->n[q], P->pstart, st);
}

// ---------------------------------------------------------------------------
// Fused single-precision KDK (complex64 psi).
// ---------------------------------------------------------------------------
// Per-step coefficients of a variable-step run (quantum-cosmo.py:173-181):
// kick_half[n] = m_per_hbar dt_n pot_fac_n / 2, drift[n] = dt_n kin_fac_n.
// Null = the constant-dt step of quantum-stars.py (pot_fac = kin_fac = 1).
struct StepCoefs {
  std::vector<double> kick_half, drift;
};

// One fused pass of a run: its mode, axis and arguments.
struct Phase {
  int mode, axis;
  FusedArgs a;
};
int run_phase(const qj_plan *P, const Phase &ph, cudaStream_t st) {
  return launch_fused(ph.mode, P->n[ph.axis], ph.a, st);
}

// A fused KDK run of one plan, phase by phase.  fused_kdk runs the phases in
// order; an ensemble runs each phase for all its plans (as one launch per
// fused pass where the plans' sizes allow) with the same sequence:
//   begin, density, then for k = 0..nsteps: step_begin, fft_fwd, poisson,
//   ifft2, kick, stars; unless k == nsteps: drift, join, drift_density,
//   step_end; finally end.
// Consecutive half kicks of adjacent steps share their potential (the density
// |psi|^2 and the star positions do not change between them), so nsteps
// steps take nsteps + 1 Poisson solves; each kick still advances the star
// velocities by two separate dt/2 half kicks and records dt_s between them,
// as the reference's step boundary does.
struct KdkRun {
  qj_plan *P;
  float2 *psi;
  float *pos, *vel;
  int n_s;
  double m_s, dt;
  int nsteps, si;
  const float *vext;
  double *diag;
  const StepCoefs *sc;
  void *save;
  float *vsave;
  const float *rho_src;
  bool parts = false, use_phi = false;
  int q = 2;  // the axis of the density build before kick k (and of kick k)

  double half(int n) const { return sc ? sc->kick_half[n] : P->ph.m_per_hbar * dt / 2.0; }
  double drift_dt(int n) const { return sc ? sc->drift[n] : dt; }
  double kick_coef(int k, bool last) const {
    return (k > 0 ? half(k - 1) : 0.0) + (last ? 0.0 : half(k));
  }
  int r() const { return 2 - q; }

  int begin(cudaStream_t st) {
    parts = n_s > 0;
    const int nb = P->nbox;  // boxes: fields [nb][nx][ny][nz], stars [nb][n_s][3]
    P->cur_stars = n_s;
    // the uniform potential's phase is carried in float64 (FusedArgs::phi),
    // except on the adjoint's recompute path, whose saved potentials include it
    use_phi = save == nullptr && vsave == nullptr;
    q = 2;
    if (use_phi) QJ_CK(cudaMemsetAsync(P->phi, 0, (size_t)nb * sizeof(double), st));
    QJ_TRY(launch_diag_load(false, diag, P->amax, st, nb));
    if (parts) QJ_TRY(launch_set_scalar(false, P->dts, INFINITY, st, nb));
    if (parts) {
      if (prof_on()) prof_mark_begin(st);
      QJ_TRY(launch_stars_prepare(pos, n_s * nb, nullptr, m_s, geom(P), q, P->sb, st));
      QJ_TRY(launch_bucket_sort(n_s, n_pencils(P, q), bucket_nv(P, q), P->sb, st, nb,
                                P->bstart_stride));
      if (prof_on()) prof_mark_end(7, st);
    }
    return 0;
  }
  Phase density() const {
    FusedArgs a = fused_args(P, q, M_DENSITY);
    a.psi = psi;
    if (parts) set_stars(a, P);
    a.rho_src = rho_src;
    a.half = 1;  // the passes after it read k <= n/2 of R
    return {M_DENSITY, q, a};
  }
  int step_begin(int k, cudaStream_t st) {
    if (k < nsteps) QJ_TRY(ensure_prop(P, drift_dt(k), st));
    return 0;
  }
  // The potential's passes (forward y, Poisson, inverse y, kick) each follow
  // another fused pass directly on the stream, so each launches as its
  // programmatic dependent (pdl); forward y follows the drift + density pass,
  // or on the first step the density build or the drift table.
  Phase fft_fwd() const {
    FusedArgs a = fused_args(P, 1, M_FFT_FWD);
    half_spectrum(a, P, q);
    a.pdl = 1;
    return {M_FFT_FWD, 1, a};
  }
  Phase poisson(int k) const {
    FusedArgs a = fused_args(P, r(), M_POISSON);
    a.half = 1;
    half_spectrum(a, P, q);
    a.part_in = P->part;
    a.n_part = density_parts(P, q);
    if (use_phi) {
      a.phi = P->phi;
      a.phi_coef = kick_coef(k, k == nsteps);
    }
    a.pdl = 1;
    return {M_POISSON, r(), a};
  }
  Phase ifft2() const {
    FusedArgs a = fused_args(P, 1, M_IFFT2);
    a.half = 1;
    half_spectrum(a, P, q);
    a.pdl = 1;
    return {M_IFFT2, 1, a};
  }
  Phase kick(int k) const {
    const bool last = k == nsteps;
    FusedArgs a = fused_args(P, q, M_KICK);
    a.psi = psi;
    // kick k = second half kick of step k-1 and first half kick of step k
    a.kick_coef = kick_coef(k, last);
    if (use_phi) {
      a.phi = P->phi;
      a.phi_final = last ? 1 : 0;
    }
    a.b_coeff = si ? (float)P->ph.b_coeff : 0.0f;
    a.v_ext = vext;
    a.rho_src = rho_src;
    a.do_drift = last ? 0 : 1;
    if (vsave) a.v_out = vsave + (size_t)k * P->ncell;  // V of kick k (adjoint)
    if (parts) set_stars(a, P);
    a.pdl = 1;
    return {M_KICK, q, a};
  }
  // fork: the star update and bucket sort run on the side stream while the y
  // drift pass runs on st; joined before the next density build
  int stars(int k, cudaStream_t st) {
    if (!parts) return 0;
    const bool last = k == nsteps;
    QJ_CK(cudaEventRecord(P->ev_kick, st));
    QJ_CK(cudaStreamWaitEvent(P->side, P->ev_kick, 0));
    cudaStream_t pst = P->side;
    if (prof_on()) prof_mark_begin(pst);
    UpdateArgs u;
    std::memset(&u, 0, sizeof(u));
    u.n = n_s * P->nbox;
    u.box_stars = n_s;
    u.dt = dt;
    u.k2 = k > 0;
    u.k1 = !last;
    u.drift = !last;
    u.dts_bits = P->dts;
    u.q_next = last ? -1 : r();
    u.m_s = m_s;
    QJ_TRY(launch_update_fused(pos, vel, geom(P), u, P->sb, pst));
    if (!last)
      QJ_TRY(launch_bucket_sort(n_s, n_pencils(P, r()), bucket_nv(P, r()), P->sb, pst, P->nbox,
                                P->bstart_stride));
    if (prof_on()) prof_mark_end(8, pst);
    QJ_CK(cudaEventRecord(P->ev_parts, pst));
    return 0;
  }
  // the y drift follows the kick on the stream (the star fork between them
  // is an event record, no wait), so it too launches as the kick's
  // programmatic dependent; the drift + density pass waits for the star
  // stream's event, and launches plainly
  Phase drift() const {
    FusedArgs a = fused_args(P, 1, M_DRIFT);
    a.psi = psi;
    a.pdl = 1;
    return {M_DRIFT, 1, a};
  }
  int join(cudaStream_t st) {
    if (parts) QJ_CK(cudaStreamWaitEvent(st, P->ev_parts, 0));
    return 0;
  }
  Phase drift_density() const {
    FusedArgs a = fused_args(P, r(), M_DRIFT_DENSITY);
    a.psi = psi;
    if (parts) set_stars(a, P);
    a.rho_src = rho_src;
    a.half = 1;  // the passes after it read k <= n/2 of R
    return {M_DRIFT_DENSITY, r(), a};
  }
  int step_end(int k, cudaStream_t st) {
    if (save)  // the state after drift k (before kick k + 1), for the adjoint
      QJ_CK(cudaMemcpyAsync((char *)save + (size_t)k * P->ncell * P->csz, psi,
                            P->ncell * P->csz, cudaMemcpyDeviceToDevice, st));
    q = r();
    return 0;
  }
  int end(cudaStream_t st) {
    QJ_TRY(join(st));
    return launch_diag_store(false, diag, P->amax, P->dts, parts ? 1 : 0, nsteps * dt, st,
                             P->nbox);
  }
};

int fused_kdk(qj_plan *P, float2 *psi, float *pos, float *vel, int n_s, double m_s, double dt,
              int nsteps, int si, const float *vext, double *diag, cudaStream_t st,
              const StepCoefs *sc = nullptr, void *save = nullptr, float *vsave = nullptr,
              const float *rho_src = nullptr) {
  KdkRun R{P, psi, pos, vel, n_s, m_s, dt, nsteps, si, vext, diag, sc, save, vsave, rho_src};
  QJ_TRY(R.begin(st));
  QJ_TRY(run_phase(P, R.density(), st));
  for (int k = 0; k <= nsteps; ++k) {
    QJ_TRY(R.step_begin(k, st));
    QJ_TRY(run_phase(P, R.fft_fwd(), st));
    QJ_TRY(run_phase(P, R.poisson(k), st));
    QJ_TRY(run_phase(P, R.ifft2(), st));
    QJ_TRY(run_phase(P, R.kick(k), st));
    QJ_TRY(R.stars(k, st));
    if (k == nsteps) break;
    QJ_TRY(run_phase(P, R.drift(), st));
    QJ_TRY(R.join(st));
    QJ_TRY(run_phase(P, R.drift_density(), st));
    QJ_TRY(R.step_end(k, st));
  }
  return R.end(st);
}

// ---------------------------------------------------------------------------
// Plain path: the reference's compute_step call for call (quantum-stars.py:295-330).
// ---------------------------------------------------------------------------

// get_potential(rho) -> V (rho given as rho_in, or |psi|^2 + rho_s).
int plain_potential(qj_plan *P, const void *psi, const void *rho_s, const void *rho_in, void *V,
                    int si, const void *vext, cudaStream_t st, const void *rho_gas = nullptr) {
  QJ_TRY(launch_build_rho(P->dbl, psi, rho_s, rho_gas, rho_in, 4.0 * M_PI * P->ph.G, P->ph.rho_bar,
                          P->rho_tot, P->c0, P->ncell, st));
  QJ_TRY(fft3d(P, P->c0, -1, st));
  QJ_TRY(launch_poisson_div(P->dbl, P->c0, ktabs(P), P->ncell, st));
  QJ_TRY(fft3d(P, P->c0, +1, st));
  return launch_real_part(P->dbl, P->c0, 1.0, si ? P->rho_tot : nullptr, P->ph.b_coeff, vext, V,
                          P->ncell, st);
}

// Grid accelerations of get_acceleration (:254-260) from P->rho_tot (or rho_in).
int plain_accel(qj_plan *P, const void *rho_in, void *amax_bits, cudaStream_t st) {
  QJ_TRY(launch_build_rho(P->dbl, nullptr, nullptr, nullptr, rho_in ? rho_in : P->rho_tot,
                          4.0 * M_PI * P->ph.G, P->ph.rho_bar, nullptr, P->c0, P->ncell, st));
  QJ_TRY(fft3d(P, P->c0, -1, st));
  QJ_TRY(launch_poisson_div(P->dbl, P->c0, ktabs(P), P->ncell, st));
  void *ag[3] = {P->ax, P->ay, P->az};
  for (int d = 0; d < 3; ++d) {
    QJ_TRY(launch_mul_ik(P->dbl, P->c0, d, ktabs(P), P->c1, P->ncell, st));
    QJ_TRY(fft3d(P, P->c1, +1, st));
    QJ_TRY(launch_real_part(P->dbl, P->c1, -1.0, nullptr, 0.0, nullptr, ag[d], P->ncell, st));
  }
  return launch_amax3(P->dbl, P->ax, P->ay, P->az, P->ncell, amax_bits, st);
}

int plain_bin(qj_plan *P, const void *pos, int n, double m_s, const void *masses, void *rho_s,
              cudaStream_t st) {
  QJ_CK(cudaMemsetAsync(rho_s, 0, P->ncell * P->rsz, st));
  if (n <= 0) return 0;
  QJ_TRY(deposit_list(P, pos, n, m_s, masses, 2, false, nullptr, st));
  return launch_scatter_unique(P->dbl, P->ukey, P->uval, P->n_unique, 8 * n, rho_s, st);
}

int plain_kdk(qj_plan *P, void *psi, void *pos, void *vel, int n_s, double m_s, double dt,
              int nsteps, int si, const void *vext, double *diag, cudaStream_t st,
              const StepCoefs *sc = nullptr, void *save = nullptr,
              const void *rho_src = nullptr) {
  QJ_TRY(ensure_plain_ws(P));
  QJ_TRY(launch_diag_load(P->dbl, diag, P->amax, st));
  for (int step = 0; step < nsteps; ++step) {
    const double coef = sc ? sc->kick_half[step] : P->ph.m_per_hbar * dt / 2.0;
    const double dtk = sc ? sc->drift[step] : dt;
    for (int half = 0; half < 2; ++half) {
      // (1/2) kick; a fixed source density (no stars) takes the stars' place
      if (!rho_src) QJ_TRY(plain_bin(P, pos, n_s, m_s, nullptr, P->rho_s, st));
      QJ_TRY(plain_potential(P, psi, rho_src ? rho_src : P->rho_s, nullptr, P->V, si, vext, st));
      QJ_TRY(launch_kick_plain(P->dbl, psi, P->V, coef, P->ncell, st));
      QJ_TRY(plain_accel(P, nullptr, P->amax, st));
      if (n_s > 0) {
        QJ_TRY(launch_gather_dense(P->dbl, pos, n_s, geom(P), P->ax, P->ay, P->az, P->acc, st));
        if (half == 1) QJ_TRY(launch_set_scalar(P->dbl, P->dts, INFINITY, st));
        UpdateArgs u;
        std::memset(&u, 0, sizeof(u));
        u.n = n_s;
        u.dt = dt;
        u.k1 = half == 0;
        u.k2 = half == 1;
        u.drift = half == 0;
        u.dts_bits = P->dts;
        QJ_TRY(launch_particles_update(P->dbl, pos, vel, P->acc, geom(P), u, st));
      }
      if (half == 0) {
        // drift (:307-309); the particle drift ran in the update above
        QJ_TRY(fft3d(P, psi, -1, st));
        QJ_TRY(launch_drift_mul(P->dbl, psi, ktabs(P), dtk, P->ph.m_per_hbar, P->ncell, st));
        QJ_TRY(fft3d(P, psi, +1, st));
        if (save)
          QJ_CK(cudaMemcpyAsync((char *)save + (size_t)step * P->ncell * P->csz, psi,
                                P->ncell * P->csz, cudaMemcpyDeviceToDevice, st));
      }
    }
  }
  return launch_diag_store(P->dbl, diag, P->amax, P->dts, n_s > 0 ? 1 : 0, nsteps * dt, st);
}

// ---------------------------------------------------------------------------
// Adjoint of the psi-only KDK step (no particles).  A run of nsteps is split
// into chunks of K steps; each chunk is one qj_kdk_step call, i.e. kicks
// [c/2, c, ..., c, c/2] (c = m_per_hbar dt) around K drifts.  Each kick is
// psi' = exp(-i c_j V[|psi|^2]) psi with V = (L + b) |psi|^2 + V_ext and L the
// Poisson operator (real, symmetric).  With the gradient g = dL/dRe + i dL/dIm,
// its adjoint is
//     g <- exp(+i c_j V) g + 2 [(L + b) mu] psi,   mu = c_j Im(conj(g) psi'),
// one Poisson solve for V and one for (L + b) mu.  A drift's adjoint is the
// drift with -dt.  psi is checkpointed at chunk starts; the reverse sweep
// recomputes each chunk forward, saving the state before every kick.
// ---------------------------------------------------------------------------
int kdk_chunk(qj_plan *P, void *psi, int m, double dt, int si, const void *vext,
              const void *rho_src, cudaStream_t st, void *save, float *vsave = nullptr) {
  if (!P->tmp_diag) QJ_TRY(dev_alloc(P, &P->tmp_diag, 3 * sizeof(double)));
  QJ_CK(cudaMemsetAsync(P->tmp_diag, 0, 3 * sizeof(double), st));
  if (P->dbl)
    return plain_kdk(P, psi, nullptr, nullptr, 0, 0.0, dt, m, si, vext, (double *)P->tmp_diag, st,
                     nullptr, save, rho_src);
  return fused_kdk(P, (float2 *)psi, nullptr, nullptr, 0, 0.0, dt, m, si, (const float *)vext,
                   (double *)P->tmp_diag, st, nullptr, save, vsave, (const float *)rho_src);
}

int adjoint_sweep(qj_plan *P, const void *ckpt, void *g, int nsteps, int K, double dt, int si,
                  const void *vext, const void *rho_src, cudaStream_t st) {
  QJ_TRY(ensure_plain_ws(P));
  const size_t fb = P->ncell * P->csz;
  if (!P->adj_psi) QJ_TRY(dev_alloc(P, &P->adj_psi, fb));
  if (P->adj_cap < K) {
    QJ_TRY(dev_alloc(P, &P->adj_states, (size_t)K * fb));
    // single precision: the recompute also keeps each kick's potential, so
    // the reverse sweep needs one Poisson solve per kick instead of two
    if (!P->dbl) QJ_TRY(dev_alloc(P, &P->adj_V, (size_t)(K + 1) * P->ncell * sizeof(float)));
    P->adj_cap = K;
  }
  const int nseg = (nsteps + K - 1) / K;
  const double half = P->ph.m_per_hbar * dt / 2.0;
  void *mu = P->ax;
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int m = std::min(K, nsteps - seg * K);
    const void *c0 = (const char *)ckpt + (size_t)seg * fb;
    QJ_CK(cudaMemcpyAsync(P->adj_psi, c0, fb, cudaMemcpyDeviceToDevice, st));
    QJ_TRY(kdk_chunk(P, P->adj_psi, m, dt, si, vext, rho_src, st, P->adj_states,
                     (float *)P->adj_V));
    for (int j = m; j >= 0; --j) {
      const void *pre = j == 0 ? c0 : (const char *)P->adj_states + (size_t)(j - 1) * fb;
      const double coef = half * ((j == 0 || j == m) ? 1.0 : 2.0);
      const void *Vj = P->V;
      if (P->dbl)
        QJ_TRY(plain_potential(P, pre, rho_src, nullptr, P->V, si, vext, st));
      else
        Vj = (const float *)P->adj_V + (size_t)j * P->ncell;
      // W = (L + b) mu: the Poisson operator without the rho_bar shift; mu
      // itself is kept only for the self-interaction term
      if (P->dbl) {
        QJ_TRY(launch_adj_mu(P->dbl, g, pre, Vj, coef, si ? mu : nullptr, 4.0 * M_PI * P->ph.G,
                             P->c0, P->ncell, st));
        QJ_TRY(fft3d(P, P->c0, -1, st));
        QJ_TRY(launch_poisson_div(P->dbl, P->c0, ktabs(P), P->ncell, st));
        QJ_TRY(fft3d(P, P->c0, +1, st));
        QJ_TRY(launch_adj_update(P->dbl, g, pre, Vj, P->c0, si ? mu : nullptr, P->ph.b_coeff,
                                 coef, P->ncell, st));
        if (j > 0) {  // adjoint of drift j - 1: the drift with -dt
          QJ_TRY(fft3d(P, g, -1, st));
          QJ_TRY(launch_drift_mul(P->dbl, g, ktabs(P), -dt, P->ph.m_per_hbar, P->ncell, st));
          QJ_TRY(fft3d(P, g, +1, st));
        }
      } else {
        // the forward step's potential passes with mu as the density: mu,
        // its partial sums and the z transform (ADJ_SOURCE); forward y;
        // Poisson along x with no rho_bar shift and the k = 0 term kept in W;
        // inverse y; then the inverse z transform to W, the g update and the
        // z part of the drift adjoint (ADJ_UPDATE); the drift adjoint along y
        // and x (the drift with -dt)
        const int q = 2, r = 0;
        if (j > 0) QJ_TRY(ensure_prop(P, -dt, st));
        FusedArgs a = fused_args(P, q, M_ADJ_SOURCE);
        a.psi = (float2 *)g;
        a.adj_pre = (const float2 *)pre;
        a.adj_V = (const float *)Vj;
        a.adj_mu = si ? (float *)mu : nullptr;
        a.kick_coef = coef;
        a.half = 1;
        QJ_TRY(launch_fused(M_ADJ_SOURCE, P->n[q], a, st));
        // each pass from here follows another fused pass directly: launched
        // as its programmatic dependent
        a = fused_args(P, 1, M_FFT_FWD);
        half_spectrum(a, P, q);
        a.pdl = 1;
        QJ_TRY(launch_fused(M_FFT_FWD, P->n[1], a, st));
        a = fused_args(P, r, M_POISSON);
        a.half = 1;
        half_spectrum(a, P, q);
        a.part_in = P->part;
        a.n_part = pass_blocks(P->n[q], q, P->n[0], P->n[1], P->n[2], 0);  // ADJ_SOURCE's tiles
        a.rho_bar = 0.0;
        a.pdl = 1;
        QJ_TRY(launch_fused(M_POISSON, P->n[r], a, st));
        a = fused_args(P, 1, M_IFFT2);
        a.half = 1;
        half_spectrum(a, P, q);
        a.pdl = 1;
        QJ_TRY(launch_fused(M_IFFT2, P->n[1], a, st));
        a = fused_args(P, q, M_ADJ_UPDATE);
        a.psi = (float2 *)g;
        a.adj_pre = (const float2 *)pre;
        a.adj_V = (const float *)Vj;
        a.adj_mu = si ? (float *)mu : nullptr;
        a.kick_coef = coef;
        a.b_coeff = si ? (float)P->ph.b_coeff : 0.0f;
        a.do_drift = j > 0 ? 1 : 0;
        a.pdl = 1;
        QJ_TRY(launch_fused(M_ADJ_UPDATE, P->n[q], a, st));
        if (j > 0)
          for (int ax = 1; ax >= 0; --ax) {
            FusedArgs d = fused_args(P, ax, M_DRIFT);
            d.psi = (float2 *)g;
            d.pdl = 1;
            QJ_TRY(launch_fused(M_DRIFT, P->n[ax], d, st));
          }
      }
    }
  }
  return 0;
}


// ---------------------------------------------------------------------------
// Gas + black hole step, quantum-gas-bh.py:537-578 (quantum-bh.py:346-381
// without gas).  The dark-matter accretion between the second half kick and
// the next step's first half kick changes the density, so the two half kicks
// of a step keep separate Poisson solves here.
// ---------------------------------------------------------------------------
struct GasArgs {
  void *psi, *rho, *v[3], *m_bh, *pos, *vel;
  int n_bh;
  double dt;
  double sigma_v;
  int dm_accretion;
  double bondi;  // r_acc_mult, <= 0 disables the gas sink
};

int ensure_gas_ws(qj_plan *P) {
  if (!P->gas_prim) QJ_TRY(dev_alloc(P, &P->gas_prim, 16 * P->ncell * P->rsz));
  return 0;
}

int gas_hydro(qj_plan *P, const GasArgs &g, cudaStream_t st) {
  const double dx = P->g.Lx / P->n[0];
  return launch_hydro(P->dbl, g.rho, g.v[0], g.v[1], g.v[2], P->gas_prim, P->n[0], dx, g.dt,
                      P->ph.cs, (g.bondi > 0 && g.n_bh > 0) ? 1 : 0, st,
                      P->tune[9] > 0 ? P->tune[9] : 256);
}

// first / last: the call's first and last step (the uniform potential's phase
// is carried in float64 over the call, see FusedArgs::phi).
int fused_gas_step(qj_plan *P, const GasArgs &g, cudaStream_t st, bool first, bool last) {
  const bool bh = g.n_bh > 0, gas = g.rho != nullptr;
  const double dx = P->g.Lx / P->n[0];
  const double half = P->ph.m_per_hbar * g.dt / 2.0;
  QJ_TRY(ensure_prop(P, g.dt, st));
  if (first) QJ_CK(cudaMemsetAsync(P->phi, 0, sizeof(double), st));
  auto stars = [&](FusedArgs &a) {
    if (bh) set_stars(a, P);
    if (gas) {
      a.grho = (const float *)g.rho;
    }
  };
  auto poisson = [&](int q, int r) -> int {
    FusedArgs a = fused_args(P, 1, M_FFT_FWD);
    half_spectrum(a, P, q);
    QJ_TRY(launch_fused(M_FFT_FWD, P->n[1], a, st));
    a = fused_args(P, r, M_POISSON);
    a.half = 1;
    half_spectrum(a, P, q);
    a.part_in = P->part;
    a.n_part = density_parts(P, q);
    a.phi = P->phi;
    a.phi_coef = half;
    QJ_TRY(launch_fused(M_POISSON, P->n[r], a, st));
    a = fused_args(P, 1, M_IFFT2);
    a.half = 1;
    half_spectrum(a, P, q);
    return launch_fused(M_IFFT2, P->n[1], a, st);
  };
  auto kick = [&](int q, int drift) -> int {
    FusedArgs a = fused_args(P, q, M_KICK);
    a.psi = (float2 *)g.psi;
    a.kick_coef = half;
    a.do_drift = drift;
    a.phi = P->phi;
    a.phi_final = (last && !drift) ? 1 : 0;  // the call's last half kick
    if (bh) set_stars(a, P);
    if (gas) {
      for (int d = 0; d < 3; ++d) a.gv[d] = (float *)g.v[d];
      a.gas_dt = (float)(g.dt / 2.0);
    }
    return launch_fused(M_KICK, P->n[q], a, st);
  };
  UpdateArgs u;
  std::memset(&u, 0, sizeof(u));
  u.n = g.n_bh;
  u.dt = g.dt;
  u.dts_bits = P->dts;
  u.masses = g.m_bh;
  // (1/2) kick
  if (bh) {
    QJ_TRY(stars_prepare_sort(P, g.pos, g.n_bh, g.m_bh, 0.0, 2, st));
  }
  {
    FusedArgs a = fused_args(P, 2, M_DENSITY);
    a.psi = (float2 *)g.psi;
    stars(a);
    a.half = 1;  // the passes after it read k <= n/2 of R
    QJ_TRY(launch_fused(M_DENSITY, P->n[2], a, st));
  }
  QJ_TRY(poisson(2, 0));
  QJ_TRY(kick(2, 1));  // + drift along z
  if (bh) {
    u.k1 = 1;
    u.drift = 1;
    u.q_next = 0;
    QJ_TRY(launch_update_fused(g.pos, g.vel, geom(P), u, P->sb, st));
  }
  {
    FusedArgs a = fused_args(P, 1, M_DRIFT);
    a.psi = (float2 *)g.psi;
    QJ_TRY(launch_fused(M_DRIFT, P->n[1], a, st));
  }
  if (gas) QJ_TRY(gas_hydro(P, g, st));
  if (bh && gas && g.bondi > 0)
    QJ_TRY(launch_bondi(false, g.rho, g.pos, g.m_bh, P->n[0], dx, P->g.Lx, P->ph.cs, P->ph.G, g.dt,
                        g.bondi, st));
  if (bh) {
    // deposit of the drifted black holes (their mass may have changed)
    QJ_TRY(stars_prepare_sort(P, g.pos, g.n_bh, g.m_bh, 0.0, 0, st));
  }
  {
    FusedArgs a = fused_args(P, 0, M_DRIFT_DENSITY);
    a.psi = (float2 *)g.psi;
    stars(a);
    a.half = 1;  // the passes after it read k <= n/2 of R
    QJ_TRY(launch_fused(M_DRIFT_DENSITY, P->n[0], a, st));
  }
  // (1/2) kick
  QJ_TRY(poisson(0, 2));
  QJ_TRY(kick(0, 0));
  if (bh) {
    u.k1 = 0;
    u.k2 = 1;
    u.drift = 0;
    u.q_next = -1;
    QJ_TRY(launch_update_fused(g.pos, g.vel, geom(P), u, P->sb, st));
    if (g.dm_accretion)
      QJ_TRY(launch_accrete(false, g.psi, g.pos, g.vel, g.m_bh, P->n[0], dx, g.sigma_v, P->ph.G,
                            P->ph.m_per_hbar, P->ph.c_light, g.dt, st));
  }
  return 0;
}

int plain_gas_step(qj_plan *P, const GasArgs &g, cudaStream_t st) {
  const bool bh = g.n_bh > 0, gas = g.rho != nullptr;
  const double dx = P->g.Lx / P->n[0];
  const double coef = P->ph.m_per_hbar * g.dt / 2.0;
  for (int half = 0; half < 2; ++half) {
    QJ_TRY(plain_bin(P, g.pos, g.n_bh, 0.0, g.m_bh, P->rho_s, st));
    QJ_TRY(plain_potential(P, g.psi, P->rho_s, nullptr, P->V, 0, nullptr, st, gas ? g.rho : nullptr));
    QJ_TRY(launch_kick_plain(P->dbl, g.psi, P->V, coef, P->ncell, st));
    if (gas) {  // apply_grav_accel (:255-266) from rho_tot
      QJ_TRY(plain_accel(P, nullptr, P->tmp_scalar, st));
      QJ_TRY(launch_gas_kick(P->dbl, g.v[0], g.v[1], g.v[2], P->ax, P->ay, P->az, g.dt / 2.0,
                             P->ncell, st));
    }
    if (bh) {  // get_acceleration (:452-490)
      QJ_TRY(plain_accel(P, nullptr, P->tmp_scalar, st));
      QJ_TRY(launch_gather_dense(P->dbl, g.pos, g.n_bh, geom(P), P->ax, P->ay, P->az, P->acc, st));
      UpdateArgs u;
      std::memset(&u, 0, sizeof(u));
      u.n = g.n_bh;
      u.dt = g.dt;
      u.k1 = half == 0;
      u.k2 = half == 1;
      u.drift = half == 0;
      u.dts_bits = P->dts;
      QJ_TRY(launch_particles_update(P->dbl, g.pos, g.vel, P->acc, geom(P), u, st));
    }
    if (half == 0) {
      QJ_TRY(fft3d(P, g.psi, -1, st));
      QJ_TRY(launch_drift_mul(P->dbl, g.psi, ktabs(P), g.dt, P->ph.m_per_hbar, P->ncell, st));
      QJ_TRY(fft3d(P, g.psi, +1, st));
      if (gas) QJ_TRY(gas_hydro(P, g, st));
      if (bh && gas && g.bondi > 0)
        QJ_TRY(launch_bondi(true, g.rho, g.pos, g.m_bh, P->n[0], dx, P->g.Lx, P->ph.cs, P->ph.G,
                            g.dt, g.bondi, st));
    }
  }
  if (bh && g.dm_accretion)
    QJ_TRY(launch_accrete(true, g.psi, g.pos, g.vel, g.m_bh, P->n[0], dx, g.sigma_v, P->ph.G,
                          P->ph.m_per_hbar, P->ph.c_light, g.dt, st));
  return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char *qj_last_error(void) { return g_err.c_str(); }

// Entry points other than qj_kdk_step work on single-box plans.
#define QJ_ONE_BOX(P, name)                                                     \
  do {                                                                          \
    if ((P) && (P)->nbox != 1) {                                                \
      set_error("%s: batched plans (nbox > 1) support qj_kdk_step only", name); \
      return QJ_ERR_ARG;                                                        \
    }                                                                           \
  } while (0)

int qj_plan_create(qj_plan **plan, const qj_grid *grid, const qj_phys *phys, int precision,
                   int max_particles) {
  return qj_plan_create_batched(plan, grid, phys, precision, max_particles, 1);
}

int qj_plan_create_batched(qj_plan **plan, const qj_grid *grid, const qj_phys *phys, int precision,
                           int max_particles, int nbox) {
  if (!plan || !grid || !phys) {
    set_error("qj_plan_create: null argument");
    return QJ_ERR_ARG;
  }
  *plan = nullptr;
  if (nbox < 1 || nbox > 65535 || (nbox > 1 && precision != QJ_FUSED_F32)) {
    set_error("qj_plan_create_batched: nbox must be in [1, 65535], batches need QJ_FUSED_F32");
    return QJ_ERR_ARG;
  }
  if (precision != QJ_PLAIN_F64 && precision != QJ_FUSED_F32) {
    set_error("qj_plan_create: precision must be QJ_PLAIN_F64 or QJ_FUSED_F32");
    return QJ_ERR_ARG;
  }
  const int n[3] = {grid->nx, grid->ny, grid->nz};
  for (int a = 0; a < 3; ++a) {
    if (!fft_length_supported(n[a])) {
      set_error("qj_plan_create: axis %d length %d unsupported (16, 32, 64, 96, 128, 256, 512)", a,
                n[a]);
      return QJ_ERR_ARG;
    }
  }
  if (n[2] % 16) {
    set_error("qj_plan_create: nz must be a multiple of 16");
    return QJ_ERR_ARG;
  }
  if (!(grid->Lx > 0 && grid->Ly > 0 && grid->Lz > 0)) {
    set_error("qj_plan_create: box lengths must be positive");
    return QJ_ERR_ARG;
  }
  if (max_particles < 0 || max_particles > (1 << 24) / 8) {
    set_error("qj_plan_create: max_particles must be in [0, %d]", (1 << 24) / 8);
    return QJ_ERR_ARG;
  }
  qj_plan *P = new qj_plan();
  P->g = *grid;
  P->ph = *phys;
  P->prec = precision;
  P->dbl = precision == QJ_PLAIN_F64;
  P->max_particles = max_particles;
  for (int a = 0; a < 3; ++a) P->n[a] = n[a];
  P->ncell = (long long)n[0] * n[1] * n[2];
  P->rsz = P->dbl ? 8 : 4;
  P->csz = 2 * P->rsz;
  const double L[3] = {grid->Lx, grid->Ly, grid->Lz};
  int rc = 0;
  auto fail = [&](int code) {
    qj_plan_destroy(P);
    return code;
  };
  for (int a = 0; a < 3 && !rc; ++a) {
    const int N = n[a];
    std::vector<double> k(N), kt(N);
    std::vector<float> kf(N), ktf(N);
    for (int i = 0; i < N; ++i) {
      // ifftshift(2 pi / L * arange(-N/2, N/2)): index N/2 holds -pi N / L
      const int m = i < N / 2 ? i : i - N;
      k[i] = 2.0 * M_PI / L[a] * m;
      kt[i] = (i == N / 2) ? 0.0 : k[i];
      kf[i] = (float)k[i];
      ktf[i] = (float)kt[i];
    }
    if ((rc = dev_alloc_t(P, &P->kd[a], N))) break;
    if ((rc = dev_alloc_t(P, &P->kf[a], N))) break;
    if ((rc = dev_alloc_t(P, &P->ktf[a], N))) break;
    if ((rc = dev_alloc_t(P, &P->prop[a], N))) break;
    cudaError_t e = cudaMemcpy(P->kd[a], k.data(), N * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(P->kf[a], kf.data(), N * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(P->ktf[a], ktf.data(), N * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      rc = cuda_fail(e, "cudaMemcpy(tables)", __FILE__, __LINE__);
      break;
    }
    P->kr[a] = P->dbl ? (void *)P->kd[a] : (void *)P->kf[a];
    // twiddles w[m] = exp(-2 pi i m / N), long double, rounded once
    if (P->dbl) {
      std::vector<double2> w(N);
      for (int m = 0; m < N; ++m) {
        const long double th = -2.0L * 3.14159265358979323846264338327950288L * m / N;
        w[m] = double2{(double)cosl(th), (double)sinl(th)};
      }
      if ((rc = dev_alloc(P, &P->tw[a], N * sizeof(double2)))) break;
      e = cudaMemcpy(P->tw[a], w.data(), N * sizeof(double2), cudaMemcpyHostToDevice);
    } else {
      std::vector<float2> w(N);
      for (int m = 0; m < N; ++m) {
        const long double th = -2.0L * 3.14159265358979323846264338327950288L * m / N;
        w[m] = float2{(float)cosl(th), (float)sinl(th)};
      }
      if ((rc = dev_alloc(P, &P->tw[a], N * sizeof(float2)))) break;
      e = cudaMemcpy(P->tw[a], w.data(), N * sizeof(float2), cudaMemcpyHostToDevice);
      const std::vector<float2> ts = stage_twiddles(N);
      if (e == cudaSuccess && !(rc = dev_alloc_t(P, &P->tws[a], ts.size())))
        e = cudaMemcpy(P->tws[a], ts.data(), ts.size() * sizeof(float2), cudaMemcpyHostToDevice);
      if (rc) break;
      if (has_radix_variant(N)) {
        const std::vector<float2> ta = stage_twiddles(N, 1);
        if (e == cudaSuccess && !(rc = dev_alloc_t(P, &P->tws_alt[a], ta.size())))
          e = cudaMemcpy(P->tws_alt[a], ta.data(), ta.size() * sizeof(float2),
                         cudaMemcpyHostToDevice);
        if (rc) break;
      }
    }
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemcpy(twiddles)", __FILE__, __LINE__);
  }
  if (rc) return fail(rc);
  P->nbox = nbox;
  if (!P->dbl) {
    if ((rc = dev_alloc_t(P, &P->R, P->ncell * nbox))) return fail(rc);
    if ((rc = dev_alloc_t(P, &P->S1, P->ncell * nbox))) return fail(rc);
    if ((rc = dev_alloc_t(P, &P->S2, P->ncell * nbox))) return fail(rc);
    int nb = 0;  // partial sums of a density pass, over every shape variant
    for (int a = 0; a < 3; ++a)
      for (int v = 0; v < 4; ++v) nb = std::max(nb, pass_blocks(n[a], a, n[0], n[1], n[2], v));
    P->part_stride = nb;
    if ((rc = dev_alloc_t(P, &P->part, (size_t)nb * nbox))) return fail(rc);
  } else {
    if ((rc = ensure_plain_ws(P))) return fail(rc);
  }
  const size_t np8 = (size_t)8 * std::max(1, max_particles);
  for (unsigned **b : {&P->keys, &P->kA, &P->iA, &P->kB, &P->iB, &P->ukey, &P->cell_u})
    if ((rc = dev_alloc_t(P, b, np8))) return fail(rc);
  if ((rc = dev_alloc(P, &P->vals, np8 * P->rsz))) return fail(rc);
  if ((rc = dev_alloc(P, &P->uval, np8 * P->rsz))) return fail(rc);
  if ((rc = dev_alloc(P, &P->A, 3 * np8 * P->rsz * nbox))) return fail(rc);
  if ((rc = dev_alloc(P, &P->acc, 3 * (np8 / 8) * P->rsz))) return fail(rc);
  long long npen = 0;
  for (int a = 0; a < 3; ++a) npen = std::max(npen, P->ncell / n[a]);
  P->bstart_stride = (int)(npen + 1);
  if (!P->dbl) {
    const size_t np = (size_t)std::max(1, max_particles) * nbox;
    StarBufs &b = P->sb;
    if ((rc = dev_alloc_t(P, &b.sidx, np))) return fail(rc);
    if ((rc = dev_alloc_t(P, &b.sw0, np))) return fail(rc);
    if ((rc = dev_alloc_t(P, &b.sw1, np))) return fail(rc);
    if ((rc = dev_alloc_t(P, &b.bkey, np))) return fail(rc);
    if ((rc = dev_alloc_t(P, &b.perm, np))) return fail(rc);
    if ((rc = dev_alloc_t(P, &b.skey, np))) return fail(rc);
    if ((rc = dev_alloc_t(P, &b.sortbuf, 4 * np))) return fail(rc);
    if ((rc = dev_alloc_t(P, &b.bstart, (size_t)(npen + 1) * nbox))) return fail(rc);
    b.mstride = (int)((npen + 1 + 31) / 32);
    if ((rc = dev_alloc_t(P, &b.pmask, (size_t)b.mstride * nbox))) return fail(rc);
    b.A = (float *)P->A;
    int lo = 0, hi = 0;
    cudaError_t e0 = cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (e0 == cudaSuccess) e0 = cudaStreamCreateWithPriority(&P->side, cudaStreamNonBlocking, hi);
    if (e0 == cudaSuccess) e0 = cudaEventCreateWithFlags(&P->ev_kick, cudaEventDisableTiming);
    if (e0 == cudaSuccess) e0 = cudaEventCreateWithFlags(&P->ev_parts, cudaEventDisableTiming);
    if (e0 != cudaSuccess) return fail(cuda_fail(e0, "side stream", __FILE__, __LINE__));
  }
  if ((rc = dev_alloc_t(P, &P->pstart, npen + 1))) return fail(rc);
  if ((rc = dev_alloc_t(P, &P->n_unique, 1))) return fail(rc);
  if ((rc = dev_alloc(P, &P->amax, 8 * (size_t)nbox))) return fail(rc);
  if ((rc = dev_alloc(P, &P->dts, 8 * (size_t)nbox))) return fail(rc);
  if ((rc = dev_alloc(P, &P->tmp_scalar, 8))) return fail(rc);
  if ((rc = dev_alloc_t(P, &P->err, 4))) return fail(rc);
  if ((rc = dev_alloc_t(P, &P->phi, (size_t)nbox))) return fail(rc);
  if (cudaMemset(P->err, 0, 4 * sizeof(unsigned)) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "plan init", __FILE__, __LINE__));
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return fail(cuda_fail(e, "plan init", __FILE__, __LINE__));
  *plan = P;
  return QJ_OK;
}

int qj_plan_destroy(qj_plan *P) {
  if (!P) return QJ_OK;
  if (P->side) {
    cudaStreamSynchronize(P->side);
    cudaStreamDestroy(P->side);
  }
  if (P->ev_kick) cudaEventDestroy(P->ev_kick);
  if (P->ev_parts) cudaEventDestroy(P->ev_parts);
  for (void *p : P->allocs) cudaFree(p);
  delete P;
  return QJ_OK;
}

int qj_plan_set_phys(qj_plan *P, const qj_phys *phys) {
  if (!P || !phys) {
    set_error("qj_plan_set_phys: null argument");
    return QJ_ERR_ARG;
  }
  if (phys->m_per_hbar != P->ph.m_per_hbar) P->prop_dtk = NAN;
  P->ph = *phys;
  return QJ_OK;
}

int64_t qj_plan_workspace_bytes(const qj_plan *P) { return P ? P->ws_bytes : 0; }

int qj_bondi_ambient(qj_plan *P, void *rho, const void *vx, const void *vy, const void *vz,
                     const double *x_bh, const double *v_bh, double M_bh, double dt,
                     double r_acc_mult, double lam, double fmax, double ann_lo, double ann_hi,
                     double *out, void *stream) {
  if (!P || !rho || !x_bh || !out || (vx && (!vy || !vz || !v_bh)) || !(dt >= 0) ||
      !(r_acc_mult > 0) || !(M_bh >= 0)) {
    set_error("qj_bondi_ambient: bad argument");
    return QJ_ERR_ARG;
  }
  QJ_ONE_BOX(P, "qj_bondi_ambient");
  if (P->n[0] != P->n[1] || P->n[0] != P->n[2] || P->g.Lx != P->g.Ly || P->g.Lx != P->g.Lz) {
    set_error("qj_bondi_ambient: needs a cubic grid and box");
    return QJ_ERR_ARG;
  }
  const double zero[3] = {0.0, 0.0, 0.0};
  return launch_bondi_ambient(P->dbl, rho, vx, vy, vz, P->n[0], P->g.Lx / P->n[0], P->g.Lx,
                              x_bh, v_bh ? v_bh : zero, M_bh, P->ph.cs, P->ph.G, dt, r_acc_mult,
                              lam, fmax, ann_lo, ann_hi, out, (cudaStream_t)stream);
}

int qj_hydro_cfl_dt(qj_plan *P, const void *vx, const void *vy, const void *vz, double cs,
                    double cfl, double dt, double *dt_out, void *stream) {
  if (!P || !vx || !vy || !vz || !dt_out || !(cfl > 0) || !(dt > 0)) {
    set_error("qj_hydro_cfl_dt: bad argument");
    return QJ_ERR_ARG;
  }
  QJ_ONE_BOX(P, "qj_hydro_cfl_dt");
  const int nb = 592;
  if (!P->cfl_part) QJ_TRY(dev_alloc_t(P, &P->cfl_part, (size_t)nb));
  return launch_cfl_dt(P->dbl, vx, vy, vz, P->ncell, cs, P->g.Lx / P->n[0], cfl, dt,
                       P->cfl_part, nb, dt_out, (cudaStream_t)stream);
}

}  // extern "C"

namespace {
// seed_mass_from_time, quantum-fluid-accretion.py:682-690
double facc_seed(double t, double placed, const qj_facc_params &q) {
  const double pl = placed > 0.5 ? 1.0 : 0.0;
  double s;
  if (q.ramp_on)
    s = 0.5 * (1.0 + std::tanh((t - q.ramp_center) / (q.ramp_w + 1e-30))) *
        (t >= q.bh_inject_t ? 1.0 : 0.0);
  else
    s = t >= q.bh_inject_t ? 1.0 : 0.0;
  return q.bh_init_m * s * pl;
}

// One compute_step of quantum-fluid-accretion.py:695-870 (plain path).
int facc_step(qj_plan *P, void *psi, void *rho, void *v[3], qj_facc_state &S,
              const qj_facc_params &q, double dt, qj_facc_diag &D, cudaStream_t st) {
  const bool dbl = P->dbl;
  const long long nc = P->ncell;
  const int n = P->n[0];
  const double dx = P->g.Lx / n, L = P->g.Lx, G = P->ph.G, mph = P->ph.m_per_hbar, cs = q.cs;
  const double fourpiG = 4.0 * M_PI * G;
  const int nb = 592;
  double *sc = P->facc_scal;  // [0] dt_eff, [2..3] means, [4..6] sample, [8..14] Bondi, [15] argmax
  auto host = [&](int i, int cnt, double *dst) -> int {
    QJ_CK(cudaMemcpyAsync(dst, sc + i, cnt * sizeof(double), cudaMemcpyDeviceToHost, st));
    QJ_CK(cudaStreamSynchronize(st));
    return 0;
  };
  // hydro CFL cap (:697-701)
  QJ_TRY(launch_cfl_dt(dbl, v[0], v[1], v[2], nc, cs, dx, q.hydro_cfl, dt, P->cfl_part, nb, sc, st));
  double dt_eff = 0.0;
  QJ_TRY(host(0, 1, &dt_eff));
  const double M_eff = facc_seed(S.t, S.placed, q) + S.M_acc;
  const double r_soft = q.r_acc_mult * dx;
  QJ_TRY(launch_mean_dm_gas(dbl, psi, rho, nc, P->facc_part, nb, sc + 2, st));
  double means[2];
  QJ_TRY(host(2, 2, means));
  const double rho_bg = means[0] + means[1];
  const double k_cut = q.k_cut_frac * (M_PI / dx);
  const double active = S.placed > 0.5 ? 1.0 : 0.0;
  // V^ of |psi|^2 + rho (+ rho_bh) against rho_bg into c0 (get_potential_bg, :182-185)
  auto vhat = [&](const void *rho_bh) -> int {
    QJ_TRY(launch_build_rho(dbl, psi, rho, rho_bh, nullptr, fourpiG, rho_bg, nullptr, P->c0, nc, st));
    QJ_TRY(fft3d(P, P->c0, -1, st));
    return launch_poisson_div(dbl, P->c0, ktabs(P), nc, st);
  };
  // the three accelerations -Re ifftn(i k_d V^) of c0 into ax, ay, az (accel_from_Vhat)
  auto accel = [&]() -> int {
    void *ag[3] = {P->ax, P->ay, P->az};
    for (int d = 0; d < 3; ++d) {
      QJ_TRY(launch_mul_ik(dbl, P->c0, d, ktabs(P), P->c1, nc, st));
      QJ_TRY(fft3d(P, P->c1, +1, st));
      QJ_TRY(launch_real_part(dbl, P->c1, -1.0, nullptr, 0.0, nullptr, ag[d], nc, st));
    }
    return 0;
  };
  // black-hole half kick with the low-passed force of the DM + gas potential
  auto bh_kick = [&]() -> int {
    QJ_TRY(vhat(nullptr));
    QJ_TRY(launch_kfilter(dbl, P->c0, ktabs(P), 0, k_cut * k_cut, nc, st));
    QJ_TRY(accel());
    QJ_TRY(launch_cic_sample3(dbl, P->ax, P->ay, P->az, n, S.x_bh, dx, sc + 4, st));
    double a[3];
    QJ_TRY(host(4, 3, a));
    for (int d = 0; d < 3; ++d) S.v_bh[d] = S.v_bh[d] + a[d] * (dt_eff / 2.0) * active;
    return 0;
  };
  // Gaussian-softened CIC density of the black hole into facc_bh (:729-736)
  // (out = nullptr when the black hole does not gravitate this kick)
  auto soft_bh = [&](double M, double r, const void *&out) -> int {
    out = nullptr;
    if (!(q.bh_on && q.bh_grav) || !(S.placed > 0.5 && M > 0.0)) return 0;
    QJ_CK(cudaMemsetAsync(P->facc_bh, 0, nc * P->rsz, st));
    QJ_TRY(launch_cic_point(dbl, P->facc_bh, n, S.x_bh, dx, M, st));
    QJ_TRY(launch_build_rho(dbl, nullptr, nullptr, nullptr, P->facc_bh, 1.0, 0.0, nullptr, P->c1,
                            nc, st));
    QJ_TRY(fft3d(P, P->c1, -1, st));
    QJ_TRY(launch_kfilter(dbl, P->c1, ktabs(P), 1, r * r, nc, st));
    QJ_TRY(fft3d(P, P->c1, +1, st));
    QJ_TRY(launch_real_part(dbl, P->c1, 1.0, nullptr, 0.0, nullptr, P->facc_bh, nc, st));
    out = P->facc_bh;
    return 0;
  };
  // kick: psi and gas with the potential of |psi|^2 + rho + rho_bh
  auto kick = [&](const void *rho_bh) -> int {
    QJ_TRY(vhat(rho_bh));
    QJ_CK(cudaMemcpyAsync(P->c1, P->c0, nc * P->csz, cudaMemcpyDeviceToDevice, st));
    QJ_TRY(fft3d(P, P->c1, +1, st));
    QJ_TRY(launch_real_part(dbl, P->c1, 1.0, nullptr, 0.0, nullptr, P->V, nc, st));
    QJ_TRY(launch_kick_plain(dbl, psi, P->V, mph * dt_eff / 2.0, nc, st));
    QJ_TRY(accel());
    return launch_gas_kick(dbl, v[0], v[1], v[2], P->ax, P->ay, P->az, dt_eff / 2.0, nc, st);
  };
  if (q.bh_on && q.bh_move) QJ_TRY(bh_kick());
  {
    const void *bh = nullptr;
    QJ_TRY(soft_bh(M_eff, r_soft, bh));
    QJ_TRY(kick(bh));
  }
  // drift (quantum + hydro)
  QJ_TRY(fft3d(P, psi, -1, st));
  QJ_TRY(launch_drift_mul(dbl, psi, ktabs(P), dt_eff, mph, nc, st));
  QJ_TRY(fft3d(P, psi, +1, st));
  QJ_TRY(launch_hydro(dbl, rho, v[0], v[1], v[2], P->gas_prim, n, dx, dt_eff, cs, 0, st,
                      P->tune[9] > 0 ? P->tune[9] : 256, true));
  if (q.bh_on && q.bh_move)
    for (int d = 0; d < 3; ++d) {
      const double x = S.x_bh[d] + dt_eff * S.v_bh[d] * active;
      S.x_bh[d] = x - L * std::floor(x / L);
    }
  // ambient-shell Bondi accretion (:770-800)
  const double active_acc = (S.placed > 0.5 && M_eff > 0.0) ? 1.0 : 0.0;
  D.dMdt = D.dMdt_real = D.cap_ratio = D.r_B = 0.0;
  D.rho_inf = q.rho_gas;
  D.r_acc_eff = std::max(q.r_acc_mult * dx, 2.0 * (G * M_eff / (cs * cs + 1e-30)));
  if (q.bh_on && q.bh_accretion && active_acc > 0.5) {
    QJ_TRY(launch_bondi_ambient(dbl, rho, v[0], v[1], v[2], n, dx, L, S.x_bh, S.v_bh, M_eff, cs, G,
                                dt_eff, q.r_acc_mult, q.lam, q.fmax, q.ann_lo, q.ann_hi, sc + 8, st));
    double o[7];
    QJ_TRY(host(8, 7, o));
    D.dMdt = o[0];
    D.rho_inf = o[1];
    D.r_B = o[2];
    S.M_acc = S.M_acc + o[3];
    D.dMdt_real = o[3] / (dt_eff + 1e-30);
    D.cap_ratio = o[6] > 0.0 ? o[3] / (o[6] + 1e-30) : 0.0;
    D.r_acc_eff = o[4];
  }
  // second kick (:806-830)
  {
    const double M_mid = facc_seed(S.t, S.placed, q) + S.M_acc;
    const void *bh = nullptr;
    QJ_TRY(soft_bh(M_mid, D.r_acc_eff, bh));
    QJ_TRY(kick(bh));
  }
  if (q.bh_on && q.bh_move) QJ_TRY(bh_kick());
  S.t = S.t + dt_eff;
  // black-hole site at the smoothed dark-matter peak, once (:836-860)
  if (S.placed < 0.5 && S.t >= q.bh_inject_t) {
    QJ_TRY(launch_build_rho(dbl, psi, nullptr, nullptr, nullptr, 1.0, 0.0, P->rho_tot, P->c1, nc, st));
    if (q.inject_smooth_on) {
      const double s = std::max(q.inject_smooth_kpc, 1.5 * dx);
      QJ_TRY(fft3d(P, P->c1, -1, st));
      QJ_TRY(launch_kfilter(dbl, P->c1, ktabs(P), 1, s * s, nc, st));
      QJ_TRY(fft3d(P, P->c1, +1, st));
      QJ_TRY(launch_real_part(dbl, P->c1, 1.0, nullptr, 0.0, nullptr, P->rho_tot, nc, st));
    }
    QJ_TRY(launch_argmax(dbl, P->rho_tot, nc, P->facc_part, P->facc_pi, nb, sc + 15, st));
    double idx = 0.0;
    QJ_TRY(host(15, 1, &idx));
    const long long c = (long long)idx;
    const long long ii[3] = {c / ((long long)n * n), (c / n) % n, c % n};
    for (int d = 0; d < 3; ++d) {
      S.x_bh[d] = ((double)ii[d] + 0.5) * dx;
      S.v_bh[d] = 0.0;
    }
    S.placed = 1.0;
  }
  D.M_bh_eff_out = facc_seed(S.t, S.placed, q) + S.M_acc;
  D.dt_eff = dt_eff;
  return 0;
}
}  // namespace

extern "C" {

int qj_fluid_accretion_step(qj_plan *P, void *psi, void *rho, void *vx, void *vy, void *vz,
                            qj_facc_state *state, const qj_facc_params *params, double dt,
                            int nsteps, qj_facc_diag *diag, void *stream) {
  if (!P || !psi || !rho || !vx || !vy || !vz || !state || !params || !(dt > 0) || nsteps < 0) {
    set_error("qj_fluid_accretion_step: bad argument");
    return QJ_ERR_ARG;
  }
  QJ_ONE_BOX(P, "qj_fluid_accretion_step");
  if (!P->dbl) {
    set_error("qj_fluid_accretion_step: needs a PLAIN_F64 plan (the reference runs in float64)");
    return QJ_ERR_ARG;
  }
  if (P->n[0] != P->n[1] || P->n[0] != P->n[2] || P->g.Lx != P->g.Ly || P->g.Lx != P->g.Lz) {
    set_error("qj_fluid_accretion_step: needs a cubic grid and box");
    return QJ_ERR_ARG;
  }
  QJ_TRY(ensure_plain_ws(P));
  QJ_TRY(ensure_gas_ws(P));
  const int nb = 592;
  if (!P->cfl_part) QJ_TRY(dev_alloc_t(P, &P->cfl_part, (size_t)nb));
  if (!P->facc_bh) QJ_TRY(dev_alloc(P, &P->facc_bh, P->ncell * P->rsz));
  if (!P->facc_scal) QJ_TRY(dev_alloc_t(P, &P->facc_scal, 16));
  if (!P->facc_part) QJ_TRY(dev_alloc_t(P, &P->facc_part, (size_t)2 * nb));
  if (!P->facc_pi) QJ_TRY(dev_alloc_t(P, &P->facc_pi, (size_t)nb));
  void *v[3] = {vx, vy, vz};
  qj_facc_diag D;
  std::memset(&D, 0, sizeof(D));
  for (int s = 0; s < nsteps; ++s)
    QJ_TRY(facc_step(P, psi, rho, v, *state, *params, dt, D, (cudaStream_t)stream));
  if (diag) *diag = D;
  return QJ_OK;
}

int qj_plan_get_tuning(const qj_plan *P, int32_t *tune, int n) {
  if (!P || !tune || n < QJ_TUNE_N) {
    set_error("qj_plan_get_tuning: bad argument (n must be >= %d)", QJ_TUNE_N);
    return QJ_ERR_ARG;
  }
  for (int i = 0; i < QJ_TUNE_N; ++i) tune[i] = P->tune[i];
  return QJ_OK;
}

int qj_plan_set_tuning(qj_plan *P, const int32_t *tune, int n) {
  if (!P || !tune || n < QJ_TUNE_N) {
    set_error("qj_plan_set_tuning: bad argument (n must be >= %d)", QJ_TUNE_N);
    return QJ_ERR_ARG;
  }
  for (int i = 0; i < 8; ++i)
    if (tune[i] < 0 || tune[i] > 32) {
      set_error("qj_plan_set_tuning: CTAs per SM of pass %d must be 0..32", i);
      return QJ_ERR_ARG;
    }
  if (tune[8] < -1 || tune[8] > 64 || !(tune[9] == 0 || tune[9] == 64 || tune[9] == 128 ||
                                         tune[9] == 256)) {
    set_error("qj_plan_set_tuning: reserve must be -1..64, hydro block 0/64/128/256");
    return QJ_ERR_ARG;
  }
  if ((tune[QJ_TUNE_RADIX] & ~0x7f7f) != 0 || (tune[QJ_TUNE_TILE] & ~0x7f7f) != 0) {
    set_error("qj_plan_set_tuning: radix plan and tile variant are bit masks over passes 0..6 "
              "(strided) and 8..14 (contiguous)");
    return QJ_ERR_ARG;
  }
  for (int i = 0; i < QJ_TUNE_N; ++i) P->tune[i] = tune[i];
  return QJ_OK;
}

// Coordinate search over the launch tuning of the fused step.  With
// QJ_AUTOTUNE_SHAPES (and an axis of length 128 or 256): first, per pass and
// orientation (strided x / y, contiguous z), the radix plan and tile variant
// (the four combinations).  Then, per pass, the CTAs per SM (1 .. the
// occupancy maximum of its chosen shapes); then the reserved CTA slots.
// Each trial runs probe_steps steps of qj_kdk_step on a scratch copy of the
// state (the caller's arrays are only read) and takes the faster of two
// timings.
int qj_autotune_kdk(qj_plan *P, const void *psi, const void *pos, const void *vel, int n_s,
                    double m_s, double dt, int probe_steps, int flags, void *stream) {
  if (!P || !psi || n_s < 0 || (n_s > 0 && (!pos || !vel)) || probe_steps < 1 ||
      !(dt > 0) || n_s > P->max_particles || (flags & ~QJ_AUTOTUNE_SHAPES) != 0) {
    set_error("qj_autotune_kdk: bad argument");
    return QJ_ERR_ARG;
  }
  if (P->dbl) return QJ_OK;  // the plain path has no persistent passes to tune
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = P->nbox;
  const size_t psi_b = (size_t)nb * P->ncell * sizeof(float2);
  const size_t par_b = (size_t)nb * n_s * 3 * sizeof(float);
  void *s_psi = nullptr, *s_pos = nullptr, *s_vel = nullptr, *s_diag = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = QJ_OK;
  auto cleanup = [&] {
    cudaFree(s_psi);
    cudaFree(s_pos);
    cudaFree(s_vel);
    cudaFree(s_diag);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  };
  cudaError_t e = cudaMalloc(&s_psi, psi_b);
  if (e == cudaSuccess && n_s > 0) e = cudaMalloc(&s_pos, par_b);
  if (e == cudaSuccess && n_s > 0) e = cudaMalloc(&s_vel, par_b);
  if (e == cudaSuccess) e = cudaMalloc(&s_diag, (size_t)nb * 3 * sizeof(double));
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    cleanup();
    return cuda_fail(e, "autotune scratch", __FILE__, __LINE__);
  }
  std::vector<double> diag0((size_t)nb * 3);
  for (int b = 0; b < nb; ++b) {
    diag0[3 * b] = 0.0;
    diag0[3 * b + 1] = 0.0;
    diag0[3 * b + 2] = dt;
  }
  auto trial = [&](float &ms, int reps) -> int {
    float best = 1e30f;
    for (int rep = 0; rep < reps; ++rep) {
      QJ_CK(cudaMemcpyAsync(s_psi, psi, psi_b, cudaMemcpyDeviceToDevice, st));
      if (n_s > 0) {
        QJ_CK(cudaMemcpyAsync(s_pos, pos, par_b, cudaMemcpyDeviceToDevice, st));
        QJ_CK(cudaMemcpyAsync(s_vel, vel, par_b, cudaMemcpyDeviceToDevice, st));
      }
      QJ_CK(cudaMemcpyAsync(s_diag, diag0.data(), diag0.size() * sizeof(double),
                            cudaMemcpyHostToDevice, st));
      QJ_CK(cudaEventRecord(e0, st));
      QJ_TRY(fused_kdk(P, (float2 *)s_psi, (float *)s_pos, (float *)s_vel, n_s, m_s, dt,
                       probe_steps, 0, nullptr, (double *)s_diag, st));
      QJ_CK(cudaEventRecord(e1, st));
      QJ_CK(cudaEventSynchronize(e1));
      float t = 0.f;
      QJ_CK(cudaEventElapsedTime(&t, e0, e1));
      best = std::min(best, t);
    }
    ms = best;
    return 0;
  };
  int saved[QJ_TUNE_N];
  for (int i = 0; i < QJ_TUNE_N; ++i) saved[i] = P->tune[i];
  float best_ms = 0.f;
  if ((rc = trial(best_ms, 2)) == 0 && (rc = trial(best_ms, 2)) == 0) {  // warm-up, then baseline
    bool variants = false;
    for (int ax = 0; ax < 3; ++ax) variants = variants || has_radix_variant(P->n[ax]);
    const int modes[] = {M_FFT_FWD, M_POISSON, M_IFFT2, M_KICK, M_DRIFT, M_DRIFT_DENSITY};
    if ((flags & QJ_AUTOTUNE_SHAPES) && variants) {
      // per pass and orientation, each radix plan / tile combination at the
      // current CTA counts (a combination's first trial also sets up its
      // kernels: the second one, the best of three runs, counts).  A single
      // pass changes the step by a fraction of a percent, so a combination
      // is kept when it is 0.3 % faster.  The y-only passes have no
      // contiguous form.
      const int shapes0[2] = {P->tune[QJ_TUNE_RADIX], P->tune[QJ_TUNE_TILE]};
      float shape_ms = 0.f;
      rc = trial(shape_ms, 3);
      // A combination's worth is timed on its own pass: CUDA events around
      // each launch of the pass along the orientation in question, averaged
      // over a probe run, best of two runs; kept when 1 % faster.  (With the
      // caller's own pass profiling on, the whole step is timed instead.)
      const bool by_pass = !prof_on();
      auto pass_trial = [&](int m, bool contig, float &ms) -> int {
        ms = INFINITY;
        for (int rep = 0; rep < 2; ++rep) {
          prof_session(true);
          float step_ms = 0.f, t = 0.f;
          int r = trial(step_ms, 1);
          if (r == 0) r = prof_bucket_mean(m + (contig ? kProfZ : 0), t);
          prof_session(false);
          if (r) return r;
          ms = std::min(ms, t);
        }
        return 0;
      };
      for (int mb = 0; mb < 2 * 6 && rc == 0; ++mb) {
        const int m = modes[mb % 6];
        const bool contig = mb >= 6;
        if (contig && (m == M_FFT_FWD || m == M_IFFT2)) continue;
        const int bit = 1 << (m + (contig ? 8 : 0));
        auto shape_now = [&] {
          return ((P->tune[QJ_TUNE_RADIX] & bit) ? 1 : 0) | ((P->tune[QJ_TUNE_TILE] & bit) ? 2 : 0);
        };
        auto set_shape = [&](int v) {
          P->tune[QJ_TUNE_RADIX] = (P->tune[QJ_TUNE_RADIX] & ~bit) | ((v & 1) ? bit : 0);
          P->tune[QJ_TUNE_TILE] = (P->tune[QJ_TUNE_TILE] & ~bit) | ((v & 2) ? bit : 0);
        };
        const int cur = shape_now();
        int best_v = cur;
        if (by_pass) {
          float best_p = INFINITY;
          rc = pass_trial(m, contig, best_p);
          for (int v = 0; v < 4 && rc == 0 && std::isfinite(best_p); ++v) {
            if (v == cur) continue;
            set_shape(v);
            float t = 0.f, u = 0.f;
            if ((rc = trial(u, 1)) == 0 && (rc = pass_trial(m, contig, t)) == 0 &&
                t < 0.99f * best_p) {
              best_p = t;
              best_v = v;
            }
          }
        } else {
          for (int v = 0; v < 4 && rc == 0; ++v) {
            if (v == cur) continue;
            set_shape(v);
            float t = 0.f;
            if ((rc = trial(t, 1)) == 0 && (rc = trial(t, 3)) == 0 && t < 0.997f * shape_ms) {
              shape_ms = t;
              best_v = v;
            }
          }
        }
        set_shape(best_v);
      }
      // the chosen shapes against the starting ones, in alternating longer
      // runs: picks made by whole-step timing must be 0.3 % faster (so that
      // picks made on noise do not add up), picks made on their own passes
      // must not make the step slower (by more than 0.1 %)
      const int chosen[2] = {P->tune[QJ_TUNE_RADIX], P->tune[QJ_TUNE_TILE]};
      if (rc == 0 && (chosen[0] != shapes0[0] || chosen[1] != shapes0[1])) {
        float t_new = 1e30f, t_old = 1e30f;
        for (int r = 0; r < 3 && rc == 0; ++r) {
          float t = 0.f;
          P->tune[QJ_TUNE_RADIX] = shapes0[0];
          P->tune[QJ_TUNE_TILE] = shapes0[1];
          if ((rc = trial(t, 2)) == 0) t_old = std::min(t_old, t);
          P->tune[QJ_TUNE_RADIX] = chosen[0];
          P->tune[QJ_TUNE_TILE] = chosen[1];
          if (rc == 0 && (rc = trial(t, 2)) == 0) t_new = std::min(t_new, t);
        }
        const bool keep = t_new < (by_pass ? 1.001f : 0.997f) * t_old;
        P->tune[QJ_TUNE_RADIX] = keep ? chosen[0] : shapes0[0];
        P->tune[QJ_TUNE_TILE] = keep ? chosen[1] : shapes0[1];
      }
      if (rc == 0) rc = trial(best_ms, 2);  // the CTA search's baseline
    }
    for (int m : modes) {
      // occupancy of the pass, in the chosen shape, over both orientations it runs in
      int kmax = 0;
      for (int ax = 0; ax < 3; ++ax)
        kmax = std::max(kmax, fused_max_ctas_per_sm(m, P->n[ax], ax == 2,
                                                    shape_of(P->n[ax], P->tune, m, ax == 2)));
      const int cur = P->tune[m];
      int best_k = cur;
      for (int k = 1; k <= kmax && rc == 0; ++k) {
        if (k == cur || (cur == 0 && k == kmax)) continue;
        P->tune[m] = k;
        float t = 0.f;
        if ((rc = trial(t, 2)) == 0 && t < 0.99f * best_ms) {
          best_ms = t;
          best_k = k;
        }
      }
      P->tune[m] = best_k;
    }
    const int cur_r = P->tune[8];
    int best_r = cur_r;
    for (int r : {0, 2, 4, 8}) {
      if (rc) break;
      if (r == (cur_r < 0 ? 2 : cur_r)) continue;
      P->tune[8] = r;
      float t = 0.f;
      if ((rc = trial(t, 2)) == 0 && t < 0.99f * best_ms) {
        best_ms = t;
        best_r = r;
      }
    }
    P->tune[8] = best_r;
  }
  if (rc)
    for (int i = 0; i < QJ_TUNE_N; ++i) P->tune[i] = saved[i];
  const cudaError_t se = cudaStreamSynchronize(st);
  cleanup();
  if (rc) return rc;
  QJ_CK(se);
  return QJ_OK;
}

int qj_plan_status(qj_plan *P) {
  if (!P) {
    set_error("qj_plan_status: bad argument");
    return QJ_ERR_ARG;
  }
  QJ_CK(cudaDeviceSynchronize());
  unsigned w = 0;
  QJ_CK(cudaMemcpy(&w, P->err, sizeof(w), cudaMemcpyDeviceToHost));
  if (w == 0) return QJ_OK;
  QJ_CK(cudaMemset(P->err, 0, sizeof(unsigned)));
  set_error("a fused pass gave up waiting for a tile copy (bounded wait); its results are invalid");
  return QJ_ERR_TIMEOUT;
}

int qj_plan_selftest_wait(qj_plan *P, int64_t limit_ns, void *stream) {
  if (!P || limit_ns < 1000000 || limit_ns > 2000000000) {
    set_error("qj_plan_selftest_wait: bad argument (limit_ns in [1e6, 2e9])");
    return QJ_ERR_ARG;
  }
  return launch_selftest_wait(P->err, (long long)limit_ns, (cudaStream_t)stream);
}

int qj_selftest_sincos(const double *theta, float *sin_cos, int n, void *stream) {
  if (n < 0 || !theta || !sin_cos) {
    set_error("qj_selftest_sincos: bad argument (n >= 0, theta and sin_cos non-null)");
    return QJ_ERR_ARG;
  }
  if (n == 0) return QJ_OK;
  return launch_selftest_sincos(theta, reinterpret_cast<float2 *>(sin_cos), n,
                                (cudaStream_t)stream);
}

int64_t qj_launch_count(void) { return (int64_t)g_launches.load(); }

int qj_profile_enable(int on) {
  Prof &p = prof();
  std::lock_guard<std::mutex> g(p.mu);
  for (auto &m : p.marks) {
    p.pool.push_back(m.a);
    p.pool.push_back(m.b);
  }
  p.marks.clear();
  p.on = on != 0;
  return QJ_OK;
}

int qj_profile_read(double *ms, int64_t *count, int nbuckets) {
  Prof &p = prof();
  std::lock_guard<std::mutex> g(p.mu);
  for (int i = 0; i < nbuckets; ++i) {
    ms[i] = 0.0;
    count[i] = 0;
  }
  for (auto &m : p.marks) {
    cudaError_t e = cudaEventSynchronize(m.b);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventSynchronize", __FILE__, __LINE__);
    float t = 0.f;
    e = cudaEventElapsedTime(&t, m.a, m.b);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventElapsedTime", __FILE__, __LINE__);
    if (m.bucket >= 0 && m.bucket < nbuckets) {
      ms[m.bucket] += t;
      count[m.bucket] += 1;
    }
  }
  return QJ_OK;
}

int qj_fft3d(qj_plan *P, const void *in, void *out, int direction, void *stream) {
  QJ_ONE_BOX(P, "qj_fft3d");
  if (!P || !in || !out || (direction != -1 && direction != 1)) {
    set_error("qj_fft3d: bad argument");
    return QJ_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (in != out) QJ_CK(cudaMemcpyAsync(out, in, P->ncell * P->csz, cudaMemcpyDeviceToDevice, st));
  return fft3d(P, out, direction, st);
}

int qj_get_potential(qj_plan *P, const void *rho, void *V, int self_interaction, void *stream) {
  QJ_ONE_BOX(P, "qj_get_potential");
  if (!P || !rho || !V) {
    set_error("qj_get_potential: null argument");
    return QJ_ERR_ARG;
  }
  QJ_TRY(ensure_plain_ws(P));
  return plain_potential(P, nullptr, nullptr, rho, V, self_interaction, nullptr,
                         (cudaStream_t)stream);
}

int qj_bin_stars(qj_plan *P, const void *pos, int n, double m_s, const void *masses, void *rho_s,
                 void *stream) {
  QJ_ONE_BOX(P, "qj_bin_stars");
  if (!P || !rho_s || (n > 0 && !pos) || n < 0 || n > P->max_particles) {
    set_error("qj_bin_stars: bad argument (n=%d, max_particles=%d)", n, P ? P->max_particles : 0);
    return QJ_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (P->dbl) return plain_bin(P, pos, n, m_s, masses, rho_s, st);
  // single precision: the pencil-bucket deposit of the fused step
  FusedArgs a = fused_args(P, 2, M_DEPOSIT);
  a.rho_out = (float *)rho_s;
  if (n > 0) {
    QJ_TRY(launch_stars_prepare(pos, n, masses, m_s, geom(P), 2, P->sb, st));
    QJ_TRY(launch_bucket_sort(n, n_pencils(P, 2), bucket_nv(P, 2), P->sb, st));
    set_stars(a, P);
  }
  return launch_fused(M_DEPOSIT, P->n[2], a, st);
}

int qj_get_acceleration(qj_plan *P, const void *pos, int n, const void *rho, void *acc,
                        double *a_max, void *stream) {
  QJ_ONE_BOX(P, "qj_get_acceleration");
  if (!P || !rho || (n > 0 && (!pos || !acc)) || n < 0 || n > P->max_particles) {
    set_error("qj_get_acceleration: bad argument (n=%d, max_particles=%d)", n,
              P ? P->max_particles : 0);
    return QJ_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  QJ_TRY(ensure_plain_ws(P));
  QJ_CK(cudaMemsetAsync(P->tmp_scalar, 0, 8, st));
  QJ_TRY(plain_accel(P, rho, P->tmp_scalar, st));
  if (n > 0) QJ_TRY(launch_gather_dense(P->dbl, pos, n, geom(P), P->ax, P->ay, P->az, acc, st));
  if (a_max) QJ_TRY(launch_bits_to_double(P->dbl, P->tmp_scalar, a_max, st));
  return QJ_OK;
}

// quantum-cosmo.py:149-162: dt from a 1000-point midpoint quadrature of
// 1 / adot, adot = H0 sqrt(omega_m / a + omega_l a^2), in float64.
static double cosmo_dt(double a, double da, double H0, double om, double ol) {
  const int n = 1000;
  const double h = 1.0 / n;
  auto mean_inv = [&](double A) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) {
      const double at = A * (0.5 * h + i * h);
      s += 1.0 / (H0 * std::sqrt(om / at + ol * at * at));
    }
    return s / n;
  };
  const double t = mean_inv(a) * (a - 0.0);
  return mean_inv(a + da) * ((a + da) - 0.0) - t;
}

int qj_kdk_cosmo(qj_plan *P, void *psi, double *a_io, double da, double H0, double omega_m,
                 double omega_l, int nsteps, void *stream) {
  QJ_ONE_BOX(P, "qj_kdk_cosmo");
  if (!P || !psi || !a_io || nsteps < 0 || !(da > 0) || !(*a_io > 0)) {
    set_error("qj_kdk_cosmo: bad argument");
    return QJ_ERR_ARG;
  }
  if (nsteps == 0) return QJ_OK;
  StepCoefs sc;
  double a = *a_io;
  for (int n = 0; n < nsteps; ++n) {
    // quantum-cosmo.py:173-176
    const double kin_fac = 0.5 * (std::pow(a, -2.0) + std::pow(a + da, -2.0));
    const double pot_fac = 0.5 * (1.0 / a + 1.0 / (a + da));
    const double dt = cosmo_dt(a, da, H0, omega_m, omega_l);
    sc.kick_half.push_back(P->ph.m_per_hbar * dt * pot_fac / 2.0);
    sc.drift.push_back(dt * kin_fac);
    a += da;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (!P->tmp_diag) QJ_TRY(dev_alloc(P, &P->tmp_diag, 3 * sizeof(double)));
  int rc = P->dbl ? plain_kdk(P, psi, nullptr, nullptr, 0, 0.0, 1.0, nsteps, 0, nullptr,
                              (double *)P->tmp_diag, st, &sc)
                  : fused_kdk(P, (float2 *)psi, nullptr, nullptr, 0, 0.0, 1.0, nsteps, 0, nullptr,
                              (double *)P->tmp_diag, st, &sc);
  if (rc == 0) *a_io = a;
  return rc;
}

int qj_kdk_gas_bh_step(qj_plan *P, void *psi, void *rho, void *vx, void *vy, void *vz, void *m_bh,
                       void *pos, void *vel, int n_bh, double dt, int nsteps, double sigma_v,
                       int dm_accretion, double bondi_r_acc_mult, double *t_io, void *stream) {
  QJ_ONE_BOX(P, "qj_kdk_gas_bh_step");
  if (!P || !psi || nsteps < 0 || n_bh < 0 || (n_bh > 0 && (!m_bh || !pos || !vel)) ||
      (rho && (!vx || !vy || !vz)) || !(dt > 0)) {
    set_error("qj_kdk_gas_bh_step: bad argument");
    return QJ_ERR_ARG;
  }
  if (P->n[0] != P->n[1] || P->n[0] != P->n[2] || P->g.Lx != P->g.Ly || P->g.Lx != P->g.Lz) {
    set_error("qj_kdk_gas_bh_step: the gas / black-hole step needs a cubic grid and box");
    return QJ_ERR_ARG;
  }
  if (n_bh > P->max_particles) {
    set_error("qj_kdk_gas_bh_step: n_bh=%d exceeds max_particles=%d", n_bh, P->max_particles);
    return QJ_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  QJ_TRY(ensure_gas_ws(P));
  if (P->dbl) QJ_TRY(ensure_plain_ws(P));
  GasArgs g;
  g.psi = psi;
  g.rho = rho;
  g.v[0] = vx;
  g.v[1] = vy;
  g.v[2] = vz;
  g.m_bh = m_bh;
  g.pos = pos;
  g.vel = vel;
  g.n_bh = n_bh;
  g.dt = dt;
  g.sigma_v = sigma_v;
  g.dm_accretion = dm_accretion;
  g.bondi = bondi_r_acc_mult;
  for (int s = 0; s < nsteps; ++s)
    QJ_TRY(P->dbl ? plain_gas_step(P, g, st) : fused_gas_step(P, g, st, s == 0, s == nsteps - 1));
  if (t_io) *t_io += nsteps * dt;
  return QJ_OK;
}

int qj_kdk_forward_ckpt(qj_plan *P, void *psi, int nsteps, int K, void *ckpt, double dt,
                        int self_interaction, const void *v_ext, const void *rho_s,
                        void *stream) {
  QJ_ONE_BOX(P, "qj_kdk_forward_ckpt");
  if (!P || !psi || !ckpt || nsteps <= 0 || K <= 0 || !(dt > 0)) {
    set_error("qj_kdk_forward_ckpt: bad argument");
    return QJ_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const size_t fb = P->ncell * P->csz;
  for (int s0 = 0, seg = 0; s0 < nsteps; s0 += K, ++seg) {
    QJ_CK(cudaMemcpyAsync((char *)ckpt + (size_t)seg * fb, psi, fb, cudaMemcpyDeviceToDevice, st));
    QJ_TRY(kdk_chunk(P, psi, std::min(K, nsteps - s0), dt, self_interaction, v_ext, rho_s, st,
                     nullptr));
  }
  return QJ_OK;
}

int qj_kdk_adjoint(qj_plan *P, const void *ckpt, void *g, int nsteps, int K, double dt,
                   int self_interaction, const void *v_ext, const void *rho_s, void *stream) {
  QJ_ONE_BOX(P, "qj_kdk_adjoint");
  if (!P || !ckpt || !g || nsteps <= 0 || K <= 0 || !(dt > 0)) {
    set_error("qj_kdk_adjoint: bad argument");
    return QJ_ERR_ARG;
  }
  return adjoint_sweep(P, ckpt, g, nsteps, K, dt, self_interaction, v_ext, rho_s,
                       (cudaStream_t)stream);
}

int qj_kdk_step(qj_plan *P, void *psi, void *pos, void *vel, int n_s, double m_s, double dt,
                int nsteps, int self_interaction, const void *v_ext, qj_diag *diag,
                void *stream) {
  if (!P || !psi || !diag || nsteps < 0 || n_s < 0 || (n_s > 0 && (!pos || !vel))) {
    set_error("qj_kdk_step: bad argument");
    return QJ_ERR_ARG;
  }
  if (n_s > P->max_particles) {
    set_error("qj_kdk_step: n_s=%d exceeds the plan's max_particles=%d", n_s, P->max_particles);
    return QJ_ERR_ARG;
  }
  if (!(dt > 0) || !std::isfinite(dt)) {
    set_error("qj_kdk_step: dt must be positive and finite");
    return QJ_ERR_ARG;
  }
  if (nsteps == 0) return QJ_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (P->dbl)
    return plain_kdk(P, psi, pos, vel, n_s, m_s, dt, nsteps, self_interaction, v_ext,
                     (double *)diag, st);
  return fused_kdk(P, (float2 *)psi, (float *)pos, (float *)vel, n_s, m_s, dt, nsteps,
                   self_interaction, (const float *)v_ext, (double *)diag, st);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Ensembles: several batched plans (one per box size) stepped together, with
// the step body captured once into a CUDA graph and replayed.  By default each
// plan steps on its own stream.  With merge on and the plans' sizes distinct
// cubes of 64, 96 and 128 (the sizes that share a CTA shape), every fused pass
// is instead one launch for all plans' boxes (launch_fused_ens); that gives
// the same bits but measured slower on the 32-box mix (1.07 vs 0.95 ms per
// step): each pass then ends for all sizes together, while the streams let one
// size's pass overlap another size's next one.
// ---------------------------------------------------------------------------
struct qj_ensemble {
  std::vector<qj_plan *> plans;
  bool merge = false;  // use ensemble launches when the plans allow them
  std::vector<cudaStream_t> streams;
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr, done = nullptr, caller = nullptr;
  std::vector<cudaEvent_t> joins;
  cudaGraphExec_t exec = nullptr;
  std::vector<const void *> key;  // pointers and sizes the graph was captured with
  // tile counters of the ensemble launches: one per box for each launch of a
  // merged body (ens_counters)
  unsigned *ctr = nullptr;
  size_t ctr_n = 0;
};

namespace {

struct EnsArgs {
  void *const *psi;
  void *const *pos;
  void *const *vel;
  const int *n_s;
  const double *m_s;
  const double *dt;
  qj_diag *const *diag;
};

// The plans fit ensemble launches: at most one plan per size class, each a
// cube of a class size, no shape variants in their tuning.
bool ens_mergeable(const qj_ensemble *E) {
  if (!E->merge || E->plans.empty() || (int)E->plans.size() > kEnsClasses) return false;
  bool used[kEnsClasses] = {false, false, false};
  for (const qj_plan *P : E->plans) {
    const int s = ens_slot(P->n[0]);
    if (s < 0 || used[s] || P->n[1] != P->n[0] || P->n[2] != P->n[0] ||
        P->tune[QJ_TUNE_RADIX] != 0 || P->tune[QJ_TUNE_TILE] != 0)
      return false;
    used[s] = true;
  }
  return true;
}

// Boxes of all plans, and the fused launches of an m-step merged body: the
// first density build, four potential passes for each of the m + 1 kicks and
// two drift passes for each step.
int ens_boxes(const qj_ensemble *E) {
  int b = 0;
  for (const qj_plan *P : E->plans) b += P->nbox;
  return b;
}
size_t ens_launches(int m) { return 6 * (size_t)m + 5; }

// Tile counters for merged bodies of up to m steps (allocated here, never
// during a stream capture: qj_ensemble_step calls this before it captures).
int ens_counters(qj_ensemble *E, int m) {
  const size_t need = ens_launches(m) * (size_t)ens_boxes(E);
  if (E->ctr_n >= need) return 0;
  if (E->ctr) {
    QJ_CK(cudaFree(E->ctr));
    E->ctr = nullptr;
    E->ctr_n = 0;
  }
  QJ_CK(cudaMalloc(&E->ctr, need * sizeof(unsigned)));
  E->ctr_n = need;
  return 0;
}

// m steps of every plan with one launch per fused pass for all of them: the
// phases of fused_kdk (KdkRun), each run for all plans before the next.  The
// plans' star updates and sorts run on their own side streams, forked after
// the kick and joined before the drift + density pass, as in fused_kdk.
// Each launch claims tiles from its own counters, all zeroed by one memset.
int ensemble_merged_body(qj_ensemble *E, const EnsArgs &a, int m) {
  const int np = (int)E->plans.size();
  cudaStream_t st = E->origin;
  const int boxes = ens_boxes(E);
  const size_t nctr = ens_launches(m) * (size_t)boxes;
  if (E->ctr_n < nctr) {
    set_error("internal: %zu ensemble tile counters for %zu", E->ctr_n, nctr);
    return QJ_ERR_ARG;
  }
  QJ_CK(cudaMemsetAsync(E->ctr, 0, nctr * sizeof(unsigned), st));
  size_t launch = 0;
  std::vector<KdkRun> runs;
  int reserve = 0;
  for (int i = 0; i < np; ++i) {
    qj_plan *P = E->plans[i];
    runs.push_back(KdkRun{P, (float2 *)a.psi[i], (float *)(a.n_s[i] ? a.pos[i] : nullptr),
                          (float *)(a.n_s[i] ? a.vel[i] : nullptr), a.n_s[i], a.m_s[i], a.dt[i], m,
                          0, nullptr, (double *)a.diag[i], nullptr, nullptr, nullptr, nullptr});
    // each plan with stars keeps its own free CTA slots for its side stream
    if (a.n_s[i] > 0) reserve += P->tune[8] >= 0 ? P->tune[8] : 2;
  }
  FusedArgs fa[kEnsClasses];
  int fn[kEnsClasses];
  auto phase = [&](auto &&get) -> int {
    int mode = 0;
    for (int i = 0; i < np; ++i) {
      const Phase ph = get(runs[i]);
      mode = ph.mode;
      fa[i] = ph.a;
      fn[i] = runs[i].P->n[ph.axis];
    }
    if (launch >= ens_launches(m)) {
      set_error("internal: more ensemble launches than counted");
      return QJ_ERR_ARG;
    }
    unsigned *ctr = E->ctr + launch++ * (size_t)boxes;
    return launch_fused_ens(mode, np, fa, fn, reserve, ctr, boxes, st);
  };
  for (KdkRun &R : runs) QJ_TRY(R.begin(st));
  QJ_TRY(phase([](KdkRun &R) { return R.density(); }));
  for (int k = 0; k <= m; ++k) {
    for (KdkRun &R : runs) QJ_TRY(R.step_begin(k, st));
    QJ_TRY(phase([](KdkRun &R) { return R.fft_fwd(); }));
    QJ_TRY(phase([k](KdkRun &R) { return R.poisson(k); }));
    QJ_TRY(phase([](KdkRun &R) { return R.ifft2(); }));
    QJ_TRY(phase([k](KdkRun &R) { return R.kick(k); }));
    for (KdkRun &R : runs) QJ_TRY(R.stars(k, st));
    if (k == m) break;
    QJ_TRY(phase([](KdkRun &R) { return R.drift(); }));
    for (KdkRun &R : runs) QJ_TRY(R.join(st));
    QJ_TRY(phase([](KdkRun &R) { return R.drift_density(); }));
    for (KdkRun &R : runs) QJ_TRY(R.step_end(k, st));
  }
  for (KdkRun &R : runs) QJ_TRY(R.end(st));
  return 0;
}

int ensemble_body(qj_ensemble *E, const EnsArgs &a, int m) {
  if (ens_mergeable(E)) return ensemble_merged_body(E, a, m);
  QJ_CK(cudaEventRecord(E->fork, E->origin));
  for (size_t i = 0; i < E->plans.size(); ++i) {
    QJ_CK(cudaStreamWaitEvent(E->streams[i], E->fork, 0));
    QJ_TRY(fused_kdk(E->plans[i], (float2 *)a.psi[i], (float *)a.pos[i], (float *)a.vel[i],
                     a.n_s[i], a.m_s[i], a.dt[i], m, 0, nullptr, (double *)a.diag[i],
                     E->streams[i]));
    QJ_CK(cudaEventRecord(E->joins[i], E->streams[i]));
    QJ_CK(cudaStreamWaitEvent(E->origin, E->joins[i], 0));
  }
  return 0;
}

}  // namespace

extern "C" {

int qj_ensemble_create(qj_ensemble **ens, qj_plan *const *plans, int nplans) {
  if (!ens || !plans || nplans <= 0) {
    set_error("qj_ensemble_create: bad argument");
    return QJ_ERR_ARG;
  }
  *ens = nullptr;
  for (int i = 0; i < nplans; ++i) {
    if (!plans[i] || plans[i]->dbl) {
      set_error("qj_ensemble_create: plan %d is null or not QJ_FUSED_F32", i);
      return QJ_ERR_ARG;
    }
  }
  qj_ensemble *E = new qj_ensemble();
  E->plans.assign(plans, plans + nplans);
  cudaError_t e = cudaStreamCreateWithFlags(&E->origin, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&E->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&E->done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&E->caller, cudaEventDisableTiming);
  for (int i = 0; i < nplans && e == cudaSuccess; ++i) {
    cudaStream_t s = nullptr;
    cudaEvent_t j = nullptr;
    e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&j, cudaEventDisableTiming);
    E->streams.push_back(s);
    E->joins.push_back(j);
  }
  if (e != cudaSuccess) {
    qj_ensemble_destroy(E);
    return cuda_fail(e, "qj_ensemble_create", __FILE__, __LINE__);
  }
  *ens = E;
  return QJ_OK;
}

int qj_ensemble_destroy(qj_ensemble *E) {
  if (!E) return QJ_OK;
  if (E->origin) cudaStreamSynchronize(E->origin);
  if (E->exec) cudaGraphExecDestroy(E->exec);
  if (E->ctr) cudaFree(E->ctr);
  for (cudaStream_t s : E->streams)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t j : E->joins)
    if (j) cudaEventDestroy(j);
  if (E->fork) cudaEventDestroy(E->fork);
  if (E->done) cudaEventDestroy(E->done);
  if (E->caller) cudaEventDestroy(E->caller);
  if (E->origin) cudaStreamDestroy(E->origin);
  delete E;
  return QJ_OK;
}

int qj_ensemble_set_merge(qj_ensemble *E, int on) {
  if (!E) {
    set_error("qj_ensemble_set_merge: bad argument");
    return QJ_ERR_ARG;
  }
  E->merge = on != 0;
  return QJ_OK;
}

int qj_ensemble_merged(const qj_ensemble *E) {
  if (!E) {
    set_error("qj_ensemble_merged: bad argument");
    return QJ_ERR_ARG;
  }
  return ens_mergeable(E) ? 1 : 0;
}

int qj_ensemble_step(qj_ensemble *E, void *const *psi, void *const *pos, void *const *vel,
                     const int *n_s, const double *m_s, const double *dt, qj_diag *const *diag,
                     int nsteps, int chunk, int use_graph, void *stream) {
  if (!E || !psi || !n_s || !m_s || !dt || !diag || nsteps < 0 || chunk <= 0) {
    set_error("qj_ensemble_step: bad argument");
    return QJ_ERR_ARG;
  }
  const size_t np = E->plans.size();
  for (size_t i = 0; i < np; ++i) {
    if (!psi[i] || !diag[i] || n_s[i] < 0 || n_s[i] > E->plans[i]->max_particles ||
        (n_s[i] > 0 && (!pos || !vel || !pos[i] || !vel[i])) || !(dt[i] > 0)) {
      set_error("qj_ensemble_step: bad arguments for plan %d", (int)i);
      return QJ_ERR_ARG;
    }
  }
  if (nsteps == 0) return QJ_OK;
  EnsArgs a{psi, pos, vel, n_s, m_s, dt, diag};
  cudaStream_t st = (cudaStream_t)stream;
  QJ_CK(cudaEventRecord(E->caller, st));
  QJ_CK(cudaStreamWaitEvent(E->origin, E->caller, 0));
  const int full = nsteps / chunk, rem = nsteps % chunk;
  if (ens_mergeable(E)) QJ_TRY(ens_counters(E, std::max(full > 0 ? chunk : 0, rem)));
  if (use_graph && full > 0) {
    std::vector<const void *> key;
    key.push_back((const void *)(intptr_t)(ens_mergeable(E) ? 1 : 0));
    key.push_back(E->ctr);  // a graph of merged launches holds its counters
    for (size_t i = 0; i < np; ++i) {
      key.push_back(psi[i]);
      key.push_back(n_s[i] ? pos[i] : nullptr);
      key.push_back(n_s[i] ? vel[i] : nullptr);
      key.push_back(diag[i]);
      key.push_back((const void *)(intptr_t)n_s[i]);
      key.push_back((const void *)(intptr_t)chunk);
      long long mb, db;
      std::memcpy(&mb, &m_s[i], 8);
      std::memcpy(&db, &dt[i], 8);
      key.push_back((const void *)(intptr_t)mb);
      key.push_back((const void *)(intptr_t)db);
    }
    if (!E->exec || key != E->key) {
      if (E->exec) {
        QJ_CK(cudaGraphExecDestroy(E->exec));
        E->exec = nullptr;
      }
      cudaGraph_t g = nullptr;
      QJ_CK(cudaStreamBeginCapture(E->origin, cudaStreamCaptureModeThreadLocal));
      const int rc = ensemble_body(E, a, chunk);
      cudaError_t ce = cudaStreamEndCapture(E->origin, &g);
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      QJ_CK(ce);
      ce = cudaGraphInstantiate(&E->exec, g, 0);
      cudaGraphDestroy(g);
      QJ_CK(ce);
      E->key = key;
    }
    for (int c = 0; c < full; ++c) QJ_CK(cudaGraphLaunch(E->exec, E->origin));
  } else {
    for (int c = 0; c < full; ++c) QJ_TRY(ensemble_body(E, a, chunk));
  }
  if (rem) QJ_TRY(ensemble_body(E, a, rem));
  QJ_CK(cudaEventRecord(E->done, E->origin));
  QJ_CK(cudaStreamWaitEvent(st, E->done, 0));
  return QJ_OK;
}

}  // extern "C"
