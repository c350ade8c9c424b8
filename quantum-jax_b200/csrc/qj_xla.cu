// XLA custom-call targets: the JAX binding of the step and of get_potential.
//
// The reference calls its step as a jitted Python function inside
// jax.lax.fori_loop(0, nt_sub, update, ...) (quantum-stars.py:454) and its
// Poisson solve as get_potential (quantum-stars.py:189-193).  Inside a jitted
// JAX program those become XLA custom calls to the targets below, which run
// libqj's kernels on XLA's own stream.
//
// ABI: XLA's GPU custom-call convention, status-returning form (custom_call
// api_version 2; registered with jax.ffi.register_ffi_target(...,
// api_version=0)):
//   void target(cudaStream_t stream, void **buffers, const char *opaque,
//               size_t opaque_len, XlaCustomCallStatus *status)
// buffers holds the operands' device pointers, then the results'.  opaque is
// the custom call's backend_config: a packed descriptor (include/qj.h).
// No jaxlib header or library is needed to build this file.
//
// Plans (device tables and workspace) are created on the first call of a
// configuration on a device and cached until qj_xla_release_plans(); make
// that first call outside stream capture (XLA's command buffers capture
// custom calls only after a first, eager run in the usual set-up).
// get_potential on grids of at most 64^3 cells (16 / 32 / 64 per axis) uses
// the allocation-free entry point and creates no plan.
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "../../include/qj.h"
#include "qj_internal.h"

namespace qj {
namespace {

std::mutex g_xla_mu;
qj_xla_status_fn g_status_fn = nullptr;
std::atomic<int> g_last_status{0};

struct PlanKey {
  int dev, nx, ny, nz, n_s;
  double Lx, Ly, Lz;
  bool operator<(const PlanKey &o) const {
    return std::tie(dev, nx, ny, nz, n_s, Lx, Ly, Lz) <
           std::tie(o.dev, o.nx, o.ny, o.nz, o.n_s, o.Lx, o.Ly, o.Lz);
  }
};
std::map<PlanKey, qj_plan *> g_plans;

// The cached single-precision plan of (current device, grid, n_s) with the
// given constants.
int cached_plan(const qj_grid &g, const qj_phys &ph, int n_s, qj_plan **out) {
  int dev = 0;
  QJ_CK(cudaGetDevice(&dev));
  const PlanKey k{dev, g.nx, g.ny, g.nz, n_s, g.Lx, g.Ly, g.Lz};
  std::lock_guard<std::mutex> lock(g_xla_mu);
  auto it = g_plans.find(k);
  qj_plan *P = nullptr;
  if (it == g_plans.end()) {
    const int rc = qj_plan_create(&P, &g, &ph, QJ_FUSED_F32, n_s > 0 ? n_s : 1);
    if (rc) return rc;
    g_plans[k] = P;
  } else {
    P = it->second;
  }
  *out = P;
  return qj_plan_set_phys(P, &ph);
}

// Report rc of a target to XLA (when a status function and status are
// given) and to qj_xla_last_status.
void finish(void *status, int rc) {
  g_last_status.store(rc);
  if (rc == QJ_OK || !status) return;
  qj_xla_status_fn fn = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_xla_mu);
    fn = g_status_fn;
  }
  if (fn) {
    const char *msg = qj_last_error();
    fn(status, msg, std::strlen(msg));
  }
}

// Copy an operand into its result buffer when XLA did not alias them, so the
// in-place entry points can work on the result.
int into_result(const void *in, void *out, size_t bytes, cudaStream_t st) {
  if (bytes == 0 || in == out) return 0;
  if (!in || !out) {
    set_error("XLA target: null buffer");
    return QJ_ERR_ARG;
  }
  QJ_CK(cudaMemcpyAsync(out, in, bytes, cudaMemcpyDeviceToDevice, st));
  return 0;
}

int kdk_target(cudaStream_t st, void **buffers, const char *opaque, size_t len) {
  qj_xla_kdk_desc d;
  if (!opaque || len != sizeof(d)) {
    set_error("qj_xla_kdk_step_f32: descriptor of %zu bytes, expected %zu", opaque ? len : 0,
              sizeof(d));
    return QJ_ERR_ARG;
  }
  std::memcpy(&d, opaque, sizeof(d));
  if (d.version != QJ_XLA_DESC_VERSION || d.n_s < 0 || d.nsteps < 0) {
    set_error("qj_xla_kdk_step_f32: bad descriptor (version %d, n_s %d, nsteps %d)", d.version,
              d.n_s, d.nsteps);
    return QJ_ERR_ARG;
  }
  if (!buffers) {
    set_error("qj_xla_kdk_step_f32: null buffer array");
    return QJ_ERR_ARG;
  }
  const size_t ncell = (size_t)d.grid.nx * d.grid.ny * d.grid.nz;
  const int nin = 4 + (d.has_v_ext ? 1 : 0);
  void *psi = buffers[nin], *pos = buffers[nin + 1], *vel = buffers[nin + 2];
  void *diag = buffers[nin + 3];
  const size_t pbytes = (size_t)d.n_s * 3 * sizeof(float);
  int rc;
  if ((rc = into_result(buffers[0], psi, ncell * sizeof(float2), st))) return rc;
  if ((rc = into_result(buffers[1], pos, pbytes, st))) return rc;
  if ((rc = into_result(buffers[2], vel, pbytes, st))) return rc;
  if ((rc = into_result(buffers[3], diag, sizeof(qj_diag), st))) return rc;
  qj_plan *P = nullptr;
  if ((rc = cached_plan(d.grid, d.phys, d.n_s, &P))) return rc;
  return qj_kdk_step(P, psi, d.n_s ? pos : nullptr, d.n_s ? vel : nullptr, d.n_s, d.m_s, d.dt,
                     d.nsteps, d.self_interaction, d.has_v_ext ? buffers[4] : nullptr,
                     (qj_diag *)diag, st);
}

int poisson_target(cudaStream_t st, void **buffers, const char *opaque, size_t len) {
  qj_xla_poisson_desc d;
  if (!opaque || len != sizeof(d)) {
    set_error("qj_xla_get_potential_f32: descriptor of %zu bytes, expected %zu", opaque ? len : 0,
              sizeof(d));
    return QJ_ERR_ARG;
  }
  std::memcpy(&d, opaque, sizeof(d));
  if (d.version != QJ_XLA_DESC_VERSION) {
    set_error("qj_xla_get_potential_f32: bad descriptor (version %d, expected %d)", d.version,
              QJ_XLA_DESC_VERSION);
    return QJ_ERR_ARG;
  }
  if (!buffers || !buffers[0] || !buffers[1]) {
    set_error("qj_xla_get_potential_f32: null buffer");
    return QJ_ERR_ARG;
  }
  const float *rho = (const float *)buffers[0];
  float *V = (float *)buffers[1];
  auto small = [](int n) { return n == 16 || n == 32 || n == 64; };
  if (small(d.grid.nx) && small(d.grid.ny) && small(d.grid.nz))
    return qj_get_potential_f32_noalloc(&d.grid, &d.phys, rho, V, d.self_interaction, st);
  qj_plan *P = nullptr;
  const int rc = cached_plan(d.grid, d.phys, 0, &P);
  if (rc) return rc;
  return qj_get_potential(P, rho, V, d.self_interaction, st);
}

}  // namespace
}  // namespace qj

using namespace qj;

extern "C" {

void qj_xla_kdk_step_f32(void *stream, void **buffers, const char *opaque, size_t opaque_len,
                         void *status) {
  finish(status, kdk_target((cudaStream_t)stream, buffers, opaque, opaque_len));
}

void qj_xla_get_potential_f32(void *stream, void **buffers, const char *opaque,
                              size_t opaque_len, void *status) {
  finish(status, poisson_target((cudaStream_t)stream, buffers, opaque, opaque_len));
}

void qj_xla_set_status_fn(qj_xla_status_fn fn) {
  std::lock_guard<std::mutex> lock(g_xla_mu);
  g_status_fn = fn;
}

int qj_xla_last_status(void) { return g_last_status.load(); }

int qj_xla_release_plans(void) {
  std::lock_guard<std::mutex> lock(g_xla_mu);
  int rc = QJ_OK;
  for (auto &kv : g_plans) {
    const int r = qj_plan_destroy(kv.second);
    if (r && rc == QJ_OK) rc = r;
  }
  g_plans.clear();
  return rc;
}

}  // extern "C"
