// Ensemble launches of the fused passes: one persistent launch per pass for
// the boxes of up to three batched plans of sizes 64, 96 and 128 (one plan
// per size).  Those lengths share a CTA shape (128 threads on a strided pass,
// 256 on a contiguous one), so a CTA can run the pass body of any size class.
// Each CTA works on one box and claims its tiles from the box's counter
// (DynCta) until none are left, copying its next tile in while it transforms
// the current one; each class has enough CTAs to fill the GPU, and the
// classes follow one another in the launch (k_fused_ens).  Results are
// bit-identical to stepping each plan on its own (no tile's arithmetic
// depends on which CTA runs it).
#include <cmath>

#include "qj_fused_run.cuh"

namespace qj {

// Size classes, by slot: the largest first, so that the smaller classes'
// shorter tiles fill the launch's tail.
constexpr int kEnsSizes[kEnsClasses] = {128, 96, 64};

struct EnsClass {
  FusedArgs a;
  TileMaps maps;
  int nbox;  // boxes of the class (0 for an empty slot)
  int ctr0;  // the first box's tile counter in the launch's counters
  int cta0;  // the class's CTA range in the launch: the CTAs that start on it
  int ctas;
};
struct EnsLaunch {
  EnsClass c[kEnsClasses];
  unsigned *ctr;  // one tile counter per box of the launch, zeroed before it
};
static_assert(sizeof(EnsLaunch) <= 4096, "ensemble launch parameters exceed 4 KB");

template <bool CONTIG> struct EnsShape {
  using S0 = PassShape<64, CONTIG, 0>;
  using S1 = PassShape<96, CONTIG, 0>;
  using S2 = PassShape<128, CONTIG, 0>;
  static_assert(S0::THREADS == S1::THREADS && S1::THREADS == S2::THREADS,
                "ensemble size classes must share the CTA size");
  static constexpr int THREADS = S2::THREADS;
  static constexpr int MINB = S2::MINB < S0::MINB ? S2::MINB : S0::MINB;
};
template <int MODE, bool CONTIG> constexpr size_t ens_smem_bytes() {
  constexpr size_t a = fused_smem_bytes<64, CONTIG, MODE, 0>();
  constexpr size_t b = fused_smem_bytes<96, CONTIG, MODE, 0>();
  constexpr size_t c = fused_smem_bytes<128, CONTIG, MODE, 0>();
  return a > b ? (a > c ? a : c) : (b > c ? b : c);
}

// One CTA of class S: its box is its place in the class's CTA range modulo
// the class's box count, and it claims that box's tiles until none are left.
template <int S, int MODE, bool CONTIG>
__device__ __forceinline__ void ens_class_body(const EnsLaunch &L, int local, int *slot) {
  const EnsClass &c = L.c[S];
  const int b = local % c.nbox;
  FusedArgs a = c.a;
  fused_body<kEnsSizes[S], CONTIG, MODE, 0>(a, c.maps, DynCta{b, L.ctr + c.ctr0 + b, slot});
}

// The classes' CTA ranges follow one another in slot order, the largest
// class first; each range holds enough CTAs to fill the GPU on its own.  The
// hardware starts the CTAs in order, so the largest class's boxes take the
// GPU first, and as its CTAs find no tiles left and leave, the next class's
// CTAs take their slots: the classes overlap only at their ends.
template <int MODE, bool CONTIG>
__global__ void __launch_bounds__(EnsShape<CONTIG>::THREADS, EnsShape<CONTIG>::MINB)
    k_fused_ens(const __grid_constant__ EnsLaunch L) {
  __shared__ int slot;
  const int bid = (int)blockIdx.x;
  if (bid < L.c[0].cta0 + L.c[0].ctas) {
    ens_class_body<0, MODE, CONTIG>(L, bid - L.c[0].cta0, &slot);
  } else if (bid < L.c[1].cta0 + L.c[1].ctas) {
    ens_class_body<1, MODE, CONTIG>(L, bid - L.c[1].cta0, &slot);
  } else if (bid < L.c[2].cta0 + L.c[2].ctas) {
    ens_class_body<2, MODE, CONTIG>(L, bid - L.c[2].cta0, &slot);
  }
}

// Resident CTAs per SM of an ensemble launch and the SM count, per device.
template <int MODE, bool CONTIG> static cudaError_t ens_occupancy(int &per_sm, int &sms) {
  static PerDevice<Occupancy> cache;
  const Occupancy *o = nullptr;
  const cudaError_t e = per_device(cache, o, [](Occupancy &r) {
    const size_t smem = ens_smem_bytes<MODE, CONTIG>();
    r.err = cudaFuncSetAttribute(k_fused_ens<MODE, CONTIG>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int dev = 0, n_sm = 0, p = 0;
    if (r.err == cudaSuccess) r.err = cudaGetDevice(&dev);
    if (r.err == cudaSuccess) r.err = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (r.err == cudaSuccess)
      r.err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, k_fused_ens<MODE, CONTIG>,
                                                            EnsShape<CONTIG>::THREADS, smem);
    r.per_sm = std::max(1, p);
    r.sms = std::max(1, n_sm);
  });
  if (e != cudaSuccess) return e;
  per_sm = o->per_sm;
  sms = o->sms;
  return o->err;
}

template <int N, int MODE, bool CONTIG>
static int ens_class_setup(const FusedArgs &a, EnsClass &c) {
  c.a = a;
  c.a.ntiles = grid_of<N, CONTIG, 0>(a);
  c.a.rev = (!CONTIG && a.axis == 1) ? 1 : 0;
  std::memset(&c.maps, 0, sizeof(c.maps));
  if (!CONTIG && stream_count<MODE>() > 0) {
    const int rc = strided_maps<N, MODE, 0>(c.a, c.maps);
    if (rc) return rc;
  }
  c.nbox = a.nbox > 1 ? a.nbox : 1;
  return 0;
}

template <int MODE, bool CONTIG>
static int run_ens(int np, const FusedArgs *a, const int *n, int reserve, unsigned *ctr,
                   int nctr, cudaStream_t st) {
  EnsLaunch L;
  std::memset(&L, 0, sizeof(L));
  L.ctr = ctr;
  for (int i = 0; i < np; ++i) {
    const void *fields[4] = {a[i].psi, a[i].R, a[i].S1, a[i].S2};
    for (const void *f : fields)
      if ((reinterpret_cast<uintptr_t>(f) & 15) != 0) {
        set_error("fields of the fused passes must be 16-byte aligned");
        return QJ_ERR_ARG;
      }
    const int slot = ens_slot(n[i]);
    EnsClass &c = L.c[slot];
    const int rc = slot == 0   ? ens_class_setup<kEnsSizes[0], MODE, CONTIG>(a[i], c)
                   : slot == 1 ? ens_class_setup<kEnsSizes[1], MODE, CONTIG>(a[i], c)
                               : ens_class_setup<kEnsSizes[2], MODE, CONTIG>(a[i], c);
    if (rc) return rc;
  }
  // the classes' box counters follow one another in slot order
  int boxes = 0;
  for (int s = 0; s < kEnsClasses; ++s) {
    L.c[s].ctr0 = boxes;
    boxes += L.c[s].nbox;
  }
  if (boxes > nctr) {
    set_error("internal: ensemble launch of %d boxes with %d tile counters", boxes, nctr);
    return QJ_ERR_ARG;
  }
  int per_sm = 0, sms = 0;
  QJ_CK((ens_occupancy<MODE, CONTIG>(per_sm, sms)));
  // each class's range: a multiple of its box count, at least the CTAs that
  // fit at once (less the reserved slots)
  const int resident = std::max(1, per_sm * sms - reserve);
  int next = 0;
  for (int s = 0; s < kEnsClasses; ++s) {
    EnsClass &c = L.c[s];
    c.cta0 = next;
    c.ctas = c.nbox > 0 ? ((resident + c.nbox - 1) / c.nbox) * c.nbox : 0;
    next += c.ctas;
  }
  k_fused_ens<MODE, CONTIG><<<next, EnsShape<CONTIG>::THREADS, ens_smem_bytes<MODE, CONTIG>(), st>>>(L);
  QJ_CK_LAUNCH();
  return 0;
}

int ens_slot(int n) {
  for (int s = 0; s < kEnsClasses; ++s)
    if (kEnsSizes[s] == n) return s;
  return -1;
}

int launch_fused_ens(int mode, int np, const FusedArgs *a, const int *n, int reserve,
                     unsigned *ctr, int nctr, cudaStream_t st) {
  if (np < 1 || np > kEnsClasses) {
    set_error("internal: ensemble launch of %d plans", np);
    return QJ_ERR_ARG;
  }
  bool used[kEnsClasses] = {false, false, false};
  for (int i = 0; i < np; ++i) {
    const int s = ens_slot(n[i]);
    if (s < 0 || used[s] || a[i].shape != 0 || a[i].axis != a[0].axis) {
      set_error("internal: plan %d does not fit an ensemble launch", i);
      return QJ_ERR_ARG;
    }
    used[s] = true;
  }
  const bool contig = a[0].axis == 2;
  if (contig && (mode == M_FFT_FWD || mode == M_IFFT2)) {
    set_error("internal: pass mode %d requested along z", mode);
    return QJ_ERR_ARG;
  }
  const bool prof = prof_on();
  if (prof) prof_mark_begin(st);
  int rc;
#define QJ_ENS(M)                                                                        \
  case M:                                                                                \
    rc = contig ? run_ens<M, true>(np, a, n, reserve, ctr, nctr, st)                   \
                : run_ens<M, false>(np, a, n, reserve, ctr, nctr, st);                 \
    break;
  switch (mode) {
    QJ_ENS(M_DENSITY)
    QJ_ENS(M_POISSON)
    QJ_ENS(M_KICK)
    QJ_ENS(M_DRIFT)
    QJ_ENS(M_DRIFT_DENSITY)
    case M_FFT_FWD: rc = run_ens<M_FFT_FWD, false>(np, a, n, reserve, ctr, nctr, st); break;
    case M_IFFT2: rc = run_ens<M_IFFT2, false>(np, a, n, reserve, ctr, nctr, st); break;
    default:
      set_error("internal: pass mode %d has no ensemble launch", mode);
      rc = QJ_ERR_ARG;
  }
#undef QJ_ENS
  if (prof && rc == 0) prof_mark_end(mode, st);
  return rc;
}

}  // namespace qj
