// Pencil FFT core for libqj.
//
// A 1-D FFT of length N along one axis of a [nx][ny][nz] grid is computed by
// P = N / E threads ("a pencil group"), each holding E complex elements in
// registers.  Thread t of a group always holds the elements with index
// t + P * e, e = 0..E-1, both before and after the transform (natural order),
// so a forward transform, a pointwise multiply and an inverse transform chain
// in registers.  The transform is a Stockham autosort decimation in time over
// the radices of FftPlan<N, RV>; the first stage reads registers, the last stage
// writes registers, and each stage boundary is one exchange through shared
// memory.  Twiddles come from a table w[m] = exp(-2 pi i m / N) computed in
// float64 on the host and rounded once to the working precision.
//
// Direction DIR = -1 is the forward transform (numpy fftn sign), DIR = +1 the
// unnormalised inverse.
#pragma once

#include "qj_common.cuh"

namespace qj {

// cos(2 pi m / 16) for the in-register codelet twiddles.
__host__ __device__ constexpr double cos16(int m) {
  return m == 0    ? 1.0
         : m == 1  ? 0.92387953251128675613
         : m == 2  ? 0.70710678118654752440
         : m == 3  ? 0.38268343236508977173
         : m == 4  ? 0.0
         : m == 5  ? -0.38268343236508977173
         : m == 6  ? -0.70710678118654752440
         : m == 7  ? -0.92387953251128675613
         : m == 8  ? -1.0
         : m == 9  ? -0.92387953251128675613
         : m == 10 ? -0.70710678118654752440
         : m == 11 ? -0.38268343236508977173
         : m == 12 ? 0.0
         : m == 13 ? 0.38268343236508977173
         : m == 14 ? 0.70710678118654752440
                   : 0.92387953251128675613;
}
__host__ __device__ constexpr double sin16(int m) { return cos16((m + 12) % 16); }

// x * exp(DIR * 2 pi i k / R) for R | 16, k a compile-time constant after
// unrolling.
template <int R, int DIR, typename C>
__device__ __forceinline__ C twc(C x, int k) {
  using T = decltype(x.x);
  const int m = (k * (16 / R)) % 16;
  if (m == 0) return x;
  if (m == 4) return cmul_i<DIR>(x);
  if (m == 8) return C{-x.x, -x.y};
  if (m == 12) return cmul_i<-DIR>(x);
  const T c = (T)cos16(m), s = (T)(DIR * sin16(m));
  return C{x.x * c - x.y * s, x.x * s + x.y * c};
}

// In-register DFT of length R: a[k] = sum_n a[n] exp(DIR 2 pi i n k / R).
template <int R, int DIR, typename C> struct Dft {
  __device__ __forceinline__ static void run(C *a) {
    static_assert(R == 8 || R == 16, "power-of-two codelet");
    C e[R / 2], o[R / 2];
#pragma unroll
    for (int k = 0; k < R / 2; ++k) {
      e[k] = a[2 * k];
      o[k] = a[2 * k + 1];
    }
    Dft<R / 2, DIR, C>::run(e);
    Dft<R / 2, DIR, C>::run(o);
#pragma unroll
    for (int k = 0; k < R / 2; ++k) {
      C t = twc<R, DIR>(o[k], k);
      if ((k * (16 / R)) % 16 == 4) {  // t = +-i o: scalar, the sign folds into the adds
        a[k] = cadd(e[k], t);
        a[k + R / 2] = csub(e[k], t);
      } else {
        a[k] = padd(e[k], t);
        a[k + R / 2] = psub(e[k], t);
      }
    }
  }
};
template <int DIR, typename C> struct Dft<1, DIR, C> {
  __device__ __forceinline__ static void run(C *) {}
};
template <int DIR, typename C> struct Dft<2, DIR, C> {
  __device__ __forceinline__ static void run(C *a) {
    C t = a[1];
    a[1] = psub(a[0], t);
    a[0] = padd(a[0], t);
  }
};
template <int DIR, typename C> struct Dft<4, DIR, C> {
  __device__ __forceinline__ static void run(C *a) {
    C s02 = padd(a[0], a[2]), d02 = psub(a[0], a[2]);
    C s13 = padd(a[1], a[3]), d13 = psub(a[1], a[3]);
    C r = cmul_i<DIR>(d13);
    a[0] = padd(s02, s13);
    a[2] = psub(s02, s13);
    a[1] = cadd(d02, r);
    a[3] = csub(d02, r);
  }
};
template <int DIR, typename C> struct Dft<3, DIR, C> {
  __device__ __forceinline__ static void run(C *a) {
    using T = decltype(a[0].x);
    const T h = (T)0.5, s = (T)0.86602540378443864676;
    C t1 = cadd(a[1], a[2]);
    C t2 = csub(a[0], cscale(t1, h));
    C t3 = cscale(cmul_i<DIR>(csub(a[1], a[2])), s);
    a[0] = cadd(a[0], t1);
    a[1] = cadd(t2, t3);
    a[2] = csub(t2, t3);
  }
};

// Radix plans: E elements per thread, NS stages, radix(s) divides E.  RV = 0
// is each length's default; RV = 1 (n = 128, 256) holds half as many elements
// per thread, so twice the threads share a pencil over one more stage.
template <int N, int RV = 0> struct FftPlan;
template <> struct FftPlan<16> {
  static constexpr int E = 16, NS = 1;
  __host__ __device__ static constexpr int radix(int) { return 16; }
};
template <> struct FftPlan<32> {
  static constexpr int E = 8, NS = 2;
  __host__ __device__ static constexpr int radix(int s) { return s == 0 ? 8 : 4; }
};
template <> struct FftPlan<64> {
  static constexpr int E = 8, NS = 2;
  __host__ __device__ static constexpr int radix(int) { return 8; }
};
template <> struct FftPlan<96> {  // 96 = 4 * 4 * 2 * 3, 12 elements per thread
  static constexpr int E = 12, NS = 4;
  __host__ __device__ static constexpr int radix(int s) {
    return s == 0 ? 4 : (s == 1 ? 4 : (s == 2 ? 2 : 3));
  }
};
template <> struct FftPlan<128> {
  static constexpr int E = 16, NS = 2;
  __host__ __device__ static constexpr int radix(int s) { return s == 0 ? 16 : 8; }
};
template <> struct FftPlan<256> {
  static constexpr int E = 16, NS = 2;
  __host__ __device__ static constexpr int radix(int) { return 16; }
};
template <> struct FftPlan<512> {
  static constexpr int E = 16, NS = 3;
  __host__ __device__ static constexpr int radix(int s) { return s == 0 ? 16 : (s == 1 ? 8 : 4); }
};
template <> struct FftPlan<128, 1> {  // 8 * 4 * 4, 16 threads per pencil
  static constexpr int E = 8, NS = 3;
  __host__ __device__ static constexpr int radix(int s) { return s == 0 ? 8 : 4; }
};
template <> struct FftPlan<256, 1> {  // 8 * 8 * 4, 32 threads per pencil
  static constexpr int E = 8, NS = 3;
  __host__ __device__ static constexpr int radix(int s) { return s == 2 ? 4 : 8; }
};
// Lengths with a radix variant.
__host__ __device__ constexpr bool has_radix_variant(int n) { return n == 128 || n == 256; }
// The radix plan whose thread holds E elements of a length-N pencil.
template <int N, int E> __host__ __device__ constexpr int radix_variant_of() {
  return E == FftPlan<N, 0>::E ? 0 : 1;
}

template <int N, int RV = 0> __host__ __device__ constexpr int stage_ns(int s) {
  int ns = 1;
  for (int i = 0; i < s; ++i) ns *= FftPlan<N, RV>::radix(i);
  return ns;
}

// Shared-memory views of one pencil.
//  Strided passes: layout [N][TP] (pencils fastest; lanes run over pencils).
//  Contiguous passes: layout [TP][N + N/16] (elements fastest, padded so the
//  radix-r scatter of the first stage is bank-conflict free).
// A strided pencil's P threads span several warps (the CTA synchronises); a
// contiguous pencil's P <= 32 threads sit inside one warp, whose private rows
// need only a warp barrier.
template <typename C, int TP> struct SmemStrided {
  C *base;  // &sm[p]
  __device__ __forceinline__ C ld(int idx) const { return base[idx * TP]; }
  __device__ __forceinline__ void st(int idx, C v) const { base[idx * TP] = v; }
  __device__ __forceinline__ static void sync() { __syncthreads(); }
};
template <typename C> struct SmemContig {
  C *row;  // &sm[p * (N + N/16)]
  __device__ __forceinline__ C ld(int idx) const { return row[idx + (idx >> 4)]; }
  __device__ __forceinline__ void st(int idx, C v) const { row[idx + (idx >> 4)] = v; }
  __device__ __forceinline__ static void sync() { __syncwarp(); }
};

// Stage twiddle tables (read from shared memory by the fused passes): for
// stage s > 0 (Ns = product of earlier radices, radix r), row jm < Ns holds
// w_N^(jm q N / (Ns r)) for q = 1..r-1, padded to tw_row(s) entries; the
// stages are concatenated.  A thread reads its row two twiddles at a time
// (16-byte loads); the row length is 2 mod 4 entries, so eight consecutive
// rows start on eight different bank quads (conflict-free 16-byte loads).
template <int N, int RV = 0> __host__ __device__ constexpr int tw_row(int s) {
  int L = FftPlan<N, RV>::radix(s) - 1;
  while (L % 4 != 2) ++L;
  return L;
}
template <int N, int RV = 0> __host__ __device__ constexpr int stage_tw_off(int s) {
  int off = 0;
  for (int i = 1; i < s; ++i) off += stage_ns<N, RV>(i) * tw_row<N, RV>(i);
  return off;
}
template <int N, int RV = 0> __host__ __device__ constexpr int stage_tw_size() {
  return stage_tw_off<N, RV>(FftPlan<N, RV>::NS);
}

template <int N, int DIR, int S, typename C, class SM, bool TWS, int RV> struct FftStages {
  using PL = FftPlan<N, RV>;
  static constexpr int E = PL::E, P = N / E;
  static constexpr int r = PL::radix(S);
  static constexpr int B = E / r;
  static constexpr int Ns = stage_ns<N, RV>(S);
  static_assert(E % r == 0, "radix must divide E");

  __device__ __forceinline__ static void run(C (&v)[E], int t, const SM &sm,
                                             const C *__restrict__ tw) {
    if constexpr (S > 0) {
#pragma unroll
      for (int u = 0; u < B; ++u) {
        const int j = t + P * u;
#pragma unroll
        for (int q = 0; q < r; ++q) v[u + q * B] = sm.ld(j + q * (N / r));
      }
    }
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int j = t + P * u;
      C a[r];
#pragma unroll
      for (int q = 0; q < r; ++q) a[q] = v[u + q * B];
      if constexpr (Ns > 1) {
        const int jm = j % Ns;
        if constexpr (TWS) {
          // two twiddles per 16-byte load from the thread's row
          const float4 *row =
              reinterpret_cast<const float4 *>(tw + stage_tw_off<N, RV>(S) + jm * tw_row<N, RV>(S));
#pragma unroll
          for (int h = 0; 2 * h + 1 < r; ++h) {
            const float4 w2 = row[h];
            a[2 * h + 1] = DIR < 0 ? cmul(a[2 * h + 1], C{w2.x, w2.y}) : cmulc(a[2 * h + 1], C{w2.x, w2.y});
            if (2 * h + 2 < r)
              a[2 * h + 2] = DIR < 0 ? cmul(a[2 * h + 2], C{w2.z, w2.w}) : cmulc(a[2 * h + 2], C{w2.z, w2.w});
          }
        } else {
#pragma unroll
          for (int q = 1; q < r; ++q) {
            const C w = __ldg(&tw[jm * q * (N / (Ns * r))]);
            a[q] = DIR < 0 ? cmul(a[q], w) : cmulc(a[q], w);
          }
        }
      }
      Dft<r, DIR, C>::run(a);
#pragma unroll
      for (int q = 0; q < r; ++q) v[u + q * B] = a[q];
    }
    if constexpr (S + 1 < PL::NS) {
      SM::sync();  // every thread of the pencil has finished reading its rows
#pragma unroll
      for (int u = 0; u < B; ++u) {
        const int j = t + P * u;
        const int idxD = (j / Ns) * Ns * r + (j % Ns);
#pragma unroll
        for (int q = 0; q < r; ++q) sm.st(idxD + q * Ns, v[u + q * B]);
      }
      SM::sync();
      FftStages<N, DIR, S + 1, C, SM, TWS, RV>::run(v, t, sm, tw);
    }
  }
};

// Transform the pencil held by the P threads of a group.  Every thread of the
// CTA (strided) or warp (contiguous) must call this the same number of times.
// TWS: tw is the stage twiddle table of the radix plan (usually in shared
// memory); otherwise the flat table w[m] = exp(-2 pi i m / N) in global
// memory.  The radix plan follows from the thread's element count E.
template <int N, int DIR, bool TWS = false, typename C, int E, class SM>
__device__ __forceinline__ void fft_pencil(C (&v)[E], int t, const SM &sm,
                                           const C *__restrict__ tw) {
  constexpr int RV = radix_variant_of<N, E>();
  static_assert(FftPlan<N, RV>::E == E, "no radix plan of this length holds E elements");
  FftStages<N, DIR, 0, C, SM, TWS, RV>::run(v, t, sm, tw);
}

// Launch shape of a pencil pass over length N.  V selects a shape variant:
// bit 0 the radix plan (FftPlan<N, 1>), bit 1 half the pencils per CTA (a
// contiguous tile of 128 instead of 256 threads' pencils, a strided tile 8
// instead of 16 z columns wide).  Variants exist for has_radix_variant(N).
template <int N, bool CONTIG, int V = 0> struct PassShape {
  static constexpr int RV = V & 1, TV = (V >> 1) & 1;
  static constexpr int E = FftPlan<N, RV>::E;
  static constexpr int P = N / E;
  static constexpr int CT = TV ? 128 : 256;  // threads' worth of contiguous pencils
  static constexpr int TP = CONTIG ? (P >= CT ? 1 : CT / P) : (TV ? 8 : 16);
  static constexpr int THREADS = TP * P;
  // resident CTAs per SM requested from the register allocator: enough for
  // a budget of 128 registers per thread (2 x 256, 4 x 128, ... threads)
  static constexpr int MINB0 = 65536 / (THREADS * 128);
  static constexpr int MINB = MINB0 < 1 ? 1 : (MINB0 > 16 ? 16 : MINB0);
  static constexpr int ROW = N + N / 16;  // padded contiguous row
  template <typename C> static constexpr size_t smem_bytes() {
    return CONTIG ? (size_t)TP * ROW * sizeof(C) : (size_t)TP * N * sizeof(C);
  }
};

}  // namespace qj
