// Common device helpers for libqj: complex types, exact-rounding float ops,
// and the per-axis geometry of a pencil pass.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace qj {

template <typename R> struct CT;
template <> struct CT<float> { using T = float2; };
template <> struct CT<double> { using T = double2; };
template <typename R> using cplx = typename CT<R>::T;

template <typename C> __device__ __forceinline__ C cmake(double x, double y) {
  C c;
  c.x = (decltype(c.x))x;
  c.y = (decltype(c.y))y;
  return c;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) {
  return C{a.x + b.x, a.y + b.y};
}
template <typename C> __device__ __forceinline__ C csub(C a, C b) {
  return C{a.x - b.x, a.y - b.y};
}
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  return C{a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) {
  return C{a.x * s, a.y * s};
}
// i * a  (dir = +1) or -i * a (dir = -1)
template <int DIR, typename C> __device__ __forceinline__ C cmul_i(C a) {
  return DIR > 0 ? C{-a.y, a.x} : C{a.y, -a.x};
}

// a + b and a - b as one packed instruction for float2 (sm_100's
// add/sub.rn.f32x2: two IEEE round-to-nearest operations, the same results as
// the scalar pair); other types fall back to the scalar pair.  Used where both
// operands are already whole register pairs: an operand that still needs a
// swap or a sign (a +-i rotation) goes through the scalar cadd / csub, whose
// negation folds into the add.
template <typename C> __device__ __forceinline__ C padd(C a, C b) { return cadd(a, b); }
template <typename C> __device__ __forceinline__ C psub(C a, C b) { return csub(a, b); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 qa, qb, qr;\n\t"
      "mov.b64 qa, {%2, %3};\n\tmov.b64 qb, {%4, %5};\n\t"
      "add.rn.f32x2 qr, qa, qb;\n\tmov.b64 {%0, %1}, qr;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 qa, qb, qr;\n\t"
      "mov.b64 qa, {%2, %3};\n\tmov.b64 qb, {%4, %5};\n\t"
      "sub.rn.f32x2 qr, qa, qb;\n\tmov.b64 {%0, %1}, qr;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}

// float ops with explicit round-to-nearest and no contraction, used where the
// reference's float32 operation order is reproduced exactly (CIC weights).
__device__ __forceinline__ float fmul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double fmul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fadd_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fsub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double fdiv_rn(double a, double b) { return __ddiv_rn(a, b); }

// Floating modulo with the sign of the divisor (numpy / jnp.mod semantics):
// r = fmod(x, y); if r != 0 and sign(r) != sign(y): r += y.
__device__ __forceinline__ float ref_mod(float x, float y) {
  float r = fmodf(x, y);
  if (r != 0.0f && ((r < 0.0f) != (y < 0.0f))) r = __fadd_rn(r, y);
  return r;
}
__device__ __forceinline__ double ref_mod(double x, double y) {
  double r = fmod(x, y);
  if (r != 0.0 && ((r < 0.0) != (y < 0.0))) r = __dadd_rn(r, y);
  return r;
}

// Non-negative float max via integer atomics (order independent).
__device__ __forceinline__ void atomic_max_nonneg(unsigned int *addr, float v) {
  atomicMax(addr, __float_as_uint(v));
}
__device__ __forceinline__ void atomic_min_nonneg(unsigned int *addr, float v) {
  atomicMin(addr, __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *addr, double v) {
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_min_nonneg(unsigned long long *addr, double v) {
  atomicMin(addr, (unsigned long long)__double_as_longlong(v));
}

// Geometry of one pencil pass.  Axis a in {0:x, 1:y, 2:z}.  The pencils of
// a pass are numbered by `pid`; a cell's key in the orientation of axis a is
// key = pid * n_a + i_a, with
//   a = 0: pid = y * nz + z         a = 1: pid = x * nz + z
//   a = 2: pid = x * ny + y         (a = 2 keys are the natural linear index)
struct PassGeom {
  int nx, ny, nz;
  int axis;
  long long stride;  // element stride along the axis
  // strided passes (axis 0 / 1): CTA = (outer index o, z tile)
  long long outer_stride;
  int n_outer;
};

}  // namespace qj
