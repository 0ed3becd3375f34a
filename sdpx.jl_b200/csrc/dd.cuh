// Double-double (Float64x2) arithmetic on the device.
//
// A value is the unevaluated sum hi + lo of two doubles, |lo| ≤ ulp(hi)/2.
// The operations are the published error-free transformations — Knuth's
// TwoSum, Dekker's FastTwoSum, the exact product a·b = p + e with
// e = fma(a, b, −p) — and the double-double sum and product of Hida, Li and
// Bailey's QD library (accurate addition: both halves summed with TwoSum).
// The product's rounded part is an explicit __dmul_rn, so the compiler cannot
// contract it into a following sum and the results do not depend on FMA
// contraction.
#pragma once
#include <cuda_runtime.h>

namespace sdpx {

struct ddv {
  double hi, lo;
};

__device__ __forceinline__ ddv dd_two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ ddv dd_fast_two_sum(double a, double b) {
  const double s = a + b;
  return {s, b - (s - a)};
}
__device__ __forceinline__ ddv dd_two_prod(double a, double b) {
  const double p = __dmul_rn(a, b);  // never contracted into a following sum
  return {p, __fma_rn(a, b, -p)};
}
__device__ __forceinline__ ddv dd_add(ddv a, ddv b) {
  ddv s = dd_two_sum(a.hi, b.hi);
  const ddv t = dd_two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = dd_fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return dd_fast_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ ddv dd_neg(ddv a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ ddv dd_mul(ddv a, ddv b) {
  ddv p = dd_two_prod(a.hi, b.hi);
  p.lo += __fma_rn(a.hi, b.lo, a.lo * b.hi);
  return dd_fast_two_sum(p.hi, p.lo);
}
__device__ __forceinline__ ddv dd_mul_d(ddv a, double b) {
  ddv p = dd_two_prod(a.hi, b);
  p.lo = __fma_rn(a.lo, b, p.lo);
  return dd_fast_two_sum(p.hi, p.lo);
}
// a / b by two correction steps of the quotient (QD's accurate division).
__device__ __forceinline__ ddv dd_div(ddv a, ddv b) {
  const double q1 = a.hi / b.hi;
  ddv r = dd_add(a, dd_neg(dd_mul_d(b, q1)));
  const double q2 = r.hi / b.hi;
  r = dd_add(r, dd_neg(dd_mul_d(b, q2)));
  const double q3 = r.hi / b.hi;
  const ddv q = dd_fast_two_sum(q1, q2);
  return dd_add(q, {q3, 0.0});
}
__device__ __forceinline__ ddv dd_load(const double* h, const double* l, long long i) {
  return {h[i], l ? l[i] : 0.0};
}
__device__ __forceinline__ void dd_store(double* h, double* l, long long i, ddv v) {
  h[i] = v.hi;
  l[i] = v.lo;
}
__device__ __forceinline__ ddv dd_shfl_xor(ddv v, int o) {
  return {__shfl_xor_sync(0xffffffffu, v.hi, o), __shfl_xor_sync(0xffffffffu, v.lo, o)};
}

}  // namespace sdpx
