// tri_common.cuh -- constants and small device helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace tri {

// Physical constants and tolerances of the reference (constants.h:38-50,
// 117-118).  SQRTG is the reference's literal, not sqrt(9.81).
constexpr double kGravity = 9.81;
constexpr double kSqrtG = 3.132091953;
constexpr double kMaxValue = 1e10;  // "dry" cell dt sentinel (MAX_VALUE)

template <typename T>
__host__ __device__ constexpr T eps12();
template <>
__host__ __device__ constexpr double eps12<double>() { return 1e-12; }
// The FP32 form keeps the FP64 absolute threshold (the reference's
// single-precision build flushes flux contributions below 1e-6, which deletes
// the mass of thin sheet flow) and adds a relative one, kNoise32, for
// contributions that are rounding noise of larger terms.
template <>
__host__ __device__ constexpr float eps12<float>() { return 1e-12f; }

// FP32 form: relative size below which a face contribution is rounding noise
// of the terms that formed it (about 17 float ulps).
constexpr double kNoise32 = 2e-6;

__device__ __forceinline__ double dev_sqrt(double x) { return sqrt(x); }
// FP32 form: the approximate hardware square root, one PTX instruction, so it
// is the same in every kernel the solver is inlined into.
__device__ __forceinline__ float dev_sqrt(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ double dev_cbrt(double x) { return cbrt(x); }
__device__ __forceinline__ float dev_cbrt(float x) { return cbrtf(x); }
__device__ __forceinline__ double dev_fabs(double x) { return fabs(x); }
__device__ __forceinline__ float dev_fabs(float x) { return fabsf(x); }
__device__ __forceinline__ double dev_fmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float dev_fmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double dev_fmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float dev_fmin(float a, float b) { return fminf(a, b); }

__device__ __forceinline__ double dev_fma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float dev_fma(float a, float b, float c) { return fmaf(a, b, c); }

// IEEE quotient a / b, compiled out of line: for divisions on paths the
// solver rarely takes (entropy fix, dry-side tests, the fallback of
// div_shared), so their instruction sequences do not crowd the instruction
// cache of the step loop (ncu showed 17 % of warp cycles stalled on
// instruction fetch with them inline; out of line: FP64 flux launches 3-6 %
// shorter).  The same rounding as an inline '/'.  The FP32 form's quotient
// is short and stays inline (out of line measured 1 % slower there).
static __device__ __noinline__ double div_rare(double a, double b) { return a / b; }
__device__ __forceinline__ float div_rare(float a, float b) { return a / b; }

// a / b rounded to nearest from y = RN(1/b), the correctly rounded reciprocal
// (Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990): q0 = RN(a*y) is within
// one ulp of a/b, the residual r = a - b*q0 is exact in one fused
// multiply-add, and RN(q0 + r*y) is the correctly rounded quotient.  The
// theorem needs a, b and a/b normal (no overflow or underflow).  An exact
// quotient (r == 0) returns q0 itself, which also keeps the sign of a zero.
// Three operations instead of a full division when the divisor is reused.
template <typename T>
__device__ __forceinline__ T div_by_rcp(T a, T b, T y) {
  const T q0 = a * y;
  const T r = dev_fma(-q0, b, a);
  return r == T(0) ? q0 : dev_fma(r, y, q0);
}
// FP32 form: within 1.5 ulp is enough, one multiplication.
template <>
__device__ __forceinline__ float div_by_rcp<float>(float a, float, float y) {
  return a * y;
}

// div_by_rcp for a dividend that is never a zero (and never subnormal): with
// q0 != 0, an exact quotient (r == 0) gives fma(0, y, q0) == q0, so the
// zero-residual test is not needed.  The solver's uses: dt*p with |p| >=
// 1e-12 (smaller face contributions are flushed to +0 before, and dt*(+0)
// is the exact quotient +0 both ways: r = +0, fma(+0, y, +0) = +0), and
// h*dx/2 with h > 0 (a depth, far above the subnormal range; the same
// three operations as div_by_rcp there).
template <typename T>
__device__ __forceinline__ T div_nz(T a, T b, T y) {
  const T q0 = a * y;
  return dev_fma(dev_fma(-q0, b, a), y, q0);
}
template <>
__device__ __forceinline__ float div_nz<float>(float a, float, float y) {
  return a * y;
}

// a / b rounded to nearest for a divisor b shared by several quotients, from
// y = RN(1/b): div_by_rcp where Markstein's conditions provably hold (|a| >=
// 2^-900 so the residual a - b*q0 is exact, and q0 = RN(a*y) between 2^-1000
// and 2^1000 so the quotient is normal), a plain division otherwise.  A zero
// dividend gives the signed zero of a/b.  Bit-identical to a / b for every
// finite a and finite non-zero b (a NaN dividend gives a NaN, not
// necessarily with the payload IEEE division would propagate); the solver
// divides by Roe-averaged celerities, sums of sqrt(h) and the friction term
// this way.  The conditions are tested as FP64 comparisons of magnitudes:
// the same tests on the exponent bits take integer instructions from the
// issue slots of an issue-limited kernel (Thacker 2048^2 FP64 flux launch
// 0.1270 ms with them, 0.1244 ms with comparisons); on the 32-bit high words,
// with the zero residual left to fma, they measured 17 % slower.
__device__ __forceinline__ double div_shared(double a, double b, double y) {
  const double q0 = a * y;
  const double fa = fabs(a), fq = fabs(q0);
  if (a != 0.0 && (fa < 0x1p-900 || fq < 0x1p-1000 || fq > 0x1p1000)) return div_rare(a, b);
  const double r = fma(-q0, b, a);
  return r == 0.0 ? q0 : fma(r, y, q0);
}
// FP32 form: one multiplication (within 1.5 ulp).
__device__ __forceinline__ float div_shared(float a, float, float y) { return a * y; }

// Programmatic dependent launch: the step kernels are launched so that the
// next one may be scheduled while the previous one drains.  Each of them
// first waits until its predecessor has completed and its memory is visible
// (pdl_wait, before it reads or writes anything), so the order of their
// effects is exactly stream order; pdl_trigger lets the successor's launch
// begin once every block of this grid has reached it.  Both are no-ops for a
// kernel launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Integer mix of a cell index and a step number (deterministic, so a batch
// member rounds exactly as its solo run).
__device__ __forceinline__ uint32_t cell_hash(uint32_t id, uint32_t step) {
  uint32_t x = id * 0x9E3779B1u ^ (step * 0x85EBCA77u + 0x27D4EB2Fu);
  x ^= x >> 15;
  x *= 0x2C1B3C6Du;
  x ^= x >> 12;
  x *= 0x297A2D39u;
  x ^= x >> 15;
  return x;
}

// a + b rounded stochastically between its two neighbouring floats
// (unbiased), computed in FP32: the rounding error of a + b is exact by
// Knuth's TwoSum, and the sum moves to the neighbour on the error's side with
// probability |error| / gap.  r uniform in [0, 2^32).  *exact_lo receives the
// error, so (double)RN(a + b) + error is the exact sum.
__device__ __forceinline__ float sr_add(float a, float b, uint32_t r, float* exact_lo) {
  const float s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  const float err = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  *exact_lo = err;
  if (err == 0.0f) return s;
  const float t = nextafterf(s, err > 0.0f ? INFINITY : -INFINITY);
  const float u = (float)(r >> 8) * 0x1p-24f;
  return u * fabsf(t - s) < fabsf(err) ? t : s;
}

// Reciprocal of a divisor shared by several quotients.  FP64: RN(1/b), as
// div_shared requires.  FP32 form: the hardware's approximate reciprocal
// (within 2 ulp), written as an intrinsic so it is the same instruction in
// every kernel the solver is inlined into (a compiler allowed to approximate
// divisions may rewrite them differently in different contexts, and a batch
// member must compute exactly what the same domain computes alone).
__device__ __forceinline__ double recip(double b) { return 1.0 / b; }
__device__ __forceinline__ float recip(float b) { return __fdividef(1.0f, b); }
// a / b where the FP32 form accepts the approximate quotient (same reason).
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

// The CFL dt of a wet cell is RN(A / D) with A = RN(courant*dx) and the wave
// speed D = maxu + sqrt(g)*sqrt(h) (compute_dt_and_sqrt, kernels.h:167-193).
// RN(A / D) never increases with D, so the minimum over cells of the dt is
// RN(A / max D): the kernels reduce the largest D and divide once.  The slot
// holds kDtKeyInf - bits(D), an order-reversing key (bits of a non-negative
// double order like the double) under an unsigned atomic min; kDtKeyInf is
// the empty slot (no wet cell), and NaN speeds are left out (the reference's
// "a < m ? a : m" fold never selects a NaN dt).
constexpr unsigned long long kDtKeyInf = 0x7FF0000000000000ull;
__host__ __device__ inline unsigned long long speed_key(double d) {
  if (!(d >= 0.0)) return kDtKeyInf;
  unsigned long long b;
#ifdef __CUDA_ARCH__
  b = (unsigned long long)__double_as_longlong(d);
#else
  __builtin_memcpy(&b, &d, 8);
#endif
  return kDtKeyInf - (b > kDtKeyInf ? kDtKeyInf : b);
}
// dt of a slot: RN(A / D) for the largest speed, DBL_MAX for an empty slot.
__host__ __device__ inline double dt_of_key(unsigned long long key, double cfl_a) {
  if (key >= kDtKeyInf) return 1.7976931348623157e308;
  const unsigned long long b = kDtKeyInf - key;
  double d;
#ifdef __CUDA_ARCH__
  d = __longlong_as_double((long long)b);
#else
  __builtin_memcpy(&d, &b, 8);
#endif
  return cfl_a / d;
}


}  // namespace tri
