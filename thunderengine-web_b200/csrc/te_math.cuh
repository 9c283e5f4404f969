// Device arithmetic of the CM1 dynamics kernels, binary32 with the reference's rounding.
//
// Build contract (see build.py): -ftz=true -prec-div=true -prec-sqrt=true -fmad=false.
// With those flags every `a op b` below is one IEEE binary32 operation with subnormals
// flushed, `fmaf` is one fused multiply-add and `/` is the correctly rounded quotient;
// that is the arithmetic the reference's WGSL enforces with its opq() barriers and its
// correctly rounded division div_cr (data/kernels/adv_flux_x_weno.wgsl:15-50).
#pragma once
#include <cstdint>

#include "te_dims.cuh"

namespace te {


// Correctly rounded quotient.  The reference's div_cr returns the correctly rounded
// quotient in the normal range and the plain quotient for zero, huge, NaN and tiny
// results; with an IEEE divider and flushed subnormals both cases are the IEEE
// quotient, and the 2^64 pre-scaling of tiny numerators cancels exactly.
// The divisor passes through an empty asm so that the compiler cannot see a constant
// there: with -prec-div=true nvcc still turns x / c for a compile-time constant c into a
// multiplication by 1/c, which is not the correctly rounded quotient (measured on B200:
// x / 3.0f differed from the IEEE quotient for 33 % of 2^20 random x, x / 6e-05f for 64 %;
// a divisor only known at run time gave the IEEE quotient every time).
__device__ __forceinline__ float dcr(float a, float b) {
  asm("" : "+f"(b));
  return a / b;
}

// WGSL min/max on f32: min(a,b) = b if b < a else a; max(a,b) = b if a < b else a;
// a NaN operand yields the other one (fixes the sign of zero on +0/-0 ties).
__device__ __forceinline__ float wmin(float a, float b) { return (b < a || a != a) ? b : a; }
__device__ __forceinline__ float wmax(float a, float b) { return (a < b || a != a) ? b : a; }

// The reference's WGSL pow, exp and log builtins, whose precision WGSL leaves to the
// implementation, evaluated in binary64 with plain operations and rounded once to binary32:
//   ln x = e ln 2 + 2 atanh(s) for x = 2^e m, m in [sqrt(1/2), sqrt(2)), s = (m - 1) / (m + 1),
//          atanh by its odd power series to s^23;
//   2^t  = 2^n e^r, n = rint(t), r = (t - n) ln 2, e^r by its Taylor series to r^14;
//   x^y = 2^(y log2 x), e^x = 2^(x / ln 2).
// The binary64 error is far below half a binary32 ulp: each is the correctly rounded value
// except within that error of a rounding boundary.  The same operations in the same order
// on every device (no contraction).
__device__ __forceinline__ double ln_mantissa(float x, int& e) {  // x > 0 normal
  const uint32_t b = __float_as_uint(x);
  double m = (double)__uint_as_float((b & 0x7fffffu) | 0x3f800000u);
  e = (int)(b >> 23) - 127;
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    e = e + 1;
  }
  const double s = (m - 1.0) / (m + 1.0), s2 = s * s;
  double p = 1.0 / 23;
#pragma unroll
  for (int k = 21; k >= 1; k -= 2) p = p * s2 + 1.0 / k;
  return 2.0 * s * p;
}
__device__ __forceinline__ float exp2_rounded(double t) {
  if (t > 128.0) return INFINITY;
  if (t < -126.0) return 0.0f;
  const double n = rint(t), r = (t - n) * 0.6931471805599453;
  double q = 1.0;
#pragma unroll
  for (int k = 14; k >= 1; k--) q = 1.0 + (r * (1.0 / k)) * q;
  return (float)ldexp(q, (int)n);
}
__device__ __forceinline__ float pow_f64(float x, float y) {
  if (!(x > 0.0f) || x == INFINITY)
    return x == 0.0f ? (y > 0.0f ? 0.0f : INFINITY) : (x == INFINITY ? (y > 0.0f ? INFINITY : 0.0f) : NAN);
  int e;
  const double lm = ln_mantissa(x, e);
  return exp2_rounded((double)y * ((double)e + lm * 1.4426950408889634));
}
__device__ __forceinline__ float exp_f64(float x) {
  if (x != x) return x;
  return exp2_rounded((double)x * 1.4426950408889634);
}
__device__ __forceinline__ float log_f64(float x) {
  if (x != x || x < 0.0f) return NAN;
  if (x == 0.0f) return -INFINITY;
  if (x == INFINITY) return INFINITY;
  int e;
  const double lm = ln_mantissa(x, e);
  return (float)((double)e * 0.6931471805599453 + lm);
}
// log2 x = e + ln(m) / ln 2, from the same ln(m).
__device__ __forceinline__ float log2_f64(float x) {
  if (x != x || x < 0.0f) return NAN;
  if (x == 0.0f) return -INFINITY;
  if (x == INFINITY) return INFINITY;
  int e;
  const double lm = ln_mantissa(x, e);
  return (float)((double)e + lm * 1.4426950408889634);
}
// atan2(y, x) in binary64: a = min(|x|,|y|) / max(|x|,|y|) in [0, 1]; above tan(pi/12)
// atan a = pi/6 + atan((a sqrt3 - 1) / (a + sqrt3)), which leaves |u| <= tan(pi/12);
// atan u by its odd power series to u^29 (|u|^30 / 31 < 2^-57); then the octant
// (pi/2 - r where |y| > |x|, pi - r where x < 0) and the sign of y.  Zeros and infinities
// follow C's atan2f.
__device__ __forceinline__ float atan2_f64(float y, float x) {
  if (x != x || y != y) return x + y;
  const double ax = fabs((double)x), ay = fabs((double)y);
  const bool neg = __float_as_uint(y) >> 31, xneg = __float_as_uint(x) >> 31;
  double r;
  if (ax == INFINITY && ay == INFINITY) {
    r = xneg ? 2.356194490192345 : 0.7853981633974483;
  } else if (ax == 0.0 && ay == 0.0) {
    r = xneg ? 3.141592653589793 : 0.0;
  } else {
    const bool swap = ay > ax;
    const double a = swap ? ax / ay : ay / ax;
    double u = a, base = 0.0;
    if (a > 0.2679491924311227) {
      u = (a * 1.7320508075688772 - 1.0) / (a + 1.7320508075688772);
      base = 0.5235987755982988;
    }
    const double w = -(u * u);
    double p = 1.0 / 29;
#pragma unroll
    for (int k = 27; k >= 1; k -= 2) p = p * w + 1.0 / k;
    r = base + u * p;
    if (swap) r = 1.5707963267948966 - r;
    if (xneg) r = 3.141592653589793 - r;
  }
  const float f = (float)r;
  return neg ? -f : f;
}

// Quotients of constants, rounded once (the reference writes e.g. div_cr(13.0, 12.0)).
#define TE_C1312 (13.0f / 12.0f)
#define TE_C2_60 (2.0f / 60.0f)
#define TE_CM13_60 (-13.0f / 60.0f)
#define TE_C47_60 (47.0f / 60.0f)
#define TE_C27_60 (27.0f / 60.0f)
#define TE_CM3_60 (-3.0f / 60.0f)
#define TE_C2_6 (2.0f / 6.0f)
#define TE_CM1_6 (-1.0f / 6.0f)
#define TE_C5_6 (5.0f / 6.0f)
#define TE_C11_6 (11.0f / 6.0f)
#define TE_CM7_6 (-7.0f / 6.0f)
#define TE_C1_6 (1.0f / 6.0f)

// 5th-order upwind-biased linear reconstruction (2, -13, 47, 27, -3)/60.
__device__ __forceinline__ float flx5(float s1, float s2, float s3, float s4, float s5) {
  return fmaf(TE_CM3_60, s5, fmaf(TE_C27_60, s4, fmaf(TE_C47_60, s3, fmaf(TE_C2_60, s1, TE_CM13_60 * s2))));
}

// 3rd-order reconstruction (-1, 5, 2)/6.
__device__ __forceinline__ float flx3(float s1, float s2, float s3) {
  return fmaf(TE_C2_6, s3, fmaf(TE_CM1_6, s1, TE_C5_6 * s2));
}

// WENO-JS 5th-order reconstruction with clipped smoothness ratios.
__device__ __forceinline__ float weno5(float s1, float s2, float s3, float s4, float s5, float weps) {
  float e1 = fmaf(-2.0f, s2, s1) + s3;
  float d1 = fmaf(3.0f, s3, fmaf(-4.0f, s2, s1));
  float b1 = fmaf(TE_C1312 * e1, e1, (0.25f * d1) * d1);
  float e2 = fmaf(-2.0f, s3, s2) + s4;
  float d2 = s2 - s4;
  float b2 = fmaf(TE_C1312 * e2, e2, (0.25f * d2) * d2);
  float e3 = fmaf(-2.0f, s4, s3) + s5;
  float d3 = fmaf(3.0f, s3, -(4.0f * s4)) + s5;
  float b3 = fmaf(TE_C1312 * e3, e3, (0.25f * d3) * d3);
  float tau = fabsf(b1 - b3);
  float r1 = wmin(1e30f, dcr(tau, b1 + weps));
  float r2 = wmin(1e30f, dcr(tau, b2 + weps));
  float r3 = wmin(1e30f, dcr(tau, b3 + weps));
  float m = wmax(r1, wmax(r2, r3));
  float one = 1.0f;
  if (m > 1e15f) {
    float im = dcr(1.0f, m);
    r1 = r1 * im;
    r2 = r2 * im;
    r3 = r3 * im;
    one = im * im;
  }
  float w1 = 0.1f * fmaf(r1, r1, one);
  float w2 = 0.6f * fmaf(r2, r2, one);
  float w3 = 0.3f * fmaf(r3, r3, one);
  float p1 = fmaf(TE_C11_6, s3, fmaf(TE_C2_6, s1, TE_CM7_6 * s2));
  float p2 = fmaf(TE_C2_6, s4, fmaf(TE_CM1_6, s2, TE_C5_6 * s3));
  float p3 = fmaf(TE_CM1_6, s5, fmaf(TE_C2_6, s3, TE_C5_6 * s4));
  return dcr(fmaf(w3, p3, fmaf(w1, p1, w2 * p2)), (w1 + w2) + w3);
}

// Positive-definite gate: any |s| above weps.
__device__ __forceinline__ bool weno_pdef_ok(float s1, float s2, float s3, float s4, float s5, float weps) {
  float bmax = wmax(wmax(wmax(fabsf(s1), fabsf(s2)), wmax(fabsf(s3), fabsf(s4))), fabsf(s5));
  return bmax > weps;
}

// Limited 3rd-order upstream value next to the vertical boundaries.
__device__ __forceinline__ float upstrpd(float s1, float s2, float s3, float weps) {
  float dd = s2 - s1;
  float sgn = __uint_as_float((__float_as_uint(weps) & 0x7fffffffu) | (__float_as_uint(dd) & 0x80000000u));
  float rr = dcr(s3 - s2, sgn + dd);
  float phi = wmax(0.0f, wmin(rr, wmin(fmaf(TE_C2_6, rr, TE_C1_6), 1.0f)));
  return fmaf(phi, s2 - s1, s2);
}

// Horizontal metric planes of the hmetric buffer (uh, uf, vh, vf).
__device__ __forceinline__ float hm_uh(const Dims& g, const float* hm, int i) { return hm[i + 3]; }
__device__ __forceinline__ float hm_uf(const Dims& g, const float* hm, int i) { return hm[g.sJ + i + 3]; }
__device__ __forceinline__ float hm_vh(const Dims& g, const float* hm, int j) { return hm[2 * g.sJ + j + 3]; }
__device__ __forceinline__ float hm_vf(const Dims& g, const float* hm, int j) { return hm[2 * g.sJ + g.sK + j + 3]; }

// ---- two-float arithmetic for the correctly rounded pow used by the pressure glue
struct F2 {
  float x, y;
};
__device__ __forceinline__ F2 two_sum(float a, float b) {
  float s = a + b, bb = s - a;
  return F2{s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ F2 quick_two_sum(float a, float b) {
  float s = a + b;
  return F2{s, b - (s - a)};
}
__device__ __forceinline__ F2 mul_ff(F2 a, F2 b) {
  float p = a.x * b.x;
  float e = fmaf(a.x, b.x, -p);
  e = fmaf(a.x, b.y, e);
  e = fmaf(a.y, b.x, e);
  return quick_two_sum(p, e);
}
__device__ __forceinline__ F2 add_ff(F2 a, F2 b) {
  F2 s = two_sum(a.x, b.x), t = two_sum(a.y, b.y);
  F2 u = quick_two_sum(s.x, s.y + t.x);
  return quick_two_sum(u.x, u.y + t.y);
}

// log(x) as a two-float value: x = m 2^e with m in [sqrt(1/2), sqrt(2)), then
// log(m) = 2 atanh(f / (2 + f)) by an odd series in s = f / (2 + f).
__device__ __forceinline__ F2 rr_log_ff(float x) {
  int e;
  float m = frexpf(x, &e);
  if (m < 0.70710677f) {
    m = m * 2.0f;
    e = e - 1;
  }
  float f = m - 1.0f;
  F2 d = two_sum(2.0f, f);
  float sh = dcr(f, d.x);
  float r = fmaf(-sh, d.x, f);
  r = fmaf(-sh, d.y, r);
  F2 sf = quick_two_sum(sh, dcr(r, d.x));
  F2 s2 = mul_ff(sf, sf), s3 = mul_ff(s2, sf);
  F2 P{0.11764706f, -4.3826945e-10f};
  P = add_ff(mul_ff(P, s2), F2{0.13333334f, -6.9538753e-09f});
  P = add_ff(mul_ff(P, s2), F2{0.15384616f, -5.731216e-09f});
  P = add_ff(mul_ff(P, s2), F2{0.18181819f, -5.4186042e-09f});
  P = add_ff(mul_ff(P, s2), F2{0.22222222f, -1.6556846e-09f});
  P = add_ff(mul_ff(P, s2), F2{0.2857143f, -1.2772424e-08f});
  P = add_ff(mul_ff(P, s2), F2{0.4f, -5.9604646e-09f});
  P = add_ff(mul_ff(P, s2), F2{0.6666667f, -1.9868216e-08f});
  F2 l1p = add_ff(F2{2.0f * sf.x, 2.0f * sf.y}, mul_ff(s3, P));
  const float ln2h = 0.69314575f, ln2m = 1.4285906e-06f, ln2l = 1.6198487e-11f;
  float fe = (float)e;
  F2 a = add_ff(F2{fe * ln2h, fe * ln2m}, l1p);
  return add_ff(a, F2{fe * ln2l, 0.0f});
}

// exp of a two-float argument: k = round(y / ln2), Taylor series of the remainder,
// final rounding to nearest fixed up by the residual.
// f_rr_log_cr (turb_nm.wgsl): the two-float log summed; non-positive, infinite and NaN
// arguments take the log builtin's special values
__device__ __forceinline__ float rr_log_cr(float x) {
  if (!(x > 0.0f) || x == INFINITY) return x == 0.0f ? -INFINITY : (x == INFINITY ? INFINITY : NAN);
  const F2 a = rr_log_ff(x);
  return a.x + a.y;
}

__device__ __forceinline__ float rr_exp_ff(F2 y) {
  const float ln2h = 0.69314575f, ln2m = 1.4285906e-06f, ln2l = 1.6198487e-11f;
  float k = rintf(dcr(y.x, 0.6931472f));
  F2 r = add_ff(y, F2{(-k) * ln2h, (-k) * ln2m});
  r = add_ff(r, F2{(-k) * ln2l, 0.0f});
  F2 P{2.5052108e-08f, 4.417623e-16f};
  P = add_ff(mul_ff(P, r), F2{2.755732e-07f, -7.575112e-15f});
  P = add_ff(mul_ff(P, r), F2{2.7557319e-06f, 3.7935712e-14f});
  P = add_ff(mul_ff(P, r), F2{2.4801588e-05f, -3.406996e-13f});
  P = add_ff(mul_ff(P, r), F2{0.0001984127f, -2.7255969e-12f});
  P = add_ff(mul_ff(P, r), F2{0.0013888889f, -3.3631094e-11f});
  P = add_ff(mul_ff(P, r), F2{0.008333334f, -4.346172e-10f});
  P = add_ff(mul_ff(P, r), F2{0.041666668f, -1.2417635e-09f});
  P = add_ff(mul_ff(P, r), F2{0.16666667f, -4.967054e-09f});
  P = add_ff(mul_ff(P, r), F2{0.5f, 0.0f});
  P = add_ff(mul_ff(P, r), F2{1.0f, 0.0f});
  F2 Q = mul_ff(P, r);
  float s = 1.0f + Q.x;
  float t = (1.0f - s) + Q.x;
  F2 ur = two_sum(t, Q.y);
  float res = s + ur.x;
  float bb = res - s;
  float e3 = (s - (res - bb)) + (ur.x - bb);
  if (e3 != 0.0f && ur.y != 0.0f && (e3 > 0.0f) == (ur.y > 0.0f)) {
    float nb = __uint_as_float(__float_as_uint(res) + (e3 > 0.0f ? 1u : 4294967295u));
    if (e3 + e3 == nb - res) res = nb;
  }
  return ldexpf(res, (int)k);
}

__device__ __forceinline__ float rr_pow_cr(float x, float p) {
  if (!(x > 0.0f) || (__float_as_uint(x) & 0x7fffffffu) == 0x7f800000u) return powf(x, p);
  F2 L = rr_log_ff(x);
  float yh = L.x * p;
  return rr_exp_ff(quick_two_sum(yh, fmaf(L.y, p, fmaf(L.x, p, -yh))));
}

// rr_pow_cr(x, p) by a shorter route where the answer is not in doubt.  The reference's
// two-float power rounds a nearly exact x^p to the nearest binary32; here x^p is formed in
// binary64 (ln_mantissa above, p log2 x, then 2^t = 2^n e^r with e^r by its Taylor series
// to r^14; relative error below 2^-46) and rounded to the nearest binary32 f.  Unless that
// binary64 value lies within 2^-42 (relative) of a rounding boundary of f, both routes
// round the same real number the same way and give f; near a boundary, and for x outside
// [2^-6, 2^6) (over all 2^31 patterns with p = cp/rd the two routes differ at 3 inputs,
// the lowest 0x2e8000db, near 2^-34, where the two-float logarithm works with large
// magnitudes), rr_pow_cr itself runs.  For the exponents the kernels use, te_check_pow compares the two routes
// on every binary32 x.
__device__ __forceinline__ float rr_pow_fast(float x, float p) {
  if (__float_as_uint(x) - 0x3c800000u >= 0x06000000u) return rr_pow_cr(x, p);  // x outside [2^-6, 2^6)
  int e;
  const double lm = ln_mantissa(x, e);
  const double t = (double)p * ((double)e + lm * 1.4426950408889634);
  if (!(t > -125.0 && t < 125.0)) return rr_pow_cr(x, p);
  const double n = rint(t), r = (t - n) * 0.6931471805599453;
  double q = 1.0;
#pragma unroll
  for (int k = 14; k >= 1; k--) q = 1.0 + (r * (1.0 / k)) * q;
  const double y = q * __longlong_as_double((long long)((int)n + 1023) << 52);
  const float f = (float)y;
  const uint32_t fb = __float_as_uint(f);
  const double fd = (double)f;
  const double lo = 0.5 * (fd + (double)__uint_as_float(fb - 1u));  // the boundaries of f
  const double hi = 0.5 * (fd + (double)__uint_as_float(fb + 1u));
  const double tol = y * 0x1p-42;
  if (y - lo < tol || hi - y < tol) return rr_pow_cr(x, p);
  return f;
}

}  // namespace te
