// Correctly rounded double-precision cosine and sine of a rotation angle, for
// host and device alike.
//
// The reference's subpixel objective takes cos(rot) and sin(rot) of the host's
// C library (src/p-tracker.cpp:1038).  The device's own sincos may differ from
// those in the last bit, and a last-bit difference in the objective is enough
// to send Powell's line searches down another path.  This file computes both
// functions from their Taylor series in double-double arithmetic (Dekker's
// error-free sum and product, the product through a fused multiply-add) and
// rounds once at the end, so each result is the double nearest the true value
// unless that value lies within about 2^-100 (relative) of a rounding midpoint.
// A C library whose cosine and sine are correctly rounded on the angles in use
// returns the same doubles; tests/test_crtrig.py checks that against the
// host's library over millions of angles.
//
// Range: |x| <= pi/4 directly; up to 2^20 pi/2 after reduction by the nearest
// multiple of pi/2, with pi/2 held as three doubles (about 160 bits).  Beyond
// that the functions return NaN (rotation angles never get there).  Every
// operation is an explicit IEEE operation (__dadd_rn and friends on the
// device), so the results do not depend on FMA contraction settings.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define PTK_HD __host__ __device__ __forceinline__
#else
#define PTK_HD inline
#endif

namespace ptk {
namespace crtrig {

PTK_HD double add_rn(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  volatile double r = a + b;
  return r;
#endif
}
PTK_HD double sub_rn(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dsub_rn(a, b);
#else
  volatile double r = a - b;
  return r;
#endif
}
PTK_HD double mul_rn(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  volatile double r = a * b;
  return r;
#endif
}
PTK_HD double fma_rn(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return ::fma(a, b, c);
#endif
}

struct dd {
  double hi, lo;
};

// Knuth's two-sum: s + e == a + b exactly.
PTK_HD dd two_sum(double a, double b) {
  const double s = add_rn(a, b);
  const double bb = sub_rn(s, a);
  const double e = add_rn(sub_rn(a, sub_rn(s, bb)), sub_rn(b, bb));
  return dd{s, e};
}
// |a| >= |b| (or a == 0): s + e == a + b exactly.
PTK_HD dd fast_two_sum(double a, double b) {
  const double s = add_rn(a, b);
  return dd{s, sub_rn(b, sub_rn(s, a))};
}
// p + e == a * b exactly.
PTK_HD dd two_prod(double a, double b) {
  const double p = mul_rn(a, b);
  return dd{p, fma_rn(a, b, -p)};
}
PTK_HD dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  const dd t = two_sum(a.lo, b.lo);
  s.lo = add_rn(s.lo, t.hi);
  s = fast_two_sum(s.hi, s.lo);
  s.lo = add_rn(s.lo, t.lo);
  return fast_two_sum(s.hi, s.lo);
}
PTK_HD dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo = add_rn(p.lo, add_rn(mul_rn(a.hi, b.lo), mul_rn(a.lo, b.hi)));
  return fast_two_sum(p.hi, p.lo);
}

// (-1)^i / (2i+1)! and (-1)^i / (2i)! as double-double (exact rationals
// rounded to 106 bits).
#define PTK_CRT_SIN_N 16
#define PTK_CRT_COS_N 17

PTK_HD dd sin_coef(int i) {
  switch (i) {
    case 0: return dd{1.0, 0.0};
    case 1: return dd{-0.16666666666666666, -9.25185853854297e-18};
    case 2: return dd{0.008333333333333333, 1.1564823173178714e-19};
    case 3: return dd{-0.0001984126984126984, -1.7209558293420705e-22};
    case 4: return dd{2.7557319223985893e-06, -1.858393274046472e-22};
    case 5: return dd{-2.505210838544172e-08, 1.448814070935912e-24};
    case 6: return dd{1.6059043836821613e-10, 1.2585294588752098e-26};
    case 7: return dd{-7.647163731819816e-13, -7.03872877733453e-30};
    case 8: return dd{2.8114572543455206e-15, 1.6508842730861433e-31};
    case 9: return dd{-8.22063524662433e-18, -2.2141894119604265e-34};
    case 10: return dd{1.9572941063391263e-20, -1.3643503830087908e-36};
    case 11: return dd{-3.868170170630684e-23, 8.843177655482344e-40};
    case 12: return dd{6.446950284384474e-26, -1.9330404233703465e-42};
    case 13: return dd{-9.183689863795546e-29, -1.4303150396787322e-45};
    case 14: return dd{1.1309962886447716e-31, 1.0498015412959506e-47};
    default: return dd{-1.216125041553518e-34, -5.586290567888806e-51};
  }
}
PTK_HD dd cos_coef(int i) {
  switch (i) {
    case 0: return dd{1.0, 0.0};
    case 1: return dd{-0.5, 0.0};
    case 2: return dd{0.041666666666666664, 2.3129646346357427e-18};
    case 3: return dd{-0.001388888888888889, 5.300543954373577e-20};
    case 4: return dd{2.48015873015873e-05, 2.1511947866775882e-23};
    case 5: return dd{-2.755731922398589e-07, -2.3767714622250297e-23};
    case 6: return dd{2.08767569878681e-09, -1.20734505911326e-25};
    case 7: return dd{-1.1470745597729725e-11, -2.0655512752830745e-28};
    case 8: return dd{4.779477332387385e-14, 4.399205485834081e-31};
    case 9: return dd{-1.5619206968586225e-16, -1.1910679660273754e-32};
    case 10: return dd{4.110317623312165e-19, 1.4412973378659527e-36};
    case 11: return dd{-8.896791392450574e-22, 7.911402614872376e-38};
    case 12: return dd{1.6117375710961184e-24, -3.6846573564509766e-41};
    case 13: return dd{-2.4795962632247976e-27, 1.2953730964765229e-43};
    case 14: return dd{3.279889237069838e-30, 1.5117542744029879e-46};
    case 15: return dd{-3.7699876288159054e-33, -2.5870347832750324e-49};
    default: return dd{3.8003907548547434e-36, 1.7457158024652518e-52};
  }
}

// sin(r) and cos(r) for a double-double |r| <= pi/4 + tiny.
PTK_HD double sin_dd(dd r) {
  const dd z = dd_mul(r, r);
  dd s = sin_coef(PTK_CRT_SIN_N - 1);
  for (int i = PTK_CRT_SIN_N - 2; i >= 0; --i) s = dd_add(dd_mul(s, z), sin_coef(i));
  const dd v = dd_mul(s, r);
  return add_rn(v.hi, v.lo);
}
PTK_HD double cos_dd(dd r) {
  const dd z = dd_mul(r, r);
  dd c = cos_coef(PTK_CRT_COS_N - 1);
  for (int i = PTK_CRT_COS_N - 2; i >= 0; --i) c = dd_add(dd_mul(c, z), cos_coef(i));
  return add_rn(c.hi, c.lo);
}

// x - k pi/2 as a double-double, k = nearest integer to x 2/pi.  pi/2 is
// split into three doubles; k times each part is formed exactly.
PTK_HD dd reduce(double x, int* k_out) {
  const double kPio2_1 = 1.5707963267948966;       // pi/2 rounded to a double
  const double kPio2_2 = 6.123233995736766e-17;    // next 53 bits
  const double kPio2_3 = -1.4973849048591698e-33;  // next 53 bits
  const double k = rint(mul_rn(x, 0.6366197723675814));
  *k_out = (int)k;
  const dd p1 = two_prod(k, kPio2_1);
  const dd p2 = two_prod(k, kPio2_2);
  const dd p3 = two_prod(k, kPio2_3);
  dd r = dd_add(dd{x, 0.0}, dd{-p1.hi, -p1.lo});
  r = dd_add(r, dd{-p2.hi, -p2.lo});
  r = dd_add(r, dd{-p3.hi, -p3.lo});
  return r;
}

// Correctly rounded cos(x) (which == 0) or sin(x) (which == 1).
PTK_HD double cr_trig(double x, int which) {
  if (!(fabs(x) <= 1647099.0)) return x - x;  // NaN beyond 2^20 pi/2 (and for NaN / inf)
  if (fabs(x) <= 0.7853981633974483) return which ? (x == 0.0 ? x : sin_dd(dd{x, 0.0})) : cos_dd(dd{x, 0.0});
  int k;
  const dd r = reduce(x, &k);
  const int q = (k + which * 3) & 3;  // sin(x) = cos(x - pi/2)
  // cos(r + q pi/2) for q = 0..3: cos r, -sin r, -cos r, sin r
  switch (q) {
    case 0: return cos_dd(r);
    case 1: return -sin_dd(r);
    case 2: return -cos_dd(r);
    default: return sin_dd(r);
  }
}

PTK_HD double cr_cos(double x) { return cr_trig(x, 0); }
PTK_HD double cr_sin(double x) { return cr_trig(x, 1); }

}  // namespace crtrig
}  // namespace ptk
