// hadros_cr_math.cuh — sin, cos and x^(1/4) rounded to nearest, for the
// reference-arithmetic trace kernel.
//
// The reference's geodesic depends on libm in two places: sin and cos of
// theta in every inverse metric (src/kerr_metric.cpp) and pow(tol/err, 0.25)
// in the RKF45 step control (src/kerr_geodesic.cpp:317-321).  The host libm
// returns the correctly rounded value for all but a small fraction of
// arguments; CUDA's device functions are accurate to a few ulp but round
// differently more often.  A one-ulp change in a metric term moves the
// centred finite differences of the geodesic force by ~1e-11, enough to flip
// an accept/reject decision now and then.  These functions evaluate the
// results to ~2^-78 relative before the final rounding, so they agree with
// the correctly rounded value except with probability ~2^-25 per call.
//
// Method (published textbook technique, own implementation):
//   * argument reduction x = k pi/2 + r with pi/2 in three parts (the first
//     two of 33 bits, so k P1 and k P2 are exact for |k| < 2^20), carried as
//     a double-double r = rh + rl;
//   * r = j/128 + b with |b| <= 1/256; sin and cos of j/128 from a table of
//     double-double values (hadros_sincos_table.h, generated at 60 digits);
//     sin b and cos b from their Taylor series, the leading terms in
//     double-double, the rest in double;
//   * sin(a + b) = sin a cos b + cos a sin b in double-double arithmetic
//     (Dekker/Knuth two-sum, and FMA-based two-product), then the quadrant.
//   * x^(1/4) = sqrt(sqrt(x)) with each square root refined to double-double
//     by one FMA residual.
// Every operation uses an explicit rounding intrinsic, so the results are
// the same bits on the host and the device.
#pragma once

#include <cmath>

#include "hadros_sincos_table.h"

#ifdef __CUDACC__
#define CRM_HD __host__ __device__ __forceinline__
#else
#define CRM_HD inline
#endif

namespace hadros {
namespace crm {

#ifdef __CUDA_ARCH__
CRM_HD double add(double a, double b) { return __dadd_rn(a, b); }
CRM_HD double sub(double a, double b) { return __dsub_rn(a, b); }
CRM_HD double mul(double a, double b) { return __dmul_rn(a, b); }
CRM_HD double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
CRM_HD double sqrt_(double a) { return __dsqrt_rn(a); }
CRM_HD double div_(double a, double b) { return __ddiv_rn(a, b); }
#else
CRM_HD double add(double a, double b) { return a + b; }
CRM_HD double sub(double a, double b) { return a - b; }
CRM_HD double mul(double a, double b) { return a * b; }
CRM_HD double fma_(double a, double b, double c) { return std::fma(a, b, c); }
CRM_HD double sqrt_(double a) { return std::sqrt(a); }
CRM_HD double div_(double a, double b) { return a / b; }
#endif

struct DD {
    double h, l;
};

// s + e = a + b exactly
CRM_HD DD two_sum(double a, double b)
{
    const double s = add(a, b);
    const double bb = sub(s, a);
    const double e = add(sub(a, sub(s, bb)), sub(b, bb));
    return DD{s, e};
}
// s + e = a + b exactly, |a| >= |b|
CRM_HD DD fast_two_sum(double a, double b)
{
    const double s = add(a, b);
    return DD{s, sub(b, sub(s, a))};
}
CRM_HD DD dd_mul(DD a, DD b)
{
    const double p = mul(a.h, b.h);
    double e = fma_(a.h, b.h, -p);
    e = add(e, add(mul(a.h, b.l), mul(a.l, b.h)));
    return fast_two_sum(p, e);
}
CRM_HD DD dd_add(DD a, DD b)
{
    const DD s = two_sum(a.h, b.h);
    return fast_two_sum(s.h, add(s.l, add(a.l, b.l)));
}

// The table (sin hi, sin lo, cos hi, cos lo of j/128); `tab` points to it in
// the caller's memory space.
CRM_HD void sincos_dd(double x, const double* tab, DD* s, DD* c)
{
    const double kd = std::rint(mul(x, HADROS_2_OVER_PI));
    const int q = static_cast<int>(kd) & 3;
    // r = x - k pi/2 as a double-double
    const double r1 = fma_(-kd, HADROS_PIO2_1, x);          // exact
    DD r = two_sum(r1, -mul(kd, HADROS_PIO2_2));            // k P2 exact
    r.l = sub(r.l, mul(kd, HADROS_PIO2_3));
    r = fast_two_sum(r.h, r.l);
    // r = j/128 + b
    const double jd = std::rint(mul(r.h, 128.0));
    const int j = static_cast<int>(std::fabs(jd));
    const double sg = jd < 0.0 ? -1.0 : 1.0;
    const DD b = fast_two_sum(fma_(-jd, 0.0078125, r.h), r.l);   // r.h - j/128 is exact
    const double b2 = mul(b.h, b.h);
    // sin b = b - b^3/6 + b^5/120 - b^7/5040
    const double st = mul(mul(b.h, b2), fma_(b2, fma_(b2, -1.0 / 5040.0, 1.0 / 120.0), -1.0 / 6.0));
    DD sb = two_sum(b.h, st);
    sb.l = add(sb.l, b.l);
    // cos b = 1 - b^2/2 + b^4/24 - b^6/720, b^2/2 as a double-double
    const double hh = mul(b2, 0.5);
    const double hl = add(mul(fma_(b.h, b.h, -b2), 0.5), mul(b.h, b.l));
    const double ct = mul(mul(b2, b2), fma_(b2, -1.0 / 720.0, 1.0 / 24.0));
    DD cb = two_sum(1.0, -hh);
    cb.l = add(cb.l, sub(ct, hl));
    const DD sa{mul(sg, tab[4 * j]), mul(sg, tab[4 * j + 1])};
    const DD ca{tab[4 * j + 2], tab[4 * j + 3]};
    const DD sr = dd_add(dd_mul(sa, cb), dd_mul(ca, sb));
    DD cr = dd_mul(sa, sb);
    cr = dd_add(dd_mul(ca, cb), DD{-cr.h, -cr.l});
    switch (q) {
    case 0: *s = sr; *c = cr; break;
    case 1: *s = cr; *c = DD{-sr.h, -sr.l}; break;
    case 2: *s = DD{-sr.h, -sr.l}; *c = DD{-cr.h, -cr.l}; break;
    default: *s = DD{-cr.h, -cr.l}; *c = sr; break;
    }
}

// sin and cos of x rounded to nearest (|x| < 2^20; larger arguments are not
// on the geodesic path and fall back to the platform's functions).
CRM_HD void sincos_rn(double x, const double* tab, double* s, double* c)
{
    if (!(std::fabs(x) < 1048576.0)) {
        *s = std::sin(x);
        *c = std::cos(x);
        return;
    }
    DD sd, cd;
    sincos_dd(x, tab, &sd, &cd);
    *s = sd.h;
    *c = cd.h;
}

// sin and cos of x0 + d rounded to nearest from the double-doubles of x0,
// for |d| <= 1e-4: angle addition with sin d = d - d^3/6, cos d = 1 - d^2/2
// + d^4/24 (the next terms are below 2^-90 relative).
CRM_HD void sincos_shift_rn(DD s0, DD c0, double d, double* s, double* c)
{
    const double d2 = mul(d, d);
    DD sd = two_sum(d, mul(mul(d, d2), -1.0 / 6.0));
    const double hh = mul(d2, 0.5), hl = mul(fma_(d, d, -d2), 0.5);
    DD cd = two_sum(1.0, -hh);
    cd.l = add(cd.l, sub(mul(mul(d2, d2), 1.0 / 24.0), hl));
    const DD sr = dd_add(dd_mul(s0, cd), dd_mul(c0, sd));
    DD t = dd_mul(s0, sd);
    const DD cr = dd_add(dd_mul(c0, cd), DD{-t.h, -t.l});
    *s = sr.h;
    *c = cr.h;
}

// x^(1/4) rounded to nearest for finite x > 0.
CRM_HD double pow025_rn(double x)
{
    const double s = sqrt_(x);
    const double sl = div_(fma_(-s, s, x), mul(2.0, s));    // sqrt(x) = s + sl
    const double q = sqrt_(s);
    const double ql = div_(add(fma_(-q, q, s), sl), mul(2.0, q));
    return add(q, ql);
}

}  // namespace crm
}  // namespace hadros
