// hadros_trace_kernel.cuh — device code of the trace kernel, shared by the two
// translation units that instantiate it: hadros_trace.cu (reference
// arithmetic, compiled with --fmad=false) and hadros_trace_fast.cu (fast
// geodesic arithmetic, compiled with FMA contraction).  See hadros_trace.cu
// for what the kernel does.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "hadros_cr_math.cuh"
#include "hadros_internal.h"

namespace hadros {

// Minimum resident blocks per SM asked of the register allocator.  4 blocks
// of 128 threads caps the kernel at 128 registers: measured on B200 (256x256
// mixed camera) 1.72x faster than the uncapped 162 registers / 3 blocks for
// the reference-arithmetic kernel and 1.31x for the fast one; 5 blocks (96
// registers) spills more and is slower again.
#ifndef HADROS_MIN_BLOCKS
#define HADROS_MIN_BLOCKS 4
#endif
// Inline the geodesic RHS at its call sites (1) or keep one out-of-line copy (0).
#ifndef HADROS_RHS_INLINE
#define HADROS_RHS_INLINE 1
#endif
#if HADROS_RHS_INLINE
#define HADROS_RHS_ATTR __device__ __forceinline__
#else
#define HADROS_RHS_ATTR __device__ __noinline__
#endif

namespace {

// RKF45 weights of y4 and y5 (kerr_geodesic.cpp:310-311), folded at compile
// time like the reference's 25.0/216.0 etc.
constexpr double A1 = 25.0 / 216.0, A3 = 1408.0 / 2565.0, A4 = 2197.0 / 4104.0, A5 = 1.0 / 5.0;
constexpr double B1 = 16.0 / 135.0, B3 = 6656.0 / 12825.0, B4 = 28561.0 / 56430.0,
                 B5 = 9.0 / 50.0, B6 = 2.0 / 55.0;

struct K5 {
    double r, th, ph, pr, pth;
};

// -0.5 * sum dg^{mu nu} p_mu p_nu in the reference's (mu, nu) order.
__device__ __forceinline__ double fd_force(double d00, double d03, double d11, double d22,
                                           double d33, double p0, double p1, double p2, double p3)
{
    double acc = 0.0;
    acc -= 0.5 * d00 * p0 * p0;
    acc -= 0.5 * d03 * p0 * p3;
    acc -= 0.5 * d11 * p1 * p1;
    acc -= 0.5 * d22 * p2 * p2;
    acc -= 0.5 * d03 * p3 * p0;
    acc -= 0.5 * d33 * p3 * p3;
    return acc;
}

// sin/cos of j/128 (double-double) for the rounded-to-nearest sin and cos of
// the reference-arithmetic kernel (hadros_cr_math.cuh).
__device__ const double kScTab[4 * HADROS_SC_N] = HADROS_SC_TABLE;

// sin and cos of theta as double-doubles, rounded to nearest in .h.
__device__ __forceinline__ void sincos_dd(double th, crm::DD* s, crm::DD* c)
{
    if (fabs(th) < 1048576.0) {
        crm::sincos_dd(th, kScTab, s, c);
    } else {
        *s = crm::DD{sin(th), 0.0};
        *c = crm::DD{cos(th), 0.0};
    }
}

// KerrGeodesic::rhs (kerr_geodesic.cpp:83-135) with sin/cos of theta given
// (double-doubles; their .h is the value rounded to nearest, as the host
// libm gives it for all but rare arguments).  The reference evaluates
// g^{-1}(r +- eps) and g^{-1}(theta +- eps) once per (mu, nu) pair; they are
// evaluated once here (identical values).
HADROS_RHS_ATTR void geo_rhs(double a, double r, double th, const crm::DD& sd, const crm::DD& cd,
                             double pr, double pth, double pt, double pph, K5& d)
{
    const double s = sd.h, c = cd.h;
    M5 gi;
    bl_ginv(a, r, s, c, gi);
    d.r = gi.rr * pr;
    d.th = gi.thth * pth;
    d.ph = gi.tph * pt + gi.phph * pph;
    {
        const double eps = 1.0e-5 * smax(1.0, fabs(r));
        M5 gp, gm;
        bl_ginv(a, r + eps, s, c, gp);
        bl_ginv(a, r - eps, s, c, gm);
        const double den = 2.0 * eps;
        d.pr = fd_force((gp.tt - gm.tt) / den, (gp.tph - gm.tph) / den, (gp.rr - gm.rr) / den,
                        (gp.thth - gm.thth) / den, (gp.phph - gm.phph) / den, pt, pr, pth, pph);
    }
    {
        const double eps = 1.0e-5;
        const double thp = th + eps, thm = th - eps;
        double sp, cp, sm, cm;
        if (th > 1.0e-3) {   // thp - th and thm - th are exact: angle addition from theta's double-doubles
            crm::sincos_shift_rn(sd, cd, thp - th, &sp, &cp);
            crm::sincos_shift_rn(sd, cd, thm - th, &sm, &cm);
        } else {
            crm::DD a1, b1;
            sincos_dd(thp, &a1, &b1);
            sp = a1.h;
            cp = b1.h;
            sincos_dd(thm, &a1, &b1);
            sm = a1.h;
            cm = b1.h;
        }
        M5 gp, gm;
        bl_ginv(a, r, sp, cp, gp);
        bl_ginv(a, r, sm, cm, gm);
        const double den = 2.0 * eps;
        d.pth = fd_force((gp.tt - gm.tt) / den, (gp.tph - gm.tph) / den, (gp.rr - gm.rr) / den,
                         (gp.thth - gm.thth) / den, (gp.phph - gm.phph) / den, pt, pr, pth, pph);
    }
}

// ---- fast geodesic arithmetic ---------------------------------------------
// The same Hamiltonian RHS with the same centred differences, evaluated with
// fewer FP64 divisions and transcendentals: one Newton-refined reciprocal per
// inverse metric, 1/sin^2(theta) shared by the three metrics at one angle,
// sin/cos of theta +- eps by angle addition, and FMA contraction (the
// translation unit is compiled with --fmad=true).  Results differ from the
// reference by rounding only.

// 1/b to within an ulp: hardware estimate (rcp.approx.ftz.f64) and two
// Newton-Raphson steps r <- r + r (1 - b r).
__device__ __forceinline__ double rcp_nr(double b)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
    double e = fma(-b, r, 1.0);
    r = fma(r, e, r);
    e = fma(-b, r, 1.0);
    return fma(r, e, r);
}

struct Trig {
    double s2, c2, inv_s2;
};

// The radius-only terms of the inverse metric at r (shared by the metrics
// at theta and theta +- eps).
struct RTerms {
    double r2, del, rpa2, tar;
};

__device__ __forceinline__ RTerms rterms(double a, double a2, double r)
{
    RTerms t;
    t.r2 = r * r;
    t.del = t.r2 - 2.0 * r + a2;
    const double rpa = t.r2 + a2;
    t.rpa2 = rpa * rpa;
    t.tar = 2.0 * a * r;
    return t;
}

__device__ __forceinline__ void ginv_fast(double a2, const RTerms& R, const Trig& t, M5& g)
{
    const double sig = R.r2 + a2 * t.c2;
    const double bigA = R.rpa2 - a2 * R.del * t.s2;
    const double inv_sd = rcp_nr(sig * R.del);
    g.tt = -bigA * inv_sd;
    g.tph = -R.tar * inv_sd;
    g.thth = R.del * inv_sd;
    g.rr = R.del * g.thth;
    g.phph = (R.del - a2 * t.s2) * inv_sd * t.inv_s2;
}

// The momenta's products in -1/2 dg^{mu nu} p_mu p_nu (both forces use them).
struct PQ {
    double q00, q03, q11, q22, q33;
};

// -1/2 sum (gp - gm)^{mu nu} p_mu p_nu / (2 eps), with scale = -1/2 / (2 eps).
__device__ __forceinline__ double force_fast(const M5& gp, const M5& gm, double scale, const PQ& q)
{
    double acc = (gp.tt - gm.tt) * q.q00;
    acc = fma(gp.tph - gm.tph, q.q03, acc);
    acc = fma(gp.rr - gm.rr, q.q11, acc);
    acc = fma(gp.thth - gm.thth, q.q22, acc);
    acc = fma(gp.phph - gm.phph, q.q33, acc);
    return scale * acc;
}

// sin and cos of th + d for |d| ~ 1e-5 (d exact): Taylor terms to d^3.
__device__ __forceinline__ Trig trig_shift(double s, double c, double d)
{
    const double d2 = d * d;
    const double cd = 1.0 - 0.5 * d2;
    const double sd = d - d * d2 * (1.0 / 6.0);
    const double sn = s * cd + c * sd;
    const double cs = c * cd - s * sd;
    Trig t;
    t.s2 = sn * sn;
    t.c2 = cs * cs;
    t.inv_s2 = rcp_nr(t.s2);
    return t;
}

HADROS_RHS_ATTR void geo_rhs_fast(double a, double r, double th, double s, double c,
                                  double pr, double pth, double pt, double pph, K5& d)
{
    const double a2 = a * a;
    Trig t0;
    t0.s2 = s * s;
    t0.c2 = c * c;
    t0.inv_s2 = rcp_nr(t0.s2);
    const RTerms R0 = rterms(a, a2, r);
    M5 gi;
    ginv_fast(a2, R0, t0, gi);
    d.r = gi.rr * pr;
    d.th = gi.thth * pth;
    d.ph = gi.tph * pt + gi.phph * pph;
    const PQ q{pt * pt, 2.0 * pt * pph, pr * pr, pth * pth, pph * pph};
    {
        const double eps = 1.0e-5 * smax(1.0, fabs(r));
        M5 gp, gm;
        ginv_fast(a2, rterms(a, a2, r + eps), t0, gp);
        ginv_fast(a2, rterms(a, a2, r - eps), t0, gm);
        d.pr = force_fast(gp, gm, -0.25 * rcp_nr(eps), q);
    }
    {
        // the reference differentiates at fl(th +- 1e-5); use those exact offsets
        const double dp = (th + 1.0e-5) - th, dm = (th - 1.0e-5) - th;
        const Trig tp = trig_shift(s, c, dp), tm = trig_shift(s, c, dm);
        M5 gp, gm;
        ginv_fast(a2, R0, tp, gp);
        ginv_fast(a2, R0, tm, gm);
        d.pth = force_fast(gp, gm, -0.5 * (1.0 / (2.0 * 1.0e-5)), q);
    }
}

// sin and cos of th0 + d from those of th0, |d| < 0.05: Taylor series of
// sin d and cos d to d^9 and d^8 (the next terms are below 3e-20).
__device__ __forceinline__ void sincos_shift(double s0, double c0, double d, double* s, double* c)
{
    const double d2 = d * d;
    const double cd = 1.0 + d2 * (-1.0 / 2 + d2 * (1.0 / 24 + d2 * (-1.0 / 720 + d2 * (1.0 / 40320))));
    const double sd = d * (1.0 + d2 * (-1.0 / 6 + d2 * (1.0 / 120 + d2 * (-1.0 / 5040 + d2 * (1.0 / 362880)))));
    *s = s0 * cd + c0 * sd;
    *c = c0 * cd - s0 * sd;
}

// RHS at a stage point.  The fast variant reuses sin/cos of the step's base
// angle th0 (s0, c0) through sincos_shift when the stage angle is close.
template <int FAST>
__device__ __forceinline__ void geo_rhs_sel(double a, double r, double th, double pr, double pth,
                                            double pt, double pph, K5& d, double th0, double s0,
                                            double c0)
{
    double s, c;
    if (FAST) {
        const double dt = th - th0;
        if (fabs(dt) < 0.05) sincos_shift(s0, c0, dt, &s, &c);
        else sincos(th, &s, &c);
        geo_rhs_fast(a, r, th, s, c, pr, pth, pt, pph, d);
    } else {
        crm::DD sd, cd;
        sincos_dd(th, &sd, &cd);
        geo_rhs(a, r, th, sd, cd, pr, pth, pt, pph, d);
    }
}

// wrapped_delta_phi (kerr_camera.cpp:31-44)
__device__ __forceinline__ double wrapped_dphi(double phi_new, double phi_old)
{
    double dphi = phi_new - phi_old;
    int guard = 0;
    while (dphi > kPi && guard < 64) { dphi -= 2.0 * kPi; ++guard; }
    while (dphi < -kPi && guard < 128) { dphi += 2.0 * kPi; ++guard; }
    return dphi;
}

// Kahan step with rounding intrinsics: never fused with the product that
// makes x, whatever the surrounding code (the in-loop and deferred transfers
// must round alike).
__device__ __forceinline__ void kahan_add(float& s, float& c, float x)
{
    const float y = __fsub_rn(x, c);
    const float t = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
}

struct SmemLayout {
    // FP64 sigma arrays (n each): E, S, lnE, lnS; FP32: lx (n), seg (4n)
    size_t off_E, off_S, off_lnE, off_lnS, off_lx, off_seg, off_acc, total;
};

__host__ __device__ inline SmemLayout smem_layout(int precision, int n, int max_bins)
{
    SmemLayout L{};
    size_t o = 0;
    L.off_E = o; o += sizeof(double) * n;
    L.off_S = o; o += sizeof(double) * n;
    L.off_lnE = o; o += sizeof(double) * n;
    L.off_lnS = o; o += sizeof(double) * n;
    L.off_lx = o; o += sizeof(float) * n;
    o = (o + 15) & ~size_t(15);
    L.off_seg = o; o += sizeof(float) * 4 * n;
    o = (o + 15) & ~size_t(15);
    L.off_acc = o;
    o += (precision == HADROS_PRECISION_MIXED ? kAccF * sizeof(float) : 2 * sizeof(double)) *
         size_t(kTPB) * size_t(max_bins);
    L.total = o;
    return L;
}

// Shared-memory sigma tables of the block.
struct SmemTables {
    const double* E;
    const double* S;
    const double* lnE;
    const double* lnS;
    const float* lx;
    const float4* seg;
    int n;
    double Emin, Emax, scale;
    int uniform;
    float lx0, inv_dlx;
};

// This thread's column of per-bin accumulators.  FP64 mode: tau and I
// (T64, I64, stride kTPB).  Mixed mode, exponents in base 2 (kAccF = 5
// floats per bin, array j of a column at f + j * fst, bin b at b * st): S the
// intensity's integer-valued anchor (exact), T - Tc the Kahan pair of
// tau log2(e) from zero, I - Ic the Kahan pair of the intensity scaled by 2^S.

struct BinAcc {
    double* T64;
    double* I64;
    float* f;
    long fst;   // floats between the arrays S, T, Tc, I, Ic
    int st;     // stride between bins: kTPB in shared memory, 1 in a deferred slot
};

struct BinSums {
    float S, T, Tc, I, Ic;
};

__device__ __forceinline__ BinSums acc_load(const BinAcc& a, int b)
{
    const float* p = a.f + b * a.st;
    return BinSums{p[0], p[a.fst], p[2 * a.fst], p[3 * a.fst], p[4 * a.fst]};
}
__device__ __forceinline__ void acc_store(const BinAcc& a, int b, const BinSums& v)
{
    float* p = a.f + b * a.st;
    p[0] = v.S;
    p[a.fst] = v.T;
    p[2 * a.fst] = v.Tc;
    p[3 * a.fst] = v.I;
    p[4 * a.fst] = v.Ic;
}

// The mixed-precision transfer of one path point, in two parts: the
// bin-independent terms (point_terms_body, FP64 where a decision is exact)
// and the update of one bin's FP32 accumulators (bin_point).  Density and
// ln(emissivity) are FP32 (hadros_physics_f32.cuh).  Exponents are kept in
// base 2, so every exponential is one ex2.approx.
//
// Intensity: each bin's sum is kept scaled by 2^S with S an integer-valued
// anchor, stored exactly.  A contribution K w(E_loc)/w(E_mid) exp(-tau)
// enters as 2^e with e = arg + (S - tau log2 e), arg = log2(K w/w0), computed
// as ((S - T) + arg) + Tc: where the term matters, S - T is within a few
// hundred of zero (S follows tau minus the emission's own exponent), so its
// rounding is at most that of arg itself.  S moves by whole powers of two
// when the sum is empty or a term would exceed 2^57.7 (e^40); terms below
// e^-800 are below FP64's range and skipped, as the reference's FP64 sum
// rounds them away.  tau accumulates in its own Kahan pair from zero, so its
// relative precision does not depend on S, and S stays exact however large
// tau grows behind optically thick gas.

// 2^x (PTX ex2.approx.ftz.f32: relative error below 2^-22).
__device__ __forceinline__ float ex2a(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Exact 2^k for integer k <= 127; 0 below 2^-126.
__device__ __forceinline__ float pow2i(int k)
{
    return k < -126 ? 0.0f : __int_as_float((k + 127) << 23);
}

constexpr float kAnchorMax2 = 57.70780f;     // 40 / ln 2
constexpr float kUnderflow2 = -1154.156f;    // -800 / ln 2

__device__ __forceinline__ void point_terms_body(const DevCam* cam, const DevBin* bins, int B, double r,
                                                 double th, double gg, double dl_cm, PointRec& p)
{
    const float rho = torus_rho_f(cam->torus, cam->torus_f, r, th);
    const float lnC = ln_emission_f(cam->src, cam->src_f, cam->torus, cam->torus_f, r, th, rho);
    const double zp = 1.0 / gg;   // E_local / E_mid
    p.lnzp = static_cast<float>(log(zp));
    p.zm1 = static_cast<float>(zp - 1.0);
    const bool emit = cam->sp_emit && (lnC > -INFINITY) && dl_cm > 0.0;
    // log2(g^3 C dl_cm) - gamma log2(1/g), g = 1 / zp
    p.u2 = emit ? __fmul_rn(__fsub_rn(__fadd_rn(lnC, __logf(static_cast<float>(dl_cm))),
                                      __fmul_rn(__fadd_rn(3.0f, cam->sp_gamma), p.lnzp)),
                            static_cast<float>(kLog2E))
                : -INFINITY;
    p.nbdl2 = rho > 0.0f ? rho * static_cast<float>(dl_cm * cam->k_nb * kLog2E) : -1.0f;
    // The bins whose E_local = E_mid/gg lies in [E_min, E_max] of the sigma
    // table (radiative_transfer.cpp:661-668), decided in FP64 exactly as the
    // reference's compares: gg_lo[b] <= gg <= gg_hi[b], both bounds rising
    // with b, so the bins form one run b0..b1.
    int lo = 0, cnt = B;   // first b with gg_lo[b] > gg
    while (cnt > 0) {
        const int st = cnt >> 1;
        if (!(gg < bins[lo + st].gg_lo)) { lo += st + 1; cnt -= st + 1; }
        else cnt = st;
    }
    p.b1 = lo - 1;
    lo = 0;
    cnt = B;               // first b with gg_hi[b] >= gg
    while (cnt > 0) {
        const int st = cnt >> 1;
        if (bins[lo + st].gg_hi < gg) { lo += st + 1; cnt -= st + 1; }
        else cnt = st;
    }
    p.b0 = lo;
}

// false for a point the transfer skips (radiative_transfer.cpp:501-505)
__device__ __forceinline__ bool point_terms(const DevCam* cam, const DevBin* bins, int B, double r, double th,
                                            double dl, double z, PointRec& p)
{
    if (r < cam->rt_skip) return false;
    const double g = 1.0 / smax(z, 1.0e-300);
    const double gg = smax(g, 1.0e-300);
    point_terms_body(cam, bins, B, r, th, gg, dl * cam->rg_cm, p);
    return true;
}

// The fields of a DevBin the mixed transfer reads (the deferred replay keeps
// them in registers).
struct BinK {
    float lnE, kcut2, qbase;
};

__device__ __forceinline__ BinK bin_k(const DevBin& d) { return BinK{d.lnE, d.kcut2, d.qbase}; }

// One path point into bin b: emission with the optical depth before the
// point, then the point's absorption (radiative_transfer.cpp:650-671).
// Rounding intrinsics throughout: no multiply-add is fused differently in the
// in-loop and the deferred transfer.
__device__ __forceinline__ void bin_point(const PointRec& p, const BinK& bn, int b, const SmemTables& tb, BinSums& a)
{
    if (p.u2 != -INFINITY) {
        const float arg = __fmaf_rn(-bn.kcut2, p.zm1, p.u2);
        // log2 of the term itself: below -800 / ln 2 it is under FP64's range
        if (__fsub_rn(arg, __fsub_rn(a.T, a.Tc)) >= kUnderflow2) {
            float e = __fadd_rn(__fadd_rn(__fsub_rn(a.S, a.T), arg), a.Tc);
            if (a.I == 0.0f || e > kAnchorMax2) {
                const float k = -rintf(e);
                if (a.I != 0.0f) {
                    const float sc = pow2i(static_cast<int>(k));
                    a.I = __fmul_rn(a.I, sc);
                    a.Ic = __fmul_rn(a.Ic, sc);
                }
                a.S = __fadd_rn(a.S, k);
                e = __fadd_rn(__fadd_rn(__fsub_rn(a.S, a.T), arg), a.Tc);
            }
            kahan_add(a.I, a.Ic, ex2a(e));
        }
    }
    if (!(p.nbdl2 < 0.0f) && b >= p.b0 && b <= p.b1) {
        const float lnE = __fadd_rn(bn.lnE, p.lnzp);
        int k;
        if (tb.uniform) {   // evenly spaced ln E: the segment from the coordinate
            k = __float2int_rd(__fmaf_rn(p.lnzp, tb.inv_dlx, bn.qbase)) + 1;
            k = k < 1 ? 1 : (k > tb.n - 1 ? tb.n - 1 : k);
        } else {
            int lo = 0, cnt = tb.n;   // lower_bound over lx
            while (cnt > 0) {
                const int st = cnt >> 1;
                if (tb.lx[lo + st] < lnE) { lo += st + 1; cnt -= st + 1; }
                else cnt = st;
            }
            k = lo < 1 ? 1 : (lo > tb.n - 1 ? tb.n - 1 : lo);
        }
        const float4 sg = tb.seg[k];
        const float t = __fmul_rn(__fsub_rn(lnE, sg.x), sg.y);
        const float d = __fmul_rn(__fmul_rn(p.nbdl2, sg.z), ex2a(__fmul_rn(t, sg.w)));
        kahan_add(a.T, a.Tc, d);
    }
}

// One path point (r, theta, dl, redshift) into every bin: the body of
// integrate_kerr_ray's point loop (radiative_transfer.cpp:501-672, UHE terms)
// for all bins at once.  Used by the fused trace kernel and by the kernel
// over cached paths.
template <int MIXED>
__device__ __forceinline__ void transfer_point(const DevCam* cam, const DevBin* bins, int B,
                                               const SmemTables& tb, const BinAcc& acc, double r,
                                               double th, double dl, double z)
{
    if (r < cam->rt_skip) return;   // radiative_transfer.cpp:501-505
    const double g = 1.0 / smax(z, 1.0e-300);
    const double gg = smax(g, 1.0e-300);
    const double dl_cm = dl * cam->rg_cm;
    if (MIXED) {
        PointRec pr;
        point_terms_body(cam, bins, B, r, th, gg, dl_cm, pr);
        for (int b = 0; b < B; ++b) {
            BinSums a = acc_load(acc, b);
            bin_point(pr, bin_k(bins[b]), b, tb, a);
            acc_store(acc, b, a);
        }
    } else {
        const double rho = torus_rho(cam->torus, r, th);
        const double C = emissivity_factor(cam->src, cam->torus, r, th, rho);
        const double g3 = pow(g, 3.0);
        for (int b = 0; b < B; ++b) {
            const double E_loc = bins[b].E_mid / gg;
            double jj = 0.0;
            if (!(E_loc <= 0.0)) jj = C * spectral_weight(cam->src, E_loc);
            double T = acc.T64[b * acc.st];
            acc.I64[b * acc.st] += g3 * jj * exp(-T) * dl_cm;
            if (rho <= 0.0 || E_loc < tb.Emin || E_loc > tb.Emax) continue;
            // SigmaTable::log_interp (sigma_table.cpp:81-124)
            int lo = 0, cnt = tb.n;
            while (cnt > 0) {
                const int st = cnt >> 1;
                if (tb.E[lo + st] < E_loc) { lo += st + 1; cnt -= st + 1; }
                else cnt = st;
            }
            double sigma_cm2;
            if (lo == 0) sigma_cm2 = tb.S[0];
            else if (lo == tb.n) sigma_cm2 = tb.S[tb.n - 1];
            else {
                const double lx = log(E_loc);
                const double lx1 = tb.lnE[lo - 1], lx2 = tb.lnE[lo];
                const double ly1 = tb.lnS[lo - 1], ly2 = tb.lnS[lo];
                const double t = (lx - lx1) / (lx2 - lx1);
                sigma_cm2 = exp(ly1 + t * (ly2 - ly1));
            }
            const double nb = rho / kMuG;
            T += nb * sigma_cm2 * dl_cm;
            acc.T64[b * acc.st] = T;
        }
    }
}

// A finished pixel: per-bin outputs, the spectral aggregates of
// integrate_kerr_ray_spectral (radiative_transfer.cpp:730-769; monochromatic:
// the single bin), defaults for an empty ray, fate, steps and attempts.
template <int MIXED>
__device__ __forceinline__ void finish_pixel(const TraceArgs& A, const DevCam* cam, const DevBin* bins,
                                             int B, const BinAcc& acc, long long local, int step,
                                             int fate, long long att_total)
{
    const long long orow = cam->out_offset + local;
    double t_out = 0.0, p_out = 1.0, i_out = 0.0;
    double wsum = 0.0, tsum = 0.0, psum = 0.0, isum = 0.0;
    for (int b = 0; b < B; ++b) {
        double tb, ib;
        if (MIXED) {
            const BinSums a = acc_load(acc, b);
            // tau = (T - Tc) ln 2;  I = (I - Ic) 2^-S w(E_mid), S integer-valued
            tb = (static_cast<double>(a.T) - static_cast<double>(a.Tc)) * kLn2;
            ib = ldexp(static_cast<double>(a.I) - static_cast<double>(a.Ic), -static_cast<int>(a.S)) * bins[b].w0;
        } else {
            tb = acc.T64[b * acc.st];
            ib = acc.I64[b * acc.st];
        }
        const long long e = cam->binout_offset + local * B + b;
        if (MIXED) {
            if (A.tau_E) static_cast<float*>(A.tau_E)[e] = static_cast<float>(tb);
        } else {
            if (A.tau_E) static_cast<double*>(A.tau_E)[e] = tb;
        }
        if (A.I_E) A.I_E[e] = ib;
        if (cam->mono) {
            t_out = tb; p_out = exp(-tb); i_out = ib;
        } else if (bins[b].valid) {   // radiative_transfer.cpp:752-769
            const double w = bins[b].w;
            wsum += w;
            tsum += w * tb;
            psum += w * exp(-tb);
            isum += ib * bins[b].dE;
        }
    }
    if (!cam->mono && wsum > 0.0) {
        t_out = tsum / wsum;
        p_out = psum / wsum;
        i_out = isum;
    }
    if (step == 0) { t_out = 0.0; p_out = 1.0; i_out = 0.0; }
    if (A.tau) A.tau[orow] = t_out;
    if (A.P_surv) A.P_surv[orow] = p_out;
    if (A.I_obs) A.I_obs[orow] = i_out;
    if (A.fate) A.fate[orow] = static_cast<int8_t>(fate);
    if (A.steps) A.steps[orow] = step;
    if (A.attempts) A.attempts[orow] = static_cast<int32_t>(att_total > 2147483647LL ? 2147483647LL : att_total);
}

// The MeV channel's outputs of a finished pixel: its sums, or RTResult's
// defaults for a camera without the channel (every kernel writes them, so a
// requested MeV output is never left unwritten).
__device__ __forceinline__ void finish_mev(const TraceArgs& A, const DevCam* cam, const MevAcc& ma, long long local,
                                           int step)
{
    const long long orow = cam->out_offset + local;
    double t, P, I, rn, lk;
    mev_finish(cam->mev, ma, step, &t, &P, &I, &rn, &lk);
    if (A.tau_mev) A.tau_mev[orow] = t;
    if (A.P_surv_mev) A.P_surv_mev[orow] = P;
    if (A.I_obs_mev) A.I_obs_mev[orow] = I;
    if (A.r_nu) A.r_nu[orow] = rn;
    if (A.leakage) A.leakage[orow] = lk;
}

// One path point into the MeV sums (points inside r_+ + 1e-3 are skipped as
// by the UHE transfer, radiative_transfer.cpp:501-505).
__device__ __forceinline__ void mev_path_point(const DevCam* cam, MevAcc& ma, double r, double th, double dl, double z)
{
    if (!cam->mev.on || r < cam->rt_skip) return;
    mev_point(cam->mev, ma, r, th, torus_rho(cam->torus, r, th), z, dl * cam->rg_cm);
}

// Zero this thread's per-bin accumulators.
template <int MIXED>
__device__ __forceinline__ void reset_bins(const BinAcc& acc, int B)
{
    for (int b = 0; b < B; ++b) {
        if (MIXED) {
            acc_store(acc, b, BinSums{0.0f, 0.0f, 0.0f, 0.0f, 0.0f});
        } else {
            acc.T64[b * acc.st] = 0.0; acc.I64[b * acc.st] = 0.0;
        }
    }
}

enum Phase : int { kNeedRay = 0, kStepStart = 1, kAttempt = 2, kDone = 3, kWaitTransfer = 4 };

// The warp's deferred transfer: every lane's buffered points (fill each, in
// order) go into that lane's ray's bins.  Each thread takes one lane's ray
// and kDeferBins consecutive bins of it (the warp's (lane, bin group) pairs
// are numbered through a prefix sum of the lanes' group counts), so every
// buffered point is loaded once for kDeferBins independent accumulation
// chains whose bin constants sit in registers.  The per-bin arithmetic and the
// point order are those of transfer_point, so the results are the same bits.
// Not inlined: called once every kRecDepth loop iterations, its registers are
// saved around the call instead of crowding the RKF45 attempt's.
// warp_slot0 is the slot of lane 0.
#ifndef HADROS_DEFER_BINS
#define HADROS_DEFER_BINS 4
#endif
constexpr int kDeferBins = HADROS_DEFER_BINS;

__device__ __noinline__ void deferred_transfer(PointRec* rec_buf, float* rec_state, const DevBin* bins, int bmax,
                                               const SmemTables tb, long long warp_slot0, int fill, int B,
                                               const DevCam* cam)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int ng = fill > 0 ? (B + kDeferBins - 1) / kDeferBins : 0;
    int pre = ng;   // inclusive prefix sum of the lanes' bin-group counts
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(full, pre, o);
        if (lane >= o) pre += v;
    }
    const int total = __shfl_sync(full, pre, 31);
    pre -= ng;      // exclusive
    for (int k0 = 0; k0 < total; k0 += 32) {
        const int k = k0 + lane;
        int src = 0;   // the last lane whose exclusive prefix is <= k
#pragma unroll
        for (int bit = 16; bit > 0; bit >>= 1) {
            const int cand = src + bit;
            const int pc = __shfl_sync(full, pre, cand & 31);
            if (cand < 32 && pc <= k) src = cand;
        }
        const int ps = __shfl_sync(full, pre, src);
        const int n_src = __shfl_sync(full, fill, src);
        const int B_src = __shfl_sync(full, B, src);
        const DevCam* cs = reinterpret_cast<const DevCam*>(
            __shfl_sync(full, reinterpret_cast<unsigned long long>(cam), src));
        const bool act = k < total;
        const int n = act ? n_src : 0;
        const int b0 = (k - ps) * kDeferBins;
        const long long sl = warp_slot0 + src;
        float* st = rec_state + sl * kAccF * bmax;
        const BinAcc sacc{nullptr, nullptr, st, bmax, 1};
        const PointRec* rb = rec_buf + sl * kRecDepth;
        BinSums a[kDeferBins];
        BinK bk[kDeferBins];
        bool on[kDeferBins];
#pragma unroll
        for (int j = 0; j < kDeferBins; ++j) {
            const int b = b0 + j;
            on[j] = act && b < B_src;
            a[j] = BinSums{0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
            bk[j] = BinK{0.0f, 0.0f, 0.0f};
            if (on[j]) {
                bk[j] = bin_k(bins[cs->bin_offset + b]);
                a[j] = acc_load(sacc, b);
            }
        }
        int nmax = n;
        for (int o = 16; o > 0; o >>= 1) nmax = max(nmax, __shfl_xor_sync(full, nmax, o));
        // the next record is loaded while the current one is applied: the
        // buffers mostly live beyond L2, and the loop is otherwise bound by
        // the latency of one record load per point
        PointRec nxt;
        if (n > 0) nxt = rb[0];
        for (int q = 0; q < nmax; ++q) {
            if (q < n) {
                const PointRec pr = nxt;
                if (q + 1 < n) nxt = rb[q + 1];
#pragma unroll
                for (int j = 0; j < kDeferBins; ++j)
                    if (on[j]) bin_point(pr, bk[j], b0 + j, tb, a[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < kDeferBins; ++j)
            if (on[j]) acc_store(sacc, b0 + j, a[j]);
    }
}

// DEFER (mixed only): the deferred transfer; a separate instantiation so the
// in-loop kernel carries none of its code or registers.  MEV: the MeV thermal
// channel (FP64, once per point), likewise only in the kernels that need it.
template <int MIXED, int FAST, int DEFER, int MEV>
__global__ void __launch_bounds__(kTPB, HADROS_MIN_BLOCKS) trace_kernel(const TraceArgs A)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int n_sig = A.sig.n;
    // deferred transfer keeps no per-bin accumulators in shared memory
    static_assert(!DEFER || MIXED, "the deferred transfer is mixed precision only");
    constexpr bool defer = DEFER != 0;
    const SmemLayout L = smem_layout(MIXED ? 1 : 0, n_sig, defer ? 0 : A.max_bins);
    double* sE = reinterpret_cast<double*>(smem + L.off_E);
    double* sS = reinterpret_cast<double*>(smem + L.off_S);
    double* slnE = reinterpret_cast<double*>(smem + L.off_lnE);
    double* slnS = reinterpret_cast<double*>(smem + L.off_lnS);
    float* slx = reinterpret_cast<float*>(smem + L.off_lx);
    float4* sseg = reinterpret_cast<float4*>(smem + L.off_seg);
    for (int k = threadIdx.x; k < n_sig; k += blockDim.x) {
        sE[k] = A.sig.E[k];
        sS[k] = A.sig.S[k];
        slnE[k] = A.sig.lnE[k];
        slnS[k] = A.sig.lnS[k];
        slx[k] = A.sig.lx[k];
        sseg[k] = reinterpret_cast<const float4*>(A.sig.seg)[k];
    }
    __syncthreads();
    const double sigEmin = A.sig.E_min, sigEmax = A.sig.E_max;
    const double sig_scale = A.sig.sigma_scale;

    const int tid = threadIdx.x;
    // per-bin accumulators of this thread's ray, column tid, stride kTPB
    double* accT64 = reinterpret_cast<double*>(smem + L.off_acc) + tid;
    double* accI64 = accT64 + size_t(kTPB) * A.max_bins;
    float* accF = reinterpret_cast<float*>(smem + L.off_acc) + tid;
    const SmemTables tb{sE, sS, slnE, slnS, slx, sseg, n_sig, sigEmin, sigEmax, sig_scale, A.sig.uniform, A.sig.lx0, A.sig.inv_dlx};
    const long long slot = static_cast<long long>(blockIdx.x) * kTPB + tid;   // deferred-transfer slot
    float* dstate = defer ? A.rec_state + slot * kAccF * A.rec_bmax : nullptr;
    const BinAcc acc = defer ? BinAcc{nullptr, nullptr, dstate, A.rec_bmax, 1}
                             : BinAcc{accT64, accI64, accF, long(kTPB) * A.max_bins, kTPB};
    PointRec* my_rec = defer ? A.rec_buf + slot * kRecDepth : nullptr;
    int fill = 0;          // points buffered in my_rec
    unsigned iter = 0;     // loop iterations (warp-uniform)

    int phase = kNeedRay;
    // ray state
    const DevCam* cam = nullptr;
    const DevBin* bins = nullptr;
    long long item = 0, local = 0, row = 0;
    int B = 1, step = 0, att_in_step = 0;
    long long att_total = 0;
    double a = 0.0, r = 0.0, th = 0.0, ph = 0.0, pr = 0.0, pth = 0.0, pt = 0.0, pph = 0.0;
    double r_prev = 0.0, th_prev = 0.0, ph_prev = 0.0, E_obs = 1.0, h = 0.0;
    K5 k1{};
    double s_base = 0.0, c_base = 1.0;   // sin/cos of theta at the step start
    int fate = HADROS_FATE_TRUNCATED;
    MevAcc ma;
    mev_reset(ma);

    while (true) {
        while (phase == kNeedRay || phase == kStepStart) {
            if (phase == kNeedRay) {
                {   // the lanes that need a ray now take consecutive items, one atomic per warp
                    const unsigned m = __activemask();
                    const int lane = threadIdx.x & 31;
                    const int leader = __ffs(m) - 1;
                    unsigned long long base = 0;
                    if (lane == leader) base = atomicAdd(&A.counters[0], static_cast<unsigned long long>(__popc(m)));
                    base = __shfl_sync(m, base, leader);
                    item = static_cast<long long>(base) + __popc(m & ((1u << lane) - 1u));
                }
                if (item >= A.total_items) {
                    phase = kDone;
                    break;
                }
                int ci = 0;
                if (A.n_cams > 1) {   // cameras are sorted by item range
                    int lo = 0, hi = A.n_cams - 1;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (A.cams[mid].item_begin <= item) lo = mid; else hi = mid - 1;
                    }
                    ci = lo;
                }
                cam = A.cams + ci;
                bins = A.bins + cam->bin_offset;
                B = cam->n_bins;
                local = item - cam->item_begin;
                const long long pid = A.pixel_ids ? static_cast<long long>(A.pixel_ids[item])
                                      : (A.order ? static_cast<long long>(A.order[item]) : local);
                row = A.order ? pid : local;   // output row within the camera
                const int nx = cam->nx;
                const int pi = static_cast<int>(pid % nx), pj = static_cast<int>(pid / nx);
                // KerrCamera::initial_state (kerr_camera.cpp:110-186)
                a = cam->a;
                const double u = (2.0 * (pi + 0.5) / nx - 1.0) * cam->tan_half;
                const double v = (2.0 * (pj + 0.5) / cam->ny - 1.0) * cam->tan_half;
                const double norm = sqrt(1.0 + u * u + v * v);
                const double n_r = -1.0 / norm;
                const double n_theta = v / norm;
                const double n_phi = u / norm;
                const double p_t_c = cam->pt_contra;
                const double p_r_c = n_r / cam->sq_grr;
                const double p_th_c = n_theta / cam->sq_gthth;
                const double p_ph_c = n_phi / cam->sq_gphph + cam->omega_obs * p_t_c;
                pt = cam->g_tt * p_t_c + cam->g_tph * p_ph_c;
                pr = cam->g_rr * p_r_c;
                pth = cam->g_thth * p_th_c;
                pph = cam->g_tph * p_t_c + cam->g_phph * p_ph_c;
                r = cam->r_obs;
                th = cam->th_obs;
                ph = 0.0;
                r_prev = r;
                th_prev = th;
                ph_prev = ph;
                // zamo_energy at the observer (kerr_camera.cpp:16-29, :206-213)
                E_obs = -(pt + cam->omega_obs * pph) / cam->alpha_obs;
                step = 0;
                att_total = 0;
                reset_bins<MIXED>(acc, B);
                if (MEV) mev_reset(ma);
                phase = kStepStart;
            }

            // ---- step start: stop tests, path point, transfer, k1 ----------
            bool stop = false;
            if (step >= cam->max_steps) { fate = HADROS_FATE_TRUNCATED; stop = true; }
            else if (r <= cam->r_stop) { fate = HADROS_FATE_CAPTURED; stop = true; }
            else if (r >= cam->r_max && step > 10) { fate = HADROS_FATE_ESCAPED; stop = true; }
            else if (A.attempt_budget > 0 && att_total > A.attempt_budget) {
                fate = 3;   // aborted by the attempt budget
                atomicAdd(&A.counters[3], 1ULL);
                stop = true;
            }
            if (stop) {
                atomicAdd(&A.counters[1], static_cast<unsigned long long>(step));
                atomicAdd(&A.counters[2], static_cast<unsigned long long>(att_total));
                if (defer) {   // finished at the warp's next transfer
                    phase = kWaitTransfer;
                    continue;
                }
                finish_pixel<MIXED>(A, cam, bins, B, acc, row, step, fate, att_total);
                finish_mev(A, cam, ma, row, step);
                phase = kNeedRay;
                continue;
            }

            double s, c;
            crm::DD sd{0.0, 0.0}, cd{1.0, 0.0};
            if (FAST) {
                sincos(th, &s, &c);
            } else {
                sincos_dd(th, &sd, &cd);
                s = sd.h;
                c = cd.h;
            }
            // PathPoint (kerr_camera.cpp:245-273): ZAMO interval and redshift
            double dl = 0.0;
            double z;
            if (FAST) {
                // the same interval and redshift with reciprocals instead of
                // IEEE divisions and sin/cos of the midpoint by angle shift
                const double a2 = a * a;
                if (step != 0) {
                    const double r_mid = 0.5 * (r + r_prev);
                    const double th_mid = 0.5 * (th + th_prev);
                    double sm, cm;
                    const double dmid = th_mid - th;
                    if (fabs(dmid) < 0.05) sincos_shift(s, c, dmid, &sm, &cm);
                    else sincos(th_mid, &sm, &cm);
                    const double r2 = r_mid * r_mid, s2 = sm * sm;
                    const double sig = r2 + a2 * cm * cm;
                    const double del = r2 - 2.0 * r_mid + a2;
                    const double grr = sig * rcp_nr(del);
                    const double gpp = (r2 + a2 + 2.0 * a2 * r_mid * s2 * rcp_nr(sig)) * s2;
                    const double dr = r - r_prev;
                    const double dth = th - th_prev;
                    const double dph = wrapped_dphi(ph, ph_prev);
                    const double dl2 = grr * dr * dr + sig * dth * dth + gpp * dph * dph;
                    dl = sqrt(smax(dl2, 0.0));
                }
                const double r2 = r * r;
                const double sig = r2 + a2 * c * c;
                const double del = r2 - 2.0 * r + a2;
                const double rpa = r2 + a2;
                const double inv_A = rcp_nr(rpa * rpa - a2 * del * s * s);
                const double alpha = sqrt(sig * del * inv_A);
                const double omega = 2.0 * a * r * inv_A;
                z = -(pt + omega * pph) * rcp_nr(alpha) * rcp_nr(smax(E_obs, 1.0e-300));
            } else {
                if (step != 0) {
                    const double r_mid = 0.5 * (r + r_prev);
                    const double th_mid = 0.5 * (th + th_prev);
                    crm::DD smd, cmd;
                    sincos_dd(th_mid, &smd, &cmd);
                    const double sm = smd.h, cm = cmd.h;
                    M5 gmid;
                    bl_metric(a, r_mid, sm, cm, gmid);
                    const double dr = r - r_prev;
                    const double dth = th - th_prev;
                    const double dph = wrapped_dphi(ph, ph_prev);
                    const double dl2 = gmid.rr * dr * dr + gmid.thth * dth * dth + gmid.phph * dph * dph;
                    dl = sqrt(smax(dl2, 0.0));
                }
                const double alpha = bl_lapse(a, r, s, c);
                const double omega = bl_omega(a, r, s);
                z = (-(pt + omega * pph) / alpha) / smax(E_obs, 1.0e-300);
            }
            if (A.paths && step < A.path_cap) {   // PathPoint record (kerr_camera.cpp:235-273)
                double sph, cph;
                sincos(ph, &sph, &cph);
                double* q = A.paths + ((cam->out_offset + row) * static_cast<long long>(A.path_cap) + step) * 7;
                q[0] = r;
                q[1] = th;
                q[2] = r * s * cph;
                q[3] = r * s * sph;
                q[4] = r * c;
                q[5] = dl;
                q[6] = z;
            }

            // ---- transfer of this point into every bin ------------------
            if (defer) {
                PointRec pr;
                if (point_terms(cam, bins, B, r, th, dl, z, pr)) my_rec[fill++] = pr;
            } else {
                transfer_point<MIXED>(cam, bins, B, tb, acc, r, th, dl, z);
            }
            if (MEV) mev_path_point(cam, ma, r, th, dl, z);

            // ---- k1 of the coming step_adaptive (shares sin/cos) ------------
            if (FAST) geo_rhs_fast(a, r, th, s, c, pr, pth, pt, pph, k1);
            else geo_rhs(a, r, th, sd, cd, pr, pth, pt, pph, k1);
            r_prev = r;
            th_prev = th;
            ph_prev = ph;
            s_base = s;
            c_base = c;
            h = cam->h0;
            att_in_step = 0;
            phase = kAttempt;
        }

        if (defer) {
            // Every kRecDepth iterations (each adds at most one point per lane),
            // or when no lane has a ray in flight, the warp replays every lane's
            // buffered points into its bins, then finishes the waiting rays.
            ++iter;
            const bool idle = __all_sync(0xffffffffu, phase == kDone || phase == kWaitTransfer);
            if (iter % kRecDepth == 0 || idle) {
                deferred_transfer(A.rec_buf, A.rec_state, A.bins, A.rec_bmax, tb, slot - (tid & 31), fill, B, cam);
                if (phase == kWaitTransfer) {
                    finish_pixel<MIXED>(A, cam, bins, B, acc, row, step, fate, att_total);
                    finish_mev(A, cam, ma, row, step);
                    phase = kNeedRay;
                }
                fill = 0;
            }
        }
        if (__all_sync(0xffffffffu, phase == kDone)) break;
        if (phase != kAttempt) continue;

        // ---- one RKF45 attempt (kerr_geodesic.cpp:239-326) -----------------
        // Stage coefficients h * a_ij (:241-308): the camera's values at
        // h = h0 on a step's first attempt, else formed from h, each where its
        // stage uses it so that none stays live across the attempt.  The phi
        // components of k enter only y4 and y5: their weighted sums are
        // accumulated as the stages produce them, in the reference's order.
        const bool first = att_in_step == 0;
        const double* c0 = cam->c0;
#define HAD_CF(q, num, den) (first ? c0[q] : h * (num) / (den))
#define HAD_CFM(q, num) (first ? c0[q] : h * (num))
        double s4p = A1 * k1.ph, s5p = B1 * k1.ph;   // y4, y5 phi sums so far
        K5 k2, k3, k4, k5, k6;
        {
            const double c = HAD_CF(0, 1.0, 4.0);
            geo_rhs_sel<FAST>(a, r + c * k1.r, th + c * k1.th, pr + c * k1.pr, pth + c * k1.pth, pt, pph, k2,
                              th, s_base, c_base);
        }
        {
            const double c1 = HAD_CF(1, 3.0, 32.0), c2 = HAD_CF(2, 9.0, 32.0);
            geo_rhs_sel<FAST>(a, r + c1 * k1.r + c2 * k2.r, th + c1 * k1.th + c2 * k2.th,
                              pr + c1 * k1.pr + c2 * k2.pr, pth + c1 * k1.pth + c2 * k2.pth, pt, pph, k3, th,
                              s_base, c_base);
        }
        s4p = s4p + A3 * k3.ph;
        s5p = s5p + B3 * k3.ph;
        {
            const double c3 = HAD_CF(3, 1932.0, 2197.0), c4 = HAD_CF(4, -7200.0, 2197.0),
                         c5 = HAD_CF(5, 7296.0, 2197.0);
            geo_rhs_sel<FAST>(a, r + c3 * k1.r + c4 * k2.r + c5 * k3.r, th + c3 * k1.th + c4 * k2.th + c5 * k3.th,
                              pr + c3 * k1.pr + c4 * k2.pr + c5 * k3.pr,
                              pth + c3 * k1.pth + c4 * k2.pth + c5 * k3.pth, pt, pph, k4, th, s_base, c_base);
        }
        s4p = s4p + A4 * k4.ph;
        s5p = s5p + B4 * k4.ph;
        {
            const double c6 = HAD_CF(6, 439.0, 216.0), c7 = HAD_CFM(7, -8.0), c8 = HAD_CF(8, 3680.0, 513.0),
                         c9 = HAD_CF(9, -845.0, 4104.0);
            geo_rhs_sel<FAST>(a, r + c6 * k1.r + c7 * k2.r + c8 * k3.r + c9 * k4.r,
                              th + c6 * k1.th + c7 * k2.th + c8 * k3.th + c9 * k4.th,
                              pr + c6 * k1.pr + c7 * k2.pr + c8 * k3.pr + c9 * k4.pr,
                              pth + c6 * k1.pth + c7 * k2.pth + c8 * k3.pth + c9 * k4.pth, pt, pph, k5, th,
                              s_base, c_base);
        }
        s4p = s4p - A5 * k5.ph;
        s5p = s5p - B5 * k5.ph;
        {
            const double c10 = HAD_CF(10, -8.0, 27.0), c11 = HAD_CFM(11, 2.0), c12 = HAD_CF(12, -3544.0, 2565.0),
                         c13 = HAD_CF(13, 1859.0, 4104.0), c14 = HAD_CF(14, -11.0, 40.0);
            geo_rhs_sel<FAST>(a, r + c10 * k1.r + c11 * k2.r + c12 * k3.r + c13 * k4.r + c14 * k5.r,
                              th + c10 * k1.th + c11 * k2.th + c12 * k3.th + c13 * k4.th + c14 * k5.th,
                              pr + c10 * k1.pr + c11 * k2.pr + c12 * k3.pr + c13 * k4.pr + c14 * k5.pr,
                              pth + c10 * k1.pth + c11 * k2.pth + c12 * k3.pth + c13 * k4.pth + c14 * k5.pth, pt,
                              pph, k6, th, s_base, c_base);
        }
        s5p = s5p + B6 * k6.ph;
#undef HAD_CF
#undef HAD_CFM
#define HAD_Y4(f) (A1 * k1.f + A3 * k3.f + A4 * k4.f - A5 * k5.f)
#define HAD_Y5(f) (B1 * k1.f + B3 * k3.f + B4 * k4.f - B5 * k5.f + B6 * k6.f)
        const double y4r = r + h * HAD_Y4(r), y5r = r + h * HAD_Y5(r);
        const double y4t = th + h * HAD_Y4(th), y5t = th + h * HAD_Y5(th);
        const double y4p = ph + h * s4p, y5p = ph + h * s5p;
        const double y4pr = pr + h * HAD_Y4(pr), y5pr = pr + h * HAD_Y5(pr);
        const double y4pt = pth + h * HAD_Y4(pth), y5pt = pth + h * HAD_Y5(pth);
#undef HAD_Y4
#undef HAD_Y5
        double err = 0.0;   // error_norm (kerr_geodesic.cpp:219-233); p_phi term is 0
        err = smax(err, fabs(y4r - y5r));
        err = smax(err, fabs(y4t - y5t));
        err = smax(err, fabs(y4p - y5p));
        err = smax(err, fabs(y4pr - y5pr));
        err = smax(err, fabs(y4pt - y5pt));
        err = smax(err, 0.0);
        ++att_total;
        const double h_min = cam->h_min;
        if (err < cam->tol || h <= h_min) {
            r = y5r; th = y5t; ph = y5p; pr = y5pr; pth = y5pt;
            ++step;
            phase = kStepStart;
        } else {
            const double factor = 0.8 * crm::pow025_rn(cam->tol / smax(err, 1.0e-30));
            h *= sclamp(factor, 0.1, 5.0);
            if (h < h_min) h = h_min;
            ++att_in_step;
            if (att_in_step == 50) {   // step_rk4 with h0 (kerr_geodesic.cpp:137-192, :328)
                const double h0 = cam->h0;
                K5 q2, q3, q4;
                geo_rhs_sel<FAST>(a, r + 0.5 * h0 * k1.r, th + 0.5 * h0 * k1.th, pr + 0.5 * h0 * k1.pr,
                           pth + 0.5 * h0 * k1.pth, pt, pph, q2, th, s_base, c_base);
                geo_rhs_sel<FAST>(a, r + 0.5 * h0 * q2.r, th + 0.5 * h0 * q2.th, pr + 0.5 * h0 * q2.pr,
                           pth + 0.5 * h0 * q2.pth, pt, pph, q3, th, s_base, c_base);
                geo_rhs_sel<FAST>(a, r + h0 * q3.r, th + h0 * q3.th, pr + h0 * q3.pr, pth + h0 * q3.pth,
                           pt, pph, q4, th, s_base, c_base);
                r += h0 * (k1.r + 2.0 * q2.r + 2.0 * q3.r + q4.r) / 6.0;
                th += h0 * (k1.th + 2.0 * q2.th + 2.0 * q3.th + q4.th) / 6.0;
                ph += h0 * (k1.ph + 2.0 * q2.ph + 2.0 * q3.ph + q4.ph) / 6.0;
                pr += h0 * (k1.pr + 2.0 * q2.pr + 2.0 * q3.pr + q4.pr) / 6.0;
                pth += h0 * (k1.pth + 2.0 * q2.pth + 2.0 * q3.pth + q4.pth) / 6.0;
                ++att_total;
                ++step;
                phase = kStepStart;
            }
        }
    }
}


// Transfer over cached paths (compute_kerr_image_from_cache,
// apps/compute_kerr_image_from_cache.cpp:599-711): one thread per ray walks
// its recorded points (r, theta, x, y, z, dl, redshift) through the same
// transfer_point (and MeV channel) as the fused kernel.  Grid-stride over rays.
template <int MIXED, int MEV>
__global__ void __launch_bounds__(kTPB) path_transfer_kernel(const TraceArgs A)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int n_sig = A.sig.n;
    const SmemLayout L = smem_layout(MIXED ? 1 : 0, n_sig, A.max_bins);
    double* sE = reinterpret_cast<double*>(smem + L.off_E);
    double* sS = reinterpret_cast<double*>(smem + L.off_S);
    double* slnE = reinterpret_cast<double*>(smem + L.off_lnE);
    double* slnS = reinterpret_cast<double*>(smem + L.off_lnS);
    float* slx = reinterpret_cast<float*>(smem + L.off_lx);
    float4* sseg = reinterpret_cast<float4*>(smem + L.off_seg);
    for (int k = threadIdx.x; k < n_sig; k += blockDim.x) {
        sE[k] = A.sig.E[k];
        sS[k] = A.sig.S[k];
        slnE[k] = A.sig.lnE[k];
        slnS[k] = A.sig.lnS[k];
        slx[k] = A.sig.lx[k];
        sseg[k] = reinterpret_cast<const float4*>(A.sig.seg)[k];
    }
    __syncthreads();
    const int tid = threadIdx.x;
    double* accT64 = reinterpret_cast<double*>(smem + L.off_acc) + tid;
    double* accI64 = accT64 + size_t(kTPB) * A.max_bins;
    float* accF = reinterpret_cast<float*>(smem + L.off_acc) + tid;
    const SmemTables tb{sE, sS, slnE, slnS, slx, sseg, n_sig, A.sig.E_min, A.sig.E_max, A.sig.sigma_scale, A.sig.uniform, A.sig.lx0, A.sig.inv_dlx};
    const BinAcc acc{accT64, accI64, accF, long(kTPB) * A.max_bins, kTPB};
    const DevCam* cam = A.cams;
    const DevBin* bins = A.bins + cam->bin_offset;
    const int B = cam->n_bins;
    for (long long ray = static_cast<long long>(blockIdx.x) * kTPB + tid; ray < A.total_items;
         ray += static_cast<long long>(gridDim.x) * kTPB) {
        reset_bins<MIXED>(acc, B);
        MevAcc ma;
        mev_reset(ma);
        const long long k0 = A.path_offsets[ray], k1 = A.path_offsets[ray + 1];
        for (long long kk = k0; kk < k1; ++kk) {
            const double* q = A.path_points + kk * 7;
            transfer_point<MIXED>(cam, bins, B, tb, acc, q[0], q[1], q[5], q[6]);
            if (MEV) mev_path_point(cam, ma, q[0], q[1], q[5], q[6]);
        }
        const int fate = A.path_fates ? A.path_fates[ray] : HADROS_FATE_ESCAPED;
        finish_pixel<MIXED>(A, cam, bins, B, acc, ray, static_cast<int>(k1 - k0), fate, 0);
        finish_mev(A, cam, ma, ray, static_cast<int>(k1 - k0));
    }
}

// Grid-stride launch of the cached-path kernel; FAST only selects the
// translation unit (FMA contraction or not), like the trace kernel's.
template <int FAST>
int launch_paths(const TraceArgs& args, int precision, int n_sm, cudaStream_t st, std::string& err)
{
    const size_t smem = smem_layout(precision, args.sig.n, args.max_bins).total;
    const bool mixed = precision == HADROS_PRECISION_MIXED;
    auto kern = args.mev ? (mixed ? path_transfer_kernel<1, 1> : path_transfer_kernel<0, 1>)
                         : (mixed ? path_transfer_kernel<1, 0> : path_transfer_kernel<0, 0>);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTPB, smem);
    if (e != cudaSuccess || per_sm < 1) {
        err = std::string("path transfer kernel setup: ") + cudaGetErrorString(e);
        return HADROS_E_CUDA;
    }
    long long grid = static_cast<long long>(n_sm) * per_sm;
    const long long needed = (args.total_items + kTPB - 1) / kTPB;
    if (grid > needed) grid = needed > 0 ? needed : 1;
    if (args.rec_buf && grid * kTPB > args.rec_slots) grid = args.rec_slots / kTPB;   // one slot per thread
    kern<<<static_cast<unsigned>(grid), kTPB, smem, st>>>(args);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("path transfer kernel launch: ") + cudaGetErrorString(e);
        return HADROS_E_CUDA;
    }
    return HADROS_OK;
}

// The trace kernel instantiation for a precision, transfer placement and
// MeV channel.
template <int FAST, int MEV>
auto trace_kernel_mev(const TraceArgs& args, int precision) -> void (*)(const TraceArgs)
{
    if (precision != HADROS_PRECISION_MIXED) return trace_kernel<0, FAST, 0, MEV>;
    return args.rec_buf ? trace_kernel<1, FAST, 1, MEV> : trace_kernel<1, FAST, 0, MEV>;
}

template <int FAST>
auto trace_kernel_for(const TraceArgs& args, int precision) -> void (*)(const TraceArgs)
{
    return args.mev ? trace_kernel_mev<FAST, 1>(args, precision) : trace_kernel_mev<FAST, 0>(args, precision);
}

// Grid of a persistent launch: SMs x resident blocks (capped at
// blocks_per_sm when > 0), no more blocks than the work needs.
template <int FAST>
int prepare_variant(const TraceArgs& args, int precision, int n_sm, int blocks_per_sm, LaunchCfg& cfg,
                    std::string& err)
{
    cfg.smem = smem_layout(precision, args.sig.n, args.rec_buf ? 0 : args.max_bins).total;
    auto kern = trace_kernel_for<FAST>(args, precision);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTPB, cfg.smem);
    if (e != cudaSuccess) {
        err = std::string("trace kernel setup: ") + cudaGetErrorString(e);
        return HADROS_E_CUDA;
    }
    if (per_sm < 1) {
        err = "trace kernel does not fit on an SM (shared memory for sigma table and bins)";
        return HADROS_E_ARG;
    }
    if (blocks_per_sm > 0 && blocks_per_sm < per_sm) per_sm = blocks_per_sm;
    long long grid = static_cast<long long>(n_sm) * per_sm;
    const long long needed = (args.total_items + kTPB - 1) / kTPB;
    if (grid > needed) grid = needed > 0 ? needed : 1;
    if (args.rec_buf && grid * kTPB > args.rec_slots) grid = args.rec_slots / kTPB;   // one slot per thread
    cfg.grid = static_cast<unsigned>(grid);
    cfg.per_sm = per_sm;
    return HADROS_OK;
}

// Enqueue only the kernel (no host work): capturable in a CUDA graph.
template <int FAST>
int launch_prepared_variant(const TraceArgs& args, int precision, const LaunchCfg& cfg, cudaStream_t st,
                            std::string& err)
{
    auto kern = trace_kernel_for<FAST>(args, precision);
    kern<<<cfg.grid, kTPB, cfg.smem, st>>>(args);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("trace kernel launch: ") + cudaGetErrorString(e);
        return HADROS_E_CUDA;
    }
    return HADROS_OK;
}

// Occupancy-sized persistent launch of one kernel variant.
template <int FAST>
int launch_variant(const TraceArgs& args, int precision, int n_sm, cudaStream_t st, std::string& err)
{
    LaunchCfg cfg{};
    const int rc = prepare_variant<FAST>(args, precision, n_sm, args.blocks_per_sm, cfg, err);
    if (rc) return rc;
    return launch_prepared_variant<FAST>(args, precision, cfg, st, err);
}

}  // namespace

}  // namespace hadros
