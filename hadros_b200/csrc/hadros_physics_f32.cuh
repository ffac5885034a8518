// hadros_physics_f32.cuh — FP32 density and log-emissivity for the mixed-
// precision transfer (device only).
//
// Same formulas as hadros_physics.cuh (TorusProfile::rho, src/torus_profile.cpp:
// 150-272; the UHE source morphologies, src/radiative_transfer.cpp:209-395),
// with the smooth factors in FP32 on the MUFU unit and every cut, guard and
// range test still decided on the FP64 coordinates.  Divisions by parameters
// are replaced by host-computed reciprocals.  The emissivity is returned as
// ln C, built from the exponents directly (a Gaussian factor exp(-x^2)
// contributes -x^2; the bipolar sum goes through log-sum-exp), so a source
// tail far below FP32's range still carries its exact logarithm.
#pragma once

#include "hadros_physics.cuh"

namespace hadros {

// FP32 constants of a Torus (filled by make_torus_f on the host).
struct TorusF {
    float rho0, r0, inv_r0, inv_sr, inv_H, r_min, inv_rmax, rp, fdep, inv_fth, env_rho0, env_alpha,
        floor;
    // collapsar_ndaf_like
    float inv_H6, inv_s035, inv_s060, r0_075, inv_s075, inv_s18, rp_pos;
};

struct SourceF {
    float ln_norm, rc, inv_sr, inv_tw, th_mid, fth, inv_rc, q, s, ln_lo, ln_hi, inv_rho_norm;
    float gdr, gdth, inv_2gdr, inv_2gdth;
};

inline TorusF make_torus_f(const Torus& t)
{
    TorusF f{};
    f.rho0 = static_cast<float>(t.rho0);
    f.r0 = static_cast<float>(t.r0);
    f.inv_r0 = static_cast<float>(1.0 / t.r0);
    f.inv_sr = static_cast<float>(1.0 / t.sigma_r);
    f.inv_H = static_cast<float>(1.0 / t.H);
    f.r_min = static_cast<float>(t.r_min);
    f.inv_rmax = static_cast<float>(1.0 / t.r_max);
    f.rp = static_cast<float>(t.radial_power);
    f.fdep = static_cast<float>(t.funnel_depletion);
    f.inv_fth = static_cast<float>(1.0 / t.funnel_theta);
    f.env_rho0 = static_cast<float>(t.env_rho0);
    f.env_alpha = static_cast<float>(t.env_alpha);
    f.floor = static_cast<float>(t.rho_floor);
    f.inv_H6 = static_cast<float>(1.0 / smax(t.H, 1.0e-6));
    f.inv_s035 = static_cast<float>(1.0 / smax(0.35 * t.sigma_r, 1.0e-6));
    f.inv_s060 = static_cast<float>(1.0 / smax(0.60 * t.sigma_r, 1.0e-6));
    f.r0_075 = static_cast<float>(0.75 * t.r0);
    f.inv_s075 = static_cast<float>(1.0 / smax(0.75 * t.sigma_r, 1.0e-6));
    f.inv_s18 = static_cast<float>(1.0 / smax(1.8 * t.sigma_r, 1.0e-6));
    f.rp_pos = static_cast<float>(smax(t.radial_power, 0.0));
    return f;
}

inline SourceF make_source_f(const Source& s)
{
    SourceF f{};
    f.ln_norm = s.norm > 0.0 ? static_cast<float>(std::log(s.norm)) : -INFINITY;
    f.rc = static_cast<float>(s.r_center);
    f.inv_sr = s.sigma_r > 0.0 ? static_cast<float>(1.0 / s.sigma_r) : 0.0f;
    f.inv_tw = s.theta_width > 0.0 ? static_cast<float>(1.0 / s.theta_width) : 0.0f;
    f.th_mid = static_cast<float>(0.5 * kPi);
    f.fth = static_cast<float>(s.funnel_theta);
    f.inv_rc = static_cast<float>(1.0 / smax(s.r_center, 1.0e-300));
    f.q = static_cast<float>(s.q);
    f.s = static_cast<float>(s.s);
    const double lo = smax(s.cutoff_lo, 0.0), hi = smax(s.cutoff_hi, smax(s.cutoff_lo, 0.0));
    f.ln_lo = lo > 0.0 ? static_cast<float>(std::log(lo)) : -INFINITY;
    f.ln_hi = hi > 0.0 ? static_cast<float>(std::log(hi)) : -INFINITY;
    f.inv_rho_norm = static_cast<float>(1.0 / s.rho_norm);
    f.gdr = static_cast<float>(smax(s.grad_dr, 1.0e-4));
    f.gdth = static_cast<float>(smax(s.grad_dtheta, 1.0e-5));
    f.inv_2gdr = static_cast<float>(1.0 / (2.0 * smax(s.grad_dr, 1.0e-4)));
    f.inv_2gdth = static_cast<float>(1.0 / (2.0 * smax(s.grad_dtheta, 1.0e-5)));
    return f;
}

#ifdef __CUDACC__

// x^y for x > 0 (callers guarantee it), on MUFU.
__device__ __forceinline__ float powf_pos(float x, float y) { return exp2f(y * __log2f(x)); }

__device__ __forceinline__ float gauss_f(float x) { return __expf(-(x * x)); }

// TorusProfile::rho with FP32 smooth factors; cuts on the FP64 coordinates.
__device__ __forceinline__ float torus_rho_f(const Torus& t, const TorusF& f, double r, double th)
{
    const float rf = static_cast<float>(r), thf = static_cast<float>(th);
    float shape = 0.0f;
    const bool in_torus = (r >= t.r_min && r <= t.r_max);
    if (t.kind == 7) {   // collapsar_ndaf_like (:150-179)
        if (in_torus && !(r <= 0.0) && !(t.r0 <= 0.0)) {
            const float vertical = gauss_f(__cosf(thf) * f.inv_H6);
            const float inner = 1.0f / (1.0f + __expf(-(rf - f.r_min) * f.inv_s035));
            const float outer = 1.0f / (1.0f + __expf((rf - static_cast<float>(t.r_max)) * f.inv_s060));
            const float core = 0.45f * gauss_f((rf - f.r0_075) * f.inv_s075);
            const float radial = powf_pos(fmaxf(rf * f.inv_r0, 1.0e-30f), -f.rp_pos);
            const float tail = 0.08f * gauss_f((rf - f.r0) * f.inv_s18);
            shape = (radial + core + tail) * vertical * inner * outer;
        }
    } else if (t.use_powerlaw) {   // :198-217
        if (in_torus && !(r <= 0.0) && !(t.r0 <= 0.0)) {
            const float vertical = gauss_f(__cosf(thf) * f.inv_H);
            const float inner = 1.0f - gauss_f((rf - f.r_min) * f.inv_sr);
            const float x = rf * f.inv_rmax;
            const float outer = __expf(-((x * x) * (x * x)));
            const float radial = powf_pos(rf * f.inv_r0, -f.rp);
            shape = radial * vertical * inner * outer;
        }
    } else {   // gaussian (:181-196): hard cuts on the FP64 values
        const double delta = th - 0.5 * kPi;
        if (!(r <= 4.0 || r >= 18.0 || fabs(delta) >= 0.45))
            shape = gauss_f((rf - f.r0) * f.inv_sr) * gauss_f(static_cast<float>(delta) * f.inv_H);
    }
    float funnel = 1.0f;
    if (t.use_funnel) {   // :219-236
        const float n = gauss_f(thf * f.inv_fth);
        const float s = gauss_f((static_cast<float>(kPi) - thf) * f.inv_fth);
        funnel = fminf(fmaxf(1.0f - f.fdep * (n + s), 0.0f), 1.0f);
    }
    float env = 0.0f;
    if (t.use_envelope && !(t.env_rho0 <= 0.0) && !(r < t.r0) && !(r > t.r_max))   // :238-248
        env = f.env_rho0 * powf_pos(rf * f.inv_r0, -f.env_alpha);
    return fmaxf(f.rho0 * shape * funnel + env, f.floor);
}

// ln(exp(-a) + exp(-b)) for a, b >= 0.
__device__ __forceinline__ float ln_sum_gauss(float a, float b)
{
    const float m = fminf(a, b);
    return -m + __logf(__expf(m - a) + __expf(m - b));
}

// ln C of emissivity_factor (hadros_physics.cuh) in FP32: -INFINITY for none.
__device__ __forceinline__ float ln_emission_f(const Source& s, const SourceF& sf, const Torus& t,
                                               const TorusF& tf, double r, double th, float rho)
{
    const float rf = static_cast<float>(r), thf = static_cast<float>(th);
    if (s.kind == 0) {   // inner ring (radiative_transfer.cpp:335-367)
        if (s.r_center <= 0.0 || s.sigma_r <= 0.0 || s.theta_width <= 0.0 || s.emax <= 0.0) return -INFINITY;
        const float dr = (rf - sf.rc) * sf.inv_sr;
        const float dth = static_cast<float>(th - 0.5 * kPi) * sf.inv_tw;
        return sf.ln_norm - dr * dr - dth * dth;
    }
    if (r <= 0.0 || s.sigma_r <= 0.0 || s.theta_width <= 0.0) return -INFINITY;
    if (s.kind == 1) {   // funnel wall (:240-248)
        const float dr = (rf - sf.rc) * sf.inv_sr;
        const float n = (thf - sf.fth) * sf.inv_tw;
        const float so = (thf - (static_cast<float>(kPi) - sf.fth)) * sf.inv_tw;
        return sf.ln_norm - dr * dr + ln_sum_gauss(n * n, so * so);
    }
    if (s.kind == 2) {   // jet base (:250-256)
        const float x = rf * sf.inv_rc;
        const float n = thf * sf.inv_tw;
        const float so = (thf - static_cast<float>(kPi)) * sf.inv_tw;
        return sf.ln_norm - x * x + ln_sum_gauss(n * n, so * so);
    }
    if (s.kind == 4) {   // density weighted (:258-280)
        const float w = fmaxf(rho * sf.inv_rho_norm, 0.0f);
        const float lw = (w > 0.0f) ? sf.q * __logf(w) : (sf.q > 0.0f ? -INFINITY : (sf.q < 0.0f ? INFINITY : 0.0f));
        const float lr = -sf.s * __logf(fmaxf(rf * sf.inv_rc, 1.0e-30f));
        const float v = fminf(fmaxf(lw + lr, sf.ln_lo), sf.ln_hi);
        return sf.ln_norm + v;
    }
    if (s.kind == 3) {   // shock layer (:282-332): gradient of rho, FP32
        const double r_minus = smax(r - smax(s.grad_dr, 1.0e-4), 1.0e-6);
        const double dth = smax(s.grad_dtheta, 1.0e-5);
        const double th_m = sclamp(th - dth, 0.0, kPi), th_p = sclamp(th + dth, 0.0, kPi);
        const float rp = torus_rho_f(t, tf, r + smax(s.grad_dr, 1.0e-4), th);
        const float rm = torus_rho_f(t, tf, r_minus, th);
        const float tp = torus_rho_f(t, tf, r, th_p);
        const float tm = torus_rho_f(t, tf, r, th_m);
        const float d_r = (rp - rm) * sf.inv_2gdr;
        const float d_t = (tp - tm) * sf.inv_2gdth / fmaxf(rf, 1.0e-6f);
        const float grad = sqrtf(d_r * d_r + d_t * d_t) * sf.inv_rho_norm;
        const float x = rf * sf.inv_rc;
        const float lg = (grad > 0.0f) ? __logf(grad) - x * x : -INFINITY;
        return sf.ln_norm + fminf(fmaxf(lg, sf.ln_lo), sf.ln_hi);
    }
    return -INFINITY;
}

#endif  // __CUDACC__

}  // namespace hadros
