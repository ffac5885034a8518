// hadros_physics.cuh — Kerr metric, density profiles, UHE sources and spectra
// as __host__ __device__ functions.
//
// The host side (camera plans, per-camera constants) and the sm_100a trace
// kernel include the same code.  Expressions keep the reference's operand
// order (no reassociation; device code is compiled with --fmad=false) so the
// FP64 path differs from the reference CPU only through the transcendental
// functions of the two math libraries.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define HD __host__ __device__ __forceinline__
#else
#define HD inline
#endif

namespace hadros {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kLog2E = 1.442695040888963407359924681001892137;   // log2(e)
constexpr double kLn2 = 0.693147180559945309417232121458176568;     // ln(2)
// include/constants.hpp:9-13
constexpr double kCcgs = 2.99792458e10;
constexpr double kGcgs = 6.67430e-8;
constexpr double kMsunG = 1.98847e33;
constexpr double kMuG = 1.66053906660e-24;

// std::max / std::min / std::clamp, NaN behaviour included.
HD double smax(double a, double b) { return (a < b) ? b : a; }
HD double smin(double a, double b) { return (b < a) ? b : a; }
HD double sclamp(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

// Nonzero Boyer-Lindquist components.
struct M5 {
    double tt, tph, rr, thth, phph;
};

// KerrMetric::Sigma/Delta/A with sin(theta), cos(theta) supplied
// (src/kerr_metric.cpp:15-32).
HD double bl_sigma(double a, double r, double c) { return r * r + a * a * c * c; }
HD double bl_delta(double a, double r) { return r * r - 2.0 * r + a * a; }
HD double bl_A(double a, double r, double s)
{
    const double s2 = s * s;
    return (r * r + a * a) * (r * r + a * a) - a * a * bl_delta(a, r) * s2;
}

// KerrMetric::inverse_metric (src/kerr_metric.cpp:80-119).
HD void bl_ginv(double a, double r, double s, double c, M5& g)
{
    const double sig = bl_sigma(a, r, c);
    const double del = bl_delta(a, r);
    const double s2 = s * s;
    const double bigA = bl_A(a, r, s);
    g.tt = -bigA / (sig * del);
    g.tph = -2.0 * a * r / (sig * del);
    g.rr = del / sig;
    g.thth = 1.0 / sig;
    g.phph = (del - a * a * s2) / (sig * del * s2);
}

// KerrMetric::metric, rr/thth/phph (+tt, tph) (src/kerr_metric.cpp:34-78).
HD void bl_metric(double a, double r, double s, double c, M5& g)
{
    const double sig = bl_sigma(a, r, c);
    const double del = bl_delta(a, r);
    const double s2 = s * s;
    g.tt = -(1.0 - 2.0 * r / sig);
    g.tph = -2.0 * a * r * s2 / sig;
    g.rr = sig / del;
    g.thth = sig;
    g.phph = (r * r + a * a + 2.0 * a * a * r * s2 / sig) * s2;
}

// lapse and frame-drag rate (src/kerr_metric.cpp:121-145).
HD double bl_lapse(double a, double r, double s, double c)
{
    const double sig = bl_sigma(a, r, c);
    const double del = bl_delta(a, r);
    const double bigA = bl_A(a, r, s);
    return sqrt(sig * del / bigA);
}
HD double bl_omega(double a, double r, double s)
{
    const double s2 = s * s;
    return 2.0 * a * r / ((r * r + a * a) * (r * r + a * a) - a * a * bl_delta(a, r) * s2);
}

// ---- density (src/torus_profile.cpp), parameters after the constructor's
// clamps (:34-40) ----------------------------------------------------------

struct Torus {
    int32_t kind;
    int32_t use_powerlaw, use_funnel, use_envelope;
    double rho0, r0, sigma_r, H, radial_power, funnel_depletion, funnel_theta,
        env_rho0, env_alpha, r_min, r_max, rho_floor;
};

HD double torus_collapsar_shape(const Torus& t, double r, double theta)
{   // :150-179
    if (!(r >= t.r_min && r <= t.r_max) || r <= 0.0 || t.r0 <= 0.0) return 0.0;
    const double mu = cos(theta);
    const double xv = mu / smax(t.H, 1.0e-6);
    const double vertical = exp(-(xv * xv));
    const double inner_taper = 1.0 / (1.0 + exp(-(r - t.r_min) / smax(0.35 * t.sigma_r, 1.0e-6)));
    const double outer_taper = 1.0 / (1.0 + exp((r - t.r_max) / smax(0.60 * t.sigma_r, 1.0e-6)));
    const double xc = (r - 0.75 * t.r0) / smax(0.75 * t.sigma_r, 1.0e-6);
    const double inner_core = 0.45 * exp(-(xc * xc));
    const double radial = pow(smax(r / t.r0, 1.0e-300), -smax(t.radial_power, 0.0));
    const double xf = (r - t.r0) / smax(1.8 * t.sigma_r, 1.0e-6);
    const double floor_tail = 0.08 * exp(-(xf * xf));
    return (radial + inner_core + floor_tail) * vertical * inner_taper * outer_taper;
}

HD double torus_gaussian_shape(const Torus& t, double r, double theta)
{   // :181-196
    const double delta = theta - 0.5 * kPi;
    if (r <= 4.0 || r >= 18.0 || fabs(delta) >= 0.45) return 0.0;
    const double xr = (r - t.r0) / t.sigma_r;
    const double radial = exp(-(xr * xr));
    const double xv = delta / t.H;
    const double vertical = exp(-(xv * xv));
    return radial * vertical;
}

HD double torus_powerlaw_shape(const Torus& t, double r, double theta)
{   // :198-217
    if (!(r >= t.r_min && r <= t.r_max) || r <= 0.0 || t.r0 <= 0.0) return 0.0;
    const double xv = cos(theta) / t.H;
    const double vertical = exp(-(xv * xv));
    const double xi = (r - t.r_min) / t.sigma_r;
    const double inner_taper = 1.0 - exp(-(xi * xi));
    const double outer_taper = exp(-pow(r / t.r_max, 4.0));
    const double radial = pow(r / t.r0, -t.radial_power);
    return radial * vertical * inner_taper * outer_taper;
}

HD double torus_funnel_factor(const Torus& t, double theta)
{   // :219-236
    if (!t.use_funnel) return 1.0;
    const double xn = theta / t.funnel_theta;
    const double north = exp(-(xn * xn));
    const double xs = (kPi - theta) / t.funnel_theta;
    const double south = exp(-(xs * xs));
    return sclamp(1.0 - t.funnel_depletion * (north + south), 0.0, 1.0);
}

HD double torus_envelope(const Torus& t, double r)
{   // :238-248
    if (!t.use_envelope || t.env_rho0 <= 0.0 || r < t.r0 || r > t.r_max) return 0.0;
    return t.env_rho0 * pow(r / t.r0, -t.env_alpha);
}

// TorusProfile::rho (:261-272).
HD double torus_rho(const Torus& t, double r, double theta)
{
    double shape;
    if (t.kind == 7) shape = torus_collapsar_shape(t, r, theta);
    else if (t.use_powerlaw) shape = torus_powerlaw_shape(t, r, theta);
    else shape = torus_gaussian_shape(t, r, theta);
    const double disk = t.rho0 * shape * torus_funnel_factor(t, theta);
    return smax(disk + torus_envelope(t, r), t.rho_floor);
}

// ---- UHE source and spectrum (src/radiative_transfer.cpp) -----------------

struct Source {
    int32_t kind;          // enum hadros_source_kind
    int32_t spectral_kind; // enum hadros_spectral_kind
    double r_center, sigma_r, theta_width, powerlaw, emax, norm, funnel_theta,
        q, s, cutoff_lo, cutoff_hi, grad_dr, grad_dtheta;
    double rho_norm;       // rho_ref or rho(r_center, pi/2), floored at 1e-300
    double gamma, ecut;    // spectral model parameters
};

// uhe_spectral_weight (:172-207).
HD double spectral_weight(const Source& s, double E)
{
    if (E <= 0.0) return 0.0;
    const double safe_E = smax(E, 1.0e-300);
    if (s.spectral_kind == 0) {
        if (s.emax <= 0.0) return 0.0;
        return pow(safe_E, -s.powerlaw) * exp(-safe_E / s.emax);
    }
    if (s.spectral_kind == 1) return pow(safe_E, -s.gamma);
    if (s.spectral_kind == 2) {
        if (s.ecut <= 0.0) return 0.0;
        return pow(safe_E, -s.gamma) * exp(-safe_E / s.ecut);
    }
    return 0.0;
}

// bipolar_gaussian (:64-76).
HD double bipolar_gaussian(double theta, double theta0, double width)
{
    if (width <= 0.0) return 0.0;
    const double north = theta - theta0;
    const double south = theta - (kPi - theta0);
    return exp(-(north / width) * (north / width)) + exp(-(south / width) * (south / width));
}

// Bin-independent factor C of the emissivity, j = C * w(E_local):
// inner ring = emissivity_collapsar_ring's (norm*radial)*vertical (:335-367);
// other sources = norm * uhe_source_spatial_weight (:209-332, :369-395).
HD double emissivity_factor(const Source& s, const Torus& t, double r, double theta, double rho_here)
{
    if (s.kind == 0) {
        if (s.r_center <= 0.0 || s.sigma_r <= 0.0 || s.theta_width <= 0.0 || s.emax <= 0.0) return 0.0;
        const double dr = (r - s.r_center) / s.sigma_r;
        const double dth = (theta - 0.5 * kPi) / s.theta_width;
        const double radial_profile = exp(-dr * dr);
        const double vertical_profile = exp(-dth * dth);
        return s.norm * radial_profile * vertical_profile;
    }
    double S = 0.0;
    if (r <= 0.0 || s.sigma_r <= 0.0 || s.theta_width <= 0.0) {
        S = 0.0;
    } else if (s.kind == 1) {
        const double dr = (r - s.r_center) / s.sigma_r;
        S = exp(-dr * dr) * bipolar_gaussian(theta, s.funnel_theta, s.theta_width);
    } else if (s.kind == 2) {
        const double x = r / s.r_center;
        const double radial = exp(-(x * x));
        const double polar = bipolar_gaussian(theta, 0.0, s.theta_width);
        S = radial * polar;
    } else if (s.kind == 4) {
        const double density_weight = pow(smax(rho_here / s.rho_norm, 0.0), s.q);
        const double radial_weight = pow(smax(r / smax(s.r_center, 1.0e-300), 1.0e-300), -s.s);
        S = sclamp(density_weight * radial_weight, smax(s.cutoff_lo, 0.0),
                   smax(s.cutoff_hi, smax(s.cutoff_lo, 0.0)));
    } else if (s.kind == 3) {
        const double dr = smax(s.grad_dr, 1.0e-4);
        const double dtheta = smax(s.grad_dtheta, 1.0e-5);
        const double r_minus = smax(r - dr, 1.0e-6);
        const double theta_minus = sclamp(theta - dtheta, 0.0, kPi);
        const double theta_plus = sclamp(theta + dtheta, 0.0, kPi);
        const double rho_r_plus = torus_rho(t, r + dr, theta);
        const double rho_r_minus = torus_rho(t, r_minus, theta);
        const double rho_t_plus = torus_rho(t, r, theta_plus);
        const double rho_t_minus = torus_rho(t, r, theta_minus);
        const double d_r = (rho_r_plus - rho_r_minus) / (2.0 * dr);
        const double d_theta = (rho_t_plus - rho_t_minus) / (2.0 * dtheta * smax(r, 1.0e-6));
        const double gradient = sqrt(d_r * d_r + d_theta * d_theta) / s.rho_norm;
        const double x = r / smax(s.r_center, 1.0e-300);
        const double radial_taper = exp(-(x * x));
        S = sclamp(gradient * radial_taper, smax(s.cutoff_lo, 0.0),
                   smax(s.cutoff_hi, smax(s.cutoff_lo, 0.0)));
    }
    return s.norm * S;
}

}  // namespace hadros
