// hadros_mev.cuh — the MeV thermal neutrino channel as __host__ __device__
// FP64 functions.
//
// integrate_kerr_ray runs a second transfer along every ray besides the UHE
// one (src/radiative_transfer.cpp:522-638): at each path point a local
// temperature and electron fraction (mev_temperature_profile_MeV,
// mev_ye_profile), an emissivity j (URCA, pair, bremsstrahlung or the legacy
// toy proxy) and an opacity kappa (absorption on n/p, scattering on n/p/e),
// monochromatic at the redshifted energy or averaged over a Fermi-Dirac band,
// then the formal solution I = I e^{-dtau} + g^3 (j/kappa)(1 - e^{-dtau}),
// the optical depth and the neutrinosphere radius where it first reaches
// neutrinosphere_tau.  The channel does not depend on the UHE energy, so the
// trace kernel evaluates it once per point next to the per-bin UHE terms.
//
// Expressions keep the reference's operand order; std::pow(x, 2.0) is x * x
// and std::pow(x, 1.0) is x (both exact), the integer powers 3, 5, 6 and 9
// are products (a few ulp from pow, far inside the 1e-6 parity bound and
// without pow's cost), other powers call pow.
#pragma once

#include <cstdint>

#include "../../include/hadros_b200.h"
#include "hadros_physics.cuh"

namespace hadros {

// src/mev_neutrino_physics.cpp:12-15
constexpr double kHbarCMeVcm = 1.973269804e-11;
constexpr double kMeMeV = 0.510998950;
// MeVPhysicsParams::sigma_scat_e0_cm2 (include/mev_neutrino_physics.hpp:61):
// MeVThermalParams has no such field, so the channel always uses the default.
constexpr double kSigmaScatE0 = 3.4e-45;

// Per-camera constants of the channel (MeVThermalParams after the clamps the
// reference applies where it reads them).
struct Mev {
    int32_t on;         // hadros_params.mev_channel
    int32_t have_ref;   // integrate_kerr_ray_spectral keeps a first-bin result
    int32_t model, flavor, thermal, ye, band, n_bins;
    uint32_t flags;
    int32_t pad;
    double E_obs, norm, sig_abs0, sig_scat0, nu_tau;
    double T0, T_floor, T_power;                     // T0, floor: max(., 1e-12)
    double Ye_torus, Ye_funnel, Ye_envelope, Ye_lo, Ye_hi;
    double e_min, dE;                                // Fermi-Dirac band
    double rho0, r0, r_min, r_max;                   // TorusProfile accessors
};

// Running sums of one ray (RTResult's MeV fields before the final exp).
struct MevAcc {
    double tau, I, r_nu, leak;
};

HD void mev_reset(MevAcc& m)
{
    m.tau = 0.0;
    m.I = 0.0;
    m.r_nu = -1.0;
    m.leak = 0.0;
}

HD bool mev_has(const Mev& m, uint32_t bit) { return (m.flags & bit) != 0u; }
// std::isfinite: x - x is 0 for finite x, NaN for inf and NaN
HD bool mev_finite(double x) { return x - x == 0.0; }

// clamp_ye, density_shape (src/mev_neutrino_physics.cpp:17-35)
HD double mev_clamp_ye(double Ye) { return sclamp(Ye, 0.0, 1.0); }
HD double mev_density_shape(double rho, double rho0) { return sclamp(rho / smax(rho0, 1.0e-300), 0.0, 1.0); }

// mev_temperature_profile_MeV (src/mev_neutrino_physics.cpp:240-273)
HD double mev_temperature(const Mev& m, double r, double th, double rho)
{
    const double T0 = m.T0;
    const double fl = m.T_floor;
    const double shape = mev_density_shape(rho, m.rho0);
    double T = T0;
    if (m.thermal == HADROS_MEV_T_INNER_HOT_TORUS) {
        T = fl + T0 * pow(shape, smax(m.T_power, 0.0));
    } else if (m.thermal == HADROS_MEV_T_RADIAL_POWERLAW || m.thermal == HADROS_MEV_T_TORUS_PLUS_COOL_ENVELOPE ||
               m.thermal == HADROS_MEV_T_COLLAPSAR_INNER_HOT) {
        const double xe = (th - 0.5 * kPi) / 0.45;
        const double equatorial = exp(-(xe * xe));
        if (m.thermal == HADROS_MEV_T_RADIAL_POWERLAW) {
            const double radial = pow(smax(r / smax(m.r0, 1.0e-300), 1.0e-300), -m.T_power);
            T = fl + T0 * radial * (0.35 + 0.65 * equatorial);
        } else if (m.thermal == HADROS_MEV_T_TORUS_PLUS_COOL_ENVELOPE) {
            T = fl + T0 * pow(shape, smax(m.T_power, 0.0));
            const bool outside_torus = r > m.r_max || r < m.r_min;
            if (outside_torus || shape < 1.0e-3) {
                const double radial = pow(smax(r / smax(m.r0, 1.0e-300), 1.0e-300), -m.T_power);
                T = fl + 0.15 * T0 * radial;
            }
        } else {
            const double xh = (r - m.r_min) / smax(1.15 * m.r0, 1.0e-6);
            const double inner_hot = exp(-(xh * xh));
            const double radial_cooling = pow(1.0 + smax(r - m.r_min, 0.0) / smax(m.r0, 1.0e-6), -0.75);
            T = fl + T0 * (0.30 + 0.70 * pow(shape, 0.18)) * (0.45 + 0.55 * equatorial) *
                         (0.55 + 0.45 * inner_hot) * radial_cooling;
        }
    }
    return smax(T, fl);
}

// mev_ye_profile (src/mev_neutrino_physics.cpp:275-318)
HD double mev_ye(const Mev& m, double r, double th, double rho)
{
    const double shape = mev_density_shape(rho, m.rho0);
    double Ye = m.Ye_torus;
    if (m.ye == HADROS_MEV_YE_NEUTRON_RICH_TORUS) {
        const double x = (r - m.r0) / 4.0;
        Ye = m.Ye_torus + 0.05 * exp(-(x * x));
    } else if (m.ye == HADROS_MEV_YE_FUNNEL_PROTON_RICH || m.ye == HADROS_MEV_YE_COLLAPSAR_NEUTRON_RICH) {
        const double xn = th / 0.35, xs = (kPi - th) / 0.35;
        const double polar = sclamp(exp(-(xn * xn)) + exp(-(xs * xs)), 0.0, 1.0);
        if (m.ye == HADROS_MEV_YE_FUNNEL_PROTON_RICH) {
            Ye = m.Ye_torus * (1.0 - polar) + m.Ye_funnel * polar;
        } else {
            const double dense_weight = pow(shape, 0.25);
            const double x = (r - m.r0) / smax(1.2 * m.r0, 1.0e-6);
            const double radial_neutronization = exp(-(x * x));
            const double torus_ye = m.Ye_torus - 0.05 * dense_weight * radial_neutronization;
            Ye = torus_ye * (1.0 - polar) + m.Ye_funnel * polar;
        }
    } else if (m.ye == HADROS_MEV_YE_TORUS_ENVELOPE_CONTRAST) {
        const bool envelope_like = r > m.r0 && (r > m.r_max || shape < 1.0e-2);
        Ye = envelope_like ? m.Ye_envelope : m.Ye_torus;
        if (r < m.r_min && shape < 1.0e-2) Ye = m.Ye_funnel;
    }
    return sclamp(Ye, m.Ye_lo, m.Ye_hi);
}

// mev_thermal_spectral_shape without its 1/T^3 (src/mev_neutrino_physics.cpp:
// 320-340) = mev_fermi_dirac_weight (:342-354): E^2 / (e^{E/T} + 1), 0 for
// E <= 0, T <= 0 or E/T > 120.
HD double mev_fd(double E, double T)
{
    if (E <= 0.0 || T <= 0.0) return 0.0;
    const double x = E / T;
    if (x > 120.0) return 0.0;
    return E * E / (exp(x) + 1.0);
}

// electron_number_density_cm3 (:356-366)
HD double mev_ne(double rho, double Ye)
{
    if (rho <= 0.0) return 0.0;
    return rho * mev_clamp_ye(Ye) / kMuG;
}

// mev_urca_degeneracy_correction (:404-432) with electron_degeneracy_eta,
// electron_chemical_potential_MeV and electron_fermi_momentum_MeV (:368-402)
HD double mev_degeneracy(double rho, double Ye, double T, int flavor)
{
    if (flavor == HADROS_MEV_NU_X) return 1.0;
    double eta = 0.0;
    if (T > 0.0) {
        const double ne = mev_ne(rho, Ye);
        const double pF = ne <= 0.0 ? 0.0 : kHbarCMeVcm * cbrt(3.0 * kPi * kPi * ne);
        eta = sqrt(pF * pF + kMeMeV * kMeMeV) / T;
    }
    if (!mev_finite(eta)) return 1.0;
    const double shift = 0.25 * tanh((eta - 1.0) / 4.0);
    const double factor = flavor == HADROS_MEV_NU_E ? (1.0 + shift) : (1.0 - shift);
    return sclamp(factor, 0.5, 1.5);
}

// mev_total_emissivity (:511-588) with mev_emissivity_urca/pair/brems
// (:434-530); the thermal shape E^2/(e^x+1)/T^3 is the same for all three.
HD double mev_emissivity(const Mev& m, double rho, double T, double Ye, double E)
{
    if (m.model == HADROS_MEV_TOY) {
        if (rho <= 0.0 || T <= 0.0 || E <= 0.0) return 0.0;
        const double nb = rho / kMuG;
        const double neutron_fraction = sclamp(1.0 - Ye, 0.0, 1.0);
        const double proton_fraction = sclamp(Ye, 0.0, 1.0);
        const double charged_current_weight = neutron_fraction + 0.5 * proton_fraction;
        const double thermal_spectrum = E * E / (exp(smin(E / T, 120.0)) + 1.0);
        const double T3 = T * T * T, T6 = T3 * T3;
        const double capture_like = nb * charged_current_weight * T6;
        const double pair_like = 0.05 * nb * (T6 * T3);
        return m.norm * (capture_like + pair_like) * thermal_spectrum;
    }
    double shape = 0.0;
    if (T > 0.0 && E > 0.0) shape = mev_fd(E, T) / smax(T * T * T, 1.0e-300);
    const double T10 = T / 10.0;
    const double t2 = T10 * T10, t3 = t2 * T10, t6 = t3 * t3;
    const double rho10 = rho / 1.0e10;
    double total = 0.0;
    if (mev_has(m, HADROS_MEV_URCA)) {
        double urca = 0.0;
        if (!(rho <= 0.0 || T <= 0.0 || E <= 0.0) && m.flavor != HADROS_MEV_NU_X) {
            const double ye = mev_clamp_ye(Ye);
            const double flavor_factor = m.flavor == HADROS_MEV_NU_E ? ye : (1.0 - ye);
            urca = 1.0e30 * rho10 * t6 * flavor_factor * shape;
        }
        if (mev_has(m, HADROS_MEV_DEGENERACY_CORRECTION)) urca *= mev_degeneracy(rho, Ye, T, m.flavor);
        total += urca;
    }
    if (mev_has(m, HADROS_MEV_PAIR) && !(T <= 0.0 || E <= 0.0)) {
        const double flavor_factor = m.flavor == HADROS_MEV_NU_X ? 1.0 : 0.7;
        total += 3.0e28 * (t6 * t3) * flavor_factor * shape;
    }
    if (mev_has(m, HADROS_MEV_BREMS) && !(rho <= 0.0 || T <= 0.0 || E <= 0.0)) {
        const double flavor_factor = m.flavor == HADROS_MEV_NU_X ? 1.0 : 0.8;
        total += 1.0e27 * (rho10 * rho10) * (t3 * t2) * flavor_factor * shape;
    }
    return m.norm * total;
}

// mev_total_opacity_cm_inv (:762-770): absorption (:590-659) + scattering
// (:661-760), toy or per target.
HD double mev_opacity(const Mev& m, double rho, double Ye, double E)
{
    const bool absorb = mev_has(m, HADROS_MEV_ABSORPTION);
    const bool scatter = mev_has(m, HADROS_MEV_SCATTERING);
    double ka = 0.0, ks = 0.0;
    if (m.model == HADROS_MEV_TOY) {
        if (absorb && !(rho <= 0.0) && !(E <= 0.0)) {
            const double nb = rho / kMuG;
            const double target_fraction = sclamp(1.0 - Ye, 0.0, 1.0) + 0.25 * sclamp(Ye, 0.0, 1.0);
            ka = nb * m.sig_abs0 * E * E * target_fraction;
        }
        if (scatter && !(rho <= 0.0) && !(E <= 0.0)) {
            const double nb = rho / kMuG;
            const double composition_factor = 1.0 + 0.5 * sclamp(Ye, 0.0, 1.0);
            ks = nb * m.sig_scat0 * E * E * composition_factor;
        }
        return ka + ks;
    }
    if (rho <= 0.0 || E <= 0.0) return 0.0;
    const double nb = rho / kMuG;
    const double ye = mev_clamp_ye(Ye);
    double kan = 0.0, kap = 0.0, ksn = 0.0, ksp = 0.0, kse = 0.0;
    if (absorb && mev_has(m, HADROS_MEV_ABS_N) && m.flavor == HADROS_MEV_NU_E)
        kan = nb * (1.0 - ye) * m.sig_abs0 * E * E;
    if (absorb && mev_has(m, HADROS_MEV_ABS_P) && m.flavor == HADROS_MEV_ANTI_NU_E)
        kap = nb * ye * m.sig_abs0 * E * E;
    if (scatter && mev_has(m, HADROS_MEV_SCAT_N)) ksn = nb * (1.0 - ye) * m.sig_scat0 * E * E;
    if (scatter && mev_has(m, HADROS_MEV_SCAT_P)) ksp = nb * ye * 0.5 * m.sig_scat0 * E * E;
    if (scatter && mev_has(m, HADROS_MEV_SCAT_E)) kse = mev_ne(rho, Ye) * kSigmaScatE0 * E * E;
    return (kan + kap) + (ksn + ksp + kse);
}

// One path point into the ray's MeV sums: the body of integrate_kerr_ray's
// MeV block (src/radiative_transfer.cpp:507-607) for a point that passed the
// r >= r_+ + 1e-3 test; rho is TorusProfile::rho there (FP64), z the
// redshift factor, dl_cm the interval in cm.
HD void mev_point(const Mev& m, MevAcc& acc, double r, double th, double rho, double z, double dl_cm)
{
    const double g = 1.0 / smax(z, 1.0e-300);
    const double gs = smax(g, 1.0e-300);
    const double T = mev_temperature(m, r, th, rho);
    const double Ye = mev_ye(m, r, th, rho);
    double kappa = 0.0, j = 0.0;
    if (m.band) {
        double weight_sum = 0.0, kappa_weighted = 0.0;
        for (int ib = 0; ib < m.n_bins; ++ib) {
            const double E_mid = m.e_min + (static_cast<double>(ib) + 0.5) * m.dE;
            const double E_local = E_mid / gs;
            const double w = mev_fd(E_local, T) * m.dE;
            if (w <= 0.0 || !mev_finite(w)) continue;
            const double local_kappa = mev_opacity(m, rho, Ye, E_local);
            j += mev_emissivity(m, rho, T, Ye, E_local) * m.dE;
            kappa_weighted += w * local_kappa;
            weight_sum += w;
        }
        kappa = weight_sum > 0.0 ? kappa_weighted / weight_sum : 0.0;
    } else {
        const double E_local = m.E_obs / gs;
        kappa = mev_opacity(m, rho, Ye, E_local);
        j = mev_emissivity(m, rho, T, Ye, E_local);
    }
    const double dtau = kappa * dl_cm;
    const double g3 = g * g * g;
    if (kappa > 0.0 && dtau > 1.0e-12) {
        const double attenuation = exp(-smin(dtau, 700.0));
        acc.I = acc.I * attenuation + g3 * (j / kappa) * (1.0 - attenuation);
    } else {
        acc.I += g3 * j * dl_cm;
    }
    acc.leak += j * dl_cm;
    acc.tau += dtau;
    if (acc.r_nu < 0.0 && acc.tau >= m.nu_tau) acc.r_nu = r;
}

// RTResult's MeV fields of a finished ray (:673-679); a ray with no points,
// or a spectral band without a valid bin, keeps the defaults.
HD void mev_finish(const Mev& m, const MevAcc& acc, int n_points, double* tau, double* P, double* I,
                   double* r_nu, double* leak)
{
    const bool have = m.on && m.have_ref && n_points > 0;
    *tau = have ? acc.tau : 0.0;
    *P = have ? exp(-acc.tau) : 1.0;
    *I = have ? acc.I : 0.0;
    *r_nu = have ? acc.r_nu : -1.0;
    *leak = (have && acc.leak > 0.0) ? acc.leak / acc.leak : 1.0;
}

// Per-camera constants from the parameters (host).
inline Mev make_mev(const hadros_params& p, const Torus& t, bool have_ref)
{
    Mev m{};
    m.on = p.mev_channel ? 1 : 0;
    m.have_ref = have_ref ? 1 : 0;
    m.model = p.mev_model;
    m.flavor = p.mev_flavor;
    m.thermal = p.mev_thermal_profile;
    m.ye = p.mev_ye_profile;
    m.band = p.mev_spectral_mode == HADROS_MEV_FERMI_DIRAC_BAND ? 1 : 0;
    m.flags = p.mev_flags;
    m.E_obs = p.mev_Enu_obs_MeV;
    m.norm = p.mev_norm;
    m.sig_abs0 = p.mev_sigma_abs0_cm2;
    m.sig_scat0 = p.mev_sigma_scat0_cm2;
    m.nu_tau = p.mev_neutrinosphere_tau;
    m.T0 = smax(p.mev_T0_MeV, 1.0e-12);           // :250-251
    m.T_floor = smax(p.mev_T_floor_MeV, 1.0e-12);
    m.T_power = p.mev_T_power;
    m.Ye_torus = p.mev_Ye_torus;
    m.Ye_funnel = p.mev_Ye_funnel;
    m.Ye_envelope = p.mev_Ye_envelope;
    m.Ye_lo = smax(p.mev_Ye_floor, 1.0e-6);       // :313-317
    m.Ye_hi = smin(p.mev_Ye_ceil, 1.0 - 1.0e-6);
    // radiative_transfer.cpp:543-546
    m.n_bins = p.mev_n_bins > 1 ? p.mev_n_bins : 1;
    m.e_min = smax(p.mev_E_min_MeV, 1.0e-6);
    const double e_max = smax(p.mev_E_max_MeV, m.e_min);
    m.dE = (e_max - m.e_min) / static_cast<double>(m.n_bins);
    m.rho0 = t.rho0;
    m.r0 = t.r0;
    m.r_min = t.r_min;
    m.r_max = t.r_max;
    return m;
}

}  // namespace hadros
