// ref_driver.cpp — drives the REFERENCE implementation (test infrastructure).
//
// Linked by oracle/build_ref.sh against the reference's own, unmodified
// src/{kerr_metric,kerr_geodesic,kerr_camera,sigma_table,torus_profile,
// radiative_transfer,mev_neutrino_physics}.cpp into oracle/_ref/libhadros_ref.so.
// It restores the per-pixel loop that apps/compute_kerr_image.cpp:62-92
// intended (trace_pixel, then integrate_kerr_ray_spectral) for an arbitrary
// pixel subset, with the argument mapping of
// apps/compute_kerr_image_from_cache.cpp:335-351 and :612-633.
//
// The reference hard-codes a 200000-step cap (src/kerr_camera.cpp:222).  A
// smaller cap N is applied after tracing: the first N loop iterations are the
// same for any cap, so a ray still running at step N keeps its first N points
// and has captured == false.
#include "kerr_camera.hpp"
#include "radiative_transfer.hpp"
#include "sigma_table.hpp"
#include "torus_profile.hpp"

#include "../include/hadros_b200.h"

#include <cmath>
#include <cstdint>
#include <exception>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const char* profile_name(int k)
{
    static const char* names[] = {"gaussian", "powerlaw", "gaussian_funnel", "powerlaw_funnel",
                                  "gaussian_envelope", "powerlaw_envelope",
                                  "powerlaw_funnel_envelope", "collapsar_ndaf_like"};
    return (k >= 0 && k < 8) ? names[k] : "?";
}

}  // namespace

extern "C" int ref_image(const hadros_params* p, const char* sigma_path,
                         const int32_t* pixel_ids, int32_t n_pixels, double* tau,
                         double* P_surv, double* I_obs, int8_t* fate, int32_t* steps,
                         double* tau_E, double* I_E, double* tau_mev, double* P_surv_mev,
                         double* I_obs_mev, double* r_nu, double* leakage, int n_threads)
{
    try {
        if (p->max_steps > 200000 || p->tolerance != 1.0e-6) return -2;
        KerrCamera camera(p->a_spin, p->r_obs_rg, p->theta_obs_rad, p->fov_deg, p->nx, p->ny,
                          p->r_max_rg, p->h);
        SigmaTable sigma(sigma_path);
        TorusProfile torus(p->rho0_gcm3, p->r0_rg, p->sigma_r_rg, p->H_over_R,
                           profile_name(p->profile_kind), p->radial_power, p->funnel_depletion,
                           p->funnel_theta_rad, p->envelope_rho0_gcm3, p->envelope_alpha,
                           p->torus_r_min_rg, p->torus_r_max_rg, p->rho_floor_gcm3);
        UHESourceParams source;
        source.model = static_cast<UHESourceModel>(p->source_kind);
        source.model_name = radiative_transfer::uhe_source_model_name(source.model);
        source.r_center_rg = p->src_r_center_rg;
        source.sigma_r_rg = p->src_sigma_r_rg;
        source.theta_width_rad = p->src_theta_width_rad;
        source.powerlaw = p->src_powerlaw;
        source.emax_GeV = p->src_emax_GeV;
        source.norm = p->src_norm;
        source.funnel_theta_rad = p->src_funnel_theta_rad;
        source.density_power_q = p->src_density_power_q;
        source.radial_power_s = p->src_radial_power_s;
        source.rho_ref_gcm3 = p->src_rho_ref_gcm3;
        source.cutoff_min = p->src_cutoff_min;
        source.cutoff_max = p->src_cutoff_max;
        source.gradient_dr_rg = p->src_gradient_dr_rg;
        source.gradient_dtheta_rad = p->src_gradient_dtheta_rad;
        UHESpectralParams spectral;
        spectral.model = static_cast<UHESpectralModel>(p->spectral_kind);
        spectral.model_name = radiative_transfer::uhe_spectral_model_name(spectral.model);
        spectral.gamma = p->spec_gamma;
        spectral.ecut_GeV = p->spec_ecut_GeV;
        spectral.e_min_GeV = p->spec_e_min_GeV;
        spectral.e_max_GeV = p->spec_e_max_GeV;
        spectral.n_bins = p->n_bins;
        // MeV channel: the shipped defaults, or hadros_params' mev_* fields
        // when mev_channel is set (the argv 14-15 and 45-71 mapping of
        // apps/compute_kerr_image_from_cache.cpp:97-304)
        MeVThermalParams mev;
        if (p->mev_channel) {
            const uint32_t fl = p->mev_flags;
            mev.Enu_obs_MeV = p->mev_Enu_obs_MeV;
            mev.norm = p->mev_norm;
            mev.sigma_abs0_cm2 = p->mev_sigma_abs0_cm2;
            mev.sigma_scat0_cm2 = p->mev_sigma_scat0_cm2;
            mev.neutrinosphere_tau = p->mev_neutrinosphere_tau;
            mev.model = static_cast<mev_neutrino::MeVModel>(p->mev_model);
            mev.model_name = mev_neutrino::mev_model_name(mev.model);
            mev.flavor = static_cast<mev_neutrino::MeVFlavor>(p->mev_flavor);
            mev.flavor_name = mev_neutrino::mev_flavor_name(mev.flavor);
            mev.include_urca = (fl & HADROS_MEV_URCA) != 0;
            mev.include_pair = (fl & HADROS_MEV_PAIR) != 0;
            mev.include_brems = (fl & HADROS_MEV_BREMS) != 0;
            mev.include_absorption = (fl & HADROS_MEV_ABSORPTION) != 0;
            mev.include_scattering = (fl & HADROS_MEV_SCATTERING) != 0;
            mev.use_degeneracy_correction = (fl & HADROS_MEV_DEGENERACY_CORRECTION) != 0;
            mev.include_abs_n = (fl & HADROS_MEV_ABS_N) != 0;
            mev.include_abs_p = (fl & HADROS_MEV_ABS_P) != 0;
            mev.include_scat_n = (fl & HADROS_MEV_SCAT_N) != 0;
            mev.include_scat_p = (fl & HADROS_MEV_SCAT_P) != 0;
            mev.include_scat_e = (fl & HADROS_MEV_SCAT_E) != 0;
            mev.thermal_profile = static_cast<mev_neutrino::MeVThermalProfile>(p->mev_thermal_profile);
            mev.thermal_profile_name = mev_neutrino::mev_thermal_profile_name(mev.thermal_profile);
            mev.ye_profile = static_cast<mev_neutrino::MeVYeProfile>(p->mev_ye_profile);
            mev.ye_profile_name = mev_neutrino::mev_ye_profile_name(mev.ye_profile);
            mev.spectral_mode = static_cast<mev_neutrino::MeVSpectralMode>(p->mev_spectral_mode);
            mev.spectral_mode_name = mev_neutrino::mev_spectral_mode_name(mev.spectral_mode);
            mev.T0_MeV = p->mev_T0_MeV;
            mev.T_floor_MeV = p->mev_T_floor_MeV;
            mev.T_power = p->mev_T_power;
            mev.Ye_torus = p->mev_Ye_torus;
            mev.Ye_funnel = p->mev_Ye_funnel;
            mev.Ye_envelope = p->mev_Ye_envelope;
            mev.Ye_floor = p->mev_Ye_floor;
            mev.Ye_ceil = p->mev_Ye_ceil;
            mev.E_min_MeV = p->mev_E_min_MeV;
            mev.E_max_MeV = p->mev_E_max_MeV;
            mev.n_bins = p->mev_n_bins;
        }

        // Per-bin energies exactly as integrate_kerr_ray_spectral forms them.
        std::vector<double> E_mid;
        const bool mono = spectral.model == UHESpectralModel::Monochromatic;
        if (mono) {
            E_mid.push_back(p->Enu_obs_GeV);
        } else {
            const int n_bins = std::max(spectral.n_bins, 1);
            const double e_min = std::max(spectral.e_min_GeV, sigma.Emin());
            const double e_max = std::min(spectral.e_max_GeV, sigma.Emax());
            const double log_min = std::log(e_min);
            const double log_max = std::log(e_max);
            const double dlog = (log_max - log_min) / static_cast<double>(n_bins);
            for (int b = 0; b < n_bins; ++b) {
                const double log_left = log_min + dlog * static_cast<double>(b);
                const double log_right = log_left + dlog;
                E_mid.push_back(std::exp(0.5 * (log_left + log_right)));
            }
            if (e_min <= 0.0 || e_max <= e_min) E_mid.assign(n_bins, 0.0);
        }
        const int B = static_cast<int>(E_mid.size());
        const long total = pixel_ids ? static_cast<long>(n_pixels)
                                     : static_cast<long>(p->nx) * static_cast<long>(p->ny);
#ifdef _OPENMP
        if (n_threads > 0) omp_set_num_threads(n_threads);
#else
        (void)n_threads;
#endif
        int failed = 0;
#pragma omp parallel for schedule(dynamic, 1)
        for (long k = 0; k < total; ++k) {
            try {
                const long pid = pixel_ids ? static_cast<long>(pixel_ids[k]) : k;
                const int i = static_cast<int>(pid % p->nx), j = static_cast<int>(pid / p->nx);
                RayPath ray = camera.trace_pixel(i, j);
                int f = ray.captured ? HADROS_FATE_CAPTURED : HADROS_FATE_ESCAPED;
                if (ray.points.size() >= static_cast<std::size_t>(p->max_steps)) {
                    ray.points.resize(static_cast<std::size_t>(p->max_steps));
                    ray.captured = false;
                    f = HADROS_FATE_TRUNCATED;
                }
                RTResult rt;   // defaults for an empty ray, as the CPU app does
                rt.tau = 0.0;
                rt.P_surv = 1.0;
                rt.I_obs = 0.0;
                if (!ray.points.empty())
                    rt = radiative_transfer::integrate_kerr_ray_spectral(
                        ray, p->Enu_obs_GeV, p->M_bh_msun, torus, sigma, source, mev, spectral);
                if (tau) tau[k] = rt.tau;
                if (P_surv) P_surv[k] = rt.P_surv;
                if (I_obs) I_obs[k] = rt.I_obs;
                if (fate) fate[k] = static_cast<int8_t>(f);
                if (steps) steps[k] = static_cast<int32_t>(ray.points.size());
                if (tau_mev) tau_mev[k] = rt.tau_mev;
                if (P_surv_mev) P_surv_mev[k] = rt.P_surv_mev;
                if (I_obs_mev) I_obs_mev[k] = rt.I_obs_mev;
                if (r_nu) r_nu[k] = rt.r_neutrinosphere_rg;
                if (leakage) leakage[k] = rt.leakage_factor;
                if (tau_E || I_E) {
                    for (int b = 0; b < B; ++b) {
                        RTResult rb;
                        if (!ray.points.empty() && E_mid[b] > 0.0)
                            rb = radiative_transfer::integrate_kerr_ray(
                                ray, E_mid[b], p->M_bh_msun, torus, sigma, source, mev, spectral);
                        if (tau_E) tau_E[k * B + b] = rb.tau;
                        if (I_E) I_E[k * B + b] = rb.I_obs;
                    }
                }
            } catch (const std::exception&) {
#pragma omp atomic write
                failed = 1;
            }
        }
        return failed ? -3 : B;
    } catch (const std::exception&) {
        return -1;
    }
}
