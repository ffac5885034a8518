// hadros_formats.cpp — the reference's image file formats and file names.
//
//  * 13-column text image (.dat): '#'-metadata header, then one row per pixel
//    "i j alpha beta tau P_surv I captured tau_mev P_surv_mev I_mev r_nu
//    leakage" in pixel order j*nx+i, %.8e for reals
//    (apps/compute_kerr_image_from_cache.cpp:512-653,
//    apps/compute_kerr_image_cuda.cu:2509-2586);
//  * KIMG binary (.bin): "<7i4d" header (magic 0x4B494D47, version 1,
//    backend, nx, ny, ncols = 13, reserved, E_GeV, E_MeV, MeV norm,
//    theta_deg) and nx*ny rows of 13 little-endian doubles
//    (apps/compute_kerr_image_cuda.cu:279-332, read by scripts/plot_kerr_image.py:
//    108-150);
//  * output file names (apps/compute_kerr_image_cuda.cu:2108-2128 and
//    apps/compute_kerr_image_from_cache.cpp:477-500), which the Python drivers
//    re-derive to find the image.
// The five MeV columns come from the MeV channel's outputs when the caller
// passes them (hadros_write_dat_mev / hadros_write_kimg_mev) and otherwise
// carry RTResult's defaults (tau 0, P 1, I 0, r_nu -1, leakage 1).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "hadros_internal.h"

namespace {

int32_t ferr(int32_t code, const std::string& m) { return hadros::set_error(code, m); }

// make_tag (apps/compute_kerr_image_cuda.cu:377-386): printf, then
// '+' -> '_', '-' -> 'm', '.' -> 'p'.
std::string make_tag(const char* fmt, double v)
{
    char buf[64];
    std::snprintf(buf, sizeof(buf), fmt, v);
    std::string t(buf);
    for (char& ch : t) {
        if (ch == '+') ch = '_';
        else if (ch == '-') ch = 'm';
        else if (ch == '.') ch = 'p';
    }
    return t;
}

// make_compact_scientific_tag (:388-403): "%.0e" with the exponent's sign and
// leading zeros dropped ("1e+10" -> "1e10", "1e-02" -> "1e-2").
std::string compact_sci(double v)
{
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.0e", v);
    std::string t(buf);
    const size_t e = t.find('e');
    if (e == std::string::npos) return t;
    return t.substr(0, e) + "e" + std::to_string(std::atoi(t.c_str() + e + 1));
}

const char* const kProfile[8] = {"gaussian", "powerlaw", "gaussian_funnel", "powerlaw_funnel",
                                 "gaussian_envelope", "powerlaw_envelope",
                                 "powerlaw_funnel_envelope", "collapsar_ndaf_like"};
const char* const kSource[5] = {"inner_ring", "funnel_wall", "jet_base", "shock_layer",
                                "density_weighted"};
const char* const kSpectral[3] = {"monochromatic", "powerlaw", "powerlaw_cutoff"};

double rad2deg(double r) { return r * 180.0 / M_PI; }

double pixel_u(const hadros_params* p, int i)
{   // src/kerr_camera.cpp:196-200 (alpha_rg, beta_rg)
    const double fov_rad = p->fov_deg * M_PI / 180.0;
    return (2.0 * (i + 0.5) / p->nx - 1.0) * std::tan(0.5 * fov_rad);
}

double pixel_v(const hadros_params* p, int j)
{
    const double fov_rad = p->fov_deg * M_PI / 180.0;
    return (2.0 * (j + 0.5) / p->ny - 1.0) * std::tan(0.5 * fov_rad);
}

bool kinds_ok(const hadros_params* p)
{
    return p && p->profile_kind >= 0 && p->profile_kind < 8 && p->source_kind >= 0 &&
           p->source_kind < 5 && p->spectral_kind >= 0 && p->spectral_kind < 3 && p->nx > 0 &&
           p->ny > 0;
}

}  // namespace

extern "C" {

int32_t hadros_image_filename(const hadros_params* p, int32_t style, const char* dis_model,
                              double mev_E_MeV, double mev_norm, const char* ext, char* buf,
                              int32_t buflen)
{
    if (!kinds_ok(p) || !buf || buflen <= 0 || !ext) return ferr(HADROS_E_ARG, "bad argument");
    const std::string profile = kProfile[p->profile_kind];
    std::string name;
    if (style == 0) {
        // compute_kerr_image_cuda in-line mode (apps/compute_kerr_image_cuda.cu:2108-2128)
        name = "kerr_image_cuda_rho0_torus_" + compact_sci(p->rho0_gcm3) +
               (profile == "gaussian" ? "" : "_Profile_" + profile) +
               (p->source_kind == HADROS_SOURCE_INNER_RING ? "" : std::string("_Source_") + kSource[p->source_kind]) +
               "_Enu_" + make_tag("%.0e", p->Enu_obs_GeV) + "_MeVEnu_" + make_tag("%.0e", mev_E_MeV) +
               "_MeVNorm_" + make_tag("%.0e", mev_norm) + "_CamTheta_" +
               make_tag("%.1f", rad2deg(p->theta_obs_rad));
    } else {
        // compute_kerr_image_from_cache (apps/compute_kerr_image_from_cache.cpp:477-500)
        name = std::string("kerr_image_cuda_cache_") + (dis_model && *dis_model ? dis_model : "GBW") +
               "_rho0_torus_" + compact_sci(p->rho0_gcm3) +
               (profile == "gaussian" ? "" : "_Profile_" + profile) +
               (p->source_kind == HADROS_SOURCE_INNER_RING ? "" : std::string("_Source_") + kSource[p->source_kind]) +
               (p->spectral_kind == HADROS_SPECTRAL_MONOCHROMATIC ? "" : std::string("_Spectrum_") + kSpectral[p->spectral_kind]) +
               "_Enu_" + make_tag("%.0e", p->Enu_obs_GeV) + "_MeVEnu_" + make_tag("%.0e", mev_E_MeV) +
               "_MeVNorm_" + make_tag("%.0e", mev_norm) +
               (p->mev_spectral_mode == HADROS_MEV_FERMI_DIRAC_BAND
                    ? "_MeVSpectrum_fermi_dirac_band_E" + make_tag("%.0e", p->mev_E_min_MeV) + "_" +
                          make_tag("%.0e", p->mev_E_max_MeV)
                    : std::string()) +
               "_CamTheta_" + make_tag("%.1f", rad2deg(p->theta_obs_rad));
    }
    name += ext;
    if (static_cast<int32_t>(name.size()) + 1 > buflen) return ferr(HADROS_E_ARG, "buffer too small");
    std::memcpy(buf, name.c_str(), name.size() + 1);
    return HADROS_OK;
}

namespace {

// The five MeV columns of pixel k: the arrays given, else RTResult's defaults.
struct MevCols {
    const double* a[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    void row(size_t k, double* out) const
    {
        static const double def[5] = {0.0, 1.0, 0.0, -1.0, 1.0};
        for (int c = 0; c < 5; ++c) out[c] = a[c] ? a[c][k] : def[c];
    }
};

MevCols mev_cols(const hadros_image_out* h)
{
    MevCols m;
    if (h) {
        m.a[0] = h->tau_mev;
        m.a[1] = h->P_surv_mev;
        m.a[2] = h->I_obs_mev;
        m.a[3] = h->r_nu;
        m.a[4] = h->leakage;
    }
    return m;
}

const char* name_or(const char* n) { return n ? n : "?"; }

int32_t write_dat(const char* path, const hadros_params* p, const char* dis_model, double mev_E_MeV,
                  double mev_norm, const double* tau, const double* P_surv, const double* I_obs,
                  const int8_t* fate, const MevCols& mev)
{
    if (!path || !kinds_ok(p) || !tau || !P_surv || !I_obs || !fate)
        return ferr(HADROS_E_ARG, "bad argument");
    hadros::set_error(HADROS_OK, "");
    FILE* f = std::fopen(path, "w");
    if (!f) return ferr(HADROS_E_IO, std::string("Could not open ") + path);
    // metadata header: apps/compute_kerr_image_from_cache.cpp:512-597 (ostream
    // default formatting = %g)
    const char* prof = kProfile[p->profile_kind];
    const char* src = kSource[p->source_kind];
    std::fprintf(f, "# profile_type %s\n# rho0 %g\n# rho0_gcm3 %g\n# r0 %g\n# r0_rg %g\n", prof,
                 p->rho0_gcm3, p->rho0_gcm3, p->r0_rg, p->r0_rg);
    std::fprintf(f, "# sigma_r %g\n# sigma_r_rg %g\n# H_over_R %g\n# radial_power %g\n", p->sigma_r_rg,
                 p->sigma_r_rg, p->H_over_R, p->radial_power);
    std::fprintf(f, "# funnel_depletion %g\n# funnel_theta_deg %g\n# rho_floor %g\n# rho_floor_gcm3 %g\n",
                 p->funnel_depletion, rad2deg(p->funnel_theta_rad), p->rho_floor_gcm3, p->rho_floor_gcm3);
    std::fprintf(f, "# envelope_rho0 %g\n# envelope_rho0_gcm3 %g\n# envelope_alpha %g\n", p->envelope_rho0_gcm3,
                 p->envelope_rho0_gcm3, p->envelope_alpha);
    std::fprintf(f, "# R_min %g\n# R_min_rg %g\n# R_max %g\n# R_max_rg %g\n# spin %g\n", p->torus_r_min_rg,
                 p->torus_r_min_rg, p->torus_r_max_rg, p->torus_r_max_rg, p->a_spin);
    std::fprintf(f, "# observer_distance %g\n# observer_distance_rg %g\n", p->r_obs_rg, p->r_obs_rg);
    std::fprintf(f, "# observer_inclination %g\n# observer_inclination_deg %g\n", rad2deg(p->theta_obs_rad),
                 rad2deg(p->theta_obs_rad));
    std::fprintf(f, "# DIS_model %s\n# use_F3 1\n", dis_model && *dis_model ? dis_model : "GBW");
    std::fprintf(f, "# source_model %s\n# source_r_rg %g\n# source_sigma_rg %g\n# source_theta_deg %g\n", src,
                 p->src_r_center_rg, p->src_sigma_r_rg, rad2deg(p->src_theta_width_rad));
    std::fprintf(f, "# source_powerlaw %g\n# source_emax_GeV %g\n# source_norm %g\n", p->src_powerlaw,
                 p->src_emax_GeV, p->src_norm);
    std::fprintf(f, "# source_funnel_theta_deg %g\n# source_rho_ref %g\n# rho_ref %g\n",
                 rad2deg(p->src_funnel_theta_rad), p->src_rho_ref_gcm3, p->src_rho_ref_gcm3);
    std::fprintf(f, "# source_q %g\n# source_s %g\n# source_density_power_q %g\n# source_radial_power_s %g\n",
                 p->src_density_power_q, p->src_radial_power_s, p->src_density_power_q, p->src_radial_power_s);
    std::fprintf(f, "# source_cutoff_min %g\n# source_cutoff_max %g\n# source_gradient_dr_rg %g\n",
                 p->src_cutoff_min, p->src_cutoff_max, p->src_gradient_dr_rg);
    std::fprintf(f, "# source_gradient_dtheta_deg %g\n", rad2deg(p->src_gradient_dtheta_rad));
    std::fprintf(f, "# spectral_model %s\n# spectral_gamma %g\n# spectral_ecut_GeV %g\n",
                 kSpectral[p->spectral_kind], p->spec_gamma, p->spec_ecut_GeV);
    std::fprintf(f, "# spectral_E_min_GeV %g\n# spectral_E_max_GeV %g\n# spectral_N_bins %d\n", p->spec_e_min_GeV,
                 p->spec_e_max_GeV, p->n_bins);
    if (p->mev_channel) {   // apps/compute_kerr_image_from_cache.cpp:563-591
        const uint32_t fl = p->mev_flags;
        auto on = [&](uint32_t bit) { return (fl & bit) ? 1 : 0; };
        std::fprintf(f, "# MEV_MODEL %s\n# MEV_CPU_MODEL %s\n# MEV_CUDA_STATUS physical_cpu_equivalent\n",
                     name_or(hadros_mev_model_name(p->mev_model)), name_or(hadros_mev_model_name(p->mev_model)));
        std::fprintf(f, "# MEV_FLAVOR %s\n# MEV_ENERGY_MEV %g\n# MEV_NORM %g\n",
                     name_or(hadros_mev_flavor_name(p->mev_flavor)), mev_E_MeV, mev_norm);
        std::fprintf(f, "# MEV_INCLUDE_URCA %d\n# MEV_INCLUDE_PAIR %d\n# MEV_INCLUDE_BREMS %d\n",
                     on(HADROS_MEV_URCA), on(HADROS_MEV_PAIR), on(HADROS_MEV_BREMS));
        std::fprintf(f, "# MEV_INCLUDE_ABSORPTION %d\n# MEV_INCLUDE_SCATTERING %d\n", on(HADROS_MEV_ABSORPTION),
                     on(HADROS_MEV_SCATTERING));
        std::fprintf(f, "# MEV_THERMAL_PROFILE %s\n# MEV_YE_PROFILE %s\n",
                     name_or(hadros_mev_thermal_name(p->mev_thermal_profile)),
                     name_or(hadros_mev_ye_name(p->mev_ye_profile)));
        std::fprintf(f, "# MEV_T0_MEV %g\n# MEV_T_FLOOR_MEV %g\n# MEV_T_POWER %g\n", p->mev_T0_MeV,
                     p->mev_T_floor_MeV, p->mev_T_power);
        std::fprintf(f, "# MEV_YE_TORUS %g\n# MEV_YE_FUNNEL %g\n# MEV_YE_ENVELOPE %g\n# MEV_YE_FLOOR %g\n",
                     p->mev_Ye_torus, p->mev_Ye_funnel, p->mev_Ye_envelope, p->mev_Ye_floor);
        std::fprintf(f, "# MEV_YE_CEIL %g\n# MEV_SPECTRAL_MODE %s\n# MEV_E_MIN_MEV %g\n# MEV_E_MAX_MEV %g\n",
                     p->mev_Ye_ceil, name_or(hadros_mev_spectral_name(p->mev_spectral_mode)), p->mev_E_min_MeV,
                     p->mev_E_max_MeV);
        std::fprintf(f, "# MEV_N_BINS %d\n# MEV_USE_DEGENERACY_CORRECTION %d\n# MEV_INCLUDE_ABS_N %d\n",
                     p->mev_n_bins, on(HADROS_MEV_DEGENERACY_CORRECTION), on(HADROS_MEV_ABS_N));
        std::fprintf(f, "# MEV_INCLUDE_ABS_P %d\n# MEV_INCLUDE_SCAT_N %d\n# MEV_INCLUDE_SCAT_P %d\n",
                     on(HADROS_MEV_ABS_P), on(HADROS_MEV_SCAT_N), on(HADROS_MEV_SCAT_P));
        std::fprintf(f, "# MEV_INCLUDE_SCAT_E %d\n# mev_emissivity_units local_spectral_emissivity_proxy_per_MeV\n"
                        "# mev_opacity_units cm^-1\n",
                     on(HADROS_MEV_SCAT_E));
    } else {
        std::fprintf(f, "# MEV_ENERGY_MEV %g\n# MEV_NORM %g\n# MEV_CUDA_STATUS not_computed\n", mev_E_MeV, mev_norm);
    }
    std::fprintf(f, "# step_cap %d\n# rkf45_tolerance %g\n# camera_step_rg %g\n# camera_fov_deg %g\n",
                 p->max_steps, p->tolerance, p->h, p->fov_deg);
    std::fprintf(f, "# precision %s\n# backend hadros_b200\n",
                 p->precision == HADROS_PRECISION_MIXED ? "mixed_fp64_geodesic_fp32_transfer" : "fp64");
    std::fprintf(f, "# i j alpha beta tau_uhe P_surv_uhe I_obs_uhe captured "
                    "tau_mev P_surv_mev I_obs_mev r_neutrinosphere_rg leakage_mev\n");
    for (int j = 0; j < p->ny; ++j) {
        const double v = pixel_v(p, j);
        for (int i = 0; i < p->nx; ++i) {
            const size_t k = static_cast<size_t>(j) * p->nx + i;
            double m[5];
            mev.row(k, m);
            std::fprintf(f, "%d %d %.8e %.8e %.8e %.8e %.8e %d %.8e %.8e %.8e %.8e %.8e\n", i, j, pixel_u(p, i), v,
                         tau[k], P_surv[k], I_obs[k], fate[k] == HADROS_FATE_CAPTURED ? 1 : 0, m[0], m[1], m[2],
                         m[3], m[4]);
        }
    }
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    return ok ? HADROS_OK : ferr(HADROS_E_IO, std::string("write failed: ") + path);
}

int32_t write_kimg(const char* path, const hadros_params* p, double mev_E_MeV, double mev_norm, const double* tau,
                   const double* P_surv, const double* I_obs, const int8_t* fate, const MevCols& mev)
{
    if (!path || !kinds_ok(p) || !tau || !P_surv || !I_obs || !fate)
        return ferr(HADROS_E_ARG, "bad argument");
    FILE* f = std::fopen(path, "wb");
    if (!f) return ferr(HADROS_E_IO, std::string("Could not open binary output file: ") + path);
    const int32_t hdr_i[7] = {0x4B494D47, 1, 2, p->nx, p->ny, 13, 0};
    const double hdr_d[4] = {p->Enu_obs_GeV, mev_E_MeV, mev_norm, rad2deg(p->theta_obs_rad)};
    std::fwrite(hdr_i, sizeof(hdr_i), 1, f);
    std::fwrite(hdr_d, sizeof(hdr_d), 1, f);
    for (int j = 0; j < p->ny; ++j) {
        const double v = pixel_v(p, j);
        for (int i = 0; i < p->nx; ++i) {
            const size_t k = static_cast<size_t>(j) * p->nx + i;
            double row[13] = {static_cast<double>(i), static_cast<double>(j), pixel_u(p, i), v, tau[k],
                              P_surv[k], I_obs[k], fate[k] == HADROS_FATE_CAPTURED ? 1.0 : 0.0,
                              0.0, 0.0, 0.0, 0.0, 0.0};
            mev.row(k, row + 8);
            std::fwrite(row, sizeof(row), 1, f);
        }
    }
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    return ok ? HADROS_OK : ferr(HADROS_E_IO, std::string("write failed: ") + path);
}

}  // namespace

int32_t hadros_write_dat(const char* path, const hadros_params* p, const char* dis_model,
                         double mev_E_MeV, double mev_norm, const double* tau, const double* P_surv,
                         const double* I_obs, const int8_t* fate)
{
    return write_dat(path, p, dis_model, mev_E_MeV, mev_norm, tau, P_surv, I_obs, fate, MevCols{});
}

int32_t hadros_write_kimg(const char* path, const hadros_params* p, double mev_E_MeV, double mev_norm,
                          const double* tau, const double* P_surv, const double* I_obs, const int8_t* fate)
{
    return write_kimg(path, p, mev_E_MeV, mev_norm, tau, P_surv, I_obs, fate, MevCols{});
}

int32_t hadros_write_dat_mev(const char* path, const hadros_params* p, const char* dis_model,
                             const hadros_image_out* host)
{
    if (!host || !p) return ferr(HADROS_E_ARG, "bad argument");
    return write_dat(path, p, dis_model, p->mev_Enu_obs_MeV, p->mev_norm, host->tau, host->P_surv, host->I_obs,
                     host->fate, mev_cols(host));
}

int32_t hadros_write_kimg_mev(const char* path, const hadros_params* p, const hadros_image_out* host)
{
    if (!host || !p) return ferr(HADROS_E_ARG, "bad argument");
    return write_kimg(path, p, p->mev_Enu_obs_MeV, p->mev_norm, host->tau, host->P_surv, host->I_obs, host->fate,
                      mev_cols(host));
}

int32_t hadros_write_kgeo(const char* path, const hadros_params* p, int32_t n_rays, const int32_t* pixel_ids,
                          const int8_t* fate, const int32_t* npoints, const double* points)
{
    return hadros_write_kgeo_rays(path, p, n_rays, pixel_ids, fate, npoints, points, 0);
}

int32_t hadros_write_kgeo_rays(const char* path, const hadros_params* p, int32_t n_rays, const int32_t* pixel_ids,
                               const int8_t* fate, const int32_t* npoints, const double* points, int32_t append)
{
    if (!path || !kinds_ok(p) || n_rays < 0 || (n_rays > 0 && (!npoints || !points)))
        return ferr(HADROS_E_ARG, "bad argument");
    if (append) {   // rays only go after a header: the file must exist
        FILE* g = std::fopen(path, "rb");
        if (!g) return ferr(HADROS_E_IO, std::string("No KGEO file to append to: ") + path);
        std::fclose(g);
    }
    FILE* f = std::fopen(path, append ? "ab" : "wb");
    if (!f) return ferr(HADROS_E_IO, std::string("Could not open ") + path);
    if (!append) {
        const int32_t hdr[4] = {0x4B47454F, 1, p->nx, p->ny};
        std::fwrite(hdr, sizeof(hdr), 1, f);
        std::fwrite(&p->a_spin, sizeof(double), 1, f);
    }
    int64_t off = 0;
    for (int32_t k = 0; k < n_rays; ++k) {
        const int32_t pid = pixel_ids ? pixel_ids[k] : k;
        const int32_t i = pid % p->nx, j = pid / p->nx;
        unsigned char rh[40] = {0};
        const int32_t ints[5] = {i * p->ny + j, i, j, (fate && fate[k] == HADROS_FATE_CAPTURED) ? 1 : 0, npoints[k]};
        const double ab[2] = {pixel_u(p, i), pixel_v(p, j)};
        std::memcpy(rh, ints, sizeof(ints));
        std::memcpy(rh + 24, ab, sizeof(ab));
        std::fwrite(rh, sizeof(rh), 1, f);
        if (npoints[k] > 0) std::fwrite(points + 7 * off, 56, static_cast<size_t>(npoints[k]), f);
        off += npoints[k];
    }
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    return ok ? HADROS_OK : ferr(HADROS_E_IO, std::string("write failed: ") + path);
}

namespace {

// Walk a KGEO file; with sink arrays NULL only counts.
int32_t kgeo_walk(const char* path, int32_t* nx, int32_t* ny, double* a, int32_t* n_rays, int64_t* n_points,
                  int32_t* pixel_ids, int8_t* captured, int32_t* npoints, double* alpha, double* beta,
                  double* points)
{
    if (!path) return ferr(HADROS_E_ARG, "path is NULL");
    FILE* f = std::fopen(path, "rb");
    if (!f) return ferr(HADROS_E_IO, std::string("Could not open geodesic cache ") + path);
    int32_t hdr[4];
    double spin = 0.0;
    if (std::fread(hdr, sizeof(hdr), 1, f) != 1 || std::fread(&spin, sizeof(double), 1, f) != 1) {
        std::fclose(f);
        return ferr(HADROS_E_IO, "Invalid binary geodesic cache: short header");
    }
    if (hdr[0] != 0x4B47454F) {   // apps/compute_kerr_image_from_cache.cpp:385-389
        std::fclose(f);
        return ferr(HADROS_E_IO, "Invalid binary geodesic cache: bad magic number");
    }
    if (hdr[1] != 1) {
        std::fclose(f);
        return ferr(HADROS_E_IO, "Unsupported binary geodesic cache version: " + std::to_string(hdr[1]));
    }
    if (hdr[2] <= 0 || hdr[3] <= 0) {
        std::fclose(f);
        return ferr(HADROS_E_IO, "Invalid binary geodesic cache: bad image size");
    }
    int32_t rays = 0;
    int64_t pts = 0;
    unsigned char rh[40];
    while (std::fread(rh, sizeof(rh), 1, f) == 1) {
        int32_t ints[5];
        double ab[2];
        std::memcpy(ints, rh, sizeof(ints));
        std::memcpy(ab, rh + 24, sizeof(ab));
        if (ints[4] < 0) {   // :666-669
            std::fclose(f);
            return ferr(HADROS_E_IO, "Invalid ray with negative number of points");
        }
        if (ints[1] < 0 || ints[1] >= hdr[2] || ints[2] < 0 || ints[2] >= hdr[3]) {
            std::fclose(f);
            return ferr(HADROS_E_IO, "Invalid binary geodesic cache: pixel index outside the image");
        }
        if (pixel_ids) {
            pixel_ids[rays] = ints[2] * hdr[2] + ints[1];
            captured[rays] = static_cast<int8_t>(ints[3] != 0);
            npoints[rays] = ints[4];
            alpha[rays] = ab[0];
            beta[rays] = ab[1];
        }
        if (ints[4] > 0) {
            if (points) {
                if (std::fread(points + 7 * pts, 56, static_cast<size_t>(ints[4]), f) != static_cast<size_t>(ints[4])) {
                    std::fclose(f);
                    return ferr(HADROS_E_IO, "Unexpected end of file while reading points");
                }
            } else if (std::fseek(f, 56L * ints[4], SEEK_CUR) != 0) {
                std::fclose(f);
                return ferr(HADROS_E_IO, "Unexpected end of file while reading points");
            }
        }
        ++rays;
        pts += ints[4];
    }
    // the file must end exactly after the last ray (a short trailing ray
    // header or a point block cut by the end of the file is an error)
    std::fseek(f, 0, SEEK_END);
    const long end = std::ftell(f);
    std::fclose(f);
    if (24 + 40LL * rays + 56LL * pts != end) return ferr(HADROS_E_IO, "Unexpected end of file while reading points");
    if (nx) *nx = hdr[2];
    if (ny) *ny = hdr[3];
    if (a) *a = spin;
    if (n_rays) *n_rays = rays;
    if (n_points) *n_points = pts;
    return HADROS_OK;
}

}  // namespace

int32_t hadros_kgeo_info(const char* path, int32_t* nx, int32_t* ny, double* a_spin, int32_t* n_rays,
                         int64_t* n_points)
{
    return kgeo_walk(path, nx, ny, a_spin, n_rays, n_points, nullptr, nullptr, nullptr, nullptr, nullptr,
                     nullptr);
}

int32_t hadros_read_kgeo(const char* path, int32_t* pixel_ids, int8_t* captured, int32_t* npoints,
                         double* alpha, double* beta, double* points)
{
    if (!pixel_ids || !captured || !npoints || !alpha || !beta || !points)
        return ferr(HADROS_E_ARG, "NULL output array");
    return kgeo_walk(path, nullptr, nullptr, nullptr, nullptr, nullptr, pixel_ids, captured, npoints, alpha,
                     beta, points);
}

}  // extern "C"
