// compute_kerr_image — drop-in command-line front end of libhadros_b200.
//
// Positional arguments 1-44 have the order and meaning of the reference GPU
// executable (apps/compute_kerr_image_cuda.cu:2303-2358, usage at :2222-2235):
//   ENU ASPIN MBH_MSUN TORUS_RHO0 TORUS_R0 TORUS_SIGMA TORUS_H_OVER_R
//   SOURCE_R SOURCE_SIGMA SOURCE_THETA_DEG SOURCE_POWERLAW SOURCE_EMAX SOURCE_NORM
//   MEV_ENU MEV_NORM CAM_THETA_DEG CAM_R_OBS CAM_FOV CAM_NX CAM_NY CAM_R_MAX CAM_STEP
//   GPU_TILE GPU_STEPS_PER_LAUNCH GPU_MAX_STEPS GPU_TOL
//   [PROFILE RADIAL_POWER FUNNEL_DEPLETION FUNNEL_THETA_DEG ENVELOPE_RHO0
//    ENVELOPE_ALPHA R_MIN R_MAX RHO_FLOOR SOURCE_MODEL SOURCE_FUNNEL_THETA_DEG
//    SOURCE_DENSITY_Q SOURCE_RADIAL_S SOURCE_GRADIENT_DR SOURCE_GRADIENT_DTHETA_DEG
//    SOURCE_RHO_REF SOURCE_CUTOFF_MIN SOURCE_CUTOFF_MAX]
// GPU_TILE and GPU_STEPS_PER_LAUNCH are accepted and ignored: one persistent
// launch traces the whole image.  GPU_TOL defaults to the CPU image path's
// RKF45 tolerance 1e-6 (include/kerr_geodesic.hpp:12).
//
// Named options (anywhere): --sigma=FILE (default
// data/sigma/sigma_nuN_CC_GBW.dat, as the reference hard-codes at :2366),
// --spectral=MODEL --gamma=G --ecut=E --emin=E --emax=E --nbins=N (the CPU
// app's spectral arguments, apps/compute_kerr_image_from_cache.cpp:271-288),
// --precision=fp64|mixed, --device=N, --outdir=DIR (default output/images),
// and the MeV thermal channel, which the CPU app computes with arguments
// 45-71 (apps/compute_kerr_image_from_cache.cpp:201-305): --mev=physical|toy|off
// (default physical), --mev-flavor=, --mev-thermal=, --mev-ye=,
// --mev-spectral=, --mev-emin=, --mev-emax=, --mev-nbins=, --mev-t0=,
// --mev-tfloor=, --mev-tpower=, --mev-ye-torus=, --mev-ye-funnel=,
// --mev-ye-envelope=, --mev-ye-floor=, --mev-ye-ceil=, --mev-sigma-abs=,
// --mev-sigma-scat=, --mev-nusphere-tau= and the 0/1 switches --mev-urca=,
// --mev-pair=, --mev-brems=, --mev-absorption=, --mev-scattering=,
// --mev-degeneracy=, --mev-abs-n=, --mev-abs-p=, --mev-scat-n=, --mev-scat-p=,
// --mev-scat-e=.  Its five columns go into both output files.
//
// Writes DIR/<name>.bin (KIMG) and DIR/<name>.dat with the reference's file
// name (apps/compute_kerr_image_cuda.cu:2108-2128) and prints the reference's
// "Saved:" and "CUDA timing:" lines.  Errors go to stderr with exit code 1.
//
// The reference executable's two cache modes (:1624-2200) are here too:
//   --geodesic-cache ASPIN CAM_R_OBS CAM_THETA_DEG CAM_FOV_DEG CAM_NX CAM_NY
//       CAM_R_MAX CAM_STEP GPU_CACHE_RAYS GPU_CACHE_MAX_POINTS GPU_TOL
//     traces every pixel, keeps at most GPU_CACHE_MAX_POINTS points per ray (a
//     ray that reaches the limit stops there, uncaptured), and writes the KGEO
//     cache output/rays/kerr_geodesics_cuda.bin; exit code 2 when a ray was
//     cut, as the reference does;
//   --image-from-cache ENU ASPIN MBH_MSUN TORUS_RHO0 TORUS_R0 TORUS_SIGMA
//       TORUS_H_OVER_R SOURCE_R SOURCE_SIGMA SOURCE_THETA_DEG SOURCE_POWERLAW
//       SOURCE_EMAX SOURCE_NORM MEV_ENU MEV_NORM CAM_THETA_DEG GPU_CACHE_RAYS
//       [PROFILE ... SOURCE_CUTOFF_MAX, the in-line mode's arguments 27-44]
//     transfers over that cache (FP64) and writes
//     kerr_image_cuda_cache_rho0_torus_....{bin,dat}.
// GPU_CACHE_RAYS only sizes the reference's batches; here batches are sized by
// memory.  GPU_TOL defaults to 1e-6 as in the in-line mode.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "../../include/hadros_b200.h"

namespace {

constexpr double PI = 3.141592653589793238462643383279502884;

void usage(const char* argv0)
{
    std::fprintf(stderr,
                 "Usage:\n  %s ENU ASPIN MBH_MSUN TORUS_RHO0 TORUS_R0 TORUS_SIGMA TORUS_H_OVER_R"
                 " SOURCE_R SOURCE_SIGMA SOURCE_THETA_DEG SOURCE_POWERLAW SOURCE_EMAX SOURCE_NORM"
                 " MEV_ENU MEV_NORM CAM_THETA_DEG CAM_R_OBS CAM_FOV CAM_NX CAM_NY CAM_R_MAX CAM_STEP"
                 " GPU_TILE GPU_STEPS_PER_LAUNCH GPU_MAX_STEPS GPU_TOL"
                 " [PROFILE RADIAL_POWER FUNNEL_DEPLETION FUNNEL_THETA_DEG"
                 " ENVELOPE_RHO0 ENVELOPE_ALPHA R_MIN R_MAX RHO_FLOOR"
                 " SOURCE_MODEL SOURCE_FUNNEL_THETA_DEG SOURCE_DENSITY_Q"
                 " SOURCE_RADIAL_S SOURCE_GRADIENT_DR SOURCE_GRADIENT_DTHETA_DEG"
                 " SOURCE_RHO_REF SOURCE_CUTOFF_MIN SOURCE_CUTOFF_MAX]\n"
                 "  options: --sigma=FILE --spectral=MODEL --gamma=G --ecut=E --emin=E --emax=E"
                 " --nbins=N --precision=fp64|mixed --device=N --outdir=DIR\n"
                 "  MeV channel: --mev=physical|toy|off --mev-flavor=F --mev-thermal=T --mev-ye=Y"
                 " --mev-spectral=S --mev-emin=E --mev-emax=E --mev-nbins=N --mev-t0=T --mev-tfloor=T"
                 " --mev-tpower=P --mev-ye-torus=Y --mev-ye-funnel=Y --mev-ye-envelope=Y"
                 " --mev-ye-floor=Y --mev-ye-ceil=Y --mev-sigma-abs=S --mev-sigma-scat=S"
                 " --mev-nusphere-tau=T --mev-{urca,pair,brems,absorption,scattering,degeneracy,"
                 "abs-n,abs-p,scat-n,scat-p,scat-e}=0|1\n",
                 argv0);
}

int die(const char* what)
{
    std::fprintf(stderr, "%s: %s\n", what, hadros_last_error());
    return 1;
}

// One --mev-* option into the parameters; false for an unknown key, and
// *bad for a value the reference's parsers reject.
bool mev_option(hadros_params& p, const std::string& key, const std::string& val, bool* bad)
{
    const double x = std::atof(val.c_str());
    struct Num { const char* k; double* f; } nums[] = {
        {"mev-emin", &p.mev_E_min_MeV}, {"mev-emax", &p.mev_E_max_MeV}, {"mev-t0", &p.mev_T0_MeV},
        {"mev-tfloor", &p.mev_T_floor_MeV}, {"mev-tpower", &p.mev_T_power}, {"mev-ye-torus", &p.mev_Ye_torus},
        {"mev-ye-funnel", &p.mev_Ye_funnel}, {"mev-ye-envelope", &p.mev_Ye_envelope},
        {"mev-ye-floor", &p.mev_Ye_floor}, {"mev-ye-ceil", &p.mev_Ye_ceil},
        {"mev-sigma-abs", &p.mev_sigma_abs0_cm2}, {"mev-sigma-scat", &p.mev_sigma_scat0_cm2},
        {"mev-nusphere-tau", &p.mev_neutrinosphere_tau}};
    for (const Num& n : nums)
        if (key == n.k) { *n.f = x; return true; }
    struct Bit { const char* k; uint32_t bit; } bits[] = {
        {"mev-urca", HADROS_MEV_URCA}, {"mev-pair", HADROS_MEV_PAIR}, {"mev-brems", HADROS_MEV_BREMS},
        {"mev-absorption", HADROS_MEV_ABSORPTION}, {"mev-scattering", HADROS_MEV_SCATTERING},
        {"mev-degeneracy", HADROS_MEV_DEGENERACY_CORRECTION}, {"mev-abs-n", HADROS_MEV_ABS_N},
        {"mev-abs-p", HADROS_MEV_ABS_P}, {"mev-scat-n", HADROS_MEV_SCAT_N}, {"mev-scat-p", HADROS_MEV_SCAT_P},
        {"mev-scat-e", HADROS_MEV_SCAT_E}};
    for (const Bit& b : bits)
        if (key == b.k) {   // std::atoi(argv) != 0, as the CPU app reads its switches
            if (std::atoi(val.c_str()) != 0) p.mev_flags |= b.bit;
            else p.mev_flags &= ~b.bit;
            return true;
        }
    if (key == "mev-nbins") { p.mev_n_bins = std::atoi(val.c_str()); return true; }
    if (key == "mev") {
        if (val == "off") { p.mev_channel = 0; return true; }
        p.mev_channel = 1;
        *bad = hadros_parse_mev_model(val.c_str(), &p.mev_model) != 0;
        return true;
    }
    if (key == "mev-flavor") { *bad = hadros_parse_mev_flavor(val.c_str(), &p.mev_flavor) != 0; return true; }
    if (key == "mev-thermal") { *bad = hadros_parse_mev_thermal(val.c_str(), &p.mev_thermal_profile) != 0; return true; }
    if (key == "mev-ye") { *bad = hadros_parse_mev_ye(val.c_str(), &p.mev_ye_profile) != 0; return true; }
    if (key == "mev-spectral") {
        *bad = hadros_parse_mev_spectral(val.c_str(), &p.mev_spectral_mode) != 0;
        return true;
    }
    return false;
}

}  // namespace

double num(const std::vector<std::string>& pos, size_t k, double def)
{
    return pos.size() > k ? std::atof(pos[k].c_str()) : def;
}

// --geodesic-cache (apps/compute_kerr_image_cuda.cu:1624-1824)
int geodesic_cache(const std::vector<std::string>& pos, int device)
{
    hadros_params p;
    hadros_params_default(&p);
    p.a_spin = num(pos, 0, 0.9);
    p.r_obs_rg = num(pos, 1, 60.0);
    p.theta_obs_rad = num(pos, 2, 80.0) * PI / 180.0;
    p.fov_deg = num(pos, 3, 25.0);
    p.nx = pos.size() > 4 ? std::atoi(pos[4].c_str()) : 100;
    p.ny = pos.size() > 5 ? std::atoi(pos[5].c_str()) : 100;
    p.r_max_rg = num(pos, 6, 120.0);
    p.h = num(pos, 7, 0.001);
    const int cache_rays = pos.size() > 8 ? std::atoi(pos[8].c_str()) : 32;
    const int max_points = pos.size() > 9 ? std::atoi(pos[9].c_str()) : 50000;
    p.tolerance = num(pos, 10, 1.0e-6);
    if (p.nx <= 0 || p.ny <= 0 || cache_rays <= 0 || max_points <= 0) {
        std::fprintf(stderr, "Usage: compute_kerr_image --geodesic-cache ASPIN CAM_R_OBS CAM_THETA_DEG "
                             "CAM_FOV_DEG CAM_NX CAM_NY CAM_R_MAX CAM_STEP GPU_CACHE_RAYS "
                             "GPU_CACHE_MAX_POINTS GPU_TOL\n");
        return 1;
    }
    // a ray stops at its max_points-th point (trace_cache_kernel, :1478-1535)
    if (max_points < p.max_steps) p.max_steps = max_points;
    if (hadros_params_validate(&p)) return die("parameters");
    hadros_ctx* ctx = nullptr;
    if (hadros_ctx_create(device, &ctx)) return die("CUDA");
    const int64_t total = static_cast<int64_t>(p.nx) * p.ny;
    // batches of whole rays within ~512 MiB of path buffer
    int64_t batch = (512ll << 20) / (static_cast<int64_t>(max_points) * 56);
    if (batch < cache_rays) batch = cache_rays;
    if (batch > total) batch = total;
    if (batch < 1) batch = 1;
    std::printf("Geodesic cache grid: %d x %d\nBatch rays: %lld, max points/ray: %d, RKF45 tol: %g\n", p.nx,
                p.ny, static_cast<long long>(batch), max_points, p.tolerance);
    const std::string path = "output/rays/kerr_geodesics_cuda.bin";
    std::vector<double> buf(static_cast<size_t>(batch) * max_points * 7), packed;
    std::vector<int32_t> ids(static_cast<size_t>(batch)), npts(static_cast<size_t>(batch));
    std::vector<int8_t> fate(static_cast<size_t>(batch));
    int64_t total_points = 0, truncated = 0;
    const auto t0 = std::chrono::steady_clock::now();
    for (int64_t start = 0; start < total; start += batch) {
        const int32_t n = static_cast<int32_t>(std::min<int64_t>(batch, total - start));
        for (int32_t k = 0; k < n; ++k) {   // ray id = i * ny + j (init_linear_rays_kernel, :1412-1430)
            const int64_t id = start + k;
            const int32_t i = static_cast<int32_t>(id / p.ny), j = static_cast<int32_t>(id % p.ny);
            ids[k] = j * p.nx + i;
        }
        if (hadros_trace_paths(ctx, &p, ids.data(), n, max_points, buf.data(), npts.data(), fate.data()))
            return die("trace");
        packed.clear();
        for (int32_t k = 0; k < n; ++k) {
            const double* q = buf.data() + static_cast<size_t>(k) * max_points * 7;
            packed.insert(packed.end(), q, q + static_cast<size_t>(npts[k]) * 7);
            total_points += npts[k];
            if (npts[k] >= max_points && fate[k] != HADROS_FATE_CAPTURED) ++truncated;
        }
        if (hadros_write_kgeo_rays(path.c_str(), &p, n, ids.data(), fate.data(), npts.data(),
                                   packed.empty() ? nullptr : packed.data(), start > 0 ? 1 : 0))
            return die("write");
    }
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("Saved: %s\nCached points: %lld\nGeodesic GPU timing: %g s, %g rays/s\n", path.c_str(),
                static_cast<long long>(total_points), elapsed,
                static_cast<double>(total) / std::max(elapsed, 1.0e-300));
    hadros_ctx_destroy(ctx);
    if (truncated > 0) {   // :1811-1820
        std::fprintf(stderr, "ERROR: %lld rays reached GPU_CACHE_MAX_POINTS. Do not use this cache for science. "
                             "Increase GPU_CACHE_MAX_POINTS or CAM_STEP, then regenerate %s.\n",
                     static_cast<long long>(truncated), path.c_str());
        return 2;
    }
    return 0;
}

// --image-from-cache (apps/compute_kerr_image_cuda.cu:1826-2200): the
// in-line mode's physics over the cached paths, FP64, with the MeV channel.
int image_from_cache(const std::vector<std::string>& pos, int device, const std::string& sigma_path,
                     const std::string& outdir, hadros_params p)
{
    // defaults of run_image_from_cache_gpu (:1830-1868)
    p.Enu_obs_GeV = num(pos, 0, 1.0e9);
    p.a_spin = num(pos, 1, 0.9);
    p.M_bh_msun = num(pos, 2, 3.0);
    p.rho0_gcm3 = num(pos, 3, 1.0e-2);
    p.r0_rg = num(pos, 4, 10.0);
    p.sigma_r_rg = num(pos, 5, 5.0);
    p.H_over_R = num(pos, 6, 0.25);
    p.src_r_center_rg = num(pos, 7, 3.5);
    p.src_sigma_r_rg = num(pos, 8, 1.0);
    p.src_theta_width_rad = num(pos, 9, 15.0) * PI / 180.0;
    p.src_powerlaw = num(pos, 10, 2.0);
    p.src_emax_GeV = num(pos, 11, 1.0e12);
    p.src_norm = num(pos, 12, 1.0);
    p.mev_Enu_obs_MeV = num(pos, 13, 10.0);
    p.mev_norm = num(pos, 14, 1.0);
    p.theta_obs_rad = num(pos, 15, 80.0) * PI / 180.0;
    const int chunk = pos.size() > 16 ? std::atoi(pos[16].c_str()) : 256;
    if (pos.size() > 17 && hadros_parse_profile(pos[17].c_str(), &p.profile_kind)) return die("profile");
    p.radial_power = num(pos, 18, 2.0);
    p.funnel_depletion = num(pos, 19, 0.0);
    p.funnel_theta_rad = num(pos, 20, 15.0) * PI / 180.0;
    p.envelope_rho0_gcm3 = num(pos, 21, 0.0);
    p.envelope_alpha = num(pos, 22, 2.5);
    p.torus_r_min_rg = num(pos, 23, 4.0);
    p.torus_r_max_rg = num(pos, 24, 60.0);
    p.rho_floor_gcm3 = num(pos, 25, 1.0e-99);
    if (pos.size() > 26 && hadros_parse_source(pos[26].c_str(), &p.source_kind)) return die("source model");
    p.src_funnel_theta_rad = num(pos, 27, 20.0) * PI / 180.0;
    p.src_density_power_q = num(pos, 28, 1.0);
    p.src_radial_power_s = num(pos, 29, 2.0);
    p.src_gradient_dr_rg = num(pos, 30, 0.1);
    p.src_gradient_dtheta_rad = num(pos, 31, 1.0) * PI / 180.0;
    p.src_rho_ref_gcm3 = num(pos, 32, -1.0);
    p.src_cutoff_min = num(pos, 33, 0.0);
    p.src_cutoff_max = num(pos, 34, 1.0e2);
    if (chunk <= 0) {
        std::fprintf(stderr, "Usage: compute_kerr_image --image-from-cache ENU ASPIN MBH_MSUN TORUS_RHO0 TORUS_R0 "
                             "TORUS_SIGMA TORUS_H_OVER_R SOURCE_R SOURCE_SIGMA SOURCE_THETA_DEG SOURCE_POWERLAW "
                             "SOURCE_EMAX SOURCE_NORM MEV_ENU MEV_NORM CAM_THETA_DEG GPU_CACHE_RAYS [PROFILE "
                             "RADIAL_POWER FUNNEL_DEPLETION FUNNEL_THETA_DEG ENVELOPE_RHO0 ENVELOPE_ALPHA R_MIN "
                             "R_MAX RHO_FLOOR SOURCE_MODEL SOURCE_FUNNEL_THETA_DEG SOURCE_DENSITY_Q "
                             "SOURCE_RADIAL_S SOURCE_GRADIENT_DR SOURCE_GRADIENT_DTHETA_DEG]\n");
        return 1;
    }
    p.spectral_kind = HADROS_SPECTRAL_MONOCHROMATIC;
    p.precision = HADROS_PRECISION_FP64;
    const std::string path = "output/rays/kerr_geodesics_cuda.bin";
    int32_t nx = 0, ny = 0, n_rays = 0;
    double cache_a = 0.0;
    int64_t n_points = 0;
    if (hadros_kgeo_info(path.c_str(), &nx, &ny, &cache_a, &n_rays, &n_points)) return die("cache");
    p.nx = nx;
    p.ny = ny;
    if (std::fabs(cache_a - p.a_spin) > 1.0e-12)   // :1970-1975
        std::fprintf(stderr, "Warning: cache spin a=%g differs from requested ASPIN=%g\n", cache_a, p.a_spin);
    if (hadros_params_validate(&p)) return die("parameters");
    std::vector<int32_t> pid(static_cast<size_t>(n_rays)), npts(static_cast<size_t>(n_rays));
    std::vector<int8_t> captured(static_cast<size_t>(n_rays)), fate(static_cast<size_t>(n_rays));
    std::vector<double> alpha(static_cast<size_t>(n_rays)), beta(static_cast<size_t>(n_rays));
    std::vector<double> pts(static_cast<size_t>(n_points) * 7 + 1);
    if (hadros_read_kgeo(path.c_str(), pid.data(), captured.data(), npts.data(), alpha.data(), beta.data(),
                         pts.data()))
        return die("cache");
    for (int32_t k = 0; k < n_rays; ++k) fate[k] = captured[k] ? HADROS_FATE_CAPTURED : HADROS_FATE_ESCAPED;
    hadros_sigma* sig = nullptr;
    if (hadros_sigma_load(sigma_path.c_str(), &sig)) return die("sigma table");
    hadros_ctx* ctx = nullptr;
    if (hadros_ctx_create(device, &ctx)) return die("CUDA");
    std::vector<double> r_tau(static_cast<size_t>(n_rays)), r_P(static_cast<size_t>(n_rays)),
        r_I(static_cast<size_t>(n_rays)), r_mev[5];
    for (auto& v : r_mev) v.resize(static_cast<size_t>(n_rays));
    hadros_image_out ro{};
    ro.tau = r_tau.data();
    ro.P_surv = r_P.data();
    ro.I_obs = r_I.data();
    ro.tau_mev = r_mev[0].data();
    ro.P_surv_mev = r_mev[1].data();
    ro.I_obs_mev = r_mev[2].data();
    ro.r_nu = r_mev[3].data();
    ro.leakage = r_mev[4].data();
    const auto t0 = std::chrono::steady_clock::now();
    if (hadros_transfer_paths(ctx, &p, sig, n_rays, npts.data(), fate.data(), pts.data(), &ro))
        return die("transfer");
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    // rays in cache order -> pixel rows j*nx+i (a pixel missing from the cache keeps the defaults)
    const size_t P = static_cast<size_t>(nx) * ny;
    std::vector<double> tau(P, 0.0), Ps(P, 1.0), I(P, 0.0), mev[5];
    const double mev_def[5] = {0.0, 1.0, 0.0, -1.0, 1.0};
    for (int c = 0; c < 5; ++c) mev[c].assign(P, mev_def[c]);
    std::vector<int8_t> pfate(P, HADROS_FATE_ESCAPED);
    for (int32_t k = 0; k < n_rays; ++k) {
        const size_t q = static_cast<size_t>(pid[k]);
        if (q >= P) continue;
        tau[q] = r_tau[k];
        Ps[q] = r_P[k];
        I[q] = r_I[k];
        pfate[q] = fate[k];
        for (int c = 0; c < 5; ++c) mev[c][q] = r_mev[c][k];
    }
    hadros_image_out out{};
    out.tau = tau.data();
    out.P_surv = Ps.data();
    out.I_obs = I.data();
    out.fate = pfate.data();
    out.tau_mev = mev[0].data();
    out.P_surv_mev = mev[1].data();
    out.I_obs_mev = mev[2].data();
    out.r_nu = mev[3].data();
    out.leakage = mev[4].data();
    char name[512];   // the in-line name with "cache_" after "kerr_image_cuda_" (:2110-2126)
    if (hadros_image_filename(&p, 0, nullptr, p.mev_Enu_obs_MeV, p.mev_norm, "", name, sizeof(name)))
        return die("file name");
    const std::string stem = std::string("kerr_image_cuda_cache_") + (name + std::strlen("kerr_image_cuda_"));
    const std::string bin_path = outdir + "/" + stem + ".bin", dat_path = outdir + "/" + stem + ".dat";
    if (hadros_write_kimg_mev(bin_path.c_str(), &p, &out)) return die("write");
    if (hadros_write_dat_mev(dat_path.c_str(), &p, "GBW", &out)) return die("write");
    std::printf("Cache grid: %d x %d\nLoaded rays: %d\nSaved: %s\nSaved: %s\n", nx, ny, n_rays, bin_path.c_str(),
                dat_path.c_str());
    std::printf("CUDA cache image timing: %g s, %g rays/s\n", elapsed,
                static_cast<double>(n_rays) / std::max(elapsed, 1.0e-300));
    hadros_ctx_destroy(ctx);
    hadros_sigma_destroy(sig);
    return 0;
}

int main(int argc, char** argv)
{
    std::vector<std::string> pos;
    std::vector<std::pair<std::string, std::string>> mev_opts;
    std::string sigma_path = "data/sigma/sigma_nuN_CC_GBW.dat", outdir = "output/images";
    std::string spectral, precision;
    double gamma = NAN, ecut = NAN, emin = NAN, emax = NAN;
    int nbins = -1, device = 0, mode = 0;
    for (int k = 1; k < argc; ++k) {
        std::string a(argv[k]);
        if (a.rfind("--", 0) == 0) {
            const size_t eq = a.find('=');
            const std::string key = a.substr(2, eq == std::string::npos ? std::string::npos : eq - 2);
            const std::string val = eq == std::string::npos ? "" : a.substr(eq + 1);
            if (key == "sigma") sigma_path = val;
            else if (key == "outdir") outdir = val;
            else if (key == "spectral") spectral = val;
            else if (key == "precision") precision = val;
            else if (key == "gamma") gamma = std::atof(val.c_str());
            else if (key == "ecut") ecut = std::atof(val.c_str());
            else if (key == "emin") emin = std::atof(val.c_str());
            else if (key == "emax") emax = std::atof(val.c_str());
            else if (key == "nbins") nbins = std::atoi(val.c_str());
            else if (key == "device") device = std::atoi(val.c_str());
            else if (key == "help") { usage(argv[0]); return 0; }
            else if (key == "geodesic-cache") mode = 1;
            else if (key == "image-from-cache") mode = 2;
            else if (key.rfind("mev", 0) == 0) mev_opts.emplace_back(key, val);
            else { std::fprintf(stderr, "unknown option %s\n", a.c_str()); usage(argv[0]); return 1; }
        } else {
            pos.push_back(a);
        }
    }
    if (mode == 1) return geodesic_cache(pos, device);
    auto has = [&](size_t i) { return pos.size() >= i; };
    auto f = [&](size_t i) { return std::atof(pos[i - 1].c_str()); };
    auto n = [&](size_t i) { return std::atoi(pos[i - 1].c_str()); };

    hadros_params p;
    hadros_params_default(&p);
    // compute_kerr_image_cuda defaults (apps/compute_kerr_image_cuda.cu:2250-2297)
    p.Enu_obs_GeV = 1.0e9; p.a_spin = 0.9; p.M_bh_msun = 3.0;
    p.rho0_gcm3 = 1.0e-2; p.r0_rg = 10.0; p.sigma_r_rg = 5.0; p.H_over_R = 0.25;
    p.profile_kind = HADROS_PROFILE_GAUSSIAN; p.radial_power = 2.0; p.funnel_depletion = 0.0;
    p.funnel_theta_rad = 15.0 * PI / 180.0; p.envelope_rho0_gcm3 = 0.0; p.envelope_alpha = 2.5;
    p.torus_r_min_rg = 4.0; p.torus_r_max_rg = 60.0; p.rho_floor_gcm3 = 1.0e-99;
    p.src_r_center_rg = 3.5; p.src_sigma_r_rg = 1.0; p.src_theta_width_rad = 15.0 * PI / 180.0;
    p.src_powerlaw = 2.0; p.src_emax_GeV = 1.0e12; p.src_norm = 1.0;
    p.source_kind = HADROS_SOURCE_INNER_RING; p.src_funnel_theta_rad = 20.0 * PI / 180.0;
    p.src_density_power_q = 1.0; p.src_radial_power_s = 2.0; p.src_rho_ref_gcm3 = -1.0;
    p.src_cutoff_min = 0.0; p.src_cutoff_max = 1.0e2; p.src_gradient_dr_rg = 0.1;
    p.src_gradient_dtheta_rad = 1.0 * PI / 180.0;
    double mev_E = 10.0, mev_norm = 1.0;
    p.mev_channel = 1;   // the CPU app always runs its physical MeV block
    p.r_obs_rg = 60.0; p.theta_obs_rad = 80.0 * PI / 180.0; p.fov_deg = 25.0;
    p.nx = 100; p.ny = 100; p.r_max_rg = 120.0; p.h = 0.001; p.tolerance = 1.0e-6;
    p.max_steps = 200000;
    int tile = 32, steps_per_launch = 128;

    if (mode == 2) {   // the cached-image mode: its own positional order, the named MeV options
        for (const auto& kv : mev_opts) {
            bool bad = false;
            if (!mev_option(p, kv.first, kv.second, &bad)) {
                std::fprintf(stderr, "unknown option --%s\n", kv.first.c_str());
                return 1;
            }
            if (bad) return die("MeV channel");
        }
        return image_from_cache(pos, device, sigma_path, outdir, p);
    }
    if (has(1)) p.Enu_obs_GeV = f(1);
    if (has(2)) p.a_spin = f(2);
    if (has(3)) p.M_bh_msun = f(3);
    if (has(4)) p.rho0_gcm3 = f(4);
    if (has(5)) p.r0_rg = f(5);
    if (has(6)) p.sigma_r_rg = f(6);
    if (has(7)) p.H_over_R = f(7);
    if (has(8)) p.src_r_center_rg = f(8);
    if (has(9)) p.src_sigma_r_rg = f(9);
    if (has(10)) p.src_theta_width_rad = f(10) * PI / 180.0;
    if (has(11)) p.src_powerlaw = f(11);
    if (has(12)) p.src_emax_GeV = f(12);
    if (has(13)) p.src_norm = f(13);
    if (has(14)) mev_E = f(14);
    if (has(15)) mev_norm = f(15);
    if (has(16)) p.theta_obs_rad = f(16) * PI / 180.0;
    if (has(17)) p.r_obs_rg = f(17);
    if (has(18)) p.fov_deg = f(18);
    if (has(19)) p.nx = n(19);
    if (has(20)) p.ny = n(20);
    if (has(21)) p.r_max_rg = f(21);
    if (has(22)) p.h = f(22);
    if (has(23)) tile = n(23);
    if (has(24)) steps_per_launch = n(24);
    if (has(25)) p.max_steps = n(25);
    if (has(26)) p.tolerance = f(26);
    if (has(27) && hadros_parse_profile(pos[26].c_str(), &p.profile_kind)) return die("profile");
    if (has(28)) p.radial_power = f(28);
    if (has(29)) p.funnel_depletion = f(29);
    if (has(30)) p.funnel_theta_rad = f(30) * PI / 180.0;
    if (has(31)) p.envelope_rho0_gcm3 = f(31);
    if (has(32)) p.envelope_alpha = f(32);
    if (has(33)) p.torus_r_min_rg = f(33);
    if (has(34)) p.torus_r_max_rg = f(34);
    if (has(35)) p.rho_floor_gcm3 = f(35);
    if (has(36) && hadros_parse_source(pos[35].c_str(), &p.source_kind)) return die("source model");
    if (has(37)) p.src_funnel_theta_rad = f(37) * PI / 180.0;
    if (has(38)) p.src_density_power_q = f(38);
    if (has(39)) p.src_radial_power_s = f(39);
    if (has(40)) p.src_gradient_dr_rg = f(40);
    if (has(41)) p.src_gradient_dtheta_rad = f(41) * PI / 180.0;
    if (has(42)) p.src_rho_ref_gcm3 = f(42);
    if (has(43)) p.src_cutoff_min = f(43);
    if (has(44)) p.src_cutoff_max = f(44);
    if (!spectral.empty() && hadros_parse_spectral(spectral.c_str(), &p.spectral_kind)) return die("spectral model");
    if (!std::isnan(gamma)) p.spec_gamma = gamma;
    if (!std::isnan(ecut)) p.spec_ecut_GeV = ecut;
    if (!std::isnan(emin)) p.spec_e_min_GeV = emin;
    if (!std::isnan(emax)) p.spec_e_max_GeV = emax;
    if (nbins > 0) p.n_bins = nbins;
    p.mev_Enu_obs_MeV = mev_E;
    p.mev_norm = mev_norm;
    for (const auto& kv : mev_opts) {
        bool bad = false;
        if (!mev_option(p, kv.first, kv.second, &bad)) {
            std::fprintf(stderr, "unknown option --%s\n", kv.first.c_str());
            usage(argv[0]);
            return 1;
        }
        if (bad) return die("MeV channel");
    }
    if (precision == "mixed") p.precision = HADROS_PRECISION_MIXED;
    else if (!precision.empty() && precision != "fp64") { usage(argv[0]); return 1; }

    if (p.nx <= 0 || p.ny <= 0 || tile <= 0 || steps_per_launch <= 0 || p.max_steps <= 0) {
        usage(argv[0]);   // apps/compute_kerr_image_cuda.cu:2360-2364
        return 1;
    }
    if (hadros_params_validate(&p)) return die("parameters");

    hadros_sigma* sig = nullptr;
    if (hadros_sigma_load(sigma_path.c_str(), &sig)) return die("sigma table");
    hadros_ctx* ctx = nullptr;
    if (hadros_ctx_create(device, &ctx)) return die("CUDA");
    const size_t P = static_cast<size_t>(p.nx) * p.ny;
    std::vector<double> tau(P), Ps(P), I(P);
    std::vector<int8_t> fate(P);
    std::vector<int32_t> steps(P);
    std::vector<double> mev[5];
    hadros_image_out out{};
    out.tau = tau.data();
    out.P_surv = Ps.data();
    out.I_obs = I.data();
    out.fate = fate.data();
    out.steps = steps.data();
    if (p.mev_channel) {
        for (auto& v : mev) v.resize(P);
        out.tau_mev = mev[0].data();
        out.P_surv_mev = mev[1].data();
        out.I_obs_mev = mev[2].data();
        out.r_nu = mev[3].data();
        out.leakage = mev[4].data();
    }
    std::printf("Grid: %d x %d\n", p.nx, p.ny);
    const auto t0 = std::chrono::steady_clock::now();
    if (hadros_image(ctx, &p, sig, &out)) return die("trace");
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    hadros_stats st{};
    hadros_ctx_stats(ctx, &st);

    char name_bin[512], name_dat[512];
    if (hadros_image_filename(&p, 0, nullptr, mev_E, mev_norm, ".bin", name_bin, sizeof(name_bin)) ||
        hadros_image_filename(&p, 0, nullptr, mev_E, mev_norm, ".dat", name_dat, sizeof(name_dat)))
        return die("file name");
    const std::string bin_path = outdir + "/" + name_bin, dat_path = outdir + "/" + name_dat;
    if (hadros_write_kimg_mev(bin_path.c_str(), &p, &out)) return die("write");
    if (hadros_write_dat_mev(dat_path.c_str(), &p, "GBW", &out)) return die("write");
    std::printf("Saved: %s\nSaved: %s\n", bin_path.c_str(), dat_path.c_str());
    std::printf("CUDA timing: %g s, %g rays/s, tiles=1, advance launches=%d, accepted steps=%lld\n", elapsed,
                static_cast<double>(P) / std::max(elapsed, 1.0e-300), st.launches,
                static_cast<long long>(st.accepted_steps));
    hadros_ctx_destroy(ctx);
    hadros_sigma_destroy(sig);
    return 0;
}
