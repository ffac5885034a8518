// hadros_trace.cu — the sm_100a trace kernel and its host-side plan builder.
//
// One persistent kernel does the whole per-pixel pipeline of the reference:
// camera ray setup (src/kerr_camera.cpp:110-186), the RKF45 trace loop with
// the RK4 fallback (src/kerr_camera.cpp:188-283, src/kerr_geodesic.cpp:
// 194-329), the per-point ZAMO interval and redshift (kerr_camera.cpp:46-76,
// :264-271) and, fused into the same loop, the UHE transfer of every
// spectral bin (src/radiative_transfer.cpp:457-685) and the spectral
// aggregation (:687-780).  Nothing is written to HBM per step: the ray state
// lives in registers, the sigma table and the per-bin accumulators of each
// thread's ray live in shared memory, and only the finished pixel is stored.
//
// Scheduling: every thread owns one ray at a time and pulls the next work
// item (camera, pixel) from a global cursor when its ray ends, so short
// (captured) and long (escaping) rays do not leave lanes idle until the end
// of a tile; each loop iteration runs exactly one RKF45 attempt on every lane
// that has a ray, which keeps the FP64 arithmetic of a warp converged.
//
// Parity: device code is compiled with --fmad=false and IEEE division and
// square root, and every expression keeps the reference's operand order, so
// the FP64 path differs from the reference CPU only through the
// transcendental functions (sin, cos, pow, exp, log) of the two math
// libraries.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <limits>

#include "hadros_internal.h"
#include "hadros_trace_kernel.cuh"

namespace hadros {

// ===================== host: per-camera plan ===============================

namespace {

Torus resolve_torus(const hadros_params& p)
{   // TorusProfile constructor clamps, src/torus_profile.cpp:20-41
    Torus t{};
    t.kind = p.profile_kind;
    const int k = p.profile_kind;
    t.use_powerlaw = (k == 1 || k == 3 || k == 5 || k == 6);   // :125-131
    t.use_funnel = (k == 2 || k == 3 || k == 6);               // :133-139
    t.use_envelope = (k == 4 || k == 5 || k == 6);             // :141-147
    t.rho0 = p.rho0_gcm3;
    t.r0 = p.r0_rg;
    t.sigma_r = p.sigma_r_rg;
    t.H = p.H_over_R;
    t.radial_power = p.radial_power;
    t.funnel_depletion = sclamp(p.funnel_depletion, 0.0, 1.0);
    t.funnel_theta = smax(p.funnel_theta_rad, 1.0e-6);
    t.env_rho0 = smax(p.envelope_rho0_gcm3, 0.0);
    t.env_alpha = p.envelope_alpha;
    t.r_min = p.torus_r_min_rg;
    t.r_max = smax(p.torus_r_max_rg, p.torus_r_min_rg);
    t.rho_floor = smax(p.rho_floor_gcm3, 0.0);
    return t;
}

// Largest gg with fl(E/gg) >= lo, smallest gg with fl(E/gg) <= hi (division
// rounds monotonically, so the in-range test becomes two compares on gg).
double gg_upper(double E, double lo)
{
    double x = E / lo;
    for (int it = 0; it < 64 && E / x >= lo; ++it) x = std::nextafter(x, std::numeric_limits<double>::infinity());
    for (int it = 0; it < 64 && !(E / x >= lo); ++it) x = std::nextafter(x, 0.0);
    return x;
}
double gg_lower(double E, double hi)
{
    double x = E / hi;
    for (int it = 0; it < 64 && E / x <= hi; ++it) x = std::nextafter(x, 0.0);
    for (int it = 0; it < 64 && !(E / x <= hi); ++it) x = std::nextafter(x, std::numeric_limits<double>::infinity());
    return x;
}

}  // namespace

void prepare_sigma(SigmaHost& s)
{
    const size_t n = s.E.size();
    s.lnE.resize(n);
    s.lnS.resize(n);
    s.lx.resize(n);
    s.seg.assign(4 * n, 0.0f);
    double smax_v = 0.0;
    for (size_t k = 0; k < n; ++k) {
        s.lnE[k] = std::log(s.E[k]);
        s.lnS[k] = std::log(s.s_cm2[k]);
        s.lx[k] = static_cast<float>(s.lnE[k]);
        smax_v = std::max(smax_v, s.s_cm2[k]);
    }
    s.sigma_scale = smax_v > 0.0 ? smax_v : 1.0;
    // even spacing in ln E (within 1e-5 of a step): the kernel indexes the
    // segment directly from the coordinate (ln E - ln E_0) / step; a point
    // within rounding of a knot may take the neighbouring segment, whose
    // log-log line meets this one at the knot
    if (n >= 2) {
        const double step = (s.lnE[n - 1] - s.lnE[0]) / static_cast<double>(n - 1);
        bool even = step > 0.0;
        for (size_t k = 1; k < n && even; ++k)
            even = std::fabs((s.lnE[k] - s.lnE[k - 1]) - step) <= 1.0e-5 * step;
        s.uniform = even ? 1 : 0;
        s.lx0 = static_cast<float>(s.lnE[0]);
        s.inv_dlx = static_cast<float>(1.0 / step);
        s.inv_step = 1.0 / step;
    }
    for (size_t k = 1; k < n; ++k) {
        s.seg[4 * k + 0] = static_cast<float>(s.lnE[k - 1]);
        s.seg[4 * k + 1] = static_cast<float>(1.0 / (s.lnE[k] - s.lnE[k - 1]));
        s.seg[4 * k + 2] = static_cast<float>(s.s_cm2[k - 1] / s.sigma_scale);
        s.seg[4 * k + 3] = static_cast<float>((s.lnS[k] - s.lnS[k - 1]) * kLog2E);   // base-2 slope
    }
}

int build_cam_into(const hadros_params& p, const SigmaHost& sig, DevCam& cam, DevBin* bins, int cap,
                   int* n_bins_out, const char** err)
{
    std::memset(&cam, 0, sizeof(cam));
    const double a = p.a_spin;
    cam.a = a;
    cam.r_obs = p.r_obs_rg;
    cam.th_obs = p.theta_obs_rad;
    const double fov_rad = p.fov_deg * kPi / 180.0;   // deg_to_rad, kerr_camera.cpp:11-14
    cam.tan_half = std::tan(0.5 * fov_rad);
    cam.r_max = p.r_max_rg;
    cam.h0 = p.h;
    cam.h_min = p.h * 1.0e-5;                         // kerr_geodesic.cpp:237
    cam.tol = p.tolerance;
    cam.r_stop = (1.0 + std::sqrt(1.0 - a * a)) + 1.0e-3;   // kerr_camera.cpp:211-220
    {
        const double s = std::sin(p.theta_obs_rad), c = std::cos(p.theta_obs_rad);
        M5 g;
        bl_metric(a, p.r_obs_rg, s, c, g);
        cam.g_tt = g.tt;
        cam.g_tph = g.tph;
        cam.g_rr = g.rr;
        cam.g_thth = g.thth;
        cam.g_phph = g.phph;
        cam.sq_grr = std::sqrt(g.rr);
        cam.sq_gthth = std::sqrt(g.thth);
        cam.sq_gphph = std::sqrt(g.phph);
        cam.alpha_obs = bl_lapse(a, p.r_obs_rg, s, c);
        cam.omega_obs = bl_omega(a, p.r_obs_rg, s);
        cam.pt_contra = 1.0 / cam.alpha_obs;
    }
    {   // kerr_geodesic.cpp:241-308 stage coefficients at h = h0
        const double h = p.h;
        const double c[15] = {h * 1.0 / 4.0,
                              h * 3.0 / 32.0, h * 9.0 / 32.0,
                              h * 1932.0 / 2197.0, h * -7200.0 / 2197.0, h * 7296.0 / 2197.0,
                              h * 439.0 / 216.0, h * -8.0, h * 3680.0 / 513.0, h * -845.0 / 4104.0,
                              h * -8.0 / 27.0, h * 2.0, h * -3544.0 / 2565.0, h * 1859.0 / 4104.0,
                              h * -11.0 / 40.0};
        for (int k = 0; k < 15; ++k) cam.c0[k] = c[k];
    }
    {   // radiative_transfer.cpp:485-503
        const double a_bh = sclamp(a, 0.0, 0.999999);
        const double r_h = 1.0 + std::sqrt(1.0 - a_bh * a_bh);
        cam.rt_skip = r_h + 1.0e-3;
    }
    cam.rg_cm = kGcgs * p.M_bh_msun * kMsunG / (kCcgs * kCcgs);   // constants.hpp:17-20
    cam.torus = resolve_torus(p);
    {
        Source& s = cam.src;
        s.kind = p.source_kind;
        s.spectral_kind = p.spectral_kind;
        s.r_center = p.src_r_center_rg;
        s.sigma_r = p.src_sigma_r_rg;
        s.theta_width = p.src_theta_width_rad;
        s.powerlaw = p.src_powerlaw;
        s.emax = p.src_emax_GeV;
        s.norm = p.src_norm;
        s.funnel_theta = p.src_funnel_theta_rad;
        s.q = p.src_density_power_q;
        s.s = p.src_radial_power_s;
        s.cutoff_lo = p.src_cutoff_min;
        s.cutoff_hi = p.src_cutoff_max;
        s.grad_dr = p.src_gradient_dr_rg;
        s.grad_dtheta = p.src_gradient_dtheta_rad;
        s.gamma = p.spec_gamma;
        s.ecut = p.spec_ecut_GeV;
        // radiative_transfer.cpp:255-264 (density_weighted), :297-298 (shock)
        if (p.source_kind == HADROS_SOURCE_DENSITY_WEIGHTED && p.src_rho_ref_gcm3 > 0.0)
            s.rho_norm = smax(p.src_rho_ref_gcm3, 1.0e-300);
        else
            s.rho_norm = smax(torus_rho(cam.torus, p.src_r_center_rg, 0.5 * kPi), 1.0e-300);
    }
    fill_mixed_constants(cam, sig.sigma_scale);
    cam.nx = p.nx;
    cam.ny = p.ny;
    cam.max_steps = p.max_steps;
    cam.mono = (p.spectral_kind == HADROS_SPECTRAL_MONOCHROMATIC) ? 1 : 0;

    // spectral bins, radiative_transfer.cpp:711-737
    const double sEmin = sig.E.front(), sEmax = sig.E.back();
    int nb = 0;
    auto ratio_consts = [&](DevBin& b) {
        if (cam.mono) {
            b.gamma = static_cast<float>(p.src_powerlaw);
            b.kcut = p.src_emax_GeV > 0.0 ? static_cast<float>(b.E_mid / p.src_emax_GeV) : 0.0f;
        } else {
            b.gamma = static_cast<float>(p.spec_gamma);
            b.kcut = (p.spectral_kind == HADROS_SPECTRAL_POWERLAW_CUTOFF && p.spec_ecut_GeV > 0.0)
                         ? static_cast<float>(b.E_mid / p.spec_ecut_GeV) : 0.0f;
        }
        b.w0 = spectral_weight(cam.src, b.E_mid);
        b.lnE = static_cast<float>(std::log(b.E_mid));
        b.gg_lo = gg_lower(b.E_mid, sEmax);
        b.gg_hi = gg_upper(b.E_mid, sEmin);
        b.kcut2 = static_cast<float>(static_cast<double>(b.kcut) * kLog2E);
        b.qbase = sig.uniform ? static_cast<float>((std::log(b.E_mid) - sig.lnE.front()) * sig.inv_step) : 0.0f;
    };
    if (cam.mono) {
        DevBin b{};
        b.E_mid = p.Enu_obs_GeV;
        b.dE = 1.0;
        b.w = 1.0;
        b.valid = 1;
        if (!(b.E_mid > 0.0) || !std::isfinite(b.E_mid)) {
            *err = "Enu_obs_GeV must be positive and finite";
            return HADROS_E_ARG;
        }
        ratio_consts(b);
        if (nb < cap) bins[nb] = b;
        ++nb;
    } else {
        const int n_bins = std::max(p.n_bins, 1);
        if (n_bins > cap) {
            *err = "n_bins exceeds the bin capacity of this entry point";
            return HADROS_E_ARG;
        }
        const double e_min = smax(p.spec_e_min_GeV, sEmin);
        const double e_max = smin(p.spec_e_max_GeV, sEmax);
        const bool ok = !(e_min <= 0.0 || e_max <= e_min);
        const double log_min = ok ? std::log(e_min) : 0.0;
        const double log_max = ok ? std::log(e_max) : 0.0;
        const double dlog = (log_max - log_min) / static_cast<double>(n_bins);
        for (int i = 0; i < n_bins; ++i) {
            DevBin b{};
            if (ok) {
                const double log_left = log_min + dlog * static_cast<double>(i);
                const double log_right = log_left + dlog;
                b.E_mid = std::exp(0.5 * (log_left + log_right));
                b.dE = std::exp(log_right) - std::exp(log_left);
                b.w = spectral_weight(cam.src, b.E_mid) * b.dE;
                b.valid = (b.w <= 0.0 || !std::isfinite(b.w)) ? 0 : 1;
                ratio_consts(b);
            } else {
                // empty band: the reference computes no bin (RTResult{} defaults)
                b.E_mid = 0.0;
                b.valid = 0;
                b.w0 = 0.0;
                b.gg_lo = std::numeric_limits<double>::infinity();
                b.gg_hi = -std::numeric_limits<double>::infinity();
            }
            bins[nb++] = b;
        }
    }
    if (nb > cap) {
        *err = "n_bins exceeds the bin capacity of this entry point";
        return HADROS_E_ARG;
    }
    cam.n_bins = nb;
    cam.sp_gamma = cam.mono ? static_cast<float>(p.src_powerlaw) : static_cast<float>(p.spec_gamma);
    cam.sp_emit = 0;
    for (int k = 0; k < nb; ++k) cam.sp_emit |= bins[k].E_mid > 0.0 ? 1 : 0;
    // MeV channel: the spectral aggregate keeps the first valid bin's MeV
    // result (radiative_transfer.cpp:741-774), none without a valid bin
    bool have_ref = false;
    for (int k = 0; k < nb; ++k) have_ref = have_ref || bins[k].valid != 0;
    cam.mev = make_mev(p, cam.torus, have_ref);
    cam.bin_offset = 0;
    *n_bins_out = nb;
    return HADROS_OK;
}

int build_cam(const hadros_params& p, const SigmaHost& sig, DevCam& cam,
              std::vector<DevBin>& bins, std::string& err)
{
    DevBin bb[kMaxBins];
    int nb = 0;
    const char* e = "";
    const int rc = build_cam_into(p, sig, cam, bb, kMaxBins, &nb, &e);
    if (rc) {
        err = (nb > kMaxBins || p.n_bins > kMaxBins) ? "n_bins exceeds 256" : e;
        return rc;
    }
    cam.bin_offset = static_cast<int32_t>(bins.size());
    bins.insert(bins.end(), bb, bb + nb);
    return HADROS_OK;
}

size_t trace_smem_bytes(int precision, int sig_n, int max_bins)
{
    return smem_layout(precision, sig_n, max_bins).total;
}

int launch_trace(const TraceArgs& args, int precision, int n_sm, void* stream, std::string& err)
{
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (args.fast_geodesic) return launch_trace_fast(args, precision, n_sm, stream, err);
    return launch_variant<0>(args, precision, n_sm, st, err);
}

int prepare_trace(const TraceArgs& args, int precision, int fast, int n_sm, int blocks_per_sm, LaunchCfg& cfg,
                  std::string& err)
{
    if (fast) return prepare_trace_fast(args, precision, n_sm, blocks_per_sm, cfg, err);
    return prepare_variant<0>(args, precision, n_sm, blocks_per_sm, cfg, err);
}

int launch_trace_prepared(const TraceArgs& args, int precision, int fast, const LaunchCfg& cfg, void* stream,
                          std::string& err)
{
    if (fast) return launch_trace_prepared_fast(args, precision, cfg, stream, err);
    return launch_prepared_variant<0>(args, precision, cfg, static_cast<cudaStream_t>(stream), err);
}

int launch_path_transfer(const TraceArgs& args, int precision, int n_sm, void* stream, std::string& err)
{
    // the same translation unit (FMA or not) as the matching trace kernel
    if (args.fast_geodesic) return launch_path_transfer_fast(args, precision, n_sm, stream, err);
    return launch_paths<0>(args, precision, n_sm, static_cast<cudaStream_t>(stream), err);
}

}  // namespace hadros
