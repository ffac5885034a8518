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
    for (size_t k = 1; k < n; ++k) {
        s.seg[4 * k + 0] = static_cast<float>(s.lnE[k - 1]);
        s.seg[4 * k + 1] = static_cast<float>(1.0 / (s.lnE[k] - s.lnE[k - 1]));
        s.seg[4 * k + 2] = static_cast<float>(s.s_cm2[k - 1] / s.sigma_scale);
        s.seg[4 * k + 3] = static_cast<float>(s.lnS[k] - s.lnS[k - 1]);
    }
}

int build_cam(const hadros_params& p, const SigmaHost& sig, DevCam& cam,
              std::vector<DevBin>& bins, std::string& err)
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
    cam.nx = p.nx;
    cam.ny = p.ny;
    cam.max_steps = p.max_steps;
    cam.mono = (p.spectral_kind == HADROS_SPECTRAL_MONOCHROMATIC) ? 1 : 0;

    // spectral bins, radiative_transfer.cpp:711-737
    const double sEmin = sig.E.front(), sEmax = sig.E.back();
    std::vector<DevBin> bb;
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
    };
    if (cam.mono) {
        DevBin b{};
        b.E_mid = p.Enu_obs_GeV;
        b.dE = 1.0;
        b.w = 1.0;
        b.valid = 1;
        if (!(b.E_mid > 0.0) || !std::isfinite(b.E_mid)) {
            err = "Enu_obs_GeV must be positive and finite";
            return HADROS_E_ARG;
        }
        ratio_consts(b);
        bb.push_back(b);
    } else {
        const int n_bins = std::max(p.n_bins, 1);
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
            bb.push_back(b);
        }
    }
    cam.n_bins = static_cast<int32_t>(bb.size());
    if (cam.n_bins > kMaxBins) {
        err = "n_bins exceeds 256";
        return HADROS_E_ARG;
    }
    cam.bin_offset = static_cast<int32_t>(bins.size());
    bins.insert(bins.end(), bb.begin(), bb.end());
    return HADROS_OK;
}

// ===================== device ===============================================

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

// KerrGeodesic::rhs (kerr_geodesic.cpp:83-135) with sin/cos of theta given.
// The reference evaluates g^{-1}(r +- eps) and g^{-1}(theta +- eps) once per
// (mu, nu) pair; they are evaluated once here (identical values).
__device__ __forceinline__ void geo_rhs(double a, double r, double th, double s, double c,
                                        double pr, double pth, double pt, double pph, K5& d)
{
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
        double sp, cp, sm, cm;
        sincos(th + eps, &sp, &cp);
        sincos(th - eps, &sm, &cm);
        M5 gp, gm;
        bl_ginv(a, r, sp, cp, gp);
        bl_ginv(a, r, sm, cm, gm);
        const double den = 2.0 * eps;
        d.pth = fd_force((gp.tt - gm.tt) / den, (gp.tph - gm.tph) / den, (gp.rr - gm.rr) / den,
                         (gp.thth - gm.thth) / den, (gp.phph - gm.phph) / den, pt, pr, pth, pph);
    }
}

__device__ __forceinline__ void geo_rhs_at(double a, double r, double th, double pr, double pth,
                                           double pt, double pph, K5& d)
{
    double s, c;
    sincos(th, &s, &c);
    geo_rhs(a, r, th, s, c, pr, pth, pt, pph, d);
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

__device__ __forceinline__ void kahan_add(float& s, float& c, float x)
{
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
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
    o += (precision == HADROS_PRECISION_MIXED ? 5 * sizeof(float) : 2 * sizeof(double)) *
         size_t(kTPB) * size_t(max_bins);
    L.total = o;
    return L;
}

enum Phase : int { kNeedRay = 0, kStepStart = 1, kAttempt = 2, kDone = 3 };

template <int MIXED>
__global__ void __launch_bounds__(kTPB) trace_kernel(const TraceArgs A)
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
    const double sigEmin = A.sig.E_min, sigEmax = A.sig.E_max;
    const double sig_scale = A.sig.sigma_scale;

    const int tid = threadIdx.x;
    // per-bin accumulators of this thread's ray, column tid, stride kTPB
    double* accT64 = reinterpret_cast<double*>(smem + L.off_acc) + tid;
    double* accI64 = accT64 + size_t(kTPB) * A.max_bins;
    float* accT = reinterpret_cast<float*>(smem + L.off_acc) + tid;
    float* accTc = accT + size_t(kTPB) * A.max_bins;
    float* accI = accTc + size_t(kTPB) * A.max_bins;
    float* accIc = accI + size_t(kTPB) * A.max_bins;
    float* accS = accIc + size_t(kTPB) * A.max_bins;

    int phase = kNeedRay;
    // ray state
    const DevCam* cam = nullptr;
    const DevBin* bins = nullptr;
    long long item = 0, local = 0;
    int B = 1, step = 0, att_in_step = 0;
    long long att_total = 0;
    double a = 0.0, r = 0.0, th = 0.0, ph = 0.0, pr = 0.0, pth = 0.0, pt = 0.0, pph = 0.0;
    double r_prev = 0.0, th_prev = 0.0, ph_prev = 0.0, E_obs = 1.0, h = 0.0;
    K5 k1{};
    int fate = HADROS_FATE_TRUNCATED;

    while (true) {
        while (phase == kNeedRay || phase == kStepStart) {
            if (phase == kNeedRay) {
                item = static_cast<long long>(atomicAdd(&A.counters[0], 1ULL));
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
                const long long pid = A.pixel_ids ? static_cast<long long>(A.pixel_ids[local]) : local;
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
                for (int b = 0; b < B; ++b) {
                    if (MIXED) {
                        accT[b * kTPB] = 0.0f; accTc[b * kTPB] = 0.0f;
                        accI[b * kTPB] = 0.0f; accIc[b * kTPB] = 0.0f;
                        accS[b * kTPB] = 0.0f;
                    } else {
                        accT64[b * kTPB] = 0.0; accI64[b * kTPB] = 0.0;
                    }
                }
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
                // ---- finish the pixel: aggregates and stores --------------
                const long long orow = cam->out_offset + local;
                double t_out = 0.0, p_out = 1.0, i_out = 0.0;
                double wsum = 0.0, tsum = 0.0, psum = 0.0, isum = 0.0;
                for (int b = 0; b < B; ++b) {
                    double tb, ib;
                    if (MIXED) {
                        tb = static_cast<double>(accT[b * kTPB]);
                        // I = (I_s - c) * exp(-S) * w(E_mid)
                        ib = (static_cast<double>(accI[b * kTPB]) - static_cast<double>(accIc[b * kTPB])) *
                             exp(-static_cast<double>(accS[b * kTPB])) * bins[b].w0;
                    } else {
                        tb = accT64[b * kTPB];
                        ib = accI64[b * kTPB];
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
                atomicAdd(&A.counters[1], static_cast<unsigned long long>(step));
                atomicAdd(&A.counters[2], static_cast<unsigned long long>(att_total));
                phase = kNeedRay;
                continue;
            }

            double s, c;
            sincos(th, &s, &c);
            // PathPoint (kerr_camera.cpp:245-273): ZAMO interval and redshift
            double dl = 0.0;
            if (step != 0) {
                const double r_mid = 0.5 * (r + r_prev);
                const double th_mid = 0.5 * (th + th_prev);
                double sm, cm;
                sincos(th_mid, &sm, &cm);
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
            const double z = (-(pt + omega * pph) / alpha) / smax(E_obs, 1.0e-300);

            // ---- transfer of this point into every bin ------------------
            if (!(r < cam->rt_skip)) {   // radiative_transfer.cpp:501-505
                const double g = 1.0 / smax(z, 1.0e-300);
                const double gg = smax(g, 1.0e-300);
                const double dl_cm = dl * cam->rg_cm;
                const double rho = torus_rho(cam->torus, r, th);
                const double C = emissivity_factor(cam->src, cam->torus, r, th, rho);
                const double g3 = pow(g, 3.0);
                if (MIXED) {
                    // FP32 transfer.  Each bin's intensity is kept as a Kahan sum
                    // I_s scaled by exp(S): every contribution K w(E_loc)/w(E_mid)
                    // exp(-tau) enters as exp(e) with e = ln(...) - tau + S, and S is
                    // re-anchored when the sum is empty or a term would exceed e^40,
                    // so intensities behind optically thick gas (exp(-tau) far below
                    // FP32's range) keep their relative precision.
                    const double zp = 1.0 / gg;   // E_local / E_mid
                    const float lnzp = static_cast<float>(log(zp));
                    const float zm1 = static_cast<float>(zp - 1.0);
                    const double Kd = g3 * C * dl_cm;
                    const bool emit = Kd > 0.0;
                    const float lnK = emit ? static_cast<float>(log(Kd)) : 0.0f;
                    const bool have_tau = !(rho <= 0.0);
                    const float nbdl = static_cast<float>((rho / kMuG) * dl_cm * sig_scale);
                    for (int b = 0; b < B; ++b) {
                        const DevBin& bn = bins[b];
                        float T = accT[b * kTPB], Tc = accTc[b * kTPB];
                        if (emit && bn.E_mid > 0.0) {
                            float I = accI[b * kTPB], Ic = accIc[b * kTPB], S = accS[b * kTPB];
                            const float arg = lnK - bn.gamma * lnzp - bn.kcut * zm1;
                            // ln of this contribution; below -800 it is under FP64's
                            // range (the reference adds an exact or subnormal zero)
                            const double x = static_cast<double>(arg) -
                                             (static_cast<double>(T) - static_cast<double>(Tc));
                            if (x >= -800.0) {
                                double e = x + static_cast<double>(S);
                                if (I == 0.0f || e > 40.0) {
                                    const float shrink = (I == 0.0f) ? 0.0f : __expf(static_cast<float>(-e));
                                    I *= shrink;
                                    Ic *= shrink;
                                    S = static_cast<float>(-x);   // |S| < ~900: exact to 1e-4
                                    e = x + static_cast<double>(S);
                                }
                                kahan_add(I, Ic, __expf(static_cast<float>(e)));
                                accI[b * kTPB] = I; accIc[b * kTPB] = Ic; accS[b * kTPB] = S;
                            }
                        }
                        if (have_tau && gg >= bn.gg_lo && gg <= bn.gg_hi) {
                            const float lnE = bn.lnE + lnzp;
                            int lo = 0, cnt = n_sig;   // lower_bound over lx
                            while (cnt > 0) {
                                const int st = cnt >> 1;
                                if (slx[lo + st] < lnE) { lo += st + 1; cnt -= st + 1; }
                                else cnt = st;
                            }
                            const int k = lo < 1 ? 1 : (lo > n_sig - 1 ? n_sig - 1 : lo);
                            const float4 sg = sseg[k];
                            const float t = (lnE - sg.x) * sg.y;
                            kahan_add(T, Tc, nbdl * (sg.z * __expf(t * sg.w)));
                            accT[b * kTPB] = T; accTc[b * kTPB] = Tc;
                        }
                    }
                } else {
                    for (int b = 0; b < B; ++b) {
                        const double E_loc = bins[b].E_mid / gg;
                        double jj = 0.0;
                        if (!(E_loc <= 0.0)) jj = C * spectral_weight(cam->src, E_loc);
                        double T = accT64[b * kTPB];
                        accI64[b * kTPB] += g3 * jj * exp(-T) * dl_cm;
                        if (rho <= 0.0 || E_loc < sigEmin || E_loc > sigEmax) continue;
                        // SigmaTable::log_interp (sigma_table.cpp:81-124)
                        int lo = 0, cnt = n_sig;
                        while (cnt > 0) {
                            const int st = cnt >> 1;
                            if (sE[lo + st] < E_loc) { lo += st + 1; cnt -= st + 1; }
                            else cnt = st;
                        }
                        double sigma_cm2;
                        if (lo == 0) sigma_cm2 = sS[0];
                        else if (lo == n_sig) sigma_cm2 = sS[n_sig - 1];
                        else {
                            const double lx = log(E_loc);
                            const double lx1 = slnE[lo - 1], lx2 = slnE[lo];
                            const double ly1 = slnS[lo - 1], ly2 = slnS[lo];
                            const double t = (lx - lx1) / (lx2 - lx1);
                            sigma_cm2 = exp(ly1 + t * (ly2 - ly1));
                        }
                        const double nb = rho / kMuG;
                        T += nb * sigma_cm2 * dl_cm;
                        accT64[b * kTPB] = T;
                    }
                }
            }

            // ---- k1 of the coming step_adaptive (shares sin/cos) ------------
            geo_rhs(a, r, th, s, c, pr, pth, pt, pph, k1);
            r_prev = r;
            th_prev = th;
            ph_prev = ph;
            h = cam->h0;
            att_in_step = 0;
            phase = kAttempt;
        }

        if (__all_sync(0xffffffffu, phase == kDone)) break;
        if (phase != kAttempt) continue;

        // ---- one RKF45 attempt (kerr_geodesic.cpp:239-326) -----------------
        double cf[15];
        if (att_in_step == 0) {
#pragma unroll
            for (int q = 0; q < 15; ++q) cf[q] = cam->c0[q];
        } else {
            cf[0] = h * 1.0 / 4.0;
            cf[1] = h * 3.0 / 32.0; cf[2] = h * 9.0 / 32.0;
            cf[3] = h * 1932.0 / 2197.0; cf[4] = h * -7200.0 / 2197.0; cf[5] = h * 7296.0 / 2197.0;
            cf[6] = h * 439.0 / 216.0; cf[7] = h * -8.0; cf[8] = h * 3680.0 / 513.0;
            cf[9] = h * -845.0 / 4104.0;
            cf[10] = h * -8.0 / 27.0; cf[11] = h * 2.0; cf[12] = h * -3544.0 / 2565.0;
            cf[13] = h * 1859.0 / 4104.0; cf[14] = h * -11.0 / 40.0;
        }
        K5 k2, k3, k4, k5, k6;
        geo_rhs_at(a, r + cf[0] * k1.r, th + cf[0] * k1.th, pr + cf[0] * k1.pr,
                   pth + cf[0] * k1.pth, pt, pph, k2);
        geo_rhs_at(a, r + cf[1] * k1.r + cf[2] * k2.r, th + cf[1] * k1.th + cf[2] * k2.th,
                   pr + cf[1] * k1.pr + cf[2] * k2.pr, pth + cf[1] * k1.pth + cf[2] * k2.pth,
                   pt, pph, k3);
        geo_rhs_at(a, r + cf[3] * k1.r + cf[4] * k2.r + cf[5] * k3.r,
                   th + cf[3] * k1.th + cf[4] * k2.th + cf[5] * k3.th,
                   pr + cf[3] * k1.pr + cf[4] * k2.pr + cf[5] * k3.pr,
                   pth + cf[3] * k1.pth + cf[4] * k2.pth + cf[5] * k3.pth, pt, pph, k4);
        geo_rhs_at(a, r + cf[6] * k1.r + cf[7] * k2.r + cf[8] * k3.r + cf[9] * k4.r,
                   th + cf[6] * k1.th + cf[7] * k2.th + cf[8] * k3.th + cf[9] * k4.th,
                   pr + cf[6] * k1.pr + cf[7] * k2.pr + cf[8] * k3.pr + cf[9] * k4.pr,
                   pth + cf[6] * k1.pth + cf[7] * k2.pth + cf[8] * k3.pth + cf[9] * k4.pth,
                   pt, pph, k5);
        geo_rhs_at(a,
                   r + cf[10] * k1.r + cf[11] * k2.r + cf[12] * k3.r + cf[13] * k4.r + cf[14] * k5.r,
                   th + cf[10] * k1.th + cf[11] * k2.th + cf[12] * k3.th + cf[13] * k4.th + cf[14] * k5.th,
                   pr + cf[10] * k1.pr + cf[11] * k2.pr + cf[12] * k3.pr + cf[13] * k4.pr + cf[14] * k5.pr,
                   pth + cf[10] * k1.pth + cf[11] * k2.pth + cf[12] * k3.pth + cf[13] * k4.pth + cf[14] * k5.pth,
                   pt, pph, k6);
#define HAD_Y4(f) (A1 * k1.f + A3 * k3.f + A4 * k4.f - A5 * k5.f)
#define HAD_Y5(f) (B1 * k1.f + B3 * k3.f + B4 * k4.f - B5 * k5.f + B6 * k6.f)
        const double y4r = r + h * HAD_Y4(r), y5r = r + h * HAD_Y5(r);
        const double y4t = th + h * HAD_Y4(th), y5t = th + h * HAD_Y5(th);
        const double y4p = ph + h * HAD_Y4(ph), y5p = ph + h * HAD_Y5(ph);
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
            const double factor = 0.8 * pow(cam->tol / smax(err, 1.0e-30), 0.25);
            h *= sclamp(factor, 0.1, 5.0);
            if (h < h_min) h = h_min;
            ++att_in_step;
            if (att_in_step == 50) {   // step_rk4 with h0 (kerr_geodesic.cpp:137-192, :328)
                const double h0 = cam->h0;
                K5 q2, q3, q4;
                geo_rhs_at(a, r + 0.5 * h0 * k1.r, th + 0.5 * h0 * k1.th, pr + 0.5 * h0 * k1.pr,
                           pth + 0.5 * h0 * k1.pth, pt, pph, q2);
                geo_rhs_at(a, r + 0.5 * h0 * q2.r, th + 0.5 * h0 * q2.th, pr + 0.5 * h0 * q2.pr,
                           pth + 0.5 * h0 * q2.pth, pt, pph, q3);
                geo_rhs_at(a, r + h0 * q3.r, th + h0 * q3.th, pr + h0 * q3.pr, pth + h0 * q3.pth,
                           pt, pph, q4);
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

}  // namespace

size_t trace_smem_bytes(int precision, int sig_n, int max_bins)
{
    return smem_layout(precision, sig_n, max_bins).total;
}

int launch_trace(const TraceArgs& args, int precision, int n_sm, void* stream, std::string& err)
{
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t smem = trace_smem_bytes(precision, args.sig.n, args.max_bins);
    cudaError_t e;
    int per_sm = 0;
    if (precision == HADROS_PRECISION_MIXED) {
        e = cudaFuncSetAttribute(trace_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_kernel<1>, kTPB, smem);
    } else {
        e = cudaFuncSetAttribute(trace_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_kernel<0>, kTPB, smem);
    }
    if (e != cudaSuccess) {
        err = std::string("trace kernel setup: ") + cudaGetErrorString(e);
        return HADROS_E_CUDA;
    }
    if (per_sm < 1) {
        err = "trace kernel does not fit on an SM (shared memory for sigma table and bins)";
        return HADROS_E_ARG;
    }
    long long grid = static_cast<long long>(n_sm) * per_sm;
    const long long needed = (args.total_items + kTPB - 1) / kTPB;
    if (grid > needed) grid = needed > 0 ? needed : 1;
    if (precision == HADROS_PRECISION_MIXED)
        trace_kernel<1><<<static_cast<unsigned>(grid), kTPB, smem, st>>>(args);
    else
        trace_kernel<0><<<static_cast<unsigned>(grid), kTPB, smem, st>>>(args);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("trace kernel launch: ") + cudaGetErrorString(e);
        return HADROS_E_CUDA;
    }
    return HADROS_OK;
}

}  // namespace hadros
