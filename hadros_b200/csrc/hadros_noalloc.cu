// hadros_noalloc.cu — hadros_image_device_noalloc(): the trace kernel for
// callers that cannot allocate GPU memory.
//
// Who needs it: code that links this library into a process whose device
// memory is owned by someone else — a framework with its own caching
// allocator (a cudaMalloc/cudaFree behind its back fragments the pool and can
// synchronize the device), a service that reserves a fixed memory budget per
// tenant and forbids further allocation, or a host thread that must not block
// on the allocator.  Such callers already own their input and output buffers;
// what the ordinary entry points add on top is a context with device scratch
// (the work cursor and counters, the camera and bin tables, the sigma table).
// Here that scratch is one file-scope __device__ array instead.
//
// The array (kNoAllocScratchBytes, about 60 KB) is part of the library image:
// every GPU that loads the library holds it until the process exits.  Limits:
// at most 1024 sigma-table rows and 64 spectral bins per call; larger
// requests are rejected with HADROS_E_ARG before anything runs.  All calls
// share the one array and each leaves its contents behind; the work counters
// are cleared at the start of every call.  Two calls whose work overlaps on
// the GPU (different streams, or different host threads on one device) race
// on the array and corrupt each other's results: serialize them.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address with cudaGetSymbolAddress and keeps it (the array's
// name in host code is only a host-side stand-in, not a device address).
// Make that first call outside any stream capture.
//
// No cudaMalloc, cudaFree or other allocating routine is called: the plan is
// built in fixed-size local arrays and copied into the array with
// cudaMemcpyAsync; the only heap use is the text of an error message when a
// call fails.  The call waits on the caller's stream before returning, so it
// can report HADROS_E_TIMEOUT.
#include <cstring>
#include <limits>
#include <mutex>

#include "hadros_trace_kernel.cuh"

namespace hadros {
namespace {

constexpr int kNoAllocMaxSigma = 1024;
constexpr int kNoAllocMaxBins = 64;
constexpr int kNoAllocMaxDevices = 64;

constexpr size_t al256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffCounters = 0;
constexpr size_t kOffCam = 256;
constexpr size_t kOffBins = al256(kOffCam + sizeof(DevCam));
constexpr size_t kOffE = al256(kOffBins + sizeof(DevBin) * kNoAllocMaxBins);
constexpr size_t kOffS = al256(kOffE + 8 * kNoAllocMaxSigma);
constexpr size_t kOffLnE = al256(kOffS + 8 * kNoAllocMaxSigma);
constexpr size_t kOffLnS = al256(kOffLnE + 8 * kNoAllocMaxSigma);
constexpr size_t kOffLx = al256(kOffLnS + 8 * kNoAllocMaxSigma);
constexpr size_t kOffSeg = al256(kOffLx + 4 * kNoAllocMaxSigma);
constexpr size_t kNoAllocScratchBytes = al256(kOffSeg + 16 * kNoAllocMaxSigma);

// The scratch of every no-alloc call (see the file comment).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_addr_mu;
unsigned char* g_addr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up once.
int32_t scratch_address(int dev, unsigned char** out)
{
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return set_error(HADROS_E_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                                                cudaGetErrorString(e));
        g_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_addr[dev];
    return HADROS_OK;
}

// Per-camera constants and bins into fixed arrays: the same values as
// build_cam in hadros_trace.cu, without containers.
Torus na_resolve_torus(const hadros_params& p)
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

double na_gg_upper(double E, double lo)
{
    double x = E / lo;
    for (int it = 0; it < 64 && E / x >= lo; ++it) x = std::nextafter(x, std::numeric_limits<double>::infinity());
    for (int it = 0; it < 64 && !(E / x >= lo); ++it) x = std::nextafter(x, 0.0);
    return x;
}
double na_gg_lower(double E, double hi)
{
    double x = E / hi;
    for (int it = 0; it < 64 && E / x <= hi; ++it) x = std::nextafter(x, 0.0);
    for (int it = 0; it < 64 && !(E / x <= hi); ++it) x = std::nextafter(x, std::numeric_limits<double>::infinity());
    return x;
}

int na_build_cam(const hadros_params& p, const SigmaHost& sig, DevCam& cam, DevBin* bins,
                 int cap, int* n_bins, const char** err)
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
    cam.torus = na_resolve_torus(p);
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
        b.gg_lo = na_gg_lower(b.E_mid, sEmax);
        b.gg_hi = na_gg_upper(b.E_mid, sEmin);
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
        bins[nb++] = b;
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
            if (nb < cap) bins[nb] = b;
            ++nb;
        }
    }
    if (nb > cap) {
        *err = "n_bins exceeds the no-alloc maximum of 64 spectral bins";
        return HADROS_E_ARG;
    }
    cam.n_bins = nb;
    bool have_ref = false;   // MeV result of the first valid bin (radiative_transfer.cpp:741-774)
    for (int k = 0; k < nb; ++k) have_ref = have_ref || bins[k].valid != 0;
    cam.mev = make_mev(p, cam.torus, have_ref);
    cam.bin_offset = 0;
    *n_bins = nb;
    return HADROS_OK;
}

}  // namespace
}  // namespace hadros

using namespace hadros;

extern "C" int32_t hadros_image_device_noalloc(const hadros_params* p, const hadros_sigma* s,
                                               const hadros_image_out* dev_out, void* stream)
{
    if (!p || !s || !dev_out) return set_error(HADROS_E_ARG, "NULL argument");
    int32_t rc = hadros_params_validate(p);
    if (rc) return rc;
    if (p->fast_geodesic)
        return set_error(HADROS_E_ARG, "the no-alloc entry point runs the reference-arithmetic kernel only "
                                       "(fast_geodesic must be 0)");
    const int n_sig = static_cast<int>(s->h.E.size());
    if (n_sig > kNoAllocMaxSigma)
        return set_error(HADROS_E_ARG, "sigma table has more rows than the no-alloc maximum of 1024");
    const int want_bins = p->spectral_kind == HADROS_SPECTRAL_MONOCHROMATIC ? 1 : std::max(p->n_bins, 1);
    if (want_bins > kNoAllocMaxBins)
        return set_error(HADROS_E_ARG, "n_bins exceeds the no-alloc maximum of 64 spectral bins");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices)
        return set_error(HADROS_E_CUDA, "no usable current CUDA device");
    int n_sm = 0;
    e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return set_error(HADROS_E_CUDA, cudaGetErrorString(e));

    DevCam cam;
    DevBin bins[kNoAllocMaxBins];
    int nb = 0;
    const char* perr = "";
    rc = na_build_cam(*p, s->h, cam, bins, kNoAllocMaxBins, &nb, &perr);
    if (rc) return set_error(rc, perr);
    const int64_t P = static_cast<int64_t>(p->nx) * p->ny;
    cam.item_begin = 0;
    cam.item_end = P;
    cam.out_offset = 0;
    cam.binout_offset = 0;

    unsigned char* base = nullptr;
    if ((rc = scratch_address(dev, &base))) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const SigmaHost& h = s->h;
    struct Up { size_t off; const void* src; size_t n; } ups[] = {
        {kOffCam, &cam, sizeof(DevCam)}, {kOffBins, bins, sizeof(DevBin) * nb},
        {kOffE, h.E.data(), 8u * n_sig}, {kOffS, h.s_cm2.data(), 8u * n_sig},
        {kOffLnE, h.lnE.data(), 8u * n_sig}, {kOffLnS, h.lnS.data(), 8u * n_sig},
        {kOffLx, h.lx.data(), 4u * n_sig}, {kOffSeg, h.seg.data(), 16u * n_sig}};
    for (const Up& u : ups) {
        e = cudaMemcpyAsync(base + u.off, u.src, u.n, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return set_error(HADROS_E_CUDA, std::string("upload: ") + cudaGetErrorString(e));
    }
    e = cudaMemsetAsync(base + kOffCounters, 0, 4 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return set_error(HADROS_E_CUDA, std::string("counter reset: ") + cudaGetErrorString(e));

    TraceArgs A{};
    A.cams = reinterpret_cast<const DevCam*>(base + kOffCam);
    A.n_cams = 1;
    A.max_bins = nb;
    A.total_items = P;
    A.pixel_ids = nullptr;
    A.bins = reinterpret_cast<const DevBin*>(base + kOffBins);
    A.sig.n = n_sig;
    A.sig.E_min = h.E.front();
    A.sig.E_max = h.E.back();
    A.sig.sigma_scale = h.sigma_scale;
    A.sig.uniform = h.uniform;
    A.sig.lx0 = h.lx0;
    A.sig.inv_dlx = h.inv_dlx;
    A.sig.E = reinterpret_cast<const double*>(base + kOffE);
    A.sig.S = reinterpret_cast<const double*>(base + kOffS);
    A.sig.lnE = reinterpret_cast<const double*>(base + kOffLnE);
    A.sig.lnS = reinterpret_cast<const double*>(base + kOffLnS);
    A.sig.lx = reinterpret_cast<const float*>(base + kOffLx);
    A.sig.seg = reinterpret_cast<const float*>(base + kOffSeg);
    A.tau = dev_out->tau;
    A.P_surv = dev_out->P_surv;
    A.I_obs = dev_out->I_obs;
    A.fate = dev_out->fate;
    A.steps = dev_out->steps;
    A.attempts = dev_out->attempts;
    A.tau_E = dev_out->tau_E;
    A.I_E = static_cast<double*>(dev_out->I_E);
    A.tau_mev = dev_out->tau_mev;
    A.P_surv_mev = dev_out->P_surv_mev;
    A.I_obs_mev = dev_out->I_obs_mev;
    A.r_nu = dev_out->r_nu;
    A.leakage = dev_out->leakage;
    A.mev = p->mev_channel ? 1 : 0;
    A.counters = reinterpret_cast<unsigned long long*>(base + kOffCounters);
    A.attempt_budget = static_cast<int64_t>(p->max_steps) * 51 + 1;
    A.fast_geodesic = 0;
    if (P > 0) {
        std::string lerr;
        rc = launch_variant<0>(A, p->precision, n_sm, st, lerr);
        if (rc) return set_error(rc, lerr);
    }
    unsigned long long c[4] = {0, 0, 0, 0};
    e = cudaMemcpyAsync(c, base + kOffCounters, sizeof(c), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_error(HADROS_E_CUDA, std::string("trace kernel: ") + cudaGetErrorString(e));
    if (c[3] > 0) return set_error(HADROS_E_TIMEOUT, "rays exceeded the attempt budget");
    return set_error(HADROS_OK, "");
}
