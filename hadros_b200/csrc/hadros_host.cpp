// hadros_host.cpp — the C ABI (include/hadros_b200.h): parameters, model
// names, sigma tables, device contexts and the image calls.
//
// No function lets a C++ exception or a CUDA error escape: every entry point
// returns a status code and leaves a message for hadros_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

#include "hadros_internal.h"

using namespace hadros;

namespace {

thread_local std::string g_last_error;

int32_t fail(int32_t code, const std::string& msg)
{
    g_last_error = msg;
    return code;
}

int32_t ok()
{
    g_last_error.clear();
    return HADROS_OK;
}

const char* const kProfileNames[8] = {"gaussian", "powerlaw", "gaussian_funnel", "powerlaw_funnel",
                                      "gaussian_envelope", "powerlaw_envelope",
                                      "powerlaw_funnel_envelope", "collapsar_ndaf_like"};
const char* const kSourceNames[5] = {"inner_ring", "funnel_wall", "jet_base", "shock_layer",
                                     "density_weighted"};
const char* const kSpectralNames[3] = {"monochromatic", "powerlaw", "powerlaw_cutoff"};

// One MeV name table: the accepted spellings of each kind and the
// reference's error text (src/mev_neutrino_physics.cpp:37-238).
int32_t parse_names(const char* name, int32_t* kind, std::initializer_list<std::initializer_list<const char*>> kinds,
                    const char* what, const char* choices)
{
    if (!name || !kind) return fail(HADROS_E_ARG, "NULL argument");
    const std::string n(name);
    int32_t k = 0;
    for (const auto& names : kinds) {
        for (const char* a : names)
            if (n == a) {
                *kind = k;
                return ok();
            }
        ++k;
    }
    return fail(HADROS_E_ARG, std::string("Unknown ") + what + " '" + n + "'. Use " + choices + ".");
}
const char* const kMevModelNames[2] = {"toy", "physical"};
const char* const kMevFlavorNames[3] = {"nu_e", "anti_nu_e", "nu_x"};
const char* const kMevThermalNames[5] = {"constant", "inner_hot_torus", "radial_powerlaw",
                                         "torus_plus_cool_envelope", "collapsar_inner_hot"};
const char* const kMevYeNames[5] = {"constant", "neutron_rich_torus", "funnel_proton_rich",
                                    "torus_envelope_contrast", "collapsar_neutron_rich"};
const char* const kMevSpectralNames[2] = {"monochromatic", "fermi_dirac_band"};

std::atomic<uint64_t> g_sigma_serial{1};

}  // namespace

int32_t hadros::set_error(int32_t code, const std::string& msg) { return fail(code, msg); }

// A device context: one stream, device buffers grown on demand, the sigma
// table last uploaded, and the statistics of the last call.
struct hadros_ctx {
    int device = 0;
    int n_sm = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t attempt_budget = 0;
    hadros_stats stats{};
    std::string err;
    bool failed = false;

    // device buffers
    void* d_cams = nullptr; size_t cams_cap = 0;
    void* d_bins = nullptr; size_t bins_cap = 0;
    void* d_pix = nullptr; size_t pix_cap = 0;
    void* d_out = nullptr; size_t out_cap = 0;
    unsigned long long* d_counters = nullptr;
    void* d_sig = nullptr; size_t sig_cap = 0;
    void* d_rec = nullptr; size_t rec_cap = 0;   // deferred-transfer slots
    int32_t transfer_mode = HADROS_TRANSFER_AUTO;
    const hadros_sigma* sig_key = nullptr;
    uint64_t sig_serial = 0;
    SigmaDev sig_dev{};
};

namespace {

// Deferred transfer (mixed precision): the trace kernel buffers each ray's
// path points and replays them warp-wide into the bins every kRecDepth
// iterations, so the per-bin accumulators leave shared memory and the
// occupancy no longer falls with the bin count.  Auto picks it from
// kDeferMinBins bins (measured crossover between 16 and 32 bins).
bool want_defer(int32_t mode, int precision, int max_bins)
{
    if (precision != HADROS_PRECISION_MIXED) return false;
    if (mode == HADROS_TRANSFER_DEFERRED) return true;
    if (mode == HADROS_TRANSFER_IN_LOOP) return false;
    return max_bins >= kDeferMinBins;
}

// Slots for every thread of the largest persistent grid (8 blocks per SM).
int64_t defer_slots(int n_sm) { return static_cast<int64_t>(n_sm) * 8 * kTPB; }

void set_defer(TraceArgs& A, void* base, int64_t slots, int bmax)
{
    A.rec_buf = static_cast<PointRec*>(base);
    A.rec_state = reinterpret_cast<float*>(static_cast<unsigned char*>(base) +
                                           static_cast<size_t>(slots) * kRecDepth * sizeof(PointRec));
    A.rec_bmax = bmax;
    A.rec_slots = slots;
}

int32_t cuda_fail(hadros_ctx* ctx, cudaError_t e, const char* what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (ctx) {
        ctx->err = m;
        if (e != cudaErrorMemoryAllocation) ctx->failed = true;
    }
    return fail(e == cudaErrorMemoryAllocation ? HADROS_E_NOMEM : HADROS_E_CUDA, m);
}

int32_t grow(hadros_ctx* ctx, void** buf, size_t* cap, size_t need, const char* what)
{
    if (need <= *cap && *buf) return HADROS_OK;
    if (*buf) {
        cudaFree(*buf);
        *buf = nullptr;
        *cap = 0;
    }
    size_t n = need < 256 ? 256 : need;
    cudaError_t e = cudaMalloc(buf, n);
    if (e != cudaSuccess) {
        *buf = nullptr;
        return cuda_fail(ctx, e, what);
    }
    *cap = n;
    return HADROS_OK;
}

bool finite_all(std::initializer_list<double> v)
{
    for (double x : v)
        if (!std::isfinite(x)) return false;
    return true;
}

// Device copy of a sigma table: E, S, lnE, lnS (double), lx (float), seg
// (float4), each 256-byte aligned.
int32_t upload_sigma(hadros_ctx* ctx, const hadros_sigma* s, uint64_t serial)
{
    if (ctx->sig_key == s && ctx->sig_serial == serial && ctx->d_sig) return HADROS_OK;
    const SigmaHost& h = s->h;
    const size_t n = h.E.size();
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t oE = 0, oS = al(oE + 8 * n), olnE = al(oS + 8 * n), olnS = al(olnE + 8 * n),
                 olx = al(olnS + 8 * n), oseg = al(olx + 4 * n), total = al(oseg + 16 * n);
    int32_t rc = grow(ctx, &ctx->d_sig, &ctx->sig_cap, total, "sigma table allocation");
    if (rc) return rc;
    std::vector<unsigned char> blob(total, 0);
    std::memcpy(blob.data() + oE, h.E.data(), 8 * n);
    std::memcpy(blob.data() + oS, h.s_cm2.data(), 8 * n);
    std::memcpy(blob.data() + olnE, h.lnE.data(), 8 * n);
    std::memcpy(blob.data() + olnS, h.lnS.data(), 8 * n);
    std::memcpy(blob.data() + olx, h.lx.data(), 4 * n);
    std::memcpy(blob.data() + oseg, h.seg.data(), 16 * n);
    cudaError_t e = cudaMemcpy(ctx->d_sig, blob.data(), total, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "sigma table upload");
    unsigned char* base = static_cast<unsigned char*>(ctx->d_sig);
    SigmaDev& d = ctx->sig_dev;
    d.n = static_cast<int32_t>(n);
    d.E_min = h.E.front();
    d.E_max = h.E.back();
    d.sigma_scale = h.sigma_scale;
    d.uniform = h.uniform;
    d.lx0 = h.lx0;
    d.inv_dlx = h.inv_dlx;
    d.E = reinterpret_cast<const double*>(base + oE);
    d.S = reinterpret_cast<const double*>(base + oS);
    d.lnE = reinterpret_cast<const double*>(base + olnE);
    d.lnS = reinterpret_cast<const double*>(base + olnS);
    d.lx = reinterpret_cast<const float*>(base + olx);
    d.seg = reinterpret_cast<const float*>(base + oseg);
    ctx->sig_key = s;
    ctx->sig_serial = serial;
    return HADROS_OK;
}

// Every array of hadros_image_out with its element size and extent: P rows
// per pixel, or PB per-bin elements (tau_E in the transfer's precision).
template <class F>
void each_output(size_t fsz, F&& f)
{
    f(&hadros_image_out::tau, size_t(8), false);
    f(&hadros_image_out::P_surv, size_t(8), false);
    f(&hadros_image_out::I_obs, size_t(8), false);
    f(&hadros_image_out::steps, size_t(4), false);
    f(&hadros_image_out::attempts, size_t(4), false);
    f(&hadros_image_out::fate, size_t(1), false);
    f(&hadros_image_out::tau_E, fsz, true);
    f(&hadros_image_out::I_E, size_t(8), true);
    f(&hadros_image_out::tau_mev, size_t(8), false);
    f(&hadros_image_out::P_surv_mev, size_t(8), false);
    f(&hadros_image_out::I_obs_mev, size_t(8), false);
    f(&hadros_image_out::r_nu, size_t(8), false);
    f(&hadros_image_out::leakage, size_t(8), false);
}

// Device staging of a call with host outputs: one 256-byte aligned slice of
// ctx->d_out per requested array, after `head` bytes the caller keeps.
struct Staged {
    hadros_image_out d{};
    struct Cp { void* h; const void* d; size_t n; };
    std::vector<Cp> copies;
    unsigned char* base = nullptr;
};

int32_t stage_outputs(hadros_ctx* ctx, const hadros_image_out* out, int64_t P, int64_t PB, size_t fsz, size_t head,
                      Staged& st)
{
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    std::vector<size_t> offs;
    size_t o = al(head);
    each_output(fsz, [&](auto m, size_t esz, bool per_bin) {
        offs.push_back(o);
        if (out->*m) o = al(o + esz * static_cast<size_t>(per_bin ? PB : P));
    });
    const int32_t rc = grow(ctx, &ctx->d_out, &ctx->out_cap, o, "output buffers");
    if (rc) return rc;
    st.base = static_cast<unsigned char*>(ctx->d_out);
    st.copies.clear();
    size_t k = 0;
    each_output(fsz, [&](auto m, size_t esz, bool per_bin) {
        using T = std::remove_reference_t<decltype(st.d.*m)>;
        const size_t off = offs[k++];
        if (!(out->*m)) {
            st.d.*m = nullptr;
            return;
        }
        st.d.*m = static_cast<T>(static_cast<void*>(st.base + off));
        st.copies.push_back({static_cast<void*>(out->*m), static_cast<const void*>(st.d.*m),
                             esz * static_cast<size_t>(per_bin ? PB : P)});
    });
    return HADROS_OK;
}

// Enqueue the device-to-host copies of a staged call; adds their bytes to *d2h.
int32_t download_outputs(hadros_ctx* ctx, const Staged& st, cudaStream_t stream, int64_t* d2h)
{
    for (const Staged::Cp& c : st.copies) {
        if (c.n == 0) continue;
        *d2h += static_cast<int64_t>(c.n);
        const cudaError_t e = cudaMemcpyAsync(c.h, c.d, c.n, cudaMemcpyDeviceToHost, stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "output download");
    }
    return HADROS_OK;
}

// Output pointers of a launch (DEVICE pointers).
void set_outputs(TraceArgs& A, const hadros_image_out& d)
{
    A.tau = d.tau;
    A.P_surv = d.P_surv;
    A.I_obs = d.I_obs;
    A.fate = d.fate;
    A.steps = d.steps;
    A.attempts = d.attempts;
    A.tau_E = d.tau_E;
    A.I_E = static_cast<double*>(d.I_E);
    A.tau_mev = d.tau_mev;
    A.P_surv_mev = d.P_surv_mev;
    A.I_obs_mev = d.I_obs_mev;
    A.r_nu = d.r_nu;
    A.leakage = d.leakage;
}

bool any_mev(const hadros_params* cams, int32_t n)
{
    for (int32_t c = 0; c < n; ++c)
        if (cams[c].mev_channel) return true;
    return false;
}

}  // namespace

namespace {
uint64_t sigma_serial(const hadros_sigma* s) { return s->serial; }
}  // namespace

extern "C" {

int32_t hadros_abi_version(void) { return HADROS_ABI_VERSION; }

const char* hadros_status_string(int32_t status)
{
    switch (status) {
    case HADROS_OK: return "ok";
    case HADROS_E_ARG: return "invalid argument";
    case HADROS_E_IO: return "i/o error";
    case HADROS_E_CUDA: return "CUDA error";
    case HADROS_E_RANGE: return "energy outside sigma table range";
    case HADROS_E_TIMEOUT: return "attempt budget exhausted";
    case HADROS_E_NOMEM: return "out of memory";
    case HADROS_E_STATE: return "invalid handle or state";
    default: return "unknown status";
    }
}

const char* hadros_last_error(void) { return g_last_error.c_str(); }

void hadros_params_default(hadros_params* p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->struct_size = sizeof(hadros_params);
    // KerrCamera arguments of compute_kerr_geodesics (apps/compute_kerr_geodesics.cpp:26-34)
    p->a_spin = 0.9;
    p->r_obs_rg = 60.0;
    p->theta_obs_rad = M_PI * 74.0 / 180.0;
    p->fov_deg = 45.0;
    p->nx = 100;
    p->ny = 100;
    p->r_max_rg = 120.0;
    p->h = 0.001;
    p->tolerance = 1.0e-6;   // include/kerr_geodesic.hpp:12
    p->max_steps = 200000;   // src/kerr_camera.cpp:222
    // compute_kerr_image_from_cache argv defaults (apps/compute_kerr_image_from_cache.cpp:33-55)
    p->Enu_obs_GeV = 1.0e9;
    p->M_bh_msun = 3.0;
    p->rho0_gcm3 = 1.0e10;
    p->r0_rg = 10.0;
    p->sigma_r_rg = 5.0;
    p->H_over_R = 0.01;
    p->profile_kind = HADROS_PROFILE_GAUSSIAN;
    p->radial_power = 2.0;
    p->funnel_depletion = 0.0;
    p->funnel_theta_rad = 15.0 * M_PI / 180.0;
    p->envelope_rho0_gcm3 = 0.0;
    p->envelope_alpha = 2.5;
    p->torus_r_min_rg = 4.0;
    p->torus_r_max_rg = 60.0;
    p->rho_floor_gcm3 = 1.0e-99;
    // UHESourceParams defaults (include/radiative_transfer.hpp:45-62)
    p->source_kind = HADROS_SOURCE_INNER_RING;
    p->src_r_center_rg = 3.5;
    p->src_sigma_r_rg = 1.0;
    p->src_theta_width_rad = 8.0 * 3.141592653589793238462643383279502884 / 180.0;
    p->src_powerlaw = 2.0;
    p->src_emax_GeV = 1.0e12;
    p->src_norm = 1.0;
    p->src_funnel_theta_rad = 20.0 * 3.141592653589793238462643383279502884 / 180.0;
    p->src_density_power_q = 1.0;
    p->src_radial_power_s = 2.0;
    p->src_rho_ref_gcm3 = -1.0;
    p->src_cutoff_min = 0.0;
    p->src_cutoff_max = 1.0e2;
    p->src_gradient_dr_rg = 0.1;
    p->src_gradient_dtheta_rad = 1.0 * 3.141592653589793238462643383279502884 / 180.0;
    // UHESpectralParams defaults (include/radiative_transfer.hpp:29-35)
    p->spectral_kind = HADROS_SPECTRAL_MONOCHROMATIC;
    p->spec_gamma = 2.0;
    p->spec_ecut_GeV = 1.0e12;
    p->spec_e_min_GeV = 1.0e5;
    p->spec_e_max_GeV = 1.0e12;
    p->n_bins = 8;
    p->precision = HADROS_PRECISION_FP64;
    p->fast_geodesic = 1;
    // MeVThermalParams defaults (include/radiative_transfer.hpp:64-101); the
    // channel itself is off until mev_channel is set
    p->mev_channel = 0;
    p->mev_model = HADROS_MEV_PHYSICAL;
    p->mev_flavor = HADROS_MEV_ANTI_NU_E;
    p->mev_thermal_profile = HADROS_MEV_T_INNER_HOT_TORUS;
    p->mev_ye_profile = HADROS_MEV_YE_NEUTRON_RICH_TORUS;
    p->mev_spectral_mode = HADROS_MEV_MONOCHROMATIC;
    p->mev_n_bins = 8;
    p->mev_flags = HADROS_MEV_FLAGS_DEFAULT;
    p->mev_Enu_obs_MeV = 10.0;
    p->mev_norm = 1.0;
    p->mev_sigma_abs0_cm2 = 9.6e-44;
    p->mev_sigma_scat0_cm2 = 1.7e-44;
    p->mev_neutrinosphere_tau = 2.0 / 3.0;
    p->mev_T0_MeV = 6.0;
    p->mev_T_floor_MeV = 0.1;
    p->mev_T_power = 0.2;
    p->mev_Ye_torus = 0.25;
    p->mev_Ye_funnel = 0.55;
    p->mev_Ye_envelope = 0.45;
    p->mev_Ye_floor = 0.01;
    p->mev_Ye_ceil = 0.60;
    p->mev_E_min_MeV = 3.0;
    p->mev_E_max_MeV = 50.0;
}

int32_t hadros_params_validate(const hadros_params* p)
{
    if (!p) return fail(HADROS_E_ARG, "params is NULL");
    if (p->struct_size != sizeof(hadros_params))
        return fail(HADROS_E_ARG, "params.struct_size does not match this library (use hadros_params_default)");
    if (p->nx <= 0 || p->ny <= 0)
        return fail(HADROS_E_ARG, "nx and ny must be positive");
    if (static_cast<int64_t>(p->nx) * p->ny > 2147483647LL)
        return fail(HADROS_E_ARG, "nx*ny exceeds 2^31-1 pixels");
    if (p->max_steps <= 0) return fail(HADROS_E_ARG, "max_steps must be positive");
    if (p->profile_kind < 0 || p->profile_kind > 7) return fail(HADROS_E_ARG, "profile_kind out of range");
    if (p->source_kind < 0 || p->source_kind > 4) return fail(HADROS_E_ARG, "source_kind out of range");
    if (p->spectral_kind < 0 || p->spectral_kind > 2) return fail(HADROS_E_ARG, "spectral_kind out of range");
    if (p->fast_geodesic != 0 && p->fast_geodesic != 1)
        return fail(HADROS_E_ARG, "fast_geodesic must be 0 or 1");
    if (p->precision != HADROS_PRECISION_FP64 && p->precision != HADROS_PRECISION_MIXED)
        return fail(HADROS_E_ARG, "precision must be HADROS_PRECISION_FP64 or HADROS_PRECISION_MIXED");
    if (p->spectral_kind != HADROS_SPECTRAL_MONOCHROMATIC && (p->n_bins > kMaxBins))
        return fail(HADROS_E_ARG, "n_bins must be <= 256");
    if (!(p->h > 0.0) || !std::isfinite(p->h)) return fail(HADROS_E_ARG, "step h must be positive and finite");
    if (!(p->tolerance > 0.0) || !std::isfinite(p->tolerance))
        return fail(HADROS_E_ARG, "tolerance must be positive and finite");
    if (!finite_all({p->a_spin, p->r_obs_rg, p->theta_obs_rad, p->fov_deg, p->r_max_rg,
                     p->Enu_obs_GeV, p->M_bh_msun}))
        return fail(HADROS_E_ARG, "camera parameters must be finite");
    if (p->mev_channel != 0 && p->mev_channel != 1) return fail(HADROS_E_ARG, "mev_channel must be 0 or 1");
    if (p->mev_channel) {
        if (p->mev_model < 0 || p->mev_model > 1) return fail(HADROS_E_ARG, "mev_model out of range");
        if (p->mev_flavor < 0 || p->mev_flavor > 2) return fail(HADROS_E_ARG, "mev_flavor out of range");
        if (p->mev_thermal_profile < 0 || p->mev_thermal_profile > 4)
            return fail(HADROS_E_ARG, "mev_thermal_profile out of range");
        if (p->mev_ye_profile < 0 || p->mev_ye_profile > 4) return fail(HADROS_E_ARG, "mev_ye_profile out of range");
        if (p->mev_spectral_mode < 0 || p->mev_spectral_mode > 1)
            return fail(HADROS_E_ARG, "mev_spectral_mode out of range");
        if (p->mev_spectral_mode == HADROS_MEV_FERMI_DIRAC_BAND && p->mev_n_bins > 4096)
            return fail(HADROS_E_ARG, "mev_n_bins must be <= 4096");
        if (!finite_all({p->mev_Enu_obs_MeV, p->mev_norm, p->mev_sigma_abs0_cm2, p->mev_sigma_scat0_cm2,
                         p->mev_neutrinosphere_tau, p->mev_T0_MeV, p->mev_T_floor_MeV, p->mev_T_power,
                         p->mev_Ye_torus, p->mev_Ye_funnel, p->mev_Ye_envelope, p->mev_Ye_floor, p->mev_Ye_ceil,
                         p->mev_E_min_MeV, p->mev_E_max_MeV}))
            return fail(HADROS_E_ARG, "MeV channel parameters must be finite");
    }
    return ok();
}

int32_t hadros_parse_profile(const char* name, int32_t* kind)
{   // src/torus_profile.cpp:44-91
    if (!name || !kind) return fail(HADROS_E_ARG, "NULL argument");
    const std::string n(name);
    int32_t k = -1;
    if (n == "gaussian" || n == "torus" || n == "gaussian_torus") k = 0;
    else if (n == "powerlaw" || n == "powerlaw_disk") k = 1;
    else if (n == "funnel" || n == "gaussian_funnel") k = 2;
    else if (n == "powerlaw_funnel") k = 3;
    else if (n == "gaussian_envelope") k = 4;
    else if (n == "powerlaw_envelope") k = 5;
    else if (n == "powerlaw_funnel_envelope") k = 6;
    else if (n == "collapsar_ndaf_like" || n == "collapsar_ndaf") k = 7;
    if (k < 0)
        return fail(HADROS_E_ARG,
                    "Unknown density profile '" + n +
                        "'. Use gaussian, powerlaw, gaussian_funnel, powerlaw_funnel, "
                        "gaussian_envelope, powerlaw_envelope, powerlaw_funnel_envelope, "
                        "or collapsar_ndaf_like.");
    *kind = k;
    return ok();
}

int32_t hadros_parse_source(const char* name, int32_t* kind)
{   // src/radiative_transfer.cpp:80-112
    if (!name || !kind) return fail(HADROS_E_ARG, "NULL argument");
    const std::string n(name);
    int32_t k = -1;
    if (n == "inner_ring" || n == "INNER_RING" || n == "ring") k = 0;
    else if (n == "funnel_wall" || n == "FUNNEL_WALL") k = 1;
    else if (n == "jet_base" || n == "JET_BASE") k = 2;
    else if (n == "shock_layer" || n == "SHOCK_LAYER") k = 3;
    else if (n == "density_weighted" || n == "DENSITY_WEIGHTED") k = 4;
    if (k < 0)
        return fail(HADROS_E_ARG, "Unknown UHE source model '" + n +
                                      "'. Use inner_ring, funnel_wall, jet_base, shock_layer, or density_weighted.");
    *kind = k;
    return ok();
}

int32_t hadros_parse_spectral(const char* name, int32_t* kind)
{   // src/radiative_transfer.cpp:132-156
    if (!name || !kind) return fail(HADROS_E_ARG, "NULL argument");
    const std::string n(name);
    int32_t k = -1;
    if (n == "monochromatic" || n == "MONOCHROMATIC" || n == "mono") k = 0;
    else if (n == "powerlaw" || n == "POWERLAW" || n == "power_law") k = 1;
    else if (n == "powerlaw_cutoff" || n == "POWERLAW_CUTOFF" || n == "power_law_cutoff") k = 2;
    if (k < 0)
        return fail(HADROS_E_ARG, "Unknown UHE spectral model '" + n +
                                      "'. Use monochromatic, powerlaw, or powerlaw_cutoff.");
    *kind = k;
    return ok();
}


int32_t hadros_parse_mev_model(const char* name, int32_t* kind)
{   // parse_mev_model, src/mev_neutrino_physics.cpp:37-51
    return parse_names(name, kind, {{"toy", "TOY"}, {"physical", "PHYSICAL", "phys"}}, "MEV_MODEL",
                       "toy or physical");
}

int32_t hadros_parse_mev_flavor(const char* name, int32_t* kind)
{   // parse_mev_flavor, :65-90
    return parse_names(name, kind,
                       {{"nu_e", "nue", "NU_E"}, {"anti_nu_e", "antinue", "anti-nu-e", "ANTI_NU_E"},
                        {"nu_x", "nux", "NU_X"}},
                       "MEV_FLAVOR", "nu_e, anti_nu_e, or nu_x");
}

int32_t hadros_parse_mev_thermal(const char* name, int32_t* kind)
{   // parse_mev_thermal_profile, :106-130
    return parse_names(name, kind,
                       {{"constant", "CONSTANT"}, {"inner_hot_torus", "INNER_HOT_TORUS"},
                        {"radial_powerlaw", "RADIAL_POWERLAW"},
                        {"torus_plus_cool_envelope", "TORUS_PLUS_COOL_ENVELOPE"},
                        {"collapsar_inner_hot", "COLLAPSAR_INNER_HOT"}},
                       "MEV_THERMAL_PROFILE",
                       "constant, inner_hot_torus, radial_powerlaw, torus_plus_cool_envelope, or collapsar_inner_hot");
}

int32_t hadros_parse_mev_ye(const char* name, int32_t* kind)
{   // parse_mev_ye_profile, :149-173
    return parse_names(name, kind,
                       {{"constant", "CONSTANT"}, {"neutron_rich_torus", "NEUTRON_RICH_TORUS"},
                        {"funnel_proton_rich", "FUNNEL_PROTON_RICH"},
                        {"torus_envelope_contrast", "TORUS_ENVELOPE_CONTRAST"},
                        {"collapsar_neutron_rich", "COLLAPSAR_NEUTRON_RICH"}},
                       "MEV_YE_PROFILE",
                       "constant, neutron_rich_torus, funnel_proton_rich, torus_envelope_contrast, or "
                       "collapsar_neutron_rich");
}

int32_t hadros_parse_mev_spectral(const char* name, int32_t* kind)
{   // parse_mev_spectral_mode, :192-209
    return parse_names(name, kind,
                       {{"monochromatic", "MONOCHROMATIC", "mono"}, {"fermi_dirac_band", "FERMI_DIRAC_BAND", "fd_band"}},
                       "MEV_SPECTRAL_MODE", "monochromatic or fermi_dirac_band");
}

const char* hadros_mev_model_name(int32_t k) { return (k >= 0 && k < 2) ? kMevModelNames[k] : nullptr; }
const char* hadros_mev_flavor_name(int32_t k) { return (k >= 0 && k < 3) ? kMevFlavorNames[k] : nullptr; }
const char* hadros_mev_thermal_name(int32_t k) { return (k >= 0 && k < 5) ? kMevThermalNames[k] : nullptr; }
const char* hadros_mev_ye_name(int32_t k) { return (k >= 0 && k < 5) ? kMevYeNames[k] : nullptr; }
const char* hadros_mev_spectral_name(int32_t k) { return (k >= 0 && k < 2) ? kMevSpectralNames[k] : nullptr; }

const char* hadros_profile_name(int32_t kind) { return (kind >= 0 && kind < 8) ? kProfileNames[kind] : nullptr; }
const char* hadros_source_name(int32_t kind) { return (kind >= 0 && kind < 5) ? kSourceNames[kind] : nullptr; }
const char* hadros_spectral_name(int32_t kind) { return (kind >= 0 && kind < 3) ? kSpectralNames[kind] : nullptr; }

// ---- sigma tables --------------------------------------------------------

static int32_t sigma_finish(std::vector<double>& E, std::vector<double>& g2, std::vector<double>& cm2,
                            hadros_sigma** out)
{   // src/sigma_table.cpp:38-53
    if (E.size() < 2)
        return fail(HADROS_E_IO, "Sigma table must contain at least two valid data lines.");
    for (size_t i = 1; i < E.size(); ++i)
        if (E[i] <= E[i - 1])
            return fail(HADROS_E_IO, "Energy grid in sigma table must be strictly increasing.");
    if (E.size() > static_cast<size_t>(kMaxSigma))
        return fail(HADROS_E_ARG, "sigma table has more than 4096 rows");
    hadros_sigma* box = new (std::nothrow) hadros_sigma();
    if (!box) return fail(HADROS_E_NOMEM, "out of host memory");
    box->serial = g_sigma_serial.fetch_add(1);
    box->h.E.swap(E);
    box->h.s_GeV2.swap(g2);
    box->h.s_cm2.swap(cm2);
    prepare_sigma(box->h);
    *out = box;
    return ok();
}

int32_t hadros_sigma_load(const char* path, hadros_sigma** out)
{   // SigmaTable::SigmaTable (src/sigma_table.cpp:9-53)
    if (!path || !out) return fail(HADROS_E_ARG, "NULL argument");
    *out = nullptr;
    std::ifstream in(path);
    if (!in) return fail(HADROS_E_IO, std::string("Could not open sigma table: ") + path);
    std::vector<double> E, g2, cm2;
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty()) continue;
        if (line[0] == '#') continue;
        std::istringstream iss(line);
        double e, sg, sc;
        if (!(iss >> e >> sg >> sc)) continue;
        if (e <= 0.0 || sg <= 0.0 || sc <= 0.0) continue;
        E.push_back(e);
        g2.push_back(sg);
        cm2.push_back(sc);
    }
    return sigma_finish(E, g2, cm2, out);
}

int32_t hadros_sigma_from_arrays(const double* E_GeV, const double* sigma_GeV2, const double* sigma_cm2,
                                 int32_t n, hadros_sigma** out)
{
    if (!E_GeV || !sigma_cm2 || !out || n < 0) return fail(HADROS_E_ARG, "NULL argument or negative n");
    *out = nullptr;
    std::vector<double> E, g2, cm2;
    for (int32_t i = 0; i < n; ++i) {
        const double sg = sigma_GeV2 ? sigma_GeV2[i] : 1.0;
        if (E_GeV[i] <= 0.0 || sg <= 0.0 || sigma_cm2[i] <= 0.0) continue;
        E.push_back(E_GeV[i]);
        g2.push_back(sigma_GeV2 ? sg : 0.0);
        cm2.push_back(sigma_cm2[i]);
    }
    return sigma_finish(E, g2, cm2, out);
}

int32_t hadros_sigma_info(const hadros_sigma* s, int32_t* n, double* E_min, double* E_max)
{
    if (!s) return fail(HADROS_E_STATE, "sigma handle is NULL");
    if (n) *n = static_cast<int32_t>(s->h.E.size());
    if (E_min) *E_min = s->h.E.front();
    if (E_max) *E_max = s->h.E.back();
    return ok();
}

int32_t hadros_sigma_eval_cm2(const hadros_sigma* s, double x, double* out)
{   // SigmaTable::log_interp (src/sigma_table.cpp:81-124)
    if (!s || !out) return fail(HADROS_E_ARG, "NULL argument");
    const auto& xs = s->h.E;
    const auto& ys = s->h.s_cm2;
    if (x <= 0.0) return fail(HADROS_E_RANGE, "Interpolation energy must be positive.");
    if (x < xs.front() || x > xs.back()) return fail(HADROS_E_RANGE, "Requested energy outside sigma table range.");
    auto it = std::lower_bound(xs.begin(), xs.end(), x);
    if (it == xs.begin()) { *out = ys.front(); return ok(); }
    if (it == xs.end()) { *out = ys.back(); return ok(); }
    const size_t i = static_cast<size_t>(it - xs.begin());
    const double lx = std::log(x), lx1 = std::log(xs[i - 1]), lx2 = std::log(xs[i]);
    const double ly1 = std::log(ys[i - 1]), ly2 = std::log(ys[i]);
    const double t = (lx - lx1) / (lx2 - lx1);
    *out = std::exp(ly1 + t * (ly2 - ly1));
    return ok();
}

void hadros_sigma_destroy(hadros_sigma* s)
{
    delete s;
}

int32_t hadros_spectral_bins(const hadros_params* p, const hadros_sigma* s, double* E_mid, double* dE,
                             double* weight, int8_t* valid, int32_t* n_bins_out)
{
    int32_t rc = hadros_params_validate(p);
    if (rc) return rc;
    if (!s) return fail(HADROS_E_STATE, "sigma handle is NULL");
    DevCam cam;
    std::vector<DevBin> bins;
    std::string err;
    rc = build_cam(*p, s->h, cam, bins, err);
    if (rc) return fail(rc, err);
    for (size_t b = 0; b < bins.size(); ++b) {
        if (E_mid) E_mid[b] = bins[b].E_mid;
        if (dE) dE[b] = bins[b].dE;
        if (weight) weight[b] = bins[b].w;
        if (valid) valid[b] = static_cast<int8_t>(bins[b].valid);
    }
    if (n_bins_out) *n_bins_out = static_cast<int32_t>(bins.size());
    return ok();
}

// ---- contexts -----------------------------------------------------------------

int32_t hadros_ctx_create(int32_t device, hadros_ctx** out)
{
    if (!out) return fail(HADROS_E_ARG, "NULL argument");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= 0) return fail(HADROS_E_CUDA, "no CUDA device available");
    if (device < 0 || device >= count) return fail(HADROS_E_ARG, "device index out of range");
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaSetDevice");
    cudaDeviceProp prop{};
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDeviceProperties");
    if (prop.major != 10 || prop.minor != 0)
        return fail(HADROS_E_CUDA, std::string("this library is built for sm_100a (B200); device is ") + prop.name);
    hadros_ctx* ctx = new (std::nothrow) hadros_ctx();
    if (!ctx) return fail(HADROS_E_NOMEM, "out of host memory");
    ctx->device = device;
    ctx->n_sm = prop.multiProcessorCount;
    if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&ctx->ev0)) != cudaSuccess || (e = cudaEventCreate(&ctx->ev1)) != cudaSuccess ||
        (e = cudaMalloc(reinterpret_cast<void**>(&ctx->d_counters), 4 * sizeof(unsigned long long))) != cudaSuccess) {
        hadros_ctx_destroy(ctx);
        return cuda_fail(nullptr, e, "context setup");
    }
    *out = ctx;
    return ok();
}

void hadros_ctx_destroy(hadros_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_cams);
    cudaFree(ctx->d_bins);
    cudaFree(ctx->d_pix);
    cudaFree(ctx->d_out);
    cudaFree(ctx->d_counters);
    cudaFree(ctx->d_sig);
    cudaFree(ctx->d_rec);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int32_t hadros_ctx_set_transfer(hadros_ctx* ctx, int32_t mode)
{
    if (!ctx) return fail(HADROS_E_STATE, "context is NULL");
    if (mode != HADROS_TRANSFER_AUTO && mode != HADROS_TRANSFER_IN_LOOP && mode != HADROS_TRANSFER_DEFERRED)
        return fail(HADROS_E_ARG, "unknown transfer mode");
    ctx->transfer_mode = mode;
    return ok();
}

int32_t hadros_ctx_stats(const hadros_ctx* ctx, hadros_stats* out)
{
    if (!ctx || !out) return fail(HADROS_E_STATE, "NULL argument");
    *out = ctx->stats;
    return ok();
}

int32_t hadros_ctx_set_attempt_budget(hadros_ctx* ctx, int64_t attempts_per_ray)
{
    if (!ctx) return fail(HADROS_E_STATE, "context is NULL");
    if (attempts_per_ray < 0) return fail(HADROS_E_ARG, "budget must be >= 0");
    ctx->attempt_budget = attempts_per_ray;
    return ok();
}

}  // extern "C"

namespace {

// Path recording requested by hadros_trace_paths for the next run_image.
struct PathRec {
    double* buf;
    int32_t cap;
};
thread_local PathRec g_path_rec{nullptr, 0};

// Shared body of the image calls.  dev_out holds DEVICE pointers.
// With pixel_ids_dev (a DEVICE list of n_pixels ids), the list is traced
// as it is, without the host range check: an id only sets the ray's screen
// position, and outputs go to list rows.
int32_t run_image(hadros_ctx* ctx, const hadros_params* p, const hadros_sigma* s,
                  const int32_t* pixel_ids_host, int32_t n_pixels, const hadros_image_out& dev_out,
                  cudaStream_t st, bool time_kernel, const int32_t* pixel_ids_dev = nullptr)
{
    if (!ctx) return fail(HADROS_E_STATE, "context is NULL");
    if (ctx->failed) return fail(HADROS_E_STATE, "context is in a failed state: " + ctx->err);
    if (!s) return fail(HADROS_E_STATE, "sigma handle is NULL");
    int32_t rc = hadros_params_validate(p);
    if (rc) return rc;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");

    DevCam cam;
    std::vector<DevBin> bins;
    std::string err;
    rc = build_cam(*p, s->h, cam, bins, err);
    if (rc) return fail(rc, err);
    const bool listed = pixel_ids_host || pixel_ids_dev;
    const int64_t P = listed ? n_pixels : static_cast<int64_t>(p->nx) * p->ny;
    if (pixel_ids_host) {
        const int64_t total = static_cast<int64_t>(p->nx) * p->ny;
        for (int32_t k = 0; k < n_pixels; ++k)
            if (pixel_ids_host[k] < 0 || pixel_ids_host[k] >= total)
                return fail(HADROS_E_ARG, "pixel id out of range");
    }
    cam.item_begin = 0;
    cam.item_end = P;
    cam.out_offset = 0;
    cam.binout_offset = 0;

    const bool sigma_new = !(ctx->sig_key == s && ctx->sig_serial == sigma_serial(s) && ctx->d_sig);
    if ((rc = upload_sigma(ctx, s, sigma_serial(s)))) return rc;
    if ((rc = grow(ctx, &ctx->d_cams, &ctx->cams_cap, sizeof(DevCam), "camera table"))) return rc;
    if ((rc = grow(ctx, &ctx->d_bins, &ctx->bins_cap, sizeof(DevBin) * bins.size(), "bin table"))) return rc;
    if ((e = cudaMemcpyAsync(ctx->d_cams, &cam, sizeof(DevCam), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(ctx, e, "camera upload");
    if ((e = cudaMemcpyAsync(ctx->d_bins, bins.data(), sizeof(DevBin) * bins.size(), cudaMemcpyHostToDevice, st)) !=
        cudaSuccess)
        return cuda_fail(ctx, e, "bin upload");
    int64_t h2d = static_cast<int64_t>(sizeof(DevCam) + sizeof(DevBin) * bins.size());
    if (sigma_new) h2d += static_cast<int64_t>(ctx->sig_cap);
    const int32_t* d_pix = pixel_ids_dev;
    if (pixel_ids_host && n_pixels > 0) {
        h2d += static_cast<int64_t>(sizeof(int32_t)) * n_pixels;
        if ((rc = grow(ctx, &ctx->d_pix, &ctx->pix_cap, sizeof(int32_t) * n_pixels, "pixel list"))) return rc;
        if ((e = cudaMemcpyAsync(ctx->d_pix, pixel_ids_host, sizeof(int32_t) * n_pixels, cudaMemcpyHostToDevice,
                                 st)) != cudaSuccess)
            return cuda_fail(ctx, e, "pixel list upload");
        d_pix = static_cast<const int32_t*>(ctx->d_pix);
    }
    if ((e = cudaMemsetAsync(ctx->d_counters, 0, 4 * sizeof(unsigned long long), st)) != cudaSuccess)
        return cuda_fail(ctx, e, "counter reset");

    TraceArgs A{};
    A.cams = static_cast<const DevCam*>(ctx->d_cams);
    A.n_cams = 1;
    A.max_bins = cam.n_bins;
    A.total_items = P;
    A.pixel_ids = d_pix;
    A.bins = static_cast<const DevBin*>(ctx->d_bins);
    A.sig = ctx->sig_dev;
    set_outputs(A, dev_out);
    A.mev = p->mev_channel ? 1 : 0;
    A.counters = ctx->d_counters;
    A.fast_geodesic = p->fast_geodesic;
    A.paths = g_path_rec.buf;
    A.path_cap = g_path_rec.cap;
    A.attempt_budget = ctx->attempt_budget > 0 ? ctx->attempt_budget
                                               : static_cast<int64_t>(p->max_steps) * 51 + 1;
    if (want_defer(ctx->transfer_mode, p->precision, cam.n_bins)) {
        const int64_t slots = defer_slots(ctx->n_sm);
        if ((rc = grow(ctx, &ctx->d_rec, &ctx->rec_cap, rec_bytes(slots, cam.n_bins), "deferred transfer buffers")))
            return rc;
        set_defer(A, ctx->d_rec, slots, cam.n_bins);
    }

    if (P > 0) {
        if (time_kernel) cudaEventRecord(ctx->ev0, st);
        rc = launch_trace(A, p->precision, ctx->n_sm, st, err);
        if (rc) {
            ctx->err = err;
            return fail(rc, err);
        }
        if (time_kernel) cudaEventRecord(ctx->ev1, st);
    }
    ctx->stats.rays = P;
    ctx->stats.launches = P > 0 ? 1 : 0;
    ctx->stats.h2d_bytes = h2d;
    ctx->stats.d2h_bytes = 0;
    return HADROS_OK;
}


// Many cameras in one persistent launch.  dev_out holds DEVICE pointers to
// the concatenated outputs (camera order).
// With `counts`, camera c traces counts[c] pixels whose ids (j*nx+i) follow
// one another in the host array `pix` (outputs in list order).
int32_t run_batch(hadros_ctx* ctx, const hadros_params* cams, int32_t n_cams, const hadros_sigma* s,
                  const hadros_image_out& dev_out, cudaStream_t st, bool time_kernel, int64_t* P_total,
                  int64_t* PB_total, const int32_t* pix = nullptr, const int32_t* counts = nullptr)
{
    if (!ctx) return fail(HADROS_E_STATE, "context is NULL");
    if (ctx->failed) return fail(HADROS_E_STATE, "context is in a failed state: " + ctx->err);
    if (!s) return fail(HADROS_E_STATE, "sigma handle is NULL");
    if (!cams || n_cams <= 0) return fail(HADROS_E_ARG, "camera list is NULL or empty");
    for (int32_t c = 0; c < n_cams; ++c) {
        int32_t rc = hadros_params_validate(&cams[c]);
        if (rc) return fail(rc, "camera " + std::to_string(c) + ": " + g_last_error);
        if (cams[c].precision != cams[0].precision || cams[c].fast_geodesic != cams[0].fast_geodesic)
            return fail(HADROS_E_ARG, "all cameras of a batch need the same precision and fast_geodesic");
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    std::vector<DevCam> dc(static_cast<size_t>(n_cams));
    std::vector<DevBin> bins;
    std::string err;
    int64_t items = 0, binout = 0;
    int32_t max_bins = 1;
    for (int32_t c = 0; c < n_cams; ++c) {
        int32_t rc = build_cam(cams[c], s->h, dc[c], bins, err);
        if (rc) return fail(rc, "camera " + std::to_string(c) + ": " + err);
        const int64_t full = static_cast<int64_t>(cams[c].nx) * cams[c].ny;
        const int64_t P = counts ? counts[c] : full;
        if (counts) {
            if (P < 0) return fail(HADROS_E_ARG, "camera " + std::to_string(c) + ": negative pixel count");
            for (int64_t k = 0; k < P; ++k)
                if (pix[items + k] < 0 || pix[items + k] >= full)
                    return fail(HADROS_E_ARG, "camera " + std::to_string(c) + ": pixel id outside the image");
        }
        dc[c].item_begin = items;
        dc[c].item_end = items + P;
        dc[c].out_offset = items;
        dc[c].binout_offset = binout;
        items += P;
        binout += P * dc[c].n_bins;
        max_bins = std::max(max_bins, dc[c].n_bins);
    }
    *P_total = items;
    *PB_total = binout;
    int32_t rc;
    const bool sigma_new = !(ctx->sig_key == s && ctx->sig_serial == sigma_serial(s) && ctx->d_sig);
    if ((rc = upload_sigma(ctx, s, sigma_serial(s)))) return rc;
    if ((rc = grow(ctx, &ctx->d_cams, &ctx->cams_cap, sizeof(DevCam) * dc.size(), "camera table"))) return rc;
    if ((rc = grow(ctx, &ctx->d_bins, &ctx->bins_cap, sizeof(DevBin) * bins.size(), "bin table"))) return rc;
    if ((e = cudaMemcpyAsync(ctx->d_cams, dc.data(), sizeof(DevCam) * dc.size(), cudaMemcpyHostToDevice, st)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(ctx->d_bins, bins.data(), sizeof(DevBin) * bins.size(), cudaMemcpyHostToDevice, st)) !=
            cudaSuccess)
        return cuda_fail(ctx, e, "camera upload");
    const int32_t* d_pix = nullptr;
    if (counts && items > 0) {
        if ((rc = grow(ctx, &ctx->d_pix, &ctx->pix_cap, sizeof(int32_t) * items, "pixel list"))) return rc;
        if ((e = cudaMemcpyAsync(ctx->d_pix, pix, sizeof(int32_t) * items, cudaMemcpyHostToDevice, st)) !=
            cudaSuccess)
            return cuda_fail(ctx, e, "pixel list upload");
        d_pix = static_cast<const int32_t*>(ctx->d_pix);
    }
    if ((e = cudaMemsetAsync(ctx->d_counters, 0, 4 * sizeof(unsigned long long), st)) != cudaSuccess)
        return cuda_fail(ctx, e, "counter reset");
    TraceArgs A{};
    A.cams = static_cast<const DevCam*>(ctx->d_cams);
    A.n_cams = n_cams;
    A.max_bins = max_bins;
    A.total_items = items;
    A.pixel_ids = d_pix;
    A.bins = static_cast<const DevBin*>(ctx->d_bins);
    A.sig = ctx->sig_dev;
    set_outputs(A, dev_out);
    A.mev = any_mev(cams, n_cams) ? 1 : 0;
    A.counters = ctx->d_counters;
    int32_t max_cap = 0;
    for (int32_t c = 0; c < n_cams; ++c) max_cap = std::max(max_cap, cams[c].max_steps);
    A.attempt_budget = ctx->attempt_budget > 0 ? ctx->attempt_budget : static_cast<int64_t>(max_cap) * 51 + 1;
    A.fast_geodesic = cams[0].fast_geodesic;
    if (want_defer(ctx->transfer_mode, cams[0].precision, max_bins)) {
        const int64_t slots = defer_slots(ctx->n_sm);
        if ((rc = grow(ctx, &ctx->d_rec, &ctx->rec_cap, rec_bytes(slots, max_bins), "deferred transfer buffers")))
            return rc;
        set_defer(A, ctx->d_rec, slots, max_bins);
    }
    if (items > 0) {
        if (time_kernel) cudaEventRecord(ctx->ev0, st);
        rc = launch_trace(A, cams[0].precision, ctx->n_sm, st, err);
        if (rc) {
            ctx->err = err;
            return fail(rc, err);
        }
        if (time_kernel) cudaEventRecord(ctx->ev1, st);
    }
    ctx->stats.rays = items;
    ctx->stats.launches = items > 0 ? 1 : 0;
    ctx->stats.h2d_bytes = static_cast<int64_t>(sizeof(DevCam) * dc.size() + sizeof(DevBin) * bins.size()) +
                           (sigma_new ? static_cast<int64_t>(ctx->sig_cap) : 0) +
                           (counts ? static_cast<int64_t>(sizeof(int32_t)) * items : 0);
    ctx->stats.d2h_bytes = 0;
    return HADROS_OK;
}

// Finish a synchronous call: wait, read counters, fill stats.
int32_t finish_sync(hadros_ctx* ctx, bool timed)
{
    unsigned long long c[4] = {0, 0, 0, 0};
    cudaError_t e = cudaMemcpyAsync(c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "trace kernel");
    ctx->stats.accepted_steps = static_cast<int64_t>(c[1]);
    ctx->stats.attempts = static_cast<int64_t>(c[2]);
    ctx->stats.aborted_rays = static_cast<int32_t>(c[3]);
    if (timed && ctx->stats.rays > 0) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) ctx->stats.kernel_ms = ms;
    }
    if (c[3] > 0)
        return fail(HADROS_E_TIMEOUT, std::to_string(c[3]) + " rays exceeded the attempt budget");
    return ok();
}

int32_t image_host(hadros_ctx* ctx, const hadros_params* p, const hadros_sigma* s, const int32_t* pix,
                   int32_t n_pix, const hadros_image_out* out)
{
    const auto t0 = std::chrono::steady_clock::now();
    if (!ctx) return fail(HADROS_E_STATE, "context is NULL");
    if (!out) return fail(HADROS_E_ARG, "output struct is NULL");
    int32_t rc = hadros_params_validate(p);
    if (rc) return rc;
    if (!s) return fail(HADROS_E_STATE, "sigma handle is NULL");
    const int64_t P = pix ? n_pix : static_cast<int64_t>(p->nx) * p->ny;
    const int64_t B = p->spectral_kind == HADROS_SPECTRAL_MONOCHROMATIC ? 1 : std::max(p->n_bins, 1);
    const size_t fsz = p->precision == HADROS_PRECISION_MIXED ? 4 : 8;
    Staged sg;
    if ((rc = stage_outputs(ctx, out, P, P * B, fsz, 0, sg))) return rc;
    rc = run_image(ctx, p, s, pix, n_pix, sg.d, ctx->stream, true);
    if (rc) return rc;
    int64_t d2h = 4 * sizeof(unsigned long long);
    if ((rc = download_outputs(ctx, sg, ctx->stream, &d2h))) return rc;
    rc = finish_sync(ctx, true);
    ctx->stats.d2h_bytes = d2h;
    ctx->stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

}  // namespace

extern "C" {

int32_t hadros_image(hadros_ctx* ctx, const hadros_params* p, const hadros_sigma* s, const hadros_image_out* out)
{
    try {
        return image_host(ctx, p, s, nullptr, 0, out);
    } catch (const std::exception& ex) {
        return fail(HADROS_E_NOMEM, ex.what());
    }
}

int32_t hadros_image_pixels(hadros_ctx* ctx, const hadros_params* p, const hadros_sigma* s,
                            const int32_t* pixel_ids, int32_t n_pixels, const hadros_image_out* out)
{
    if (!pixel_ids || n_pixels < 0) return fail(HADROS_E_ARG, "pixel list is NULL or negative length");
    try {
        return image_host(ctx, p, s, pixel_ids, n_pixels, out);
    } catch (const std::exception& ex) {
        return fail(HADROS_E_NOMEM, ex.what());
    }
}

int32_t hadros_image_device(hadros_ctx* ctx, const hadros_params* p, const hadros_sigma* s,
                            const hadros_image_out* dev_out, void* stream)
{
    if (!dev_out) return fail(HADROS_E_ARG, "output struct is NULL");
    try {
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : (ctx ? ctx->stream : nullptr);
        const int32_t rc = run_image(ctx, p, s, nullptr, 0, *dev_out, st, false);
        return rc ? rc : ok();
    } catch (const std::exception& ex) {
        return fail(HADROS_E_NOMEM, ex.what());
    }
}

int32_t hadros_image_pixels_device(hadros_ctx* ctx, const hadros_params* p, const hadros_sigma* s,
                                   const int32_t* dev_pixel_ids, int32_t n_pixels,
                                   const hadros_image_out* dev_out, void* stream)
{
    if (!dev_out) return fail(HADROS_E_ARG, "output struct is NULL");
    if (n_pixels < 0 || (n_pixels > 0 && !dev_pixel_ids))
        return fail(HADROS_E_ARG, "pixel list is NULL or negative length");
    try {
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : (ctx ? ctx->stream : nullptr);
        const int32_t rc = run_image(ctx, p, s, nullptr, n_pixels, *dev_out, st, false,
                                     n_pixels > 0 ? dev_pixel_ids : nullptr);
        return rc ? rc : ok();
    } catch (const std::exception& ex) {
        return fail(HADROS_E_NOMEM, ex.what());
    }
}

int32_t hadros_batch_device(hadros_ctx* ctx, const hadros_params* cams, int32_t n_cams, const hadros_sigma* s,
                            const hadros_image_out* dev_out, void* stream)
{
    if (!dev_out) return fail(HADROS_E_ARG, "output struct is NULL");
    try {
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : (ctx ? ctx->stream : nullptr);
        int64_t P = 0, PB = 0;
        const int32_t rc = run_batch(ctx, cams, n_cams, s, *dev_out, st, false, &P, &PB);
        return rc ? rc : ok();
    } catch (const std::exception& ex) {
        return fail(HADROS_E_NOMEM, ex.what());
    }
}

namespace {
int32_t batch_host(hadros_ctx* ctx, const hadros_params* cams, int32_t n_cams, const hadros_sigma* s,
                   const hadros_image_out* out, const int32_t* pix, const int32_t* counts)
{
    if (!ctx) return fail(HADROS_E_STATE, "context is NULL");
    if (!out || !cams || n_cams <= 0) return fail(HADROS_E_ARG, "NULL argument or empty camera list");
    try {
        const auto t0 = std::chrono::steady_clock::now();
        int64_t P = 0, PB = 0;
        for (int32_t c = 0; c < n_cams; ++c) {
            if (hadros_params_validate(&cams[c])) return fail(HADROS_E_ARG, "camera " + std::to_string(c) + ": " + g_last_error);
            const int64_t pc = counts ? std::max<int64_t>(counts[c], 0) : static_cast<int64_t>(cams[c].nx) * cams[c].ny;
            P += pc;
            PB += pc * (cams[c].spectral_kind == HADROS_SPECTRAL_MONOCHROMATIC ? 1 : std::max(cams[c].n_bins, 1));
        }
        const size_t fsz = cams[0].precision == HADROS_PRECISION_MIXED ? 4 : 8;
        Staged sg;
        int32_t rc = stage_outputs(ctx, out, P, PB, fsz, 0, sg);
        if (rc) return rc;
        int64_t P2 = 0, PB2 = 0;
        rc = run_batch(ctx, cams, n_cams, s, sg.d, ctx->stream, true, &P2, &PB2, pix, counts);
        if (rc) return rc;
        int64_t d2h = 4 * sizeof(unsigned long long);
        if ((rc = download_outputs(ctx, sg, ctx->stream, &d2h))) return rc;
        rc = finish_sync(ctx, true);
        ctx->stats.d2h_bytes = d2h;
        ctx->stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return rc;
    } catch (const std::exception& ex) {
        return fail(HADROS_E_NOMEM, ex.what());
    }
}
}  // namespace

int32_t hadros_batch(hadros_ctx* ctx, const hadros_params* cams, int32_t n_cams, const hadros_sigma* s,
                     const hadros_image_out* out)
{
    return batch_host(ctx, cams, n_cams, s, out, nullptr, nullptr);
}

int32_t hadros_batch_pixels(hadros_ctx* ctx, const hadros_params* cams, int32_t n_cams, const hadros_sigma* s,
                            const int32_t* pixel_ids, const int32_t* counts, const hadros_image_out* out)
{
    if (!pixel_ids || !counts) return fail(HADROS_E_ARG, "pixel list or counts is NULL");
    return batch_host(ctx, cams, n_cams, s, out, pixel_ids, counts);
}

int32_t hadros_trace_paths(hadros_ctx* ctx, const hadros_params* p, const int32_t* pixel_ids, int32_t n_pixels,
                           int32_t max_points, double* points, int32_t* npoints, int8_t* fate)
{
    if (!ctx) return fail(HADROS_E_STATE, "context is NULL");
    if (!points || !npoints || max_points <= 0) return fail(HADROS_E_ARG, "points/npoints NULL or max_points <= 0");
    int32_t rc = hadros_params_validate(p);
    if (rc) return rc;
    const int64_t rows = pixel_ids ? n_pixels : static_cast<int64_t>(p->nx) * p->ny;
    if (pixel_ids && n_pixels < 0) return fail(HADROS_E_ARG, "negative pixel count");
    const size_t path_bytes = static_cast<size_t>(rows) * static_cast<size_t>(max_points) * 7 * sizeof(double);
    try {
        // a path-only trace: monochromatic, no per-bin outputs
        hadros_params q = *p;
        q.spectral_kind = HADROS_SPECTRAL_MONOCHROMATIC;
        q.mev_channel = 0;
        if (!(q.Enu_obs_GeV > 0.0)) q.Enu_obs_GeV = 1.0e9;
        void* d_paths = nullptr;
        cudaError_t e = cudaSetDevice(ctx->device);
        if (e == cudaSuccess) e = cudaMalloc(&d_paths, path_bytes > 0 ? path_bytes : 8);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "path buffer allocation");
        auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
        const size_t o_st = 0, o_f = al(4 * rows), total = al(o_f + rows);
        rc = grow(ctx, &ctx->d_out, &ctx->out_cap, total, "output buffers");
        if (rc) { cudaFree(d_paths); return rc; }
        unsigned char* base = static_cast<unsigned char*>(ctx->d_out);
        hadros_image_out d{};
        d.steps = reinterpret_cast<int32_t*>(base + o_st);
        d.fate = reinterpret_cast<int8_t*>(base + o_f);
        // the geometry does not depend on sigma: a fixed two-row table
        static hadros_sigma* dummy = [] {
            hadros_sigma* t = new hadros_sigma();
            t->serial = g_sigma_serial.fetch_add(1);
            t->h.E = {1.0, 1.0e30};
            t->h.s_GeV2 = {1.0, 1.0};
            t->h.s_cm2 = {1.0e-40, 1.0e-40};
            prepare_sigma(t->h);
            return t;
        }();
        g_path_rec = {static_cast<double*>(d_paths), max_points};
        rc = run_image(ctx, &q, dummy, pixel_ids, n_pixels, d, ctx->stream, true);
        g_path_rec = {nullptr, 0};
        if (!rc) {
            e = cudaMemcpyAsync(npoints, d.steps, 4 * rows, cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess && fate) e = cudaMemcpyAsync(fate, d.fate, rows, cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(points, d_paths, path_bytes, cudaMemcpyDeviceToHost, ctx->stream);
            if (e != cudaSuccess) rc = cuda_fail(ctx, e, "path download");
            else rc = finish_sync(ctx, true);
        }
        cudaFree(d_paths);
        return rc;
    } catch (const std::exception& ex) {
        g_path_rec = {nullptr, 0};
        return fail(HADROS_E_NOMEM, ex.what());
    }
}

int32_t hadros_transfer_paths(hadros_ctx* ctx, const hadros_params* p, const hadros_sigma* s, int32_t n_rays,
                              const int32_t* npoints, const int8_t* fate, const double* points,
                              const hadros_image_out* out)
{
    if (!ctx) return fail(HADROS_E_STATE, "context is NULL");
    if (ctx->failed) return fail(HADROS_E_STATE, "context is in a failed state: " + ctx->err);
    if (!s) return fail(HADROS_E_STATE, "sigma handle is NULL");
    if (!out || !npoints || (!points && n_rays > 0) || n_rays < 0) return fail(HADROS_E_ARG, "NULL argument");
    int32_t rc = hadros_params_validate(p);
    if (rc) return rc;
    const auto t0 = std::chrono::steady_clock::now();
    try {
        std::vector<int64_t> offs(static_cast<size_t>(n_rays) + 1, 0);
        for (int32_t k = 0; k < n_rays; ++k) {
            if (npoints[k] < 0) return fail(HADROS_E_ARG, "Invalid ray with negative number of points");
            offs[k + 1] = offs[k] + npoints[k];
        }
        const int64_t n_pts = offs.back();
        DevCam cam;
        std::vector<DevBin> bins;
        std::string err;
        rc = build_cam(*p, s->h, cam, bins, err);
        if (rc) return fail(rc, err);
        cam.item_begin = 0;
        cam.item_end = n_rays;
        cam.out_offset = 0;
        cam.binout_offset = 0;
        const int64_t B = cam.n_bins;
        const size_t fsz = p->precision == HADROS_PRECISION_MIXED ? 4 : 8;
        auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
        const int64_t P = n_rays;
        size_t o = 0;
        const size_t o_pts = o; o = al(o + 56 * static_cast<size_t>(n_pts));
        const size_t o_off = o; o = al(o + 8 * offs.size());
        const size_t o_fin = o; o = al(o + P);
        Staged sg;   // the cached paths, then the outputs
        if ((rc = stage_outputs(ctx, out, P, P * B, fsz, o, sg))) return rc;
        if ((rc = upload_sigma(ctx, s, sigma_serial(s)))) return rc;
        if ((rc = grow(ctx, &ctx->d_cams, &ctx->cams_cap, sizeof(DevCam), "camera table"))) return rc;
        if ((rc = grow(ctx, &ctx->d_bins, &ctx->bins_cap, sizeof(DevBin) * bins.size(), "bin table"))) return rc;
        unsigned char* base = static_cast<unsigned char*>(ctx->d_out);
        cudaStream_t st = ctx->stream;
        cudaError_t e = cudaSetDevice(ctx->device);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->d_cams, &cam, sizeof(DevCam), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->d_bins, bins.data(), sizeof(DevBin) * bins.size(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && n_pts > 0) e = cudaMemcpyAsync(base + o_pts, points, 56 * static_cast<size_t>(n_pts), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(base + o_off, offs.data(), 8 * offs.size(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && fate) e = cudaMemcpyAsync(base + o_fin, fate, P, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_counters, 0, 4 * sizeof(unsigned long long), st);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "path upload");
        TraceArgs A{};
        A.cams = static_cast<const DevCam*>(ctx->d_cams);
        A.n_cams = 1;
        A.max_bins = cam.n_bins;
        A.total_items = P;
        A.bins = static_cast<const DevBin*>(ctx->d_bins);
        A.sig = ctx->sig_dev;
        set_outputs(A, sg.d);
        A.mev = p->mev_channel ? 1 : 0;
        A.counters = ctx->d_counters;
        A.path_offsets = reinterpret_cast<const int64_t*>(base + o_off);
        A.path_points = reinterpret_cast<const double*>(base + o_pts);
        A.path_fates = fate ? reinterpret_cast<const int8_t*>(base + o_fin) : nullptr;
        A.fast_geodesic = p->fast_geodesic;
        if (P > 0) {
            cudaEventRecord(ctx->ev0, st);
            rc = launch_path_transfer(A, p->precision, ctx->n_sm, st, err);
            if (rc) { ctx->err = err; return fail(rc, err); }
            cudaEventRecord(ctx->ev1, st);
        }
        ctx->stats.rays = P;
        ctx->stats.launches = P > 0 ? 1 : 0;
        ctx->stats.h2d_bytes = static_cast<int64_t>(56 * n_pts + 8 * offs.size() + (fate ? P : 0));
        int64_t d2h = 0;
        if ((rc = download_outputs(ctx, sg, st, &d2h))) return rc;
        rc = finish_sync(ctx, true);
        ctx->stats.d2h_bytes = d2h;
        ctx->stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return rc;
    } catch (const std::exception& ex) {
        return fail(HADROS_E_NOMEM, ex.what());
    }
}

int32_t hadros_ctx_synchronize(hadros_ctx* ctx)
{
    if (!ctx) return fail(HADROS_E_STATE, "context is NULL");
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "synchronize");
    unsigned long long c[4] = {0, 0, 0, 0};
    e = cudaMemcpy(c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "counter read");
    ctx->stats.accepted_steps = static_cast<int64_t>(c[1]);
    ctx->stats.attempts = static_cast<int64_t>(c[2]);
    ctx->stats.aborted_rays = static_cast<int32_t>(c[3]);
    if (c[3] > 0) return fail(HADROS_E_TIMEOUT, std::to_string(c[3]) + " rays exceeded the attempt budget");
    return ok();
}

}  // extern "C"

// ---- plans: uploaded scans, capturable launches ---------------------------

struct hadros_plan {
    int device = 0;
    int precision = 0, fast = 0;
    int64_t P = 0, PB = 0;
    void* d_tabs = nullptr;          // cams | bins | order | sigma
    unsigned long long* d_counters = nullptr;
    void* d_rec = nullptr;           // deferred-transfer slots (owned by the plan)
    TraceArgs A{};
    LaunchCfg cfg{};
    hadros_schedule sched{};
};

namespace {

// Per-pixel cost estimate of a camera from a coarse pre-pass (accepted
// steps on every `stride`-th pixel; nearest coarse sample elsewhere), and the
// pixel order by descending cost (ties: pixel order).
int32_t cost_order(hadros_ctx* ctx, const hadros_params& p, const hadros_sigma* s, int stride,
                   std::vector<int32_t>& order, double& total_cost)
{
    const int nx = p.nx, ny = p.ny;
    const int cx = (nx + stride - 1) / stride, cy = (ny + stride - 1) / stride;
    std::vector<int32_t> ids;
    ids.reserve(static_cast<size_t>(cx) * cy);
    for (int j = 0; j < ny; j += stride)
        for (int i = 0; i < nx; i += stride) ids.push_back(j * nx + i);
    std::vector<int32_t> steps(ids.size());
    hadros_image_out o{};
    o.steps = steps.data();
    hadros_params q = p;
    q.spectral_kind = HADROS_SPECTRAL_MONOCHROMATIC;   // geometry only
    q.mev_channel = 0;
    int32_t rc = hadros_image_pixels(ctx, &q, s, ids.data(), static_cast<int32_t>(ids.size()), &o);
    if (rc) return rc;
    std::vector<float> cost(static_cast<size_t>(nx) * ny);
    total_cost = 0.0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const int ci = std::min((i + stride / 2) / stride, cx - 1), cj = std::min((j + stride / 2) / stride, cy - 1);
            cost[static_cast<size_t>(j) * nx + i] = static_cast<float>(steps[static_cast<size_t>(cj) * cx + ci]);
            total_cost += steps[static_cast<size_t>(cj) * cx + ci];
        }
    order.resize(cost.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = static_cast<int32_t>(k);
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return cost[x] > cost[y]; });
    return HADROS_OK;
}

// Pixel order walking 8x4 tiles, so a warp's 32 rays are a compact patch.
void tile_order(const hadros_params& p, std::vector<int32_t>& order)
{
    order.clear();
    order.reserve(static_cast<size_t>(p.nx) * p.ny);
    for (int tj = 0; tj < p.ny; tj += 4)
        for (int ti = 0; ti < p.nx; ti += 8)
            for (int j = tj; j < std::min(tj + 4, p.ny); ++j)
                for (int i = ti; i < std::min(ti + 8, p.nx); ++i) order.push_back(j * p.nx + i);
}

}  // namespace

extern "C" {

void hadros_schedule_default(hadros_schedule* s)
{
    if (!s) return;
    s->blocks_per_sm = 0;
    s->order = HADROS_ORDER_ROWS;
    s->coarse_stride = 16;
    s->camera_order = 1;
}

int32_t hadros_plan_create(hadros_ctx* ctx, const hadros_params* cams, int32_t n_cams, const hadros_sigma* s,
                           const hadros_schedule* sched, hadros_plan** out)
{
    if (!ctx) return fail(HADROS_E_STATE, "context is NULL");
    if (!out || !cams || n_cams <= 0 || !s) return fail(HADROS_E_ARG, "NULL argument or empty camera list");
    *out = nullptr;
    hadros_schedule sc;
    hadros_schedule_default(&sc);
    if (sched) sc = *sched;
    if (sc.order < 0 || sc.order > 2 || sc.blocks_per_sm < 0 || sc.coarse_stride <= 0)
        return fail(HADROS_E_ARG, "bad schedule");
    try {
        for (int32_t c = 0; c < n_cams; ++c) {
            int32_t rc = hadros_params_validate(&cams[c]);
            if (rc) return fail(rc, "camera " + std::to_string(c) + ": " + g_last_error);
            if (cams[c].precision != cams[0].precision || cams[c].fast_geodesic != cams[0].fast_geodesic)
                return fail(HADROS_E_ARG, "all cameras of a batch need the same precision and fast_geodesic");
        }
        // per-camera pixel orders and costs
        std::vector<std::vector<int32_t>> orders(static_cast<size_t>(n_cams));
        std::vector<double> cost(static_cast<size_t>(n_cams), 0.0);
        for (int32_t c = 0; c < n_cams; ++c) {
            cost[c] = static_cast<double>(cams[c].nx) * cams[c].ny;
            if (sc.order == HADROS_ORDER_COST) {
                int32_t rc = cost_order(ctx, cams[c], s, sc.coarse_stride, orders[c], cost[c]);
                if (rc) return rc;
            } else if (sc.order == HADROS_ORDER_TILES) {
                tile_order(cams[c], orders[c]);
            }
        }
        // queue order of cameras: most expensive first (outputs stay in caller order)
        std::vector<int32_t> qorder(static_cast<size_t>(n_cams));
        for (int32_t c = 0; c < n_cams; ++c) qorder[c] = c;
        if (sc.camera_order)
            std::stable_sort(qorder.begin(), qorder.end(), [&](int32_t x, int32_t y) { return cost[x] > cost[y]; });
        std::vector<DevCam> dc(static_cast<size_t>(n_cams));
        std::vector<DevBin> bins;
        std::string err;
        std::vector<int64_t> out_off(static_cast<size_t>(n_cams)), bin_off(static_cast<size_t>(n_cams));
        int64_t P = 0, PB = 0;
        for (int32_t c = 0; c < n_cams; ++c) {   // output layout: caller order
            const int64_t Pc = static_cast<int64_t>(cams[c].nx) * cams[c].ny;
            const int64_t Bc = cams[c].spectral_kind == HADROS_SPECTRAL_MONOCHROMATIC ? 1 : std::max(cams[c].n_bins, 1);
            out_off[c] = P;
            bin_off[c] = PB;
            P += Pc;
            PB += Pc * Bc;
        }
        std::vector<int32_t> order_all;
        const bool use_order = sc.order != HADROS_ORDER_ROWS;
        if (use_order) order_all.reserve(static_cast<size_t>(P));
        int64_t item = 0;
        int32_t max_bins = 1, max_cap = 0;
        for (int32_t k = 0; k < n_cams; ++k) {   // queue layout: cost order
            const int32_t c = qorder[k];
            DevCam& d = dc[k];
            int32_t rc = build_cam(cams[c], s->h, d, bins, err);
            if (rc) return fail(rc, "camera " + std::to_string(c) + ": " + err);
            const int64_t Pc = static_cast<int64_t>(cams[c].nx) * cams[c].ny;
            d.item_begin = item;
            d.item_end = item + Pc;
            d.out_offset = out_off[c];
            d.binout_offset = bin_off[c];
            item += Pc;
            max_bins = std::max(max_bins, d.n_bins);
            max_cap = std::max(max_cap, cams[c].max_steps);
            if (use_order) order_all.insert(order_all.end(), orders[c].begin(), orders[c].end());
        }
        hadros_plan* pl = new hadros_plan();
        pl->device = ctx->device;
        pl->precision = cams[0].precision;
        pl->fast = cams[0].fast_geodesic;
        pl->P = P;
        pl->PB = PB;
        pl->sched = sc;
        const SigmaHost& h = s->h;
        const size_t n = h.E.size();
        auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
        size_t o = 0;
        const size_t o_cam = o; o = al(o + sizeof(DevCam) * dc.size());
        const size_t o_bin = o; o = al(o + sizeof(DevBin) * bins.size());
        const size_t o_ord = o; o = al(o + sizeof(int32_t) * order_all.size());
        const size_t oE = o; o = al(o + 8 * n);
        const size_t oS = o; o = al(o + 8 * n);
        const size_t olnE = o; o = al(o + 8 * n);
        const size_t olnS = o; o = al(o + 8 * n);
        const size_t olx = o; o = al(o + 4 * n);
        const size_t oseg = o; o = al(o + 16 * n);
        std::vector<unsigned char> blob(o, 0);
        std::memcpy(blob.data() + o_cam, dc.data(), sizeof(DevCam) * dc.size());
        std::memcpy(blob.data() + o_bin, bins.data(), sizeof(DevBin) * bins.size());
        if (use_order) std::memcpy(blob.data() + o_ord, order_all.data(), sizeof(int32_t) * order_all.size());
        std::memcpy(blob.data() + oE, h.E.data(), 8 * n);
        std::memcpy(blob.data() + oS, h.s_cm2.data(), 8 * n);
        std::memcpy(blob.data() + olnE, h.lnE.data(), 8 * n);
        std::memcpy(blob.data() + olnS, h.lnS.data(), 8 * n);
        std::memcpy(blob.data() + olx, h.lx.data(), 4 * n);
        std::memcpy(blob.data() + oseg, h.seg.data(), 16 * n);
        cudaError_t e = cudaSetDevice(ctx->device);
        if (e == cudaSuccess) e = cudaMalloc(&pl->d_tabs, o);
        if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&pl->d_counters), 4 * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMemcpy(pl->d_tabs, blob.data(), o, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            hadros_plan_destroy(pl);
            return cuda_fail(nullptr, e, "plan upload");
        }
        unsigned char* base = static_cast<unsigned char*>(pl->d_tabs);
        TraceArgs& A = pl->A;
        A.cams = reinterpret_cast<const DevCam*>(base + o_cam);
        A.n_cams = n_cams;
        A.max_bins = max_bins;
        A.total_items = P;
        A.bins = reinterpret_cast<const DevBin*>(base + o_bin);
        A.order = use_order ? reinterpret_cast<const int32_t*>(base + o_ord) : nullptr;
        A.blocks_per_sm = sc.blocks_per_sm;
        A.sig.n = static_cast<int32_t>(n);
        A.sig.uniform = h.uniform;
        A.sig.lx0 = h.lx0;
        A.sig.inv_dlx = h.inv_dlx;
        A.sig.E_min = h.E.front();
        A.sig.E_max = h.E.back();
        A.sig.sigma_scale = h.sigma_scale;
        A.sig.E = reinterpret_cast<const double*>(base + oE);
        A.sig.S = reinterpret_cast<const double*>(base + oS);
        A.sig.lnE = reinterpret_cast<const double*>(base + olnE);
        A.sig.lnS = reinterpret_cast<const double*>(base + olnS);
        A.sig.lx = reinterpret_cast<const float*>(base + olx);
        A.sig.seg = reinterpret_cast<const float*>(base + oseg);
        A.counters = pl->d_counters;
        A.attempt_budget = ctx->attempt_budget > 0 ? ctx->attempt_budget : static_cast<int64_t>(max_cap) * 51 + 1;
        A.fast_geodesic = pl->fast;
        A.mev = any_mev(cams, n_cams) ? 1 : 0;
        if (want_defer(ctx->transfer_mode, pl->precision, max_bins)) {
            const int64_t slots = defer_slots(ctx->n_sm);
            cudaError_t e2 = cudaMalloc(&pl->d_rec, rec_bytes(slots, max_bins));
            if (e2 != cudaSuccess) {
                hadros_plan_destroy(pl);
                return fail(HADROS_E_NOMEM, std::string("plan deferred transfer buffers: ") + cudaGetErrorString(e2));
            }
            set_defer(A, pl->d_rec, slots, max_bins);
        }
        int32_t rc = prepare_trace(A, pl->precision, pl->fast, ctx->n_sm, sc.blocks_per_sm, pl->cfg, err);
        if (rc) {
            hadros_plan_destroy(pl);
            return fail(rc, err);
        }
        *out = pl;
        return ok();
    } catch (const std::exception& ex) {
        return fail(HADROS_E_NOMEM, ex.what());
    }
}

int32_t hadros_plan_info(const hadros_plan* pl, int64_t* n_pixels, int64_t* n_pixel_bins, int32_t* grid,
                         int32_t* blocks_per_sm)
{
    if (!pl) return fail(HADROS_E_STATE, "plan is NULL");
    if (n_pixels) *n_pixels = pl->P;
    if (n_pixel_bins) *n_pixel_bins = pl->PB;
    if (grid) *grid = static_cast<int32_t>(pl->cfg.grid);
    if (blocks_per_sm) *blocks_per_sm = pl->cfg.per_sm;
    return ok();
}

int32_t hadros_plan_launch(hadros_plan* pl, const hadros_image_out* dev_out, void* stream)
{
    if (!pl) return fail(HADROS_E_STATE, "plan is NULL");
    if (!dev_out) return fail(HADROS_E_ARG, "output struct is NULL");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    TraceArgs A = pl->A;
    set_outputs(A, *dev_out);
    cudaError_t e = cudaMemsetAsync(pl->d_counters, 0, 4 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return fail(HADROS_E_CUDA, std::string("plan counter reset: ") + cudaGetErrorString(e));
    if (pl->P == 0) return ok();
    std::string err;
    const int32_t rc = launch_trace_prepared(A, pl->precision, pl->fast, pl->cfg, st, err);
    return rc ? fail(rc, err) : ok();
}

int32_t hadros_plan_counters(hadros_plan* pl, void* stream, int64_t* steps, int64_t* attempts, int32_t* aborted)
{
    if (!pl) return fail(HADROS_E_STATE, "plan is NULL");
    unsigned long long c[4] = {0, 0, 0, 0};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(c, pl->d_counters, sizeof(c), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(HADROS_E_CUDA, std::string("plan counters: ") + cudaGetErrorString(e));
    if (steps) *steps = static_cast<int64_t>(c[1]);
    if (attempts) *attempts = static_cast<int64_t>(c[2]);
    if (aborted) *aborted = static_cast<int32_t>(c[3]);
    return c[3] > 0 ? fail(HADROS_E_TIMEOUT, "rays exceeded the attempt budget") : ok();
}

void hadros_plan_destroy(hadros_plan* pl)
{
    if (!pl) return;
    cudaSetDevice(pl->device);
    cudaFree(pl->d_tabs);
    cudaFree(pl->d_counters);
    cudaFree(pl->d_rec);
    delete pl;
}

}  // extern "C"
