// hadros_internal.h — structures shared by the C-ABI host code and the
// sm_100a trace kernel.  Not part of the public ABI.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/hadros_b200.h"
#include "hadros_physics.cuh"
#include "hadros_physics_f32.cuh"
#include "hadros_mev.cuh"

namespace hadros {

constexpr int kTPB = 128;        // threads per block of the trace kernel
constexpr int kMaxBins = 256;    // per-camera spectral bins
constexpr int kMaxSigma = 4096;  // sigma table rows staged in shared memory

// Per-camera constants, computed once on the host with the host libm (so the
// observer-side quantities are the reference's own values bit for bit).
struct DevCam {
    // camera and integrator (src/kerr_camera.cpp:79-186, kerr_geodesic.cpp)
    double a;
    double r_obs, th_obs, tan_half;
    double r_max, h0, h_min, tol;
    double r_stop;                    // r_+ + 1e-3
    double g_tt, g_tph, g_rr, g_thth, g_phph;
    double sq_grr, sq_gthth, sq_gphph;
    double alpha_obs, omega_obs, pt_contra;
    double c0[15];                    // RKF45 stage coefficients at h = h0
    // transfer (src/radiative_transfer.cpp:457-685)
    double rt_skip;                   // r_+(clamped a) + 1e-3
    double rg_cm;
    Torus torus;
    Source src;
    TorusF torus_f;                   // FP32 constants for the mixed transfer
    SourceF src_f;
    double k_nb;                      // sigma_scale / m_u (mixed transfer)
    Mev mev;                          // MeV thermal channel (radiative_transfer.cpp:522-638)
    int32_t nx, ny, max_steps, n_bins;
    int32_t mono;
    int32_t sp_emit;                  // some bin has E_mid > 0 (an empty band emits nothing)
    float sp_gamma;                   // spectral index shared by the bins' w(E)/w(E_mid)
    int32_t bin_offset;               // first row in the bin tables
    int64_t item_begin;               // first work item of this camera
    int64_t item_end;
    int64_t out_offset;               // first output row
    int64_t binout_offset;            // first per-bin output element
};

// Per-bin constants (one row per camera bin).
struct DevBin {
    double E_mid;       // bin centre energy (monochromatic: Enu_obs)
    double dE;          // bin width (1 for monochromatic)
    double w;           // aggregation weight w(E_mid)*dE (1 for monochromatic)
    double w0;          // spectral_weight(E_mid): scale of the FP32 intensity
    double gg_lo, gg_hi;// E_mid/gg in [E_min, E_max]  <=>  gg in [gg_lo, gg_hi]
    float lnE;          // log(E_mid)
    float kcut;         // E_mid / E_cut (or / E_max for monochromatic), 0 if none
    float gamma;        // spectral index of the ratio w(E)/w(E_mid)
    int32_t valid;      // counted in the spectral aggregates
    float kcut2;        // kcut * log2(e): the cutoff term in base-2 exponents
    float qbase;        // (log(E_mid) - log(E_0)) / (sigma table step): segment coordinate at g = 1
};

// Sigma table staged in shared memory.  FP64 arrays follow SigmaTable::
// log_interp (src/sigma_table.cpp:81-124); the FP32 segment form is the
// mixed-precision lookup sigma = sigma_scale * s1[k] * exp(t * dly[k]).
struct SigmaDev {
    int32_t n;
    int32_t uniform;     // ln E nearly evenly spaced: direct segment index
    float lx0, inv_dlx;
    double E_min, E_max, sigma_scale;
    const double* E;     // [n]
    const double* S;     // [n]  sigma_cm2
    const double* lnE;   // [n]  log(E_k)
    const double* lnS;   // [n]  log(sigma_k)
    const float* lx;     // [n]  (float)log(E_k)
    const float* seg;    // [4n] per segment k>=1: lx1, 1/(lx2-lx1), s1, dly*log2(e)
};

// One path point's bin-independent transfer terms in mixed precision (24
// bytes; the deferred transfer buffers them).  Exponents are base 2.
struct PointRec {
    float lnzp;    // ln(E_local / E_mid) = ln(1/g)
    float zm1;     // E_local / E_mid - 1
    float u2;      // log2(g^3 C dl_cm) - gamma log2(1/g); -inf: no emission at this point
    float nbdl2;   // n_b dl_cm log2(e); negative: no density
    int32_t b0, b1;// bins whose E_local lies in the sigma table's range: b0..b1 (decided in FP64)
};
// Points a thread buffers between deferred transfers.  Each replay moves a
// lane's accumulator slot (20 bytes per bin) in and out of device memory, so
// a deeper buffer halves that traffic per point; 128 measured 2.5 % faster
// than 64 on the 64-bin production camera (the buffers of all resident
// threads exceed L2 either way).
#ifndef HADROS_REC_DEPTH
#define HADROS_REC_DEPTH 128
#endif
constexpr int kRecDepth = HADROS_REC_DEPTH;   // points a thread buffers between deferred transfers
constexpr int kDeferMinBins = 24;   // bins from which the host picks deferred transfer
constexpr int kAccF = 5;            // FP32 accumulators per bin in mixed precision

struct TraceArgs {
    const DevCam* cams;
    int32_t n_cams;
    int32_t max_bins;
    int64_t total_items;
    const int32_t* pixel_ids;   // optional list (single camera)
    const DevBin* bins;
    SigmaDev sig;
    // outputs (device); any may be null
    double* tau;
    double* P_surv;
    double* I_obs;
    int8_t* fate;
    int32_t* steps;
    int32_t* attempts;
    void* tau_E;        // float (mixed) or double (fp64)
    double* I_E;
    double* tau_mev;    // MeV channel per pixel
    double* P_surv_mev;
    double* I_obs_mev;
    double* r_nu;
    double* leakage;
    int32_t mev;        // some camera has mev_channel set: the kernel variant that computes it
    // scratch
    unsigned long long* counters;   // [0] work cursor, [1] steps, [2] attempts, [3] aborted
    int64_t attempt_budget;
    int32_t fast_geodesic;          // 1: geo_rhs_fast (hadros_trace_fast.cu)
    // path recording (trace kernel): [rows][path_cap][7] PathPoint doubles
    double* paths;
    int32_t path_cap;
    // cached paths (path transfer kernel): points [n][7], ray offsets [rays+1]
    const int64_t* path_offsets;
    const double* path_points;
    const int8_t* path_fates;
    // schedule: optional item -> pixel order (outputs stay in pixel order)
    // and a cap on resident blocks per SM (0 = occupancy)
    const int32_t* order;
    int32_t blocks_per_sm;
    // deferred transfer (mixed only; rec_buf null = per-point transfer in the
    // loop): per thread slot kRecDepth PointRecs and kAccF x rec_bmax FP32
    // accumulators (S, T, Tc, I, Ic); at most rec_slots threads in the grid
    PointRec* rec_buf;
    float* rec_state;
    int32_t rec_bmax;
    int64_t rec_slots;
};

inline size_t rec_bytes(int64_t slots, int bmax)
{
    return static_cast<size_t>(slots) * (kRecDepth * sizeof(PointRec) + kAccF * sizeof(float) * static_cast<size_t>(bmax));
}

struct LaunchCfg {
    unsigned grid;
    size_t smem;
    int per_sm;
};

// Host-side handle of an uploaded sigma table.
struct SigmaHost {
    std::vector<double> E, s_GeV2, s_cm2;
    std::vector<double> lnE, lnS;
    std::vector<float> lx, seg;
    double sigma_scale = 1.0;
    int32_t uniform = 0;
    float lx0 = 0.0f, inv_dlx = 0.0f;
    double inv_step = 0.0;   // 1 / (ln E step) of an evenly spaced table
};

// FP32 constants of the mixed transfer (torus_f, src_f, k_nb) from a camera's
// torus and source; called by every camera builder.
inline void fill_mixed_constants(DevCam& cam, double sigma_scale)
{
    cam.torus_f = make_torus_f(cam.torus);
    cam.src_f = make_source_f(cam.src);
    cam.k_nb = sigma_scale / kMuG;
}

// Camera plan building (host, hadros_trace.cu).  build_cam_into writes the
// camera's bins into caller storage of `cap` rows with no heap use (n_bins_out
// rows; bin_offset 0) and fails with HADROS_E_ARG beyond cap; build_cam appends
// them to `bins` and sets bin_offset.
int build_cam_into(const hadros_params& p, const SigmaHost& sig, DevCam& cam, DevBin* bins, int cap,
                   int* n_bins_out, const char** err);
int build_cam(const hadros_params& p, const SigmaHost& sig, DevCam& cam,
              std::vector<DevBin>& bins, std::string& err);
void prepare_sigma(SigmaHost& s);

// Kernel launch (hadros_trace.cu).  `stream` is a cudaStream_t.
int launch_trace(const TraceArgs& args, int precision, int n_sm, void* stream,
                 std::string& err);
int launch_trace_fast(const TraceArgs& args, int precision, int n_sm, void* stream,
                      std::string& err);
int launch_path_transfer(const TraceArgs& args, int precision, int n_sm, void* stream,
                         std::string& err);
int launch_path_transfer_fast(const TraceArgs& args, int precision, int n_sm, void* stream,
                              std::string& err);
// Prepared launches (plans): the setup once, then only the kernel enqueue.
int prepare_trace(const TraceArgs& args, int precision, int fast, int n_sm, int blocks_per_sm,
                  LaunchCfg& cfg, std::string& err);
int launch_trace_prepared(const TraceArgs& args, int precision, int fast, const LaunchCfg& cfg,
                          void* stream, std::string& err);
int prepare_trace_fast(const TraceArgs& args, int precision, int n_sm, int blocks_per_sm,
                       LaunchCfg& cfg, std::string& err);
int launch_trace_prepared_fast(const TraceArgs& args, int precision, const LaunchCfg& cfg,
                               void* stream, std::string& err);
size_t trace_smem_bytes(int precision, int sig_n, int max_bins);

// Record the calling thread's hadros_last_error() message; returns `code`.
int32_t set_error(int32_t code, const std::string& msg);

}  // namespace hadros

// hadros_sigma is the public opaque handle.
struct hadros_sigma {
    hadros::SigmaHost h;
    uint64_t serial = 0;   // distinguishes handles that reuse an address
};
