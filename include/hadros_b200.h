/*
 * hadros_b200.h — C ABI of the B200-native HADROS per-pixel image pipeline.
 *
 * The pipeline is the one HADROS runs per pixel: Kerr camera ray setup,
 * RKF45 null-geodesic integration in Boyer-Lindquist coordinates, DIS optical
 * depth tau_E = sum n_b sigma_CC(E_local) dl and UHE radiative transfer
 * I_E += g^3 j(r, theta, E_local) exp(-tau_E) dl per spectral bin.
 *
 * In the reference these stages are C++ classes driven by command-line
 * executables (no library API):
 *   KerrCamera::trace_pixel                  src/kerr_camera.cpp:188-283
 *   KerrGeodesic::step_adaptive              src/kerr_geodesic.cpp:194-329
 *   SigmaTable                               src/sigma_table.cpp:9-124
 *   TorusProfile::rho                        src/torus_profile.cpp:261-272
 *   radiative_transfer::integrate_kerr_ray_spectral
 *                                            src/radiative_transfer.cpp:687-780
 *   executables compute_kerr_geodesics + compute_kerr_image_from_cache
 *   (CPU) and compute_kerr_image_cuda (GPU).
 * This header replaces that boundary with plain C: POD parameters, caller-owned
 * output buffers, integer status codes and a per-thread error message.
 *
 * Conventions
 *  - Pixel p = j * nx + i, i in [0, nx) along alpha (u), j in [0, ny) along
 *    beta (v); the reference's KIMG row order (apps/compute_kerr_image_cuda.cu:
 *    279-332).
 *  - No function throws or aborts; every entry point returns HADROS_OK (0) or
 *    a HADROS_E_* code and leaves a message for hadros_last_error().
 *  - A hadros_ctx owns one CUDA stream and its device buffers; one context is
 *    used by one host thread at a time. Distinct contexts may run concurrently.
 *  - A hadros_sigma handle is immutable after creation and may be shared.
 */
#ifndef HADROS_B200_H
#define HADROS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HADROS_ABI_VERSION 2

/* Status codes.  The reference reports errors by throwing std::runtime_error
 * (e.g. src/torus_profile.cpp:85-90, src/sigma_table.cpp:14-16) or by exiting
 * with code 1/2 (apps/compute_kerr_image_cuda.cu:2607-2610, :1822). */
enum hadros_status {
    HADROS_OK = 0,
    HADROS_E_ARG = 1,     /* bad argument, unknown model name, bad sizes   */
    HADROS_E_IO = 2,      /* file missing, unreadable or malformed          */
    HADROS_E_CUDA = 3,    /* CUDA runtime error or no usable device         */
    HADROS_E_RANGE = 4,   /* energy outside the sigma table                 */
    HADROS_E_TIMEOUT = 5, /* device attempt budget exhausted (rays aborted) */
    HADROS_E_NOMEM = 6,   /* host or device allocation failed               */
    HADROS_E_STATE = 7    /* null handle or call on a failed context        */
};

/* Density morphologies, in the order of DensityProfileKind
 * (include/torus_profile.hpp:6-15). */
enum hadros_profile_kind {
    HADROS_PROFILE_GAUSSIAN = 0,
    HADROS_PROFILE_POWERLAW = 1,
    HADROS_PROFILE_GAUSSIAN_FUNNEL = 2,
    HADROS_PROFILE_POWERLAW_FUNNEL = 3,
    HADROS_PROFILE_GAUSSIAN_ENVELOPE = 4,
    HADROS_PROFILE_POWERLAW_ENVELOPE = 5,
    HADROS_PROFILE_POWERLAW_FUNNEL_ENVELOPE = 6,
    HADROS_PROFILE_COLLAPSAR_NDAF_LIKE = 7
};

/* UHE source morphologies (include/radiative_transfer.hpp:37-43). */
enum hadros_source_kind {
    HADROS_SOURCE_INNER_RING = 0,
    HADROS_SOURCE_FUNNEL_WALL = 1,
    HADROS_SOURCE_JET_BASE = 2,
    HADROS_SOURCE_SHOCK_LAYER = 3,
    HADROS_SOURCE_DENSITY_WEIGHTED = 4
};

/* UHE spectral models (include/radiative_transfer.hpp:23-27). */
enum hadros_spectral_kind {
    HADROS_SPECTRAL_MONOCHROMATIC = 0,
    HADROS_SPECTRAL_POWERLAW = 1,
    HADROS_SPECTRAL_POWERLAW_CUTOFF = 2
};

/* Arithmetic of the transfer stage.  The geodesic is FP64 in both.
 * Independently, hadros_params.fast_geodesic = 1 evaluates the same RKF45 /
 * centred-difference geodesic with fewer FP64 divisions and transcendentals
 * and with FMA contraction: same algorithm, different rounding. */
enum hadros_precision {
    HADROS_PRECISION_FP64 = 0,  /* every stage FP64, reference operation order */
    HADROS_PRECISION_MIXED = 1  /* FP64 geodesic; FP32 Kahan tau and I per bin */
};

/* Ray fate.  The reference keeps only `captured` (include/ray.hpp:25); a ray
 * that hits the step cap has captured == false (src/kerr_camera.cpp:222). */
enum hadros_fate {
    HADROS_FATE_ESCAPED = 0,   /* r >= r_max after more than 10 steps     */
    HADROS_FATE_CAPTURED = 1,  /* r <= r_+ + 1e-3                          */
    HADROS_FATE_TRUNCATED = 2  /* step cap reached first ("neither")      */
};

/* MeV thermal neutrino channel: the second transfer that integrate_kerr_ray
 * runs along the same path (src/radiative_transfer.cpp:522-638) with the
 * microphysics of src/mev_neutrino_physics.cpp.  Enums in the order of
 * include/mev_neutrino_physics.hpp:8-37. */
enum hadros_mev_model { HADROS_MEV_TOY = 0, HADROS_MEV_PHYSICAL = 1 };
enum hadros_mev_flavor { HADROS_MEV_NU_E = 0, HADROS_MEV_ANTI_NU_E = 1, HADROS_MEV_NU_X = 2 };
enum hadros_mev_thermal {
    HADROS_MEV_T_CONSTANT = 0,
    HADROS_MEV_T_INNER_HOT_TORUS = 1,
    HADROS_MEV_T_RADIAL_POWERLAW = 2,
    HADROS_MEV_T_TORUS_PLUS_COOL_ENVELOPE = 3,
    HADROS_MEV_T_COLLAPSAR_INNER_HOT = 4
};
enum hadros_mev_ye {
    HADROS_MEV_YE_CONSTANT = 0,
    HADROS_MEV_YE_NEUTRON_RICH_TORUS = 1,
    HADROS_MEV_YE_FUNNEL_PROTON_RICH = 2,
    HADROS_MEV_YE_TORUS_ENVELOPE_CONTRAST = 3,
    HADROS_MEV_YE_COLLAPSAR_NEUTRON_RICH = 4
};
enum hadros_mev_spectral { HADROS_MEV_MONOCHROMATIC = 0, HADROS_MEV_FERMI_DIRAC_BAND = 1 };
/* The include_* / use_* switches of MeVThermalParams
 * (include/radiative_transfer.hpp:71-81) as bits of hadros_params.mev_flags. */
enum hadros_mev_flag {
    HADROS_MEV_URCA = 1 << 0,
    HADROS_MEV_PAIR = 1 << 1,
    HADROS_MEV_BREMS = 1 << 2,
    HADROS_MEV_ABSORPTION = 1 << 3,
    HADROS_MEV_SCATTERING = 1 << 4,
    HADROS_MEV_DEGENERACY_CORRECTION = 1 << 5,
    HADROS_MEV_ABS_N = 1 << 6,
    HADROS_MEV_ABS_P = 1 << 7,
    HADROS_MEV_SCAT_N = 1 << 8,
    HADROS_MEV_SCAT_P = 1 << 9,
    HADROS_MEV_SCAT_E = 1 << 10
};
/* every switch of the reference's defaults: all on but the degeneracy correction */
#define HADROS_MEV_FLAGS_DEFAULT 0x7DF

/* All parameters of one camera/image.  Fill with hadros_params_default()
 * and override fields.  Angles are radians except fov_deg, which KerrCamera
 * takes in degrees (src/kerr_camera.cpp:79-98). */
typedef struct hadros_params {
    uint32_t struct_size;    /* = sizeof(hadros_params); set by _default   */
    int32_t nx, ny;          /* image size                                  */
    int32_t max_steps;       /* step cap; reference hard-codes 200000      */
    int32_t profile_kind;    /* enum hadros_profile_kind                    */
    int32_t source_kind;     /* enum hadros_source_kind                     */
    int32_t spectral_kind;   /* enum hadros_spectral_kind                   */
    int32_t n_bins;          /* spectral bins (ignored for monochromatic)  */
    int32_t precision;       /* enum hadros_precision                       */
    int32_t fast_geodesic;   /* 1: fast geodesic arithmetic (default); 0: reference */

    /* camera and integrator: KerrCamera(a, r_obs, theta_obs, fov_deg, nx,
     * ny, r_max, h) with KerrGeodesic tolerance (include/kerr_geodesic.hpp:
     * 10-13; the CPU image path uses the default 1e-6). */
    double a_spin;
    double r_obs_rg;
    double theta_obs_rad;
    double fov_deg;
    double r_max_rg;
    double h;
    double tolerance;

    /* observed energy (monochromatic) and black-hole mass */
    double Enu_obs_GeV;
    double M_bh_msun;

    /* TorusProfile constructor arguments (include/torus_profile.hpp:19-33) */
    double rho0_gcm3;
    double r0_rg;
    double sigma_r_rg;
    double H_over_R;
    double radial_power;
    double funnel_depletion;
    double funnel_theta_rad;
    double envelope_rho0_gcm3;
    double envelope_alpha;
    double torus_r_min_rg;
    double torus_r_max_rg;
    double rho_floor_gcm3;

    /* UHESourceParams (include/radiative_transfer.hpp:45-62) */
    double src_r_center_rg;
    double src_sigma_r_rg;
    double src_theta_width_rad;
    double src_powerlaw;
    double src_emax_GeV;
    double src_norm;
    double src_funnel_theta_rad;
    double src_density_power_q;
    double src_radial_power_s;
    double src_rho_ref_gcm3;
    double src_cutoff_min;
    double src_cutoff_max;
    double src_gradient_dr_rg;
    double src_gradient_dtheta_rad;

    /* UHESpectralParams (include/radiative_transfer.hpp:29-35) */
    double spec_gamma;
    double spec_ecut_GeV;
    double spec_e_min_GeV;
    double spec_e_max_GeV;

    /* MeV thermal channel: MeVThermalParams (include/radiative_transfer.hpp:
     * 64-101), defaults as there.  mev_channel = 0 skips the channel (no cost;
     * the MeV outputs hold RTResult's defaults tau 0, P 1, I 0, r_nu -1,
     * leakage 1); 1 computes it.  FP64 in both precisions. */
    int32_t mev_channel;
    int32_t mev_model;            /* enum hadros_mev_model                    */
    int32_t mev_flavor;           /* enum hadros_mev_flavor                   */
    int32_t mev_thermal_profile;  /* enum hadros_mev_thermal                  */
    int32_t mev_ye_profile;       /* enum hadros_mev_ye                       */
    int32_t mev_spectral_mode;    /* enum hadros_mev_spectral                 */
    int32_t mev_n_bins;           /* Fermi-Dirac band bins                    */
    uint32_t mev_flags;           /* enum hadros_mev_flag bits                */
    double mev_Enu_obs_MeV;
    double mev_norm;
    double mev_sigma_abs0_cm2;
    double mev_sigma_scat0_cm2;
    double mev_neutrinosphere_tau;
    double mev_T0_MeV;
    double mev_T_floor_MeV;
    double mev_T_power;
    double mev_Ye_torus;
    double mev_Ye_funnel;
    double mev_Ye_envelope;
    double mev_Ye_floor;
    double mev_Ye_ceil;
    double mev_E_min_MeV;
    double mev_E_max_MeV;
} hadros_params;

/* Caller-owned outputs.  Any pointer may be NULL (that output is skipped).
 * Per-pixel arrays hold nx*ny entries (or n_pixels for the pixel-list call);
 * per-bin arrays hold that many rows of n_bins entries (1 for
 * monochromatic): tau_E is float in HADROS_PRECISION_MIXED and double in FP64,
 * I_E is always double (intensities span far more than FP32's range).
 * tau/P_surv/I_obs are integrate_kerr_ray_spectral's aggregates
 * (src/radiative_transfer.cpp:687-780); tau_E/I_E are integrate_kerr_ray
 * at each bin's E_mid (src/radiative_transfer.cpp:457-685). */
typedef struct hadros_image_out {
    double* tau;
    double* P_surv;
    double* I_obs;
    int8_t* fate;       /* enum hadros_fate                                */
    int32_t* steps;     /* accepted steps = RayPath::points.size()         */
    int32_t* attempts;  /* RKF45 attempts (>= steps)                       */
    void* tau_E;
    void* I_E;
    /* MeV channel per pixel (RTResult, include/radiative_transfer.hpp:16-20):
     * tau_mev, exp(-tau_mev), I_obs_mev, r of the first point whose
     * tau_mev >= mev_neutrinosphere_tau (-1 if none) and leakage_factor. */
    double* tau_mev;
    double* P_surv_mev;
    double* I_obs_mev;
    double* r_nu;
    double* leakage;
} hadros_image_out;

/* Run statistics of the last image/batch call on a context. */
typedef struct hadros_stats {
    double kernel_ms;        /* device time of the trace kernel(s)          */
    double total_ms;         /* host wall time of the whole call            */
    int64_t rays;
    int64_t accepted_steps;  /* sum of steps                                */
    int64_t attempts;        /* sum of attempts                             */
    int64_t h2d_bytes;       /* host->device bytes copied by the call       */
    int64_t d2h_bytes;       /* device->host bytes copied by the call       */
    int32_t launches;        /* kernels this library launched in the call  */
    int32_t aborted_rays;    /* rays stopped by the attempt budget          */
} hadros_stats;

/* ---- library info, names and parameters --------------------------------- */

int32_t hadros_abi_version(void);
const char* hadros_status_string(int32_t status);
/* Message of the last failing call on this host thread ("" if none). */
const char* hadros_last_error(void);

/* Reference defaults (and fast_geodesic = 1): KerrCamera args of compute_kerr_geodesics
 * (apps/compute_kerr_geodesics.cpp:26-34), argv defaults of
 * compute_kerr_image_from_cache (apps/compute_kerr_image_from_cache.cpp:
 * 33-55), tolerance 1e-6, max_steps 200000, UHESourceParams/UHESpectralParams
 * member defaults. */
void hadros_params_default(hadros_params* p);
/* Validate sizes, kinds and finiteness; HADROS_E_ARG with a message. */
int32_t hadros_params_validate(const hadros_params* p);

/* Name -> kind with the reference's aliases and error text
 * (src/torus_profile.cpp:44-91, src/radiative_transfer.cpp:80-156). */
int32_t hadros_parse_profile(const char* name, int32_t* kind);
int32_t hadros_parse_source(const char* name, int32_t* kind);
int32_t hadros_parse_spectral(const char* name, int32_t* kind);
const char* hadros_profile_name(int32_t kind);
const char* hadros_source_name(int32_t kind);
const char* hadros_spectral_name(int32_t kind);
/* MeV channel names with the reference's aliases and error text
 * (src/mev_neutrino_physics.cpp:37-238): parse_mev_model, parse_mev_flavor,
 * parse_mev_thermal_profile, parse_mev_ye_profile, parse_mev_spectral_mode
 * and their *_name inverses. */
int32_t hadros_parse_mev_model(const char* name, int32_t* kind);
int32_t hadros_parse_mev_flavor(const char* name, int32_t* kind);
int32_t hadros_parse_mev_thermal(const char* name, int32_t* kind);
int32_t hadros_parse_mev_ye(const char* name, int32_t* kind);
int32_t hadros_parse_mev_spectral(const char* name, int32_t* kind);
const char* hadros_mev_model_name(int32_t kind);
const char* hadros_mev_flavor_name(int32_t kind);
const char* hadros_mev_thermal_name(int32_t kind);
const char* hadros_mev_ye_name(int32_t kind);
const char* hadros_mev_spectral_name(int32_t kind);

/* ---- sigma_CC(E) table (SigmaTable, src/sigma_table.cpp) ------------------ */

typedef struct hadros_sigma hadros_sigma;

/* Parse a 3-column "E_GeV sigma_GeV^-2 sigma_cm2" file: '#' and empty lines
 * and non-positive rows skipped, >= 2 rows, strictly increasing E
 * (src/sigma_table.cpp:9-53). */
int32_t hadros_sigma_load(const char* path, hadros_sigma** out);
/* Same validation from arrays (sigma_GeV2 may be NULL). */
int32_t hadros_sigma_from_arrays(const double* E_GeV, const double* sigma_GeV2,
                                 const double* sigma_cm2, int32_t n,
                                 hadros_sigma** out);
int32_t hadros_sigma_info(const hadros_sigma* s, int32_t* n, double* E_min,
                          double* E_max);
/* SigmaTable::sigma_cm2: log-log interpolation, HADROS_E_RANGE outside
 * [E_min, E_max] (src/sigma_table.cpp:81-124).  Host-side. */
int32_t hadros_sigma_eval_cm2(const hadros_sigma* s, double E_GeV, double* out);
void hadros_sigma_destroy(hadros_sigma* s);

/* Spectral bins integrate_kerr_ray_spectral uses (src/radiative_transfer.cpp:
 * 711-737): *n_bins_out entries of E_mid, dE, weight and valid (weight > 0
 * and finite).  Monochromatic: one bin at Enu_obs_GeV, dE = weight = 1.
 * Arrays must hold max(n_bins, 1) entries; any may be NULL. */
int32_t hadros_spectral_bins(const hadros_params* p, const hadros_sigma* s,
                             double* E_mid, double* dE, double* weight,
                             int8_t* valid, int32_t* n_bins_out);

/* ---- device contexts and the image call ----------------------------------- */

typedef struct hadros_ctx hadros_ctx;

/* Create a context on CUDA device `device` (its own non-blocking stream).
 * HADROS_E_CUDA when the device or the kernels for sm_100a are unusable. */
int32_t hadros_ctx_create(int32_t device, hadros_ctx** out);
void hadros_ctx_destroy(hadros_ctx* ctx);
int32_t hadros_ctx_stats(const hadros_ctx* ctx, hadros_stats* out);
/* Upper bound on RKF45 attempts per ray before the ray is aborted with
 * HADROS_E_TIMEOUT (0 = max_steps * 51, the most step_adaptive can take). */
int32_t hadros_ctx_set_attempt_budget(hadros_ctx* ctx, int64_t attempts_per_ray);

/* Where the mixed-precision transfer runs.  IN_LOOP: each thread adds every
 * path point to its ray's bins as the point is reached (accumulators in shared
 * memory, so resident rays per SM fall as bins grow).  DEFERRED: each thread
 * buffers 64 points (24 bytes each) and the warp replays them into the bins
 * together, 32 threads sharing the bins (accumulators in a device slot per
 * thread); the same per-bin arithmetic, so with fast_geodesic = 0 the
 * results are the same bits (the fast arithmetic's FMA contraction may differ
 * between the two kernels, as between any two builds).  AUTO (default):
 * deferred from 24 bins.
 * FP64 mode always transfers in the loop.  Applies to later calls and plans. */
enum hadros_transfer_mode { HADROS_TRANSFER_AUTO = 0, HADROS_TRANSFER_IN_LOOP = 1,
                            HADROS_TRANSFER_DEFERRED = 2 };
int32_t hadros_ctx_set_transfer(hadros_ctx* ctx, int32_t mode);

/* Whole image.  Replaces compute_kerr_geodesics + compute_kerr_image_from_
 * cache (apps/compute_kerr_geodesics.cpp:24-146, apps/compute_kerr_image_
 * from_cache.cpp:31-722) and compute_kerr_image_cuda's in-line mode
 * (apps/compute_kerr_image_cuda.cu:2239-2611).  Outputs are HOST buffers;
 * the call returns when they are filled. */
int32_t hadros_image(hadros_ctx* ctx, const hadros_params* p,
                     const hadros_sigma* s, const hadros_image_out* out);

/* Subset of pixels (ids j*nx+i); outputs indexed by list position.  The
 * oracle harness's trace_pixel-over-a-subset, used for strided CPU baselines
 * and for judging a random pixel subset. */
int32_t hadros_image_pixels(hadros_ctx* ctx, const hadros_params* p,
                            const hadros_sigma* s, const int32_t* pixel_ids,
                            int32_t n_pixels, const hadros_image_out* out);

/* Whole image into DEVICE buffers on `stream` (a cudaStream_t, NULL = the
 * context's stream, which is non-blocking: a caller whose work is on the
 * legacy default stream passes cudaStreamLegacy, not NULL; the same holds
 * for every `stream` of the image, batch and plan entry points).
 * Asynchronous: returns after enqueueing.  For callers that keep results in
 * HBM (batched scans, benchmarks). */
int32_t hadros_image_device(hadros_ctx* ctx, const hadros_params* p,
                            const hadros_sigma* s,
                            const hadros_image_out* dev_out, void* stream);
/* Pixel subset whose ids (j*nx+i) are already in DEVICE memory (the
 * surrogate's fallback list, a judge subset drawn on the device), outputs
 * into DEVICE buffers in list order, on `stream`; asynchronous.  Ids are not
 * range-checked (they are device data): an id outside the image only moves
 * the ray off the screen.  Replaces, for device-resident scans, the judge
 * and fallback traces the reference would run as separate executables per
 * parameter point (scripts/run_robustness_scans.py:81-145). */
int32_t hadros_image_pixels_device(hadros_ctx* ctx, const hadros_params* p,
                                   const hadros_sigma* s, const int32_t* dev_pixel_ids,
                                   int32_t n_pixels, const hadros_image_out* dev_out,
                                   void* stream);
/* Many cameras in one persistent launch (parameter scans: cameras of
 * different size, spin, inclination, profile, rho0 and bins).  Outputs are
 * concatenated in camera order: per-pixel arrays hold sum(nx*ny) entries,
 * per-bin arrays sum(nx*ny*n_bins).  All cameras share the sigma table and
 * must share precision and fast_geodesic.  Replaces the reference's serial
 * per-tile host loop (apps/compute_kerr_image_cuda.cu:2418-2483) repeated per
 * parameter point by the scan drivers (scripts/run_robustness_scans.py:81-145). */
int32_t hadros_batch(hadros_ctx* ctx, const hadros_params* cams, int32_t n_cams,
                     const hadros_sigma* s, const hadros_image_out* out);
/* Pixel subsets of many cameras in one launch: camera c traces counts[c]
 * pixels whose ids (j*nx+i) follow one another in pixel_ids (host arrays);
 * outputs in list order, concatenated as hadros_batch's.  The random pixel
 * subsets the surrogate is trained on, and strided subsets of many cameras. */
int32_t hadros_batch_pixels(hadros_ctx* ctx, const hadros_params* cams, int32_t n_cams,
                            const hadros_sigma* s, const int32_t* pixel_ids,
                            const int32_t* counts, const hadros_image_out* out);
int32_t hadros_batch_device(hadros_ctx* ctx, const hadros_params* cams, int32_t n_cams,
                            const hadros_sigma* s, const hadros_image_out* dev_out,
                            void* stream);

/* ---- plans: scans uploaded once, launches capturable in CUDA graphs -------- */

/* Work schedule of a plan (what the autotuner searches). */
enum hadros_order {
    HADROS_ORDER_ROWS = 0,   /* pixels in row order j*nx+i                          */
    HADROS_ORDER_TILES = 1,  /* 8x4 pixel tiles: a warp traces a compact patch      */
    HADROS_ORDER_COST = 2    /* by descending cost from a coarse pre-pass           */
};
typedef struct hadros_schedule {
    int32_t blocks_per_sm;   /* resident blocks per SM, 0 = occupancy limit         */
    int32_t order;           /* enum hadros_order                                   */
    int32_t coarse_stride;   /* pre-pass stride for HADROS_ORDER_COST (default 16)  */
    int32_t camera_order;    /* 1: queue costly cameras first (outputs keep order)  */
} hadros_schedule;

typedef struct hadros_plan hadros_plan;
void hadros_schedule_default(hadros_schedule* s);
/* Upload cameras, bins and the sigma table once (and, for
 * HADROS_ORDER_COST, run the pre-pass).  Replaces the reference's per-tile
 * host loop with its per-launch synchronization and 4-byte readback
 * (apps/compute_kerr_image_cuda.cu:2418-2483) for repeated scans. */
int32_t hadros_plan_create(hadros_ctx* ctx, const hadros_params* cams, int32_t n_cams,
                           const hadros_sigma* s, const hadros_schedule* sched,
                           hadros_plan** out);
int32_t hadros_plan_info(const hadros_plan* plan, int64_t* n_pixels, int64_t* n_pixel_bins,
                         int32_t* grid, int32_t* blocks_per_sm);
/* Enqueue the plan on `stream` into DEVICE buffers (concatenated outputs as
 * hadros_batch): a 32-byte counter reset and one kernel launch, nothing on
 * the host, so the call can be captured in a CUDA graph and replayed.  One
 * launch of a plan in flight at a time. */
int32_t hadros_plan_launch(hadros_plan* plan, const hadros_image_out* dev_out, void* stream);
/* Wait for `stream` and read the last launch's step/attempt totals. */
int32_t hadros_plan_counters(hadros_plan* plan, void* stream, int64_t* steps, int64_t* attempts,
                             int32_t* aborted);
void hadros_plan_destroy(hadros_plan* plan);

/* ---- geodesic cache (compute_kerr_geodesics / --image-from-cache) ---------- */

/* Trace pixels (all: pixel_ids NULL; or a list) and record every path point
 * as compute_kerr_geodesics stores it: (r, theta, x, y, z, dl_rg, redshift),
 * KerrCamera::trace_pixel's PathPoint (src/kerr_camera.cpp:235-273).
 * points: host buffer of rows x max_points x 7 doubles; npoints[k] = the
 * ray's accepted steps (a value above max_points means the stored path was
 * cut at max_points); fate may be NULL.  Replaces
 * apps/compute_kerr_geodesics.cpp:95-138 and the CUDA --geodesic-cache mode
 * (apps/compute_kerr_image_cuda.cu:1624-1826). */
int32_t hadros_trace_paths(hadros_ctx* ctx, const hadros_params* p, const int32_t* pixel_ids,
                           int32_t n_pixels, int32_t max_points, double* points,
                           int32_t* npoints, int8_t* fate);
/* Radiative transfer over cached paths: n_rays rays with npoints[k] points
 * each, packed back to back in `points` (7 doubles per point, as in KGEO);
 * fate may be NULL (then 0).  Outputs as hadros_image, one row per ray, with
 * steps = npoints and attempts unused.  p supplies the spin (the cache's),
 * mass, medium, source, spectrum and precision.  Replaces
 * apps/compute_kerr_image_from_cache.cpp:599-711 and the CUDA
 * --image-from-cache mode (apps/compute_kerr_image_cuda.cu:1828-2220). */
int32_t hadros_transfer_paths(hadros_ctx* ctx, const hadros_params* p, const hadros_sigma* s,
                              int32_t n_rays, const int32_t* npoints, const int8_t* fate,
                              const double* points, const hadros_image_out* out);

/* Wait for the context's work and report the first deferred error. */
int32_t hadros_ctx_synchronize(hadros_ctx* ctx);

/* Whole image into DEVICE buffers without allocating any GPU memory.  No
 * counterpart in the reference.  For callers that cannot call cudaMalloc
 * (a framework's caching allocator owns the device memory, or a fixed
 * per-tenant memory budget forbids new allocations): it needs no context,
 * and its scratch (work counters, camera and bin tables, sigma table) is a
 * static ~60 KB device array inside this library, held by every GPU that
 * loads it until the process exits.  Runs on the current device, on `stream`
 * (a cudaStream_t; NULL = the legacy default stream), with the
 * reference-arithmetic kernel, and returns when the image is done.  Limits:
 * at most 1024 sigma rows and 64 spectral bins (else HADROS_E_ARG);
 * fast_geodesic must be 0.  Every call looks up the array's address in the
 * current context (a device reset or another current context cannot leave
 * it stale); the first call on a device loads the library's kernels there,
 * so make that first call outside stream capture.  All calls share the
 * array, which keeps the last call's contents (the work counters are cleared
 * at the start of each call): calls that overlap on the GPU race; serialize
 * them.  With 64 bins in mixed precision the kernel keeps the bins in shared
 * memory (up to ~213 KB per block with a 1024-row table): one block per SM. */
int32_t hadros_image_device_noalloc(const hadros_params* p, const hadros_sigma* s,
                                    const hadros_image_out* dev_out, void* stream);

/* ---- the reference's image files (host only) ------------------------------ */

/* Output file name the reference apps use, so scripts that re-derive it find
 * the image: style 0 = compute_kerr_image_cuda in-line mode
 * (apps/compute_kerr_image_cuda.cu:2108-2128), style 1 =
 * compute_kerr_image_from_cache (apps/compute_kerr_image_from_cache.cpp:
 * 477-500; dis_model NULL -> "GBW").  `ext` is appended (".dat", ".bin").
 * The name has no directory part. */
int32_t hadros_image_filename(const hadros_params* p, int32_t style, const char* dis_model,
                              double mev_E_MeV, double mev_norm, const char* ext, char* buf,
                              int32_t buflen);
/* 13-column text image with the reference's '#' metadata header
 * (apps/compute_kerr_image_from_cache.cpp:512-653); rows in j*nx+i order.
 * The MeV columns carry RTResult's defaults (tau 0, P 1, I 0, r_nu -1,
 * leakage 1); hadros_write_dat_mev writes computed ones.  Arrays hold nx*ny
 * entries. */
int32_t hadros_write_dat(const char* path, const hadros_params* p, const char* dis_model,
                         double mev_E_MeV, double mev_norm, const double* tau,
                         const double* P_surv, const double* I_obs, const int8_t* fate);
/* KIMG binary image (apps/compute_kerr_image_cuda.cu:279-332), MeV columns
 * as hadros_write_dat. */
int32_t hadros_write_kimg(const char* path, const hadros_params* p, double mev_E_MeV,
                          double mev_norm, const double* tau, const double* P_surv,
                          const double* I_obs, const int8_t* fate);
/* The same files with the MeV columns of a host hadros_image_out (tau_mev,
 * P_surv_mev, I_obs_mev, r_nu, leakage; a NULL array writes its default) and,
 * in the text header, the MeV parameters of `p` as the CPU app lists them
 * (apps/compute_kerr_image_from_cache.cpp:563-591) when p->mev_channel is
 * set.  The MeV energy and norm of the file name/header are p's. */
int32_t hadros_write_dat_mev(const char* path, const hadros_params* p, const char* dis_model,
                             const hadros_image_out* host);
int32_t hadros_write_kimg_mev(const char* path, const hadros_params* p, const hadros_image_out* host);

/* KGEO geodesic cache files (apps/compute_kerr_geodesics.cpp:14-22, :95-138):
 * header <int32 magic 0x4B47454F, int32 version 1, int32 nx, int32 ny,
 * double a>, then per ray a 40-byte header <int32 ray_id, pixel_i, pixel_j,
 * captured, npoints, 4 pad bytes, double alpha, double beta> and npoints
 * PathPoints of 7 doubles.  The writer takes the packed layout of
 * hadros_transfer_paths (ray_id = i*ny + j, alpha/beta from the camera). */
int32_t hadros_write_kgeo(const char* path, const hadros_params* p, int32_t n_rays,
                          const int32_t* pixel_ids, const int8_t* fate,
                          const int32_t* npoints, const double* points);
/* The same rays written in batches, as the reference's cache writers stream
 * them (apps/compute_kerr_image_cuda.cu:1718-1780): append = 0 creates the
 * file with its header, append = 1 adds rays to it (HADROS_E_IO if the file
 * does not exist). */
int32_t hadros_write_kgeo_rays(const char* path, const hadros_params* p, int32_t n_rays,
                               const int32_t* pixel_ids, const int8_t* fate,
                               const int32_t* npoints, const double* points, int32_t append);
/* First pass: sizes of a KGEO file (reference read loop,
 * apps/compute_kerr_image_from_cache.cpp:374-406, :655-707). */
int32_t hadros_kgeo_info(const char* path, int32_t* nx, int32_t* ny, double* a_spin,
                         int32_t* n_rays, int64_t* n_points);
/* Second pass: per ray pixel id (j*nx+i), captured flag, npoints, alpha,
 * beta, and the packed points.  Arrays sized from hadros_kgeo_info. */
int32_t hadros_read_kgeo(const char* path, int32_t* pixel_ids, int8_t* captured,
                         int32_t* npoints, double* alpha, double* beta, double* points);

/* ---- surrogate network (no counterpart in the reference) -------------------
 * A BF16 tensor-core MLP trained on (pixel, bin) samples that this library
 * traces; it predicts ln tau_E and ln I_E for parameter scans, and an
 * ensemble of such networks marks, through its spread, the pixels the exact
 * tracer must redo.  Inputs: 16 raw features per sample (alpha, beta, a,
 * cos theta_obs, log10 rho0, one-hot profile kind x8, r0, H/R, log10 E_mid);
 * network 64 -> 4 x 256 (SiLU) -> 2 whose inputs are the normalized features
 * split into hi/lo BF16 pairs plus Fourier features of alpha and beta, with
 * an FP32 linear skip.  Pointers are DEVICE pointers
 * unless stated; calls are asynchronous on `stream` (a cudaStream_t; NULL =
 * the legacy default stream) and allocate nothing. */
typedef struct hadros_mlp_norm {   /* host struct, passed by pointer          */
    float feat_mu[16];             /* x = (raw - mu) * inv_sd                 */
    float feat_inv_sd[16];
    float out_mu[2];               /* ln value = mu + sd * network output     */
    float out_sd[2];
    float out_floor[2];            /* targets are ln(value + floor)           */
} hadros_mlp_norm;

typedef struct hadros_adam {
    float lr, beta1, beta2, eps;
} hadros_adam;

/* FP32 master parameters of one network, BF16 elements of its row-major
 * working copy, and training workspace bytes for a batch. */
int64_t hadros_mlp_param_count(void);
int64_t hadros_mlp_packed_count(void);
int64_t hadros_mlp_workspace_bytes(int64_t batch);
/* Offsets (in floats) of W1, b1, W2, b2, W3, b3, W4, b4, W5, b5, Ws and the
 * end of the used parameters in the master array (12 slots). */
int32_t hadros_mlp_layout(int64_t* offsets, int32_t n);
/* master FP32 -> BF16 working copy (W1 twice for the hi/lo columns). */
int32_t hadros_mlp_pack(const float* master, void* packed, void* stream);
/* raw [n][16] FP32 -> X [n][64] BF16 (normalized: hi[16], lo[16], then
 * sin/cos of 8 frequencies of alpha and of beta). */
int32_t hadros_mlp_featurize(const float* raw, int64_t n, const hadros_mlp_norm* norm, void* X,
                             void* stream);
/* Raw features of the samples (pixel_ids[k], bin b) of a camera, rows
 * k * n_bins + b; pixel_ids NULL = pixels 0..n_pixels-1.  The same function
 * the inference kernel evaluates. */
int32_t hadros_mlp_raw_features(const hadros_params* p, const hadros_sigma* s,
                                const int32_t* pixel_ids, int64_t n_pixels, float* raw,
                                void* stream);
/* Forward pass of a batch (stores activations in `workspace` for backward);
 * out [n][2] standardized predictions. */
int32_t hadros_mlp_forward(const float* master, const void* packed, const void* X, int64_t n,
                           void* workspace, float* out, void* stream);
/* Backward pass after hadros_mlp_forward on the same workspace: adds the
 * gradient of sum(dout * out) to grad (master layout; zero it first). */
int32_t hadros_mlp_backward(const void* packed, const void* X, int64_t n, const float* dout,
                            void* workspace, float* grad, void* stream);
/* loss += sum w (out - target)^2 / (2n); dout its gradient; weight may be NULL. */
int32_t hadros_mlp_loss(const float* out, const float* target, const float* weight, int64_t n,
                        float* dout, float* loss, void* stream);
/* One Adam update of the master parameters (step counts from 1). */
int32_t hadros_mlp_adam(float* master, float* m, float* v, const float* grad,
                        const hadros_adam* opt, int64_t step, void* stream);
/* forward + loss + backward + Adam + repack, for one batch. */
int32_t hadros_mlp_train_step(float* master, void* packed, float* m, float* v, const void* X,
                              const float* target, const float* weight, int64_t n,
                              const hadros_adam* opt, int64_t step, void* workspace, float* grad,
                              float* out, float* dout, float* loss, void* stream);

/* Training workspace bytes of hadros_mlp_train_members. */
int64_t hadros_mlp_members_workspace_bytes(int32_t members, int64_t batch);
/* One Adam step of `members` networks (an ensemble) trained side by side in
 * the same launches, each on its own batch of n rows of the shared training
 * set: member k's rows are idx[k * idx_stride + s], s < n, of X_all
 * [rows][64] (featurized), T_all [rows][2] and W_all [rows] (may be NULL).
 * masters, m, v, grad [members][param_count], packed [members][packed_count];
 * loss[k] += member k's batch loss (a NaN there reports a timed-out wait in
 * a tensor-core kernel). */
int32_t hadros_mlp_train_members(int32_t members, int64_t n, const void* X_all, const float* T_all,
                                 const float* W_all, const int64_t* idx, int64_t idx_stride,
                                 float* masters, void* packed, float* m, float* v, float* grad,
                                 const hadros_adam* opt, int64_t step, void* workspace, float* loss,
                                 void* stream);

/* The schedule of a training run whose steps replay from a CUDA graph. */
typedef struct hadros_train_sched {
    float lr_max, lr_min;      /* cosine from lr_max (step 1) to lr_min (step total_steps) */
    float beta1, beta2, eps;   /* Adam */
    int64_t total_steps;
    int64_t steps_per_epoch;   /* batches per pass over each member's index list */
} hadros_train_sched;
/* hadros_mlp_train_members with the step counter in DEVICE memory: the call
 * increments *step_dev on the device and takes the step's learning rate,
 * bias corrections and batch (rows idx[k * idx_stride + ((step - 1) mod
 * steps_per_epoch) * n + s]) from it, so a sequence of calls captured once in
 * a CUDA graph replays the following steps.  Launches only (asynchronous). */
int32_t hadros_mlp_train_members_dev(int32_t members, int64_t n, const void* X_all, const float* T_all,
                                     const float* W_all, const int64_t* idx, int64_t idx_stride,
                                     float* masters, void* packed, float* m, float* v, float* grad,
                                     const hadros_train_sched* sched, int64_t* step_dev,
                                     void* workspace, float* loss, void* stream);

/* Bytes of one network's inference image (weights pre-swizzled for the
 * tensor-core kernel) and its construction from the BF16 working copy. */
int64_t hadros_mlp_image_bytes(void);
int32_t hadros_mlp_pack_image(const void* packed, void* image, void* stream);

/* Schedule of the inference kernel's two 128-sample halves: LOCKSTEP (each
 * streamed weight stage feeds both halves; tensor cores idle during the
 * epilogue) or PINGPONG (the halves alternate on the tensor cores, one half's
 * epilogue overlapping the other's products; default).  Process-wide;
 * hadros_surrogate_schedule(-1) returns the current one. */
enum hadros_surrogate_schedule_kind { HADROS_SURROGATE_LOCKSTEP = 0, HADROS_SURROGATE_PINGPONG = 1 };
int32_t hadros_surrogate_schedule(int32_t schedule);

typedef struct hadros_surrogate_out {   /* DEVICE buffers                        */
    float* ln_tau_E;       /* [P][B] ensemble mean of ln tau_E (may be NULL)   */
    float* ln_I_E;         /* [P][B] ensemble mean of ln I_E (may be NULL)     */
    double* tau;           /* [P] spectral aggregates as integrate_kerr_ray_   */
    double* P_surv;        /*     spectral forms them from the mean prediction */
    double* I_obs;
    float* spread;         /* [P] ensemble standard deviation (see spread_of)  */
    int32_t* fallback_ids; /* [P] pixel ids with spread > threshold, unordered */
    int32_t* counters;     /* [2]: fallback count, abort flag (set by the call) */
} hadros_surrogate_out;

/* Surrogate image of pixels [pixel_begin, pixel_end) of camera p with an
 * ensemble of n_members (1..8) networks: masters [n][param_count] FP32,
 * images [n][image_bytes] (16-byte aligned).  P = pixel_end - pixel_begin,
 * outputs indexed from pixel_begin; B = bins of p, which must divide 256.
 * The spread is the ensemble standard deviation of ln I_obs (spread_of 0)
 * or of ln tau (spread_of 1, for media whose intensity vanishes); pixels
 * above spread_threshold go to fallback_ids.  Asynchronous; after the stream
 * completes, counters[1] != 0 means a wait in the kernel timed out and the
 * outputs are not valid. */
int32_t hadros_surrogate_image(const hadros_params* p, const hadros_sigma* s, int32_t n_members,
                               const float* masters, const void* images,
                               const hadros_mlp_norm* norm, int64_t pixel_begin,
                               int64_t pixel_end, float spread_threshold, int32_t spread_of,
                               const hadros_surrogate_out* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HADROS_B200_H */
