/*
 * hadros_oracle.h — CPU ORACLE (test infrastructure only; see hadros_oracle.c).
 * Parameters use the POD hadros_params of include/hadros_b200.h so tests pass
 * the same struct to the oracle and to the CUDA library.
 */
#ifndef HADROS_ORACLE_H
#define HADROS_ORACLE_H

#include <stdint.h>
#include "../include/hadros_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define HOR_MAX_BINS 256

/* include/constants.hpp:9-13 */
#define HOR_C_CGS 2.99792458e10
#define HOR_G_CGS 6.67430e-8
#define HOR_MSUN_G 1.98847e33
#define HOR_M_U_G 1.66053906660e-24

/* GeodesicState, include/geodesic_state.hpp:4-16 */
typedef struct { double t, r, theta, phi, pt, pr, ptheta, pphi; } hor_state;
/* nonzero Boyer-Lindquist components: tt, t-phi, rr, theta-theta, phi-phi */
typedef struct { double tt, tph, rr, thth, phph; } hor_m5;

/* TorusProfile after its constructor clamps (src/torus_profile.cpp:20-41) */
typedef struct {
    int kind;
    double rho0, r0, sigma_r, H, radial_power, funnel_depletion, funnel_theta,
           env_rho0, env_alpha, r_min, r_max, rho_floor;
} hor_torus;

/* per-camera constants of one image */
typedef struct {
    const hadros_params* p;
    hor_torus torus;
    double rho_norm;
    const double* sigE;
    const double* sigS;
    int sig_n;
    double rg_cm;
    double rt_r_skip;   /* r_+(a clamped to [0,0.999999]) + 1e-3 */
    double r_stop;      /* r_+ + 1e-3 */
    int n_bins;
    const double* E_mid;
} hor_cam;

typedef void (*hor_point_cb)(void* user, double r, double theta, double phi,
                             double dl_rg, double redshift);

double hor_sigma_fn(double a, double r, double th);
double hor_delta_fn(double a, double r);
double hor_A_fn(double a, double r, double th);
void hor_metric(double a, double r, double th, hor_m5* g);
void hor_inverse_metric(double a, double r, double th, hor_m5* gi);
double hor_lapse(double a, double r, double th);
double hor_omega(double a, double r, double th);
void hor_rhs(double a, const hor_state* y, hor_state* d);
int hor_step_adaptive(double a, double h0, double tol, hor_state* y);
double hor_pixel_u(const hadros_params* p, int i);
double hor_pixel_v(const hadros_params* p, int j);
void hor_initial_state(const hadros_params* p, int i, int j, hor_state* y);
double hor_sigma_interp(const double* xs, const double* ys, int n, double x);
double hor_rho(const hor_torus* t, double r, double theta);
double hor_spectral_weight(const hadros_params* p, double E);
int hor_spectral_bins(const hadros_params* p, double sig_Emin, double sig_Emax,
                      double* E_mid, double* dE, double* w, int8_t* valid);

int hor_cam_init(hor_cam* cam, const hadros_params* p, const double* sigE,
                 const double* sigS_cm2, int sig_n, const double* E_mid, int n_bins);
/* Trace one pixel; fills tau_b/I_b[n_bins] and, when mev5 is not NULL, the
 * MeV channel's tau, P, I, r_nu, leakage; returns enum hadros_fate. */
int hor_trace_pixel(const hor_cam* cam, int i, int j, double* tau_b, double* I_b,
                    int32_t* steps_out, int32_t* attempts_out, double* mev5,
                    hor_point_cb cb, void* cb_user);

/* Whole image (pixel_ids == NULL) or a pixel list, OpenMP over pixels.
 * Returns the number of bins written per pixel (or -1). */
int hor_image(const hadros_params* p, const double* sigE, const double* sigS_cm2, int sig_n,
              const int32_t* pixel_ids, int32_t n_pixels,
              double* tau, double* P_surv, double* I_obs, int8_t* fate,
              int32_t* steps, int32_t* attempts, double* tau_E, double* I_E,
              double* tau_mev, double* P_surv_mev, double* I_obs_mev, double* r_nu,
              double* leakage, int n_threads);

/* Helpers for tests (ctypes-friendly, no structs by value). */
void hor_inverse_metric5(double a, double r, double th, double* out5);
void hor_metric5(double a, double r, double th, double* out5);
double hor_rho_params(const hadros_params* p, double r, double theta);
int hor_rkf45_step(double a, double h0, double tol, double* state8);
int hor_trace_points(const hadros_params* p, const double* sigE, const double* sigS_cm2,
                     int sig_n, int i, int j, int max_points, double* out_points5,
                     int32_t* n_points, int32_t* fate);

#ifdef __cplusplus
}
#endif

#endif
