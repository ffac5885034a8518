/*
 * hadros_oracle.c — CPU ORACLE for the HADROS per-pixel image pipeline.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; the product (hadros_b200/) never links, loads or calls it.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * It restates, in plain C, the reference algorithm for one camera image:
 *   Kerr metric            src/kerr_metric.cpp:10-145
 *   geodesic RHS (FD)      src/kerr_geodesic.cpp:47-135
 *   RK4 / RKF45 stepping   src/kerr_geodesic.cpp:137-329
 *   camera + trace loop    src/kerr_camera.cpp:14-283
 *   sigma table            src/sigma_table.cpp:9-124
 *   density profiles       src/torus_profile.cpp:12-272
 *   UHE sources/spectra    src/radiative_transfer.cpp:64-76, :172-395
 *   transfer along a ray   src/radiative_transfer.cpp:457-685 (UHE terms)
 *   spectral aggregation   src/radiative_transfer.cpp:687-780
 * Every expression keeps the reference's operand order so that, compiled by
 * gcc with the reference flags (-O3, x86-64 baseline: no FMA contraction)
 * against the same libm, results are bit-identical to the reference.  That
 * claim is checked by tests against the reference itself, built from its own
 * sources by oracle/build_ref.sh, and against fixtures made from it.
 *
 *   MeV thermal channel    src/radiative_transfer.cpp:522-638 with
 *                          src/mev_neutrino_physics.cpp:240-770
 * Deliberate differences from the reference, none of which changes a result:
 *   - the MeV thermal channel is evaluated only when its outputs are asked
 *     for: it never feeds tau/P_surv/I_obs;
 *   - the four off-centre inverse metrics of each RHS are evaluated once
 *     instead of once per (mu, nu) pair (same arguments, same values);
 *   - terms that are exactly zero (g^{01}, g^{02}, derivatives of zero
 *     components) are skipped: adding +-0 to a finite value is exact;
 *   - the step cap is a parameter (the reference hard-codes 200000 at
 *     src/kerr_camera.cpp:222);
 *   - RKF45 attempts are counted (for FLOP accounting).
 */
#include "hadros_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static const double PI = 3.141592653589793238462643383279502884;

/* std::max / std::min / std::clamp semantics, NaN behaviour included. */
static inline double smax(double a, double b) { return (a < b) ? b : a; }
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double sclamp(double v, double lo, double hi)
{
    return (v < lo) ? lo : (hi < v) ? hi : v;
}

/* ---------------- Kerr metric (src/kerr_metric.cpp) ---------------------- */

double hor_sigma_fn(double a, double r, double th)
{   /* kerr_metric.cpp:15-18 */
    return r*r + a*a * cos(th)*cos(th);
}

double hor_delta_fn(double a, double r)
{   /* kerr_metric.cpp:20-23 */
    return r*r - 2.0*r + a*a;
}

double hor_A_fn(double a, double r, double th)
{   /* kerr_metric.cpp:25-32 */
    const double s2 = sin(th)*sin(th);
    return (r*r + a*a)*(r*r + a*a) - a*a * hor_delta_fn(a, r) * s2;
}

void hor_metric(double a, double r, double th, hor_m5* g)
{   /* kerr_metric.cpp:34-78 */
    const double sig = hor_sigma_fn(a, r, th);
    const double del = hor_delta_fn(a, r);
    const double s = sin(th);
    const double s2 = s*s;
    g->tt = -(1.0 - 2.0*r/sig);
    g->tph = -2.0*a*r*s2/sig;
    g->rr = sig / del;
    g->thth = sig;
    g->phph = (r*r + a*a + 2.0*a*a*r*s2/sig) * s2;
}

void hor_inverse_metric(double a, double r, double th, hor_m5* gi)
{   /* kerr_metric.cpp:80-119 */
    const double sig = hor_sigma_fn(a, r, th);
    const double del = hor_delta_fn(a, r);
    const double s = sin(th);
    const double s2 = s*s;
    const double bigA = hor_A_fn(a, r, th);
    gi->tt = -bigA / (sig * del);
    gi->tph = -2.0*a*r / (sig * del);
    gi->rr = del / sig;
    gi->thth = 1.0 / sig;
    gi->phph = (del - a*a*s2) / (sig * del * s2);
}

double hor_lapse(double a, double r, double th)
{   /* kerr_metric.cpp:121-131 */
    const double sig = hor_sigma_fn(a, r, th);
    const double del = hor_delta_fn(a, r);
    const double bigA = hor_A_fn(a, r, th);
    return sqrt(sig * del / bigA);
}

double hor_omega(double a, double r, double th)
{   /* kerr_metric.cpp:133-145 */
    const double s2 = sin(th)*sin(th);
    return 2.0*a*r / ((r*r + a*a)*(r*r + a*a) - a*a*hor_delta_fn(a, r)*s2);
}

/* ---------------- geodesic RHS (src/kerr_geodesic.cpp:47-135) ------------ */

/* d/dlambda of (t, r, theta, phi, p_t, p_r, p_theta, p_phi).  p_t and p_phi
 * are constants of motion (dydl.pt = dydl.pphi = 0, :112-113). */
void hor_rhs(double a, const hor_state* y, hor_state* d)
{
    hor_m5 gi, gp, gm;
    const double p0 = y->pt, p1 = y->pr, p2 = y->ptheta, p3 = y->pphi;
    hor_inverse_metric(a, y->r, y->theta, &gi);

    /* :102-107  dx^mu = g^{mu nu} p_nu, summed nu = 0..3 */
    d->t = gi.tt * p0 + gi.tph * p3;
    d->r = gi.rr * p1;
    d->theta = gi.thth * p2;
    d->phi = gi.tph * p0 + gi.phph * p3;
    d->pt = 0.0;
    d->pphi = 0.0;

    /* :47-81 centred differences; :118-132 summation order (mu, nu) =
     * (0,0),(0,3),(1,1),(2,2),(3,0),(3,3) of -0.5 * dg * p_mu * p_nu. */
    {
        const double eps = 1.0e-5 * smax(1.0, fabs(y->r));
        hor_inverse_metric(a, y->r + eps, y->theta, &gp);
        hor_inverse_metric(a, y->r - eps, y->theta, &gm);
        const double d00 = (gp.tt - gm.tt) / (2.0 * eps);
        const double d03 = (gp.tph - gm.tph) / (2.0 * eps);
        const double d11 = (gp.rr - gm.rr) / (2.0 * eps);
        const double d22 = (gp.thth - gm.thth) / (2.0 * eps);
        const double d33 = (gp.phph - gm.phph) / (2.0 * eps);
        double acc = 0.0;
        acc -= 0.5 * d00 * p0 * p0;
        acc -= 0.5 * d03 * p0 * p3;
        acc -= 0.5 * d11 * p1 * p1;
        acc -= 0.5 * d22 * p2 * p2;
        acc -= 0.5 * d03 * p3 * p0;
        acc -= 0.5 * d33 * p3 * p3;
        d->pr = acc;
    }
    {
        const double eps = 1.0e-5;
        hor_inverse_metric(a, y->r, y->theta + eps, &gp);
        hor_inverse_metric(a, y->r, y->theta - eps, &gm);
        const double d00 = (gp.tt - gm.tt) / (2.0 * eps);
        const double d03 = (gp.tph - gm.tph) / (2.0 * eps);
        const double d11 = (gp.rr - gm.rr) / (2.0 * eps);
        const double d22 = (gp.thth - gm.thth) / (2.0 * eps);
        const double d33 = (gp.phph - gm.phph) / (2.0 * eps);
        double acc = 0.0;
        acc -= 0.5 * d00 * p0 * p0;
        acc -= 0.5 * d03 * p0 * p3;
        acc -= 0.5 * d11 * p1 * p1;
        acc -= 0.5 * d22 * p2 * p2;
        acc -= 0.5 * d03 * p3 * p0;
        acc -= 0.5 * d33 * p3 * p3;
        d->ptheta = acc;
    }
}

/* ---------------- RK4 and RKF45 (src/kerr_geodesic.cpp:137-329) --------- */

/* y0 + c1*k1 (+ c2*k2 ...), component by component, left to right
 * (add_scaled, :141-161).  Trailing terms 0.0 * {} add +0 exactly. */
#define HOR_AXPY1(o, y0, c1, k1) do { \
    (o).t = (y0).t + (c1)*(k1).t; (o).r = (y0).r + (c1)*(k1).r; \
    (o).theta = (y0).theta + (c1)*(k1).theta; (o).phi = (y0).phi + (c1)*(k1).phi; \
    (o).pt = (y0).pt + (c1)*(k1).pt; (o).pr = (y0).pr + (c1)*(k1).pr; \
    (o).ptheta = (y0).ptheta + (c1)*(k1).ptheta; (o).pphi = (y0).pphi + (c1)*(k1).pphi; } while (0)

static void hor_step_rk4(double a, double h, hor_state* y)
{   /* :137-192, fixed step h_ */
    hor_state k1, k2, k3, k4, tmp;
    hor_rhs(a, y, &k1);
    HOR_AXPY1(tmp, *y, 0.5 * h, k1); hor_rhs(a, &tmp, &k2);
    HOR_AXPY1(tmp, *y, 0.5 * h, k2); hor_rhs(a, &tmp, &k3);
    HOR_AXPY1(tmp, *y, h, k3);       hor_rhs(a, &tmp, &k4);
#define HOR_RK4C(f) y->f += h * (k1.f + 2.0*k2.f + 2.0*k3.f + k4.f) / 6.0
    HOR_RK4C(t); HOR_RK4C(r); HOR_RK4C(theta); HOR_RK4C(phi);
    HOR_RK4C(pt); HOR_RK4C(pr); HOR_RK4C(ptheta); HOR_RK4C(pphi);
#undef HOR_RK4C
}

/* One step_adaptive call (:194-329).  Returns the attempts made (1..50, or
 * 51 when the RK4 fallback ran). */
int hor_step_adaptive(double a, double h0, double tol, hor_state* y)
{
    double h = h0;
    const double h_min = h0 * 1.0e-5;
    hor_state k1, k2, k3, k4, k5, k6, s, y4, y5;
    int attempt;
    for (attempt = 0; attempt < 50; ++attempt) {
        hor_rhs(a, y, &k1);
        {
            const double c1 = h * 1.0/4.0;
            HOR_AXPY1(s, *y, c1, k1);
        }
        hor_rhs(a, &s, &k2);
        {
            const double c1 = h * 3.0/32.0, c2 = h * 9.0/32.0;
#define ST(f) s.f = y->f + c1*k1.f + c2*k2.f
            ST(t); ST(r); ST(theta); ST(phi); ST(pt); ST(pr); ST(ptheta); ST(pphi);
#undef ST
        }
        hor_rhs(a, &s, &k3);
        {
            const double c1 = h * 1932.0/2197.0, c2 = h * -7200.0/2197.0,
                         c3 = h * 7296.0/2197.0;
#define ST(f) s.f = y->f + c1*k1.f + c2*k2.f + c3*k3.f
            ST(t); ST(r); ST(theta); ST(phi); ST(pt); ST(pr); ST(ptheta); ST(pphi);
#undef ST
        }
        hor_rhs(a, &s, &k4);
        {
            const double c1 = h * 439.0/216.0, c2 = h * -8.0,
                         c3 = h * 3680.0/513.0, c4 = h * -845.0/4104.0;
#define ST(f) s.f = y->f + c1*k1.f + c2*k2.f + c3*k3.f + c4*k4.f
            ST(t); ST(r); ST(theta); ST(phi); ST(pt); ST(pr); ST(ptheta); ST(pphi);
#undef ST
        }
        hor_rhs(a, &s, &k5);
        {
            const double c1 = h * -8.0/27.0, c2 = h * 2.0,
                         c3 = h * -3544.0/2565.0, c4 = h * 1859.0/4104.0,
                         c5 = h * -11.0/40.0;
#define ST(f) s.f = y->f + c1*k1.f + c2*k2.f + c3*k3.f + c4*k4.f + c5*k5.f
            ST(t); ST(r); ST(theta); ST(phi); ST(pt); ST(pr); ST(ptheta); ST(pphi);
#undef ST
        }
        hor_rhs(a, &s, &k6);

#define Y4(f) y4.f = y->f + h*(25.0/216.0*k1.f + 1408.0/2565.0*k3.f + 2197.0/4104.0*k4.f - 1.0/5.0*k5.f)
#define Y5(f) y5.f = y->f + h*(16.0/135.0*k1.f + 6656.0/12825.0*k3.f + 28561.0/56430.0*k4.f - 9.0/50.0*k5.f + 2.0/55.0*k6.f)
        Y4(t); Y4(r); Y4(theta); Y4(phi); Y4(pt); Y4(pr); Y4(ptheta); Y4(pphi);
        Y5(t); Y5(r); Y5(theta); Y5(phi); Y5(pt); Y5(pr); Y5(ptheta); Y5(pphi);
#undef Y4
#undef Y5
        /* error_norm, :219-233 */
        double err = 0.0;
        err = smax(err, fabs(y4.r - y5.r));
        err = smax(err, fabs(y4.theta - y5.theta));
        err = smax(err, fabs(y4.phi - y5.phi));
        err = smax(err, fabs(y4.pr - y5.pr));
        err = smax(err, fabs(y4.ptheta - y5.ptheta));
        err = smax(err, fabs(y4.pphi - y5.pphi));

        if (err < tol || h <= h_min) {   /* :312-315 */
            *y = y5;
            return attempt + 1;
        }
        {   /* :317-325 */
            const double safety = 0.8;
            const double factor = safety * pow(tol / smax(err, 1.0e-30), 0.25);
            h *= sclamp(factor, 0.1, 5.0);
            if (h < h_min) h = h_min;
        }
    }
    hor_step_rk4(a, h0, y);   /* :328 */
    return 51;
}

/* ---------------- camera (src/kerr_camera.cpp) --------------------------- */

static double deg_to_rad(double x) { return x * PI / 180.0; }   /* :11-14 */

static double zamo_energy(double a, double r, double th, double p_t, double p_phi)
{   /* :16-29 */
    const double alpha = hor_lapse(a, r, th);
    const double omega = hor_omega(a, r, th);
    return -(p_t + omega * p_phi) / alpha;
}

static double wrapped_delta_phi(double phi_new, double phi_old)
{   /* :31-44 */
    double dphi = phi_new - phi_old;
    while (dphi > PI) dphi -= 2.0 * PI;
    while (dphi < -PI) dphi += 2.0 * PI;
    return dphi;
}

static double zamo_spatial_interval_rg(double a, const hor_state* cur, const hor_state* prev)
{   /* :46-76 */
    const double r_mid = 0.5 * (cur->r + prev->r);
    const double theta_mid = 0.5 * (cur->theta + prev->theta);
    hor_m5 g;
    hor_metric(a, r_mid, theta_mid, &g);
    const double dr = cur->r - prev->r;
    const double dtheta = cur->theta - prev->theta;
    const double dphi = wrapped_delta_phi(cur->phi, prev->phi);
    const double dl2 = g.rr * dr * dr + g.thth * dtheta * dtheta + g.phph * dphi * dphi;
    return sqrt(smax(dl2, 0.0));
}

double hor_pixel_u(const hadros_params* p, int i)
{   /* :112-113 (and :196-197) */
    const double fov_rad = deg_to_rad(p->fov_deg);
    return (2.0 * (i + 0.5) / p->nx - 1.0) * tan(0.5 * fov_rad);
}

double hor_pixel_v(const hadros_params* p, int j)
{   /* :115-116 (and :199-200) */
    const double fov_rad = deg_to_rad(p->fov_deg);
    return (2.0 * (j + 0.5) / p->ny - 1.0) * tan(0.5 * fov_rad);
}

void hor_initial_state(const hadros_params* p, int i, int j, hor_state* y)
{   /* :110-186 */
    const double a = p->a_spin, r_obs = p->r_obs_rg, th_obs = p->theta_obs_rad;
    const double u = hor_pixel_u(p, i);
    const double v = hor_pixel_v(p, j);
    const double norm = sqrt(1.0 + u*u + v*v);
    const double n_r = -1.0 / norm;
    const double n_theta = v / norm;
    const double n_phi = u / norm;
    hor_m5 g;
    hor_metric(a, r_obs, th_obs, &g);
    const double alpha = hor_lapse(a, r_obs, th_obs);
    const double omega = hor_omega(a, r_obs, th_obs);
    const double p_t_contra = 1.0 / alpha;
    const double p_r_contra = n_r / sqrt(g.rr);
    const double p_theta_contra = n_theta / sqrt(g.thth);
    const double p_phi_contra = n_phi / sqrt(g.phph) + omega * p_t_contra;
    /* :162-168 p_mu = g_{mu nu} p^nu, zero components skipped */
    y->t = 0.0;
    y->r = r_obs;
    y->theta = th_obs;
    y->phi = 0.0;
    y->pt = g.tt * p_t_contra + g.tph * p_phi_contra;
    y->pr = g.rr * p_r_contra;
    y->ptheta = g.thth * p_theta_contra;
    y->pphi = g.tph * p_t_contra + g.phph * p_phi_contra;
}

/* ---------------- sigma table (src/sigma_table.cpp:81-124) --------------- */

/* lower_bound + log-log interpolation.  Caller guarantees E in range. */
double hor_sigma_interp(const double* xs, const double* ys, int n, double x)
{
    int lo = 0, cnt = n;   /* std::lower_bound: first xs[k] >= x */
    while (cnt > 0) {
        const int step = cnt / 2;
        const int mid = lo + step;
        if (xs[mid] < x) { lo = mid + 1; cnt -= step + 1; }
        else cnt = step;
    }
    if (lo == 0) return ys[0];
    if (lo == n) return ys[n - 1];
    {
        const double x1 = xs[lo - 1], x2 = xs[lo];
        const double y1 = ys[lo - 1], y2 = ys[lo];
        const double lx = log(x);
        const double lx1 = log(x1);
        const double lx2 = log(x2);
        const double ly1 = log(y1);
        const double ly2 = log(y2);
        const double t = (lx - lx1) / (lx2 - lx1);
        return exp(ly1 + t * (ly2 - ly1));
    }
}

/* ---------------- density (src/torus_profile.cpp) ------------------------ */

/* Constructor clamps, :34-40. */
static void torus_resolve(const hadros_params* p, hor_torus* t)
{
    t->kind = p->profile_kind;
    t->rho0 = p->rho0_gcm3;
    t->r0 = p->r0_rg;
    t->sigma_r = p->sigma_r_rg;
    t->H = p->H_over_R;
    t->radial_power = p->radial_power;
    t->funnel_depletion = sclamp(p->funnel_depletion, 0.0, 1.0);
    t->funnel_theta = smax(p->funnel_theta_rad, 1.0e-6);
    t->env_rho0 = smax(p->envelope_rho0_gcm3, 0.0);
    t->env_alpha = p->envelope_alpha;
    t->r_min = p->torus_r_min_rg;
    t->r_max = smax(p->torus_r_max_rg, p->torus_r_min_rg);
    t->rho_floor = smax(p->rho_floor_gcm3, 0.0);
}

static int uses_powerlaw_disk(int k)
{   /* :125-131 */
    return k == HADROS_PROFILE_POWERLAW || k == HADROS_PROFILE_POWERLAW_FUNNEL ||
           k == HADROS_PROFILE_POWERLAW_ENVELOPE || k == HADROS_PROFILE_POWERLAW_FUNNEL_ENVELOPE;
}

static int uses_funnel(int k)
{   /* :133-139 */
    return k == HADROS_PROFILE_GAUSSIAN_FUNNEL || k == HADROS_PROFILE_POWERLAW_FUNNEL ||
           k == HADROS_PROFILE_POWERLAW_FUNNEL_ENVELOPE;
}

static int uses_envelope(int k)
{   /* :141-147 */
    return k == HADROS_PROFILE_GAUSSIAN_ENVELOPE || k == HADROS_PROFILE_POWERLAW_ENVELOPE ||
           k == HADROS_PROFILE_POWERLAW_FUNNEL_ENVELOPE;
}

static int in_torus(const hor_torus* t, double r)
{   /* :118-123 */
    return r >= t->r_min && r <= t->r_max;
}

static double collapsar_ndaf_shape(const hor_torus* t, double r, double theta)
{   /* :150-179 */
    if (!in_torus(t, r) || r <= 0.0 || t->r0 <= 0.0) return 0.0;
    const double mu = cos(theta);
    const double vertical = exp(-pow(mu / smax(t->H, 1.0e-6), 2.0));
    const double inner_taper =
        1.0 / (1.0 + exp(-(r - t->r_min) / smax(0.35 * t->sigma_r, 1.0e-6)));
    const double outer_taper =
        1.0 / (1.0 + exp((r - t->r_max) / smax(0.60 * t->sigma_r, 1.0e-6)));
    const double inner_core =
        0.45 * exp(-pow((r - 0.75 * t->r0) / smax(0.75 * t->sigma_r, 1.0e-6), 2.0));
    const double radial =
        pow(smax(r / t->r0, 1.0e-300), -smax(t->radial_power, 0.0));
    const double floor_tail =
        0.08 * exp(-pow((r - t->r0) / smax(1.8 * t->sigma_r, 1.0e-6), 2.0));
    return (radial + inner_core + floor_tail) * vertical * inner_taper * outer_taper;
}

static double gaussian_shape(const hor_torus* t, double r, double theta)
{   /* :181-196 */
    const double delta = theta - 0.5 * PI;
    if (r <= 4.0 || r >= 18.0 || fabs(delta) >= 0.45) return 0.0;
    const double radial = exp(-pow((r - t->r0) / t->sigma_r, 2.0));
    const double vertical = exp(-pow(delta / t->H, 2.0));
    return radial * vertical;
}

static double powerlaw_shape(const hor_torus* t, double r, double theta)
{   /* :198-217 */
    if (!in_torus(t, r) || r <= 0.0 || t->r0 <= 0.0) return 0.0;
    const double vertical = exp(-pow(cos(theta) / t->H, 2.0));
    const double inner_taper = 1.0 - exp(-pow((r - t->r_min) / t->sigma_r, 2.0));
    const double outer_taper = exp(-pow(r / t->r_max, 4.0));
    const double radial = pow(r / t->r0, -t->radial_power);
    return radial * vertical * inner_taper * outer_taper;
}

static double funnel_factor(const hor_torus* t, double theta)
{   /* :219-236 */
    if (!uses_funnel(t->kind)) return 1.0;
    const double north = exp(-pow(theta / t->funnel_theta, 2.0));
    const double south = exp(-pow((PI - theta) / t->funnel_theta, 2.0));
    return sclamp(1.0 - t->funnel_depletion * (north + south), 0.0, 1.0);
}

static double envelope_rho(const hor_torus* t, double r)
{   /* :238-248 */
    if (!uses_envelope(t->kind) || t->env_rho0 <= 0.0 || r < t->r0 || r > t->r_max)
        return 0.0;
    return t->env_rho0 * pow(r / t->r0, -t->env_alpha);
}

static double disk_shape(const hor_torus* t, double r, double theta)
{   /* :250-259 */
    if (t->kind == HADROS_PROFILE_COLLAPSAR_NDAF_LIKE) return collapsar_ndaf_shape(t, r, theta);
    return uses_powerlaw_disk(t->kind) ? powerlaw_shape(t, r, theta) : gaussian_shape(t, r, theta);
}

double hor_rho(const hor_torus* t, double r, double theta)
{   /* :261-272 */
    const double disk = t->rho0 * disk_shape(t, r, theta) * funnel_factor(t, theta);
    const double raw = disk + envelope_rho(t, r);
    return smax(raw, t->rho_floor);
}

/* ---------------- UHE sources and spectra -------------------------------- */

static double spectral_weight(const hadros_params* p, double E)
{   /* radiative_transfer.cpp:172-207 */
    if (E <= 0.0) return 0.0;
    const double safe_E = smax(E, 1.0e-300);
    if (p->spectral_kind == HADROS_SPECTRAL_MONOCHROMATIC) {
        if (p->src_emax_GeV <= 0.0) return 0.0;
        return pow(safe_E, -p->src_powerlaw) * exp(-safe_E / p->src_emax_GeV);
    }
    if (p->spectral_kind == HADROS_SPECTRAL_POWERLAW) return pow(safe_E, -p->spec_gamma);
    if (p->spectral_kind == HADROS_SPECTRAL_POWERLAW_CUTOFF) {
        if (p->spec_ecut_GeV <= 0.0) return 0.0;
        return pow(safe_E, -p->spec_gamma) * exp(-safe_E / p->spec_ecut_GeV);
    }
    return 0.0;
}

double hor_spectral_weight(const hadros_params* p, double E) { return spectral_weight(p, E); }

static double bipolar_gaussian(double theta, double theta0, double width)
{   /* radiative_transfer.cpp:64-76 */
    if (width <= 0.0) return 0.0;
    const double north = theta - theta0;
    const double south = theta - (PI - theta0);
    return exp(-(north / width) * (north / width)) + exp(-(south / width) * (south / width));
}

/* uhe_source_spatial_weight, radiative_transfer.cpp:209-332 (not InnerRing). */
static double source_spatial_weight(const hadros_params* p, const hor_torus* t,
                                    double rho_norm, double r, double theta, double rho_here)
{
    if (r <= 0.0 || p->src_sigma_r_rg <= 0.0 || p->src_theta_width_rad <= 0.0) return 0.0;
    switch (p->source_kind) {
    case HADROS_SOURCE_INNER_RING: {
        const double delta_r = (r - p->src_r_center_rg) / p->src_sigma_r_rg;
        const double delta_theta = (theta - 0.5 * PI) / p->src_theta_width_rad;
        return exp(-delta_r * delta_r) * exp(-delta_theta * delta_theta);
    }
    case HADROS_SOURCE_FUNNEL_WALL: {
        const double delta_r = (r - p->src_r_center_rg) / p->src_sigma_r_rg;
        return exp(-delta_r * delta_r) *
               bipolar_gaussian(theta, p->src_funnel_theta_rad, p->src_theta_width_rad);
    }
    case HADROS_SOURCE_JET_BASE: {
        const double radial = exp(-pow(r / p->src_r_center_rg, 2.0));
        const double polar = bipolar_gaussian(theta, 0.0, p->src_theta_width_rad);
        return radial * polar;
    }
    case HADROS_SOURCE_DENSITY_WEIGHTED: {
        const double density_weight = pow(smax(rho_here / rho_norm, 0.0), p->src_density_power_q);
        const double radial_weight =
            pow(smax(r / smax(p->src_r_center_rg, 1.0e-300), 1.0e-300), -p->src_radial_power_s);
        return sclamp(density_weight * radial_weight, smax(p->src_cutoff_min, 0.0),
                      smax(p->src_cutoff_max, smax(p->src_cutoff_min, 0.0)));
    }
    case HADROS_SOURCE_SHOCK_LAYER: {
        const double dr = smax(p->src_gradient_dr_rg, 1.0e-4);
        const double dtheta = smax(p->src_gradient_dtheta_rad, 1.0e-5);
        const double r_minus = smax(r - dr, 1.0e-6);
        const double theta_minus = sclamp(theta - dtheta, 0.0, PI);
        const double theta_plus = sclamp(theta + dtheta, 0.0, PI);
        const double rho_r_plus = hor_rho(t, r + dr, theta);
        const double rho_r_minus = hor_rho(t, r_minus, theta);
        const double rho_t_plus = hor_rho(t, r, theta_plus);
        const double rho_t_minus = hor_rho(t, r, theta_minus);
        const double d_r = (rho_r_plus - rho_r_minus) / (2.0 * dr);
        const double d_theta = (rho_t_plus - rho_t_minus) / (2.0 * dtheta * smax(r, 1.0e-6));
        const double gradient = sqrt(d_r * d_r + d_theta * d_theta) / rho_norm;
        const double radial_taper = exp(-pow(r / smax(p->src_r_center_rg, 1.0e-300), 2.0));
        return sclamp(gradient * radial_taper, smax(p->src_cutoff_min, 0.0),
                      smax(p->src_cutoff_max, smax(p->src_cutoff_min, 0.0)));
    }
    default:
        return 0.0;
    }
}

/* Norm of the density-weighted and shock-layer sources (:255-264, :297-298):
 * rho_ref if positive (density_weighted only), else rho(r_center, pi/2). */
static double source_rho_norm(const hadros_params* p, const hor_torus* t)
{
    if (p->source_kind == HADROS_SOURCE_DENSITY_WEIGHTED)
        return smax(p->src_rho_ref_gcm3 > 0.0 ? p->src_rho_ref_gcm3
                                              : hor_rho(t, p->src_r_center_rg, 0.5 * PI),
                    1.0e-300);
    return smax(hor_rho(t, p->src_r_center_rg, 0.5 * PI), 1.0e-300);
}

/* Bin-independent factor of the emissivity at a point: j = C * w(E_local).
 * InnerRing: emissivity_collapsar_ring (:335-367) = (norm*radial)*vertical;
 * others: emissivity_uhe (:369-395) = norm * S(r, theta). */
static double emissivity_factor(const hadros_params* p, const hor_torus* t, double rho_norm,
                                double r, double theta, double rho_here)
{
    if (p->source_kind == HADROS_SOURCE_INNER_RING) {
        if (p->src_r_center_rg <= 0.0 || p->src_sigma_r_rg <= 0.0 ||
            p->src_theta_width_rad <= 0.0 || p->src_emax_GeV <= 0.0)
            return 0.0;
        const double delta_r = (r - p->src_r_center_rg) / p->src_sigma_r_rg;
        const double delta_theta = (theta - 0.5 * PI) / p->src_theta_width_rad;
        const double radial_profile = exp(-delta_r * delta_r);
        const double vertical_profile = exp(-delta_theta * delta_theta);
        return p->src_norm * radial_profile * vertical_profile;
    }
    return p->src_norm * source_spatial_weight(p, t, rho_norm, r, theta, rho_here);
}

/* ---------------- spectral bins (radiative_transfer.cpp:711-737) --------- */

int hor_spectral_bins(const hadros_params* p, double sig_Emin, double sig_Emax,
                      double* E_mid, double* dE, double* w, int8_t* valid)
{
    if (p->spectral_kind == HADROS_SPECTRAL_MONOCHROMATIC) {
        E_mid[0] = p->Enu_obs_GeV; dE[0] = 1.0; w[0] = 1.0; valid[0] = 1;
        return 1;
    }
    const int n_bins = p->n_bins > 1 ? p->n_bins : 1;
    const double e_min = smax(p->spec_e_min_GeV, sig_Emin);
    const double e_max = smin(p->spec_e_max_GeV, sig_Emax);
    if (e_min <= 0.0 || e_max <= e_min) {
        for (int b = 0; b < n_bins; ++b) { E_mid[b] = 0.0; dE[b] = 0.0; w[b] = 0.0; valid[b] = 0; }
        return n_bins;
    }
    const double log_min = log(e_min);
    const double log_max = log(e_max);
    const double dlog = (log_max - log_min) / (double)n_bins;
    for (int b = 0; b < n_bins; ++b) {
        const double log_left = log_min + dlog * (double)b;
        const double log_right = log_left + dlog;
        E_mid[b] = exp(0.5 * (log_left + log_right));
        dE[b] = exp(log_right) - exp(log_left);
        w[b] = spectral_weight(p, E_mid[b]) * dE[b];
        valid[b] = (w[b] <= 0.0 || !isfinite(w[b])) ? 0 : 1;
    }
    return n_bins;
}

/* ---------------- MeV thermal channel ------------------------------------
 * mev_neutrino_physics.cpp with the MeVThermalParams of hadros_params
 * (mev_* fields; switches as HADROS_MEV_* bits). */

#define HOR_HBAR_C_MEV_CM 1.973269804e-11   /* mev_neutrino_physics.cpp:14 */
#define HOR_M_E_MEV 0.510998950             /* :15 */
#define HOR_SIGMA_SCAT_E0 3.4e-45           /* MeVPhysicsParams default (mev_neutrino_physics.hpp:61) */

static int mev_flag(const hadros_params* p, unsigned bit) { return (p->mev_flags & bit) != 0u; }
static double mev_clamp_ye(double Ye) { return sclamp(Ye, 0.0, 1.0); }          /* :17-20 */
static double mev_safe_pow(double x, double e) { return pow(smax(x, 0.0), e); }   /* :22-25 */
static double mev_density_shape(double rho, double rho0)                        /* :27-35 */
{
    return sclamp(rho / smax(rho0, 1.0e-300), 0.0, 1.0);
}

static double mev_temperature(const hadros_params* p, const hor_torus* t, double r, double th, double rho)
{   /* mev_temperature_profile_MeV, :240-273 */
    const double T0 = smax(p->mev_T0_MeV, 1.0e-12);
    const double fl = smax(p->mev_T_floor_MeV, 1.0e-12);
    const double shape = mev_density_shape(rho, t->rho0);
    const double radial = pow(smax(r / smax(t->r0, 1.0e-300), 1.0e-300), -p->mev_T_power);
    const double equatorial = exp(-pow((th - 0.5 * PI) / 0.45, 2.0));
    const int outside_torus = r > t->r_max || r < t->r_min;
    double T = T0;
    switch (p->mev_thermal_profile) {
    case HADROS_MEV_T_INNER_HOT_TORUS:
        T = fl + T0 * pow(shape, smax(p->mev_T_power, 0.0));
        break;
    case HADROS_MEV_T_RADIAL_POWERLAW:
        T = fl + T0 * radial * (0.35 + 0.65 * equatorial);
        break;
    case HADROS_MEV_T_TORUS_PLUS_COOL_ENVELOPE:
        T = fl + T0 * pow(shape, smax(p->mev_T_power, 0.0));
        if (outside_torus || shape < 1.0e-3) T = fl + 0.15 * T0 * radial;
        break;
    case HADROS_MEV_T_COLLAPSAR_INNER_HOT: {
        const double inner_hot = exp(-pow((r - t->r_min) / smax(1.15 * t->r0, 1.0e-6), 2.0));
        const double radial_cooling = pow(1.0 + smax(r - t->r_min, 0.0) / smax(t->r0, 1.0e-6), -0.75);
        T = fl + T0 * (0.30 + 0.70 * pow(shape, 0.18)) * (0.45 + 0.55 * equatorial) *
                 (0.55 + 0.45 * inner_hot) * radial_cooling;
        break;
    }
    default:
        T = T0;
    }
    return smax(T, fl);
}

static double mev_ye(const hadros_params* p, const hor_torus* t, double r, double th, double rho)
{   /* mev_ye_profile, :275-318 */
    const double shape = mev_density_shape(rho, t->rho0);
    const double polar = exp(-pow(th / 0.35, 2.0)) + exp(-pow((PI - th) / 0.35, 2.0));
    const int envelope_like = r > t->r0 && (r > t->r_max || shape < 1.0e-2);
    double Ye = p->mev_Ye_torus;
    switch (p->mev_ye_profile) {
    case HADROS_MEV_YE_NEUTRON_RICH_TORUS:
        Ye = p->mev_Ye_torus + 0.05 * exp(-pow((r - t->r0) / 4.0, 2.0));
        break;
    case HADROS_MEV_YE_FUNNEL_PROTON_RICH:
        Ye = p->mev_Ye_torus * (1.0 - sclamp(polar, 0.0, 1.0)) + p->mev_Ye_funnel * sclamp(polar, 0.0, 1.0);
        break;
    case HADROS_MEV_YE_TORUS_ENVELOPE_CONTRAST:
        Ye = envelope_like ? p->mev_Ye_envelope : p->mev_Ye_torus;
        if (r < t->r_min && shape < 1.0e-2) Ye = p->mev_Ye_funnel;
        break;
    case HADROS_MEV_YE_COLLAPSAR_NEUTRON_RICH: {
        const double polar_weight = sclamp(polar, 0.0, 1.0);
        const double dense_weight = pow(shape, 0.25);
        const double radial_neutronization = exp(-pow((r - t->r0) / smax(1.2 * t->r0, 1.0e-6), 2.0));
        const double torus_ye = p->mev_Ye_torus - 0.05 * dense_weight * radial_neutronization;
        Ye = torus_ye * (1.0 - polar_weight) + p->mev_Ye_funnel * polar_weight;
        break;
    }
    default:
        Ye = p->mev_Ye_torus;
    }
    return sclamp(Ye, smax(p->mev_Ye_floor, 1.0e-6), smin(p->mev_Ye_ceil, 1.0 - 1.0e-6));
}

static double mev_thermal_shape(double E, double T)
{   /* mev_thermal_spectral_shape, :320-340 */
    if (E <= 0.0 || T <= 0.0) return 0.0;
    const double x = E / T;
    if (x > 120.0) return 0.0;
    const double T3 = smax(T * T * T, 1.0e-300);
    return E * E / (exp(x) + 1.0) / T3;
}

static double mev_fd_weight(double E, double T)
{   /* mev_fermi_dirac_weight, :342-354 */
    if (E <= 0.0 || T <= 0.0) return 0.0;
    const double x = E / T;
    if (x > 120.0) return 0.0;
    return E * E / (exp(x) + 1.0);
}

static double mev_electron_density(double rho, double Ye)
{   /* electron_number_density_cm3, :356-366 */
    if (rho <= 0.0) return 0.0;
    return rho * mev_clamp_ye(Ye) / HOR_M_U_G;
}

static double mev_degeneracy_correction(double rho, double Ye, double T, int flavor)
{   /* mev_urca_degeneracy_correction with electron_degeneracy_eta and the
     * zero-temperature chemical potential, :368-432 */
    if (flavor == HADROS_MEV_NU_X) return 1.0;
    double eta = 0.0;
    if (T > 0.0) {
        const double ne = mev_electron_density(rho, Ye);
        const double pF = ne <= 0.0 ? 0.0 : HOR_HBAR_C_MEV_CM * cbrt(3.0 * PI * PI * ne);
        eta = sqrt(pF * pF + HOR_M_E_MEV * HOR_M_E_MEV) / T;
    }
    if (!isfinite(eta)) return 1.0;
    const double shift = 0.25 * tanh((eta - 1.0) / 4.0);
    const double factor = flavor == HADROS_MEV_NU_E ? (1.0 + shift) : (1.0 - shift);
    return sclamp(factor, 0.5, 1.5);
}

static double mev_emissivity(const hadros_params* p, double rho, double T, double Ye, double E)
{   /* mev_total_emissivity with the URCA, pair and bremsstrahlung terms, :434-588 */
    const int flavor = p->mev_flavor;
    if (p->mev_model == HADROS_MEV_TOY) {
        if (rho <= 0.0 || T <= 0.0 || E <= 0.0) return 0.0;
        const double nb = rho / HOR_M_U_G;
        const double neutron_fraction = sclamp(1.0 - Ye, 0.0, 1.0);
        const double proton_fraction = sclamp(Ye, 0.0, 1.0);
        const double charged_current_weight = neutron_fraction + 0.5 * proton_fraction;
        const double thermal_spectrum = E * E / (exp(smin(E / T, 120.0)) + 1.0);
        const double capture_like = nb * charged_current_weight * pow(T, 6.0);
        const double pair_like = 0.05 * nb * pow(T, 9.0);
        return p->mev_norm * (capture_like + pair_like) * thermal_spectrum;
    }
    double total = 0.0;
    if (mev_flag(p, HADROS_MEV_URCA)) {
        double urca = 0.0;
        if (!(rho <= 0.0 || T <= 0.0 || E <= 0.0) && flavor != HADROS_MEV_NU_X) {
            const double ye = mev_clamp_ye(Ye);
            const double flavor_factor = flavor == HADROS_MEV_NU_E ? ye : (1.0 - ye);
            urca = 1.0e30 * mev_safe_pow(rho / 1.0e10, 1.0) * mev_safe_pow(T / 10.0, 6.0) * flavor_factor *
                   mev_thermal_shape(E, T);
        }
        if (mev_flag(p, HADROS_MEV_DEGENERACY_CORRECTION)) urca *= mev_degeneracy_correction(rho, Ye, T, flavor);
        total += urca;
    }
    if (mev_flag(p, HADROS_MEV_PAIR) && !(T <= 0.0 || E <= 0.0)) {
        const double flavor_factor = flavor == HADROS_MEV_NU_X ? 1.0 : 0.7;
        total += 3.0e28 * mev_safe_pow(T / 10.0, 9.0) * flavor_factor * mev_thermal_shape(E, T);
    }
    if (mev_flag(p, HADROS_MEV_BREMS) && !(rho <= 0.0 || T <= 0.0 || E <= 0.0)) {
        const double flavor_factor = flavor == HADROS_MEV_NU_X ? 1.0 : 0.8;
        total += 1.0e27 * mev_safe_pow(rho / 1.0e10, 2.0) * mev_safe_pow(T / 10.0, 5.0) * flavor_factor *
                 mev_thermal_shape(E, T);
    }
    return p->mev_norm * total;
}

static double mev_opacity(const hadros_params* p, double rho, double Ye, double E)
{   /* mev_total_opacity_cm_inv = absorption + scattering, :590-770 */
    const int absorb = mev_flag(p, HADROS_MEV_ABSORPTION), scatter = mev_flag(p, HADROS_MEV_SCATTERING);
    const double nb = rho / HOR_M_U_G;
    double ka = 0.0, ks = 0.0;
    if (p->mev_model == HADROS_MEV_TOY) {
        if (absorb && !(rho <= 0.0 || E <= 0.0)) {
            const double target_fraction = sclamp(1.0 - Ye, 0.0, 1.0) + 0.25 * sclamp(Ye, 0.0, 1.0);
            ka = nb * p->mev_sigma_abs0_cm2 * E * E * target_fraction;
        }
        if (scatter && !(rho <= 0.0 || E <= 0.0)) {
            const double composition_factor = 1.0 + 0.5 * sclamp(Ye, 0.0, 1.0);
            ks = nb * p->mev_sigma_scat0_cm2 * E * E * composition_factor;
        }
        return ka + ks;
    }
    const int dense = !(rho <= 0.0 || E <= 0.0);
    double abs_n = 0.0, abs_p = 0.0, scat_n = 0.0, scat_p = 0.0, scat_e = 0.0;
    if (dense && absorb && mev_flag(p, HADROS_MEV_ABS_N) && p->mev_flavor == HADROS_MEV_NU_E)
        abs_n = nb * (1.0 - mev_clamp_ye(Ye)) * p->mev_sigma_abs0_cm2 * E * E;
    if (dense && absorb && mev_flag(p, HADROS_MEV_ABS_P) && p->mev_flavor == HADROS_MEV_ANTI_NU_E)
        abs_p = nb * mev_clamp_ye(Ye) * p->mev_sigma_abs0_cm2 * E * E;
    if (dense && scatter && mev_flag(p, HADROS_MEV_SCAT_N))
        scat_n = nb * (1.0 - mev_clamp_ye(Ye)) * p->mev_sigma_scat0_cm2 * E * E;
    if (dense && scatter && mev_flag(p, HADROS_MEV_SCAT_P))
        scat_p = nb * mev_clamp_ye(Ye) * 0.5 * p->mev_sigma_scat0_cm2 * E * E;
    if (dense && scatter && mev_flag(p, HADROS_MEV_SCAT_E))
        scat_e = mev_electron_density(rho, Ye) * HOR_SIGMA_SCAT_E0 * E * E;
    return (abs_n + abs_p) + (scat_n + scat_p + scat_e);
}

/* MeV sums of one ray: tau, I, r_nu, leakage sum and weight. */
typedef struct { double tau, I, r_nu, leak_sum, leak_weight; } hor_mev_acc;

static void mev_point(const hadros_params* p, const hor_torus* t, hor_mev_acc* m, double r, double th,
                      double rho, double g, double dl_cm)
{   /* integrate_kerr_ray, radiative_transfer.cpp:507-607 */
    const double T = mev_temperature(p, t, r, th, rho);
    const double Ye = mev_ye(p, t, r, th, rho);
    double kappa = 0.0, j = 0.0;
    if (p->mev_spectral_mode == HADROS_MEV_FERMI_DIRAC_BAND) {
        const int n_bins = p->mev_n_bins > 1 ? p->mev_n_bins : 1;
        const double e_min = smax(p->mev_E_min_MeV, 1.0e-6);
        const double e_max = smax(p->mev_E_max_MeV, e_min);
        const double dE = (e_max - e_min) / (double)n_bins;
        double weight_sum = 0.0, kappa_weighted = 0.0;
        for (int ib = 0; ib < n_bins; ++ib) {
            const double E_mid = e_min + ((double)ib + 0.5) * dE;
            const double E_local = E_mid / smax(g, 1.0e-300);
            const double w = mev_fd_weight(E_local, T) * dE;
            if (w <= 0.0 || !isfinite(w)) continue;
            const double local_kappa = mev_opacity(p, rho, Ye, E_local);
            j += mev_emissivity(p, rho, T, Ye, E_local) * dE;
            kappa_weighted += w * local_kappa;
            weight_sum += w;
        }
        kappa = weight_sum > 0.0 ? kappa_weighted / weight_sum : 0.0;
    } else {
        const double E_local = p->mev_Enu_obs_MeV / smax(g, 1.0e-300);
        kappa = mev_opacity(p, rho, Ye, E_local);
        j = mev_emissivity(p, rho, T, Ye, E_local);
    }
    const double dtau = kappa * dl_cm;
    if (kappa > 0.0 && dtau > 1.0e-12) {
        const double attenuation = exp(-smin(dtau, 700.0));
        m->I = m->I * attenuation + pow(g, 3.0) * (j / kappa) * (1.0 - attenuation);
    } else {
        m->I += pow(g, 3.0) * j * dl_cm;
    }
    m->leak_sum += j * dl_cm;
    m->leak_weight += j * dl_cm;
    m->tau += dtau;
    if (m->r_nu < 0.0 && m->tau >= p->mev_neutrinosphere_tau) m->r_nu = r;
}

/* ---------------- one pixel, all bins ------------------------------------ */


int hor_trace_pixel(const hor_cam* cam, int i, int j,
                    double* tau_b, double* I_b, int32_t* steps_out, int32_t* attempts_out,
                    double* mev5, hor_point_cb cb, void* cb_user)
{
    hor_mev_acc mev = {0.0, 0.0, -1.0, 0.0, 0.0};
    const hadros_params* p = cam->p;
    const double a = p->a_spin;
    hor_state y, y_prev;
    hor_initial_state(p, i, j, &y);
    y_prev = y;
    const double energy_obs = zamo_energy(a, p->r_obs_rg, p->theta_obs_rad, y.pt, y.pphi);
    const int B = cam->n_bins;
    for (int b = 0; b < B; ++b) { tau_b[b] = 0.0; I_b[b] = 0.0; }

    int fate = HADROS_FATE_TRUNCATED;
    int step;
    long attempts = 0;
    for (step = 0; step < p->max_steps; ++step) {   /* kerr_camera.cpp:222 */
        if (y.r <= cam->r_stop) { fate = HADROS_FATE_CAPTURED; break; }
        if (y.r >= p->r_max_rg && step > 10) { fate = HADROS_FATE_ESCAPED; break; }

        /* PathPoint (:245-273) */
        const double pr_r = y.r, pr_th = y.theta;
        const double dl_rg = (step == 0) ? 0.0 : zamo_spatial_interval_rg(a, &y, &y_prev);
        const double redshift =
            zamo_energy(a, y.r, y.theta, y.pt, y.pphi) / smax(energy_obs, 1.0e-300);
        if (cb) cb(cb_user, pr_r, pr_th, y.phi, dl_rg, redshift);

        /* integrate_kerr_ray body for this point (radiative_transfer.cpp:501-672),
         * UHE terms only, for every bin. */
        if (!(pr_r < cam->rt_r_skip)) {
            const double g = 1.0 / smax(redshift, 1.0e-300);
            const double dl_cm = dl_rg * cam->rg_cm;
            const double rho = hor_rho(&cam->torus, pr_r, pr_th);
            if (mev5) mev_point(p, &cam->torus, &mev, pr_r, pr_th, rho, g, dl_cm);
            const double C = emissivity_factor(p, &cam->torus, cam->rho_norm, pr_r, pr_th, rho);
            const double g3 = pow(g, 3.0);
            for (int b = 0; b < B; ++b) {
                const double E_loc = cam->E_mid[b] / smax(g, 1.0e-300);
                double jj = 0.0;
                if (!(E_loc <= 0.0)) jj = C * spectral_weight(p, E_loc);
                I_b[b] += g3 * jj * exp(-tau_b[b]) * dl_cm;
                if (rho <= 0.0 || E_loc < cam->sigE[0] || E_loc > cam->sigE[cam->sig_n - 1])
                    continue;
                const double sigma_cm2 = hor_sigma_interp(cam->sigE, cam->sigS, cam->sig_n, E_loc);
                const double nb = rho / HOR_M_U_G;
                const double dtau = nb * sigma_cm2 * dl_cm;
                tau_b[b] += dtau;
            }
        }
        y_prev = y;
        attempts += hor_step_adaptive(a, p->h, p->tolerance, &y);
    }
    *steps_out = step;
    *attempts_out = (int32_t)(attempts > 2147483647L ? 2147483647L : attempts);
    if (mev5) {   /* radiative_transfer.cpp:673-679 */
        mev5[0] = mev.tau;
        mev5[1] = exp(-mev.tau);
        mev5[2] = mev.I;
        mev5[3] = mev.r_nu;
        mev5[4] = mev.leak_weight > 0.0 ? mev.leak_sum / mev.leak_weight : 1.0;
    }
    return fate;
}

int hor_cam_init(hor_cam* cam, const hadros_params* p, const double* sigE,
                 const double* sigS_cm2, int sig_n, const double* E_mid, int n_bins)
{
    memset(cam, 0, sizeof(*cam));
    cam->p = p;
    torus_resolve(p, &cam->torus);
    cam->rho_norm = source_rho_norm(p, &cam->torus);
    cam->sigE = sigE;
    cam->sigS = sigS_cm2;
    cam->sig_n = sig_n;
    cam->rg_cm = HOR_G_CGS * p->M_bh_msun * HOR_MSUN_G / (HOR_C_CGS * HOR_C_CGS);
    {
        const double a_bh = sclamp(p->a_spin, 0.0, 0.999999);
        const double r_h = 1.0 + sqrt(1.0 - a_bh * a_bh);
        cam->rt_r_skip = r_h + 1.0e-3;
    }
    cam->r_stop = (1.0 + sqrt(1.0 - p->a_spin * p->a_spin)) + 1.0e-3;
    cam->n_bins = n_bins;
    cam->E_mid = E_mid;
    return 0;
}

/* ---------------- whole image / pixel list ------------------------------- */

int hor_image(const hadros_params* p, const double* sigE, const double* sigS_cm2, int sig_n,
              const int32_t* pixel_ids, int32_t n_pixels,
              double* tau, double* P_surv, double* I_obs, int8_t* fate,
              int32_t* steps, int32_t* attempts, double* tau_E, double* I_E,
              double* tau_mev, double* P_surv_mev, double* I_obs_mev, double* r_nu, double* leakage,
              int n_threads)
{
    double* const mev_out[5] = {tau_mev, P_surv_mev, I_obs_mev, r_nu, leakage};
    const int want_mev = tau_mev || P_surv_mev || I_obs_mev || r_nu || leakage;
    double E_mid[HOR_MAX_BINS], dE[HOR_MAX_BINS], w[HOR_MAX_BINS];
    int8_t valid[HOR_MAX_BINS];
    if (p->n_bins > HOR_MAX_BINS) return -1;
    const int B = hor_spectral_bins(p, sigE[0], sigE[sig_n - 1], E_mid, dE, w, valid);
    const int mono = (p->spectral_kind == HADROS_SPECTRAL_MONOCHROMATIC);
    hor_cam cam;
    hor_cam_init(&cam, p, sigE, sigS_cm2, sig_n, E_mid, B);
    const long total = pixel_ids ? (long)n_pixels : (long)p->nx * (long)p->ny;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif

#pragma omp parallel for schedule(dynamic, 1)
    for (long k = 0; k < total; ++k) {
        const long pid = pixel_ids ? (long)pixel_ids[k] : k;
        const int i = (int)(pid % p->nx), j = (int)(pid / p->nx);
        double tb[HOR_MAX_BINS], ib[HOR_MAX_BINS];
        double m5[5] = {0.0, 1.0, 0.0, -1.0, 1.0};   /* RTResult defaults */
        int32_t st = 0, at = 0;
        const int f = hor_trace_pixel(&cam, i, j, tb, ib, &st, &at, want_mev ? m5 : NULL, NULL, NULL);
        /* the spectral aggregate keeps the first valid bin's MeV fields
         * (radiative_transfer.cpp:741-774); an empty ray keeps the defaults */
        int have_ref = mono;
        for (int b = 0; b < B && !have_ref; ++b) have_ref = valid[b];
        if (want_mev && (st == 0 || !have_ref)) {
            m5[0] = 0.0; m5[1] = 1.0; m5[2] = 0.0; m5[3] = -1.0; m5[4] = 1.0;
        }
        for (int c = 0; c < 5; ++c)
            if (mev_out[c]) mev_out[c][k] = m5[c];
        double t_out = 0.0, p_out = 1.0, i_out = 0.0;
        if (st > 0) {   /* compute_kerr_image_from_cache.cpp:617-633: empty rays keep defaults */
            if (mono) {
                t_out = tb[0]; p_out = exp(-tb[0]); i_out = ib[0];
            } else {   /* radiative_transfer.cpp:730-769 */
                double weight_sum = 0.0, tau_sum = 0.0, psurv_sum = 0.0, intensity_sum = 0.0;
                for (int b = 0; b < B; ++b) {
                    if (!valid[b]) continue;
                    weight_sum += w[b];
                    tau_sum += w[b] * tb[b];
                    psurv_sum += w[b] * exp(-tb[b]);
                    intensity_sum += ib[b] * dE[b];
                }
                if (weight_sum > 0.0) {
                    t_out = tau_sum / weight_sum;
                    p_out = psurv_sum / weight_sum;
                    i_out = intensity_sum;
                }
            }
        }
        if (tau) tau[k] = t_out;
        if (P_surv) P_surv[k] = p_out;
        if (I_obs) I_obs[k] = i_out;
        if (fate) fate[k] = (int8_t)f;
        if (steps) steps[k] = st;
        if (attempts) attempts[k] = at;
        for (int b = 0; b < B; ++b) {
            if (tau_E) tau_E[k * B + b] = tb[b];
            if (I_E) I_E[k * B + b] = ib[b];
        }
    }
    return B;
}

/* ---------------- ctypes-friendly helpers for tests ---------------------- */

void hor_inverse_metric5(double a, double r, double th, double* out5)
{
    hor_m5 g;
    hor_inverse_metric(a, r, th, &g);
    out5[0] = g.tt; out5[1] = g.tph; out5[2] = g.rr; out5[3] = g.thth; out5[4] = g.phph;
}

void hor_metric5(double a, double r, double th, double* out5)
{
    hor_m5 g;
    hor_metric(a, r, th, &g);
    out5[0] = g.tt; out5[1] = g.tph; out5[2] = g.rr; out5[3] = g.thth; out5[4] = g.phph;
}

double hor_rho_params(const hadros_params* p, double r, double theta)
{
    hor_torus t;
    torus_resolve(p, &t);
    return hor_rho(&t, r, theta);
}

int hor_rkf45_step(double a, double h0, double tol, double* s8)
{
    hor_state y = {s8[0], s8[1], s8[2], s8[3], s8[4], s8[5], s8[6], s8[7]};
    const int att = hor_step_adaptive(a, h0, tol, &y);
    s8[0] = y.t; s8[1] = y.r; s8[2] = y.theta; s8[3] = y.phi;
    s8[4] = y.pt; s8[5] = y.pr; s8[6] = y.ptheta; s8[7] = y.pphi;
    return att;
}

typedef struct { double* out; int cap; int n; } hor_pt_sink;

static void hor_pt_collect(void* user, double r, double theta, double phi, double dl, double z)
{
    hor_pt_sink* s = (hor_pt_sink*)user;
    if (s->n < s->cap) {
        double* o = s->out + 5 * (long)s->n;
        o[0] = r; o[1] = theta; o[2] = phi; o[3] = dl; o[4] = z;
    }
    s->n++;
}

int hor_trace_points(const hadros_params* p, const double* sigE, const double* sigS_cm2,
                     int sig_n, int i, int j, int max_points, double* out_points5,
                     int32_t* n_points, int32_t* fate)
{
    double E_mid[1] = {p->Enu_obs_GeV};
    double tb[1], ib[1];
    int32_t st = 0, at = 0;
    hadros_params q = *p;
    q.spectral_kind = HADROS_SPECTRAL_MONOCHROMATIC;
    hor_cam cam;
    hor_cam_init(&cam, &q, sigE, sigS_cm2, sig_n, E_mid, 1);
    hor_pt_sink sink = {out_points5, max_points, 0};
    *fate = hor_trace_pixel(&cam, i, j, tb, ib, &st, &at, NULL, hor_pt_collect, &sink);
    *n_points = st;
    return sink.n;
}
