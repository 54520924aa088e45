/*
 * dim_oracle.c — TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * Plain-C restatement of the reference DIM step of SegunOwoeye/
 * diffuse_vs_GFM_MMS.  Each function cites the reference lines it restates
 * (paths relative to the reference project root).  Operation order follows
 * the reference exactly; build with -ffp-contract=off and no -march so no FMA
 * contraction changes a rounding (the reference is built the same way).
 * std::max(a,b) is `(a < b) ? b : a` and std::min(a,b) is `(b < a) ? b : a`
 * in libstdc++; MAXD/MIND below keep those NaN / signed-zero semantics.
 *
 * The pressure recovery is the reference's literal doubling + bisection loop
 * (src/dim/eos.hpp:77-143), residual evaluation by residual evaluation.
 */
#include "dim_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXM DIMGPU_MAX_MATERIALS
#define MAXV (2 * MAXM + 3)

static __thread char g_err[256];

static void set_err(const char* m) { snprintf(g_err, sizeof g_err, "%s", m); }

const char* oracle_last_error(void) { return g_err; }

int oracle_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* ---- src/math/numerical_safety.hpp ------------------------------------- */
static inline double MAXD(double a, double b) { return (a < b) ? b : a; }
static inline double MIND(double a, double b) { return (b < a) ? b : a; }

/* numerical_safety.hpp:12-18 */
static inline double clamp_min_t(double x, double tol) { return isfinite(x) ? MAXD(x, tol) : tol; }
static inline double clamp_min(double x) { return clamp_min_t(x, 1e-10); }
/* numerical_safety.hpp:21-24 */
static inline double finite_or(double x, double fb) { return isfinite(x) ? x : fb; }
/* numerical_safety.hpp:27-39 */
static inline double safe_denom(double d, double tol)
{
    if (!isfinite(d)) return (d < 0.0) ? -tol : tol;
    if (fabs(d) < tol) return (d < 0.0) ? -tol : tol;
    return d;
}
/* numerical_safety.hpp:41-45 */
static inline double safe_div(double n, double d, double tol)
{
    return finite_or(n, 0.0) / safe_denom(d, tol);
}

/* ---- per-material laws, src/euler/eos.hpp ------------------------------- */
typedef struct {
    int dim, nmat;
    int kind[MAXM];
    double gamma[MAXM], p_inf[MAXM];
    int lambda;
    double asf;
} ctx_t;

static void make_ctx(const dimgpu_desc* d, ctx_t* c)
{
    memset(c, 0, sizeof *c);
    c->dim = d->dim;
    c->nmat = d->nmat;
    for (int k = 0; k < d->nmat; ++k) {
        c->kind[k] = d->mat[k].kind;
        c->gamma[k] = d->mat[k].gamma;
        c->p_inf[k] = d->mat[k].p_inf;
    }
    c->lambda = d->lambda_model;
    c->asf = d->alpha_source_floor;
}

static int validate(const dimgpu_desc* d)
{
    if (!d || d->dim < 1 || d->dim > 3) { set_err("bad dim"); return DIMGPU_E_INVALID_ARG; }
    if (d->nmat < 1 || d->nmat > MAXM) { set_err("bad nmat"); return DIMGPU_E_INVALID_ARG; }
    for (int k = 0; k < d->nmat; ++k) {
        if (d->mat[k].kind != DIMGPU_EOS_IDEAL_GAS && d->mat[k].kind != DIMGPU_EOS_STIFFENED_GAS) {
            set_err("oracle restates the ideal and stiffened-gas laws only");
            return DIMGPU_E_UNSUPPORTED_EOS;
        }
        if (!(d->mat[k].gamma > 1.0)) { set_err("dim::EOSParams: gamma must be > 1"); return DIMGPU_E_INVALID_ARG; }
    }
    return 0;
}

/* IdealGasEOS::internal_energy eos.hpp:488-495; StiffenedGasEOS eos.hpp:601-609 */
static inline double mat_internal_energy(const ctx_t* c, int k, double rho, double p)
{
    const double g = c->gamma[k];
    if (c->kind[k] == DIMGPU_EOS_STIFFENED_GAS)
        return safe_div((p + g * c->p_inf[k]), ((g - 1.0) * rho), 1e-10);
    return safe_div(p, ((g - 1.0) * rho), 1e-10);
}

/* pressure<1>(U) with U.mom = 0: IdealGasEOS::pressure eos.hpp:450-466,
 * StiffenedGasEOS::pressure eos.hpp:555-572. */
static inline double mat_pressure_rest(const ctx_t* c, int k, double Urho, double UE)
{
    const double g = c->gamma[k];
    const double rho = clamp_min(Urho);
    double mom2 = 0.0;
    mom2 += 0.0 * 0.0;
    const double kineticE = 0.5 * safe_div(mom2, rho, 1e-10);
    double p_raw;
    if (c->kind[k] == DIMGPU_EOS_STIFFENED_GAS)
        p_raw = (g - 1.0) * (UE - kineticE) - g * c->p_inf[k];
    else
        p_raw = (g - 1.0) * (UE - kineticE);
    return clamp_min(p_raw);
}

/* sound_speed<1>(U) with U.mom = 0: eos.hpp:469-479 (ideal), eos.hpp:575-585
 * (stiffened). */
static inline double mat_sound_speed_rest(const ctx_t* c, int k, double Urho, double UE)
{
    const double g = c->gamma[k];
    const double rho = clamp_min(Urho);
    const double p = mat_pressure_rest(c, k, Urho, UE);
    if (c->kind[k] == DIMGPU_EOS_STIFFENED_GAS)
        return sqrt(g * safe_div((p + c->p_inf[k]), rho, 1e-10));
    return sqrt(g * safe_div(p, rho, 1e-10));
}

/* ---- dim::MixtureEOS, src/dim/eos.hpp ----------------------------------- */
/* eos.hpp:16-27 */
static inline double material_pressure_from_density_energy(const ctx_t* c, int k, double rho, double e)
{
    const double Urho = clamp_min(rho);
    const double UE = Urho * MAXD(e, 0.0);
    return mat_pressure_rest(c, k, Urho, UE);
}

/* eos.hpp:29-40 */
static inline double material_sound_speed(const ctx_t* c, int k, double rho, double p)
{
    const double Urho = clamp_min(rho);
    const double UE = Urho * mat_internal_energy(c, k, Urho, p);
    return mat_sound_speed_rest(c, k, Urho, UE);
}

/* eos.hpp:42-57 */
static inline double material_energy_pressure_derivative(const ctx_t* c, int k, double rho, double p)
{
    rho = clamp_min(rho);
    p = clamp_min(p);
    const double dp = MAXD(1e-6 * MAXD(fabs(p), 1.0), 1e-8);
    const double p_lo = MAXD(p - dp, 1e-12);
    const double p_hi = p + dp;
    const double e_lo = mat_internal_energy(c, k, rho, p_lo);
    const double e_hi = mat_internal_energy(c, k, rho, p_hi);
    return MAXD(safe_div(e_hi - e_lo, p_hi - p_lo, 1e-14), 1e-14);
}

/* eos.hpp:59-75 */
static inline double mixture_internal_energy_density(const ctx_t* c, double p, const double* alpha,
                                                     const double* rho)
{
    double energy_density = 0.0;
    for (int k = 0; k < c->nmat; ++k) {
        const double alpha_k = MAXD(finite_or(alpha[k], 0.0), 0.0);
        const double rho_k = clamp_min(rho[k]);
        const double p_k = clamp_min(p);
        energy_density += alpha_k * rho_k * mat_internal_energy(c, k, rho_k, p_k);
    }
    return finite_or(energy_density, 0.0);
}

/* eos.hpp:77-143: literal doubling + bisection. */
static double pressure_from_internal_energy(const ctx_t* c, double rho_total, double e,
                                            const double* alpha, const double* rho)
{
    rho_total = clamp_min(rho_total);
    e = finite_or(e, 0.0);
    const double target = finite_or(rho_total * e, 0.0);
    double fallback_pressure = 0.0;
    for (int k = 0; k < c->nmat; ++k) {
        const double ek = target / rho_total;
        fallback_pressure += MAXD(finite_or(alpha[k], 0.0), 0.0) *
            material_pressure_from_density_energy(c, k, clamp_min(rho[k]), ek);
    }
    fallback_pressure = clamp_min(fallback_pressure);

    double lo = 1e-12;
    double hi = MAXD(1.0, fallback_pressure);

    double flo = mixture_internal_energy_density(c, lo, alpha, rho) - target;
    double fhi = mixture_internal_energy_density(c, hi, alpha, rho) - target;

    for (int n = 0; n < 80 && isfinite(fhi) && fhi < 0.0; ++n) {
        hi *= 2.0;
        fhi = mixture_internal_energy_density(c, hi, alpha, rho) - target;
    }

    if (!isfinite(flo) || !isfinite(fhi) || !(flo <= 0.0 && fhi >= 0.0))
        return clamp_min(fallback_pressure);

    for (int n = 0; n < 80; ++n) {
        const double mid = 0.5 * (lo + hi);
        const double fmid = mixture_internal_energy_density(c, mid, alpha, rho) - target;
        if (!isfinite(fmid)) return clamp_min(fallback_pressure);
        if (fabs(fmid) <= 1e-10 * MAXD(1.0, target)) return clamp_min(mid);
        if (fmid > 0.0) hi = mid;
        else lo = mid;
    }
    return clamp_min(0.5 * (lo + hi));
}

/* eos.hpp:195-221 */
static double mixture_sound_speed(const ctx_t* c, double rho_total, double p, const double* alpha,
                                  const double* rho)
{
    rho_total = clamp_min(rho_total);
    p = clamp_min(p);
    double beta_mix = 0.0;
    for (int k = 0; k < c->nmat; ++k) {
        const double rho_k = clamp_min(rho[k]);
        const double cs = material_sound_speed(c, k, rho_k, p);
        beta_mix += MAXD(finite_or(alpha[k], 0.0), 0.0) / safe_denom(rho_k * cs * cs, 1e-14);
    }
    return sqrt(1.0 / (rho_total * safe_denom(beta_mix, 1e-14)));
}

/* eos.hpp:223-275 */
static double generic_mixture_sound_speed(const ctx_t* c, double rho_total, double p,
                                          const double* alpha, const double* rho)
{
    if (c->lambda == DIMGPU_LAMBDA_KAPILA) return mixture_sound_speed(c, rho_total, p, alpha, rho);

    double sound_speed[MAXM], xi[MAXM];
    double xi_mix = 0.0, inverse_sound_sum = 0.0;
    for (int k = 0; k < c->nmat; ++k) {
        const double alpha_k = MAXD(finite_or(alpha[k], 0.0), 0.0);
        const double rho_k = clamp_min(rho[k]);
        sound_speed[k] = material_sound_speed(c, k, rho_k, p);
        xi[k] = rho_k * material_energy_pressure_derivative(c, k, rho_k, p);
        xi_mix += alpha_k * xi[k];
        inverse_sound_sum += alpha_k / safe_denom(sound_speed[k], 1e-14);
    }
    xi_mix = safe_denom(xi_mix, 1e-14);
    inverse_sound_sum = safe_denom(inverse_sound_sum, 1e-14);

    double rho_c_squared = 0.0;
    for (int k = 0; k < c->nmat; ++k) {
        const double alpha_k = MAXD(finite_or(alpha[k], 0.0), 0.0);
        double lambda_k = 1.0;
        if (c->lambda == DIMGPU_LAMBDA_EQUAL_VELOCITY)
            lambda_k = safe_div(1.0 / safe_denom(sound_speed[k], 1e-14), inverse_sound_sum, 1e-14);
        rho_c_squared += lambda_k * alpha_k * xi[k] * sound_speed[k] * sound_speed[k] / xi_mix;
    }
    return sqrt(MAXD(rho_c_squared / clamp_min(rho_total), 1e-14));
}

/* ---- src/dim/primitives.hpp --------------------------------------------- */
typedef struct {
    double m[MAXM];
    double mom[3];
    double E;
    double a[MAXM]; /* nmat-1 independent fractions */
} st_t;

typedef struct {
    double rho[MAXM];
    double alpha[MAXM];
    double vel[3];
    double p;
} pr_t;

typedef struct {
    double m[MAXM];
    double mom[3];
    double E;
} fl_t;

/* primitives.hpp:18-42 */
static void full_alpha(const ctx_t* c, const st_t* U, double* alpha)
{
    const int expected = (c->nmat > 1) ? (c->nmat - 1) : 0;
    double sum = 0.0;
    for (int k = 0; k < expected; ++k) {
        alpha[k] = U->a[k];
        sum += alpha[k];
    }
    alpha[c->nmat - 1] = 1.0 - sum;
}

/* primitives.hpp:45-70 */
static void sanitise_alpha(double* alpha, int n, double alpha_floor)
{
    double sum = 0.0;
    for (int k = 0; k < n; ++k) {
        alpha[k] = finite_or(alpha[k], alpha_floor);
        alpha[k] = MAXD(alpha[k], alpha_floor);
        sum += alpha[k];
    }
    if (!isfinite(sum) || sum <= 0.0) {
        for (int k = 0; k < n; ++k) alpha[k] = 0.0;
        alpha[0] = 1.0;
        return;
    }
    for (int k = 0; k < n; ++k) alpha[k] /= sum;
}

/* primitives.hpp:83-96 */
static void independent_alpha(const ctx_t* c, const double* alpha, st_t* U)
{
    for (int k = 0; k < c->nmat - 1; ++k) U->a[k] = alpha[k];
}

/* primitives.hpp:99-108 */
static double total_density(const ctx_t* c, const st_t* U)
{
    double r = 0.0;
    for (int k = 0; k < c->nmat; ++k) r += finite_or(U->m[k], 0.0);
    return r;
}

/* primitives.hpp:111-162 */
static void cons_to_prim(const ctx_t* c, const st_t* U, pr_t* P)
{
    const double rho_floor = 1e-12, p_floor = 1e-12, alpha_floor = 1e-12;
    memset(P, 0, sizeof *P);
    full_alpha(c, U, P->alpha);
    sanitise_alpha(P->alpha, c->nmat, alpha_floor);
    for (int k = 0; k < c->nmat; ++k) P->rho[k] = rho_floor;

    double rho_total = 0.0;
    for (int k = 0; k < c->nmat; ++k) rho_total += finite_or(U->m[k], 0.0);
    rho_total = MAXD(rho_total, rho_floor);

    double velocity_squared = 0.0;
    for (int d = 0; d < c->dim; ++d) {
        P->vel[d] = safe_div(U->mom[d], rho_total, 1e-10);
        velocity_squared += P->vel[d] * P->vel[d];
    }
    for (int k = 0; k < c->nmat; ++k) {
        const double alpha_k = MAXD(P->alpha[k], alpha_floor);
        P->rho[k] = MAXD(safe_div(finite_or(U->m[k], 0.0), alpha_k, 1e-10), rho_floor);
    }
    const double kinetic = 0.5 * rho_total * velocity_squared;
    const double internal_energy = safe_div(finite_or(U->E, kinetic) - kinetic, rho_total, 1e-10);
    P->p = MAXD(pressure_from_internal_energy(c, rho_total, internal_energy, P->alpha, P->rho), p_floor);
}

/* primitives.hpp:165-212 */
static void prim_to_cons(const ctx_t* c, const pr_t* P_in, st_t* U)
{
    const double rho_floor = 1e-12, p_floor = 1e-12, alpha_floor = 1e-12;
    pr_t P = *P_in;
    sanitise_alpha(P.alpha, c->nmat, alpha_floor);
    memset(U, 0, sizeof *U);

    double rho_total = 0.0;
    for (int k = 0; k < c->nmat; ++k) {
        P.rho[k] = MAXD(P.rho[k], rho_floor);
        U->m[k] = P.alpha[k] * P.rho[k];
        rho_total += U->m[k];
    }
    rho_total = MAXD(rho_total, rho_floor);
    P.p = MAXD(P.p, p_floor);

    double velocity_squared = 0.0;
    for (int d = 0; d < c->dim; ++d) {
        U->mom[d] = rho_total * P.vel[d];
        velocity_squared += P.vel[d] * P.vel[d];
    }
    /* MixtureEOS::internal_energy_from_pressure, eos.hpp:146-166 */
    const double rt = clamp_min(rho_total);
    const double pp = clamp_min(P.p);
    const double internal_energy = mixture_internal_energy_density(c, pp, P.alpha, P.rho) / rt;

    U->E = rho_total * internal_energy + 0.5 * rho_total * velocity_squared;
    independent_alpha(c, P.alpha, U);
}

/* primitives.hpp:216-322 */
static void alpha_rhs_coefficients(const ctx_t* c, const pr_t* P, double* rhs)
{
    const double floor_ = 1e-12;
    const double active_alpha_floor = c->asf;
    for (int k = 0; k < c->nmat; ++k) rhs[k] = P->alpha[k];
    sanitise_alpha(rhs, c->nmat, 0.0);

    if (c->lambda == DIMGPU_LAMBDA_ALLAIRE) return;

    if (c->lambda == DIMGPU_LAMBDA_EQUAL_VELOCITY) {
        double inverse_sound_sum = 0.0;
        double sound_speed[MAXM];
        for (int k = 0; k < c->nmat; ++k) sound_speed[k] = floor_;
        for (int k = 0; k < c->nmat; ++k) {
            const double alpha_k = MAXD(finite_or(rhs[k], 0.0), 0.0);
            if (alpha_k <= floor_ || alpha_k < MAXD(active_alpha_floor, 0.0)) continue;
            sound_speed[k] = material_sound_speed(c, k, MAXD(finite_or(P->rho[k], 0.0), floor_),
                                                  MAXD(finite_or(P->p, 0.0), floor_));
            inverse_sound_sum += alpha_k / safe_denom(sound_speed[k], 1e-14);
        }
        if (inverse_sound_sum <= floor_ || !isfinite(inverse_sound_sum)) return;
        for (int k = 0; k < c->nmat; ++k) {
            const double alpha_k = MAXD(finite_or(rhs[k], 0.0), 0.0);
            if (alpha_k <= floor_) { rhs[k] = 0.0; continue; }
            const double lambda_k = safe_div(1.0 / safe_denom(sound_speed[k], 1e-14), inverse_sound_sum, 1e-14);
            rhs[k] = alpha_k * lambda_k;
        }
        return;
    }

    const double source_alpha_floor = MAXD(active_alpha_floor, 0.0);
    double beta_mix = 0.0;
    double acoustic_impedance[MAXM];
    int active[MAXM];
    for (int k = 0; k < c->nmat; ++k) { acoustic_impedance[k] = floor_; active[k] = 0; }

    for (int k = 0; k < c->nmat; ++k) {
        const double alpha_k = MAXD(finite_or(rhs[k], 0.0), 0.0);
        if (alpha_k <= floor_ || alpha_k < source_alpha_floor) continue;
        active[k] = 1;
        const double rho_k = MAXD(finite_or(P->rho[k], 0.0), floor_);
        const double c_k = material_sound_speed(c, k, rho_k, MAXD(finite_or(P->p, 0.0), floor_));
        acoustic_impedance[k] = MAXD(rho_k * c_k * c_k, floor_);
        beta_mix += alpha_k / acoustic_impedance[k];
    }
    if (beta_mix <= floor_ || !isfinite(beta_mix)) return;

    const double q_mix = 1.0 / beta_mix;
    for (int k = 0; k < c->nmat; ++k) {
        const double alpha_k = MAXD(finite_or(rhs[k], 0.0), 0.0);
        if (!active[k] || alpha_k <= floor_) { rhs[k] = 0.0; continue; }
        const double K_k = alpha_k * (q_mix / acoustic_impedance[k] - 1.0);
        rhs[k] = alpha_k + K_k;
    }
}

/* primitives.hpp:325-457 */
static void repair_state(const ctx_t* c, st_t* U)
{
    const double mass_floor = 1e-12, p_floor = 1e-12, inactive_alpha_floor = 1e-10;
    const int nm = c->nmat, D = c->dim;

    for (int k = 0; k < nm; ++k) U->m[k] = MAXD(finite_or(U->m[k], 0.0), 0.0);
    for (int k = 0; k < nm - 1; ++k) U->a[k] = finite_or(U->a[k], 0.0);
    for (int d = 0; d < D; ++d) U->mom[d] = finite_or(U->mom[d], 0.0);
    U->E = finite_or(U->E, 0.0);

    const double rho_before = MAXD(total_density(c, U), mass_floor);
    double velocity_before[3] = {0.0, 0.0, 0.0};
    double velocity_squared_before = 0.0;
    for (int d = 0; d < D; ++d) {
        velocity_before[d] = safe_div(U->mom[d], rho_before, 1e-10);
        velocity_squared_before += velocity_before[d] * velocity_before[d];
    }

    double alpha_before[MAXM];
    full_alpha(c, U, alpha_before);
    sanitise_alpha(alpha_before, nm, 0.0);
    double rho_material_before[MAXM];
    for (int k = 0; k < nm; ++k) {
        const double alpha_k = MAXD(alpha_before[k], inactive_alpha_floor);
        rho_material_before[k] = MAXD(safe_div(MAXD(U->m[k], 0.0), alpha_k, 1e-10), mass_floor);
    }
    const double kinetic_before = 0.5 * rho_before * velocity_squared_before;
    const double internal_before = safe_div(finite_or(U->E, kinetic_before) - kinetic_before, rho_before, 1e-10);
    const double pressure_before = MAXD(
        pressure_from_internal_energy(c, rho_before, internal_before, alpha_before, rho_material_before),
        p_floor);

    for (int k = 0; k < nm; ++k) U->m[k] = MAXD(finite_or(U->m[k], 0.0), 0.0);

    double alpha_full[MAXM];
    full_alpha(c, U, alpha_full);
    sanitise_alpha(alpha_full, nm, 0.0);
    independent_alpha(c, alpha_full, U);

    int removed_inactive_mass = 0;
    for (int k = 0; k < nm; ++k) {
        if (alpha_full[k] <= inactive_alpha_floor && U->m[k] > mass_floor) {
            U->m[k] = 0.0;
            removed_inactive_mass = 1;
        }
    }

    double rho_total = total_density(c, U);
    if (!isfinite(rho_total) || rho_total <= 0.0) {
        int dominant = 0;
        for (int k = 1; k < nm; ++k)
            if (alpha_full[k] > alpha_full[dominant]) dominant = k;
        U->m[dominant] = mass_floor;
        rho_total = mass_floor;
    }

    if (removed_inactive_mass) {
        for (int d = 0; d < D; ++d) U->mom[d] = rho_total * velocity_before[d];
        double rho_material[MAXM];
        for (int k = 0; k < nm; ++k) {
            const double alpha_k = MAXD(alpha_full[k], inactive_alpha_floor);
            rho_material[k] = MAXD(safe_div(U->m[k], alpha_k, 1e-10), mass_floor);
        }
        const double rt = clamp_min(rho_total);
        const double pp = clamp_min(pressure_before);
        const double internal_energy = mixture_internal_energy_density(c, pp, alpha_full, rho_material) / rt;
        U->E = rho_total * internal_energy + 0.5 * rho_total * velocity_squared_before;
    }

    double velocity_squared = 0.0;
    for (int d = 0; d < D; ++d) {
        const double v = safe_div(U->mom[d], rho_total, 1e-10);
        velocity_squared += v * v; /* std::pow(v, 2) */
    }
    double rho_material[MAXM];
    for (int k = 0; k < nm; ++k) {
        const double alpha_k = MAXD(alpha_full[k], inactive_alpha_floor);
        rho_material[k] = MAXD(safe_div(U->m[k], alpha_k, 1e-10), mass_floor);
    }
    const double kinetic = 0.5 * rho_total * velocity_squared;
    const double minimum_internal = mixture_internal_energy_density(c, p_floor, alpha_full, rho_material);
    U->E = MAXD(finite_or(U->E, 0.0), kinetic + minimum_internal);
}

/* ---- src/dim/reconstruction/muscl.hpp ----------------------------------- */
/* src/core/fv/limiters.hpp:9-15 */
static inline double minmod(double a, double b)
{
    if (a * b <= 0.0) return 0.0;
    return fabs(a) < fabs(b) ? a : b;
}

/* muscl.hpp:26-40 */
static void enforce_positive_primitive(const ctx_t* c, pr_t* P)
{
    for (int k = 0; k < c->nmat; ++k) P->rho[k] = MAXD(P->rho[k], 1e-12);
    sanitise_alpha(P->alpha, c->nmat, 0.0);
    P->p = MAXD(P->p, 1e-12);
}

/* muscl.hpp:43-112 */
static void reconstruct_cell_faces(const ctx_t* c, const pr_t* PL, const pr_t* PC, const pr_t* PR,
                                   pr_t* Lf, pr_t* Rf)
{
    pr_t s;
    memset(&s, 0, sizeof s);
    for (int k = 0; k < c->nmat; ++k) s.rho[k] = minmod(PC->rho[k] - PL->rho[k], PR->rho[k] - PC->rho[k]);
    for (int k = 0; k < c->nmat; ++k) s.alpha[k] = minmod(PC->alpha[k] - PL->alpha[k], PR->alpha[k] - PC->alpha[k]);
    for (int d = 0; d < c->dim; ++d) s.vel[d] = minmod(PC->vel[d] - PL->vel[d], PR->vel[d] - PC->vel[d]);
    s.p = minmod(PC->p - PL->p, PR->p - PC->p);

    *Lf = *PC;
    *Rf = *PC;
    for (int k = 0; k < c->nmat; ++k) {
        Lf->rho[k] = PC->rho[k] - 0.5 * s.rho[k];
        Rf->rho[k] = PC->rho[k] + 0.5 * s.rho[k];
    }
    for (int k = 0; k < c->nmat; ++k) {
        Lf->alpha[k] = PC->alpha[k] - 0.5 * s.alpha[k];
        Rf->alpha[k] = PC->alpha[k] + 0.5 * s.alpha[k];
    }
    for (int d = 0; d < c->dim; ++d) {
        Lf->vel[d] = PC->vel[d] - 0.5 * s.vel[d];
        Rf->vel[d] = PC->vel[d] + 0.5 * s.vel[d];
    }
    Lf->p = PC->p - 0.5 * s.p;
    Rf->p = PC->p + 0.5 * s.p;
    enforce_positive_primitive(c, Lf);
    enforce_positive_primitive(c, Rf);
}

/* src/dim/flux.hpp:11-43 with an axis normal e_dir (norm 1, so n = e_dir). */
static void compute_flux_normal(const ctx_t* c, const st_t* U, const pr_t* P, int dir, fl_t* F)
{
    double n[3] = {0.0, 0.0, 0.0};
    n[dir] = 1.0;
    const double rho_total = total_density(c, U);
    double un = 0.0;
    for (int d = 0; d < c->dim; ++d) un += P->vel[d] * n[d];
    for (int k = 0; k < c->nmat; ++k) F->m[k] = U->m[k] * un;
    for (int d = 0; d < c->dim; ++d) F->mom[d] = rho_total * P->vel[d] * un + P->p * n[d];
    F->E = (U->E + P->p) * un;
}

/* muscl.hpp:115-140 */
static void apply_flux_difference(const ctx_t* c, const st_t* U, const fl_t* FL, const fl_t* FR,
                                  double factor, st_t* out)
{
    *out = *U;
    for (int k = 0; k < c->nmat; ++k) out->m[k] -= factor * (FR->m[k] - FL->m[k]);
    for (int d = 0; d < c->dim; ++d) out->mom[d] -= factor * (FR->mom[d] - FL->mom[d]);
    out->E -= factor * (FR->E - FL->E);
}

/* muscl.hpp:143-191 */
static void hancock_predict(const ctx_t* c, const st_t* Uc, const pr_t* Pc, const st_t* Ul,
                            const st_t* Ur, const pr_t* Pl, const pr_t* Pr, int dir, double dt,
                            double dx, st_t* out)
{
    fl_t FL, FR;
    compute_flux_normal(c, Ul, Pl, dir, &FL);
    compute_flux_normal(c, Ur, Pr, dir, &FR);
    const double factor = 0.5 * dt / dx;
    apply_flux_difference(c, Uc, &FL, &FR, factor, out);

    const double u_left = Pl->vel[dir];
    const double u_right = Pr->vel[dir];
    const double div_u = (u_right - u_left) / dx;
    double rhs[MAXM];
    alpha_rhs_coefficients(c, Pc, rhs);

    double alpha_new[MAXM];
    for (int k = 0; k < c->nmat; ++k) alpha_new[k] = Pc->alpha[k];
    for (int k = 0; k < c->nmat; ++k) {
        alpha_new[k] -= factor * (Pr->alpha[k] * u_right - Pl->alpha[k] * u_left);
        alpha_new[k] += 0.5 * dt * rhs[k] * div_u;
    }
    sanitise_alpha(alpha_new, c->nmat, 0.0);
    independent_alpha(c, alpha_new, out);
    repair_state(c, out);
}

/* muscl.hpp:197-329.  UL_face/UR_face have n-1 entries. */
static void reconstruct_line_interfaces(const ctx_t* c, int n, const st_t* U, int dir, double dt,
                                        double dx, st_t* UL_face, st_t* UR_face, pr_t* work_p,
                                        st_t* work_s)
{
    if (n < 3) {
        for (int f = 0; f < n - 1; ++f) {
            UL_face[f] = U[f];
            UR_face[f] = U[f + 1];
        }
        return;
    }
    pr_t* P_line = work_p;          /* n */
    pr_t* P_left = work_p + n;      /* n */
    pr_t* P_right = work_p + 2 * n; /* n */
    pr_t* P_half = work_p + 3 * n;  /* n */
    st_t* U_left = work_s;          /* n */
    st_t* U_right = work_s + n;
    st_t* U_half = work_s + 2 * n;
    st_t* U_left_half = work_s + 3 * n;
    st_t* U_right_half = work_s + 4 * n;

    for (int i = 0; i < n; ++i) {
        cons_to_prim(c, &U[i], &P_line[i]);
        enforce_positive_primitive(c, &P_line[i]);
    }
    P_left[0] = P_line[0];
    P_right[0] = P_line[0];
    U_left[0] = U[0];
    U_right[0] = U[0];
    P_left[n - 1] = P_line[n - 1];
    P_right[n - 1] = P_line[n - 1];
    U_left[n - 1] = U[n - 1];
    U_right[n - 1] = U[n - 1];

    for (int i = 1; i < n - 1; ++i) {
        reconstruct_cell_faces(c, &P_line[i - 1], &P_line[i], &P_line[i + 1], &P_left[i], &P_right[i]);
        prim_to_cons(c, &P_left[i], &U_left[i]);
        prim_to_cons(c, &P_right[i], &U_right[i]);
        repair_state(c, &U_left[i]);
        repair_state(c, &U_right[i]);
    }

    U_half[0] = U[0];
    U_half[n - 1] = U[n - 1];
    for (int i = 1; i < n - 1; ++i)
        hancock_predict(c, &U[i], &P_line[i], &U_left[i], &U_right[i], &P_left[i], &P_right[i], dir,
                        dt, dx, &U_half[i]);

    for (int i = 0; i < n; ++i) {
        cons_to_prim(c, &U_half[i], &P_half[i]);
        enforce_positive_primitive(c, &P_half[i]);
    }

    U_left_half[0] = U_half[0];
    U_right_half[0] = U_half[0];
    U_left_half[n - 1] = U_half[n - 1];
    U_right_half[n - 1] = U_half[n - 1];
    for (int i = 1; i < n - 1; ++i) {
        pr_t Lh, Rh;
        reconstruct_cell_faces(c, &P_half[i - 1], &P_half[i], &P_half[i + 1], &Lh, &Rh);
        prim_to_cons(c, &Lh, &U_left_half[i]);
        prim_to_cons(c, &Rh, &U_right_half[i]);
        repair_state(c, &U_left_half[i]);
        repair_state(c, &U_right_half[i]);
    }
    for (int f = 0; f < n - 1; ++f) {
        UL_face[f] = U_right_half[f];
        UR_face[f] = U_left_half[f + 1];
    }
}

/* ---- src/dim/riemann/hllc.hpp -------------------------------------------- */
/* hllc.hpp:15-24 */
static inline double star_density(double rho, double sK, double unK, double s_star)
{
    return rho * safe_div(sK - unK, sK - s_star, 1e-10);
}

/* hllc.hpp:27-41 */
static inline double star_energy(double rho_star, double E, double rho, double p, double sK,
                                 double unK, double s_star)
{
    return rho_star * (safe_div(E, rho, 1e-10) + (s_star - unK) * (s_star + safe_div(p, rho * (sK - unK), 1e-10)));
}

static void state_to_flux_diff(const ctx_t* c, const st_t* A, const st_t* B, fl_t* out)
{
    for (int k = 0; k < c->nmat; ++k) out->m[k] = A->m[k] - B->m[k];
    for (int d = 0; d < c->dim; ++d) out->mom[d] = A->mom[d] - B->mom[d];
    out->E = A->E - B->E;
}

/* hllc.hpp:47-59: (sR*FL - sL*FR + (sL*sR)*delta) / (sR - sL), where the
 * Flux division is a multiplication by 1.0/s (src/dim/conservative.hpp:81-88). */
static void hll_flux(const ctx_t* c, const st_t* UL, const st_t* UR, const fl_t* FL, const fl_t* FR,
                     double sL, double sR, fl_t* out)
{
    fl_t delta;
    state_to_flux_diff(c, UR, UL, &delta);
    const double inv = 1.0 / (sR - sL);
    const double sLsR = sL * sR;
    for (int k = 0; k < c->nmat; ++k) out->m[k] = inv * ((sR * FL->m[k] - sL * FR->m[k]) + sLsR * delta.m[k]);
    for (int d = 0; d < c->dim; ++d) out->mom[d] = inv * ((sR * FL->mom[d] - sL * FR->mom[d]) + sLsR * delta.mom[d]);
    out->E = inv * ((sR * FL->E - sL * FR->E) + sLsR * delta.E);
}

static void flux_avg(const ctx_t* c, const fl_t* A, const fl_t* B, fl_t* out)
{
    for (int k = 0; k < c->nmat; ++k) out->m[k] = 0.5 * (A->m[k] + B->m[k]);
    for (int d = 0; d < c->dim; ++d) out->mom[d] = 0.5 * (A->mom[d] + B->mom[d]);
    out->E = 0.5 * (A->E + B->E);
}

/* hllc.hpp:62-195.  Returns 0, or DIMGPU_E_NONFINITE where the reference's
 * require_positive throws (hllc.hpp:88-91). */
static int hllc_flux_normal(const ctx_t* c, const st_t* UL, const st_t* UR, int dir, fl_t* F, double* s_face)
{
    double n[3] = {0.0, 0.0, 0.0};
    n[dir] = 1.0;
    pr_t PL, PR;
    cons_to_prim(c, UL, &PL);
    cons_to_prim(c, UR, &PR);

    double rhoL = total_density(c, UL), rhoR = total_density(c, UR);
    double pL = PL.p, pR = PR.p;
    if (!isfinite(rhoL) || !isfinite(rhoR) || !isfinite(pL) || !isfinite(pR)) {
        set_err("dim::hllc_flux_normal: invalid density or pressure (non-finite)");
        return DIMGPU_E_NONFINITE;
    }
    if (rhoL <= 0.0) rhoL = 1e-10;
    if (rhoR <= 0.0) rhoR = 1e-10;
    if (pL <= 0.0) pL = 1e-10;
    if (pR <= 0.0) pR = 1e-10;

    double unL = 0.0, unR = 0.0;
    for (int d = 0; d < c->dim; ++d) unL += PL.vel[d] * n[d];
    for (int d = 0; d < c->dim; ++d) unR += PR.vel[d] * n[d];

    const double cL = generic_mixture_sound_speed(c, rhoL, pL, PL.alpha, PL.rho);
    const double cR = generic_mixture_sound_speed(c, rhoR, pR, PR.alpha, PR.rho);

    const double sL = MIND(unL - cL, unR - cR);
    const double sR = MAXD(unL + cL, unR + cR);

    const double numerator = (pR - pL) + rhoL * unL * (sL - unL) - rhoR * unR * (sR - unR);
    const double denom = rhoL * (sL - unL) - rhoR * (sR - unR);
    double s_star = safe_div(numerator, denom, 1e-10);
    if (fabs(pL - pR) < 1e-10 && fabs(unL - unR) < 1e-10) s_star = unL;

    fl_t FL, FR;
    compute_flux_normal(c, UL, &PL, dir, &FL);
    compute_flux_normal(c, UR, &PR, dir, &FR);

    if (!isfinite(sL) || !isfinite(sR) || !isfinite(s_star)) {
        flux_avg(c, &FL, &FR, F);
        *s_face = 0.5 * (unL + unR);
        return 0;
    }
    if (0.0 <= sL) { *F = FL; *s_face = unL; return 0; }
    if (sR <= 0.0) { *F = FR; *s_face = unR; return 0; }
    if (!(sL < sR)) {
        flux_avg(c, &FL, &FR, F);
        *s_face = 0.5 * (unL + unR);
        return 0;
    }

    const st_t* UK = (sL <= 0.0 && 0.0 <= s_star) ? UL : UR;
    const pr_t* PK = (UK == UL) ? &PL : &PR;
    const fl_t* FK = (UK == UL) ? &FL : &FR;
    const double rhoK = (UK == UL) ? rhoL : rhoR;
    const double pK = (UK == UL) ? pL : pR;
    const double unK = (UK == UL) ? unL : unR;
    const double sK = (UK == UL) ? sL : sR;

    const double rho_star = star_density(rhoK, sK, unK, s_star);
    const double E_star = star_energy(rho_star, UK->E, rhoK, pK, sK, unK, s_star);
    if (rho_star <= 0.0 || !isfinite(rho_star) || !isfinite(E_star)) {
        hll_flux(c, UL, UR, &FL, &FR, sL, sR, F);
        *s_face = s_star;
        return 0;
    }
    st_t Us;
    memset(&Us, 0, sizeof Us);
    const double mass_scale = safe_div(rho_star, rhoK, 1e-10);
    for (int k = 0; k < c->nmat; ++k) Us.m[k] = UK->m[k] * mass_scale;
    const double delta = s_star - unK;
    for (int d = 0; d < c->dim; ++d) {
        const double u_star = PK->vel[d] + delta * n[d];
        Us.mom[d] = rho_star * u_star;
    }
    Us.E = E_star;
    fl_t diff;
    state_to_flux_diff(c, &Us, UK, &diff);
    for (int k = 0; k < c->nmat; ++k) F->m[k] = FK->m[k] + sK * diff.m[k];
    for (int d = 0; d < c->dim; ++d) F->mom[d] = FK->mom[d] + sK * diff.mom[d];
    F->E = FK->E + sK * diff.E;
    *s_face = s_star;
    return 0;
}

/* ---- src/dim/conservative.hpp:116-141 ----------------------------------- */
static void conservative_update(const ctx_t* c, const st_t* U, const fl_t* Fl, const fl_t* Fr,
                                double lambda, st_t* out)
{
    *out = *U;
    for (int k = 0; k < c->nmat; ++k) out->m[k] -= lambda * (Fr->m[k] - Fl->m[k]);
    for (int d = 0; d < c->dim; ++d) out->mom[d] -= lambda * (Fr->mom[d] - Fl->mom[d]);
    out->E -= lambda * (Fr->E - Fl->E);
}

/* ---- src/dim/solver/advance/sweep_core.hpp:16-149 ---------------------- */
typedef struct {
    pr_t* p;  /* 4n primitives for the reconstruction + n for solve_line */
    st_t* s;  /* 5n states for the reconstruction + 2(n-1) faces         */
    fl_t* f;  /* n+1 fluxes */
    double* fv;
    pr_t* pf; /* 2(n-1) face primitives */
} line_work_t;

static int solve_line(const ctx_t* c, int n, const st_t* U_in, st_t* U_out, double dx, double dt,
                      int dir, line_work_t* w)
{
    if (n == 1) { U_out[0] = U_in[0]; return 0; }
    const int nm = c->nmat;
    const double lambda = dt / dx;
    pr_t* primitive = w->p + 4 * n;
    st_t* UL_face = w->s + 5 * n;
    st_t* UR_face = UL_face + (n - 1);
    pr_t* PL_face = w->pf;
    pr_t* PR_face = w->pf + (n - 1);
    fl_t* F = w->f;
    double* fv = w->fv;

    for (int i = 0; i < n; ++i) cons_to_prim(c, &U_in[i], &primitive[i]);

    reconstruct_line_interfaces(c, n, U_in, dir, dt, dx, UL_face, UR_face, w->p, w->s);

    for (int f = 0; f < n - 1; ++f) {
        cons_to_prim(c, &UL_face[f], &PL_face[f]);
        cons_to_prim(c, &UR_face[f], &PR_face[f]);
    }
    for (int i = 0; i < n - 1; ++i) {
        const int rc = hllc_flux_normal(c, &UL_face[i], &UR_face[i], dir, &F[i + 1], &fv[i + 1]);
        if (rc) return rc;
    }
    F[0] = F[1];
    F[n] = F[n - 1];
    fv[0] = fv[1];
    fv[n] = fv[n - 1];

    for (int i = 0; i < n; ++i) {
        conservative_update(c, &U_in[i], &F[i], &F[i + 1], lambda, &U_out[i]);
        repair_state(c, &U_out[i]);
    }

    /* alpha_flux[face][k] */
    for (int i = 0; i < n; ++i) {
        double flux_lo[MAXM], flux_hi[MAXM];
        for (int side = 0; side < 2; ++side) {
            const int face = i + side;
            double* out = side ? flux_hi : flux_lo;
            if (face == 0) {
                for (int k = 0; k < nm; ++k) out[k] = primitive[0].alpha[k] * fv[0];
            }
            else if (face == n) {
                for (int k = 0; k < nm; ++k) out[k] = primitive[n - 1].alpha[k] * fv[n];
            }
            else {
                const int iface = face - 1;
                const double* up = (fv[face] >= 0.0) ? PL_face[iface].alpha : PR_face[iface].alpha;
                for (int k = 0; k < nm; ++k) out[k] = up[k] * fv[face];
            }
        }
        double alpha_new[MAXM], rhs[MAXM];
        for (int k = 0; k < nm; ++k) alpha_new[k] = primitive[i].alpha[k];
        alpha_rhs_coefficients(c, &primitive[i], rhs);
        const double div_u = (fv[i + 1] - fv[i]) / dx;
        for (int k = 0; k < nm; ++k) {
            alpha_new[k] -= lambda * (flux_hi[k] - flux_lo[k]);
            alpha_new[k] += dt * rhs[k] * div_u;
        }
        sanitise_alpha(alpha_new, nm, 0.0);
        independent_alpha(c, alpha_new, &U_out[i]);
        repair_state(c, &U_out[i]);
    }
    return 0;
}

/* ---- field helpers --------------------------------------------------------- */
static size_t field_cells(const dimgpu_desc* d)
{
    size_t n = 1;
    for (int a = 0; a < d->dim; ++a) n *= (size_t)d->N[a];
    return n;
}

static void load_cell(const ctx_t* c, const double* soa, size_t stride, size_t i, st_t* U)
{
    int q = 0;
    memset(U, 0, sizeof *U);
    for (int k = 0; k < c->nmat; ++k) U->m[k] = soa[(size_t)(q++) * stride + i];
    for (int d = 0; d < c->dim; ++d) U->mom[d] = soa[(size_t)(q++) * stride + i];
    U->E = soa[(size_t)(q++) * stride + i];
    for (int k = 0; k < c->nmat - 1; ++k) U->a[k] = soa[(size_t)(q++) * stride + i];
}

static void store_cell(const ctx_t* c, double* soa, size_t stride, size_t i, const st_t* U)
{
    int q = 0;
    for (int k = 0; k < c->nmat; ++k) soa[(size_t)(q++) * stride + i] = U->m[k];
    for (int d = 0; d < c->dim; ++d) soa[(size_t)(q++) * stride + i] = U->mom[d];
    soa[(size_t)(q++) * stride + i] = U->E;
    for (int k = 0; k < c->nmat - 1; ++k) soa[(size_t)(q++) * stride + i] = U->a[k];
}

static void strides_of(const dimgpu_desc* d, size_t* stride)
{
    stride[0] = 1;
    for (int a = 1; a < 3; ++a) stride[a] = stride[a - 1] * (size_t)(a - 1 < d->dim ? d->N[a - 1] : 1);
}

/* sweep_core.hpp:151-202 with extract_line / write_line
 * (src/dim/solver/advance/line_ops.hpp:13-50). */
static int sweep_field(const dimgpu_desc* d, const ctx_t* c, int dir, double dt, const double* in,
                       double* out)
{
    const size_t total = field_cells(d);
    const int n = d->N[dir];
    const size_t lines = total / (size_t)n;
    size_t stride[3];
    strides_of(d, stride);
    int rc_all = 0;

#pragma omp parallel
    {
        st_t* lin = (st_t*)malloc(sizeof(st_t) * (size_t)n);
        st_t* lout = (st_t*)malloc(sizeof(st_t) * (size_t)n);
        line_work_t w;
        w.p = (pr_t*)malloc(sizeof(pr_t) * (size_t)(5 * n + 2));
        w.s = (st_t*)malloc(sizeof(st_t) * (size_t)(7 * n + 2));
        w.f = (fl_t*)malloc(sizeof(fl_t) * (size_t)(n + 1));
        w.fv = (double*)malloc(sizeof(double) * (size_t)(n + 1));
        w.pf = (pr_t*)malloc(sizeof(pr_t) * (size_t)(2 * n + 2));

#pragma omp for schedule(dynamic, 4)
        for (long long linear = 0; linear < (long long)lines; ++linear) {
            int idx[3] = {0, 0, 0};
            long long tmp = linear;
            for (int a = d->dim - 1; a >= 0; --a) {
                if (a == dir) continue;
                idx[a] = (int)(tmp % d->N[a]);
                tmp /= d->N[a];
            }
            size_t base = 0;
            for (int a = 0; a < d->dim; ++a) base += (size_t)idx[a] * stride[a];
            for (int i = 0; i < n; ++i) load_cell(c, in, total, base + (size_t)i * stride[dir], &lin[i]);
            const int rc = solve_line(c, n, lin, lout, d->dx[dir], dt, dir, &w);
            if (rc) {
#pragma omp atomic write
                rc_all = rc;
            }
            for (int i = 0; i < n; ++i) store_cell(c, out, total, base + (size_t)i * stride[dir], &lout[i]);
        }
        free(lin); free(lout); free(w.p); free(w.s); free(w.f); free(w.fv); free(w.pf);
    }
    return rc_all;
}

/* ---- src/dim/solver/cfl.hpp:16-119 -------------------------------------- */
static double cfl_field(const dimgpu_desc* d, const ctx_t* c, const double* soa, double cfl,
                        double dt_max, int unsplit)
{
    const size_t total = field_cells(d);
    double dt = dt_max;
#pragma omp parallel for reduction(min : dt) schedule(static)
    for (long long i = 0; i < (long long)total; ++i) {
        st_t U;
        pr_t P;
        load_cell(c, soa, total, (size_t)i, &U);
        cons_to_prim(c, &U, &P);
        const double cs = generic_mixture_sound_speed(c, total_density(c, &U), P.p, P.alpha, P.rho);
        if (unsplit) {
            double spectral_sum = 0.0;
            for (int a = 0; a < d->dim; ++a) spectral_sum += (fabs(P.vel[a]) + cs) / d->dx[a];
            if (spectral_sum > 1e-14) dt = MIND(dt, cfl / spectral_sum);
        }
        else {
            for (int a = 0; a < d->dim; ++a) {
                const double wave_speed = fabs(P.vel[a]) + cs;
                if (wave_speed > 1e-14) dt = MIND(dt, cfl * d->dx[a] / wave_speed);
            }
        }
    }
    return dt;
}

/* ---- src/dim/solver/advance/boundary.hpp -------------------------------- */
static void unflatten(const dimgpu_desc* d, size_t linear, int* idx)
{
    size_t s = 1;
    for (int a = 0; a < d->dim; ++a) {
        idx[a] = (int)((linear / s) % (size_t)d->N[a]);
        s *= (size_t)d->N[a];
    }
}

static size_t flatten(const dimgpu_desc* d, const int* idx)
{
    size_t stride[3];
    strides_of(d, stride);
    size_t l = 0;
    for (int a = 0; a < d->dim; ++a) l += (size_t)idx[a] * stride[a];
    return l;
}

/* boundary.hpp:113-163 */
static void nonreflective_state(const dimgpu_desc* d, const ctx_t* c, const double* soa, size_t total,
                                const int* idx, const int* src_idx, st_t* out)
{
    int second[3] = {src_idx[0], src_idx[1], src_idx[2]};
    for (int a = 0; a < d->dim; ++a) {
        if (idx[a] == 0 && d->N[a] > 2) second[a] = 2;
        else if (idx[a] == d->N[a] - 1 && d->N[a] > 2) second[a] = d->N[a] - 3;
    }
    st_t first, sec, state, ex;
    load_cell(c, soa, total, flatten(d, src_idx), &first);
    load_cell(c, soa, total, flatten(d, second), &sec);
    state = first;
    ex = first;
    for (int k = 0; k < c->nmat; ++k) ex.m[k] = first.m[k] + (first.m[k] - sec.m[k]);
    for (int a = 0; a < d->dim; ++a) ex.mom[a] = first.mom[a] + (first.mom[a] - sec.mom[a]);
    ex.E = first.E + (first.E - sec.E);
    for (int k = 0; k < c->nmat - 1; ++k) ex.a[k] = first.a[k] + (first.a[k] - sec.a[k]);

    int axis = 0;
    for (int a = 0; a < d->dim; ++a) {
        if (idx[a] == 0 || idx[a] == d->N[a] - 1) { axis = a; break; }
    }
    const int outward = (idx[axis] == 0) ? -1 : 1;
    const double ex_rho = MAXD(total_density(c, &ex), 1e-12);
    const double ex_un = outward * safe_div(ex.mom[axis], ex_rho, 1e-10);
    if (ex_un > 0.0) {
        const double rho = MAXD(total_density(c, &state), 1e-12);
        double b = 0.0, af = 0.0;
        for (int a = 0; a < d->dim; ++a) b += state.mom[a] * state.mom[a];
        state.mom[axis] = ex.mom[axis];
        for (int a = 0; a < d->dim; ++a) af += state.mom[a] * state.mom[a];
        state.E += 0.5 * (af - b) / rho;
    }
    repair_state(c, &state);
    *out = state;
}

/* boundary.hpp:165-226: serial, in place, x-fastest order. */
static void bc_field(const dimgpu_desc* d, const ctx_t* c, double* soa)
{
    const size_t total = field_cells(d);
    for (size_t linear = 0; linear < total; ++linear) {
        int idx[3] = {0, 0, 0}, src[3] = {0, 0, 0};
        unflatten(d, linear, idx);
        int is_boundary = 0;
        for (int a = 0; a < d->dim; ++a) {
            src[a] = idx[a];
            if (d->N[a] <= 1) continue;
            if (idx[a] == 0) { src[a] = 1; is_boundary = 1; }
            else if (idx[a] == d->N[a] - 1) { src[a] = d->N[a] - 2; is_boundary = 1; }
        }
        if (!is_boundary) continue;

        /* boundary_name_for_cell, boundary.hpp:23-41 */
        int bc = DIMGPU_BC_TRANSMISSIVE;
        for (int a = 0; a < d->dim; ++a) {
            if (idx[a] == 0) { bc = d->bc_lo[a]; break; }
            if (idx[a] == d->N[a] - 1) { bc = d->bc_hi[a]; break; }
        }
        st_t U;
        if (bc == DIMGPU_BC_NONREFLECTIVE) {
            nonreflective_state(d, c, soa, total, idx, src, &U);
            store_cell(c, soa, total, linear, &U);
            continue;
        }
        load_cell(c, soa, total, flatten(d, src), &U);
        for (int a = 0; a < d->dim; ++a) {
            if ((idx[a] == 0 && d->bc_lo[a] == DIMGPU_BC_REFLECTIVE) ||
                (idx[a] == d->N[a] - 1 && d->bc_hi[a] == DIMGPU_BC_REFLECTIVE))
                U.mom[a] *= -1.0;
        }
        store_cell(c, soa, total, linear, &U);
    }
}

/* ---- public entry points -------------------------------------------------- */
int oracle_compute_dt_cfl(const dimgpu_desc* d, const double* soa, double cfl, double dt_max,
                          double* dt_out)
{
    const int rc = validate(d);
    if (rc) return rc;
    if (!(cfl > 0.0) || !(dt_max > 0.0)) { set_err("cfl and dt_max must be positive"); return DIMGPU_E_INVALID_ARG; }
    ctx_t c;
    make_ctx(d, &c);
    *dt_out = cfl_field(d, &c, soa, cfl, dt_max, d->time_update == DIMGPU_TIME_UNSPLIT);
    return 0;
}

int oracle_sweep_direction(const dimgpu_desc* d, int dir, double dt, const double* in, double* out)
{
    const int rc = validate(d);
    if (rc) return rc;
    ctx_t c;
    make_ctx(d, &c);
    return sweep_field(d, &c, dir, dt, in, out);
}

int oracle_apply_boundary_conditions(const dimgpu_desc* d, double* soa)
{
    const int rc = validate(d);
    if (rc) return rc;
    ctx_t c;
    make_ctx(d, &c);
    bc_field(d, &c, soa);
    return 0;
}

/* src/dim/solver/advance_step.hpp:29-149 (split and unsplit). */
int oracle_advance(const dimgpu_desc* d, const double* soa_in, double* soa_out, double cfl,
                   double dt_max, int nsteps, double* dt_out)
{
    int rc = validate(d);
    if (rc) return rc;
    ctx_t c;
    make_ctx(d, &c);
    const size_t total = field_cells(d);
    const int V = 2 * d->nmat + d->dim;
    const size_t bytes = sizeof(double) * total * (size_t)V;
    double* cur = soa_out;
    double* a = (double*)malloc(bytes);
    double* b = (double*)malloc(bytes);
    memcpy(cur, soa_in, bytes);
    for (int s = 0; s < nsteps && !rc; ++s) {
        const int unsplit = d->time_update == DIMGPU_TIME_UNSPLIT;
        if (!(cfl > 0.0) || !(dt_max > 0.0)) { set_err("cfl and dt_max must be positive"); rc = DIMGPU_E_INVALID_ARG; break; }
        const double dt = cfl_field(d, &c, cur, cfl, dt_max, unsplit);
        if (dt_out) dt_out[s] = dt;
        if (!unsplit) {
            for (int dir = 0; dir < d->dim && !rc; ++dir) {
                rc = sweep_field(d, &c, dir, dt, cur, a);
                bc_field(d, &c, a);
                memcpy(cur, a, bytes);
            }
        }
        else {
            memcpy(b, cur, bytes); /* accumulated = base */
            for (int dir = 0; dir < d->dim && !rc; ++dir) {
                rc = sweep_field(d, &c, dir, dt, cur, a);
#pragma omp parallel for schedule(static)
                for (long long i = 0; i < (long long)total; ++i) {
                    st_t acc, di, ba;
                    load_cell(&c, b, total, (size_t)i, &acc);
                    load_cell(&c, a, total, (size_t)i, &di);
                    load_cell(&c, cur, total, (size_t)i, &ba);
                    for (int k = 0; k < c.nmat; ++k) acc.m[k] += di.m[k] - ba.m[k];
                    for (int q = 0; q < c.dim; ++q) acc.mom[q] += di.mom[q] - ba.mom[q];
                    acc.E += di.E - ba.E;
                    for (int k = 0; k < c.nmat - 1; ++k) acc.a[k] += di.a[k] - ba.a[k];
                    repair_state(&c, &acc);
                    store_cell(&c, b, total, (size_t)i, &acc);
                }
            }
            bc_field(d, &c, b);
            memcpy(cur, b, bytes);
        }
    }
    free(a);
    free(b);
    return rc;
}

/* compute_dim_conservation_totals, src/app/io/conservation_report.hpp:188-218:
 * out = {material_mass[nmat], mass, momentum[dim], energy}. */
int oracle_totals(const dimgpu_desc* d, const double* soa, double* out)
{
    const int rc = validate(d);
    if (rc) return rc;
    ctx_t c;
    make_ctx(d, &c);
    const size_t total = field_cells(d);
    double volume = 1.0;
    for (int a = 0; a < d->dim; ++a) volume *= d->dx[a];
    double mm[MAXM] = {0}, mass = 0.0, mom[3] = {0}, energy = 0.0;
    for (size_t i = 0; i < total; ++i) {
        st_t U;
        load_cell(&c, soa, total, i, &U);
        double cell_mass = 0.0;
        for (int k = 0; k < c.nmat; ++k) {
            const double partial = U.m[k] * volume;
            mm[k] += partial;
            cell_mass += partial;
        }
        mass += cell_mass;
        energy += U.E * volume;
        for (int a = 0; a < c.dim; ++a) mom[a] += U.mom[a] * volume;
    }
    int q = 0;
    for (int k = 0; k < c.nmat; ++k) out[q++] = mm[k];
    out[q++] = mass;
    for (int a = 0; a < c.dim; ++a) out[q++] = mom[a];
    out[q++] = energy;
    return 0;
}

/* ---- per-function record entry points ----------------------------------- */
static void load_rec(const ctx_t* c, const double* r, st_t* U) { load_cell(c, r, 1, 0, U); }
static void store_rec(const ctx_t* c, double* r, const st_t* U) { store_cell(c, r, 1, 0, U); }

static void store_prim(const ctx_t* c, double* o, const pr_t* P)
{
    int q = 0;
    for (int k = 0; k < c->nmat; ++k) o[q++] = P->rho[k];
    for (int k = 0; k < c->nmat; ++k) o[q++] = P->alpha[k];
    for (int a = 0; a < c->dim; ++a) o[q++] = P->vel[a];
    o[q++] = P->p;
}

static void load_prim(const ctx_t* c, const double* in, pr_t* P)
{
    int q = 0;
    memset(P, 0, sizeof *P);
    for (int k = 0; k < c->nmat; ++k) P->rho[k] = in[q++];
    for (int k = 0; k < c->nmat; ++k) P->alpha[k] = in[q++];
    for (int a = 0; a < c->dim; ++a) P->vel[a] = in[q++];
    P->p = in[q++];
}

/* compute_dim_boundary_flux + add_dim_flux_to_totals,
 * src/app/io/conservation_report.hpp:149-167, 253-305: per axis, per
 * transverse line (highest axis fastest), add area * F(right end cell), then
 * -area * F(left end cell), in that order. */
int oracle_boundary_flux(const dimgpu_desc* d, const double* soa, double* out)
{
    const int rc = validate(d);
    if (rc) return rc;
    ctx_t c;
    make_ctx(d, &c);
    const size_t total = field_cells(d);
    double mm[MAXM] = {0}, mass = 0.0, mom[3] = {0}, energy = 0.0;
    for (int dir = 0; dir < c.dim; ++dir) {
        double area = 1.0;
        for (int a = 0; a < c.dim; ++a)
            if (a != dir) area *= d->dx[a];
        long long lines = 1;
        for (int a = 0; a < c.dim; ++a)
            if (a != dir) lines *= d->N[a];
        for (long long line = 0; line < lines; ++line) {
            int idx[3] = {0, 0, 0};
            long long tmp = line;
            for (int a = c.dim - 1; a >= 0; --a) {
                if (a == dir) continue;
                idx[a] = (int)(tmp % d->N[a]);
                tmp /= d->N[a];
            }
            for (int side = 1; side >= 0; --side) {
                idx[dir] = side ? d->N[dir] - 1 : 0;
                size_t lin = (size_t)idx[0];
                size_t stride = (size_t)d->N[0];
                for (int a = 1; a < c.dim; ++a) {
                    lin += (size_t)idx[a] * stride;
                    stride *= (size_t)d->N[a];
                }
                st_t U;
                pr_t P;
                fl_t F;
                load_cell(&c, soa, total, lin, &U);
                cons_to_prim(&c, &U, &P);
                compute_flux_normal(&c, &U, &P, dir, &F);
                const double scale = side ? area : -area;
                double mass_flux = 0.0;
                for (int k = 0; k < c.nmat; ++k) {
                    const double v = scale * F.m[k];
                    mm[k] += v;
                    mass_flux += v;
                }
                mass += mass_flux;
                energy += scale * F.E;
                for (int a = 0; a < c.dim; ++a) mom[a] += scale * F.mom[a];
            }
        }
    }
    int q = 0;
    for (int k = 0; k < c.nmat; ++k) out[q++] = mm[k];
    out[q++] = mass;
    for (int a = 0; a < c.dim; ++a) out[q++] = mom[a];
    out[q++] = energy;
    return 0;
}

int oracle_cons_to_prim(const dimgpu_desc* d, int n, const double* U, double* P)
{
    const int rc = validate(d);
    if (rc) return rc;
    ctx_t c;
    make_ctx(d, &c);
    const int V = 2 * c.nmat + c.dim, PV = V + 1;
    for (int i = 0; i < n; ++i) {
        st_t s;
        pr_t p;
        load_rec(&c, U + (size_t)i * V, &s);
        cons_to_prim(&c, &s, &p);
        store_prim(&c, P + (size_t)i * PV, &p);
    }
    return 0;
}

int oracle_prim_to_cons(const dimgpu_desc* d, int n, const double* P, double* U)
{
    const int rc = validate(d);
    if (rc) return rc;
    ctx_t c;
    make_ctx(d, &c);
    const int V = 2 * c.nmat + c.dim, PV = V + 1;
    for (int i = 0; i < n; ++i) {
        st_t s;
        pr_t p;
        load_prim(&c, P + (size_t)i * PV, &p);
        prim_to_cons(&c, &p, &s);
        store_rec(&c, U + (size_t)i * V, &s);
    }
    return 0;
}

int oracle_repair_state(const dimgpu_desc* d, int n, double* U)
{
    const int rc = validate(d);
    if (rc) return rc;
    ctx_t c;
    make_ctx(d, &c);
    const int V = 2 * c.nmat + c.dim;
    for (int i = 0; i < n; ++i) {
        st_t s;
        load_rec(&c, U + (size_t)i * V, &s);
        repair_state(&c, &s);
        store_rec(&c, U + (size_t)i * V, &s);
    }
    return 0;
}

int oracle_mixture_pressure(const dimgpu_desc* d, int n, const double* in, double* p)
{
    const int rc = validate(d);
    if (rc) return rc;
    ctx_t c;
    make_ctx(d, &c);
    const int R = 2 + 2 * c.nmat;
    for (int i = 0; i < n; ++i) {
        const double* r = in + (size_t)i * R;
        p[i] = pressure_from_internal_energy(&c, r[0], r[1], r + 2, r + 2 + c.nmat);
    }
    return 0;
}

int oracle_mixture_sound_speed(const dimgpu_desc* d, int n, const double* in, double* cs)
{
    const int rc = validate(d);
    if (rc) return rc;
    ctx_t c;
    make_ctx(d, &c);
    const int R = 2 + 2 * c.nmat;
    for (int i = 0; i < n; ++i) {
        const double* r = in + (size_t)i * R;
        cs[i] = generic_mixture_sound_speed(&c, r[0], r[1], r + 2, r + 2 + c.nmat);
    }
    return 0;
}

int oracle_alpha_rhs(const dimgpu_desc* d, int n, const double* P, double* rhs)
{
    const int rc = validate(d);
    if (rc) return rc;
    ctx_t c;
    make_ctx(d, &c);
    const int PV = 2 * c.nmat + c.dim + 1;
    for (int i = 0; i < n; ++i) {
        pr_t p;
        load_prim(&c, P + (size_t)i * PV, &p);
        alpha_rhs_coefficients(&c, &p, rhs + (size_t)i * c.nmat);
    }
    return 0;
}

int oracle_hllc(const dimgpu_desc* d, int n, int dir, const double* UL, const double* UR, double* out)
{
    const int rc0 = validate(d);
    if (rc0) return rc0;
    ctx_t c;
    make_ctx(d, &c);
    const int V = 2 * c.nmat + c.dim, F = c.nmat + c.dim + 2;
    for (int i = 0; i < n; ++i) {
        st_t l, r;
        fl_t f;
        double s;
        load_rec(&c, UL + (size_t)i * V, &l);
        load_rec(&c, UR + (size_t)i * V, &r);
        const int rc = hllc_flux_normal(&c, &l, &r, dir, &f, &s);
        if (rc) return rc;
        double* o = out + (size_t)i * F;
        int q = 0;
        for (int k = 0; k < c.nmat; ++k) o[q++] = f.m[k];
        for (int a = 0; a < c.dim; ++a) o[q++] = f.mom[a];
        o[q++] = f.E;
        o[q++] = s;
    }
    return 0;
}

int oracle_solve_line(const dimgpu_desc* d, int n, int dir, double dt, double dx, const double* U_in,
                      double* U_out)
{
    const int rc0 = validate(d);
    if (rc0) return rc0;
    if (n < 1) { set_err("dim::solve_line: empty line"); return DIMGPU_E_INVALID_ARG; }
    ctx_t c;
    make_ctx(d, &c);
    const int V = 2 * c.nmat + c.dim;
    st_t* lin = (st_t*)malloc(sizeof(st_t) * (size_t)n);
    st_t* lout = (st_t*)malloc(sizeof(st_t) * (size_t)n);
    line_work_t w;
    w.p = (pr_t*)malloc(sizeof(pr_t) * (size_t)(5 * n + 2));
    w.s = (st_t*)malloc(sizeof(st_t) * (size_t)(7 * n + 2));
    w.f = (fl_t*)malloc(sizeof(fl_t) * (size_t)(n + 1));
    w.fv = (double*)malloc(sizeof(double) * (size_t)(n + 1));
    w.pf = (pr_t*)malloc(sizeof(pr_t) * (size_t)(2 * n + 2));
    for (int i = 0; i < n; ++i) load_rec(&c, U_in + (size_t)i * V, &lin[i]);
    const int rc = solve_line(&c, n, lin, lout, dx, dt, dir, &w);
    for (int i = 0; i < n; ++i) store_rec(&c, U_out + (size_t)i * V, &lout[i]);
    free(lin); free(lout); free(w.p); free(w.s); free(w.f); free(w.fv); free(w.pf);
    return rc;
}

/* dim::write_csv, src/io/dim_write_csv.hpp:15-125: header, then one row per
 * cell in linear order with the values std::ostream prints by default
 * ("%.6g"): cell centre (compute_cell_center, geometry.hpp:75-87, with
 * dx = (max - min) / N), total density, velocity, pressure, internal energy
 * max(safe_div(E - kinetic, rho), 0), fractions, material densities, masses. */
int oracle_write_csv(const dimgpu_desc* d, const double* soa, const double* domain_min,
                     const double* domain_max, const char* filename)
{
    const int rc0 = validate(d);
    if (rc0) return rc0;
    ctx_t c;
    make_ctx(d, &c);
    FILE* f = fopen(filename, "wb");
    if (!f) { set_err("dim::write_csv: failed to open file"); return DIMGPU_E_INVALID_ARG; }
    double dx[3];
    for (int a = 0; a < c.dim; ++a) dx[a] = (domain_max[a] - domain_min[a]) / (double)d->N[a];
    for (int a = 0; a < c.dim; ++a) fprintf(f, "x%d,", a);
    fprintf(f, "rho,");
    for (int a = 0; a < c.dim; ++a) fprintf(f, "u%d,", a);
    fprintf(f, "p,e");
    for (int k = 0; k < c.nmat; ++k) fprintf(f, ",alpha%d", k);
    for (int k = 0; k < c.nmat; ++k) fprintf(f, ",rho_mat%d", k);
    for (int k = 0; k < c.nmat; ++k) fprintf(f, ",mass%d", k);
    fprintf(f, "\n");
    const size_t n = field_cells(d);
    for (size_t i = 0; i < n; ++i) {
        st_t U;
        pr_t P;
        load_cell(&c, soa, n, i, &U);
        cons_to_prim(&c, &U, &P);
        const double rho = total_density(&c, &U);
        double v2 = 0.0;
        for (int a = 0; a < c.dim; ++a) v2 += P.vel[a] * P.vel[a];
        const double kinetic = 0.5 * rho * v2;
        const double ie = MAXD(safe_div(U.E - kinetic, rho, 1e-10), 0.0);
        size_t rem = i;
        for (int a = 0; a < c.dim; ++a) {
            const size_t idx = rem % (size_t)d->N[a];
            rem /= (size_t)d->N[a];
            fprintf(f, "%.6g,", domain_min[a] + ((double)idx + 0.5) * dx[a]);
        }
        fprintf(f, "%.6g,", rho);
        for (int a = 0; a < c.dim; ++a) fprintf(f, "%.6g,", P.vel[a]);
        fprintf(f, "%.6g,%.6g", P.p, ie);
        for (int k = 0; k < c.nmat; ++k) fprintf(f, ",%.6g", P.alpha[k]);
        for (int k = 0; k < c.nmat; ++k) fprintf(f, ",%.6g", P.rho[k]);
        for (int k = 0; k < c.nmat; ++k) fprintf(f, ",%.6g", U.m[k]);
        fprintf(f, "\n");
    }
    if (fclose(f) != 0) { set_err("dim::write_csv: failed to write file"); return DIMGPU_E_INVALID_ARG; }
    return 0;
}
