/*
 * euler_oracle.c — TEST INFRASTRUCTURE ONLY: a plain-C restatement of the
 * reference's single-material Euler step (the sharp-interface solver's
 * one-material, no-level-set fast path), used by tests/ as the checker of
 * the CUDA Euler path.  Never linked into the product.
 *
 * Follows, function by function (paths in SegunOwoeye/diffuse_vs_GFM_MMS):
 *   advance_one_step            src/sim/solver/advance_step.hpp:489-866
 *                               (phi_list empty, one material: CFL, split or
 *                               unsplit sweeps, boundary fill)
 *   advance_line fast path      src/sim/solver/advance/sweep_core.hpp:65-111
 *   reconstruct_line_interfaces src/euler/reconstruction/muscl.hpp:139-304
 *   enforce_positive_*          src/euler/reconstruction/muscl.hpp:24-48
 *   hancock_predict             src/euler/reconstruction/muscl.hpp:114-135
 *   hllc_flux_normal            src/euler/riemann/hllc.hpp:18-152
 *   compute_flux_normal         src/euler/flux.hpp:14-53
 *   compute_thermo              src/euler/thermo_compute.hpp:10-26
 *   cons_to_prim / prim_to_cons src/euler/conservative.hpp:12-50,
 *                               src/euler/primitives.hpp:7-34
 *   Ideal / StiffenedGasEOS     src/euler/eos.hpp:447-662 (MaterialEOS
 *                               dispatch :983-1116)
 *   compute_dt_cfl_materials    src/sim/solver/cfl.hpp:64-125 (unsplit
 *                               :128-187)
 *   apply_boundary_conditions   src/sim/solver/advance/boundary.hpp:149-201
 *                               (local_nonreflective_state :96-147)
 *   numerical safety helpers    src/math/numerical_safety.hpp:12-78
 *
 * State layout: SoA, component c of cell i at U[c * ncell + i], components
 * rho, mom[0..dim-1], E (Conserved<DIM> in declaration order).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dimgpu.h"
#include "euler_oracle.h"

#define MAXD 3

typedef struct { double rho, mom[MAXD], E; } EU;
typedef struct { double rho, vel[MAXD], p; } EP;

typedef struct {
    int dim, stiff;
    double gamma, p_inf;
} Mat;

static int g_err = 0;  /* set where the reference throws */

static double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */
static double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */
static int fin(double x) { return isfinite(x); }
static double clamp_min(double x) { return fin(x) ? dmax(x, 1e-10) : 1e-10; }
static double finite_or(double x) { return fin(x) ? x : 0.0; }
static double safe_denom(double d)
{
    if (!fin(d)) return (d < 0.0) ? -1e-10 : 1e-10;
    if (fabs(d) < 1e-10) return (d < 0.0) ? -1e-10 : 1e-10;
    return d;
}
static double safe_div(double n, double d) { return finite_or(n) / safe_denom(d); }
static double require_positive(double x)
{
    if (!fin(x)) { g_err = 1; return 1e-10; }
    if (x <= 0.0) return 1e-10;
    return x;
}
static double minmod(double a, double b)
{
    if (a * b <= 0.0) return 0.0;
    return fabs(a) < fabs(b) ? a : b;
}

/* EOS::pressure: (gamma-1)(E - 0.5 |mom|^2 / rho) [- gamma p_inf], clamped. */
static double pressure(const Mat* M, const EU* U)
{
    const double rho = clamp_min(U->rho);
    double mom2 = 0.0;
    for (int d = 0; d < M->dim; ++d) mom2 += U->mom[d] * U->mom[d];
    const double kin = 0.5 * safe_div(mom2, rho);
    double p_raw = (M->gamma - 1.0) * (U->E - kin);
    if (M->stiff) p_raw = p_raw - M->gamma * M->p_inf;
    return clamp_min(p_raw);
}

static double sound_speed_p(const Mat* M, const EU* U, double p)
{
    const double rho = clamp_min(U->rho);
    if (M->stiff) return sqrt(M->gamma * safe_div(p + M->p_inf, rho));
    return sqrt(M->gamma * safe_div(p, rho));
}

static double internal_energy(const Mat* M, double rho, double p)
{
    if (M->stiff) return safe_div(p + M->gamma * M->p_inf, (M->gamma - 1.0) * rho);
    return safe_div(p, (M->gamma - 1.0) * rho);
}

static EP cons_to_prim(const Mat* M, const EU* U)
{
    EP P;
    memset(&P, 0, sizeof P);
    const double rho = dmax(U->rho, 1e-10);
    P.rho = rho;
    for (int d = 0; d < M->dim; ++d) P.vel[d] = safe_div(U->mom[d], rho);
    P.p = dmax(pressure(M, U), 1e-10);
    return P;
}

static EU prim_to_cons(const Mat* M, const EP* P)
{
    EU U;
    memset(&U, 0, sizeof U);
    const double rho = dmax(P->rho, 1e-10);
    const double p = dmax(P->p, 1e-10);
    U.rho = rho;
    double v2 = 0.0;
    for (int d = 0; d < M->dim; ++d) {
        U.mom[d] = rho * P->vel[d];
        v2 += P->vel[d] * P->vel[d];
    }
    const double kin = 0.5 * rho * v2;
    U.E = rho * internal_energy(M, rho, p) + kin;
    return U;
}

static void enforce_prim(EP* P)
{
    P->rho = dmax(P->rho, 1e-10);
    P->p = dmax(P->p, 1e-10);
}

static void enforce_cons(const Mat* M, EU* U)
{
    EP P = cons_to_prim(M, U);
    enforce_prim(&P);
    *U = prim_to_cons(M, &P);
}

static void faces(const Mat* M, const EP* L, const EP* C, const EP* R, EP* Lf, EP* Rf)
{
    const double sr = minmod(C->rho - L->rho, R->rho - C->rho);
    const double sp = minmod(C->p - L->p, R->p - C->p);
    memset(Lf, 0, sizeof *Lf);
    memset(Rf, 0, sizeof *Rf);
    Lf->rho = C->rho - 0.5 * sr;
    Rf->rho = C->rho + 0.5 * sr;
    Lf->p = C->p - 0.5 * sp;
    Rf->p = C->p + 0.5 * sp;
    for (int d = 0; d < M->dim; ++d) {
        const double s = minmod(C->vel[d] - L->vel[d], R->vel[d] - C->vel[d]);
        Lf->vel[d] = C->vel[d] - 0.5 * s;
        Rf->vel[d] = C->vel[d] + 0.5 * s;
    }
    enforce_prim(Lf);
    enforce_prim(Rf);
}

static EU flux(const Mat* M, const EU* U, int dir)
{
    EU F;
    memset(&F, 0, sizeof F);
    const double rho = require_positive(U->rho);
    const double p = require_positive(pressure(M, U));
    double vel[MAXD], n[MAXD];
    for (int d = 0; d < M->dim; ++d) {
        vel[d] = U->mom[d] / rho;
        n[d] = 1.0 * (d == dir ? 1.0 : 0.0);
    }
    double un = 0.0;
    for (int d = 0; d < M->dim; ++d) un += vel[d] * n[d];
    F.rho = rho * un;
    for (int d = 0; d < M->dim; ++d) F.mom[d] = rho * vel[d] * un + p * n[d];
    F.E = (U->E + p) * un;
    return F;
}

static EU add(const Mat* M, const EU* A, const EU* B)
{
    EU C = *A;
    C.rho = A->rho + B->rho;
    for (int d = 0; d < M->dim; ++d) C.mom[d] = A->mom[d] + B->mom[d];
    C.E = A->E + B->E;
    return C;
}
static EU sub(const Mat* M, const EU* A, const EU* B)
{
    EU C = *A;
    C.rho = A->rho - B->rho;
    for (int d = 0; d < M->dim; ++d) C.mom[d] = A->mom[d] - B->mom[d];
    C.E = A->E - B->E;
    return C;
}
static EU scal(const Mat* M, double a, const EU* U)
{
    EU R = *U;
    R.rho = a * U->rho;
    for (int d = 0; d < M->dim; ++d) R.mom[d] = a * U->mom[d];
    R.E = a * U->E;
    return R;
}

/* compute_thermo: rho = require_positive(U.rho), vel = mom / rho, p and c. */
static void thermo(const Mat* M, const EU* U, double* rho, double* vel, double* p, double* c)
{
    *rho = require_positive(U->rho);
    for (int d = 0; d < M->dim; ++d) vel[d] = U->mom[d] / *rho;
    *p = pressure(M, U);
    *c = sound_speed_p(M, U, *p);
}

EU hllc(const Mat* M, const EU* UL, const EU* UR, int dir)
{
    double rhoL, rhoR, vL[MAXD], vR[MAXD], pL, pR, cL, cR;
    thermo(M, UL, &rhoL, vL, &pL, &cL);
    thermo(M, UR, &rhoR, vR, &pR, &cR);
    double n[MAXD];
    for (int d = 0; d < M->dim; ++d) n[d] = (d == dir) ? 1.0 : 0.0;
    double mag2 = 0.0;
    for (int d = 0; d < M->dim; ++d) mag2 += n[d] * n[d];
    const double mag = sqrt(mag2);
    const double inv_mag = (mag < 1e-10) ? 1.0 : 1.0 / mag;
    double dL = 0.0, dR = 0.0;
    for (int d = 0; d < M->dim; ++d) dL += vL[d] * n[d];
    for (int d = 0; d < M->dim; ++d) dR += vR[d] * n[d];
    const double unL = dL * inv_mag, unR = dR * inv_mag;
    const double sL = dmin(unL - cL, unR - cR);
    const double sR = dmax(unL + cL, unR + cR);
    const double num = (pR - pL) + rhoL * unL * (sL - unL) - rhoR * unR * (sR - unR);
    const double den = rhoL * (sL - unL) - rhoR * (sR - unR);
    const double s_star = safe_div(num, den);
    const double rhoL_star = rhoL * safe_div((sL - unL), (sL - s_star));
    const double rhoR_star = rhoR * safe_div((sR - unR), (sR - s_star));
    const double EL_star =
        rhoL_star * (safe_div(UL->E, rhoL) + (s_star - unL) * (s_star + safe_div(pL, rhoL * (sL - unL))));
    const double ER_star =
        rhoR_star * (safe_div(UR->E, rhoR) + (s_star - unR) * (s_star + safe_div(pR, rhoR * (sR - unR))));
    if (!fin(rhoL_star) || !fin(EL_star) || rhoL_star <= 0.0) g_err = 1;
    if (!fin(rhoR_star) || !fin(ER_star) || rhoR_star <= 0.0) g_err = 1;
    const EU FL = flux(M, UL, dir);
    const EU FR = flux(M, UR, dir);
    if (0.0 <= sL) return FL;
    if (sL <= 0.0 && 0.0 <= s_star) {
        EU S = *UL;
        S.rho = rhoL_star;
        const double delta = s_star - unL;
        for (int d = 0; d < M->dim; ++d) {
            const double u = vL[d] + delta * n[d];
            S.mom[d] = rhoL_star * u;
        }
        S.E = EL_star;
        EU dU = sub(M, &S, UL);
        EU t = scal(M, sL, &dU);
        return add(M, &FL, &t);
    }
    if (s_star <= 0.0 && 0.0 <= sR) {
        EU S = *UR;
        S.rho = rhoR_star;
        const double delta = s_star - unR;
        for (int d = 0; d < M->dim; ++d) {
            const double u = vR[d] + delta * n[d];
            S.mom[d] = rhoR_star * u;
        }
        S.E = ER_star;
        EU dU = sub(M, &S, UR);
        EU t = scal(M, sR, &dU);
        return add(M, &FR, &t);
    }
    return FR;
}

/* advance_line, one-material fast path; writes the interior cells of the
 * line into out[] (end cells untouched), or sets g_err where the reference
 * throws (a line of 2 cells: reconstruct_line_interfaces needs 3). */
static void advance_line(const Mat* M, int L, const EU* U, EU* out, int dir, double dt, double dx)
{
    if (L < 2) return;
    if (L < 3) { g_err = 1; return; }
    EP* P = (EP*)malloc(sizeof(EP) * L);
    EU* Ul = (EU*)malloc(sizeof(EU) * L);
    EU* Ur = (EU*)malloc(sizeof(EU) * L);
    EU* Uh = (EU*)malloc(sizeof(EU) * L);
    EU* F = (EU*)malloc(sizeof(EU) * L);
    for (int i = 0; i < L; ++i) {
        P[i] = cons_to_prim(M, &U[i]);
        enforce_prim(&P[i]);
    }
    Ul[0] = Ur[0] = U[0];
    Ul[L - 1] = Ur[L - 1] = U[L - 1];
    for (int i = 1; i < L - 1; ++i) {
        EP a, b;
        faces(M, &P[i - 1], &P[i], &P[i + 1], &a, &b);
        Ul[i] = prim_to_cons(M, &a);
        Ur[i] = prim_to_cons(M, &b);
        enforce_cons(M, &Ul[i]);
        enforce_cons(M, &Ur[i]);
    }
    Uh[0] = U[0];
    Uh[L - 1] = U[L - 1];
    for (int i = 1; i < L - 1; ++i) {
        const EU Fl = flux(M, &Ul[i], dir);
        const EU Fr = flux(M, &Ur[i], dir);
        const double factor = 0.5 * dt / dx;
        const EU dF = sub(M, &Fr, &Fl);
        const EU t = scal(M, factor, &dF);
        Uh[i] = sub(M, &U[i], &t);
        enforce_cons(M, &Uh[i]);
    }
    for (int i = 0; i < L; ++i) {
        P[i] = cons_to_prim(M, &Uh[i]);
        enforce_prim(&P[i]);
    }
    Ul[0] = Ur[0] = Uh[0];
    Ul[L - 1] = Ur[L - 1] = Uh[L - 1];
    for (int i = 1; i < L - 1; ++i) {
        EP a, b;
        faces(M, &P[i - 1], &P[i], &P[i + 1], &a, &b);
        Ul[i] = prim_to_cons(M, &a);
        Ur[i] = prim_to_cons(M, &b);
        enforce_cons(M, &Ul[i]);
        enforce_cons(M, &Ur[i]);
    }
    for (int i = 0; i < L - 1; ++i) {
        EU a = Ur[i], b = Ul[i + 1];
        enforce_cons(M, &a);
        enforce_cons(M, &b);
        F[i] = hllc(M, &a, &b, dir);
    }
    const double factor = dt / dx;
    for (int i = 1; i < L - 1; ++i) {
        const EU dF = sub(M, &F[i], &F[i - 1]);
        const EU t = scal(M, factor, &dF);
        EU n = sub(M, &U[i], &t);
        enforce_cons(M, &n);
        out[i] = n;
    }
    free(P); free(Ul); free(Ur); free(Uh); free(F);
}

/* ---- SoA plumbing -------------------------------------------------------- */

typedef struct {
    int dim, N[3];
    long long ncell, stride[3];
    double dx[3];
    int bc_lo[3], bc_hi[3];
    Mat M;
} Grid;

static int make_grid(const dimgpu_desc* d, Grid* g)
{
    if (!d || d->dim < 1 || d->dim > 3 || d->nmat != 1) return DIMGPU_E_INVALID_ARG;
    if (d->mat[0].kind != DIMGPU_EOS_IDEAL_GAS && d->mat[0].kind != DIMGPU_EOS_STIFFENED_GAS)
        return DIMGPU_E_UNSUPPORTED_EOS;
    memset(g, 0, sizeof *g);
    g->dim = d->dim;
    g->ncell = 1;
    for (int a = 0; a < 3; ++a) {
        g->N[a] = a < d->dim ? d->N[a] : 1;
        g->dx[a] = d->dx[a];
        g->bc_lo[a] = d->bc_lo[a];
        g->bc_hi[a] = d->bc_hi[a];
        if (a < d->dim && (g->N[a] < 1 || !(d->dx[a] > 0.0))) return DIMGPU_E_INVALID_ARG;
    }
    g->stride[0] = 1;
    g->stride[1] = g->N[0];
    g->stride[2] = (long long)g->N[0] * g->N[1];
    g->ncell = (long long)g->N[0] * g->N[1] * g->N[2];
    g->M.dim = d->dim;
    g->M.stiff = d->mat[0].kind == DIMGPU_EOS_STIFFENED_GAS;
    g->M.gamma = d->mat[0].gamma;
    g->M.p_inf = d->mat[0].p_inf;
    return DIMGPU_OK;
}

static EU get(const Grid* g, const double* s, long long i)
{
    EU U;
    memset(&U, 0, sizeof U);
    U.rho = s[i];
    for (int d = 0; d < g->dim; ++d) U.mom[d] = s[(1 + d) * g->ncell + i];
    U.E = s[(1 + g->dim) * g->ncell + i];
    return U;
}

static void put(const Grid* g, double* s, long long i, const EU* U)
{
    s[i] = U->rho;
    for (int d = 0; d < g->dim; ++d) s[(1 + d) * g->ncell + i] = U->mom[d];
    s[(1 + g->dim) * g->ncell + i] = U->E;
}

/* sweep_lines_flat + advance_line over every line of axis dir.  `out` holds
 * the caller's initial contents (zeros for the split update, the base state
 * for the unsplit one); interior cells of each line are overwritten. */
static int sweep(const Grid* g, int dir, double dt, const double* in, double* out)
{
    const int L = g->N[dir];
    const long long lines = g->ncell / L;
    EU* lu = (EU*)malloc(sizeof(EU) * (L + 1));
    EU* lo = (EU*)malloc(sizeof(EU) * (L + 1));
    g_err = 0;
    for (long long line = 0; line < lines; ++line) {
        int idx[3] = {0, 0, 0};
        long long t = line;
        for (int a = 0; a < g->dim; ++a) {
            if (a == dir) continue;
            idx[a] = (int)(t % g->N[a]);
            t /= g->N[a];
        }
        long long base = 0;
        for (int a = 0; a < g->dim; ++a) base += (long long)idx[a] * g->stride[a];
        for (int i = 0; i < L; ++i) lu[i] = get(g, in, base + (long long)i * g->stride[dir]);
        for (int i = 0; i < L; ++i) lo[i] = get(g, out, base + (long long)i * g->stride[dir]);
        advance_line(&g->M, L, lu, lo, dir, dt, g->dx[dir]);
        for (int i = 1; i + 1 < L; ++i) put(g, out, base + (long long)i * g->stride[dir], &lo[i]);
    }
    free(lu);
    free(lo);
    return g_err ? DIMGPU_E_NONFINITE : DIMGPU_OK;
}

static int has_physical_energy(const Grid* g, const EU* U)
{
    if (!fin(U->rho) || U->rho <= 0.0 || !fin(U->E)) return 0;
    double mom2 = 0.0;
    for (int d = 0; d < g->dim; ++d) {
        if (!fin(U->mom[d])) return 0;
        mom2 += U->mom[d] * U->mom[d];
    }
    return U->E > 0.5 * mom2 / dmax(U->rho, 1e-12);
}

static long long flat(const Grid* g, const int* idx)
{
    long long id = 0;
    for (int a = 0; a < g->dim; ++a) id += (long long)idx[a] * g->stride[a];
    return id;
}

/* apply_boundary_conditions: in place, in linear order. */
static void boundary(const Grid* g, double* s)
{
    for (long long id = 0; id < g->ncell; ++id) {
        int idx[3] = {0, 0, 0}, src[3];
        long long t = id;
        for (int a = 0; a < g->dim; ++a) {
            idx[a] = (int)(t % g->N[a]);
            t /= g->N[a];
        }
        int is_b = 0;
        for (int a = 0; a < 3; ++a) src[a] = idx[a];
        for (int a = 0; a < g->dim; ++a) {
            if (idx[a] == 0) { src[a] = 1; is_b = 1; }
            else if (idx[a] == g->N[a] - 1) { src[a] = g->N[a] - 2; is_b = 1; }
        }
        if (!is_b) continue;
        const long long sid = flat(g, src);
        int bc = DIMGPU_BC_TRANSMISSIVE;
        for (int a = 0; a < g->dim; ++a) {
            if (idx[a] == 0) { bc = g->bc_lo[a]; break; }
            if (idx[a] == g->N[a] - 1) { bc = g->bc_hi[a]; break; }
        }
        if (bc == DIMGPU_BC_NONREFLECTIVE) {
            int second[3];
            for (int a = 0; a < 3; ++a) second[a] = src[a];
            for (int a = 0; a < g->dim; ++a) {
                if (idx[a] == 0 && g->N[a] > 2) second[a] = 2;
                else if (idx[a] == g->N[a] - 1 && g->N[a] > 2) second[a] = g->N[a] - 3;
            }
            const EU Us = get(g, s, sid);
            const EU U2 = get(g, s, flat(g, second));
            EU st = Us;
            const EU dU = sub(&g->M, &Us, &U2);
            const EU ex = add(&g->M, &Us, &dU);
            int axis = 0;
            for (int a = 0; a < g->dim; ++a)
                if (idx[a] == 0 || idx[a] == g->N[a] - 1) { axis = a; break; }
            const int sign = (idx[axis] == 0) ? -1 : 1;
            const double vn = sign * safe_div(ex.mom[axis], ex.rho);
            if (has_physical_energy(g, &ex) && vn > 0.0) {
                const double rho = dmax(st.rho, 1e-12);
                double m2b = 0.0, m2a = 0.0;
                for (int d = 0; d < g->dim; ++d) m2b += st.mom[d] * st.mom[d];
                st.mom[axis] = ex.mom[axis];
                for (int d = 0; d < g->dim; ++d) m2a += st.mom[d] * st.mom[d];
                st.E += 0.5 * (m2a - m2b) / rho;
            }
            enforce_cons(&g->M, &st);
            put(g, s, id, &st);
            continue;
        }
        EU U = get(g, s, sid);
        for (int a = 0; a < g->dim; ++a) {
            if (idx[a] == 0 && g->bc_lo[a] == DIMGPU_BC_REFLECTIVE) U.mom[a] *= -1.0;
            else if (idx[a] == g->N[a] - 1 && g->bc_hi[a] == DIMGPU_BC_REFLECTIVE) U.mom[a] *= -1.0;
        }
        put(g, s, id, &U);
    }
}

static double cfl_dt(const Grid* g, const double* s, double cfl, double dt_max, int unsplit)
{
    double dt = dt_max;
    g_err = 0;
    for (long long i = 0; i < g->ncell; ++i) {
        const EU U = get(g, s, i);
        double rho, vel[MAXD], p, c;
        thermo(&g->M, &U, &rho, vel, &p, &c);
        if (unsplit) {
            double sum = 0.0;
            for (int d = 0; d < g->dim; ++d) sum += (fabs(vel[d]) + c) / g->dx[d];
            if (sum > 1e-14) dt = dmin(dt, cfl / sum);
        }
        else {
            for (int d = 0; d < g->dim; ++d) {
                const double ws = fabs(vel[d]) + c;
                if (ws > 1e-14) dt = dmin(dt, cfl * g->dx[d] / ws);
            }
        }
    }
    return dt;
}

/* ---- exported ------------------------------------------------------------ */

int euler_oracle_compute_dt_cfl(const dimgpu_desc* d, const double* soa, double cfl, double dt_max, double* dt)
{
    Grid g;
    int rc = make_grid(d, &g);
    if (rc) return rc;
    if (!(cfl > 0.0) || !(dt_max > 0.0)) return DIMGPU_E_INVALID_ARG;
    *dt = cfl_dt(&g, soa, cfl, dt_max, d->time_update == DIMGPU_TIME_UNSPLIT);
    return g_err ? DIMGPU_E_NONFINITE : DIMGPU_OK;
}

int euler_oracle_sweep_direction(const dimgpu_desc* d, int dir, double dt, const double* in, double* out)
{
    Grid g;
    int rc = make_grid(d, &g);
    if (rc) return rc;
    if (dir < 0 || dir >= d->dim) return DIMGPU_E_INVALID_ARG;
    return sweep(&g, dir, dt, in, out);
}

int euler_oracle_apply_boundary_conditions(const dimgpu_desc* d, double* soa)
{
    Grid g;
    int rc = make_grid(d, &g);
    if (rc) return rc;
    boundary(&g, soa);
    return DIMGPU_OK;
}

int euler_oracle_hllc(const dimgpu_desc* d, int n, int dir, const double* UL, const double* UR, double* out)
{
    Grid g;
    int rc = make_grid(d, &g);
    if (rc) return rc;
    const int V = 2 + d->dim;
    g_err = 0;
    for (int i = 0; i < n; ++i) {
        EU a, b;
        memset(&a, 0, sizeof a);
        memset(&b, 0, sizeof b);
        a.rho = UL[i * V];
        b.rho = UR[i * V];
        for (int k = 0; k < d->dim; ++k) {
            a.mom[k] = UL[i * V + 1 + k];
            b.mom[k] = UR[i * V + 1 + k];
        }
        a.E = UL[i * V + 1 + d->dim];
        b.E = UR[i * V + 1 + d->dim];
        const EU F = hllc(&g.M, &a, &b, dir);
        out[i * V] = F.rho;
        for (int k = 0; k < d->dim; ++k) out[i * V + 1 + k] = F.mom[k];
        out[i * V + 1 + d->dim] = F.E;
    }
    return g_err ? DIMGPU_E_NONFINITE : DIMGPU_OK;
}

/* One advance_one_step: CFL dt, then the split (x, y, z sweeps, each into a
 * zeroed buffer and followed by the boundary fill) or unsplit update. */
static int step(const Grid* g, const dimgpu_desc* d, double* s, double cfl, double dt_max, double* dt_out)
{
    const size_t bytes = sizeof(double) * (size_t)(2 + g->dim) * (size_t)g->ncell;
    const double dt = cfl_dt(g, s, cfl, dt_max, d->time_update == DIMGPU_TIME_UNSPLIT);
    if (g_err) return DIMGPU_E_NONFINITE;
    if (!(dt > 0.0) || !fin(dt)) return DIMGPU_E_NONFINITE;
    double* next = (double*)malloc(bytes);
    int rc = DIMGPU_OK;
    if (d->time_update == DIMGPU_TIME_UNSPLIT) {
        double* acc = (double*)malloc(bytes);
        memcpy(acc, s, bytes);
        for (int dir = 0; dir < g->dim && !rc; ++dir) {
            memcpy(next, s, bytes);
            rc = sweep(g, dir, dt, s, next);
            for (long long i = 0; i < g->ncell && !rc; ++i) {
                EU a = get(g, acc, i);
                const EU u = get(g, next, i), b = get(g, s, i);
                const EU du = sub(&g->M, &u, &b);
                a = add(&g->M, &a, &du);
                put(g, acc, i, &a);
            }
        }
        if (!rc) {
            for (long long i = 0; i < g->ncell; ++i) {
                EU a = get(g, acc, i);
                enforce_cons(&g->M, &a);
                put(g, acc, i, &a);
            }
            boundary(g, acc);
            memcpy(s, acc, bytes);
        }
        free(acc);
    }
    else {
        for (int dir = 0; dir < g->dim && !rc; ++dir) {
            memset(next, 0, bytes);
            rc = sweep(g, dir, dt, s, next);
            if (!rc) {
                boundary(g, next);
                memcpy(s, next, bytes);
            }
        }
    }
    free(next);
    if (dt_out) *dt_out = dt;
    return rc;
}

int euler_oracle_advance(const dimgpu_desc* d, const double* soa_in, double* soa_out, double cfl, double dt_max,
                         int steps, double* dts)
{
    Grid g;
    int rc = make_grid(d, &g);
    if (rc) return rc;
    if (!(cfl > 0.0) || !(dt_max > 0.0)) return DIMGPU_E_INVALID_ARG;
    const size_t count = (size_t)(2 + g.dim) * (size_t)g.ncell;
    memcpy(soa_out, soa_in, sizeof(double) * count);
    for (int k = 0; k < steps; ++k) {
        rc = step(&g, d, soa_out, cfl, dt_max, dts ? &dts[k] : NULL);
        if (rc) return rc;
    }
    return DIMGPU_OK;
}
