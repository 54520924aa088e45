// dim_mixed.h — the mixed-precision line step (precision MIXED).
//
// Same five stages as the FP64 step (dim_line.h).  FP32 carries the small
// quantities of the two MUSCL reconstructions and of the HLLC star state;
// FP64 carries every quantity whose absolute size is the solution:
//  * slopes: the one-sided differences are formed in FP64 and limited
//    (minmod) in FP32, and the half slope is added to the FP64 cell value in
//    FP64, so a face value carries the FP32 rounding of its slope, not of
//    itself;
//  * HLLC: the contact speed is the FP64 mean normal velocity plus an FP32
//    increment formed from the FP64 pressure and velocity jumps; the
//    star-state ratios (chi - 1, s* - u_K, s_K rho_K (s* - u_K)) are FP32,
//    and the flux is FP64 state times FP64 coefficients built from them;
//  * FP64: the cell recoveries (cons_to_prim of U and of the half-step
//    state, where (gamma-1)(E - kinetic) - gamma p_inf cancels; in closed
//    form, pressure_closed_form below), every sound speed and wave-speed
//    estimate, the physical fluxes, the Hancock and cell updates, the alpha
//    update and the CFL dt.
// A face state is built from its reconstructed primitive without the FP64
// step's repair / re-recovery round trip (prim_to_cons -> repair_state ->
// cons_to_prim), and HLLC takes the reconstructed primitive itself; the
// round trip returns that primitive to within the recovery's bisection
// tolerance.  Results differ from the FP64 step at the FP32 rounding of
// slopes and star increments; the tests state the L1 / Linf error against
// the FP64 oracle.
#pragma once

#include <cfloat>

#include "dim_line.h"

namespace dimgpu {

DHD bool finf(float x) { return fabsf(x) <= FLT_MAX; }

// The small-quantity arithmetic is a template over its type R: float is the
// mixed form; double gives its FP64 twin (DIMGPU_PRECISION_MIXED_FP64), the
// same algorithm — closed-form recovery, no face round trip, the increment
// form of HLLC — with every quantity in FP64, so that (mixed - twin) is what
// FP32 costs and (twin - FP64 step) what the algorithm's shortcuts cost.
template<typename R>
DHD bool fin_r(R x)
{
    return fabs((double)x) <= (double)(sizeof(R) == 4 ? FLT_MAX : DBL_MAX);
}
template<typename R>
DHD R safe_div_r(R n, R d)
{
    const R tol = (R)1e-10;
    const R nn = fin_r<R>(n) ? n : (R)0;
    R dd = d;
    if (!fin_r<R>(d) || (R)fabs((double)d) < tol) dd = (d < (R)0) ? -tol : tol;
    return nn / dd;
}
template<typename R>
DHD R minmod_r(R a, R b)
{
    if (a * b <= (R)0) return (R)0;
    return fabs((double)a) < fabs((double)b) ? a : b;
}

// One limited half slope: FP64 differences, minmod in R, FP64 half slope.
template<typename R = float>
DHD double half_slope_mixed(double lo, double c, double hi)
{
    return 0.5 * (double)minmod_r<R>((R)(c - lo), (R)(hi - c));
}

// reconstruct_cell_faces with FP32-limited slopes (see the file comment).
template<int NM, int D, typename R = float>
DHD void reconstruct_mixed(const Prim<NM, D>& PL, const Prim<NM, D>& PC, const Prim<NM, D>& PR, Prim<NM, D>& Lf,
                           Prim<NM, D>& Rf)
{
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        const double h = half_slope_mixed<R>(PL.rho[k], PC.rho[k], PR.rho[k]);
        Lf.rho[k] = PC.rho[k] - h;
        Rf.rho[k] = PC.rho[k] + h;
        const double a = half_slope_mixed<R>(PL.alpha[k], PC.alpha[k], PR.alpha[k]);
        Lf.alpha[k] = PC.alpha[k] - a;
        Rf.alpha[k] = PC.alpha[k] + a;
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const double h = half_slope_mixed<R>(PL.vel[d], PC.vel[d], PR.vel[d]);
        Lf.vel[d] = PC.vel[d] - h;
        Rf.vel[d] = PC.vel[d] + h;
    }
    const double h = half_slope_mixed<R>(PL.p, PC.p, PR.p);
    Lf.p = PC.p - h;
    Rf.p = PC.p + h;
    enforce_positive_primitive<NM, D>(Lf);
    enforce_positive_primitive<NM, D>(Rf);
}

// The mixed form's pressure recovery: for ideal and stiffened gases the
// residual the reference bisects (pressure_from_internal_energy,
// src/dim/eos.hpp:77-143) is affine in p above its 1e-10 clamp,
// f(p) = A p + B - rho e, so its root is (rho e - B) / A in FP64, one
// subtraction (where the gamma p_inf terms cancel) and one division.  The
// bisection stops anywhere within 1e-10 * max(1, rho e) / A of that root; the
// mixed step takes the root itself.  Where the root is not a plain positive
// number above 1e-8 (the reference then falls back or clamps), the reference
// bisection runs instead.
template<int NM>
DHD double pressure_closed_form(const Mats& M, double rho_total, double e, const double* alpha, const double* rho)
{
    const double rt = clamp_min(rho_total);
    const double target = finite_or(rt * finite_or(e));
    double A = 0.0, B = 0.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        const double alpha_k = dmax(finite_or(alpha[k]), 0.0);
        const double rho_k = clamp_min(rho[k]);
        const double w = (alpha_k * rho_k) / safe_denom(M.gm1[k] * rho_k);
        A += w;
        if (M.stiff[k]) B += w * M.gpinf[k];
    }
    const double p = (target - B) / A;
    if (fin(A) && fin(B) && A > 1e-200 && fin(p) && p >= 1e-8 && p < 1e290 / A) return p;
    return pressure_from_internal_energy<NM>(M, rho_total, e, alpha, rho);
}

// cons_to_prim (primitives.hpp:111-162) with the closed-form recovery.
template<int NM, int D>
DHD Prim<NM, D> cons_to_prim_mixed_t(const Mats& M, State<NM, D> U)
{
    Prim<NM, D> P;
    full_alpha<NM, D>(U, P.alpha);
    sanitise_alpha<NM>(P.alpha, 1e-12);
    double rho_total = 0.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) rho_total += finite_or(U.m[k]);
    rho_total = dmax(rho_total, 1e-12);
    double velocity_squared = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        P.vel[d] = safe_div(U.mom[d], rho_total);
        velocity_squared += P.vel[d] * P.vel[d];
    }
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        const double alpha_k = dmax(P.alpha[k], 1e-12);
        P.rho[k] = dmax(safe_div(finite_or(U.m[k]), alpha_k), 1e-12);
    }
    const double kinetic = 0.5 * rho_total * velocity_squared;
    const double internal_energy = safe_div(finite_or(U.E, kinetic) - kinetic, rho_total);
    P.p = dmax(pressure_closed_form<NM>(M, rho_total, internal_energy, P.alpha, P.rho), 1e-12);
    return P;
}

template<int NM, int D>
DNI Prim<NM, D> cons_to_prim_mixed_v(const Mats& M, State<NM, D> U)
{
    return cons_to_prim_mixed_t<NM, D>(M, U);
}

template<int NM, int D>
DHD void cons_to_prim_mixed(const Mats& M, const State<NM, D>& U, Prim<NM, D>& P)
{
    P = cons_to_prim_mixed_v<NM, D>(M, U);
}

// The mixed recovery inlined (IL, kernels with one call site) or out of line.
template<int NM, int D, bool IL>
DHD Prim<NM, D> c2p_mixed(const Mats& M, const State<NM, D>& U)
{
    if constexpr (IL) return cons_to_prim_mixed_t<NM, D>(M, U);
    else return cons_to_prim_mixed_v<NM, D>(M, U);
}

// Stage A of the mixed step (stage_a with the closed-form recovery).
template<int NM, int D, bool IL = false>
DHD void stage_a_mixed(const Mats& M, const State<NM, D>& U, CellA<NM, D>& A)
{
    A.P = c2p_mixed<NM, D, IL>(M, U);
    A.Pe = A.P;
    enforce_positive_primitive<NM, D>(A.Pe);
    rhs_sound_speeds<NM, D>(M, A.P, A.ck);
}

// HLLC with the star state in FP32 increment form.  Same wave-speed
// estimates, case selection and fallbacks (average, HLL) as hllc_flux.  With
//   a_K = rho_K (s_K - u_K),
//   s* = u_L + (p_R - p_L) / (a_L - a_R) + (a_R / (a_L - a_R)) (u_L - u_R),
//   chi = (s_K - u_K) / (s_K - s*) = 1 + (s* - u_K) / (s_K - s*),
// hllc_flux's star flux F_K + s_K (U*_K - U_K) is, term by term,
//   mass   chi s* m_k
//   mom    chi s* mom_d + [d = dir] (p_K + s_K chi rho_K (s* - u_K))
//   energy chi s* (E_K + p_K + s_K rho_K (s* - u_K)).
// The two quotients of s*, chi - 1 and the bracketed increments are FP32,
// the sums and products with the state FP64, so the flux carries the FP32
// rounding of the increments only.  For mirror states at a wall
// (p_L = p_R, a_L = -a_R, u_L = -u_R) a_R / (a_L - a_R) is exactly -1/2, s*
// is exactly 0, and so are the mass and energy fluxes.
template<int NM, int D, typename R = float, bool IL = false>
DHD bool hllc_mixed(const Mats& M, const State<NM, D>& UL, const State<NM, D>& UR, const Prim<NM, D>& PL,
                    const Prim<NM, D>& PR, int dir, Flux<NM, D>& F, double& s_face)
{
    double rhoL = total_density<NM, D>(UL), rhoR = total_density<NM, D>(UR);
    double pL = PL.p, pR = PR.p;
    if (!fin(rhoL) || !fin(rhoR) || !fin(pL) || !fin(pR)) return false;
    if (rhoL <= 0.0) rhoL = 1e-10;
    if (rhoR <= 0.0) rhoR = 1e-10;
    if (pL <= 0.0) pL = 1e-10;
    if (pR <= 0.0) pR = 1e-10;
    const double unL = PL.vel[dir], unR = PR.vel[dir];
    const double cL = sound<NM, IL>(M, rhoL, pL, PL.alpha, PL.rho);
    const double cR = sound<NM, IL>(M, rhoR, pR, PR.alpha, PR.rho);
    const double sL = dmin(unL - cL, unR - cR);
    const double sR = dmax(unL + cL, unR + cR);

    const R aL = (R)(rhoL * (sL - unL)), aR = (R)(rhoR * (sR - unR));
    const R den = aL - aR;
    const R w = safe_div_r<R>(aR, den);
    double s_star = unL + (double)safe_div_r<R>((R)(pR - pL), den) + (double)w * (unL - unR);
    if (fabs(pL - pR) < 1e-10 && fabs(unL - unR) < 1e-10) s_star = unL;

    const bool average = !fin(sL) || !fin(sR) || !fin(s_star);
    const bool star = !average && sL < 0.0 && 0.0 < sR;
    const bool left = (sL <= 0.0 && 0.0 <= s_star);
    const State<NM, D>& UK = left ? UL : UR;
    const double rhoK = left ? rhoL : rhoR;
    const double pK = left ? pL : pR;
    const double sK = left ? sL : sR;
    const double unK = left ? unL : unR;
    if (star) {
        const R ds = (R)(s_star - unK);                   // s* - u_K
        const R chi_m1 = safe_div_r<R>(ds, (R)(sK - s_star));
        const double chi = 1.0 + (double)chi_m1;
        const R sKrK = (R)sK * (R)rhoK;
        const double a = chi * s_star;
        const double E = a * (UK.E + pK + (double)(sKrK * ds));
        s_face = s_star;
        if (chi > 0.0 && fin_r<R>(chi_m1) && fin(E)) {
#pragma unroll
            for (int k = 0; k < NM; ++k) F.m[k] = a * UK.m[k];
#pragma unroll
            for (int d = 0; d < D; ++d)
                F.mom[d] = a * UK.mom[d] + (d == dir ? pK + chi * (double)(sKrK * ds) : 0.0);
            F.E = E;
            return true;
        }
    }
    Flux<NM, D> FL, FR;
    flux_normal<NM, D>(UL, PL, dir, FL);
    flux_normal<NM, D>(UR, PR, dir, FR);
    if (!average && 0.0 <= sL) { F = FL; s_face = unL; return true; }
    if (!average && sR <= 0.0) { F = FR; s_face = unR; return true; }
    if (average || !(sL < sR)) {
#pragma unroll
        for (int k = 0; k < NM; ++k) F.m[k] = 0.5 * (FL.m[k] + FR.m[k]);
#pragma unroll
        for (int d = 0; d < D; ++d) F.mom[d] = 0.5 * (FL.mom[d] + FR.mom[d]);
        F.E = 0.5 * (FL.E + FR.E);
        s_face = 0.5 * (unL + unR);
        return true;
    }
    // hll_flux, where the star density is not positive or not finite
    s_face = s_star;
    const double inv = 1.0 / (sR - sL);
    const double sLsR = sL * sR;
#pragma unroll
    for (int k = 0; k < NM; ++k) F.m[k] = inv * ((sR * FL.m[k] - sL * FR.m[k]) + sLsR * (UR.m[k] - UL.m[k]));
#pragma unroll
    for (int d = 0; d < D; ++d) F.mom[d] = inv * ((sR * FL.mom[d] - sL * FR.mom[d]) + sLsR * (UR.mom[d] - UL.mom[d]));
    F.E = inv * ((sR * FL.E - sL * FR.E) + sLsR * (UR.E - UL.E));
    return true;
}

// Stage B of the mixed step: FP32-limited faces, face states without the
// repair round trip, FP64 Hancock half step (hancock_predict's arithmetic,
// muscl.hpp:143-191, evaluated face by face as in stage_b) and FP64
// recovery into Ph.
template<int NM, int D, typename R = float, bool IL = false>
DHD void stage_b_mixed(const Mats& M, const State<NM, D>& U, const CellA<NM, D>& A, const Prim<NM, D>& Pe_lo,
                       const Prim<NM, D>& Pe_hi, bool end, int dir, double dt, double dx, Prim<NM, D>& Ph)
{
    if (end) {
        Ph = A.Pe;
        return;
    }
    double rhs[NM];
    alpha_rhs_coefficients<NM, D>(M, A.Pe, A.ck, rhs);
    Prim<NM, D> Pl, Pr;
    reconstruct_mixed<NM, D, R>(Pe_lo, A.Pe, Pe_hi, Pl, Pr);
    Flux<NM, D> FL, FR;
    {
        const State<NM, D> Ul = p2c<NM, D, IL>(M, Pl);
        flux_normal<NM, D>(Ul, Pl, dir, FL);
    }
    {
        const State<NM, D> Ur = p2c<NM, D, IL>(M, Pr);
        flux_normal<NM, D>(Ur, Pr, dir, FR);
    }
    const double factor = 0.5 * dt / dx;
    State<NM, D> Uh = U;
#pragma unroll
    for (int k = 0; k < NM; ++k) Uh.m[k] -= factor * (FR.m[k] - FL.m[k]);
#pragma unroll
    for (int d = 0; d < D; ++d) Uh.mom[d] -= factor * (FR.mom[d] - FL.mom[d]);
    Uh.E -= factor * (FR.E - FL.E);
    const double u_left = Pl.vel[dir];
    const double u_right = Pr.vel[dir];
    const double div_u = (u_right - u_left) / dx;
    double alpha_new[NM];
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        alpha_new[k] = A.Pe.alpha[k];
        alpha_new[k] -= factor * (Pr.alpha[k] * u_right - Pl.alpha[k] * u_left);
        alpha_new[k] += 0.5 * dt * rhs[k] * div_u;
    }
    sanitise_alpha<NM>(alpha_new, 0.0);
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) Uh.a[k] = alpha_new[k];
    Uh = repair<NM, D, IL>(M, Uh);
    Ph = c2p_mixed<NM, D, IL>(M, Uh);
    enforce_positive_primitive<NM, D>(Ph);
}

// One face state of the mixed step's second reconstruction: the right (or
// left) face of a cell from the half-step primitives of the cell and its
// neighbours (reconstruct_mixed, one side only).  An end cell's face state
// is its own state U and primitive P instead (as in stage_c).
template<int NM, int D, typename R = float, bool IL = false>
DHD void face_mixed(const Mats& M, const Prim<NM, D>& Ph_lo, const Prim<NM, D>& Ph, const Prim<NM, D>& Ph_hi,
                    bool right, State<NM, D>& Uf, Prim<NM, D>& Pf)
{
    const double sg = right ? 1.0 : -1.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        Pf.rho[k] = Ph.rho[k] + sg * half_slope_mixed<R>(Ph_lo.rho[k], Ph.rho[k], Ph_hi.rho[k]);
        Pf.alpha[k] = Ph.alpha[k] + sg * half_slope_mixed<R>(Ph_lo.alpha[k], Ph.alpha[k], Ph_hi.alpha[k]);
    }
#pragma unroll
    for (int d = 0; d < D; ++d) Pf.vel[d] = Ph.vel[d] + sg * half_slope_mixed<R>(Ph_lo.vel[d], Ph.vel[d], Ph_hi.vel[d]);
    Pf.p = Ph.p + sg * half_slope_mixed<R>(Ph_lo.p, Ph.p, Ph_hi.p);
    enforce_positive_primitive<NM, D>(Pf);
    Uf = p2c<NM, D, IL>(M, Pf);
}

// Stage D of the mixed step: HLLC at face i|i+1 and the upwind alpha flux.
template<int NM, int D, typename R = float, bool IL = false>
DHD bool stage_d_mixed(const Mats& M, const State<NM, D>& UL, const Prim<NM, D>& PL, const State<NM, D>& UR,
                       const Prim<NM, D>& PR, int dir, FaceD<NM, D>& out)
{
    const bool ok = hllc_mixed<NM, D, R, IL>(M, UL, UR, PL, PR, dir, out.F, out.fv);
    const double* up = (out.fv >= 0.0) ? PL.alpha : PR.alpha;
#pragma unroll
    for (int k = 0; k < NM; ++k) out.af[k] = up[k] * out.fv;
    return ok;
}

}  // namespace dimgpu
