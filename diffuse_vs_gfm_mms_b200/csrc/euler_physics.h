// euler_physics.h — device arithmetic of the single-material Euler step
// (the sharp-interface solver's one-material, no-level-set fast path,
// advance_line in src/sim/solver/advance/sweep_core.hpp:65-111), shared by
// the CUDA kernels and the host test harness.
//
// Same discipline as dim_physics.h: the reference's operations in the
// reference's order (compiled with -fmad=false), libstdc++ std::max /
// std::min, the numerical-safety helpers of src/math/numerical_safety.hpp.
// The EoS is closed form (ideal or stiffened gas, MaterialEOS dispatch of
// src/euler/eos.hpp:983-1116), so a recovery costs a few operations and no
// bisection.
//
// Line stages of one sweep (cell i of a line of n >= 3 cells; ends are
// i = 0 and i = n-1):
//   A  P_i  = enforce(cons_to_prim(U_i))
//   B  interior: faces of P_{i-1}, P_i, P_{i+1} -> U_left_n, U_right_n
//      (prim_to_cons + enforce_positive_conserved), Hancock half step,
//      enforce -> U_half_i;  ends: U_half_i = U_i;   Ph_i = enforce(c2p(U_half_i))
//   C  interior: faces of Ph_{i-1}, Ph_i, Ph_{i+1} -> U_left_half,
//      U_right_half (prim_to_cons + enforce);  ends: both = U_half_i = U_i;
//      then advance_line's own enforce of each face state
//   D  face i|i+1: HLLC(RS_i, LS_{i+1})
//   E  interior: U_i - dt/dx (F_{i|i+1} - F_{i-1|i}), enforce
#pragma once

#include "dim_physics.h"

namespace dimgpu {

template<int D>
struct EState {
    double rho;
    double mom[D];
    double E;
};

template<int D>
struct EPrim {
    double rho;
    double vel[D];
    double p;
};

// EOS::pressure (IdealGasEOS / StiffenedGasEOS, src/euler/eos.hpp:449-466,
// 551-569); material 0 of M.
template<int D>
DHD double e_pressure(const Mats& M, const EState<D>& U)
{
    const double rho = clamp_min(U.rho);
    double mom2 = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) mom2 += U.mom[d] * U.mom[d];
    const double kin = 0.5 * safe_div(mom2, rho);
    double p_raw = M.gm1[0] * (U.E - kin);
    if (M.stiff[0]) p_raw = p_raw - M.gpinf[0];
    return clamp_min(p_raw);
}

// EOS::sound_speed given that pressure (eos.hpp:469-478, 572-581).
template<int D>
DHD double e_sound_speed(const Mats& M, const EState<D>& U, double p)
{
    const double rho = clamp_min(U.rho);
    if (M.stiff[0]) return sqrt(M.gamma[0] * safe_div(p + M.p_inf[0], rho));
    return sqrt(M.gamma[0] * safe_div(p, rho));
}

// EOS::internal_energy (eos.hpp:482-489, 585-592).
DHD double e_internal_energy(const Mats& M, double rho, double p)
{
    if (M.stiff[0]) return safe_div(p + M.gpinf[0], M.gm1[0] * rho);
    return safe_div(p, M.gm1[0] * rho);
}

// cons_to_prim, src/euler/conservative.hpp:12-50 (its internal energy is
// computed and discarded there; nothing reads it).
template<int D>
DHD EPrim<D> e_cons_to_prim(const Mats& M, const EState<D>& U)
{
    EPrim<D> P;
    const double rho = dmax(U.rho, 1e-10);
    P.rho = rho;
#pragma unroll
    for (int d = 0; d < D; ++d) P.vel[d] = safe_div(U.mom[d], rho);
    P.p = dmax(e_pressure<D>(M, U), 1e-10);
    return P;
}

// prim_to_cons, src/euler/primitives.hpp:7-34.
template<int D>
DHD EState<D> e_prim_to_cons(const Mats& M, const EPrim<D>& P)
{
    EState<D> U;
    const double rho = dmax(P.rho, 1e-10);
    const double p = dmax(P.p, 1e-10);
    U.rho = rho;
    double v2 = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        U.mom[d] = rho * P.vel[d];
        v2 += P.vel[d] * P.vel[d];
    }
    const double kin = 0.5 * rho * v2;
    U.E = rho * e_internal_energy(M, rho, p) + kin;
    return U;
}

// enforce_positive_primitive / enforce_positive_conserved,
// src/euler/reconstruction/muscl.hpp:24-48 (floors 1e-10).
template<int D>
DHD void e_enforce_prim(EPrim<D>& P)
{
    P.rho = dmax(P.rho, 1e-10);
    P.p = dmax(P.p, 1e-10);
}

template<int D>
DHD void e_enforce(const Mats& M, EState<D>& U)
{
    EPrim<D> P = e_cons_to_prim<D>(M, U);
    e_enforce_prim<D>(P);
    U = e_prim_to_cons<D>(M, P);
}

// compute_limited_slope + reconstruct_cell_faces, muscl.hpp:51-111; `right`
// picks the face (the other one is not formed).
template<int D>
DHD EPrim<D> e_face(const EPrim<D>& L, const EPrim<D>& C, const EPrim<D>& R, bool right)
{
    EPrim<D> f;
    const double sr = minmod(C.rho - L.rho, R.rho - C.rho);
    const double sp = minmod(C.p - L.p, R.p - C.p);
    f.rho = right ? C.rho + 0.5 * sr : C.rho - 0.5 * sr;
    f.p = right ? C.p + 0.5 * sp : C.p - 0.5 * sp;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const double s = minmod(C.vel[d] - L.vel[d], R.vel[d] - C.vel[d]);
        f.vel[d] = right ? C.vel[d] + 0.5 * s : C.vel[d] - 0.5 * s;
    }
    e_enforce_prim<D>(f);
    return f;
}

// Face state of a reconstruction: prim_to_cons of the face, then
// enforce_positive_conserved (muscl.hpp:217-221, 278-282).
template<int D>
DHD EState<D> e_face_state(const Mats& M, const EPrim<D>& L, const EPrim<D>& C, const EPrim<D>& R, bool right)
{
    const EPrim<D> f = e_face<D>(L, C, R, right);
    EState<D> U = e_prim_to_cons<D>(M, f);
    e_enforce<D>(M, U);
    return U;
}

// compute_flux_normal, src/euler/flux.hpp:14-53, normal e_dir (its
// normalisation 1/|n| = 1 leaves n unchanged).  Returns false where
// require_positive throws (non-finite density).
template<int D>
DHD bool e_flux(const Mats& M, const EState<D>& U, int dir, EState<D>& F)
{
    if (!fin(U.rho)) return false;
    const double rho = (U.rho <= 0.0) ? 1e-10 : U.rho;
    const double p0 = e_pressure<D>(M, U);
    const double p = (p0 <= 0.0) ? 1e-10 : p0;  // finite: e_pressure clamps
    double vel[D];
#pragma unroll
    for (int d = 0; d < D; ++d) vel[d] = U.mom[d] / rho;
    double un = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) un += vel[d] * (d == dir ? 1.0 : 0.0);
    F.rho = rho * un;
#pragma unroll
    for (int d = 0; d < D; ++d) F.mom[d] = rho * vel[d] * un + p * (d == dir ? 1.0 : 0.0);
    F.E = (U.E + p) * un;
    return true;
}

// Hancock half step of an interior cell, muscl.hpp:114-135, with the
// enforce of muscl.hpp:236.
template<int D>
DHD bool e_hancock(const Mats& M, const EState<D>& U, const EState<D>& Ul, const EState<D>& Ur, int dir, double dt,
                   double dx, EState<D>& Uh)
{
    EState<D> FL, FR;
    const bool ok = e_flux<D>(M, Ul, dir, FL) & e_flux<D>(M, Ur, dir, FR);
    const double factor = 0.5 * dt / dx;
    Uh.rho = U.rho - factor * (FR.rho - FL.rho);
#pragma unroll
    for (int d = 0; d < D; ++d) Uh.mom[d] = U.mom[d] - factor * (FR.mom[d] - FL.mom[d]);
    Uh.E = U.E - factor * (FR.E - FL.E);
    e_enforce<D>(M, Uh);
    return ok;
}

// compute_thermo, src/euler/thermo_compute.hpp:10-26: rho by
// require_positive, vel = mom / rho, p and c from the EoS.
template<int D>
DHD bool e_thermo(const Mats& M, const EState<D>& U, double& rho, double* vel, double& p, double& c)
{
    if (!fin(U.rho)) return false;
    rho = (U.rho <= 0.0) ? 1e-10 : U.rho;
#pragma unroll
    for (int d = 0; d < D; ++d) vel[d] = U.mom[d] / rho;
    p = e_pressure<D>(M, U);
    c = e_sound_speed<D>(M, U, p);
    return true;
}

// hllc_flux_normal, src/euler/riemann/hllc.hpp:18-152, normal e_dir.
// Returns false where the reference throws: a non-finite density, or an
// invalid left or right star state (both are checked whatever the region).
template<int D>
DHD bool e_hllc(const Mats& M, const EState<D>& UL, const EState<D>& UR, int dir, EState<D>& F)
{
    double rhoL, rhoR, vL[D], vR[D], pL, pR, cL, cR;
    if (!e_thermo<D>(M, UL, rhoL, vL, pL, cL)) return false;
    if (!e_thermo<D>(M, UR, rhoR, vR, pR, cR)) return false;
    double unL = 0.0, unR = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) unL += vL[d] * (d == dir ? 1.0 : 0.0);
#pragma unroll
    for (int d = 0; d < D; ++d) unR += vR[d] * (d == dir ? 1.0 : 0.0);
    unL = unL * 1.0;
    unR = unR * 1.0;
    const double sL = dmin(unL - cL, unR - cR);
    const double sR = dmax(unL + cL, unR + cR);
    const double num = (pR - pL) + rhoL * unL * (sL - unL) - rhoR * unR * (sR - unR);
    const double den = rhoL * (sL - unL) - rhoR * (sR - unR);
    const double s_star = safe_div(num, den);
    const double rhoL_star = rhoL * safe_div((sL - unL), (sL - s_star));
    const double rhoR_star = rhoR * safe_div((sR - unR), (sR - s_star));
    const double EL_star =
        rhoL_star * (safe_div(UL.E, rhoL) + (s_star - unL) * (s_star + safe_div(pL, rhoL * (sL - unL))));
    const double ER_star =
        rhoR_star * (safe_div(UR.E, rhoR) + (s_star - unR) * (s_star + safe_div(pR, rhoR * (sR - unR))));
    if (!fin(rhoL_star) || !fin(EL_star) || rhoL_star <= 0.0) return false;
    if (!fin(rhoR_star) || !fin(ER_star) || rhoR_star <= 0.0) return false;
    // Region selection (hllc.hpp:112-151).  The face values of the chosen
    // side are picked element by element, so no array is addressed through
    // a runtime-selected pointer (which would put the states in local memory).
    const bool useL = (0.0 <= sL) || (sL <= 0.0 && 0.0 <= s_star);
    EState<D> UK;
    UK.rho = useL ? UL.rho : UR.rho;
#pragma unroll
    for (int d = 0; d < D; ++d) UK.mom[d] = useL ? UL.mom[d] : UR.mom[d];
    UK.E = useL ? UL.E : UR.E;
    EState<D> FK;
    if (!e_flux<D>(M, UK, dir, FK)) return false;
    if (0.0 <= sL) { F = FK; return true; }
    const bool left = (sL <= 0.0 && 0.0 <= s_star);
    const bool right = !left && (s_star <= 0.0 && 0.0 <= sR);
    if (!left && !right) { F = FK; return true; }
    const double rs = left ? rhoL_star : rhoR_star;
    const double Es = left ? EL_star : ER_star;
    const double sK = left ? sL : sR;
    const double delta = s_star - (left ? unL : unR);
    F.rho = FK.rho + sK * (rs - UK.rho);
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const double u = (left ? vL[d] : vR[d]) + delta * (d == dir ? 1.0 : 0.0);
        F.mom[d] = FK.mom[d] + sK * (rs * u - UK.mom[d]);
    }
    F.E = FK.E + sK * (Es - UK.E);
    return true;
}

// Interior update + enforce (sweep_core.hpp:102-108).
template<int D>
DHD void e_update(const Mats& M, const EState<D>& U, const EState<D>& Flo, const EState<D>& Fhi, double dt, double dx,
                  EState<D>& out)
{
    const double factor = dt / dx;
    out.rho = U.rho - factor * (Fhi.rho - Flo.rho);
#pragma unroll
    for (int d = 0; d < D; ++d) out.mom[d] = U.mom[d] - factor * (Fhi.mom[d] - Flo.mom[d]);
    out.E = U.E - factor * (Fhi.E - Flo.E);
    e_enforce<D>(M, out);
}

// CFL candidate of one cell (compute_dt_cfl_materials body,
// src/sim/solver/cfl.hpp:106-122; unsplit :169-183).  false: non-finite
// density (compute_thermo throws).
template<int D>
DHD bool e_cfl_candidate(const Mats& M, const EState<D>& U, const double* dx, double cfl, bool unsplit, double& best)
{
    double rho, vel[D], p, c;
    best = HUGE_VAL;
    if (!e_thermo<D>(M, U, rho, vel, p, c)) return false;
    if (unsplit) {
        double sum = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) sum += (fabs(vel[d]) + c) / dx[d];
        if (sum > 1e-14) best = cfl / sum;
        return true;
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const double ws = fabs(vel[d]) + c;
        if (ws > 1e-14) best = dmin(best, cfl * dx[d] / ws);
    }
    return true;
}

}  // namespace dimgpu
