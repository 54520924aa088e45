// dim_line.h — the split sweep of one line (dim::solve_line,
// src/dim/solver/advance/sweep_core.hpp:16-149, with
// reconstruct_line_interfaces, src/dim/reconstruction/muscl.hpp:197-329)
// factored into five per-cell stages whose only coupling is to the nearest
// neighbour of the previous stage:
//
//   A  cell i:  P_i = cons_to_prim(U_i)                    (one bisection)
//   B  cell i:  needs Pe_{i-1}, Pe_{i+1} -> U_half_i, Ph_i  (one bisection)
//   C  cell i:  needs Ph_{i-1}, Ph_{i+1} -> face states LS_i, RS_i and their
//               primitives PLS_i, PRS_i                     (two bisections)
//   D  face i|i+1: needs RS_i, PRS_i, LS_{i+1}, PLS_{i+1} -> HLLC flux F,
//               face velocity s*, upwind alpha flux
//   E  cell i:  needs the faces i-1|i and i|i+1 -> U_out_i
//
// The CUDA kernel runs the stages over a shared-memory tile with one
// __syncthreads between them; tests/native runs them over a host array.  The
// reference computes the same quantities line-wide; the factorisation
// removes its duplicate recoveries without changing any value:
//  * primitive[i] and P_line[i] share one cons_to_prim (P_line = enforce(P));
//  * P_half of an end cell is P_line of that cell (U_half = U there);
//  * the face primitives PL_face / PR_face are the cons_to_prim calls inside
//    hllc_flux_normal (same states), computed once per face state;
//  * the material sound speeds of alpha_rhs_coefficients depend on (rho_k, p)
//    only, which P and enforce(P) share.
#pragma once

#include "dim_physics.h"

namespace dimgpu {

// Routine selectors: IL = true inlines the routine's body (the staged
// kernels, which call each routine from one site), false calls its single
// out-of-line copy (kernels that call it from many sites).
template<int NM, int D, bool IL>
DHD Prim<NM, D> c2p(const Mats& M, const State<NM, D>& U)
{
    if constexpr (IL) return cons_to_prim_t<NM, D, true>(M, U);
    else return cons_to_prim_v<NM, D>(M, U);
}

template<int NM, int D, bool IL>
DHD State<NM, D> p2c(const Mats& M, const Prim<NM, D>& P)
{
    if constexpr (IL) return prim_to_cons_t<NM, D>(M, P);
    else return prim_to_cons_v<NM, D>(M, P);
}

template<int NM, int D, bool IL>
DHD State<NM, D> repair(const Mats& M, const State<NM, D>& U)
{
    if constexpr (IL) return repair_state_t<NM, D, false>(M, U);
    else return repair_state_v<NM, D>(M, U);
}

// ck (inlined form only): material sound speeds of the same primitive to
// reuse where their arguments agree, or nullptr.
template<int NM, bool IL>
DHD double sound(const Mats& M, double rho_total, double p, const double* alpha, const double* rho,
                 const double* ck = nullptr)
{
    if constexpr (IL) return sound_speed_generic<NM>(M, rho_total, p, mix_of<NM>(alpha, rho), ck);
    else return generic_mixture_sound_speed<NM>(M, rho_total, p, alpha, rho);
}

template<int NM, int D>
struct CellA {
    Prim<NM, D> P;   // cons_to_prim(U): un-enforced (primitive[i] in solve_line)
    Prim<NM, D> Pe;  // enforce_positive_primitive(P)  (P_line[i])
    double ck[NM];   // material sound speeds for alpha_rhs_coefficients
};

// Stage A.
template<int NM, int D, bool IL = false>
DHD void stage_a(const Mats& M, const State<NM, D>& U, CellA<NM, D>& A)
{
    A.P = c2p<NM, D, IL>(M, U);
    A.Pe = A.P;
    enforce_positive_primitive<NM, D>(A.Pe);
    rhs_sound_speeds<NM, D>(M, A.P, A.ck);
}

// Stage B.  `end` is true for the first and last cell of the line and for
// every cell of a line shorter than 3 (no reconstruction there,
// muscl.hpp:213-226, 244-252, 271-272).  hancock_predict's arithmetic
// (muscl.hpp:143-191) is evaluated face by face: each face state is built,
// repaired and turned into its flux (face_flux), then the cell's half-step
// update combines the two fluxes (stage_b_update) — the same operations on
// the same values; only independent work is reordered.  The staged kernels
// run face_flux as one thread per face state and stage_b_update as one
// thread per cell.
template<int NM, int D, bool IL = false>
DHD void face_flux(const Mats& M, const Prim<NM, D>& Pf, int dir, Flux<NM, D>& F)
{
    const State<NM, D> Uf = repair<NM, D, IL>(M, p2c<NM, D, IL>(M, Pf));
    flux_normal<NM, D>(Uf, Pf, dir, F);
}

// The half-step update of stage B from the cell's face primitives Pl, Pr
// and their fluxes FL, FR.
template<int NM, int D, bool IL = false>
DHD void stage_b_update(const Mats& M, const State<NM, D>& U, const CellA<NM, D>& A, const Prim<NM, D>& Pl,
                        const Prim<NM, D>& Pr, const Flux<NM, D>& FL, const Flux<NM, D>& FR, int dir, double dt,
                        double dx, State<NM, D>& Uh, Prim<NM, D>& Ph)
{
    double rhs[NM];
    alpha_rhs_coefficients<NM, D>(M, A.Pe, A.ck, rhs);
    const double factor = 0.5 * dt / dx;
    Uh = U;
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
    Ph = c2p<NM, D, IL>(M, Uh);
    enforce_positive_primitive<NM, D>(Ph);
}

template<int NM, int D, bool IL = false>
DHD void stage_b(const Mats& M, const State<NM, D>& U, const CellA<NM, D>& A, const Prim<NM, D>& Pe_lo,
                 const Prim<NM, D>& Pe_hi, bool end, int dir, double dt, double dx, State<NM, D>& Uh,
                 Prim<NM, D>& Ph)
{
    if (end) {
        Uh = U;
        Ph = A.Pe;
        return;
    }
    Prim<NM, D> Pl, Pr;
    reconstruct_cell_faces<NM, D>(Pe_lo, A.Pe, Pe_hi, Pl, Pr);
    Flux<NM, D> FL, FR;
    face_flux<NM, D, IL>(M, Pl, dir, FL);
    face_flux<NM, D, IL>(M, Pr, dir, FR);
    stage_b_update<NM, D, IL>(M, U, A, Pl, Pr, FL, FR, dir, dt, dx, Uh, Ph);
}

// One face state of stage C: the conservative state of the reconstructed
// half-step primitive Pf, repaired, and its primitive.  The staged kernel
// runs it as one thread per face state.
template<int NM, int D, bool IL = false>
DHD void face_state(const Mats& M, const Prim<NM, D>& Pf, State<NM, D>& S, Prim<NM, D>& P)
{
    S = repair<NM, D, IL>(M, p2c<NM, D, IL>(M, Pf));
    P = c2p<NM, D, IL>(M, S);
}

// Stage C: the half-step face states of cell i (U_left_half[i],
// U_right_half[i]) and their primitives (the cons_to_prim of PL_face /
// PR_face and of hllc_flux_normal).
template<int NM, int D, bool IL = false>
DHD void stage_c(const Mats& M, const State<NM, D>& U, const CellA<NM, D>& A, const Prim<NM, D>& Ph,
                 const Prim<NM, D>& Ph_lo, const Prim<NM, D>& Ph_hi, bool end, State<NM, D>& LS,
                 State<NM, D>& RS, Prim<NM, D>& PLS, Prim<NM, D>& PRS)
{
    if (end) {
        LS = U;
        RS = U;
        PLS = A.P;
        PRS = A.P;
        return;
    }
    Prim<NM, D> Lh, Rh;
    reconstruct_cell_faces<NM, D>(Ph_lo, Ph, Ph_hi, Lh, Rh);
    face_state<NM, D, IL>(M, Lh, LS, PLS);
    face_state<NM, D, IL>(M, Rh, RS, PRS);
}

// Stage D output per face.
template<int NM, int D>
struct FaceD {
    Flux<NM, D> F;
    double fv;       // face velocity s*
    double af[NM];   // upwind alpha flux (sweep_core.hpp:119-127)
};

// Stage D: face between cell i (UL = RS_i) and cell i+1 (UR = LS_{i+1}).
template<int NM, int D, bool IL = false>
DHD bool stage_d(const Mats& M, const State<NM, D>& UL, const Prim<NM, D>& PL, const State<NM, D>& UR,
                 const Prim<NM, D>& PR, int dir, FaceD<NM, D>& out)
{
    const bool ok = hllc_flux<NM, D, IL>(M, UL, UR, PL, PR, dir, out.F, out.fv);
    const double* up = (out.fv >= 0.0) ? PL.alpha : PR.alpha;
#pragma unroll
    for (int k = 0; k < NM; ++k) out.af[k] = up[k] * out.fv;
    return ok;
}

// Stage E: conservative update + repair, then the non-conservative alpha
// update + repair (sweep_core.hpp:96-148).  lo / hi are the faces i-1|i and
// i|i+1; first / last mark the line's end cells, whose outer face copies the
// inner one (F[0] = F[1], F[n] = F[n-1]) and whose outer alpha flux is the
// cell-centred fraction times that face velocity.
template<int NM, int D, bool IL = false>
DHD void stage_e(const Mats& M, const State<NM, D>& U, const CellA<NM, D>& A, const FaceD<NM, D>* lo,
                 const FaceD<NM, D>* hi, bool first, bool last, double dt, double dx, State<NM, D>& out)
{
    const FaceD<NM, D>& Flo = first ? *hi : *lo;
    const FaceD<NM, D>& Fhi = last ? *lo : *hi;
    const double lambda = dt / dx;
    out = U;
#pragma unroll
    for (int k = 0; k < NM; ++k) out.m[k] -= lambda * (Fhi.F.m[k] - Flo.F.m[k]);
#pragma unroll
    for (int d = 0; d < D; ++d) out.mom[d] -= lambda * (Fhi.F.mom[d] - Flo.F.mom[d]);
    out.E -= lambda * (Fhi.F.E - Flo.F.E);

    // The fraction update reads only A and the faces, not the repaired
    // state, so it is formed before the first repair: only alpha_new stays
    // live across that call.
    double af_lo[NM], af_hi[NM];
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        af_lo[k] = first ? A.P.alpha[k] * Flo.fv : Flo.af[k];
        af_hi[k] = last ? A.P.alpha[k] * Fhi.fv : Fhi.af[k];
    }
    double rhs[NM];
    alpha_rhs_coefficients<NM, D>(M, A.P, A.ck, rhs);
    const double div_u = (Fhi.fv - Flo.fv) / dx;
    double alpha_new[NM];
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        alpha_new[k] = A.P.alpha[k];
        alpha_new[k] -= lambda * (af_hi[k] - af_lo[k]);
        alpha_new[k] += dt * rhs[k] * div_u;
    }
    sanitise_alpha<NM>(alpha_new, 0.0);

    out = repair<NM, D, IL>(M, out);
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) out.a[k] = alpha_new[k];
    out = repair<NM, D, IL>(M, out);
}

// CFL candidate of one cell (dim::compute_dt_cfl body, src/dim/solver/cfl.hpp:
// 46-62, and the unsplit variant :94-115): the smallest cfl*dx_d/wave_speed
// over the axes (or cfl/spectral_sum); +inf when no axis contributes.
// P = cons_to_prim(U); ck: rhs_sound_speeds of P (stage A has them), or
// nullptr.
template<int NM, int D, bool IL = false>
DHD double cfl_candidate(const Mats& M, const State<NM, D>& U, const Prim<NM, D>& P, const double* dx,
                         double cfl, bool unsplit, const double* ck = nullptr)
{
    const double c = sound<NM, IL>(M, total_density<NM, D>(U), P.p, P.alpha, P.rho, ck);
    double best = HUGE_VAL;
    if (unsplit) {
        double spectral_sum = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) spectral_sum += (fabs(P.vel[d]) + c) / dx[d];
        if (spectral_sum > 1e-14) best = cfl / spectral_sum;
        return best;
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const double wave_speed = fabs(P.vel[d]) + c;
        if (wave_speed > 1e-14) best = dmin(best, cfl * dx[d] / wave_speed);
    }
    return best;
}

}  // namespace dimgpu
