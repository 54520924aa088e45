// dim_physics.h — per-state arithmetic of the DIM step, shared by the CUDA
// kernels (compiled by nvcc with -fmad=false) and by the host-side equivalence
// tests (compiled by g++ without -march, so without FMA either).
//
// Every function reproduces the rounding of the reference's double-precision
// code (SegunOwoeye/diffuse_vs_GFM_MMS; file:line cited per function): the
// same operations in the same order, IEEE division and square root, and
// libstdc++'s std::max / std::min semantics.  What differs is what is NOT
// computed; each shortcut below returns the bit pattern the reference would
// have returned:
//
//  * sanitise_alpha skips its divisions when the sum is exactly 1.0 (x/1.0 == x);
//  * repair_state computes its "pressure before" bisection only on the branch
//    that reads it (src/dim/primitives.hpp:413-434), and skips the energy floor
//    arithmetic when a rigorous upper bound of the floor is already below E;
//  * the mixture-pressure bisection (src/dim/eos.hpp:77-143) decides each
//    doubling / bisection step from a closed-form bracket of the (affine)
//    residual and evaluates the literal residual only inside a guard band
//    around the termination window; see MixtureBisection below.
#pragma once

#include <cfloat>
#include <cmath>

// DHD: small helpers, inlined.  DNI: the large routines every sweep calls at
// many sites (pressure recovery, cons_to_prim, prim_to_cons, repair_state,
// the generic sound speed), kept as single out-of-line copies on the device
// so the sweep kernel's code fits the instruction cache.  The out-of-line
// copies take and return their records by value (the *_v functions): a
// record passed by reference or pointer must live in addressable (local)
// memory, which turns every call into local stores and loads; by value it
// stays in registers.  Inline wrappers with the by-reference signatures sit
// in front of them.  Each out-of-line copy wraps an always-inlined body
// (pressure_recover, sound_speed_generic, cons_to_prim_t, prim_to_cons_t,
// repair_state_t): a kernel that calls a routine from one site only (the
// staged sweep's per-face-state kernels) inlines the body and pays no call
// (no argument moves, no callee-saved registers spilled to local memory).
#ifdef __CUDACC__
#define DHD __host__ __device__ __forceinline__
#define DNI __host__ __device__ __noinline__
#else
#define DHD inline
#define DNI inline
#endif

namespace dimgpu {

constexpr int kMaxMat = 4;

// Operation counts of a host profiling build: the host harness defines
// DIMGPU_OPCOUNT(k) to count the events below; every other build compiles
// the counts away.
enum OpCount {
    kOpRecover,       // mixture pressure recoveries
    kOpDouble,        // doubling steps of the upper bracket
    kOpCertain,       // bisection steps decided by the certain bracket
    kOpLiteral,       // literal residual evaluations
    kOpNotFast,       // recoveries without a certain bracket
    kOpRepair,        // repair_state calls
    kOpRepairBisect,  // repair_state "pressure before" recoveries
    kOpRepairFloor,   // repair_state exact energy floors
    kOpSound,         // generic mixture sound speeds
    kOpDoubleSkipped, // doubling steps skipped in one step (bracket-decided)
    kOpCountN
};
#ifndef DIMGPU_OPCOUNT
#define DIMGPU_OPCOUNT(k) ((void)0)
#define DIMGPU_OPCOUNT_ADD(k, n) ((void)0)
#endif

// ---- constants per material (filled on the host from dimgpu_desc) --------
struct Mats {
    double gamma[kMaxMat];
    double p_inf[kMaxMat];
    double gm1[kMaxMat];      // gamma - 1.0            (same value the reference forms)
    double gpinf[kMaxMat];    // gamma * p_inf          (same value the reference forms)
    double einf_ub[kMaxMat];  // upper bound of (1e-10 + gamma p_inf) / (gamma - 1)
    int stiff[kMaxMat];       // 1 = stiffened gas, 0 = ideal gas
    int nmat;
    int lambda_model;         // 0 kapila, 1 allaire, 2 equal_velocity
    double alpha_source_floor;
};

// ---- src/math/numerical_safety.hpp -----------------------------------------
DHD bool fin(double x) { return fabs(x) <= DBL_MAX; }
DHD double dmax(double a, double b) { return (a < b) ? b : a; }   // std::max
DHD double dmin(double a, double b) { return (b < a) ? b : a; }   // std::min
// numerical_safety.hpp:12-18
DHD double clamp_min(double x, double tol = 1e-10) { return fin(x) ? dmax(x, tol) : tol; }
// numerical_safety.hpp:21-24
DHD double finite_or(double x, double fb = 0.0) { return fin(x) ? x : fb; }
// numerical_safety.hpp:27-39
DHD double safe_denom(double d, double tol = 1e-10)
{
    if (!fin(d)) return (d < 0.0) ? -tol : tol;
    if (fabs(d) < tol) return (d < 0.0) ? -tol : tol;
    return d;
}
// numerical_safety.hpp:41-45
DHD double safe_div(double n, double d, double tol = 1e-10) { return finite_or(n) / safe_denom(d, tol); }

// ---- state records -----------------------------------------------------------
template<int NM, int D>
struct State {
    double m[NM];
    double mom[D];
    double E;
    double a[NM > 1 ? NM - 1 : 1];
};

template<int NM, int D>
struct Prim {
    double rho[NM];
    double alpha[NM];
    double vel[D];
    double p;
};

template<int NM, int D>
struct Flux {
    double m[NM];
    double mom[D];
    double E;
};

// ---- per-material laws (src/euler/eos.hpp) -----------------------------------
// IdealGasEOS::internal_energy eos.hpp:488-495, StiffenedGasEOS eos.hpp:601-609
DHD double mat_ie(const Mats& M, int k, double rho, double p)
{
    return M.stiff[k] ? safe_div(p + M.gpinf[k], M.gm1[k] * rho) : safe_div(p, M.gm1[k] * rho);
}

// pressure<1>(U) with zero momentum, eos.hpp:450-466 / 555-572.  The kinetic
// term is 0.5 * safe_div(0.0, rho) == +0.0 for the clamped rho, and E - (+0.0)
// == E for every E, so it is dropped.
DHD double mat_p_rest(const Mats& M, int k, double UE)
{
    const double p_raw = M.stiff[k] ? (M.gm1[k] * UE - M.gpinf[k]) : (M.gm1[k] * UE);
    return clamp_min(p_raw);
}

// sound_speed<1>(U) with zero momentum, eos.hpp:469-479 / 575-585
DHD double mat_c_rest(const Mats& M, int k, double Urho, double UE)
{
    const double rho = clamp_min(Urho);
    const double p = mat_p_rest(M, k, UE);
    return M.stiff[k] ? sqrt(M.gamma[k] * safe_div(p + M.p_inf[k], rho))
                      : sqrt(M.gamma[k] * safe_div(p, rho));
}

// MixtureEOS::material_sound_speed, src/dim/eos.hpp:29-40
DHD double material_sound_speed(const Mats& M, int k, double rho, double p)
{
    const double Urho = clamp_min(rho);
    const double UE = Urho * mat_ie(M, k, Urho, p);
    return mat_c_rest(M, k, Urho, UE);
}

// MixtureEOS::material_energy_pressure_derivative, src/dim/eos.hpp:42-57
DHD double material_energy_pressure_derivative(const Mats& M, int k, double rho, double p)
{
    rho = clamp_min(rho);
    p = clamp_min(p);
    const double dp = dmax(1e-6 * dmax(fabs(p), 1.0), 1e-8);
    const double p_lo = dmax(p - dp, 1e-12);
    const double p_hi = p + dp;
    const double e_lo = mat_ie(M, k, rho, p_lo);
    const double e_hi = mat_ie(M, k, rho, p_hi);
    return dmax(safe_div(e_hi - e_lo, p_hi - p_lo, 1e-14), 1e-14);
}

// MixtureEOS::mixture_internal_energy_density, src/dim/eos.hpp:59-75
template<int NM>
DHD double mixture_ie_density(const Mats& M, double p, const double* alpha, const double* rho)
{
    double energy_density = 0.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        const double alpha_k = dmax(finite_or(alpha[k]), 0.0);
        const double rho_k = clamp_min(rho[k]);
        const double p_k = clamp_min(p);
        energy_density += alpha_k * rho_k * mat_ie(M, k, rho_k, p_k);
    }
    return finite_or(energy_density);
}

// ---- mixture pressure recovery, src/dim/eos.hpp:77-143 -----------------------
//
// The residual f(p) = sum_k (a_k r_k) * (pc + c_k) / d_k - T (pc = max(p,1e-10),
// c_k = gamma_k p_inf_k or 0, d_k = safe_denom((gamma_k-1) r_k)) is affine in
// pc with non-negative terms, so its computed value lies within
// 8u * (A pc + B + |T|) of the exact line A pc + B - T, where
// A = sum a_k r_k / d_k and B = sum a_k r_k c_k / d_k (u = 2^-53; nmat <= 4).
// The bracket below uses kRel = 256u, which also covers the rounding of A, B
// and of the two bounds.  Outside [P_lo, P_hi] the literal residual is
// certainly < -thresh (p < P_lo) or > thresh (p > P_hi): the bisection step
// it drives, and the termination test (false), are known without evaluating
// it.  Inside, and wherever a quantity could overflow, the literal residual
// is evaluated exactly as the reference does.
template<int NM>
struct MixtureBisection {
    double ar[NM];   // alpha_k * rho_k
    double den[NM];  // safe_denom((gamma_k - 1) * rho_k)
    double T;

    DHD double literal(const Mats& M, double p) const
    {
        const double pc = clamp_min(p);
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NM; ++k) {
            const double num = M.stiff[k] ? (pc + M.gpinf[k]) : pc;
            s += ar[k] * (finite_or(num) / den[k]);
        }
        return finite_or(s) - T;
    }
};

// Volume fractions and material densities of a mixture state, passed by value.
template<int NM>
struct MixVec {
    double alpha[NM];
    double rho[NM];
};

template<int NM>
DHD MixVec<NM> mix_of(const double* alpha, const double* rho)
{
    MixVec<NM> x;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        x.alpha[k] = alpha[k];
        x.rho[k] = rho[k];
    }
    return x;
}

template<int NM>
DNI double pressure_from_internal_energy_v(const Mats& M, double rho_total, double e, MixVec<NM> x);

// FULL = false is the inlined form: it carries only the certain-bracket
// path, which every recovery of the benchmarked fields takes, and hands a
// state without a certain bracket to the out-of-line full form (which
// recomputes it from the same inputs: the same result, less inlined code).
template<int NM, bool FULL = true>
DHD double pressure_recover(const Mats& M, double rho_total_in, double e_in, MixVec<NM> x)
{
    const double* alpha = x.alpha;
    const double* rho = x.rho;
    DIMGPU_OPCOUNT(kOpRecover);
    double rho_total = clamp_min(rho_total_in);
    double e = finite_or(e_in);
    const double target = finite_or(rho_total * e);

    double fallback_pressure = 0.0;
    const double ek = target / rho_total;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        // material_pressure_from_density_energy, src/dim/eos.hpp:16-27
        const double Urho = clamp_min(clamp_min(rho[k]));
        const double UE = Urho * dmax(ek, 0.0);
        fallback_pressure += dmax(finite_or(alpha[k]), 0.0) * mat_p_rest(M, k, UE);
    }
    fallback_pressure = clamp_min(fallback_pressure);

    MixtureBisection<NM> R;
    R.T = target;
    double A = 0.0, B = 0.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        const double alpha_k = dmax(finite_or(alpha[k]), 0.0);
        const double rho_k = clamp_min(rho[k]);
        R.ar[k] = alpha_k * rho_k;
        R.den[k] = safe_denom(M.gm1[k] * rho_k);
        const double w = R.ar[k] / R.den[k];
        A += w;
        if (M.stiff[k]) B += w * M.gpinf[k];
    }
    const double thresh = 1e-10 * dmax(1.0, target);

    // Certain-decision bracket (see the comment above MixtureBisection).
    constexpr double kRel = 256.0 * 1.1102230246251565e-16;
    constexpr double kInvOneMinusRel = 1.0 / (1.0 - kRel);
    constexpr double kInvOnePlusRel = 1.0 / (1.0 + kRel);
    bool fast = fin(A) && fin(B) && A > 1e-200 && (B + fabs(target)) < 1e290;
    double P_lo = 0.0, P_hi = 0.0, P_fin = 0.0;
    if (fast) {
        // One division: the bounds are products with 1/A.  Each product is
        // within 4u of the quotient it replaces (the rounding of 1/A, of the
        // constant 1/(1 -+ kRel) and of two products), far inside the 1e-13
        // relative widening that follows, so the bounds stay outer bounds;
        // P_fin only guards against overflow and needs no precision.
        const double rA = 1.0 / A;
        const double slack = kRel * (B + fabs(target));
        P_hi = (thresh + target - B + slack) * (rA * kInvOneMinusRel);
        P_lo = (target - B - thresh - slack) * (rA * kInvOnePlusRel);
        P_hi = P_hi + fabs(P_hi) * 1e-13 + 1e-300;
        P_lo = P_lo - fabs(P_lo) * 1e-13 - 1e-300;
        P_fin = 1e290 * rA;
        fast = fin(P_hi) && fin(P_lo);
    }
    if constexpr (!FULL) {
        if (!fast) return pressure_from_internal_energy_v<NM>(M, rho_total_in, e_in, x);
    }
    if (!fast) DIMGPU_OPCOUNT(kOpNotFast);
    // status: -1 certainly f < -thresh, +1 certainly f > thresh, 0 unknown
    auto status = [&](double p) -> int {
        if (!fast) return 0;
        const double pc = clamp_min(p);
        if (!(pc < P_fin)) return 0;
        if (pc > P_hi) return 1;
        if (pc < P_lo) return -1;
        return 0;
    };

    double lo = 1e-12;
    double hi = dmax(1.0, fallback_pressure);

    // flo / fhi: their signs and finiteness are all the reference reads.
    bool flo_ok;
    int s = status(lo);
    if (s < 0) flo_ok = true;
    else if (s > 0) flo_ok = false;
    else {
        DIMGPU_OPCOUNT(kOpLiteral);
        const double flo = R.literal(M, lo);
        flo_ok = fin(flo) && flo <= 0.0;
    }

    bool fhi_neg, fhi_finite;
    s = status(hi);
    if (s != 0) { fhi_neg = s < 0; fhi_finite = true; }
    else {
        DIMGPU_OPCOUNT(kOpLiteral);
        const double fhi = R.literal(M, hi);
        fhi_finite = fin(fhi);
        fhi_neg = fhi_finite && fhi < 0.0;
    }
    // Doublings the bracket decides (hi * 2^n < min(P_lo, P_fin): status -1)
    // are skipped in one step: hi * 2^n is exact, and the first n with
    // hi * 2^n >= Q is ilogb(Q) - ilogb(hi) or one more (hi >= 1 and Q > hi
    // are normal numbers here).  The loop resumes at that doubling, with the
    // same 80-doubling cap.
    int n0 = 0;
    if (s < 0) {
        const double Q = dmin(P_lo, P_fin);
        int m = ilogb(Q) - ilogb(hi);
        if (ldexp(hi, m) < Q) ++m;
        n0 = m - 1 < 80 ? m - 1 : 80;
        hi = ldexp(hi, n0);
        DIMGPU_OPCOUNT_ADD(kOpDoubleSkipped, n0);
    }
    for (int n = n0; n < 80 && fhi_finite && fhi_neg; ++n) {
        DIMGPU_OPCOUNT(kOpDouble);
        hi *= 2.0;
        s = status(hi);
        if (s != 0) { fhi_neg = s < 0; fhi_finite = true; }
        else {
            DIMGPU_OPCOUNT(kOpLiteral);
            const double fhi = R.literal(M, hi);
            fhi_finite = fin(fhi);
            fhi_neg = fhi_finite && fhi < 0.0;
        }
    }
    const bool fhi_ok = fhi_finite && !fhi_neg;  // fhi >= 0.0

    if (!flo_ok || !fhi_ok) return clamp_min(fallback_pressure);

    // Inside the loop lo <= mid <= hi, all finite and positive, so
    // clamp_min(mid) == max(mid, 1e-10); below P_fin the certain decisions
    // are two compares and two selects.  When P_lo > 1e-10 the clamp cannot
    // change either decision (mid < 1e-10 is below P_lo clamped or not), so
    // the dependency chain of a step is add, multiply, compare, select.
    const bool fast_loop = fast && clamp_min(hi) < P_fin;
    if constexpr (!FULL) {
        if (!fast_loop) return pressure_from_internal_energy_v<NM>(M, rho_total_in, e_in, x);
    }
    const bool no_clamp = fast_loop && P_lo > 1e-10;
    for (int n = 0; n < 80; ++n) {
        const double mid = 0.5 * (lo + hi);
        if (no_clamp) {
            const bool up = mid > P_hi, dn = mid < P_lo;
            if (up || dn) {
                DIMGPU_OPCOUNT(kOpCertain);
                hi = up ? mid : hi;
                lo = dn ? mid : lo;
                continue;
            }
        }
        else if (fast_loop) {
            const double pc = dmax(mid, 1e-10);
            const bool up = pc > P_hi, dn = pc < P_lo;
            if (up || dn) {
                DIMGPU_OPCOUNT(kOpCertain);
                hi = up ? mid : hi;
                lo = dn ? mid : lo;
                continue;
            }
        }
        else {
            s = status(mid);
            if (s > 0) { DIMGPU_OPCOUNT(kOpCertain); hi = mid; continue; }
            if (s < 0) { DIMGPU_OPCOUNT(kOpCertain); lo = mid; continue; }
        }
        DIMGPU_OPCOUNT(kOpLiteral);
        const double fmid = R.literal(M, mid);
        if (!fin(fmid)) return clamp_min(fallback_pressure);
        if (fabs(fmid) <= thresh) return clamp_min(mid);
        if (fmid > 0.0) hi = mid;
        else lo = mid;
    }
    return clamp_min(0.5 * (lo + hi));
}

template<int NM>
DNI double pressure_from_internal_energy_v(const Mats& M, double rho_total, double e, MixVec<NM> x)
{
    return pressure_recover<NM>(M, rho_total, e, x);
}

template<int NM>
DHD double pressure_from_internal_energy(const Mats& M, double rho_total, double e, const double* alpha,
                                         const double* rho)
{
    return pressure_from_internal_energy_v<NM>(M, rho_total, e, mix_of<NM>(alpha, rho));
}

// material_sound_speed(M, k, clamp_min(rho_raw), p_arg), taken from ck[k]
// where the caller already evaluated it on the same arguments: ck from
// rhs_sound_speeds of the same primitive, which passes max(finite_or(x),
// 1e-12) for rho_k and p, and clamp_min leaves x itself as well when x is
// finite and at least 1e-10 (p_ok: the raw pressure is; p_arg is then the
// raw pressure, clamped or not).  ck == nullptr: always evaluated.
DHD double material_speed_or(const Mats& M, int k, double rho_raw, double p_arg, bool p_ok, const double* ck)
{
    if (ck && p_ok && fin(rho_raw) && rho_raw >= 1e-10) return ck[k];
    return material_sound_speed(M, k, clamp_min(rho_raw), p_arg);
}

// MixtureEOS::mixture_sound_speed, src/dim/eos.hpp:195-221
template<int NM>
DHD double mixture_sound_speed(const Mats& M, double rho_total, double p, const double* alpha,
                               const double* rho, const double* ck = nullptr)
{
    rho_total = clamp_min(rho_total);
    const bool p_ok = fin(p) && p >= 1e-10;
    p = clamp_min(p);
    double beta_mix = 0.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        const double rho_k = clamp_min(rho[k]);
        const double c = material_speed_or(M, k, rho[k], p, p_ok, ck);
        beta_mix += dmax(finite_or(alpha[k]), 0.0) / safe_denom(rho_k * c * c, 1e-14);
    }
    return sqrt(1.0 / (rho_total * safe_denom(beta_mix, 1e-14)));
}

// MixtureEOS::generic_mixture_sound_speed, src/dim/eos.hpp:223-275
// ck: the material sound speeds of the same primitive (rhs_sound_speeds),
// reused where their arguments agree (material_speed_or), or nullptr.
template<int NM>
DHD double sound_speed_generic(const Mats& M, double rho_total, double p, MixVec<NM> x,
                               const double* ck = nullptr)
{
    const double* alpha = x.alpha;
    const double* rho = x.rho;
    DIMGPU_OPCOUNT(kOpSound);
    if (M.lambda_model == 0) return mixture_sound_speed<NM>(M, rho_total, p, alpha, rho, ck);
    const bool p_ok = fin(p) && p >= 1e-10;
    double sound_speed[NM], xi[NM];
    double xi_mix = 0.0, inverse_sound_sum = 0.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        const double alpha_k = dmax(finite_or(alpha[k]), 0.0);
        const double rho_k = clamp_min(rho[k]);
        sound_speed[k] = material_speed_or(M, k, rho[k], p, p_ok, ck);
        xi[k] = rho_k * material_energy_pressure_derivative(M, k, rho_k, p);
        xi_mix += alpha_k * xi[k];
        inverse_sound_sum += alpha_k / safe_denom(sound_speed[k], 1e-14);
    }
    xi_mix = safe_denom(xi_mix, 1e-14);
    inverse_sound_sum = safe_denom(inverse_sound_sum, 1e-14);
    double rho_c_squared = 0.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        const double alpha_k = dmax(finite_or(alpha[k]), 0.0);
        double lambda_k = 1.0;
        if (M.lambda_model == 2)
            lambda_k = safe_div(1.0 / safe_denom(sound_speed[k], 1e-14), inverse_sound_sum, 1e-14);
        rho_c_squared += lambda_k * alpha_k * xi[k] * sound_speed[k] * sound_speed[k] / xi_mix;
    }
    return sqrt(dmax(rho_c_squared / clamp_min(rho_total), 1e-14));
}

template<int NM>
DNI double generic_mixture_sound_speed_v(const Mats& M, double rho_total, double p, MixVec<NM> x)
{
    return sound_speed_generic<NM>(M, rho_total, p, x);
}

template<int NM>
DHD double generic_mixture_sound_speed(const Mats& M, double rho_total, double p, const double* alpha,
                                       const double* rho)
{
    return generic_mixture_sound_speed_v<NM>(M, rho_total, p, mix_of<NM>(alpha, rho));
}

// ---- src/dim/primitives.hpp ----------------------------------------------------
// full_alpha_from_independent, primitives.hpp:18-42
template<int NM, int D>
DHD void full_alpha(const State<NM, D>& U, double* alpha)
{
    double sum = 0.0;
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) {
        alpha[k] = U.a[k];
        sum += alpha[k];
    }
    alpha[NM - 1] = 1.0 - sum;
}

// sanitise_alpha, primitives.hpp:45-70.  Dividing by a sum of exactly 1.0 is
// the identity, so it is skipped.
template<int NM>
DHD void sanitise_alpha(double* alpha, double alpha_floor)
{
    double sum = 0.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        alpha[k] = finite_or(alpha[k], alpha_floor);
        alpha[k] = dmax(alpha[k], alpha_floor);
        sum += alpha[k];
    }
    if (!fin(sum) || sum <= 0.0) {
#pragma unroll
        for (int k = 0; k < NM; ++k) alpha[k] = 0.0;
        alpha[0] = 1.0;
        return;
    }
    if (sum == 1.0) return;
#pragma unroll
    for (int k = 0; k < NM; ++k) alpha[k] /= sum;
}

// total_density, primitives.hpp:99-108
template<int NM, int D>
DHD double total_density(const State<NM, D>& U)
{
    double r = 0.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) r += finite_or(U.m[k]);
    return r;
}

// cons_to_prim, primitives.hpp:111-162
template<int NM, int D, bool IL>
DHD Prim<NM, D> cons_to_prim_t(const Mats& M, State<NM, D> U)
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
    double p;
    if constexpr (IL) p = pressure_recover<NM, false>(M, rho_total, internal_energy, mix_of<NM>(P.alpha, P.rho));
    else p = pressure_from_internal_energy<NM>(M, rho_total, internal_energy, P.alpha, P.rho);
    P.p = dmax(p, 1e-12);
    return P;
}

template<int NM, int D>
DNI Prim<NM, D> cons_to_prim_v(const Mats& M, State<NM, D> U)
{
    return cons_to_prim_t<NM, D, false>(M, U);
}

template<int NM, int D>
DHD void cons_to_prim(const Mats& M, const State<NM, D>& U, Prim<NM, D>& P)
{
    P = cons_to_prim_v<NM, D>(M, U);
}

// prim_to_cons, primitives.hpp:165-212 (internal_energy_from_pressure,
// src/dim/eos.hpp:146-166, inlined)
template<int NM, int D>
DHD State<NM, D> prim_to_cons_t(const Mats& M, Prim<NM, D> P)
{
    State<NM, D> U;
    sanitise_alpha<NM>(P.alpha, 1e-12);
    double rho_total = 0.0;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        P.rho[k] = dmax(P.rho[k], 1e-12);
        U.m[k] = P.alpha[k] * P.rho[k];
        rho_total += U.m[k];
    }
    rho_total = dmax(rho_total, 1e-12);
    P.p = dmax(P.p, 1e-12);
    double velocity_squared = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        U.mom[d] = rho_total * P.vel[d];
        velocity_squared += P.vel[d] * P.vel[d];
    }
    const double ie = mixture_ie_density<NM>(M, clamp_min(P.p), P.alpha, P.rho) / clamp_min(rho_total);
    U.E = rho_total * ie + 0.5 * rho_total * velocity_squared;
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) U.a[k] = P.alpha[k];
    return U;
}

template<int NM, int D>
DNI State<NM, D> prim_to_cons_v(const Mats& M, Prim<NM, D> P)
{
    return prim_to_cons_t<NM, D>(M, P);
}

template<int NM, int D>
DHD void prim_to_cons(const Mats& M, const Prim<NM, D>& P, State<NM, D>& U)
{
    U = prim_to_cons_v<NM, D>(M, P);
}

// Material sound speeds at a primitive's (rho_k, p) with the floors that
// alpha_rhs_coefficients applies (primitives.hpp:250-254, 295-300): they
// depend on rho and p only, so both calls of alpha_rhs_coefficients on a
// cell (with P and with enforce_positive_primitive(P)) share them.
template<int NM, int D>
DHD void rhs_sound_speeds(const Mats& M, const Prim<NM, D>& P, double* ck)
{
#pragma unroll
    for (int k = 0; k < NM; ++k)
        ck[k] = material_sound_speed(M, k, dmax(finite_or(P.rho[k]), 1e-12), dmax(finite_or(P.p), 1e-12));
}

// alpha_rhs_coefficients, primitives.hpp:216-322.  ck[] from rhs_sound_speeds
// on a primitive with the same rho and p.
template<int NM, int D>
DHD void alpha_rhs_coefficients(const Mats& M, const Prim<NM, D>& P, const double* ck, double* rhs)
{
    const double floor_ = 1e-12;
#pragma unroll
    for (int k = 0; k < NM; ++k) rhs[k] = P.alpha[k];
    sanitise_alpha<NM>(rhs, 0.0);
    if (M.lambda_model == 1) return;
    if (M.lambda_model == 2) {
        double inverse_sound_sum = 0.0;
        double sound_speed[NM];
#pragma unroll
        for (int k = 0; k < NM; ++k) {
            sound_speed[k] = floor_;
            const double alpha_k = dmax(finite_or(rhs[k]), 0.0);
            if (alpha_k <= floor_ || alpha_k < dmax(M.alpha_source_floor, 0.0)) continue;
            sound_speed[k] = ck[k];
            inverse_sound_sum += alpha_k / safe_denom(sound_speed[k], 1e-14);
        }
        if (inverse_sound_sum <= floor_ || !fin(inverse_sound_sum)) return;
#pragma unroll
        for (int k = 0; k < NM; ++k) {
            const double alpha_k = dmax(finite_or(rhs[k]), 0.0);
            if (alpha_k <= floor_) { rhs[k] = 0.0; continue; }
            const double lambda_k = safe_div(1.0 / safe_denom(sound_speed[k], 1e-14), inverse_sound_sum, 1e-14);
            rhs[k] = alpha_k * lambda_k;
        }
        return;
    }
    const double source_alpha_floor = dmax(M.alpha_source_floor, 0.0);
    double beta_mix = 0.0;
    double ai[NM];
    bool active[NM];
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        ai[k] = floor_;
        active[k] = false;
        const double alpha_k = dmax(finite_or(rhs[k]), 0.0);
        if (alpha_k <= floor_ || alpha_k < source_alpha_floor) continue;
        active[k] = true;
        const double rho_k = dmax(finite_or(P.rho[k]), floor_);
        ai[k] = dmax(rho_k * ck[k] * ck[k], floor_);
        beta_mix += alpha_k / ai[k];
    }
    if (beta_mix <= floor_ || !fin(beta_mix)) return;
    const double q_mix = 1.0 / beta_mix;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        const double alpha_k = dmax(finite_or(rhs[k]), 0.0);
        if (!active[k] || alpha_k <= floor_) { rhs[k] = 0.0; continue; }
        const double K_k = alpha_k * (q_mix / ai[k] - 1.0);
        rhs[k] = alpha_k + K_k;
    }
}

template<int NM, int D>
DNI State<NM, D> repair_state_v(const Mats& M, State<NM, D> U);

// repair_state, primitives.hpp:325-457.  FULL = false is the inlined form:
// it carries only the path where nothing is removed and E clears the energy
// floor's bound, and hands every other state — after the input clamps,
// which are idempotent — to the out-of-line full form.
template<int NM, int D, bool FULL = true>
DHD State<NM, D> repair_state_t(const Mats& M, State<NM, D> U)
{
    DIMGPU_OPCOUNT(kOpRepair);
    const double mass_floor = 1e-12, p_floor = 1e-12, inactive_alpha_floor = 1e-10;
#pragma unroll
    for (int k = 0; k < NM; ++k) U.m[k] = dmax(finite_or(U.m[k]), 0.0);
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) U.a[k] = finite_or(U.a[k]);
#pragma unroll
    for (int d = 0; d < D; ++d) U.mom[d] = finite_or(U.mom[d]);
    U.E = finite_or(U.E);

    // alpha_before (:356-357) and alpha_full (:387-388) are the same
    // sanitised vector: nothing between them touches U.alpha.
    double alpha_full[NM];
    full_alpha<NM, D>(U, alpha_full);
    sanitise_alpha<NM>(alpha_full, 0.0);

    bool remove[NM];
    bool removed_inactive_mass = false;
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        remove[k] = alpha_full[k] <= inactive_alpha_floor && U.m[k] > mass_floor;
        removed_inactive_mass = removed_inactive_mass || remove[k];
    }

    if constexpr (!FULL) {
        // the full form's steps below, on the path that removes nothing:
        // the same total density, the same bound test, the same result
        const double rho_total = total_density<NM, D>(U);
        const double E = finite_or(U.E);
        bool plain = !removed_inactive_mass && fin(rho_total) && rho_total > 0.0;
        if (plain) {
            double msq = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) msq += U.mom[d] * U.mom[d];
            double ub = 0.5 * msq / rho_total * (1.0 + 1e-12);
#pragma unroll
            for (int k = 0; k < NM; ++k) ub += dmax(alpha_full[k], 0.0) * M.einf_ub[k];
            ub = ub * (1.0 + 1e-12) + 1e-290;
            plain = fin(ub) && E >= ub;
        }
        if (!plain) return repair_state_v<NM, D>(M, U);
#pragma unroll
        for (int k = 0; k < NM - 1; ++k) U.a[k] = alpha_full[k];
        U.E = E;
        return U;
    }

    double velocity_before[D];
    double velocity_squared_before = 0.0;
    double pressure_before = 0.0;
    if (removed_inactive_mass) {
        // :348-379, evaluated from the state as it was before the removal
        const double rho_before = dmax(total_density<NM, D>(U), mass_floor);
#pragma unroll
        for (int d = 0; d < D; ++d) {
            velocity_before[d] = safe_div(U.mom[d], rho_before);
            velocity_squared_before += velocity_before[d] * velocity_before[d];
        }
        double rho_material_before[NM];
#pragma unroll
        for (int k = 0; k < NM; ++k) {
            const double alpha_k = dmax(alpha_full[k], inactive_alpha_floor);
            rho_material_before[k] = dmax(safe_div(dmax(U.m[k], 0.0), alpha_k), mass_floor);
        }
        const double kinetic_before = 0.5 * rho_before * velocity_squared_before;
        const double internal_before = safe_div(finite_or(U.E, kinetic_before) - kinetic_before, rho_before);
        DIMGPU_OPCOUNT(kOpRepairBisect);
        pressure_before = dmax(pressure_from_internal_energy<NM>(M, rho_before, internal_before,
                                                                 alpha_full, rho_material_before),
                               p_floor);
    }

#pragma unroll
    for (int k = 0; k < NM - 1; ++k) U.a[k] = alpha_full[k];
#pragma unroll
    for (int k = 0; k < NM; ++k)
        if (remove[k]) U.m[k] = 0.0;

    double rho_total = total_density<NM, D>(U);
    if (!fin(rho_total) || rho_total <= 0.0) {
        int dominant = 0;
#pragma unroll
        for (int k = 1; k < NM; ++k)
            if (alpha_full[k] > alpha_full[dominant]) dominant = k;
#pragma unroll
        for (int k = 0; k < NM; ++k)
            if (k == dominant) U.m[k] = mass_floor;
        rho_total = mass_floor;
    }

    if (removed_inactive_mass) {
#pragma unroll
        for (int d = 0; d < D; ++d) U.mom[d] = rho_total * velocity_before[d];
        double rho_material[NM];
#pragma unroll
        for (int k = 0; k < NM; ++k) {
            const double alpha_k = dmax(alpha_full[k], inactive_alpha_floor);
            rho_material[k] = dmax(safe_div(U.m[k], alpha_k), mass_floor);
        }
        const double ie = mixture_ie_density<NM>(M, clamp_min(pressure_before), alpha_full, rho_material) /
                          clamp_min(rho_total);
        U.E = rho_total * ie + 0.5 * rho_total * velocity_squared_before;
    }

    // Energy floor E >= kinetic + mixture energy at p_floor (:437-456).  Both
    // terms are bounded above without per-component divisions:
    //   kinetic <= 0.5 * |mom|^2 / rho_total (to 1e-12 relative),
    //   alpha_k rho_k e_k(1e-10) <= alpha_k (1e-10 + gamma_k p_inf_k)/(gamma_k - 1)
    // (einf_ub carries a 1e-12 relative margin; the absolute 1e-290 covers
    // squared momenta that underflow while v^2 does not: then kinetic
    // <= 0.5 |mom|^2 * 1e10 < 1e-297).  When E clears the bound,
    // std::max(E, floor) == E and the exact floor need not be formed.
    const double E = finite_or(U.E);
    {
        double msq = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) msq += U.mom[d] * U.mom[d];
        double ub = 0.5 * msq / rho_total * (1.0 + 1e-12);
#pragma unroll
        for (int k = 0; k < NM; ++k) ub += dmax(alpha_full[k], 0.0) * M.einf_ub[k];
        ub = ub * (1.0 + 1e-12) + 1e-290;
        if (fin(ub) && E >= ub) {
            U.E = E;
            return U;
        }
    }
    DIMGPU_OPCOUNT(kOpRepairFloor);
    double velocity_squared = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const double v = safe_div(U.mom[d], rho_total);
        velocity_squared += v * v;  // std::pow(v, 2)
    }
    double rho_material[NM];
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        const double alpha_k = dmax(alpha_full[k], inactive_alpha_floor);
        rho_material[k] = dmax(safe_div(U.m[k], alpha_k), mass_floor);
    }
    const double kinetic = 0.5 * rho_total * velocity_squared;
    const double minimum_internal = mixture_ie_density<NM>(M, p_floor, alpha_full, rho_material);
    U.E = dmax(E, kinetic + minimum_internal);
    return U;
}

template<int NM, int D>
DNI State<NM, D> repair_state_v(const Mats& M, State<NM, D> U)
{
    return repair_state_t<NM, D>(M, U);
}

template<int NM, int D>
DHD void repair_state(const Mats& M, State<NM, D>& U)
{
    U = repair_state_v<NM, D>(M, U);
}

// ---- src/dim/reconstruction/muscl.hpp -----------------------------------------
// core::fv::minmod, src/core/fv/limiters.hpp:9-15
DHD double minmod(double a, double b)
{
    if (a * b <= 0.0) return 0.0;
    return fabs(a) < fabs(b) ? a : b;
}

// enforce_positive_primitive, muscl.hpp:26-40
template<int NM, int D>
DHD void enforce_positive_primitive(Prim<NM, D>& P)
{
#pragma unroll
    for (int k = 0; k < NM; ++k) P.rho[k] = dmax(P.rho[k], 1e-12);
    sanitise_alpha<NM>(P.alpha, 0.0);
    P.p = dmax(P.p, 1e-12);
}

// compute_limited_slope + reconstruct_cell_faces, muscl.hpp:43-112
template<int NM, int D>
DHD void reconstruct_cell_faces(const Prim<NM, D>& PL, const Prim<NM, D>& PC, const Prim<NM, D>& PR,
                                Prim<NM, D>& Lf, Prim<NM, D>& Rf)
{
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        const double s = minmod(PC.rho[k] - PL.rho[k], PR.rho[k] - PC.rho[k]);
        Lf.rho[k] = PC.rho[k] - 0.5 * s;
        Rf.rho[k] = PC.rho[k] + 0.5 * s;
    }
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        const double s = minmod(PC.alpha[k] - PL.alpha[k], PR.alpha[k] - PC.alpha[k]);
        Lf.alpha[k] = PC.alpha[k] - 0.5 * s;
        Rf.alpha[k] = PC.alpha[k] + 0.5 * s;
    }
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const double s = minmod(PC.vel[d] - PL.vel[d], PR.vel[d] - PC.vel[d]);
        Lf.vel[d] = PC.vel[d] - 0.5 * s;
        Rf.vel[d] = PC.vel[d] + 0.5 * s;
    }
    const double s = minmod(PC.p - PL.p, PR.p - PC.p);
    Lf.p = PC.p - 0.5 * s;
    Rf.p = PC.p + 0.5 * s;
    enforce_positive_primitive<NM, D>(Lf);
    enforce_positive_primitive<NM, D>(Rf);
}

// dim::compute_flux_normal, src/dim/flux.hpp:11-43, with the axis normal e_dir
// (norm 1, so n = e_dir; un = sum_d vel_d n_d is formed literally).
template<int NM, int D>
DHD void flux_normal(const State<NM, D>& U, const Prim<NM, D>& P, int dir, Flux<NM, D>& F)
{
    const double rho_total = total_density<NM, D>(U);
    double un = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) un += P.vel[d] * (d == dir ? 1.0 : 0.0);
#pragma unroll
    for (int k = 0; k < NM; ++k) F.m[k] = U.m[k] * un;
#pragma unroll
    for (int d = 0; d < D; ++d) F.mom[d] = rho_total * P.vel[d] * un + P.p * (d == dir ? 1.0 : 0.0);
    F.E = (U.E + P.p) * un;
}

// hancock_predict, muscl.hpp:143-191 (apply_flux_difference :115-140).
// ck: rhs_sound_speeds of Pc.
template<int NM, int D>
DHD void hancock_predict(const Mats& M, const State<NM, D>& Uc, const Prim<NM, D>& Pc, const double* ck,
                         const State<NM, D>& Ul, const State<NM, D>& Ur, const Prim<NM, D>& Pl,
                         const Prim<NM, D>& Pr, int dir, double dt, double dx, State<NM, D>& out)
{
    Flux<NM, D> FL, FR;
    flux_normal<NM, D>(Ul, Pl, dir, FL);
    flux_normal<NM, D>(Ur, Pr, dir, FR);
    const double factor = 0.5 * dt / dx;
    out = Uc;
#pragma unroll
    for (int k = 0; k < NM; ++k) out.m[k] -= factor * (FR.m[k] - FL.m[k]);
#pragma unroll
    for (int d = 0; d < D; ++d) out.mom[d] -= factor * (FR.mom[d] - FL.mom[d]);
    out.E -= factor * (FR.E - FL.E);

    const double u_left = Pl.vel[dir];
    const double u_right = Pr.vel[dir];
    const double div_u = (u_right - u_left) / dx;
    double rhs[NM];
    alpha_rhs_coefficients<NM, D>(M, Pc, ck, rhs);
    double alpha_new[NM];
#pragma unroll
    for (int k = 0; k < NM; ++k) {
        alpha_new[k] = Pc.alpha[k];
        alpha_new[k] -= factor * (Pr.alpha[k] * u_right - Pl.alpha[k] * u_left);
        alpha_new[k] += 0.5 * dt * rhs[k] * div_u;
    }
    sanitise_alpha<NM>(alpha_new, 0.0);
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) out.a[k] = alpha_new[k];
    repair_state<NM, D>(M, out);
}

// ---- src/dim/riemann/hllc.hpp ---------------------------------------------------
// hllc_flux_normal, hllc.hpp:62-195 (star terms :15-41, hll_flux :47-59).
// PL / PR are cons_to_prim(UL) / cons_to_prim(UR), computed by the caller
// once per face state.  Returns false where the reference's require_positive
// throws (non-finite density or pressure, hllc.hpp:88-91).
template<int NM, int D, bool IL = false>
DHD bool hllc_flux(const Mats& M, const State<NM, D>& UL, const State<NM, D>& UR, const Prim<NM, D>& PL,
                   const Prim<NM, D>& PR, int dir, Flux<NM, D>& F, double& s_face)
{
    double rhoL = total_density<NM, D>(UL), rhoR = total_density<NM, D>(UR);
    double pL = PL.p, pR = PR.p;
    if (!fin(rhoL) || !fin(rhoR) || !fin(pL) || !fin(pR)) return false;
    if (rhoL <= 0.0) rhoL = 1e-10;
    if (rhoR <= 0.0) rhoR = 1e-10;
    if (pL <= 0.0) pL = 1e-10;
    if (pR <= 0.0) pR = 1e-10;
    double unL = 0.0, unR = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) unL += PL.vel[d] * (d == dir ? 1.0 : 0.0);
#pragma unroll
    for (int d = 0; d < D; ++d) unR += PR.vel[d] * (d == dir ? 1.0 : 0.0);

    double cL, cR;
    if constexpr (IL) {
        cL = sound_speed_generic<NM>(M, rhoL, pL, mix_of<NM>(PL.alpha, PL.rho));
        cR = sound_speed_generic<NM>(M, rhoR, pR, mix_of<NM>(PR.alpha, PR.rho));
    }
    else {
        cL = generic_mixture_sound_speed<NM>(M, rhoL, pL, PL.alpha, PL.rho);
        cR = generic_mixture_sound_speed<NM>(M, rhoR, pR, PR.alpha, PR.rho);
    }
    const double sL = dmin(unL - cL, unR - cR);
    const double sR = dmax(unL + cL, unR + cR);
    const double numerator = (pR - pL) + rhoL * unL * (sL - unL) - rhoR * unR * (sR - unR);
    const double denom = rhoL * (sL - unL) - rhoR * (sR - unR);
    double s_star = safe_div(numerator, denom);
    if (fabs(pL - pR) < 1e-10 && fabs(unL - unR) < 1e-10) s_star = unL;

    Flux<NM, D> FL, FR;
    flux_normal<NM, D>(UL, PL, dir, FL);
    flux_normal<NM, D>(UR, PR, dir, FR);

    const bool average = !fin(sL) || !fin(sR) || !fin(s_star);
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
    const bool left = (sL <= 0.0 && 0.0 <= s_star);
    const State<NM, D>& UK = left ? UL : UR;
    const Prim<NM, D>& PK = left ? PL : PR;
    const Flux<NM, D>& FK = left ? FL : FR;
    const double rhoK = left ? rhoL : rhoR;
    const double pK = left ? pL : pR;
    const double unK = left ? unL : unR;
    const double sK = left ? sL : sR;

    const double rho_star = rhoK * safe_div(sK - unK, sK - s_star);
    const double E_star = rho_star * (safe_div(UK.E, rhoK) + (s_star - unK) * (s_star + safe_div(pK, rhoK * (sK - unK))));
    s_face = s_star;
    if (rho_star <= 0.0 || !fin(rho_star) || !fin(E_star)) {
        // hll_flux: (sR FL - sL FR + (sL sR) (UR - UL)) * (1 / (sR - sL))
        const double inv = 1.0 / (sR - sL);
        const double sLsR = sL * sR;
#pragma unroll
        for (int k = 0; k < NM; ++k) F.m[k] = inv * ((sR * FL.m[k] - sL * FR.m[k]) + sLsR * (UR.m[k] - UL.m[k]));
#pragma unroll
        for (int d = 0; d < D; ++d)
            F.mom[d] = inv * ((sR * FL.mom[d] - sL * FR.mom[d]) + sLsR * (UR.mom[d] - UL.mom[d]));
        F.E = inv * ((sR * FL.E - sL * FR.E) + sLsR * (UR.E - UL.E));
        return true;
    }
    const double mass_scale = safe_div(rho_star, rhoK);
    const double delta = s_star - unK;
#pragma unroll
    for (int k = 0; k < NM; ++k) F.m[k] = FK.m[k] + sK * (UK.m[k] * mass_scale - UK.m[k]);
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const double u_star = PK.vel[d] + delta * (d == dir ? 1.0 : 0.0);
        F.mom[d] = FK.mom[d] + sK * (rho_star * u_star - UK.mom[d]);
    }
    F.E = FK.E + sK * (E_star - UK.E);
    return true;
}

// Host-side material constants from the descriptor fields.
inline void fill_mats(Mats& M, int nmat, const int* kind, const double* gamma, const double* p_inf,
                      int lambda_model, double alpha_source_floor)
{
    for (int k = 0; k < kMaxMat; ++k) {
        const bool on = k < nmat;
        M.gamma[k] = on ? gamma[k] : 1.4;
        M.p_inf[k] = on ? p_inf[k] : 0.0;
        M.stiff[k] = on ? (kind[k] == 1) : 0;
        M.gm1[k] = M.gamma[k] - 1.0;
        M.gpinf[k] = M.gamma[k] * M.p_inf[k];
        const double num = 1e-10 + (M.stiff[k] ? M.gpinf[k] : 0.0);
        M.einf_ub[k] = num / M.gm1[k] * (1.0 + 1e-12);
    }
    M.nmat = nmat;
    M.lambda_model = lambda_model;
    M.alpha_source_floor = alpha_source_floor;
}

}  // namespace dimgpu
