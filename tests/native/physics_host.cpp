// physics_host.cpp — test harness: the device arithmetic (dim_physics.h and
// the per-cell stages of dim_line.h) compiled for the host with g++, exposed
// with the same record layouts as the oracle so the CPU test suite can check
// the kernel arithmetic bit for bit against the oracle and the reference.
// The stage driver below walks a line the way the CUDA kernel walks a tile.
#include <cstdlib>
#include <cstring>
#include <vector>

// Operation counts (dimgpu::OpCount) of everything this harness runs.
static long long g_opcount[16];
#define DIMGPU_OPCOUNT(k) (++g_opcount[(k)])
#define DIMGPU_OPCOUNT_ADD(k, n) (g_opcount[(k)] += (n))

#include "../../diffuse_vs_gfm_mms_b200/csrc/dim_line.h"
#include "../../diffuse_vs_gfm_mms_b200/csrc/dim_mixed.h"
#include "../../diffuse_vs_gfm_mms_b200/csrc/euler_physics.h"
#include "../../diffuse_vs_gfm_mms_b200/csrc/fastdiv.h"
#include "dimgpu.h"

using namespace dimgpu;

namespace {

Mats mats_of(const dimgpu_desc* d)
{
    Mats M;
    int kind[kMaxMat];
    double g[kMaxMat], pi[kMaxMat];
    for (int k = 0; k < d->nmat; ++k) {
        kind[k] = d->mat[k].kind;
        g[k] = d->mat[k].gamma;
        pi[k] = d->mat[k].p_inf;
    }
    fill_mats(M, d->nmat, kind, g, pi, d->lambda_model, d->alpha_source_floor);
    return M;
}

template<int NM, int D>
void load(const double* r, State<NM, D>& U, size_t stride = 1)
{
    int q = 0;
    for (int k = 0; k < NM; ++k) U.m[k] = r[(q++) * stride];
    for (int d = 0; d < D; ++d) U.mom[d] = r[(q++) * stride];
    U.E = r[(q++) * stride];
    for (int k = 0; k < NM - 1; ++k) U.a[k] = r[(q++) * stride];
}

template<int NM, int D>
void store(double* r, const State<NM, D>& U, size_t stride = 1)
{
    int q = 0;
    for (int k = 0; k < NM; ++k) r[(q++) * stride] = U.m[k];
    for (int d = 0; d < D; ++d) r[(q++) * stride] = U.mom[d];
    r[(q++) * stride] = U.E;
    for (int k = 0; k < NM - 1; ++k) r[(q++) * stride] = U.a[k];
}

template<int NM, int D>
void store_prim(double* o, const Prim<NM, D>& P)
{
    int q = 0;
    for (int k = 0; k < NM; ++k) o[q++] = P.rho[k];
    for (int k = 0; k < NM; ++k) o[q++] = P.alpha[k];
    for (int d = 0; d < D; ++d) o[q++] = P.vel[d];
    o[q++] = P.p;
}

template<int NM, int D>
void load_prim(const double* in, Prim<NM, D>& P)
{
    int q = 0;
    for (int k = 0; k < NM; ++k) P.rho[k] = in[q++];
    for (int k = 0; k < NM; ++k) P.alpha[k] = in[q++];
    for (int d = 0; d < D; ++d) P.vel[d] = in[q++];
    P.p = in[q++];
}

// One line through stages A..E (the kernel's tile schedule, untiled).
// IL = true: the inlined forms of the routines, as the staged kernels run
// them (their common paths inline, the rest through the out-of-line forms).
template<int NM, int D, bool IL = true>
int solve_line_stages(const Mats& M, int n, const State<NM, D>* U, State<NM, D>* out, int dir, double dt,
                      double dx)
{
    if (n == 1) {
        out[0] = U[0];
        return 0;
    }
    std::vector<CellA<NM, D>> A(n);
    std::vector<State<NM, D>> Uh(n), LS(n), RS(n);
    std::vector<Prim<NM, D>> Ph(n), PLS(n), PRS(n);
    std::vector<FaceD<NM, D>> F(n);
    auto is_end = [&](int i) { return i == 0 || i == n - 1 || n < 3; };
    for (int i = 0; i < n; ++i) stage_a<NM, D, IL>(M, U[i], A[i]);
    for (int i = 0; i < n; ++i) {
        const Prim<NM, D>& lo = A[i > 0 ? i - 1 : i].Pe;
        const Prim<NM, D>& hi = A[i < n - 1 ? i + 1 : i].Pe;
        stage_b<NM, D, IL>(M, U[i], A[i], lo, hi, is_end(i), dir, dt, dx, Uh[i], Ph[i]);
    }
    for (int i = 0; i < n; ++i) {
        const Prim<NM, D>& lo = Ph[i > 0 ? i - 1 : i];
        const Prim<NM, D>& hi = Ph[i < n - 1 ? i + 1 : i];
        stage_c<NM, D, IL>(M, U[i], A[i], Ph[i], lo, hi, is_end(i), LS[i], RS[i], PLS[i], PRS[i]);
    }
    for (int i = 0; i + 1 < n; ++i)
        if (!stage_d<NM, D, IL>(M, RS[i], PRS[i], LS[i + 1], PLS[i + 1], dir, F[i])) return DIMGPU_E_NONFINITE;
    for (int i = 0; i < n; ++i) {
        const FaceD<NM, D>* lo = i > 0 ? &F[i - 1] : nullptr;
        const FaceD<NM, D>* hi = i < n - 1 ? &F[i] : nullptr;
        stage_e<NM, D, IL>(M, U[i], A[i], lo, hi, i == 0, i == n - 1, dt, dx, out[i]);
    }
    return 0;
}

// The mixed-precision line schedule (stage A, stage_b_mixed, face_mixed +
// stage_d_mixed, stage E), untiled.
template<int NM, int D>
int solve_line_mixed(const Mats& M, int n, const State<NM, D>* U, State<NM, D>* out, int dir, double dt, double dx)
{
    if (n == 1) {
        out[0] = U[0];
        return 0;
    }
    std::vector<CellA<NM, D>> A(n);
    std::vector<Prim<NM, D>> Ph(n);
    std::vector<FaceD<NM, D>> F(n);
    auto is_end = [&](int i) { return i == 0 || i == n - 1 || n < 3; };
    for (int i = 0; i < n; ++i) stage_a_mixed<NM, D>(M, U[i], A[i]);
    for (int i = 0; i < n; ++i) {
        const Prim<NM, D>& lo = A[i > 0 ? i - 1 : i].Pe;
        const Prim<NM, D>& hi = A[i < n - 1 ? i + 1 : i].Pe;
        stage_b_mixed<NM, D>(M, U[i], A[i], lo, hi, is_end(i), dir, dt, dx, Ph[i]);
    }
    for (int i = 0; i + 1 < n; ++i) {
        State<NM, D> UL, UR;
        Prim<NM, D> PL, PR;
        if (is_end(i)) { UL = U[i]; PL = A[i].P; }
        else face_mixed<NM, D>(M, Ph[i - 1], Ph[i], Ph[i + 1], true, UL, PL);
        if (is_end(i + 1)) { UR = U[i + 1]; PR = A[i + 1].P; }
        else face_mixed<NM, D>(M, Ph[i], Ph[i + 1], Ph[i + 2], false, UR, PR);
        if (!stage_d_mixed<NM, D>(M, UL, PL, UR, PR, dir, F[i])) return DIMGPU_E_NONFINITE;
    }
    for (int i = 0; i < n; ++i) {
        const FaceD<NM, D>* lo = i > 0 ? &F[i - 1] : nullptr;
        const FaceD<NM, D>* hi = i < n - 1 ? &F[i] : nullptr;
        stage_e<NM, D>(M, U[i], A[i], lo, hi, i == 0, i == n - 1, dt, dx, out[i]);
    }
    return 0;
}


// The Euler sweep of one line through the device stages of euler_physics.h
// (the order euler_sweep_kernel evaluates them), untiled.
template<int D>
int euler_line(const Mats& M, int n, const EState<D>* U, EState<D>* out, int dir, double dt, double dx,
               int ends_copy)
{
    std::vector<EPrim<D>> P(n), Ph(n);
    std::vector<EState<D>> LS(n), RS(n), F(n);
    bool ok = true;
    for (int i = 0; i < n; ++i) {
        P[i] = e_cons_to_prim<D>(M, U[i]);
        e_enforce_prim<D>(P[i]);
    }
    for (int i = 0; i < n; ++i) {
        if (i == 0 || i == n - 1) { Ph[i] = P[i]; continue; }
        const EState<D> Ul = e_face_state<D>(M, P[i - 1], P[i], P[i + 1], false);
        const EState<D> Ur = e_face_state<D>(M, P[i - 1], P[i], P[i + 1], true);
        EState<D> Uh;
        ok &= e_hancock<D>(M, U[i], Ul, Ur, dir, dt, dx, Uh);
        Ph[i] = e_cons_to_prim<D>(M, Uh);
        e_enforce_prim<D>(Ph[i]);
    }
    for (int i = 0; i < n; ++i) {
        if (i == 0 || i == n - 1) { LS[i] = U[i]; RS[i] = U[i]; }
        else {
            LS[i] = e_face_state<D>(M, Ph[i - 1], Ph[i], Ph[i + 1], false);
            RS[i] = e_face_state<D>(M, Ph[i - 1], Ph[i], Ph[i + 1], true);
        }
        e_enforce<D>(M, LS[i]);
        e_enforce<D>(M, RS[i]);
    }
    for (int i = 0; i + 1 < n; ++i) ok &= e_hllc<D>(M, RS[i], LS[i + 1], dir, F[i]);
    for (int i = 0; i < n; ++i) {
        if (i == 0 || i == n - 1) {
            if (ends_copy) out[i] = U[i];
            else {
                out[i].rho = 0.0;
                for (int d = 0; d < D; ++d) out[i].mom[d] = 0.0;
                out[i].E = 0.0;
            }
            continue;
        }
        e_update<D>(M, U[i], F[i - 1], F[i], dt, dx, out[i]);
    }
    return ok ? 0 : DIMGPU_E_NONFINITE;
}

template<int D>
int euler_sweep_impl(const dimgpu_desc* d, int dir, double dt, const double* in, double* out, int ends_copy)
{
    const Mats M = mats_of(d);
    size_t total = 1, stride[3] = {1, 1, 1};
    for (int a = 0; a < D; ++a) total *= (size_t)d->N[a];
    for (int a = 1; a < D; ++a) stride[a] = stride[a - 1] * (size_t)d->N[a - 1];
    const int n = d->N[dir];
    const size_t lines = total / (size_t)n;
    int rc = 0;
    std::vector<EState<D>> lin(n), lout(n);
    for (size_t line = 0; line < lines; ++line) {
        int idx[3] = {0, 0, 0};
        size_t tmp = line;
        for (int a = D - 1; a >= 0; --a) {
            if (a == dir) continue;
            idx[a] = (int)(tmp % (size_t)d->N[a]);
            tmp /= (size_t)d->N[a];
        }
        size_t base = 0;
        for (int a = 0; a < D; ++a) base += (size_t)idx[a] * stride[a];
        for (int i = 0; i < n; ++i) {
            const size_t c = base + (size_t)i * stride[dir];
            lin[i].rho = in[c];
            for (int a = 0; a < D; ++a) lin[i].mom[a] = in[(1 + a) * total + c];
            lin[i].E = in[(1 + D) * total + c];
        }
        const int r = euler_line<D>(M, n, lin.data(), lout.data(), dir, dt, d->dx[dir], ends_copy);
        if (r) rc = r;
        for (int i = 0; i < n; ++i) {
            const size_t c = base + (size_t)i * stride[dir];
            out[c] = lout[i].rho;
            for (int a = 0; a < D; ++a) out[(1 + a) * total + c] = lout[i].mom[a];
            out[(1 + D) * total + c] = lout[i].E;
        }
    }
    return rc;
}

template<int D>
int euler_hllc_impl(const dimgpu_desc* d, int n, int dir, const double* UL, const double* UR, double* out)
{
    const Mats M = mats_of(d);
    const int V = 2 + D;
    int rc = 0;
    for (int i = 0; i < n; ++i) {
        EState<D> a, b, F;
        a.rho = UL[i * V];
        b.rho = UR[i * V];
        for (int k = 0; k < D; ++k) {
            a.mom[k] = UL[i * V + 1 + k];
            b.mom[k] = UR[i * V + 1 + k];
        }
        a.E = UL[i * V + 1 + D];
        b.E = UR[i * V + 1 + D];
        if (!e_hllc<D>(M, a, b, dir, F)) { rc = DIMGPU_E_NONFINITE; continue; }
        out[i * V] = F.rho;
        for (int k = 0; k < D; ++k) out[i * V + 1 + k] = F.mom[k];
        out[i * V + 1 + D] = F.E;
    }
    return rc;
}

template<int NM, int D>
int sweep_impl(const dimgpu_desc* d, int dir, double dt, const double* in, double* out)
{
    const Mats M = mats_of(d);
    size_t total = 1, stride[3] = {1, 1, 1};
    for (int a = 0; a < D; ++a) total *= (size_t)d->N[a];
    for (int a = 1; a < D; ++a) stride[a] = stride[a - 1] * (size_t)d->N[a - 1];
    const int n = d->N[dir];
    const size_t lines = total / (size_t)n;
    int rc = 0;
    std::vector<State<NM, D>> lin(n), lout(n);
    for (size_t line = 0; line < lines; ++line) {
        int idx[3] = {0, 0, 0};
        size_t tmp = line;
        for (int a = D - 1; a >= 0; --a) {
            if (a == dir) continue;
            idx[a] = (int)(tmp % (size_t)d->N[a]);
            tmp /= (size_t)d->N[a];
        }
        size_t base = 0;
        for (int a = 0; a < D; ++a) base += (size_t)idx[a] * stride[a];
        for (int i = 0; i < n; ++i) load<NM, D>(in + base + (size_t)i * stride[dir], lin[i], total);
        const int r = d->precision == DIMGPU_PRECISION_MIXED
                          ? solve_line_mixed<NM, D>(M, n, lin.data(), lout.data(), dir, dt, d->dx[dir])
                          : solve_line_stages<NM, D>(M, n, lin.data(), lout.data(), dir, dt, d->dx[dir]);
        if (r) rc = r;
        for (int i = 0; i < n; ++i) store<NM, D>(out + base + (size_t)i * stride[dir], lout[i], total);
    }
    return rc;
}

#define DISPATCH(d, FN, ...)                                                           \
    do {                                                                              \
        switch ((d)->nmat * 10 + (d)->dim) {                                          \
            case 11: return FN<1, 1>(__VA_ARGS__);                                    \
            case 12: return FN<1, 2>(__VA_ARGS__);                                    \
            case 13: return FN<1, 3>(__VA_ARGS__);                                    \
            case 21: return FN<2, 1>(__VA_ARGS__);                                    \
            case 22: return FN<2, 2>(__VA_ARGS__);                                    \
            case 23: return FN<2, 3>(__VA_ARGS__);                                    \
            case 31: return FN<3, 1>(__VA_ARGS__);                                    \
            case 32: return FN<3, 2>(__VA_ARGS__);                                    \
            case 33: return FN<3, 3>(__VA_ARGS__);                                    \
            case 41: return FN<4, 1>(__VA_ARGS__);                                    \
            case 42: return FN<4, 2>(__VA_ARGS__);                                    \
            case 43: return FN<4, 3>(__VA_ARGS__);                                    \
            default: return DIMGPU_E_INVALID_ARG;                                     \
        }                                                                             \
    } while (0)

template<int NM, int D>
int c2p_impl(const dimgpu_desc* d, int n, const double* U, double* P)
{
    const Mats M = mats_of(d);
    for (int i = 0; i < n; ++i) {
        State<NM, D> s;
        Prim<NM, D> p;
        load<NM, D>(U + (size_t)i * (2 * NM + D), s);
        cons_to_prim<NM, D>(M, s, p);
        store_prim<NM, D>(P + (size_t)i * (2 * NM + D + 1), p);
    }
    return 0;
}

template<int NM, int D>
int p2c_impl(const dimgpu_desc* d, int n, const double* P, double* U)
{
    const Mats M = mats_of(d);
    for (int i = 0; i < n; ++i) {
        State<NM, D> s;
        Prim<NM, D> p;
        load_prim<NM, D>(P + (size_t)i * (2 * NM + D + 1), p);
        prim_to_cons<NM, D>(M, p, s);
        store<NM, D>(U + (size_t)i * (2 * NM + D), s);
    }
    return 0;
}

template<int NM, int D>
int repair_impl(const dimgpu_desc* d, int n, double* U)
{
    const Mats M = mats_of(d);
    for (int i = 0; i < n; ++i) {
        State<NM, D> s;
        load<NM, D>(U + (size_t)i * (2 * NM + D), s);
        repair_state<NM, D>(M, s);
        store<NM, D>(U + (size_t)i * (2 * NM + D), s);
    }
    return 0;
}

template<int NM, int D>
int pressure_impl(const dimgpu_desc* d, int n, const double* in, double* p)
{
    const Mats M = mats_of(d);
    for (int i = 0; i < n; ++i) {
        const double* r = in + (size_t)i * (2 + 2 * NM);
        p[i] = pressure_from_internal_energy<NM>(M, r[0], r[1], r + 2, r + 2 + NM);
    }
    return 0;
}

template<int NM, int D>
int sound_impl(const dimgpu_desc* d, int n, const double* in, double* c)
{
    const Mats M = mats_of(d);
    for (int i = 0; i < n; ++i) {
        const double* r = in + (size_t)i * (2 + 2 * NM);
        c[i] = generic_mixture_sound_speed<NM>(M, r[0], r[1], r + 2, r + 2 + NM);
    }
    return 0;
}

// The generic sound speed with and without stage A's material speeds ck
// (rhs_sound_speeds of a primitive with the record's rho_k and p).
template<int NM, int D>
int sound_ck_impl(const dimgpu_desc* d, int n, const double* in, double* with_ck, double* without_ck)
{
    const Mats M = mats_of(d);
    for (int i = 0; i < n; ++i) {
        const double* r = in + (size_t)i * (2 + 2 * NM);
        Prim<NM, D> P{};
        P.p = r[1];
        for (int k = 0; k < NM; ++k) P.rho[k] = r[2 + NM + k];
        double ck[NM];
        rhs_sound_speeds<NM, D>(M, P, ck);
        with_ck[i] = sound_speed_generic<NM>(M, r[0], r[1], mix_of<NM>(r + 2, r + 2 + NM), ck);
        without_ck[i] = sound_speed_generic<NM>(M, r[0], r[1], mix_of<NM>(r + 2, r + 2 + NM), nullptr);
    }
    return 0;
}

template<int NM, int D>
int rhs_impl(const dimgpu_desc* d, int n, const double* P, double* rhs)
{
    const Mats M = mats_of(d);
    for (int i = 0; i < n; ++i) {
        Prim<NM, D> p;
        load_prim<NM, D>(P + (size_t)i * (2 * NM + D + 1), p);
        double ck[NM];
        rhs_sound_speeds<NM, D>(M, p, ck);
        alpha_rhs_coefficients<NM, D>(M, p, ck, rhs + (size_t)i * NM);
    }
    return 0;
}

template<int NM, int D>
int hllc_impl(const dimgpu_desc* d, int n, int dir, const double* UL, const double* UR, double* out)
{
    const Mats M = mats_of(d);
    for (int i = 0; i < n; ++i) {
        State<NM, D> l, r;
        Prim<NM, D> pl, pr;
        load<NM, D>(UL + (size_t)i * (2 * NM + D), l);
        load<NM, D>(UR + (size_t)i * (2 * NM + D), r);
        cons_to_prim<NM, D>(M, l, pl);
        cons_to_prim<NM, D>(M, r, pr);
        Flux<NM, D> F;
        double s;
        if (!hllc_flux<NM, D>(M, l, r, pl, pr, dir, F, s)) return DIMGPU_E_NONFINITE;
        double* o = out + (size_t)i * (NM + D + 2);
        int q = 0;
        for (int k = 0; k < NM; ++k) o[q++] = F.m[k];
        for (int a = 0; a < D; ++a) o[q++] = F.mom[a];
        o[q++] = F.E;
        o[q++] = s;
    }
    return 0;
}

template<int NM, int D>
int line_impl(const dimgpu_desc* d, int n, int dir, double dt, double dx, const double* in, double* out)
{
    const Mats M = mats_of(d);
    std::vector<State<NM, D>> a(n), b(n);
    for (int i = 0; i < n; ++i) load<NM, D>(in + (size_t)i * (2 * NM + D), a[i]);
    const int rc = solve_line_stages<NM, D>(M, n, a.data(), b.data(), dir, dt, dx);
    for (int i = 0; i < n; ++i) store<NM, D>(out + (size_t)i * (2 * NM + D), b[i]);
    return rc;
}

}  // namespace

extern "C" {

int host_cons_to_prim(const dimgpu_desc* d, int n, const double* U, double* P) { DISPATCH(d, c2p_impl, d, n, U, P); }
int host_prim_to_cons(const dimgpu_desc* d, int n, const double* P, double* U) { DISPATCH(d, p2c_impl, d, n, P, U); }
int host_repair_state(const dimgpu_desc* d, int n, double* U) { DISPATCH(d, repair_impl, d, n, U); }
int host_mixture_pressure(const dimgpu_desc* d, int n, const double* in, double* p) { DISPATCH(d, pressure_impl, d, n, in, p); }
int host_mixture_sound_speed(const dimgpu_desc* d, int n, const double* in, double* c) { DISPATCH(d, sound_impl, d, n, in, c); }
int host_alpha_rhs(const dimgpu_desc* d, int n, const double* P, double* rhs) { DISPATCH(d, rhs_impl, d, n, P, rhs); }
int host_sound_ck(const dimgpu_desc* d, int n, const double* in, double* with_ck, double* without_ck)
{
    DISPATCH(d, sound_ck_impl, d, n, in, with_ck, without_ck);
}
int host_hllc(const dimgpu_desc* d, int n, int dir, const double* UL, const double* UR, double* out)
{
    DISPATCH(d, hllc_impl, d, n, dir, UL, UR, out);
}
int host_solve_line(const dimgpu_desc* d, int n, int dir, double dt, double dx, const double* in, double* out)
{
    DISPATCH(d, line_impl, d, n, dir, dt, dx, in, out);
}
int host_euler_sweep_direction(const dimgpu_desc* d, int dir, double dt, const double* in, double* out,
                               int ends_copy)
{
    switch (d->dim) {
        case 1: return euler_sweep_impl<1>(d, dir, dt, in, out, ends_copy);
        case 2: return euler_sweep_impl<2>(d, dir, dt, in, out, ends_copy);
        case 3: return euler_sweep_impl<3>(d, dir, dt, in, out, ends_copy);
        default: return DIMGPU_E_INVALID_ARG;
    }
}
int host_euler_hllc(const dimgpu_desc* d, int n, int dir, const double* UL, const double* UR, double* out)
{
    switch (d->dim) {
        case 1: return euler_hllc_impl<1>(d, n, dir, UL, UR, out);
        case 2: return euler_hllc_impl<2>(d, n, dir, UL, UR, out);
        case 3: return euler_hllc_impl<3>(d, n, dir, UL, UR, out);
        default: return DIMGPU_E_INVALID_ARG;
    }
}
int host_sweep_direction(const dimgpu_desc* d, int dir, double dt, const double* in, double* out)
{
    DISPATCH(d, sweep_impl, d, dir, dt, in, out);
}

// q[i] = x[i] / d and r[i] = x[i] % d through the staged kernels' FastDiv.
int host_fastdiv(unsigned d, int n, const unsigned* x, unsigned* q, unsigned* r)
{
    if (d == 0) return DIMGPU_E_INVALID_ARG;
    dimgpu::FastDiv f;
    f.set(d);
    for (int i = 0; i < n; ++i) {
        q[i] = f.div(x[i]);
        r[i] = x[i] - q[i] * d;
    }
    return DIMGPU_OK;
}

// Copies the operation counts into out[0 .. n) and, if reset, zeroes them.
int host_opcounts(long long* out, int n, int reset)
{
    for (int k = 0; k < n && k < 16; ++k) out[k] = g_opcount[k];
    if (reset) std::memset(g_opcount, 0, sizeof(g_opcount));
    return dimgpu::kOpCountN;
}

}  // extern "C"
