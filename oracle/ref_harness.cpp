// ref_harness.cpp — TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own header-only DIM step (SegunOwoeye/
// diffuse_vs_GFM_MMS, include path = the reference project root) into
// oracle/_ref/libdimref.so with the reference's compiler flags
// (g++ -std=c++17 -O2 -fopenmp, no -march, so no FMA contraction).
// Nothing from the reference is copied here: this file only converts between
// the library's SoA layout (include/dimgpu.h) and the reference's AoS
// std::vector<dim::State<DIM>> and calls the reference functions.
//
// Used by tests/ (golden vectors, parity), by __graft_entry__.smoke() as a
// checker, and by bench.py's reference arm as the timed CPU baseline.
#include <omp.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "src/app/io/conservation_report.hpp"
#include "src/dim/solver/advance_step.hpp"
#include "src/io/dim_write_csv.hpp"

#include "dimgpu.h"

namespace {

thread_local std::string g_err;

dim::EOSParams make_params(const dimgpu_desc* d)
{
    dim::EOSParams p;
    for (int k = 0; k < d->nmat; ++k) {
        ::EOSParams m{};
        m.kind = static_cast<EOSKind>(d->mat[k].kind);
        m.gamma = d->mat[k].gamma;
        m.p_inf = d->mat[k].p_inf;
        p.material.push_back(m);
    }
    return p;
}

const char* bc_name(int b)
{
    switch (b) {
        case DIMGPU_BC_REFLECTIVE: return "reflective";
        case DIMGPU_BC_NONREFLECTIVE: return "nonreflective";
        default: return "transmissive";
    }
}

const char* lambda_name(int l)
{
    switch (l) {
        case DIMGPU_LAMBDA_ALLAIRE: return "allaire";
        case DIMGPU_LAMBDA_EQUAL_VELOCITY: return "equal_velocity";
        default: return "kapila";
    }
}

template<int DIM>
Config<DIM> make_cfg(const dimgpu_desc* d)
{
    Config<DIM> cfg;
    for (int a = 0; a < DIM; ++a) {
        cfg.bc_lo[a] = bc_name(d->bc_lo[a]);
        cfg.bc_hi[a] = bc_name(d->bc_hi[a]);
    }
    cfg.time_update = (d->time_update == DIMGPU_TIME_UNSPLIT) ? "unsplit" : "split";
    cfg.dim_lambda_model = lambda_name(d->lambda_model);
    cfg.dim_alpha_source_floor = d->alpha_source_floor;
    cfg.interface_method = "DIM";
    return cfg;
}

template<int DIM>
int nvar(int nmat) { return 2 * nmat + DIM; }

// Cell `i` of a strided buffer: component c at base[c * stride + i].
template<int DIM>
dim::State<DIM> load_state(const double* base, size_t stride, size_t i, int nmat)
{
    dim::State<DIM> U = dim::make_state<DIM>(nmat);
    int c = 0;
    for (int k = 0; k < nmat; ++k) U.partial_mass[k] = base[(c++) * stride + i];
    for (int d = 0; d < DIM; ++d) U.mom[d] = base[(c++) * stride + i];
    U.E = base[(c++) * stride + i];
    for (int k = 0; k < nmat - 1; ++k) U.alpha[k] = base[(c++) * stride + i];
    return U;
}

template<int DIM>
void store_state(double* base, size_t stride, size_t i, const dim::State<DIM>& U, int nmat)
{
    int c = 0;
    for (int k = 0; k < nmat; ++k) base[(c++) * stride + i] = U.partial_mass[k];
    for (int d = 0; d < DIM; ++d) base[(c++) * stride + i] = U.mom[d];
    base[(c++) * stride + i] = U.E;
    for (int k = 0; k < nmat - 1; ++k) base[(c++) * stride + i] = U.alpha[k];
}

// Primitive record: rho[nmat], alpha[nmat], vel[DIM], p.
template<int DIM>
void store_prim(double* out, const dim::Primitive<DIM>& P, int nmat)
{
    int c = 0;
    for (int k = 0; k < nmat; ++k) out[c++] = P.rho[k];
    for (int k = 0; k < nmat; ++k) out[c++] = P.alpha[k];
    for (int d = 0; d < DIM; ++d) out[c++] = P.vel[d];
    out[c++] = P.p;
}

template<int DIM>
dim::Primitive<DIM> load_prim(const double* in, int nmat)
{
    dim::Primitive<DIM> P{};
    P.rho.assign(nmat, 0.0);
    P.alpha.assign(nmat, 0.0);
    int c = 0;
    for (int k = 0; k < nmat; ++k) P.rho[k] = in[c++];
    for (int k = 0; k < nmat; ++k) P.alpha[k] = in[c++];
    for (int d = 0; d < DIM; ++d) P.vel[d] = in[c++];
    P.p = in[c++];
    return P;
}

size_t ncells(const dimgpu_desc* d)
{
    size_t n = 1;
    for (int a = 0; a < d->dim; ++a) n *= static_cast<size_t>(d->N[a]);
    return n;
}

template<int DIM>
std::array<int, DIM> grid_n(const dimgpu_desc* d)
{
    std::array<int, DIM> N{};
    for (int a = 0; a < DIM; ++a) N[a] = d->N[a];
    return N;
}

template<int DIM>
std::array<double, DIM> grid_dx(const dimgpu_desc* d)
{
    std::array<double, DIM> dx{};
    for (int a = 0; a < DIM; ++a) dx[a] = d->dx[a];
    return dx;
}

template<int DIM>
std::vector<dim::State<DIM>> load_field(const dimgpu_desc* d, const double* soa)
{
    const size_t n = ncells(d);
    std::vector<dim::State<DIM>> U(n);
    for (size_t i = 0; i < n; ++i) U[i] = load_state<DIM>(soa, n, i, d->nmat);
    return U;
}

template<int DIM>
void store_field(const dimgpu_desc* d, double* soa, const std::vector<dim::State<DIM>>& U)
{
    const size_t n = ncells(d);
    for (size_t i = 0; i < n; ++i) store_state<DIM>(soa, n, i, U[i], d->nmat);
}

template<int DIM>
int advance_impl(const dimgpu_desc* d, const double* in, double* out, double cfl,
                 double dt_max, int nsteps, double* dt_out, double* phase_s)
{
    const auto params = make_params(d);
    const auto cfg = make_cfg<DIM>(d);
    const auto N = grid_n<DIM>(d);
    const auto dx = grid_dx<DIM>(d);
    std::vector<dim::State<DIM>> U = load_field<DIM>(d, in);
    for (int s = 0; s < nsteps; ++s) {
        dim::StepResult<DIM> r = dim::advance_one_step<DIM>(U, N, dx, params, cfg, cfl, dt_max);
        U = r.U_new;
        if (dt_out) dt_out[s] = r.dt;
        if (phase_s) {
            phase_s[0] += r.phase_timings.cfl_seconds;
            phase_s[1] += r.phase_timings.sweep_seconds;
            phase_s[2] += r.phase_timings.boundary_seconds;
        }
    }
    store_field<DIM>(d, out, U);
    return 0;
}

#define DISPATCH_DIM(d, ...)                                    \
    switch ((d)->dim) {                                         \
        case 1: { constexpr int D = 1; __VA_ARGS__; } break;    \
        case 2: { constexpr int D = 2; __VA_ARGS__; } break;    \
        case 3: { constexpr int D = 3; __VA_ARGS__; } break;    \
        default: g_err = "bad dim"; return 1;                   \
    }

#define GUARD(...)                                              \
    try { __VA_ARGS__ } catch (const std::exception& e) {       \
        g_err = e.what(); return 1;                             \
    }

} // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

void ref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

int ref_max_threads(void) { return omp_get_max_threads(); }

// nsteps calls of dim::advance_one_step with constant cfl / dt_max.
// phase_s (may be NULL) accumulates {cfl, sweep, boundary} seconds.
int ref_advance(const dimgpu_desc* d, const double* soa_in, double* soa_out, double cfl,
                double dt_max, int nsteps, double* dt_out, double* phase_s)
{
    GUARD(DISPATCH_DIM(d, return advance_impl<D>(d, soa_in, soa_out, cfl, dt_max, nsteps, dt_out, phase_s));)
    return 0;
}

// dim::compute_dt_cfl / compute_dt_cfl_unsplit over a SoA field.
int ref_compute_dt_cfl(const dimgpu_desc* d, const double* soa, double cfl, double dt_max,
                       double* dt_out)
{
    GUARD(DISPATCH_DIM(d, {
        const auto params = make_params(d);
        const auto cfg = make_cfg<D>(d);
        const auto U = load_field<D>(d, soa);
        const auto dx = grid_dx<D>(d);
        *dt_out = (cfg.time_update == "unsplit")
            ? dim::compute_dt_cfl_unsplit<D>(U, dx, params, cfg.dim_lambda_model, cfl, dt_max)
            : dim::compute_dt_cfl<D>(U, dx, params, cfg.dim_lambda_model, cfl, dt_max);
    });)
    return 0;
}

// One dim::sweep_direction_dispatch (no boundary fill).
int ref_sweep_direction(const dimgpu_desc* d, int dir, double dt, const double* soa_in,
                        double* soa_out)
{
    GUARD(DISPATCH_DIM(d, {
        const auto params = make_params(d);
        const auto cfg = make_cfg<D>(d);
        const auto U = load_field<D>(d, soa_in);
        std::vector<dim::State<D>> next(U.size());
        dim::sweep_direction_dispatch<D>(dir, U, grid_n<D>(d), grid_dx<D>(d), params, dt,
                                         cfg.dim_alpha_source_floor, cfg.dim_lambda_model, next);
        store_field<D>(d, soa_out, next);
    });)
    return 0;
}

// dim::apply_boundary_conditions in place.
int ref_apply_boundary_conditions(const dimgpu_desc* d, double* soa)
{
    GUARD(DISPATCH_DIM(d, {
        const auto params = make_params(d);
        const auto cfg = make_cfg<D>(d);
        auto U = load_field<D>(d, soa);
        dim::apply_boundary_conditions<D>(U, grid_n<D>(d), cfg, params);
        store_field<D>(d, soa, U);
    });)
    return 0;
}

// ---- per-function known-answer generators (n independent records) --------
// States are packed record-major here: record i at U[i*V .. i*V+V-1].

int ref_cons_to_prim(const dimgpu_desc* d, int n, const double* U, double* P)
{
    GUARD(DISPATCH_DIM(d, {
        const auto params = make_params(d);
        const int V = nvar<D>(d->nmat);
        const int PV = 2 * d->nmat + D + 1;
        for (int i = 0; i < n; ++i) {
            const auto s = load_state<D>(U + (size_t)i * V, 1, 0, d->nmat);
            store_prim<D>(P + (size_t)i * PV, dim::cons_to_prim<D>(s, params), d->nmat);
        }
    });)
    return 0;
}

int ref_prim_to_cons(const dimgpu_desc* d, int n, const double* P, double* U)
{
    GUARD(DISPATCH_DIM(d, {
        const auto params = make_params(d);
        const int V = nvar<D>(d->nmat);
        const int PV = 2 * d->nmat + D + 1;
        for (int i = 0; i < n; ++i) {
            const auto p = load_prim<D>(P + (size_t)i * PV, d->nmat);
            store_state<D>(U + (size_t)i * V, 1, 0, dim::prim_to_cons<D>(p, params), d->nmat);
        }
    });)
    return 0;
}

int ref_repair_state(const dimgpu_desc* d, int n, double* U)
{
    GUARD(DISPATCH_DIM(d, {
        const auto params = make_params(d);
        const int V = nvar<D>(d->nmat);
        for (int i = 0; i < n; ++i) {
            auto s = load_state<D>(U + (size_t)i * V, 1, 0, d->nmat);
            dim::repair_state<D>(s, params);
            store_state<D>(U + (size_t)i * V, 1, 0, s, d->nmat);
        }
    });)
    return 0;
}

// in record: rho_total, e, alpha[nmat], rho[nmat]  ->  p
int ref_mixture_pressure(const dimgpu_desc* d, int n, const double* in, double* p)
{
    GUARD({
        const auto params = make_params(d);
        const int nm = d->nmat;
        const int R = 2 + 2 * nm;
        for (int i = 0; i < n; ++i) {
            const double* r = in + (size_t)i * R;
            std::vector<double> a(r + 2, r + 2 + nm), rho(r + 2 + nm, r + 2 + 2 * nm);
            p[i] = dim::MixtureEOS::pressure_from_internal_energy(r[0], r[1], a, rho, params);
        }
    })
    return 0;
}

// in record: rho_total, p, alpha[nmat], rho[nmat]  ->  c (generic, lambda model)
int ref_mixture_sound_speed(const dimgpu_desc* d, int n, const double* in, double* c)
{
    GUARD({
        const auto params = make_params(d);
        const int nm = d->nmat;
        const int R = 2 + 2 * nm;
        const std::string lm = lambda_name(d->lambda_model);
        for (int i = 0; i < n; ++i) {
            const double* r = in + (size_t)i * R;
            std::vector<double> a(r + 2, r + 2 + nm), rho(r + 2 + nm, r + 2 + 2 * nm);
            c[i] = dim::MixtureEOS::generic_mixture_sound_speed(r[0], r[1], a, rho, params, lm);
        }
    })
    return 0;
}

// primitive record -> rhs[nmat]
int ref_alpha_rhs(const dimgpu_desc* d, int n, const double* P, double* rhs)
{
    GUARD(DISPATCH_DIM(d, {
        const auto params = make_params(d);
        const int PV = 2 * d->nmat + D + 1;
        for (int i = 0; i < n; ++i) {
            const auto p = load_prim<D>(P + (size_t)i * PV, d->nmat);
            const auto r = dim::alpha_rhs_coefficients<D>(p, params, 1e-12, d->alpha_source_floor,
                                                          lambda_name(d->lambda_model));
            for (int k = 0; k < d->nmat; ++k) rhs[(size_t)i * d->nmat + k] = r[k];
        }
    });)
    return 0;
}

// hllc_flux_normal along axis `dir`: out record = flux[nmat+DIM+1], s*.
int ref_hllc(const dimgpu_desc* d, int n, int dir, const double* UL, const double* UR, double* out)
{
    GUARD(DISPATCH_DIM(d, {
        const auto params = make_params(d);
        const int V = nvar<D>(d->nmat);
        const int F = d->nmat + D + 2;
        std::array<double, D> normal{};
        normal[dir] = 1.0;
        for (int i = 0; i < n; ++i) {
            const auto l = load_state<D>(UL + (size_t)i * V, 1, 0, d->nmat);
            const auto r = load_state<D>(UR + (size_t)i * V, 1, 0, d->nmat);
            const auto res = dim::hllc_flux_normal<D>(l, r, params, normal, lambda_name(d->lambda_model));
            double* o = out + (size_t)i * F;
            int c = 0;
            for (int k = 0; k < d->nmat; ++k) o[c++] = res.flux.partial_mass[k];
            for (int a = 0; a < D; ++a) o[c++] = res.flux.mom[a];
            o[c++] = res.flux.E;
            o[c++] = res.face_velocity;
        }
    });)
    return 0;
}

// dim::solve_line on one line of n cells (record-major in/out).
int ref_solve_line(const dimgpu_desc* d, int n, int dir, double dt, double dx,
                   const double* U_in, double* U_out)
{
    GUARD(DISPATCH_DIM(d, {
        const auto params = make_params(d);
        const int V = nvar<D>(d->nmat);
        std::vector<dim::State<D>> in(n), out;
        for (int i = 0; i < n; ++i) in[i] = load_state<D>(U_in + (size_t)i * V, 1, 0, d->nmat);
        dim::solve_line<D>(in, out, dx, dt, params, dir, d->alpha_source_floor,
                           lambda_name(d->lambda_model));
        for (int i = 0; i < n; ++i) store_state<D>(U_out + (size_t)i * V, 1, 0, out[i], d->nmat);
    });)
    return 0;
}

int ref_boundary_flux(const dimgpu_desc* d, const double* soa, double* out)
{
    GUARD(DISPATCH_DIM(d, {
        const auto params = make_params(d);
        const auto U = load_field<D>(d, soa);
        const auto t = app_io::compute_dim_boundary_flux<D>(U, grid_n<D>(d), grid_dx<D>(d), params);
        int q = 0;
        for (int k = 0; k < d->nmat; ++k) out[q++] = t.material_mass[k];
        out[q++] = t.mass;
        for (int a = 0; a < D; ++a) out[q++] = t.momentum[a];
        out[q++] = t.energy;
    });)
    return 0;
}

// dim::write_csv (src/io/dim_write_csv.hpp:15-125) of a SoA field.
int ref_write_csv(const dimgpu_desc* d, const double* soa, const double* domain_min, const double* domain_max,
                  const char* filename)
{
    GUARD(DISPATCH_DIM(d, {
        const auto params = make_params(d);
        const auto U = load_field<D>(d, soa);
        std::array<double, D> lo{}, hi{};
        for (int a = 0; a < D; ++a) {
            lo[a] = domain_min[a];
            hi[a] = domain_max[a];
        }
        dim::write_csv<D>(filename, U, grid_n<D>(d), lo, hi, params);
    });)
    return 0;
}

} // extern "C"
