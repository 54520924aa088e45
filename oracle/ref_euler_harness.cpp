// ref_euler_harness.cpp — TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own single-material sharp-interface step
// (SegunOwoeye/diffuse_vs_GFM_MMS, advance_one_step<DIM, MaterialEOS> of
// src/sim/solver/advance_step.hpp with no level set and one material) into
// oracle/_ref/libeulerref.so with the reference's compiler flags
// (g++ -std=c++17 -O2 -fopenmp, no -march).  Nothing from the reference is
// copied: this file builds a SolverContext<DIM>, converts between the SoA
// layout (rho, mom[0..dim-1], E per cell) and std::vector<Conserved<DIM>>,
// and calls the reference functions.  Used by tests/ to pin the C
// restatement (euler_oracle.c) and by bench.py's reference arm.
#include <omp.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "src/sim/solver/advance_step.hpp"

#include "dimgpu.h"

namespace {

thread_local std::string g_err;

BoundaryConditionType bc_of(int b)
{
    switch (b) {
        case DIMGPU_BC_REFLECTIVE: return BoundaryConditionType::reflective;
        case DIMGPU_BC_NONREFLECTIVE: return BoundaryConditionType::nonreflective;
        default: return BoundaryConditionType::transmissive;
    }
}

template<int DIM>
SolverContext<DIM> make_ctx(const dimgpu_desc* d, double cfl, double dt_max)
{
    SolverContext<DIM> ctx;
    long long n = 1;
    for (int a = 0; a < DIM; ++a) {
        ctx.N[a] = d->N[a];
        ctx.dx[a] = d->dx[a];
        ctx.bc_lo[a] = bc_of(d->bc_lo[a]);
        ctx.bc_hi[a] = bc_of(d->bc_hi[a]);
        n *= d->N[a];
    }
    ctx.cfl = cfl;
    ctx.dt_max = dt_max;
    ctx.initialise_level_set_grid();
    ctx.time_update = (d->time_update == DIMGPU_TIME_UNSPLIT) ? "unsplit" : "split";
    EOSParams m{};
    m.kind = static_cast<EOSKind>(d->mat[0].kind);
    m.gamma = d->mat[0].gamma;
    m.p_inf = d->mat[0].p_inf;
    ctx.material_params = {m};
    ctx.material_id.assign((size_t)n, 0);
    return ctx;
}

template<int DIM>
std::vector<Conserved<DIM>> load_field(const dimgpu_desc* d, const double* soa)
{
    size_t n = 1;
    for (int a = 0; a < DIM; ++a) n *= (size_t)d->N[a];
    std::vector<Conserved<DIM>> U(n);
    for (size_t i = 0; i < n; ++i) {
        U[i].rho = soa[i];
        for (int a = 0; a < DIM; ++a) U[i].mom[a] = soa[(1 + a) * n + i];
        U[i].E = soa[(1 + DIM) * n + i];
    }
    return U;
}

template<int DIM>
void store_field(double* soa, const std::vector<Conserved<DIM>>& U)
{
    const size_t n = U.size();
    for (size_t i = 0; i < n; ++i) {
        soa[i] = U[i].rho;
        for (int a = 0; a < DIM; ++a) soa[(1 + a) * n + i] = U[i].mom[a];
        soa[(1 + DIM) * n + i] = U[i].E;
    }
}

template<int DIM>
int advance_impl(const dimgpu_desc* d, const double* in, double* out, double cfl, double dt_max, int steps,
                 double* dts)
{
    SolverContext<DIM> ctx = make_ctx<DIM>(d, cfl, dt_max);
    std::vector<Conserved<DIM>> U = load_field<DIM>(d, in);
    for (int k = 0; k < steps; ++k) {
        StepResult<DIM> r = advance_one_step<DIM, MaterialEOS>(U, ctx);
        U = std::move(r.U_new);
        if (dts) dts[k] = r.dt;
    }
    store_field<DIM>(out, U);
    return 0;
}

template<int DIM>
int dt_impl(const dimgpu_desc* d, const double* soa, double cfl, double dt_max, double* dt)
{
    SolverContext<DIM> ctx = make_ctx<DIM>(d, cfl, dt_max);
    const std::vector<Conserved<DIM>> U = load_field<DIM>(d, soa);
    *dt = (ctx.time_update == "unsplit")
              ? compute_dt_cfl_materials_unsplit<DIM, MaterialEOS>(U, ctx.material_id, ctx.material_params, ctx.dx,
                                                                  cfl, dt_max)
              : compute_dt_cfl_materials<DIM, MaterialEOS>(U, ctx.material_id, ctx.material_params, ctx.dx, cfl,
                                                           dt_max);
    return 0;
}

template<int DIM>
int hllc_impl(const dimgpu_desc* d, int n, int dir, const double* UL, const double* UR, double* out)
{
    EOSParams m{};
    m.kind = static_cast<EOSKind>(d->mat[0].kind);
    m.gamma = d->mat[0].gamma;
    m.p_inf = d->mat[0].p_inf;
    const int V = 2 + DIM;
    std::array<double, DIM> nrm{};
    nrm[dir] = 1.0;
    for (int i = 0; i < n; ++i) {
        Conserved<DIM> a, b;
        a.rho = UL[i * V];
        b.rho = UR[i * V];
        for (int k = 0; k < DIM; ++k) {
            a.mom[k] = UL[i * V + 1 + k];
            b.mom[k] = UR[i * V + 1 + k];
        }
        a.E = UL[i * V + 1 + DIM];
        b.E = UR[i * V + 1 + DIM];
        const Conserved<DIM> F = hllc_flux_normal<DIM, MaterialEOS>(a, b, nrm, m, m);
        out[i * V] = F.rho;
        for (int k = 0; k < DIM; ++k) out[i * V + 1 + k] = F.mom[k];
        out[i * V + 1 + DIM] = F.E;
    }
    return 0;
}

#define DISPATCH_DIM(d, FN, ...)                                \
    switch ((d)->dim) {                                         \
        case 1: return FN<1>(__VA_ARGS__);                      \
        case 2: return FN<2>(__VA_ARGS__);                      \
        case 3: return FN<3>(__VA_ARGS__);                      \
        default: g_err = "dim must be 1..3"; return DIMGPU_E_INVALID_ARG; \
    }

#define GUARD(...)                                              \
    try { __VA_ARGS__ }                                         \
    catch (const std::exception& e) { g_err = e.what(); return DIMGPU_E_NONFINITE; }

}  // namespace

extern "C" {

const char* eref_last_error(void) { return g_err.c_str(); }

void eref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

int eref_advance(const dimgpu_desc* d, const double* soa_in, double* soa_out, double cfl, double dt_max, int steps,
                 double* dts)
{
    GUARD(DISPATCH_DIM(d, advance_impl, d, soa_in, soa_out, cfl, dt_max, steps, dts))
}

int eref_compute_dt_cfl(const dimgpu_desc* d, const double* soa, double cfl, double dt_max, double* dt)
{
    GUARD(DISPATCH_DIM(d, dt_impl, d, soa, cfl, dt_max, dt))
}

int eref_hllc(const dimgpu_desc* d, int n, int dir, const double* UL, const double* UR, double* out)
{
    GUARD(DISPATCH_DIM(d, hllc_impl, d, n, dir, UL, UR, out))
}

}  // extern "C"
