// dimgpu_sm_shim.hpp — C++ drop-in for the reference's single-material
// sharp-interface step.
//
// Include AFTER the reference's src/sim/solver/advance_step.hpp (it uses
// Conserved<DIM>, SolverContext<DIM>, StepResult<DIM>, EOSParams and the EOS
// structs).  It provides
//
//   dimgpu::sm_advance_one_step<DIM, EOS>(U, ctx)
//
// with the signature and return type of advance_one_step<DIM, EOS>
// (src/sim/solver/advance_step.hpp:489-492) for the case that function runs
// through its single-material fast path: no level set (ctx.phi_list empty)
// and one material.  Anything else is the rGFM path, which stays on the
// reference's CPU code, so the call throws std::runtime_error and the caller
// keeps its own dispatch:
//
//   auto r = (ctx.phi_list.empty() && ctx.material_params.size() == 1)
//                ? dimgpu::sm_advance_one_step<DIM, EOS>(U, ctx)
//                : advance_one_step<DIM, EOS>(U, ctx);
//
// EOS = IdealGasEOS / StiffenedGasEOS evaluate their own law whatever the
// material's kind (as the reference's templates do); MaterialEOS follows the
// kind.  The step runs in one cached device session per thread and grid.
#pragma once

#include <array>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "dimgpu.h"

namespace dimgpu {

inline int sm_bc_code(BoundaryConditionType b)
{
    switch (b) {
        case BoundaryConditionType::reflective: return DIMGPU_BC_REFLECTIVE;
        case BoundaryConditionType::nonreflective: return DIMGPU_BC_NONREFLECTIVE;
        default: return DIMGPU_BC_TRANSMISSIVE;
    }
}

template<int DIM, class EOS>
dimgpu_desc sm_make_desc(const SolverContext<DIM>& ctx)
{
    if (!ctx.phi_list.empty() || ctx.material_params.size() != 1)
        throw std::runtime_error("dimgpu::sm_advance_one_step: level sets or several materials are the rGFM "
                                 "path, which stays on the reference's CPU code");
    dimgpu_desc d;
    std::memset(&d, 0, sizeof d);
    d.dim = DIM;
    for (int a = 0; a < 3; ++a) {
        d.N[a] = a < DIM ? ctx.N[a] : 1;
        d.dx[a] = a < DIM ? ctx.dx[a] : 1.0;
        d.bc_lo[a] = a < DIM ? sm_bc_code(ctx.bc_lo[a]) : 0;
        d.bc_hi[a] = a < DIM ? sm_bc_code(ctx.bc_hi[a]) : 0;
    }
    d.nmat = 1;
    const EOSParams& m = ctx.material_params[0];
    int kind = static_cast<int>(m.kind);
    if (std::is_same<EOS, IdealGasEOS>::value) kind = DIMGPU_EOS_IDEAL_GAS;
    if (std::is_same<EOS, StiffenedGasEOS>::value) kind = DIMGPU_EOS_STIFFENED_GAS;
    d.mat[0].kind = kind;
    d.mat[0].gamma = m.gamma;
    d.mat[0].p_inf = m.p_inf;
    d.precision = DIMGPU_PRECISION_FP64;
    d.time_update = ctx.time_update == "unsplit" ? DIMGPU_TIME_UNSPLIT : DIMGPU_TIME_SPLIT;
    d.model = DIMGPU_MODEL_EULER;
    return d;
}

template<int DIM>
void sm_pack(const std::vector<Conserved<DIM>>& U, std::vector<double>& soa)
{
    const size_t n = U.size();
    soa.resize(n * (DIM + 2));
    for (size_t i = 0; i < n; ++i) {
        soa[i] = U[i].rho;
        for (int a = 0; a < DIM; ++a) soa[(1 + a) * n + i] = U[i].mom[a];
        soa[(1 + DIM) * n + i] = U[i].E;
    }
}

template<int DIM>
void sm_unpack(const std::vector<double>& soa, std::vector<Conserved<DIM>>& U)
{
    const size_t n = U.size();
    for (size_t i = 0; i < n; ++i) {
        U[i].rho = soa[i];
        for (int a = 0; a < DIM; ++a) U[i].mom[a] = soa[(1 + a) * n + i];
        U[i].E = soa[(1 + DIM) * n + i];
    }
}

// Drop-in for advance_one_step<DIM, EOS> without level sets and with one
// material: host vectors in and out, ctx.completed_steps advanced.
template<int DIM, class EOS>
StepResult<DIM> sm_advance_one_step(const std::vector<Conserved<DIM>>& U, SolverContext<DIM>& ctx)
{
    if (U.empty()) throw std::runtime_error("advance_one_step: empty state");
    ctx.validate(static_cast<int>(U.size()));
    const dimgpu_desc d = sm_make_desc<DIM, EOS>(ctx);
    std::vector<double> in, out;
    sm_pack<DIM>(U, in);
    out.resize(in.size());
    double dt = 0.0;
    dimgpu_phase_times t{};
    if (dimgpu_advance_one_step(&d, in.data(), out.data(), ctx.cfl, ctx.dt_max, &dt, &t) != DIMGPU_OK)
        throw std::runtime_error(dimgpu_last_error(nullptr));
    StepResult<DIM> r{};
    r.U_new = U;
    sm_unpack<DIM>(out, r.U_new);
    r.phi_list_new = ctx.phi_list;
    r.dt = dt;
    r.phase_timings.cfl_seconds = t.cfl_ms * 1e-3;
    r.phase_timings.sweep_seconds = t.sweep_ms * 1e-3;
    r.phase_timings.boundary_seconds = t.boundary_ms * 1e-3;
    ctx.completed_steps += 1;
    return r;
}

}  // namespace dimgpu
