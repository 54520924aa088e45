// dimgpu_reference_shim.hpp — C++ drop-in for the reference's DIM step.
//
// Include AFTER the reference's own headers (it uses dim::State, dim::EOSParams,
// dim::StepResult and Config<DIM> from src/dim and src/io).  It provides
//
//   dimgpu::advance_one_step<DIM>(U, N, dx, params, cfg, cfl, dt_max)
//
// with exactly the signature and return type of dim::advance_one_step
// (src/dim/solver/advance_step.hpp:28-37), so a caller such as run_dim_case
// (src/app/solver/run_dim.hpp:94) switches by changing the namespace, and
// dimgpu::ResidentDim<DIM>, which keeps the state on the GPU across steps and
// converts the reference's AoS std::vector<dim::State<DIM>> to and from the
// library's SoA layout only when the caller needs host data (CSV output,
// conservation reports).  Errors throw std::runtime_error, as the reference does.
#pragma once

#include <array>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "dimgpu.h"

namespace dimgpu {

inline int bc_code(const std::string& name)
{
    if (name == "reflective") return DIMGPU_BC_REFLECTIVE;
    if (name == "nonreflective" || name == "non_reflective") return DIMGPU_BC_NONREFLECTIVE;
    return DIMGPU_BC_TRANSMISSIVE;
}

inline int lambda_code(const std::string& name)
{
    if (name == "allaire") return DIMGPU_LAMBDA_ALLAIRE;
    if (name == "equal_velocity") return DIMGPU_LAMBDA_EQUAL_VELOCITY;
    if (name == "kapila" || name.empty()) return DIMGPU_LAMBDA_KAPILA;
    throw std::runtime_error("dim::alpha_rhs_coefficients: unknown lambda model");
}

inline void check(int rc, const dimgpu_session* s = nullptr)
{
    if (rc != DIMGPU_OK) throw std::runtime_error(dimgpu_last_error(s));
}

// dimgpu_desc from the arguments of dim::advance_one_step.
template<int DIM, class EOSParamsT, class ConfigT>
dimgpu_desc make_desc(const std::array<int, DIM>& N, const std::array<double, DIM>& dx, const EOSParamsT& params,
                      const ConfigT& cfg)
{
    dimgpu_desc d;
    std::memset(&d, 0, sizeof d);
    d.dim = DIM;
    for (int a = 0; a < 3; ++a) {
        d.N[a] = a < DIM ? N[a] : 1;
        d.dx[a] = a < DIM ? dx[a] : 1.0;
        d.bc_lo[a] = a < DIM ? bc_code(cfg.bc_lo[a]) : 0;
        d.bc_hi[a] = a < DIM ? bc_code(cfg.bc_hi[a]) : 0;
    }
    d.nmat = static_cast<int>(params.material.size());
    if (d.nmat < 1 || d.nmat > DIMGPU_MAX_MATERIALS) throw std::runtime_error("dimgpu: 1..4 materials supported");
    for (int k = 0; k < d.nmat; ++k) {
        d.mat[k].kind = static_cast<int>(params.material[k].kind);
        d.mat[k].gamma = params.material[k].gamma;
        d.mat[k].p_inf = params.material[k].p_inf;
    }
    d.lambda_model = lambda_code(cfg.dim_lambda_model);
    d.alpha_source_floor = cfg.dim_alpha_source_floor;
    d.precision = DIMGPU_PRECISION_FP64;
    d.time_update = cfg.time_update == "unsplit" ? DIMGPU_TIME_UNSPLIT : DIMGPU_TIME_SPLIT;
    return d;
}

// AoS (one dim::State per cell) -> SoA, component-major.
template<int DIM, class StateT>
void pack(const std::vector<StateT>& U, int nmat, std::vector<double>& soa)
{
    const size_t n = U.size();
    const int V = 2 * nmat + DIM;
    soa.resize(n * static_cast<size_t>(V));
    for (size_t i = 0; i < n; ++i) {
        int c = 0;
        for (int k = 0; k < nmat; ++k) soa[(c++) * n + i] = U[i].partial_mass[k];
        for (int a = 0; a < DIM; ++a) soa[(c++) * n + i] = U[i].mom[a];
        soa[(c++) * n + i] = U[i].E;
        for (int k = 0; k < nmat - 1; ++k) soa[(c++) * n + i] = U[i].alpha[k];
    }
}

template<int DIM, class StateT>
void unpack(const std::vector<double>& soa, int nmat, std::vector<StateT>& U)
{
    const size_t n = U.size();
    for (size_t i = 0; i < n; ++i) {
        int c = 0;
        U[i].partial_mass.resize(nmat);
        U[i].alpha.resize(nmat > 1 ? nmat - 1 : 0);
        for (int k = 0; k < nmat; ++k) U[i].partial_mass[k] = soa[(c++) * n + i];
        for (int a = 0; a < DIM; ++a) U[i].mom[a] = soa[(c++) * n + i];
        U[i].E = soa[(c++) * n + i];
        for (int k = 0; k < nmat - 1; ++k) U[i].alpha[k] = soa[(c++) * n + i];
    }
}

// Drop-in for dim::advance_one_step: one call, host vectors in and out.
template<int DIM, class StateT, class EOSParamsT, class ConfigT>
auto advance_one_step(const std::vector<StateT>& U, const std::array<int, DIM>& N,
                      const std::array<double, DIM>& dx, const EOSParamsT& params, const ConfigT& cfg, double cfl,
                      double dt_max)
{
    if (U.empty()) throw std::runtime_error("dim::advance_one_step: empty state");
    const dimgpu_desc d = make_desc<DIM>(N, dx, params, cfg);
    size_t expected = 1;
    for (int a = 0; a < DIM; ++a) expected *= static_cast<size_t>(N[a]);
    if (expected != U.size()) throw std::runtime_error("dim::advance_one_step: grid size mismatch");
    std::vector<double> in, out;
    pack<DIM>(U, d.nmat, in);
    out.resize(in.size());
    double dt = 0.0;
    dimgpu_phase_times t{};
    check(dimgpu_advance_one_step(&d, in.data(), out.data(), cfl, dt_max, &dt, &t));
    dim::StepResult<DIM> r;
    r.U_new = U;
    unpack<DIM>(out, d.nmat, r.U_new);
    r.dt = dt;
    r.phase_timings.cfl_seconds = t.cfl_ms * 1e-3;
    r.phase_timings.sweep_seconds = t.sweep_ms * 1e-3;
    r.phase_timings.boundary_seconds = t.boundary_ms * 1e-3;
    return r;
}

// Device-resident state for a time loop: upload once, step many times,
// download only for output.
template<int DIM>
class ResidentDim {
public:
    template<class StateT, class EOSParamsT, class ConfigT>
    ResidentDim(const std::vector<StateT>& U, const std::array<int, DIM>& N, const std::array<double, DIM>& dx,
                const EOSParamsT& params, const ConfigT& cfg)
        : desc_(make_desc<DIM>(N, dx, params, cfg))
    {
        check(dimgpu_create(&desc_, &s_));
        upload(U);
    }
    ~ResidentDim() { dimgpu_destroy(s_); }
    ResidentDim(const ResidentDim&) = delete;
    ResidentDim& operator=(const ResidentDim&) = delete;

    template<class StateT>
    void upload(const std::vector<StateT>& U)
    {
        pack<DIM>(U, desc_.nmat, buf_);
        check(dimgpu_upload(s_, buf_.data(), buf_.size()), s_);
    }

    template<class StateT>
    void download(std::vector<StateT>& U)
    {
        buf_.resize(static_cast<size_t>(dimgpu_components(&desc_)) * U.size());
        check(dimgpu_download(s_, buf_.data(), buf_.size()), s_);
        unpack<DIM>(buf_, desc_.nmat, U);
    }

    double step(double cfl, double dt_max)
    {
        double dt = 0.0;
        check(dimgpu_step(s_, cfl, dt_max, &dt, nullptr), s_);
        return dt;
    }

    dimgpu_session* session() { return s_; }

private:
    dimgpu_desc desc_;
    dimgpu_session* s_ = nullptr;
    std::vector<double> buf_;
};

}  // namespace dimgpu
