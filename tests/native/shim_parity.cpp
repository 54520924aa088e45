// shim_parity.cpp — the reference's own time loop run twice in one process:
// once with dim::advance_one_step (the reference's OpenMP code) and once with
// the drop-in dimgpu::advance_one_step / dimgpu::ResidentDim from
// include/dimgpu_reference_shim.hpp (the GPU).  Built by oracle/Makefile
// where the reference sources exist; exit status 0 iff every double of every
// step is identical.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "src/dim/solver/advance_step.hpp"

#include "dimgpu_reference_shim.hpp"

template<int DIM>
static std::vector<dim::State<DIM>> initial(const std::array<int, DIM>& N, const dim::EOSParams& params)
{
    size_t n = 1;
    for (int a = 0; a < DIM; ++a) n *= N[a];
    std::vector<dim::State<DIM>> U(n);
    for (size_t i = 0; i < n; ++i) {
        const double x = (double)(i % N[0]) / N[0];
        double r2 = (x - 0.6) * (x - 0.6);
        if (DIM > 1) {
            const double y = (double)((i / N[0]) % N[1]) / N[1];
            r2 += (y - 0.5) * (y - 0.5);
        }
        const double ind = 0.5 * (1.0 - std::tanh((std::sqrt(r2) - 0.2) * 40.0));
        dim::Primitive<DIM> P{};
        P.alpha = {1.0 - ind, ind};
        P.rho = {x < 0.25 ? 1.4 : 1.0, 0.14};
        P.vel[0] = x < 0.25 ? 0.4 : 0.0;
        P.p = x < 0.25 ? 1.6 : 1.0;
        U[i] = dim::prim_to_cons<DIM>(P, params);
    }
    return U;
}

template<int DIM>
static int run(const std::array<int, DIM>& N, int steps)
{
    dim::EOSParams params;
    ::EOSParams air{}, gas{};
    air.kind = EOSKind::ideal_gas;
    air.gamma = 1.4;
    gas.kind = EOSKind::stiffened_gas;
    gas.gamma = 1.67;
    gas.p_inf = 0.1;
    params.material = {air, gas};
    Config<DIM> cfg;
    cfg.interface_method = "DIM";
    if (DIM > 1) { cfg.bc_lo[1] = "reflective"; cfg.bc_hi[1] = "reflective"; }
    std::array<double, DIM> dx{};
    for (int a = 0; a < DIM; ++a) dx[a] = 1.0 / N[a];

    auto Uref = initial<DIM>(N, params);
    auto Ugpu = Uref;
    dimgpu::ResidentDim<DIM> resident(Uref, N, dx, params, cfg);
    size_t bad = 0;
    for (int s = 0; s < steps; ++s) {
        const auto r = dim::advance_one_step<DIM>(Uref, N, dx, params, cfg, 0.8, 1e300);
        const auto g = dimgpu::advance_one_step<DIM>(Ugpu, N, dx, params, cfg, 0.8, 1e300);
        const double dt_res = resident.step(0.8, 1e300);
        Uref = r.U_new;
        Ugpu = g.U_new;
        if (r.dt != g.dt || r.dt != dt_res) ++bad;
    }
    std::vector<dim::State<DIM>> Ures(Uref.size());
    resident.download(Ures);
    for (size_t i = 0; i < Uref.size(); ++i) {
        for (size_t k = 0; k < Uref[i].partial_mass.size(); ++k) {
            bad += Uref[i].partial_mass[k] != Ugpu[i].partial_mass[k];
            bad += Uref[i].partial_mass[k] != Ures[i].partial_mass[k];
        }
        for (int a = 0; a < DIM; ++a) bad += (Uref[i].mom[a] != Ugpu[i].mom[a]) + (Uref[i].mom[a] != Ures[i].mom[a]);
        bad += (Uref[i].E != Ugpu[i].E) + (Uref[i].E != Ures[i].E);
        for (size_t k = 0; k < Uref[i].alpha.size(); ++k)
            bad += (Uref[i].alpha[k] != Ugpu[i].alpha[k]) + (Uref[i].alpha[k] != Ures[i].alpha[k]);
    }
    std::printf("DIM=%d cells=%zu steps=%d mismatches=%zu\n", DIM, Uref.size(), steps, bad);
    return bad == 0 ? 0 : 1;
}

int main()
{
    int rc = 0;
    rc |= run<1>({400}, 40);
    rc |= run<2>({64, 32}, 20);
    rc |= run<3>({16, 12, 10}, 5);
    std::printf(rc == 0 ? "shim parity: identical\n" : "shim parity: MISMATCH\n");
    return rc;
}
