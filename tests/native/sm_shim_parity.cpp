// sm_shim_parity.cpp — the reference's single-material sharp-interface step
// run twice in one process: advance_one_step<DIM, EOS> (the reference's
// OpenMP code) and dimgpu::sm_advance_one_step<DIM, EOS> from
// include/dimgpu_sm_shim.hpp (the GPU), for MaterialEOS and IdealGasEOS,
// split and unsplit.  Built by oracle/Makefile where the reference sources
// exist; exit status 0 iff every double of every step is identical.
#include <cmath>
#include <cstdio>

#include "src/sim/solver/advance_step.hpp"

#include "dimgpu_sm_shim.hpp"

template<int DIM>
static std::vector<Conserved<DIM>> blast(const std::array<int, DIM>& N, const EOSParams& m)
{
    size_t n = 1;
    for (int a = 0; a < DIM; ++a) n *= N[a];
    std::vector<Conserved<DIM>> U(n);
    for (size_t i = 0; i < n; ++i) {
        size_t r = i;
        double r2 = 0.0;
        Primitive<DIM> P{};
        for (int a = 0; a < DIM; ++a) {
            const double x = ((double)(r % N[a]) + 0.5) / N[a];
            r /= N[a];
            r2 += (x - 0.47) * (x - 0.47);
            P.vel[a] = 0.1 * std::sin(7.0 * x + a);
        }
        const bool in = r2 < 0.02;
        P.rho = in ? 1.0 : 0.125;
        P.p = in ? 1.0 : 0.1;
        U[i] = prim_to_cons<DIM, MaterialEOS>(P, m);
    }
    return U;
}

template<int DIM, class EOS>
static int run(const std::array<int, DIM>& N, int steps, const char* time_update, BoundaryConditionType bc)
{
    SolverContext<DIM> ctx;
    for (int a = 0; a < DIM; ++a) {
        ctx.N[a] = N[a];
        ctx.dx[a] = 1.0 / N[a];
        ctx.bc_lo[a] = bc;
        ctx.bc_hi[a] = a == 0 ? BoundaryConditionType::transmissive : bc;
    }
    ctx.cfl = 0.6;
    ctx.dt_max = 1e300;
    ctx.time_update = time_update;
    ctx.initialise_level_set_grid();
    EOSParams m{};
    m.kind = EOSKind::ideal_gas;
    m.gamma = 1.4;
    ctx.material_params = {m};
    size_t n = 1;
    for (int a = 0; a < DIM; ++a) n *= N[a];
    ctx.material_id.assign(n, 0);
    SolverContext<DIM> ctx_gpu = ctx;

    auto Uref = blast<DIM>(N, m);
    auto Ugpu = Uref;
    size_t bad = 0;
    for (int s = 0; s < steps; ++s) {
        const auto r = advance_one_step<DIM, EOS>(Uref, ctx);
        const auto g = dimgpu::sm_advance_one_step<DIM, EOS>(Ugpu, ctx_gpu);
        Uref = r.U_new;
        Ugpu = g.U_new;
        bad += r.dt != g.dt;
    }
    bad += ctx.completed_steps != ctx_gpu.completed_steps;
    for (size_t i = 0; i < Uref.size(); ++i) {
        bad += Uref[i].rho != Ugpu[i].rho;
        for (int a = 0; a < DIM; ++a) bad += Uref[i].mom[a] != Ugpu[i].mom[a];
        bad += Uref[i].E != Ugpu[i].E;
    }
    std::printf("DIM=%d cells=%zu steps=%d %s mismatches=%zu\n", DIM, Uref.size(), steps, time_update, bad);
    return bad == 0 ? 0 : 1;
}

int main()
{
    int rc = 0;
    rc |= run<1, MaterialEOS>({400}, 40, "split", BoundaryConditionType::transmissive);
    rc |= run<2, MaterialEOS>({64, 48}, 20, "split", BoundaryConditionType::reflective);
    rc |= run<2, IdealGasEOS>({40, 36}, 10, "unsplit", BoundaryConditionType::nonreflective);
    rc |= run<3, MaterialEOS>({16, 12, 10}, 6, "split", BoundaryConditionType::reflective);
    std::printf(rc == 0 ? "sm shim parity: identical\n" : "sm shim parity: MISMATCH\n");
    return rc;
}
