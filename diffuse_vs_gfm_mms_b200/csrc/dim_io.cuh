// dim_io.cuh — device-side initial fields and CSV records of the DIM state.
//
// Initial fields: the shock-bubble and bubble-cloud workloads are generated
// cell by cell on the device instead of being built on the host and copied
// (a 512^3 field is 7.5 GB).  The diffuse interfaces use the reference's tanh
// indicator 0.5 (1 - tanh(a s / thickness)) (smooth_indicator,
// src/setup/dim_initial_conditions.hpp:224-236) with a tanh of our own made
// of IEEE +, -, *, / and exact scaling only, and every primitive -> conservative
// conversion is written in the same order as the host generator
// (diffuse_vs_gfm_mms_b200/workloads.py), so the device field and the host
// field are the same bits.
//
// CSV records: the per-cell values dim::write_csv prints
// (src/io/dim_write_csv.hpp:15-125) — cell centre, total density,
// velocity, pressure, internal energy, volume fractions, material densities,
// partial masses — computed on the device with the step's own bit-faithful
// cons_to_prim, for the host to format.
#pragma once

#include "dim_kernels.cuh"

namespace dimgpu {

// ---- portable exp / tanh (same arithmetic as workloads.portable_exp) --------------
// Cody-Waite reduction with fdlibm's split of ln 2, then the degree-13
// Taylor polynomial of exp on |r| <= ln2 / 2 in Horner form.
DHD double portable_exp(double x)
{
    const double kLn2Hi = 6.93147180369123816490e-01;
    const double kLn2Lo = 1.90821492927058770002e-10;
    const double kInvLn2 = 1.44269504088896338700e+00;
    const double k = floor(x * kInvLn2 + 0.5);
    const double r = (x - k * kLn2Hi) - k * kLn2Lo;
    // 1/n!, n = 0 .. 13: quotients of exactly representable integers
    const double c[14] = {1.0 / 1.0,         1.0 / 1.0,        1.0 / 2.0,         1.0 / 6.0,
                          1.0 / 24.0,        1.0 / 120.0,      1.0 / 720.0,       1.0 / 5040.0,
                          1.0 / 40320.0,     1.0 / 362880.0,   1.0 / 3628800.0,   1.0 / 39916800.0,
                          1.0 / 479001600.0, 1.0 / 6227020800.0};
    double p = c[13];
#pragma unroll
    for (int n = 12; n >= 0; --n) p = p * r + c[n];
    return ldexp(p, (int)k);
}

// tanh(y) = (e - 1) / (e + 1), e = exp(2|y|); odd; 1 beyond |y| = 20.
DHD double portable_tanh(double y)
{
    const double a = fmin(fabs(y), 20.0);
    const double e = portable_exp(2.0 * a);
    double t = (e - 1.0) / (e + 1.0);
    if (fabs(y) > 20.0) t = 1.0;
    return (y < 0.0) ? -t : t;
}

// smooth_indicator (src/setup/dim_initial_conditions.hpp:224-236).
DHD double smooth_indicator(double signed_distance, double thickness, double sharpness)
{
    return 0.5 * (1.0 - portable_tanh(dmax(sharpness, 1e-12) * signed_distance / thickness));
}

// Primitive -> conservative of one two-material cell exactly as the host
// generator forms it (workloads.prim_to_cons_np): masses alpha_k rho_k,
// rho = max(m0 + m1, 1e-12), rho e = sum_k (alpha_k rho_k) e_k with
// e_k = (p + gamma_k p_inf_k) / ((gamma_k - 1) rho_k), E = rho e + 0.5 rho |u|^2.
template<int D>
DHD void ic_prim_to_cons(const Mats& M, double a0, double a1, double r0, double r1, const double* vel, double p,
                         State<2, D>& U)
{
    const double al[2] = {a0, a1};
    const double rh[2] = {r0, r1};
    U.m[0] = a0 * r0;
    U.m[1] = a1 * r1;
    const double rho_t = dmax(U.m[0] + U.m[1], 1e-12);
    double rho_e = 0.0;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const double e_k = (p + M.gpinf[k]) / (M.gm1[k] * rh[k]);
        rho_e += al[k] * rh[k] * e_k;
    }
    double v2 = vel[0] * vel[0];
#pragma unroll
    for (int d = 1; d < D; ++d) v2 += vel[d] * vel[d];
#pragma unroll
    for (int d = 0; d < D; ++d) U.mom[d] = rho_t * vel[d];
    U.E = rho_e + 0.5 * rho_t * v2;
    U.a[0] = a0;
}

// The 2D shock-bubble field: material 1 fills a circle (tanh-smeared edge),
// material 0 the rest; left of shock_x the ambient gas carries the
// post-shock state.  Parameters as in dimgpu_ic_shock_bubble (include/dimgpu.h).
struct ShockBubbleIC {
    double cx, cy, radius, thickness, sharpness, shock_x, zero_below;
    double rho_post, u_post, p_post, rho_pre, p_pre, rho_bubble, p_bubble;
};

__global__ void __launch_bounds__(256) ic_shock_bubble_kernel(double* __restrict__ st, __grid_constant__ const Grid g,
                                                              __grid_constant__ const Mats M, ShockBubbleIC ic)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.ncell) return;
    const int i = (int)(c % g.N[0]);
    const int j = (int)(c / g.N[0]);
    const double x = ((double)i + 0.5) * g.dx[0];
    const double y = ((double)j + 0.5) * g.dx[1];
    const double sd = sqrt((x - ic.cx) * (x - ic.cx) + (y - ic.cy) * (y - ic.cy)) - ic.radius;
    double ab = smooth_indicator(sd, ic.thickness, ic.sharpness);
    if (ab <= ic.zero_below) ab = 0.0;
    const bool post = x < ic.shock_x;
    const double rho_amb = post ? ic.rho_post : ic.rho_pre;
    const double p_amb = post ? ic.p_post : ic.p_pre;
    const double u_amb = post ? ic.u_post : 0.0;
    const double a0 = 1.0 - ab;
    const double vel[2] = {a0 * u_amb, 0.0};
    const double p = a0 * p_amb + ab * ic.p_bubble;
    State<2, 2> U;
    ic_prim_to_cons<2>(M, a0, ab, rho_amb, ic.rho_bubble, vel, p, U);
    store_cell<2, 2>(st, g.ncell, c, U);
}

// The 3D bubble cloud: material 1 (gas) in tanh-smeared spheres, each
// evaluated only inside its box [lo, hi) of cells, the gas fraction the
// largest of them; material 0 (liquid) elsewhere; pressure p_pulse in the
// slab x < pulse_width, p_ambient beyond; at rest.
struct CloudIC {
    double thickness, sharpness, zero_below, pulse_width;
    double rho_liquid, rho_gas, p_ambient, p_pulse;
    int nbubbles;
};

struct BubbleIC {
    double c[3];
    double radius;
    int lo[3], hi[3];
};

__global__ void __launch_bounds__(256) ic_bubble_cloud_kernel(double* __restrict__ st, __grid_constant__ const Grid g,
                                                              __grid_constant__ const Mats M, CloudIC ic,
                                                              const BubbleIC* __restrict__ bub)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.ncell) return;
    const int i = (int)(c % g.N[0]);
    const int j = (int)((c / g.N[0]) % g.N[1]);
    const int k = (int)(c / ((long long)g.N[0] * g.N[1]));
    const double x = ((double)i + 0.5) * g.dx[0];
    const double y = ((double)j + 0.5) * g.dx[1];
    const double z = ((double)k + 0.5) * g.dx[2];
    double air = 0.0;
    for (int b = 0; b < ic.nbubbles; ++b) {
        const BubbleIC B = bub[b];
        if (i < B.lo[0] || i >= B.hi[0] || j < B.lo[1] || j >= B.hi[1] || k < B.lo[2] || k >= B.hi[2]) continue;
        const double sd = sqrt((x - B.c[0]) * (x - B.c[0]) + (y - B.c[1]) * (y - B.c[1]) +
                               (z - B.c[2]) * (z - B.c[2])) - B.radius;
        air = dmax(air, smooth_indicator(sd, ic.thickness, ic.sharpness));
    }
    if (air <= ic.zero_below) air = 0.0;
    const double p = (x < ic.pulse_width) ? ic.p_pulse : ic.p_ambient;
    const double vel[3] = {0.0, 0.0, 0.0};
    State<2, 3> U;
    ic_prim_to_cons<3>(M, 1.0 - air, air, ic.rho_liquid, ic.rho_gas, vel, p, U);
    store_cell<2, 3>(st, g.ncell, c, U);
}

// ---- CSV records (dim::write_csv, src/io/dim_write_csv.hpp:70-118) ----------------
// Record of cell c at rec[(c - c0) * R + ...]:
//   x[D], rho, vel[D], p, e, alpha[NM], rho_k[NM], partial_mass[NM]
// with x_d = domain_min_d + (idx_d + 0.5) dx_d (compute_cell_center,
// src/dim/solver/advance/geometry.hpp:75-87) and e = max(safe_div(E - kinetic, rho), 0).
__host__ __device__ constexpr int csv_record_width(int nm, int d) { return 2 * d + 3 + 3 * nm; }

struct CsvGeom {
    double xmin[3];
    double dx[3];
};

template<int NM, int D>
__global__ void __launch_bounds__(256) csv_records_kernel(const double* __restrict__ st, __grid_constant__ const Grid g,
                                                          __grid_constant__ const Mats M, CsvGeom geo, long long c0,
                                                          long long n, double* __restrict__ rec)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const long long c = c0 + t;
    State<NM, D> U;
    load_cell<NM, D>(st, g.ncell, c, U);
    const Prim<NM, D> P = cons_to_prim_v<NM, D>(M, U);
    const double rho = total_density<NM, D>(U);
    double v2 = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) v2 += P.vel[d] * P.vel[d];
    const double kinetic = 0.5 * rho * v2;
    const double ie = dmax(safe_div(U.E - kinetic, rho), 0.0);
    double* r = rec + t * csv_record_width(NM, D);
    int q = 0;
    long long rem = c;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const long long idx = rem % g.N[d];
        rem /= g.N[d];
        r[q++] = geo.xmin[d] + ((double)idx + 0.5) * geo.dx[d];
    }
    r[q++] = rho;
#pragma unroll
    for (int d = 0; d < D; ++d) r[q++] = P.vel[d];
    r[q++] = P.p;
    r[q++] = ie;
#pragma unroll
    for (int k = 0; k < NM; ++k) r[q++] = P.alpha[k];
#pragma unroll
    for (int k = 0; k < NM; ++k) r[q++] = P.rho[k];
#pragma unroll
    for (int k = 0; k < NM; ++k) r[q++] = U.m[k];
}

}  // namespace dimgpu
