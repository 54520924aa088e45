/*
 * dim_oracle.h — TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's
 * DIM step, used as the checker of the CUDA path (tests/, smoke()) and as the
 * "port" CPU baseline.  Never linked into the product library.
 *
 * Every function follows the reference line by line (same operations in the
 * same order, literal bisection pressure recovery) so that a correctly
 * rounded FP64 implementation without FMA contraction reproduces the
 * reference bit for bit.  Its parity with the reference is pinned by the
 * golden vectors under tests/golden/, which were produced by the reference
 * itself (oracle/_ref, built from the reference sources by oracle/Makefile).
 *
 * Record layouts are those of include/dimgpu.h: a state is
 * {partial_mass[nmat], mom[dim], E, alpha[nmat-1]}; a primitive is
 * {rho[nmat], alpha[nmat], vel[dim], p}.
 */
#ifndef DIM_ORACLE_H
#define DIM_ORACLE_H

#include <stddef.h>

#include "dimgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

const char* oracle_last_error(void);

/* Whole-step and sweep-level functions over a SoA field (component-major). */
int oracle_advance(const dimgpu_desc* d, const double* soa_in, double* soa_out, double cfl,
                   double dt_max, int nsteps, double* dt_out);
int oracle_compute_dt_cfl(const dimgpu_desc* d, const double* soa, double cfl, double dt_max,
                          double* dt_out);
int oracle_sweep_direction(const dimgpu_desc* d, int dir, double dt, const double* soa_in,
                           double* soa_out);
int oracle_apply_boundary_conditions(const dimgpu_desc* d, double* soa);
int oracle_boundary_flux(const dimgpu_desc* d, const double* soa, double* out);
int oracle_totals(const dimgpu_desc* d, const double* soa, double* out);

/* Per-function records (record-major, n records). */
int oracle_cons_to_prim(const dimgpu_desc* d, int n, const double* U, double* P);
int oracle_prim_to_cons(const dimgpu_desc* d, int n, const double* P, double* U);
int oracle_repair_state(const dimgpu_desc* d, int n, double* U);
int oracle_mixture_pressure(const dimgpu_desc* d, int n, const double* in, double* p);
int oracle_mixture_sound_speed(const dimgpu_desc* d, int n, const double* in, double* c);
int oracle_alpha_rhs(const dimgpu_desc* d, int n, const double* P, double* rhs);
int oracle_hllc(const dimgpu_desc* d, int n, int dir, const double* UL, const double* UR,
                double* out);
int oracle_solve_line(const dimgpu_desc* d, int n, int dir, double dt, double dx,
                      const double* U_in, double* U_out);

/* dim::write_csv of a SoA field (src/io/dim_write_csv.hpp:15-125). */
int oracle_write_csv(const dimgpu_desc* d, const double* soa, const double* domain_min,
                     const double* domain_max, const char* filename);

/* OpenMP threads used by the sweep / CFL loops (<= 0 leaves the default). */
int oracle_set_threads(int n);

#ifdef __cplusplus
}
#endif

#endif
