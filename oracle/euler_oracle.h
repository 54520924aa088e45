/* euler_oracle.h — TEST INFRASTRUCTURE ONLY: entry points of the plain-C
 * restatement of the reference's single-material Euler step
 * (euler_oracle.c).  SoA state: rho, mom[0..dim-1], E per cell. */
#ifndef EULER_ORACLE_H
#define EULER_ORACLE_H

#include "dimgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

int euler_oracle_compute_dt_cfl(const dimgpu_desc* d, const double* soa, double cfl, double dt_max, double* dt);
int euler_oracle_sweep_direction(const dimgpu_desc* d, int dir, double dt, const double* in, double* out);
int euler_oracle_apply_boundary_conditions(const dimgpu_desc* d, double* soa);
int euler_oracle_hllc(const dimgpu_desc* d, int n, int dir, const double* UL, const double* UR, double* out);
int euler_oracle_advance(const dimgpu_desc* d, const double* soa_in, double* soa_out, double cfl, double dt_max,
                         int steps, double* dts);

#ifdef __cplusplus
}
#endif

#endif
