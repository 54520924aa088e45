// dimgpu_validate.h — the descriptor checks every entry point that takes a
// dimgpu_desc applies before any device work (internal; not part of the
// C-ABI).  One definition, so the session API and the allocation-free entry
// point refuse exactly the same descriptors with the same status.
#pragma once

#include <string>

#include "dimgpu.h"

namespace dimgpu {

// Returns DIMGPU_OK, or a status with its message in *msg.  The messages name
// the reference routine that throws on the same input where there is one.
inline int check_desc(const dimgpu_desc* d, std::string* msg)
{
    auto bad = [&](int code, const std::string& m) {
        *msg = m;
        return code;
    };
    if (!d) return bad(DIMGPU_E_INVALID_ARG, "null descriptor");
    if (d->dim < 1 || d->dim > 3) return bad(DIMGPU_E_INVALID_ARG, "dim must be 1, 2 or 3");
    if (d->nmat < 1 || d->nmat > DIMGPU_MAX_MATERIALS)
        return bad(DIMGPU_E_INVALID_ARG, "dim::EOSParams: nmat must be 1..4");
    for (int a = 0; a < 3; ++a) {
        const int n = d->N[a];
        if (a < d->dim && n < 1) return bad(DIMGPU_E_INVALID_ARG, "dim::total_cells: grid size must be positive");
        if (a >= d->dim && n != 1) return bad(DIMGPU_E_INVALID_ARG, "unused axes must have N = 1");
        if (a < d->dim && !(d->dx[a] > 0.0))
            return bad(DIMGPU_E_INVALID_ARG, "dim::compute_dt_cfl: grid spacing must be positive");
    }
    for (int k = 0; k < d->nmat; ++k) {
        const int kind = d->mat[k].kind;
        if (kind != DIMGPU_EOS_IDEAL_GAS && kind != DIMGPU_EOS_STIFFENED_GAS)
            return bad(DIMGPU_E_UNSUPPORTED_EOS,
                       "material " + std::to_string(k) + ": only ideal_gas and stiffened_gas run on the GPU");
        if (!(d->mat[k].gamma > 1.0)) return bad(DIMGPU_E_INVALID_ARG, "dim::EOSParams: gamma must be > 1");
    }
    if (d->lambda_model < 0 || d->lambda_model > 2)
        return bad(DIMGPU_E_INVALID_ARG, "dim::alpha_rhs_coefficients: unknown lambda model");
    if (d->precision != DIMGPU_PRECISION_FP64 && d->precision != DIMGPU_PRECISION_MIXED &&
        d->precision != DIMGPU_PRECISION_MIXED_FP64)
        return bad(DIMGPU_E_INVALID_ARG, "precision must be DIMGPU_PRECISION_FP64, _MIXED or _MIXED_FP64");
    if (d->time_update != DIMGPU_TIME_SPLIT && d->time_update != DIMGPU_TIME_UNSPLIT)
        return bad(DIMGPU_E_INVALID_ARG, "time_update must be split or unsplit");
    if (d->model != DIMGPU_MODEL_DIM && d->model != DIMGPU_MODEL_EULER)
        return bad(DIMGPU_E_INVALID_ARG, "model must be DIMGPU_MODEL_DIM or DIMGPU_MODEL_EULER");
    if (d->model == DIMGPU_MODEL_EULER) {
        if (d->nmat != 1) return bad(DIMGPU_E_INVALID_ARG, "the Euler step runs exactly one material (nmat = 1)");
        if (d->precision != DIMGPU_PRECISION_FP64)
            return bad(DIMGPU_E_UNSUPPORTED, "the Euler step runs in FP64 only");
        for (int a = 0; a < d->dim; ++a)
            if (d->N[a] < 3)
                return bad(DIMGPU_E_INVALID_ARG, "reconstruct_line_interfaces: need at least 3 cells");
    }
    return DIMGPU_OK;
}

}  // namespace dimgpu
