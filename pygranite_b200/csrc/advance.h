// advance.h — the step-kernel variants, instantiated per wind storage type in advance.cu
// (compiled once per type so the variants build in parallel).
#pragma once

#include "granite_kernels.cuh"

namespace granite_b200 {

using AdvanceFn = void (*)(const KParams);

// The feature set (FT_* in granite_kernels.cuh) a launch with parameters P may use: a lean
// variant when every option it leaves out is off in P (window-pair layouts only), else generic.
// defer: the caller runs deferred_extras_kernel after every launch, which ends at each record.
inline int kernel_features(const KParams &P, bool pair, bool defer = false) {
    if (!pair || P.uplift_mode != 0 || P.abort_mode != 0 || P.topography || P.sphere || P.border_mode != 0 ||
        P.alive_at != nullptr || P.filter_weights || (P.curvature_mode != 0 && P.curvature_mode != 1))
        return FT_GENERIC;
    const bool extras = (P.volume_mode != 0 && P.nvol > 0) || P.nexpr > 0;
    if (P.compensated) return extras ? FT_GENERIC : (FT_LEAN | FT_COMP | (P.curvature_mode == 1 ? FT_CURV : 0));
    return FT_LEAN | (P.curvature_mode == 1 ? FT_CURV : 0) | (extras ? (defer ? FT_DEFER : FT_EXTRAS) : 0);
}

// Step kernel for a dimension, integrator, wind layout (pair = window-pair buffer) and feature
// set (kernel_features).
AdvanceFn advance_f32(int dim, bool rk4, bool pair, int ft);
AdvanceFn advance_bf16(int dim, bool rk4, bool pair, int ft);
AdvanceFn advance_f16(int dim, bool rk4, bool pair, int ft);

}  // namespace granite_b200
