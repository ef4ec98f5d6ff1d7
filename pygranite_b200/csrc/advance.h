// advance.h — the step-kernel variants, instantiated per wind storage type in advance.cu
// (compiled once per type so the variants build in parallel).
#pragma once

#include "granite_kernels.cuh"

namespace granite_b200 {

using AdvanceFn = void (*)(const KParams);

// Step kernel for a dimension, integrator and wind layout (pair = window-pair buffer).
AdvanceFn advance_f32(int dim, bool rk4, bool pair);
AdvanceFn advance_bf16(int dim, bool rk4, bool pair);
AdvanceFn advance_f16(int dim, bool rk4, bool pair);

}  // namespace granite_b200
