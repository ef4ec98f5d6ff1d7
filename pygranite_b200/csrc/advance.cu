// advance.cu — instantiates the step kernel (granite_kernels.cuh) for one wind storage type,
// chosen by the build: GR_ADVANCE_F32, GR_ADVANCE_BF16 or GR_ADVANCE_F16.
#include "advance.h"

namespace granite_b200 {

namespace {

template <typename T>
AdvanceFn pick(int dim, bool rk4, bool pair) {
    if (pair) {
        if (dim == 3) return rk4 ? advance_kernel<3, true, Pair<T>> : advance_kernel<3, false, Pair<T>>;
        return rk4 ? advance_kernel<2, true, Pair<T>> : advance_kernel<2, false, Pair<T>>;
    }
    if (dim == 3) return rk4 ? advance_kernel<3, true, T> : advance_kernel<3, false, T>;
    return rk4 ? advance_kernel<2, true, T> : advance_kernel<2, false, T>;
}

}  // namespace

#if defined(GR_ADVANCE_F32)
AdvanceFn advance_f32(int dim, bool rk4, bool pair) { return pick<float>(dim, rk4, pair); }
#elif defined(GR_ADVANCE_BF16)
AdvanceFn advance_bf16(int dim, bool rk4, bool pair) { return pick<__nv_bfloat16>(dim, rk4, pair); }
#elif defined(GR_ADVANCE_F16)
AdvanceFn advance_f16(int dim, bool rk4, bool pair) { return pick<__half>(dim, rk4, pair); }
#else
#error "define GR_ADVANCE_F32, GR_ADVANCE_BF16 or GR_ADVANCE_F16"
#endif

}  // namespace granite_b200
