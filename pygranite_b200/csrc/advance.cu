// advance.cu — instantiates the step kernel (granite_kernels.cuh) for one wind storage type,
// chosen by the build: GR_ADVANCE_F32, GR_ADVANCE_BF16 or GR_ADVANCE_F16.  Ring layouts get the
// generic variant only; window-pair layouts also the eight lean ones (advance.h).
#include "advance.h"

namespace granite_b200 {

namespace {

template <int DIM, bool RK4, typename T>
AdvanceFn pick_pair(int ft) {
    switch (ft) {
        case FT_LEAN: return advance_kernel<DIM, RK4, Pair<T>, FT_LEAN>;
        case FT_LEAN | FT_CURV: return advance_kernel<DIM, RK4, Pair<T>, FT_LEAN | FT_CURV>;
        case FT_LEAN | FT_EXTRAS: return advance_kernel<DIM, RK4, Pair<T>, FT_LEAN | FT_EXTRAS>;
        case FT_LEAN | FT_CURV | FT_EXTRAS: return advance_kernel<DIM, RK4, Pair<T>, FT_LEAN | FT_CURV | FT_EXTRAS>;
        case FT_LEAN | FT_COMP: return advance_kernel<DIM, RK4, Pair<T>, FT_LEAN | FT_COMP>;
        case FT_LEAN | FT_COMP | FT_CURV: return advance_kernel<DIM, RK4, Pair<T>, FT_LEAN | FT_COMP | FT_CURV>;
        case FT_LEAN | FT_DEFER: return advance_kernel<DIM, RK4, Pair<T>, FT_LEAN | FT_DEFER>;
        case FT_LEAN | FT_CURV | FT_DEFER: return advance_kernel<DIM, RK4, Pair<T>, FT_LEAN | FT_CURV | FT_DEFER>;
        default: return advance_kernel<DIM, RK4, Pair<T>, FT_GENERIC>;
    }
}

template <typename T>
AdvanceFn pick(int dim, bool rk4, bool pair, int ft) {
    if (pair) {
        if (dim == 3) return rk4 ? pick_pair<3, true, T>(ft) : pick_pair<3, false, T>(ft);
        return rk4 ? pick_pair<2, true, T>(ft) : pick_pair<2, false, T>(ft);
    }
    if (dim == 3) return rk4 ? advance_kernel<3, true, T, FT_GENERIC> : advance_kernel<3, false, T, FT_GENERIC>;
    return rk4 ? advance_kernel<2, true, T, FT_GENERIC> : advance_kernel<2, false, T, FT_GENERIC>;
}

}  // namespace

#if defined(GR_ADVANCE_F32)
AdvanceFn advance_f32(int dim, bool rk4, bool pair, int ft) { return pick<float>(dim, rk4, pair, ft); }
#elif defined(GR_ADVANCE_BF16)
AdvanceFn advance_bf16(int dim, bool rk4, bool pair, int ft) { return pick<__nv_bfloat16>(dim, rk4, pair, ft); }
#elif defined(GR_ADVANCE_F16)
AdvanceFn advance_f16(int dim, bool rk4, bool pair, int ft) { return pick<__half>(dim, rk4, pair, ft); }
#else
#error "define GR_ADVANCE_F32, GR_ADVANCE_BF16 or GR_ADVANCE_F16"
#endif

}  // namespace granite_b200
