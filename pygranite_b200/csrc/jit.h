// jit.h — run-time compiled deferred volume / expression kernel (jit.cu).
#pragma once

#include <string>

#include <cuda_runtime.h>

#include "expr.h"

namespace granite_b200 {

// Source of the deferred kernel with expressions progs[0 .. nexpr) as straight-line code
// ("" if some program cannot be translated).
std::string jit_source(const Program *progs, int nexpr, int dim);

// The compiled kernel gr_jit_deferred_extras(KParams, rec, irec, k_end, all) for these
// expressions, compiled once per distinct source and process; null (and `why`) where run-time
// compilation is unavailable or fails.
cudaKernel_t jit_deferred_kernel(const Program *progs, int nexpr, int dim, std::string &why);

}  // namespace granite_b200
