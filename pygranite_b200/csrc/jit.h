// jit.h — run-time compiled deferred volume / expression kernel (jit.cu).
#pragma once

#include <string>

#include <cuda_runtime.h>

#include "expr.h"

namespace granite_b200 {

// A run's volume / expression options (the KParams fields of the same names), compiled into
// the kernel as constants.
struct JitOptions {
    int nvol, nexpr, ncon, volume_mode, constants_mode, curvature_mode, dyn_any;
};

// Source of the deferred kernel with expressions progs[0 .. o.nexpr) as straight-line code
// ("" if some program cannot be translated).
std::string jit_source(const Program *progs, const JitOptions &o, int dim);

// The compiled kernel gr_jit_deferred_extras(KParams, rec, irec, k_end, all) for these
// expressions and options, compiled once per distinct source and process; null (and `why`)
// where run-time compilation is unavailable or fails.  The kernel must be launched with KParams
// whose option fields equal `o`.
cudaKernel_t jit_deferred_kernel(const Program *progs, const JitOptions &o, int dim, std::string &why);

}  // namespace granite_b200
