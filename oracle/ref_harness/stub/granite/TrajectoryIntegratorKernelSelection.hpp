// Stand-in for the header the reference's code generator writes
// (source/granite/TrajectoryIntegrator.gen.py:264-274): no compute_<...> dispatch members are
// needed, because the harness instantiates granite::integrate<...> directly.
#pragma once
#define PYGRANITE_KERNEL_SELECTION()
