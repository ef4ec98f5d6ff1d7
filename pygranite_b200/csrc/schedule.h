// schedule.h — the host-side step schedule of one simulation.
//
// Restates the reference's host loop: computeLoop_ (source/granite/TrajectoryIntegrator.tpp:
// 778-918) and computeLoopGPU_ (tpp:920-995).  The step count, the window each step runs in,
// the save steps and the float32 time weights are reproduced exactly, including the float32
// time accumulator `data.Time += DeltaT` and the window switch `Time >= max_windfield_time`.
// The schedule assumes the loader never runs dry and MinimumAliveParticles never triggers;
// the engine truncates it when either happens.
#pragma once

#include <cstdint>
#include <vector>

namespace granite_b200 {

struct HostStep {
    int64_t window;        // back snapshot = window, front = window + 1
    bool save;             // a record is written after the step
    bool time_pos;         // data.Time > 0 at the start of the step
    float t0, t1, t2;      // float32 time weights (reference arithmetic or float64-derived)
    double t0d, t1d, t2d;  // float64 weights
};

struct ScheduleInput {
    bool dyn_any;              // some quantity is Dynamic
    bool wind_dynamic;
    float delta_t, data_time_distance, maximum_simulation_time;
    int64_t save_interval;
    int time_mode;             // 0 float32 accumulator weights, 1 float64
};

struct Schedule {
    std::vector<HostStep> steps;
    std::vector<int64_t> window_begin;   // first step of each window; size windows + 1
    bool time_positive_at_end = false;   // data.Time > 0 after the last step
};

Schedule build_schedule(const ScheduleInput &in);

}  // namespace granite_b200
