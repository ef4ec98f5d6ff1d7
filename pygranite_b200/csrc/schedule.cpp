// schedule.cpp — see schedule.h.  Compiled without floating-point contraction so the
// float32 time arithmetic is exactly the reference's.
#include "schedule.h"

namespace granite_b200 {

Schedule build_schedule(const ScheduleInput &in) {
    Schedule out;
    const float h = in.delta_t;
    const float dtd = in.data_time_distance;
    // _simulation_counter < MaximumSimulationTime / DeltaT, compared in float (tpp:973-974)
    const float limit = in.maximum_simulation_time / in.delta_t;
    float time = 0.0f;          // data.Time (tpp:781)
    double time_d = 0.0;
    float max_wt = dtd;         // max_windfield_time (tpp:783)
    int64_t counter = 0;        // window counter
    int64_t sim = 0;            // _simulation_counter

    for (;;) {
        out.window_begin.push_back(static_cast<int64_t>(out.steps.size()));
        // computeLoopGPU_: dynamic runs stop at the window end, constant ones at the end time
        const float window_end = in.dyn_any ? max_wt : in.maximum_simulation_time;
        const float tb = static_cast<float>(counter) * dtd;
        const float tf = static_cast<float>(counter + 1) * dtd;
        while (static_cast<float>(sim) < limit) {
            HostStep s;
            s.window = counter;
            s.save = in.save_interval != 0 && (sim % in.save_interval) == 0;
            s.time_pos = time > 0.0f;
            const float t1 = time + 0.5f * h, t2 = time + h;
            s.t0 = (time - tb) / (tf - tb);
            s.t1 = (t1 - tb) / (tf - tb);
            s.t2 = (t2 - tb) / (tf - tb);
            if (in.time_mode == 1) {
                const double tbd = static_cast<double>(counter) * static_cast<double>(dtd);
                const double tfd = static_cast<double>(counter + 1) * static_cast<double>(dtd);
                const double hd = static_cast<double>(h);
                s.t0d = (time_d - tbd) / (tfd - tbd);
                s.t1d = ((time_d + 0.5 * hd) - tbd) / (tfd - tbd);
                s.t2d = ((time_d + hd) - tbd) / (tfd - tbd);
                s.t0 = static_cast<float>(s.t0d);
                s.t1 = static_cast<float>(s.t1d);
                s.t2 = static_cast<float>(s.t2d);
            } else {
                const double tbd = tb, tfd = tf, td = time, hd = h;
                s.t0d = (td - tbd) / (tfd - tbd);
                s.t1d = ((td + 0.5 * hd) - tbd) / (tfd - tbd);
                s.t2d = ((td + hd) - tbd) / (tfd - tbd);
            }
            out.steps.push_back(s);
            time = time + h;          // data.Time += data.DeltaT (tpp:990)
            time_d += static_cast<double>(h);
            ++sim;
            if (time >= window_end) break;   // tpp:993
        }
        // computeLoop_ after the window (tpp:882-912): the loader is assumed to deliver
        if (in.dyn_any) {
            max_wt += dtd;
            ++counter;
        }
        if (!(in.wind_dynamic && static_cast<float>(sim) < limit)) break;
    }
    out.window_begin.push_back(static_cast<int64_t>(out.steps.size()));
    out.time_positive_at_end = time > 0.0f;
    return out;
}

}  // namespace granite_b200
