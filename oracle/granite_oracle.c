/*
 * granite_oracle.c — CPU restatement of pygranite's step path (TEST INFRASTRUCTURE ONLY).
 *
 * The schedule below restates the reference's host loop: computeLoop_
 * (source/granite/TrajectoryIntegrator.tpp:778-918) and computeLoopGPU_ (tpp:920-995), with
 * the initial loader step of initializeData (source/granite/TrajectoryIntegrator.cpp:247-256).
 * The precision-generic particle step is oracle_step.inc, included once per precision.
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off, no fast-math).
 */
#include "granite_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static double or_now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ---------------------------------------------------------------- schedule */

typedef struct {
    const or_input *in;
    int dyn_any;
    int error;
    int done;
    int in_window;
    int abort_due_alive;
    int time_positive;     /* data.Time > 0 after the loop (for the SaveInterval == 0 record) */
    int64_t loaded;        /* snapshots handed over by the loader so far */
    int64_t counter;       /* window counter (tpp:782) */
    int64_t sim_counter;   /* _simulation_counter */
    int64_t windows;
    float time;            /* data.Time, float accumulator (tpp:990) */
    double time_d;         /* float64 accumulator (time_mode 1) */
    float max_wt;          /* max_windfield_time (tpp:783, 892) */
    float window_end;
    float tback, tfront;
    float limit;           /* MaximumSimulationTime / DeltaT, as the float the loop compares with */
} or_sched;

static void or_sched_init(or_sched *s, const or_input *in)
{
    memset(s, 0, sizeof *s);
    s->in = in;
    s->dyn_any = in->windfield_mode == 1 || in->uplift_mode == 2 || in->volume_mode == 2 ||
                 in->constants_mode == 2;
    s->loaded = 1;
    if (s->dyn_any) {
        /* initializeData: loader.step() must succeed once (cpp:247-256) */
        if (in->n_snapshots < 2) s->error = 1;
        s->loaded = 2;
    }
    s->max_wt = in->data_time_distance;
    s->limit = in->maximum_simulation_time / in->delta_t;
}

/* End of one computeLoopGPU_ call: the loader step and texture rotation of computeLoop_
 * (tpp:882-912). */
static void or_sched_after_window(or_sched *s)
{
    const or_input *in = s->in;
    s->in_window = 0;
    if (s->dyn_any) {
        if (s->loaded < in->n_snapshots) {   /* _loader.step() returned true */
            s->loaded++;
            if (s->abort_due_alive) { s->done = 1; return; }
            s->max_wt += in->data_time_distance;
            s->counter++;
        } else {
            s->done = 1;
            return;
        }
    }
    if (!(in->windfield_mode == 1 && (float)s->sim_counter < s->limit)) s->done = 1;
}

/* Produces the next step, or returns 0 when the simulation is over.  alive_ok is the value
 * alive() would return now (number alive >= MinimumAliveParticles). */
static int or_sched_next(or_sched *s, int alive_ok, or_step *st)
{
    const or_input *in = s->in;
    for (;;) {
        if (s->done || s->error) return 0;
        if (!s->in_window) {
            /* computeLoopGPU_ entry (tpp:933-934) */
            s->window_end = s->dyn_any ? s->max_wt : in->maximum_simulation_time;
            s->tback = (float)s->counter * in->data_time_distance;
            s->tfront = (float)(s->counter + 1) * in->data_time_distance;
            s->in_window = 1;
            s->windows++;
        }
        int cond = (float)s->sim_counter < s->limit;
        if (cond && in->minimum_alive) {
            s->abort_due_alive = !alive_ok;
            cond = alive_ok;
        }
        if (!cond) {
            or_sched_after_window(s);
            continue;
        }
        const float h = in->delta_t;
        const float T = s->time, TB = s->tback, TF = s->tfront;
        st->window = s->counter;
        st->save = in->save_interval != 0 && (s->sim_counter % in->save_interval) == 0;
        st->time_pos = T > 0.0f;
        /* unit_interval(x, front, back) = (x - back) / (front - back)  (LinearAlgebra.hpp:651-655) */
        st->t0f = (T - TB) / (TF - TB);
        st->t1f = ((T + 0.5f * h) - TB) / (TF - TB);
        st->t2f = ((T + h) - TB) / (TF - TB);
        if (in->time_mode == 1) {
            const double tb = (double)s->counter * (double)in->data_time_distance;
            const double tf = (double)(s->counter + 1) * (double)in->data_time_distance;
            const double td = s->time_d, hd = (double)h;
            st->t0 = (td - tb) / (tf - tb);
            st->t1 = ((td + 0.5 * hd) - tb) / (tf - tb);
            st->t2 = ((td + hd) - tb) / (tf - tb);
            st->t0f = (float)st->t0;
            st->t1f = (float)st->t1;
            st->t2f = (float)st->t2;
        } else {
            const double tb = TB, tf = TF, td = T, hd = h;
            st->t0 = (td - tb) / (tf - tb);
            st->t1 = ((td + 0.5 * hd) - tb) / (tf - tb);
            st->t2 = ((td + hd) - tb) / (tf - tb);
        }
        /* advance (tpp:990-993) */
        s->time = T + h;
        s->time_d += (double)h;
        s->sim_counter++;
        s->time_positive = s->time > 0.0f;
        if (s->time >= s->window_end) or_sched_after_window(s);
        return 1;
    }
}

int64_t oracle_schedule(const or_input *in, or_step *steps, int64_t cap, int64_t *windows_out)
{
    or_sched s;
    or_sched_init(&s, in);
    if (s.error) return -1;
    int64_t k = 0;
    or_step st;
    while (or_sched_next(&s, 1, &st)) {
        if (steps && k < cap) steps[k] = st;
        ++k;
    }
    if (windows_out) *windows_out = s.windows;
    return k;
}

/* ---------------------------------------------------------------- float64 reference */
#define REAL double
#define SUF(x) x##_f64
#define OR_IS_DOUBLE 1
#define R_FMA fma
#define R_SQRT sqrt
#define R_FLOOR floor
#define R_FABS fabs
#define R_COS cos
#define R_ACOS acos
#define R_FMOD fmod
#define R_FMIN fmin
#define R_FMAX fmax
#define R_EXP exp
#define R_LOG log
#define R_SIN sin
#define R_TAN tan
#define R_ASIN asin
#define R_ATAN atan
#define R_ATAN2 atan2
#include "oracle_step.inc"
#undef REAL
#undef SUF
#undef OR_IS_DOUBLE
#undef R_FMA
#undef R_SQRT
#undef R_FLOOR
#undef R_FABS
#undef R_COS
#undef R_ACOS
#undef R_FMOD
#undef R_FMIN
#undef R_FMAX
#undef R_EXP
#undef R_LOG
#undef R_SIN
#undef R_TAN
#undef R_ASIN
#undef R_ATAN
#undef R_ATAN2

/* ---------------------------------------------------------------- float32 mirror */
#define REAL float
#define SUF(x) x##_f32
#define OR_IS_DOUBLE 0
#define R_FMA fmaf
#define R_SQRT sqrtf
#define R_FLOOR floorf
#define R_FABS fabsf
#define R_COS cosf
#define R_ACOS acosf
#define R_FMOD fmodf
#define R_FMIN fminf
#define R_FMAX fmaxf
#define R_EXP expf
#define R_LOG logf
#define R_SIN sinf
#define R_TAN tanf
#define R_ASIN asinf
#define R_ATAN atanf
#define R_ATAN2 atan2f
#include "oracle_step.inc"
