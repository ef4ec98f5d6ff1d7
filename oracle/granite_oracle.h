/*
 * granite_oracle.h — CPU restatement of pygranite's trajectory step path.
 *
 * TEST INFRASTRUCTURE ONLY.  The CUDA engine in pygranite_b200/ is verified against
 * this oracle; only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg may
 * load it.  It is never the thing measured or shipped.
 *
 * Parity pins: the reference (catheart97/pygranite v1.5.0) ships no tests, golden
 * vectors or known-answer tests (its PYGRANITE_TEST hook points at a file that does
 * not exist, source/pygranite.cpp:37-39).  This oracle is pinned by (1) analytic
 * known answers (uniform wind, linear-in-time wind, solid-body rotation) in
 * tests/test_oracle.py and (2) fixtures produced by the reference's own `integrate`
 * kernel built from its sources and run on a B200 (tests/golden/, tests/test_golden.py).
 *
 * One source, both precisions in liboracle.so:
 *   *_f64  REAL = double : the accuracy reference (ideal arithmetic, exact 1/scale).
 *   *_f32  REAL = float  : follows the CUDA kernel's float operation order (explicit
 *                          fmaf, no contraction) so positions, status, lengths and
 *                          curvature compare bit for bit.
 */
#ifndef GRANITE_ORACLE_H
#define GRANITE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Flat pre-order AST node, same layout and meaning as granite::ASTANode
 * (source/granite/Language.hpp:80-86): Left child at i+1, Right at 1+|left| (cpp:770-798). */
typedef struct {
    uint32_t type;
    float value;
    int32_t left;
    int32_t right;
} or_node;

typedef struct {
    /* resolved settings (reference TrajectoryIntegrator.tpp:521-574 done by the caller) */
    int32_t dim;              /* 2 or 3 */
    int32_t rk4;              /* Integrator::ClassicRungeKutta */
    int32_t border_mode;      /* BorderMode (2D only; 3D runs Block) */
    int32_t curvature_mode;   /* CurvatureMode */
    int32_t abort_mode;       /* AbortMode */
    int32_t uplift_mode;      /* UpLiftMode (3D only) */
    int32_t windfield_mode;   /* WindfieldMode */
    int32_t constants_mode;   /* ConstantsMode */
    int32_t volume_mode;      /* AdditionalVolumeMode */
    int32_t use_topography;
    int32_t reverse;
    int32_t use_sphere;       /* 2D and SphereRadius > 0 */
    int32_t time_mode;        /* 0: weights from the float32 accumulator (reference); 1: from float64 time */
    int32_t minimum_alive;
    int32_t compensated;      /* Kahan-compensated position update (the engine's precision form) */
    int64_t save_interval;
    float sphere_radius, delta_t, data_time_distance, maximum_length, maximum_simulation_time;
    float scale[3], offset[3], domain[3];
    int64_t nx, ny, nz;
    int32_t n_volumes, n_constants, n_expr, n_snapshots;
    const float *const *wind;      /* [n_snapshots * dim] planes, (nz,ny,nx) or (ny,nx) */
    const float *const *volumes;   /* [n_snapshots * n_volumes] planes */
    const float *const *constants; /* [n_snapshots * n_constants], n floats each */
    const float *const *uplift;    /* [n_snapshots], n*dim floats each */
    const float *topography;       /* (ny,nx) or NULL */
    const or_node *const *expr;    /* [n_expr] */
    const int32_t *expr_len;       /* [n_expr] */
    int64_t n;
    const float *seeds;            /* n*dim */
    int32_t threads;               /* OpenMP threads, 0 = runtime default */
    int64_t step_limit;            /* >= 0: stop after this many steps (bounded timing sample) */
    int32_t filter_weights;        /* 0: exact filter fractions; 1 / 2: fractions rounded / truncated
                                      to 1/256 like texture hardware (reference GPU comparisons) */
    int64_t start_step;            /* particles integrate from this step of the clock on (a request
                                      joining mid-run); earlier steps leave them where they are */
} or_input;

typedef struct {
    int64_t max_records;
    float *positions;         /* [max_records][n][dim] */
    int32_t *status;          /* [n] */
    float *lengths;           /* [n] */
    float *total_curvature;   /* [n] */
    float *curvature;         /* [max_records][n] */
    float *volume_info;       /* [n_volumes][max_records][n] */
    float *compute_info;      /* [n_expr][max_records][n] */
    int64_t *step_of_abort;   /* [n] step index at which status left Time, -1 if never */
    /* results */
    int64_t records;
    int64_t curvature_records;
    int64_t info_records;
    int64_t steps;
    int64_t particle_steps;
    int64_t windows;
    double seconds;           /* wall time of the step loop */
    int32_t error;
    char message[256];
} or_output;

/* Per-step schedule entry (reference TrajectoryIntegrator.tpp:852-912, 973-994). */
typedef struct {
    int64_t window;      /* snapshot window counter: back = window, front = window+1 */
    int32_t save;        /* a position record is written after this step */
    int32_t time_pos;    /* data.Time > 0 at the start of the step */
    double t0, t1, t2;   /* time weights of the stages, float64 */
    float t0f, t1f, t2f; /* time weights as the float32 kernel uses them */
} or_step;

int oracle_run_f64(const or_input *in, or_output *out);
int oracle_run_f32(const or_input *in, or_output *out);

/* Builds the step schedule without integrating (alive checks disabled).  Returns the
 * number of steps written (<= cap), or -1.  *windows_out = number of windows run. */
int64_t oracle_schedule(const or_input *in, or_step *steps, int64_t cap, int64_t *windows_out);

/* Evaluates one flat AST on one reference vector, the way interpret() does
 * (source/granite/TrajectoryIntegrator.hpp:539-627). */
float oracle_interpret_f32(const or_node *nodes, int64_t n, const float *ref, int64_t i);
double oracle_interpret_f64(const or_node *nodes, int64_t n, const double *ref, int64_t i);

#ifdef __cplusplus
}
#endif

#endif
