/*
 * granite_b200.h — C ABI of the B200 trajectory engine (libgranite_b200.so).
 *
 * This is the boundary under pygranite's Python surface.  The reference binds its C++
 * classes directly with pybind11 (source/pygranite.cpp:41-152); it has no C ABI.  Each
 * entry point below states which reference interface it replaces.  The pybind11 module
 * pygranite_b200/_pygranite (same class, method and enum names as the reference) is one
 * caller; ctypes, cgo or JNI callers bind the same symbols.
 *
 * Conventions: every call returns GR_OK (0) or a negative status; no call exits the
 * process or throws.  gr_last_error() returns the message of the last failure on the
 * calling thread, prefixed like the reference's exceptions ("ERROR < USER INPUT | ..." for
 * bad input, "ERROR < RUNTIME | ..." for CUDA or internal faults).  Host buffers belong to
 * the caller and are copied before the call returns; device memory belongs to the engine.
 * One engine is driven by one host thread at a time.
 */
#ifndef GRANITE_B200_H
#define GRANITE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GR_OK 0
#define GR_ERR_USER (-1)      /* invalid input; the reference throws MY_USER_ERROR */
#define GR_ERR_RUNTIME (-2)   /* CUDA or internal failure; the reference calls exit(1) */
#define GR_ERR_CALLBACK (-3)  /* the loader callback reported a failure */

#define GR_MAX_VOLUMES 8      /* MAX_ADDITIONAL_VOLUMES, source/granite/Constants.hpp:9 */
#define GR_MAX_EXPRESSIONS 4  /* MAX_ADDITIONAL_COMPUTE, Constants.hpp:10 */
#define GR_MAX_CONSTANTS 4    /* MAX_CONSTANT_ADDITIONAL_COMPUTE, Constants.hpp:12 */

/* Wind storage type of the device snapshot ring. */
#define GR_STORE_F32 0
#define GR_STORE_BF16 1
#define GR_STORE_F16 2

/* Settings.  Enum fields take the reference's values (IntegratorSettings.hpp:16-76);
 * float/int fields mirror IntegratorSettings.hpp:83-181.  GridScale/Offset keep the
 * reference's 1..3-entry lists (grid_scale_len / offset_len). */
typedef struct gr_settings {
    int32_t space;                 /* Space: 0 Space3D, 1 Space2D */
    int32_t integrator;            /* Integrator: 0 ExplicitEuler, 1 ClassicRungeKutta */
    int32_t windfield_mode;        /* WindfieldMode: 0 Constant, 1 Dynamic */
    int32_t constants_mode;        /* ConstantsMode: 0 Off, 1 Constant, 2 Dynamic */
    int32_t volume_mode;           /* AdditionalVolumeMode: 0 Off, 1 Constant, 2 Dynamic */
    int32_t uplift_mode;           /* UpLiftMode: 0 Off, 1 Constant, 2 Dynamic */
    int32_t border_mode;           /* BorderMode: 0 Block, 1 LoopX, 2 LoopY, 3 LoopXY */
    int32_t curvature_mode;        /* CurvatureMode: 0 Off, 1 Total, 2 FastTotal, 3 IndividualAndTotal */
    int32_t abort_mode;            /* AbortMode: 0 Time, 1 Length, 2 FitLength */
    int32_t reverse;               /* Reverse */
    int32_t minimum_alive;         /* MinimumAliveParticles */
    int32_t grid_scale_len;        /* entries used in grid_scale (1..3) */
    int32_t offset_len;            /* entries used in offset (1..3) */
    float sphere_radius;           /* SphereRadius */
    float delta_t;                 /* DeltaT */
    float data_time_distance;      /* DataTimeDistance */
    float maximum_length;          /* MaximumLength */
    float maximum_simulation_time; /* MaximumSimulationTime */
    float grid_scale[3];           /* GridScale */
    float offset[3];               /* Offset */
    int64_t save_interval;         /* SaveInterval */
    /* engine options beyond the reference (0 = reference behaviour) */
    int32_t storage;               /* GR_STORE_*: wind storage in the device ring */
    int32_t time_mode;             /* 0: time weights from the float32 accumulator the reference
                                      keeps; 1: from a float64 accumulator */
    int32_t compensated;           /* 1: Kahan-compensated float32 position update */
    int32_t ring_slots;            /* device ring depth (>= 3); 0 = 3 */
    int32_t steps_per_launch;      /* steps fused into one launch; 0 = one snapshot window */
    int32_t sort_interval;         /* launches between Morton re-sorts / compactions; 0 = off; negative
                                    * (the default): every 8 launches from 65,536 particles, else off */
    int32_t block_size;            /* threads per block; 0 = autotuned default; capped at the step
                                      kernel's launch bound (128 for the float32 3D window-pair
                                      kernel, 256 for the others) */
    int32_t device;                /* CUDA device ordinal */
    int32_t layout;                /* wind layout read by the step kernel: 0 = window pairs when the
                                      windfield is dynamic (one load returns the back and the front
                                      snapshot), 1 = the ring slots directly */
    int32_t grid_waves;            /* graph runs: resident waves of step-kernel blocks in the
                                      persistent grid (each thread walks live particles with a
                                      grid stride); 0 = 1 */
    int32_t filter_weights;        /* 0: exact interpolation weights (float32 software filter);
                                      1: fractions rounded to the nearest 1/256, the 8-bit weights
                                      of the texture unit the reference filters with
                                      (TrajectoryIntegrator.icc:22-50; cpp:444-583), which
                                      reproduces its 2D results bit for bit */
} gr_settings;

/* Fills *s with the reference's IntegratorSettings defaults (IntegratorSettings.hpp:89-181). */
void gr_settings_default(gr_settings *s);

typedef struct gr_engine gr_engine;

/* Loader callback: called with the snapshot index the run needs next (the reference's
 * `_loader.step()` followed by updateData, TrajectoryIntegrator.tpp:887-889,
 * TrajectoryIntegrator.cpp:261-360).  It must push that snapshot's dynamic quantities
 * with gr_load_* and return 1, return 0 when the loader is exhausted (step() == False),
 * or a negative value on failure.  Called on the thread that called gr_run. */
typedef int (*gr_loader_fn)(void *user, gr_engine *engine, int64_t snapshot);

/* Result sizes after gr_run. */
typedef struct gr_result_info {
    int64_t n;                   /* particles */
    int32_t dim;                 /* 2 or 3 */
    int64_t records;             /* position records incl. the seed record (lengthTrajectories) */
    int64_t curvature_records;   /* per-step curvature records (IndividualAndTotalCurvature) */
    int64_t info_records;        /* volume / compute records */
    int64_t steps;               /* integrator steps run */
    int64_t windows;             /* snapshot windows run */
    int64_t particle_steps;      /* alive particles advanced, summed over steps */
    int32_t n_volumes;
    int32_t n_expressions;
} gr_result_info;

/* Timing and traffic counters of the last gr_run. */
typedef struct gr_stats {
    double kernel_ms;            /* summed device time of the step launches (CUDA events) */
    double run_ms;               /* device time from first upload to last result byte */
    int64_t launches;            /* step-kernel launches */
    int64_t aux_launches;        /* pack / sort / save kernels */
    int64_t particle_steps;
    int64_t h2d_bytes;
    int64_t d2h_bytes;
    int64_t jit_launches;        /* deferred volume / expression launches of run-time compiled code */
} gr_stats;

/* Step plan of a run whose loader never runs dry: counts and, if the arrays are non-null,
 * per step the window index, flags (1 = record after the step, 2 = data.Time > 0 at its
 * start) and the three float32 time weights.  Restates the bookkeeping of computeLoop_ /
 * computeLoopGPU_ (TrajectoryIntegrator.tpp:778-995); needs no GPU, so callers can size
 * result buffers before a run. */
typedef struct gr_plan_info {
    int64_t steps;
    int64_t windows;
    int64_t records;             /* position records incl. the seed record */
    int64_t curvature_records;
    int64_t info_records;
} gr_plan_info;

int gr_plan(const gr_settings *settings, gr_plan_info *out, int64_t capacity, int64_t *window,
            int32_t *flags, float *weights);

/* Create / destroy.  Replaces the TrajectoryIntegrator constructor's resource setup
 * (TrajectoryIntegrator.hpp:138-147) and destructor (TrajectoryIntegrator.cpp:362-422). */
int gr_create(const gr_settings *settings, gr_engine **out);
void gr_destroy(gr_engine *engine);

/* Message of the last failure on this thread ("" if none). */
const char *gr_last_error(void);

/* Snapshot loads.  Replace loadTexture3D / loadTexture2D (TrajectoryIntegrator.cpp:444-609)
 * and the constants / uplift uploads (cpp:195-245, 305-359).  `snapshot` is the loader
 * step the data belongs to (0 = the data present at construction).  Planes are C-order
 * (z, y, x) for 3D and (y, x) for 2D, float32.  The first wind load fixes the grid. */
int gr_load_windfield(gr_engine *engine, int64_t snapshot, const float *const *components,
                      int32_t n_components, int64_t nz, int64_t ny, int64_t nx);
int gr_load_volume(gr_engine *engine, int64_t snapshot, int32_t index, const float *data,
                   int64_t nz, int64_t ny, int64_t nx);
int gr_load_constant(gr_engine *engine, int64_t snapshot, int32_t index, const float *data,
                     int64_t n);
int gr_load_uplift(gr_engine *engine, int64_t snapshot, const float *data, int64_t n, int32_t dim);
/* Topography (IntegratorSettings.Topography; initializeTopography, cpp:635-663). */
int gr_set_topography(gr_engine *engine, const float *data, int64_t ny, int64_t nx);

/* Compiles one AdditionalCompute expression to device bytecode.  Replaces parse /
 * replace_environment / contains / flatten (TrajectoryIntegrator.cpp:4-144, 744-798,
 * TrajectoryIntegrator.tpp:647-712).  volume_names[k] binds to volume index k and
 * constant_names[k] to constant index k. */
int gr_compile_expression(gr_engine *engine, int32_t index, const char *code,
                          const char *const *volume_names, int32_t n_volumes,
                          const char *const *constant_names, int32_t n_constants);

/* Compiles `code` like gr_compile_expression and evaluates it on the host for one
 * reference vector ref[19] = {x, y, z, cv, f0..f7, c0..c3, u, v, w}
 * (TrajectoryIntegrator.tpp:381-439).  Needs no GPU; returns GR_ERR_USER with the
 * reference's message for an invalid expression. */
int gr_expression_evaluate(const char *code, const char *const *volume_names, int32_t n_volumes,
                           const char *const *constant_names, int32_t n_constants, int32_t dim,
                           int32_t curvature_mode, const float *ref, float *out);

/* Seeds (the last record of the TrajectorySet handed to the constructor,
 * TrajectoryIntegrator::initSet, cpp:424-442). */
int gr_set_seeds(gr_engine *engine, const float *positions, int64_t n, int32_t dim);

/* Runs the whole simulation.  Replaces compute() (cpp:687-693) with compute_ /
 * computeLoop_ / computeLoopGPU_ (TrajectoryIntegrator.tpp:467-995). */
int gr_run(gr_engine *engine, gr_loader_fn loader, void *user);

int gr_result_info_get(gr_engine *engine, gr_result_info *out);
int gr_stats_get(gr_engine *engine, gr_stats *out);

/* Results, copied into caller buffers.  Shapes follow the reference's accessors
 * (TrajectorySet.cpp:90-253): positions (n, records, dim); status (n); lengths (n);
 * total curvature (n); curvatures (n, curvature_records); volume / compute info
 * (n, info_records). */
int gr_fetch_positions(gr_engine *engine, float *out, int64_t capacity_floats);
int gr_fetch_status(gr_engine *engine, int32_t *out, int64_t capacity);
int gr_fetch_lengths(gr_engine *engine, float *out, int64_t capacity);
int gr_fetch_total_curvature(gr_engine *engine, float *out, int64_t capacity);
int gr_fetch_curvatures(gr_engine *engine, float *out, int64_t capacity_floats);
int gr_fetch_volume_info(gr_engine *engine, int32_t index, float *out, int64_t capacity_floats);
int gr_fetch_compute_info(gr_engine *engine, int32_t index, float *out, int64_t capacity_floats);
/* The last position record of every particle, (n, dim). */
int gr_fetch_final_positions(gr_engine *engine, float *out, int64_t capacity_floats);

/* Result streaming.  The reference copies every saved step to the host synchronously inside
 * its step loop (copyParticleInfo, TrajectoryIntegrator.tpp:997-1049).  Here the records stay
 * in a device history, and with destinations set, gr_run also copies the position, volume and
 * compute records into these caller arrays while it runs: whenever enough records are complete
 * (rows of at least 256 bytes per particle), one pitched DMA per array on a separate stream,
 * overlapped with the steps and the snapshot uploads; the remainder when the run ends.  When
 * gr_run returns, record r of particle i is at positions[(i * records_capacity + r) * dim + d]
 * for r < records (gr_result_info_get), volume k's record r at
 * volume_info[k][i * info_capacity + r] and expression e's at compute_info[e][i *
 * info_capacity + r] for r < info_records.  The capacities must cover the run's records (the
 * counts of gr_plan for the same settings), and every non-null array must lie in page-locked
 * host memory (gr_host_alloc, cudaHostAlloc, cudaHostRegister): GR_ERR_USER at gr_run
 * otherwise.  Null arrays are not copied.  Runs with MinimumAliveParticles copy at the end
 * only; graph runs (gr_batch_*) do not stream.  The device history stays valid, so the
 * gr_fetch_* calls still work.  The destinations apply to every later gr_run of the engine
 * until gr_set_result_destinations(engine, NULL). */
typedef struct gr_result_destinations {
    float *positions;                           /* (n, records_capacity, dim) */
    int64_t records_capacity;
    float *volume_info[GR_MAX_VOLUMES];         /* (n, info_capacity) each */
    float *compute_info[GR_MAX_EXPRESSIONS];    /* (n, info_capacity) each */
    int64_t info_capacity;
} gr_result_destinations;

int gr_set_result_destinations(gr_engine *engine, const gr_result_destinations *dest);

/* Page-locked host memory.  No counterpart in the reference, whose uploads and result copies
 * are synchronous copies from and to pageable memory (TrajectoryIntegrator.cpp:444-609,
 * TrajectoryIntegrator.tpp:997-1049).  Every load above whose source, and every fetch whose
 * destination, lies wholly in page-locked memory (from gr_host_alloc, cudaHostAlloc or
 * cudaHostRegister) is one DMA with no staging copy; a load from such memory returns once the
 * DMA has read it.  Other buffers go through the engine's pinned staging and a parallel host
 * copy.
 * gr_host_alloc serves requests up to 4 KiB from 4 KiB slots of shared 2 MiB slabs; larger ones
 * round up to 2 MiB and get a cached block when one of the size (up to a quarter larger) is free; gr_host_free returns a block to the cache while the cached total
 * stays within the limit (default: a quarter of physical memory; gr_host_cache_limit), and
 * frees it otherwise.  gr_host_free of a pointer not from gr_host_alloc is GR_ERR_USER.
 * gr_host_is_pinned returns 1 if `p` lies in page-locked memory known to CUDA, else 0. */
typedef struct gr_host_cache_stats {
    int64_t live_bytes;     /* handed out, not yet freed */
    int64_t cached_bytes;   /* freed, kept for reuse */
    int64_t limit_bytes;
    int64_t allocations;    /* page-locked allocations made */
    int64_t reuses;         /* requests served from the cache */
} gr_host_cache_stats;

int gr_host_alloc(int64_t bytes, void **out);
int gr_host_free(void *p);
int gr_host_cache_limit(int64_t bytes);
int gr_host_cache_trim(void);
int gr_host_cache_stats_get(gr_host_cache_stats *out);
int gr_host_is_pinned(const void *p);

/* Device memory.  Every device buffer of engines, servers and fields comes from one CUDA memory
 * pool per device that keeps freed memory mapped for reuse (the reference calls cudaMalloc /
 * cudaFree per run and per integrator, TrajectoryIntegrator.tpp:477-503, 577-771 and
 * TrajectoryIntegrator.cpp:362-422).  A failed allocation trims the pool and retries once.
 * gr_device_cache_stats_get reports the pool's mapped and in-use bytes (0 / 0 before its first
 * use); gr_device_cache_trim returns the idle memory of every pool to the driver. */
int gr_device_cache_stats_get(int32_t device, int64_t *reserved_bytes, int64_t *used_bytes);
int gr_device_cache_trim(void);

/* Device-resident variants for callers that keep data on the GPU: the same loads and
 * seeds from device pointers (no host copy). */
int gr_load_windfield_device(gr_engine *engine, int64_t snapshot, const float *const *components,
                             int32_t n_components, int64_t nz, int64_t ny, int64_t nx);
int gr_set_seeds_device(gr_engine *engine, const float *positions, int64_t n, int32_t dim);

/* Run options between runs.  No counterpart in the reference (its settings are fixed at
 * construction).  Everything the loaded data was built for must stay the same: space, the
 * windfield / constants / volume / uplift modes, grid scale and offset, storage, ring slots,
 * device (GR_ERR_USER otherwise).  Integrator, border / curvature / abort modes, time step,
 * lengths, MaximumSimulationTime, SaveInterval and the engine options may change. */
int gr_update_settings(gr_engine *engine, const gr_settings *settings);
int gr_settings_get(const gr_engine *engine, gr_settings *out);

/* Per-particle lifetimes in integrator steps (n = the seed count; steps = NULL clears them).
 * No counterpart in the reference, where every particle runs until MaximumSimulationTime.  A
 * particle stops after its lifetime: it keeps status Time (0) and its later records repeat
 * its last state, exactly what a separate run of it with MaximumSimulationTime = lifetime *
 * DeltaT leaves in its last record.  A run ends after the longest lifetime.  Seed sets of
 * different lengths on one windfield are batched this way. */
int gr_set_lifetimes(gr_engine *engine, const int32_t *steps, int64_t n);

/* Batches: several engines run as one CUDA graph.  No counterpart in the reference.
 * Each engine's whole run (seeding, every step launch, compaction and re-sorting passes,
 * the final records) is enqueued with fixed launch shapes — the step kernel walks the live
 * particles with a persistent grid-stride loop over a device-side count — captured on its own
 * stream, forked from and joined to the batch stream, and instantiated once.  Every
 * gr_batch_run replays the graph, so results are those of a fresh gr_run of each engine over
 * the snapshots resident in its ring (its ring must hold every snapshot the run reads, loaded
 * before the first gr_batch_run; the loader is not called).  MinimumAliveParticles is not
 * supported (it needs host decisions between steps).  A call that changes an engine (loads,
 * seeds, lifetimes, settings, expressions, gr_run) makes the next gr_batch_run capture again.
 * All engines must use the same device.  A batch keeps pointers to its engines: destroy the
 * batch before any of them. */
typedef struct gr_batch gr_batch;
typedef struct gr_batch_stats {
    double graph_ms;             /* device time of the last replay (CUDA events) */
    int64_t nodes;               /* graph nodes */
    int64_t kernel_launches;     /* step-kernel launches per replay */
    int64_t aux_launches;        /* other kernels and memsets per replay */
    int64_t particle_steps;      /* summed over the engines, last replay */
    int64_t captures;            /* graphs built so far */
    int64_t replays;
} gr_batch_stats;
int gr_batch_create(gr_engine *const *engines, int32_t n_engines, gr_batch **out);
void gr_batch_destroy(gr_batch *batch);
int gr_batch_run(gr_batch *batch);
int gr_batch_stats_get(const gr_batch *batch, gr_batch_stats *out);

/* Autotuner: picks the wind layout, block size, sort interval and persistent-grid waves of an
 * engine by timing short runs (`trial_steps` steps each, resident snapshots, graph launch
 * shapes) and stores the fastest in its settings.  No counterpart in the reference.  Trials
 * overwrite the engine's results. */
typedef struct gr_tune_result {
    int32_t layout, block_size, sort_interval, grid_waves;
    double particle_steps_per_s;   /* of the chosen configuration */
    int32_t trials;
} gr_tune_result;
int gr_tune(gr_engine *engine, int32_t trial_steps, gr_tune_result *out);

/* Request server: continuous batching of trajectory requests over one field.  No counterpart
 * in the reference, which integrates one seed set per TrajectoryIntegrator.
 *
 * The field (n_snapshots snapshots of nz x ny x nx nodes, DataTimeDistance apart, stored as
 * settings->storage) is packed once into pinned host memory by gr_server_set_snapshot.  A
 * worker thread sweeps it window by window through a 4-slot device ring refilled from there.
 * A request is a seed set, a start time (seconds on the field's clock, rounded down to the
 * step grid DeltaT), a step count and an integrator (0 Euler, 1 RK4); it runs from its start step
 * until the step count, an abort, or the end of the field, whichever comes first.  Requests
 * whose start falls in the current window join the particle pool of their integrator, while
 * their state fits `hbm_budget_bytes` (0 = a quarter of the free device memory); all requests
 * in flight advance together, one launch per integrator and window.  A request whose start
 * window the sweep has passed waits for the next sweep.  Results (final positions and abort
 * codes) are those of an integration of the request alone.  Positions only: settings with
 * curvature, volumes, constants, uplift, length abort, MinimumAliveParticles or compensation
 * are rejected.  Submit, wait, result, cancel and stats may be called from any thread. */
#define GR_REQ_PENDING 0
#define GR_REQ_ACTIVE 1
#define GR_REQ_DONE 2
#define GR_REQ_CANCELLED 3
#define GR_REQ_FAILED 4
typedef struct gr_server gr_server;
typedef struct gr_request_info {
    int64_t n;
    int32_t dim, integrator;
    int64_t start_step;          /* on the field's step clock */
    int64_t steps;               /* steps it runs (after clipping at the field's end) */
    double submit_s, admit_s, done_s;   /* server clock, seconds since gr_server_start */
    int32_t state;               /* GR_REQ_* */
} gr_request_info;
typedef struct gr_server_stats {
    int64_t submitted, admitted, completed, cancelled;
    int64_t deferred;            /* admissions postponed for lack of HBM budget */
    int64_t windows, sweeps, jumps;
    int64_t particle_steps;
    int64_t capacity_particles;  /* particle slots per integrator pool */
    int64_t peak_particles;      /* most particles in flight at once */
    int64_t h2d_bytes, d2h_bytes;
    int64_t pending, active;
    int64_t clock_steps;         /* steps of the field's clock */
    int64_t windows_per_sweep;
    int64_t staged_later;        /* completions whose copy-out waited for pinned staging */
} gr_server_stats;
int gr_server_create(const gr_settings *settings, int64_t n_snapshots, int64_t nz, int64_t ny, int64_t nx,
                     int64_t hbm_budget_bytes, gr_server **out);
/* Snapshot k as float32 planes (z, y, x) / (y, x); device_src = 1 for device pointers. */
int gr_server_set_snapshot(gr_server *server, int64_t snapshot, const float *const *components,
                           int32_t n_components, int32_t device_src);
int gr_server_start(gr_server *server);
int gr_server_submit(gr_server *server, const float *seeds, int64_t n, int32_t dim, double start_time,
                     int32_t steps, int32_t integrator, int64_t *request_id);
/* Waits until the request is done, cancelled or failed (timeout_s < 0: no limit). */
int gr_server_wait(gr_server *server, int64_t request_id, double timeout_s, int32_t *state);
/* Info, and when done the final positions (n, dim) and abort codes (n). */
int gr_server_result(gr_server *server, int64_t request_id, gr_request_info *info, float *positions,
                     int32_t *status, int64_t capacity);
int gr_server_release(gr_server *server, int64_t request_id);
int gr_server_cancel(gr_server *server, int64_t request_id);
int gr_server_stats_get(gr_server *server, gr_server_stats *out);
void gr_server_destroy(gr_server *server);

/* Native loaders: analytic windfields evaluated on the device.  The reference feeds every
 * snapshot through a Python DataLoader returning numpy arrays (DataLoader.hpp:26-81,
 * TrajectoryIntegrator.cpp:146-360); for synthetic fields these generate each snapshot on the
 * GPU (float64 arithmetic, rounded to float32) and load it with gr_load_windfield_device, so
 * a run needs no host snapshot memory and no Python.
 *   double gyre: u = -pi A sin(pi f) cos(pi y), v = pi A cos(pi f) sin(pi y) df/dx with
 *     f = eps sin(w t) x^2 + (1 - 2 eps sin(w t)) x on nodes x_i = i lx/nx, y_j = j ly/ny, 2D;
 *   Fourier modes: component c at node (z, y, x) = scale_c * sum_m amp_cm
 *     cos(phase_cm - omega_cm t + k_cm . (z dz, y dy, x dx)), 2D or 3D; k, amp, phase, omega
 *     given per component and mode (k in the grid's axis order: (z, y, x) or (y, x)).
 * Snapshot k is the field at time k * snapshot_dt. */
typedef struct gr_field gr_field;
int gr_field_double_gyre(double A, double eps, double omega, int64_t ny, int64_t nx, double lx, double ly,
                         double snapshot_dt, int64_t n_snapshots, int32_t device, gr_field **out);
int gr_field_fourier(int32_t dim, const int64_t *shape, const double *spacing, int32_t n_modes,
                     const double *k, const double *amp, const double *phase, const double *omega,
                     const double *scale, double snapshot_dt, int64_t n_snapshots, int32_t device,
                     gr_field **out);
/* Evaluates snapshot k and loads it into the engine's ring (the engine's device). */
int gr_field_load(gr_field *field, gr_engine *engine, int64_t snapshot);
/* A gr_loader_fn for gr_run: user = the gr_field; returns 0 past its last snapshot. */
int gr_field_loader(void *user, gr_engine *engine, int64_t snapshot);
/* Snapshot k's planes copied to host memory, (dim, nz, ny, nx) float32. */
int gr_field_snapshot(gr_field *field, int64_t snapshot, float *out, int64_t capacity_floats);
void gr_field_destroy(gr_field *field);

/* Allocation-free advance of particles between two snapshots.  No counterpart in the
 * reference.  It exists for callers that cannot call cudaMalloc: plug-in hosts whose device
 * memory belongs to their own pool allocator (an allocation behind its back escapes the host's
 * accounting and limits), and real-time loops that forbid allocation after start-up (an
 * allocation may synchronise the device or take an unbounded time).  It allocates no device
 * memory and calls no allocating routine; the caller owns every input and output buffer:
 *   wind_back / wind_front: the two snapshots, node-major (z, y, x), float4 {u, v, w, 0}
 *     per node in 3D or float2 {u, v} in 2D, on the device;
 *   px, py, pz, status: particle positions and abort codes (0 = alive), device arrays of n,
 *     updated in place; pz unused in 2D.
 * It runs `steps` integrator steps starting at time_start, which must lie in
 * [time_back, time_front), with the reference's float32 time arithmetic (T = T + DeltaT; a
 * step that ends past time_front extrapolates the weights, as the reference's last step of a
 * window does), and writes the particle-steps done to *particle_steps (if non-null; this
 * synchronises `stream`).  Only the plain integrator: Euler / RK4 with dynamic wind, Reverse,
 * border modes, sphere coordinates, ReferenceFilter; no curvature, volumes, constants, uplift,
 * topography, length abort, MinimumAliveParticles, constant wind, 16-bit storage, Kahan
 * positions or float64 time weights (GR_ERR_USER otherwise).
 * Its scratch (the per-step time weights and two counters, GR_NOALLOC_SCRATCH_BYTES) is one
 * file-scope device array that every GPU loading the library holds until the process exits;
 * steps beyond GR_NOALLOC_MAX_STEPS are rejected.  The first call on a device looks up that
 * array's device address (cudaGetSymbolAddress) and keeps it for the life of the process, so
 * make that first call before any stream capture; a cudaDeviceReset between calls is not
 * supported.  Each call rebuilds the weights and clears the counters on `stream` before its
 * step kernel.  All calls share the array: calls whose work overlaps on the GPU (different
 * streams, no ordering between them) race. */
#define GR_NOALLOC_MAX_STEPS 4096
#define GR_NOALLOC_SCRATCH_BYTES (GR_NOALLOC_MAX_STEPS * 48 + 16)
int gr_advance_noalloc(const gr_settings *settings, int64_t nz, int64_t ny, int64_t nx,
                       const void *wind_back, const void *wind_front, float time_back,
                       float time_front, float time_start, int32_t steps, float *px, float *py,
                       float *pz, int32_t *status, int64_t n, void *stream,
                       int64_t *particle_steps);

#ifdef __cplusplus
}
#endif

#endif
