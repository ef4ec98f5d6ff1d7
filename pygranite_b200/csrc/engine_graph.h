// engine_graph.h — what batch.cu needs of the engine (engine.cu) to capture engine runs into
// one CUDA graph.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/granite_b200.h"

namespace granite_b200 {

// Host plan and buffers of a run over the resident snapshots, with fixed launch shapes.
int graph_prepare(gr_engine *e);
// The whole run on the engine's stream: seeding, steps, compaction passes, final records.
// Enqueues device work only (no host reads or synchronisation), so it can be captured.
int graph_enqueue(gr_engine *e);
// After the enqueued run finished: counters and result sizes.
int graph_collect(gr_engine *e);
cudaStream_t engine_stream(gr_engine *e);
int engine_device(const gr_engine *e);
uint64_t engine_generation(const gr_engine *e);
int64_t engine_launches(const gr_engine *e, int64_t *aux);
int64_t engine_particle_steps(const gr_engine *e);
void set_last_error(const char *msg);

}  // namespace granite_b200
