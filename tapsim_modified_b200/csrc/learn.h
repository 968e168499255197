// Hooks of the learned warm start (learn.cu) used by tg_solve (handle.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "kernels.cuh"

struct tg_learner;

// the device the learner's buffers live on (current at tg_learner_create)
int learner_device(const tg_learner* L);
// sizes the per-mesh scratch (global -> graph index map); fails when the
// graph width is below the mesh's longest row
int learner_attach_mesh(tg_learner* L, size_t meshNodes, int maxRow);
// graph and features of `site` from the current state; with `collect` the
// features are stored as a new sample (finished by learner_collect_end);
// with `predict` the prediction is added to the potentials of the graph's
// cells, and with `hist` also to the recorded correction of their V slots
// (slotOf: node -> slot), so that the next event recycles all of it
int learner_predict(tg_learner* L, const tgd::DevMesh& m, int site, cudaStream_t s, bool collect, bool predict,
                    const int32_t* slotOf, float* hist);
// the cells of the last graph (device list, its length on the device) and
// the list's capacity: the cells whose potentials a prediction changed
void learner_graph_cells(const tg_learner* L, const int32_t** nodes, const int32_t** count, int* capacity);
// the target of the sample started by learner_predict, from the converged state
int learner_collect_end(tg_learner* L, const tgd::DevMesh& m, cudaStream_t s);
// drops a sample that learner_predict started
void learner_collect_cancel(tg_learner* L);
