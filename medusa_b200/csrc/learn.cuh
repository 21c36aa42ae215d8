// learn.cuh -- learned-scheduler training and trace collection (internal).
#pragma once
#include "sched.cuh"

namespace mb {
struct BfsState;
struct SsspState;
struct MsBfsState;

// Gradient and loss (means over n samples, weighted by each sample's best
// time) of the MLP with parameters P on features X [n][6] and schedule
// times T [n][8]; all device pointers; loss_dev holds 2 floats (loss, and
// the weights' normaliser).
void mlp_grad(Context &ctx, const float *P_dev, const float *X_dev, const float *T_dev, int32_t n,
              float *G_dev, float *loss_dev);
// Train the weights P (device, kMlpParams floats) from a seeded
// initialisation with full-batch Adam; returns the final loss.
float mlp_train(Context &ctx, float *P, const float *X_dev, const float *T_dev, int32_t n,
                int32_t epochs, float lr, uint64_t seed);
// Training range of a model set from outside (weights given by the caller):
// unbounded.
void mlp_set_open_bounds(Context &ctx, float *P);
// Schedule the MLP with weights P picks for each of n feature rows; with
// fallback_dev (nullable), the in-run rule: fallback[i] unless the network's
// best output beats it by kOverrideMargin.
void mlp_pick(Context &ctx, const float *P, const float *X_dev, const int32_t *fallback_dev,
              int32_t n, int32_t *out_dev);
// Timing traces of one traversal (app APP_BFS / APP_SSSP from `source`;
// APP_MSBFS: batched BFS from `source` and the 63 vertices after it): per
// superstep, its features, the time of each schedule (-1: not measured; the
// batched traversal measures push 0 and pull 4) and (fixed_out, nullable)
// the fixed rule's choice.  Returns the sample count.
int32_t collect_traces(Context &ctx, Graph &g, BfsState &bst, SsspState &sst, MsBfsState &mst,
                       int app, int32_t source, float *feat_out, float *times_out,
                       int32_t *fixed_out, int32_t max_samples);
}  // namespace mb
