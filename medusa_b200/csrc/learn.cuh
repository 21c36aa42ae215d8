// learn.cuh -- learned-scheduler training and trace collection (internal).
#pragma once
#include "sched.cuh"

namespace mb {
struct BfsState;
struct SsspState;

// Gradient (mean over n samples) and mean loss of the MLP with parameters P
// on features X [n][6] and schedule times T [n][8]; all device pointers.
void mlp_grad(Context &ctx, const float *P_dev, const float *X_dev, const float *T_dev, int32_t n,
              float *G_dev, float *loss_dev);
// Train ctx.mlp from a seeded initialisation with full-batch Adam; returns the final loss.
float mlp_train(Context &ctx, const float *X_dev, const float *T_dev, int32_t n, int32_t epochs,
                float lr, uint64_t seed);
// Schedule the trained MLP picks for each of n feature rows.
void mlp_pick(Context &ctx, const float *X_dev, int32_t n, int32_t *out_dev);
// Timing traces of one traversal (app APP_BFS / APP_SSSP): per superstep, its
// features, the time of each of the 8 schedules and (fixed_out, nullable)
// the fixed rule's choice.  Returns the sample count.
int32_t collect_traces(Context &ctx, Graph &g, BfsState &bst, SsspState &sst, int app,
                       int32_t source, float *feat_out, float *times_out, int32_t *fixed_out,
                       int32_t max_samples);
}  // namespace mb
