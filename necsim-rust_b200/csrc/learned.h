// learned.h -- the learned lifetime scheduler: a small MLP that predicts a
// lineage's remaining event count from its state, trained and evaluated by
// this file's kernels, and the bucket sort that turns its predictions into
// the step kernel's queue order.  The predictor only reorders work: every
// lineage still executes exactly the events it would execute unordered.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "layout.h"

namespace necsim {

// MLP 8 -> 64 -> 64 -> 1 with ReLU hidden layers, predicting
// log(1 + remaining events).  Parameters are one flat array:
constexpr int kFeat = 8;
constexpr int kHidden = 64;
constexpr int kW1 = 0;                        // [64][8]  layer 1 weights (row = output)
constexpr int kB1 = kW1 + kHidden * kFeat;    // [64]
constexpr int kW2 = kB1 + kHidden;            // [64][64] layer 2 weights (row = output)
constexpr int kB2 = kW2 + kHidden * kHidden;  // [64]
constexpr int kW3 = kB2 + kHidden;            // [64]     output weights
constexpr int kB3 = kW3 + kHidden;            // [1]
constexpr int kMlpParams = kB3 + 1;           // 4801
constexpr int kOrderBuckets = 32;

// One trace snapshot of a live lineage: its features and the step count at
// the snapshot, keyed by (simulation, global reference).
struct TraceRow {
    float f[kFeat];
    uint64_t gref;
    uint64_t steps;
    uint32_t sim;
    uint32_t pad;
};
static_assert(sizeof(TraceRow) == 56, "TraceRow layout");

// Where a lineage left the simulation (speciation or duplicate removal) and
// its step count there.
struct TraceDeath {
    uint64_t gref;
    uint64_t steps;
    uint32_t sim;
    uint32_t pad;
};
static_assert(sizeof(TraceDeath) == 24, "TraceDeath layout");

struct TraceSink {
    TraceDeath *deaths;                  // nullptr: not tracing
    unsigned long long *n_deaths;
    uint64_t cap;
};

// Lineages whose features are read.
struct FeatureArgs {
    LineageSoA in;
    const unsigned long long *n_cur;
    const SimParams *params;
    const SimCounters *counters;
    int kind;
    uint64_t skip_at_most;  // rounds with at most this many live lineages need no order
};

// Appends a snapshot row for every live lineage of `f.in` (rows beyond `cap`
// are counted but not written).
cudaError_t launch_trace_snapshot(const FeatureArgs &f, TraceRow *rows, unsigned long long *n_rows,
                                  uint64_t cap, cudaStream_t st);
// Fills pred_end (= steps + predicted remaining events) of every live lineage
// whose prediction is unset (0) or used up.
cudaError_t launch_lineage_predict(const FeatureArgs &f, const __nv_bfloat16 *w, float *pred_end,
                                   cudaStream_t st);
// Queue order of this round: lineages bucketed by expected work in the
// round, min(events per round, predicted remaining), the largest first.
// `hist` holds 2 * kOrderBuckets counters, zero before the first call.
cudaError_t launch_order(const FeatureArgs &f, const float *pred_end, uint8_t *keys, unsigned *hist,
                         uint32_t *order, unsigned grid, cudaStream_t st);

// y[i] = MLP(X[i]) for n feature rows.
cudaError_t launch_mlp_predict(const __nv_bfloat16 *w, const float *X, uint64_t n, float *y, cudaStream_t st);
// Accumulates into `grads` (fp32, kMlpParams) the gradient of
// sum_i 0.5 * (MLP(X[r_i]) - T[r_i])^2 * inv_n over rows r_i = perm[offset + i]
// (perm nullptr: offset + i), i < n, and the loss into *loss.
cudaError_t launch_mlp_grad(const __nv_bfloat16 *w, const float *X, const float *T, const uint32_t *perm,
                            uint64_t offset, uint64_t n, float inv_n, float *grads, double *loss,
                            cudaStream_t st);
// One Adam step on the fp32 master weights, re-rounding the bf16 copy;
// clears `grads`.
cudaError_t launch_adam(float *master, float *m, float *v, float *grads, __nv_bfloat16 *w, float lr,
                        float beta1, float beta2, float eps, int step, cudaStream_t st);

}  // namespace necsim
