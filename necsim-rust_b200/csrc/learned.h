// learned.h -- the learned lifetime scheduler: a small MLP that predicts a
// lineage's remaining event count from its state, trained and evaluated by
// this file's kernels, and the bucket sort that turns its predictions into
// the step kernel's queue order.  The predictor only reorders work: every
// lineage still executes exactly the events it would execute unordered.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "layout.h"

namespace necsim {

// MLP 8 -> 64 -> 64 -> 1 with ReLU hidden layers, predicting from a
// lineage's features log(1 + remaining events) of its simulation's
// longest-lived lineage.  Parameters are one flat array:
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
constexpr uint64_t kTraceRowsPerSim = 256;

struct TraceRow {
    float f[kFeat];
    uint64_t gref;
    uint64_t steps;
    uint32_t sim;
    uint32_t snap;   // the snapshot's index in the run
    double time;     // the lineage's time (its last event) at the snapshot
};
static_assert(sizeof(TraceRow) == 64, "TraceRow layout");

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

// The eight features of a lineage, each scaled to about [0, 1]:
//   0, 1  position in the scenario's extent (x / width, y / height; the
//         metacommunity's own extent for an SI lineage outside the local
//         community; 0 on the unbounded AlmostInfinite plane)
//   2     log(1 + habitat at the location) / 8 (deme size)
//   3     entropy (nats) of the location's dispersal distribution / 16
//   4     log(1 + time of the lineage's last event) / 20
//   5     -log10(speciation probability per event at the location) / 15
//         (SI local community: speciation happens after migration, nu * m)
//   6     log(1 + live lineages of the simulation) / 16 (crowding)
//   7     log(1 + events the lineage has executed) / 20 (age)
// `se_habitat` and `se_entropy` are the SpatiallyExplicit cell's habitat and
// dispersal entropy (read from the device tables by the kernels, from the
// maps by the host).  The same source serves the kernels and the host.
__host__ __device__ inline void lineage_features_of(int kind, const SimParams &p, uint64_t n_live, uint32_t x,
                                                    uint32_t y, double last, uint64_t steps, float se_habitat,
                                                    float se_entropy, float f[kFeat]) {
    float fx = 0.f, fy = 0.f, hab = 1.f, ent = 0.f;
    float nu = (float)p.nu;
    if (kind == kNonSpatial) {
        fx = (float)x / (float)p.width;
        fy = (float)y / (float)p.height;
        hab = (float)p.deme;
        ent = logf((float)p.width * (float)p.height);
    } else if (kind == kSpatiallyImplicit) {
        if (x <= p.width - 1 && y <= p.height - 1) {  // the local community (extent at (0, 0))
            fx = (float)x / (float)p.width;
            fy = (float)y / (float)p.height;
            hab = (float)p.deme;
            // entropy of one dispersal: uniform over the local community with
            // probability 1 - m, over the metacommunity with probability m;
            // the speciation probability is the metacommunity's, where the
            // lineage must migrate to speciate
            const float m = fminf(fmaxf((float)p.migration, 0.f), 1.f);
            const float h = (m > 0.f ? -m * logf(m) : 0.f) + (m < 1.f ? -(1.f - m) * logf(1.f - m) : 0.f);
            ent = (1.f - m) * logf((float)p.width * (float)p.height) +
                  m * logf((float)p.meta_width * (float)p.meta_height) + h;
        } else {
            fx = (float)(x - p.meta_ox) / (float)p.meta_width;
            fy = (float)(y - p.meta_oy) / (float)p.meta_height;
            hab = (float)p.meta_deme;
            ent = logf((float)p.meta_width * (float)p.meta_height);
        }
    } else if (kind == kAlmostInfiniteNormal) {
        // differential entropy of the 2D dispersal kernel: normal, or a
        // Clark2Dt kernel of scale sqrt(u) (sigma 0: none)
        const float scale2 = p.clark ? (float)p.clark_shape_u : (float)p.sigma * (float)p.sigma;
        ent = logf(fmaxf(2.0f * 3.14159265f * 2.71828183f * scale2, 1.0f));
    } else if (kind == kWrappingNoise) {
        // the Normal kernel's entropy, restricted to the habitable share
        const float scale2 = (float)p.sigma * (float)p.sigma;
        ent = logf(fmaxf(2.0f * 3.14159265f * 2.71828183f * scale2 * (float)p.noise.coverage, 1.0f));
    } else {
        fx = (float)x / (float)p.width;
        fy = (float)y / (float)p.height;
        hab = se_habitat;
        ent = se_entropy;
    }
    f[0] = fx;
    f[1] = fy;
    f[2] = log1pf(hab) * 0.125f;
    f[3] = ent * 0.0625f;
    f[4] = log1pf((float)last) * 0.05f;
    f[5] = -log10f(fmaxf(nu, 1e-15f)) * (1.0f / 15.0f);
    f[6] = log1pf((float)n_live) * 0.0625f;
    f[7] = log1pf((float)steps) * 0.05f;
}

// Appends a snapshot row for about kTraceRowsPerSim live lineages of every
// active simulation of `f.in`, chosen by a hash of (global reference,
// snapshot) (rows beyond `cap` are counted but not written).
cudaError_t launch_trace_snapshot(const FeatureArgs &f, uint32_t snap, TraceRow *rows, unsigned long long *n_rows,
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
