// kernels.h -- launch arguments of the round kernels (host <-> device).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "layout.h"
#include "learned.h"

namespace necsim {

constexpr int kStepBlockMax = 256;
// block size of the cooperative kernel (one lineage per warp)
constexpr int kCoopBlock = 128;
// simulations with at most this many live lineages run in the resident kernel
constexpr int kResidentMax = 256;

// SMs set aside for the priority engine's tails.  While `on` is nonzero the
// persistent kernels of an engine with role kGateAvoid leave the SMs whose
// id (%smid) has its bit set in `mask`, and those of an engine with role
// kGateOnly run only there, so a tail's dependent event chain does not share
// its issue slots with bulk warps.  Which blocks do the work never changes
// what is computed: the work is claimed dynamically, and the last block of a
// launch to leave takes whatever is still unclaimed.
struct SmGate {
    uint32_t on;
    uint32_t mask[8];  // SM ids 0..255
};
constexpr uint32_t kGateNone = 0, kGateAvoid = 1, kGateOnly = 2;

struct StepArgs {
    LineageSoA in;                       // lineages of this round (updated in place)
    uint8_t *state;                      // per slot: 0 alive, 1 speciated, 2 dropped
    const uint32_t *order;               // queue order of slots (nullptr: identity)
    const unsigned long long *n_cur;     // live lineages in `in`
    unsigned long long *work;            // queue head (reset by the scheduler)
    const SimParams *params;
    SimCounters *counters;
    DevSpeciationEvent *spec;
    unsigned long long *n_spec_total;
    uint64_t spec_cap;
    DevDispersalEvent *disp;
    unsigned long long *n_disp_total;
    uint64_t disp_cap;
    int report_dispersal;
    uint32_t *status;
    unsigned long long *steps_total;     // optional per-launch event count
    uint32_t n_sims;                     // simulations in `params`
    TraceSink trace;                     // death records of speciated lineages (tracing only)
    uint32_t exp_sampler;                // 1: exponential event-time sampler (exp.rs), else Poisson
    // Poisson sampler: rounds with at most this many live lineages run in
    // the cooperative kernel (one warp per lineage, at most its resident
    // warps); 0: the step kernel takes every round
    uint64_t coop_max;
    // cooperative kernel: a simulation with one live lineage runs up to this
    // many of its next rounds in the same launch while other warps are busy
    // (or it is the launch's only simulation); 0: off.  `busy` counts the
    // warps holding a lineage (zero between launches)
    uint32_t free_rounds;
    unsigned int *busy;
    const SmGate *gate;                  // SM reservation (nullable) and this engine's role in it
    uint32_t gate_role;
    unsigned int *blocks_done;           // blocks of the round's kernel that have finished or left
                                         // (reset by the scheduler)
};

struct DedupArgs {
    LineageSoA arena;                    // resident arena (x == nullptr: no routing)
    uint64_t resident_max;               // route simulations that start a round with at most this many (<= kResidentMax)
    const SimParams *params;             // lineage_offset of each simulation
    LineageSoA in;
    LineageSoA out;
    const uint8_t *state;
    uint8_t *state_out;
    const unsigned long long *n_cur;
    const unsigned long long *mask;      // table slots - 1 for this round
    uint32_t *owner;                     // slot -> owning lineage (0xffffffff empty)
    unsigned long long *min_gref;        // slot -> smallest global reference
    uint32_t *slot;                      // lineage -> slot
    unsigned long long *out_count;
    SimCounters *counters;
    uint32_t *status;
    TraceSink trace;                     // death records of removed duplicates (tracing only)
};

struct ScheduleArgs {
    SimParams *params;
    SimCounters *counters;
    uint32_t n_sims;
    uint32_t dedup_pct;
    unsigned long long *n_cur;
    unsigned long long *out_count;
    unsigned long long *work;
    unsigned long long *mask;
    unsigned long long table_size;
    unsigned int *n_active;
    unsigned long long *visits;          // lineages the scheduled rounds process
    unsigned int *n_resident;            // active simulations owned by the resident kernel
    unsigned int *blocks_done;           // the next round's kernel arrivals (reset here)
};

// the step kernel on grid x block and, for the Poisson sampler with
// a.coop_max > 0, the cooperative kernel on coop_grid x kCoopBlock before it
// (a.coop_max at most coop_grid's warps); each returns at once in the
// other's rounds
cudaError_t launch_step(int kind, const StepArgs &a, unsigned grid, unsigned block, unsigned coop_grid,
                        cudaStream_t st);
cudaError_t step_kernel_occupancy(int kind, bool exp_sampler, int block, int *blocks_per_sm);
cudaError_t coop_kernel_occupancy(int kind, int *blocks_per_sm);
cudaError_t launch_dedup(const DedupArgs &a, unsigned grid, unsigned block, cudaStream_t st);
cudaError_t launch_schedule(const ScheduleArgs &a, cudaStream_t st);

struct ResidentArgs {
    LineageSoA arena;                    // lineages of resident simulations, by segment
    SimParams *params;
    SimCounters *counters;
    uint32_t n_sims;
    uint32_t budget;                     // rounds per simulation in this launch
    DevSpeciationEvent *spec;
    unsigned long long *n_spec_total;
    uint64_t spec_cap;
    uint32_t *status;
    unsigned long long *steps_total;
    unsigned long long *visits;
    unsigned int *n_resident;
    const int *stop_flag;                // set when the concurrent global rounds end (nullable)
    uint32_t exp_sampler;                // 1: exponential event-time sampler (exp.rs), else Poisson
    const SmGate *gate;                  // SM reservation (nullable) and this engine's role in it
    uint32_t gate_role;
    unsigned int *claim;                 // with a gate: next simulation to claim, and the blocks
    unsigned int *blocks_done;           // that have finished or left (both zero at launch)
};

// The SM ids present on the device: bit smid of mask[smid / 32] is set by a
// block that ran there (grid blocks of 32 threads; mask zeroed before).
cudaError_t launch_sm_census(uint32_t *mask, unsigned grid, cudaStream_t st);

cudaError_t launch_resident(int kind, const ResidentArgs &a, unsigned grid, cudaStream_t st);
cudaError_t launch_promote(SimParams *params, uint32_t n_sims, cudaStream_t st);
// AlmostInfinite displacements before rounding (kind kAlmostInfiniteNormal: a =
// sigma; else Clark2Dt: a = shape u, b = 1 / p) of n sample pairs
cudaError_t launch_displacements(int32_t kind, const uint64_t *draws, uint64_t n, double a, double b, double *dx,
                                 double *dy, unsigned grid, cudaStream_t st);
// 8 * 256 * grid * iters wymum in independent chains (the hash-issue ceiling)
cudaError_t launch_hash_peak(unsigned grid, uint64_t seed, uint32_t iters, unsigned long long *sink,
                             cudaStream_t st);

}  // namespace necsim
