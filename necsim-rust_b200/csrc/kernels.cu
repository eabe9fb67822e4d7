// kernels.cu -- sm_100a kernels of one synchronised round of the Independent
// algorithm: the persistent step kernel, the deterministic dedup (insert,
// compact, clear) and the per-simulation round scheduler.
//
// A round advances every live lineage of every active simulation to that
// simulation's horizon H (all events with time < H; the reference's
// early-stop rule `next_event_time >= level_time`,
// parallelisation/independent/monolithic/mod.rs:228-239), then removes
// lineages whose state (location, index, last event time) equals another's:
// such lineages share their whole future (the RNG is re-primed from
// (location, time) before every draw, event_time_sampler/poisson.rs:49 and
// :102-106), so this is the reference's duplicate-individual removal
// (monolithic/mod.rs:205-220) made exact and order-independent.  The
// survivor of each group is the lineage with the smallest global reference.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_core.cuh"
#include "kernels.h"

namespace necsim {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kEmpty = 0xffffffffu;

__device__ __forceinline__ void set_status(uint32_t *status, uint32_t bit) { atomicOr(status, bit); }

__device__ __forceinline__ unsigned long long f64_bits(double v) {
    return (unsigned long long)__double_as_longlong(v);
}

// ceil(speciation probability * 2^53) at a location
// (speciation_probability/uniform.rs; speciation_probability/spatially_implicit.rs:31-44)
template <int KIND>
__device__ __forceinline__ uint64_t speciation_threshold(const SimParams &p, uint32_t x, uint32_t y) {
    if (KIND == kSpatiallyImplicit && in_local(p, x, y)) return 0;
    return p.nu_threshold;
}

// Per-lane lineage registers.
struct Lane {
    uint32_t slot;
    uint32_t x, y, i, s;
    double last, next, horizon;
    uint64_t reprime, gref, steps;
    bool has_next;
    Rng g;
    CellRecord rec;  // SpatiallyExplicit: record of the current cell
};

template <int KIND>
__device__ __forceinline__ uint64_t lane_injection(const Lane &l, const SimParams &p) {
    if (KIND == kNonSpatial) return non_spatial_injection(0, 0, p.width, p.deme, l.x, l.y, l.i);
    if (KIND == kSpatiallyImplicit) {
        // habitat/spatially_implicit.rs:106-120
        if (in_local(p, l.x, l.y)) return non_spatial_injection(0, 0, p.width, p.deme, l.x, l.y, l.i);
        return non_spatial_injection(p.meta_ox, p.meta_oy, p.meta_width, p.meta_deme, l.x, l.y, l.i);
    }
    if (KIND == kAlmostInfiniteNormal) return ((uint64_t)l.y << 32) | (uint64_t)l.x;  // almost_infinite.rs:66-70
    return l.rec.injection + (uint64_t)l.i;                                          // in_memory.rs:70-80
}

__device__ __forceinline__ bool load_cell(const SimParams &p, uint32_t x, uint32_t y, CellRecord &rec,
                                          uint32_t *status) {
    const uint64_t cell = (uint64_t)y * p.width + (uint64_t)x;
    if (cell >= p.n_cells) {
        set_status(status, kErrCellIndex);
        return false;
    }
    rec = p.cells[cell];
    return true;
}

// packed_separable_alias/dispersal.rs:16-77 and alias/packed.rs:135-163, fed
// with the event's samples 2..4: the self-dispersal test (when taken) uses
// the first, the alias draw the next; `d_coal` receives the sample after them.
__device__ __forceinline__ bool spatially_explicit_dispersal_draw(
    uint64_t e2, uint64_t e3, uint64_t e4, const SimParams &p, uint32_t x, uint32_t y,
    const CellRecord &rec, uint32_t &tx, uint32_t &ty, uint64_t &d_coal, uint32_t *status) {
    const uint64_t cell = (uint64_t)y * p.width + (uint64_t)x;
    uint64_t target;
    const double sd = rec.self_dispersal;
    bool use_alias;
    uint64_t d_alias;
    if (sd == 1.0) {
        use_alias = false;
        d_alias = 0;
        d_coal = e2;
    } else if (sd == 0.0 || (uint64_t)rec.non_self_event != cell) {
        use_alias = true;
        d_alias = e2;
        d_coal = e3;
    } else {
        use_alias = unit_closed_open(e2) >= sd;
        d_alias = e3;
        d_coal = use_alias ? e4 : e3;
    }
    if (!use_alias) {
        target = cell;
    } else {
        const uint64_t len = rec.atom_count;
        const double f = __dmul_rn(__dmul_rn(unit_closed_open(d_alias), 1.0), __ull2double_rn(len));
        const uint64_t i = f64_to_u64(floor(f));
        const double frac = __dsub_rn(f, __ull2double_rn(i));
        const uint64_t at = (uint64_t)rec.atom_start + i;
        if (i >= len || at >= p.n_atoms) {
            set_status(status, kErrAtomIndex);
            return false;
        }
        const AliasAtom atom = p.atoms[at];
        target = (frac < atom.u) ? atom.e : atom.k;
    }
    // cell indices are < 2^32 (one CellRecord per cell): 32-bit divide
    const uint32_t t32 = (uint32_t)target, w32 = p.width;
    const uint32_t q = t32 / w32;
    tx = t32 - q * w32;
    ty = q;
    return true;
}

}  // namespace

// One lane per lineage at a time; a lane whose lineage reaches the horizon
// (or speciates) takes the next lineage of the queue, so warps stay full
// while lineages of very different event counts drain.
template <int KIND, bool SINGLE>
__global__ void __launch_bounds__(kStepBlockMax) step_kernel(StepArgs a) {
    // one simulation: its parameters live in shared memory for the launch
    __shared__ __align__(16) unsigned char params_smem[SINGLE ? sizeof(SimParams) : 16];
    if (SINGLE) {
        const uint4 *src = reinterpret_cast<const uint4 *>(a.params);
        uint4 *dst = reinterpret_cast<uint4 *>(params_smem);
        for (unsigned w = threadIdx.x; w < sizeof(SimParams) / 16; w += blockDim.x) dst[w] = src[w];
        __syncthreads();
    }
    const SimParams *P = SINGLE ? reinterpret_cast<const SimParams *>(params_smem) : a.params;
    const uint64_t n = *a.n_cur;
    const unsigned lane_id = threadIdx.x & 31u;
    const unsigned lanemask_lt = (1u << lane_id) - 1u;
    bool have = false;
    bool exhausted = (n == 0);
    Lane l;
    uint64_t local_steps = 0;

    for (;;) {
        const unsigned need = __ballot_sync(kFull, !have && !exhausted);
        if (need) {
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if ((int)lane_id == leader) base = atomicAdd(a.work, (unsigned long long)__popc(need));
            base = __shfl_sync(kFull, base, leader);
            if (!have && !exhausted) {
                const unsigned long long k = base + __popc(need & lanemask_lt);
                if (k < n) {
                    const uint32_t slot = a.order ? a.order[k] : (uint32_t)k;
                    const uint32_t s = a.in.sim[slot];
                    const SimParams &p = P[SINGLE ? 0 : s];
                    if (p.active) {
                        l.slot = slot;
                        l.s = s;
                        l.x = a.in.x[slot];
                        l.y = a.in.y[slot];
                        l.i = a.in.idx[slot];
                        l.last = a.in.last[slot];
                        l.next = a.in.next[slot];
                        l.reprime = a.in.reprime[slot];
                        l.gref = a.in.gref[slot];
                        l.steps = a.in.steps[slot];
                        l.has_next = a.in.has_next[slot] != 0;
                        l.horizon = p.horizon;
                        l.g.seed = p.seed;
                        l.g.state = p.seed;
                        have = true;
                        if (KIND == kSpatiallyExplicit) have = load_cell(p, l.x, l.y, l.rec, a.status);
                    }
                } else {
                    exhausted = true;
                }
            }
        }
        if (!__any_sync(kFull, have)) break;
        if (!have) continue;

        const SimParams &p = P[SINGLE ? 0 : l.s];
        const uint64_t loc_term = location_term(p.seed, lane_injection<KIND>(l, p));
        uint64_t rs;  // WyHash state re-primed for the event
        if (!l.has_next) {
            // IndependentActiveLineageSampler::pop_active_lineage_and_event_time
            // (active_lineage_sampler/independent/sampler.rs:69-116)
            const double before = l.last > p.min_event_time ? l.last : p.min_event_time;
            const double t = poisson_next_event_time_ilp(loc_term, before, p, l.reprime, rs);
            l.next = max_after(before, t);
            l.has_next = true;
        } else {
            rs = primed_state(loc_term, l.reprime);
        }

        if (__double_as_longlong(l.next) >= __double_as_longlong(l.horizon)) {  // non-negative
            // early stop: keep the peeked time for the next round
            a.in.x[l.slot] = l.x;
            a.in.y[l.slot] = l.y;
            a.in.idx[l.slot] = l.i;
            a.in.last[l.slot] = l.last;
            a.in.next[l.slot] = l.next;
            a.in.reprime[l.slot] = l.reprime;
            a.in.steps[l.slot] = l.steps;
            a.in.has_next[l.slot] = 1;
            have = false;
            continue;
        }

        // IndependentEventSampler::sample_event_for_lineage_at_event_time_or_emigrate
        // (event_sampler/independent.rs:112-222)
        l.steps += 1;
        local_steps += 1;
        // the event's samples 1..4 after the re-prime, drawn up front; which
        // of them the dispersal and coalescence use depends on the branch
        const uint64_t e1 = draw_at(rs, 1);
        const uint64_t e2 = draw_at(rs, 2);
        const uint64_t e3 = draw_at(rs, 3);
        const uint64_t e4 = (KIND == kNonSpatial) ? 0 : draw_at(rs, 4);
        // speciation iff U[0,1) < nu  <=>  (e1 >> 11) < ceil(nu * 2^53)
        if ((e1 >> 11) < speciation_threshold<KIND>(p, l.x, l.y)) {
            const unsigned long long e = atomicAdd(a.n_spec_total, 1ULL);
            if (e < a.spec_cap) {
                DevSpeciationEvent ev;
                ev.gref = l.gref;
                ev.prior_time = l.last;
                ev.event_time = l.next;
                ev.x = l.x;
                ev.y = l.y;
                ev.idx = l.i;
                ev.sim = l.s;
                a.spec[e] = ev;
            } else {
                set_status(a.status, kErrEventOverflow);
            }
            a.state[l.slot] = 1;
            SimCounters &c = a.counters[l.s];
            atomicAdd(&c.steps, (unsigned long long)l.steps);
            atomicMax(&c.max_time_bits, f64_bits(l.next));
            atomicAdd(&c.n_speciation, 1ULL);
            have = false;
            continue;
        }

        uint32_t tx, ty, ti;
        if (KIND == kNonSpatial) {
            non_spatial_dispersal_draw(e2, 0, 0, p.width, p.height, tx, ty);
            ti = coalescence_index(e3, p.deme);
        } else if (KIND == kSpatiallyImplicit) {
            // dispersal_sampler/spatially_implicit.rs:58-86
            const bool local = in_local(p, l.x, l.y);
            const bool to_meta = !local || (e2 >> 11) < p.migration_threshold;
            const uint64_t d_index = local ? e3 : e2;
            const uint64_t d_coal = local ? e4 : e3;
            if (to_meta)
                non_spatial_dispersal_draw(d_index, p.meta_ox, p.meta_oy, p.meta_width, p.meta_height, tx, ty);
            else
                non_spatial_dispersal_draw(d_index, 0, 0, p.width, p.height, tx, ty);
            // habitat/spatially_implicit.rs:95-103: local extent first
            ti = coalescence_index(d_coal, in_local(p, tx, ty) ? p.deme : p.meta_deme);
        } else if (KIND == kAlmostInfiniteNormal) {
            // sample e4 is CoalescenceRngSample::new's draw; singleton demes -> index 0
            normal_dispersal_draw(e2, e3, p.sigma, l.x, l.y, tx, ty);
            ti = 0;
        } else {
            uint64_t d_coal;
            if (!spatially_explicit_dispersal_draw(e2, e3, e4, p, l.x, l.y, l.rec, tx, ty, d_coal,
                                                   a.status) ||
                !load_cell(p, tx, ty, l.rec, a.status)) {
                a.state[l.slot] = 2;  // dropped by a failed bound check
                have = false;
                continue;
            }
            ti = coalescence_index(d_coal, l.rec.habitat);
        }
        if (a.report_dispersal) {
            const unsigned long long e = atomicAdd(a.n_disp_total, 1ULL);
            if (e < a.disp_cap) {
                DevDispersalEvent ev;
                ev.gref = l.gref;
                ev.prior_time = l.last;
                ev.event_time = l.next;
                ev.x = l.x;
                ev.y = l.y;
                ev.idx = l.i;
                ev.tx = tx;
                ev.ty = ty;
                ev.tidx = ti;
                ev.sim = l.s;
                ev.pad = 0;
                a.disp[e] = ev;
            } else {
                set_status(a.status, kErrDispersalOverflow);
            }
        }
        l.x = tx;
        l.y = ty;
        l.i = ti;
        l.last = l.next;
        l.has_next = false;
    }
    if (a.steps_total) {
        // one atomic per warp for the launch's event count
        unsigned long long w = local_steps;
        for (int off = 16; off > 0; off >>= 1) w += __shfl_down_sync(kFull, w, off);
        if (lane_id == 0 && w) atomicAdd(a.steps_total, w);
    }
}

namespace {

__device__ __forceinline__ uint64_t dedup_hash(uint32_t s, uint32_t x, uint32_t y, uint32_t i,
                                               double last) {
    uint64_t h = seahash_diffuse(((uint64_t)y << 32) | x);
    h ^= seahash_diffuse(((uint64_t)s << 32) | i) + 0x9e3779b97f4a7c15ULL;
    h ^= seahash_diffuse((uint64_t)__double_as_longlong(last) ^ 0x632be59bd9b4e019ULL);
    return seahash_diffuse(h);
}

__device__ __forceinline__ bool same_state(const LineageSoA &in, uint32_t a, uint32_t b) {
    return in.x[a] == in.x[b] && in.y[a] == in.y[b] && in.idx[a] == in.idx[b] &&
           in.sim[a] == in.sim[b] &&
           __double_as_longlong(in.last[a]) == __double_as_longlong(in.last[b]);
}

}  // namespace

__global__ void dedup_insert_kernel(DedupArgs a) {
    const uint64_t n = *a.n_cur;
    const uint64_t mask = *a.mask;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x * blockDim.x) {
        if (a.state[j] != 0) continue;
        uint64_t h = dedup_hash(a.in.sim[j], a.in.x[j], a.in.y[j], a.in.idx[j], a.in.last[j]) & mask;
        uint32_t slot = kEmpty;
        for (uint64_t probe = 0; probe <= mask; ++probe) {
            const uint32_t o = atomicCAS(&a.owner[h], kEmpty, (uint32_t)j);
            if (o == kEmpty || same_state(a.in, o, (uint32_t)j)) {
                atomicMin(&a.min_gref[h], (unsigned long long)a.in.gref[j]);
                slot = (uint32_t)h;
                break;
            }
            h = (h + 1) & mask;
        }
        if (slot == kEmpty) set_status(a.status, kErrDedupFull);
        a.slot[j] = slot;
    }
}

// Survivors (alive and holding their group's smallest global reference) are
// appended to the output arrays; duplicates hand their counters to the
// simulation.  Warp-aggregated appends keep the output dense.
__global__ void dedup_compact_kernel(DedupArgs a) {
    const uint64_t n = *a.n_cur;
    const unsigned lane_id = threadIdx.x & 31u;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint64_t j = base + threadIdx.x;
        bool survivor = false;
        bool dup = false;
        uint32_t s = 0;
        if (j < n && a.state[j] == 0) {
            s = a.in.sim[j];
            const uint32_t slot = a.slot[j];
            survivor = (slot == kEmpty) || a.min_gref[slot] == a.in.gref[j];
            dup = !survivor;
        }
        const unsigned sv = __ballot_sync(kFull, survivor);
        unsigned long long dst_base = 0;
        if (sv) {
            const int leader = __ffs(sv) - 1;
            if ((int)lane_id == leader) dst_base = atomicAdd(a.out_count, (unsigned long long)__popc(sv));
            dst_base = __shfl_sync(kFull, dst_base, leader);
        }
        if (survivor) {
            const uint64_t d = dst_base + __popc(sv & ((1u << lane_id) - 1u));
            a.out.x[d] = a.in.x[j];
            a.out.y[d] = a.in.y[j];
            a.out.idx[d] = a.in.idx[j];
            a.out.sim[d] = s;
            a.out.last[d] = a.in.last[j];
            a.out.next[d] = a.in.next[j];
            a.out.reprime[d] = a.in.reprime[j];
            a.out.gref[d] = a.in.gref[j];
            a.out.steps[d] = a.in.steps[j];
            a.out.has_next[d] = a.in.has_next[j];
            a.state_out[d] = 0;
        }
        // per-simulation live counts, aggregated over lanes of the same simulation
        const unsigned same = __match_any_sync(kFull, survivor ? s : 0xffffffffu);
        if (survivor && (__ffs(same) - 1) == (int)lane_id)
            atomicAdd(&a.counters[s].n_live_next, (unsigned long long)__popc(same));
        if (dup) {
            SimCounters &c = a.counters[s];
            atomicAdd(&c.steps, (unsigned long long)a.in.steps[j]);
            atomicMax(&c.max_time_bits, f64_bits(a.in.last[j]));
            atomicAdd(&c.n_dedup, 1ULL);
        }
    }
}

__global__ void dedup_clear_kernel(DedupArgs a) {
    const uint64_t n = *a.n_cur;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x * blockDim.x) {
        if (a.state[j] != 0) continue;
        const uint32_t slot = a.slot[j];
        if (slot == kEmpty) continue;
        a.owner[slot] = kEmpty;
        a.min_gref[slot] = ~0ULL;
    }
}

// Picks each simulation's next horizon from its live count:
// H' = min(H + clamp(ceil(min_round_events / n), step_slice, step_slice_max) / lambda, pause).
__global__ void schedule_kernel(ScheduleArgs a) {
    __shared__ unsigned int active_sum;
    if (threadIdx.x == 0) active_sum = 0;
    __syncthreads();
    unsigned int my_active = 0;
    for (uint32_t s = threadIdx.x; s < a.n_sims; s += blockDim.x) {
        SimParams &p = a.params[s];
        SimCounters &c = a.counters[s];
        const unsigned long long live = c.n_live_next;
        c.n_live = live;
        c.n_live_next = 0;
        const bool paused = p.pause_before >= 0.0 && !(p.horizon < p.pause_before);
        if (live > 0 && !paused) {
            const unsigned long long step_slice = p.step_slice ? p.step_slice : 1ULL;
            unsigned long long per = (p.min_round_events + live - 1) / live;
            if (p.step_slice_max && per > p.step_slice_max) per = p.step_slice_max;
            if (per < step_slice) per = step_slice;
            double h = __dadd_rn(p.horizon, __ddiv_rn(__ull2double_rn(per), p.lambda));
            if (p.pause_before >= 0.0 && p.pause_before < h) h = p.pause_before;
            p.horizon = h;
            p.active = 1;
            c.n_rounds += 1;
            my_active += 1;
        } else {
            p.active = 0;
        }
    }
    atomicAdd(&active_sum, my_active);
    __syncthreads();
    if (threadIdx.x == 0) {
        *a.n_active = active_sum;
        if (active_sum > 0) *a.visits += *a.out_count;
        const unsigned long long n = *a.out_count;
        *a.n_cur = n;
        *a.out_count = 0;
        *a.work = 0;
        unsigned long long want = (n * (unsigned long long)a.dedup_pct + 99ULL) / 100ULL;
        if (want < 2) want = 2;
        unsigned long long size = 1;
        while (size < want) size <<= 1;
        if (size > a.table_size) size = a.table_size;
        *a.mask = size - 1;
    }
}

// ---- host-side launchers ----
template <int KIND>
static cudaError_t launch_step_t(const StepArgs &a, unsigned grid, unsigned block, cudaStream_t st) {
    if (a.n_sims == 1)
        step_kernel<KIND, true><<<grid, block, 0, st>>>(a);
    else
        step_kernel<KIND, false><<<grid, block, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_step(int kind, const StepArgs &a, unsigned grid, unsigned block, cudaStream_t st) {
    switch (kind) {
    case kNonSpatial: return launch_step_t<kNonSpatial>(a, grid, block, st);
    case kSpatiallyImplicit: return launch_step_t<kSpatiallyImplicit>(a, grid, block, st);
    case kAlmostInfiniteNormal: return launch_step_t<kAlmostInfiniteNormal>(a, grid, block, st);
    case kSpatiallyExplicit: return launch_step_t<kSpatiallyExplicit>(a, grid, block, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t step_kernel_occupancy(int kind, int block, int *blocks_per_sm) {
    switch (kind) {
    case kNonSpatial:
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, step_kernel<kNonSpatial, false>, block, 0);
    case kSpatiallyImplicit:
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, step_kernel<kSpatiallyImplicit, false>, block, 0);
    case kAlmostInfiniteNormal:
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, step_kernel<kAlmostInfiniteNormal, false>, block, 0);
    case kSpatiallyExplicit:
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, step_kernel<kSpatiallyExplicit, false>, block, 0);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_dedup(const DedupArgs &a, unsigned grid, unsigned block, cudaStream_t st) {
    dedup_insert_kernel<<<grid, block, 0, st>>>(a);
    dedup_compact_kernel<<<grid, block, 0, st>>>(a);
    dedup_clear_kernel<<<grid, block, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_schedule(const ScheduleArgs &a, cudaStream_t st) {
    schedule_kernel<<<1, 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace necsim
