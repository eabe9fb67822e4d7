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
#include "wrapping_noise.h"

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

// The event-time samplers' constants at the lineage's location: per cell
// under a SpatiallyExplicit turnover map (turnover_rate/in_memory.rs:22-40,
// the cell of a loaded lineage is in range), else the simulation's.
template <int KIND>
__device__ __forceinline__ const PoissonConsts &poisson_consts(const Lane &l, const SimParams &p) {
    if (KIND == kSpatiallyExplicit && p.turnover_cells) return p.turnover_cells[(uint64_t)l.y * p.width + l.x];
    return p.pois;
}

// The record of cell (x, y); false (and no read) when it lies outside the table.
__device__ __forceinline__ bool fetch_cell(const SimParams &p, uint32_t x, uint32_t y, CellRecord &rec) {
    const uint64_t cell = (uint64_t)y * p.width + (uint64_t)x;
    if (cell >= p.n_cells) return false;
    rec = p.cells[cell];
    return true;
}

__device__ __forceinline__ bool load_cell(const SimParams &p, uint32_t x, uint32_t y, CellRecord &rec,
                                          uint32_t *status) {
    if (fetch_cell(p, x, y, rec)) return true;
    set_status(status, kErrCellIndex);
    return false;
}

// packed_separable_alias/dispersal.rs:16-77 and alias/packed.rs:135-163, fed
// with the event's samples 2..4: the self-dispersal test (when taken) uses
// the first, the alias draw the next; `d_coal` receives the sample after them.
// A failed bound check returns false with its status bit in `err` (nothing
// is read out of range).
template <bool EAGER>
__device__ __forceinline__ bool spatially_explicit_dispersal_draw(
    uint64_t e2, uint64_t e3, uint64_t e4, uint64_t rs, const SimParams &p, uint32_t x, uint32_t y,
    const CellRecord &rec, uint32_t &tx, uint32_t &ty, uint64_t &d_coal, uint32_t &err) {
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
        d_coal = use_alias ? (EAGER ? e4 : draw_at(rs, 4)) : e3;
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
            err |= kErrAtomIndex;
            return false;
        }
        const AliasAtom atom = p.atoms[at];
        target = (frac < atom.u) ? atom.e : atom.k;
    }
    // cell indices are < 2^32 (one CellRecord per cell): 32-bit quotient
    const uint32_t t32 = (uint32_t)target, w32 = p.width;
    const uint32_t q = div_by_magic(t32, p.width_magic);
    tx = t32 - q * w32;
    ty = q;
    return true;
}

}  // namespace

// Where an event left the lineage.
enum StepResult : int { kStepStop = 0, kStepMoved = 1, kStepSpeciated = 2, kStepDropped = 3 };

// Outputs of lineage_step besides the lineage itself.
struct EventSink {
    DevSpeciationEvent *spec;
    unsigned long long *n_spec_total;
    uint64_t spec_cap;
    DevDispersalEvent *disp;
    unsigned long long *n_disp_total;
    uint64_t disp_cap;
    int report_dispersal;
    uint32_t *status;
    SimCounters *counters;
    TraceSink trace;
};

__device__ __forceinline__ void record_death(const TraceSink &t, uint64_t gref, uint64_t steps, uint32_t sim) {
    if (!t.deaths) return;
    const unsigned long long i = atomicAdd(t.n_deaths, 1ULL);
    if (i < t.cap) {
        TraceDeath d;
        d.gref = gref;
        d.steps = steps;
        d.sim = sim;
        d.pad = 0;
        t.deaths[i] = d;
    }
}

// The location injection of (x, y, i) (habitat/*: map_indexed_location_to_u64_injective);
// `rec` is the record of (x, y) for SpatiallyExplicit.
template <int KIND>
__device__ __forceinline__ uint64_t injection_at(const SimParams &p, uint32_t x, uint32_t y, uint32_t i,
                                                 const CellRecord &rec) {
    if (KIND == kNonSpatial) return non_spatial_injection(0, 0, p.width, p.deme, x, y, i);
    if (KIND == kSpatiallyImplicit) {
        // habitat/spatially_implicit.rs:106-120
        if (in_local(p, x, y)) return non_spatial_injection(0, 0, p.width, p.deme, x, y, i);
        return non_spatial_injection(p.meta_ox, p.meta_oy, p.meta_width, p.meta_deme, x, y, i);
    }
    if (KIND == kAlmostInfiniteNormal || KIND == kWrappingNoise) return ((uint64_t)y << 32) | (uint64_t)x;
    return rec.injection + (uint64_t)i;
}

template <int KIND>
__device__ __forceinline__ uint64_t lane_injection(const Lane &l, const SimParams &p) {
    return injection_at<KIND>(p, l.x, l.y, l.i, l.rec);
}

// Writes the speciation event of the lineage (event time l.next) and hands
// its step count to the simulation's counters.
__device__ __forceinline__ void emit_speciation(const Lane &l, const EventSink &k) {
    const unsigned long long e = atomicAdd(k.n_spec_total, 1ULL);
    if (e < k.spec_cap) {
        DevSpeciationEvent ev;
        ev.gref = l.gref;
        ev.prior_time = l.last;
        ev.event_time = l.next;
        ev.x = l.x;
        ev.y = l.y;
        ev.idx = l.i;
        ev.sim = l.s;
        k.spec[e] = ev;
    } else {
        set_status(k.status, kErrEventOverflow);
    }
    SimCounters &c = k.counters[l.s];
    atomicAdd(&c.steps, (unsigned long long)l.steps);
    atomicMax(&c.max_time_bits, f64_bits(l.next));
    atomicAdd(&c.n_speciation, 1ULL);
    record_death(k.trace, l.gref, l.steps, l.s);
}

// Writes the dispersal event of the lineage (event time l.next) to (tx, ty, ti).
__device__ __forceinline__ void emit_dispersal(const Lane &l, const EventSink &k, uint32_t tx, uint32_t ty,
                                               uint32_t ti) {
    const unsigned long long e = atomicAdd(k.n_disp_total, 1ULL);
    if (e < k.disp_cap) {
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
        k.disp[e] = ev;
    } else {
        set_status(k.status, kErrDispersalOverflow);
    }
}

// Dispersal target and coalescence index of an event that is not a
// speciation (event_sampler/independent.rs:160-204), from the re-primed
// state rs and its samples 2..4 (samples DRAWN + 1.. are drawn here only
// when the branch consumes them).  No side effects: `rec` receives the
// target's record (SpatiallyExplicit); a failed bound check or a
// WrappingNoise rejection limit returns false with its status bit in `err`.
template <int KIND, int DRAWN>
__device__ __forceinline__ bool event_target(const Lane &l, const SimParams &p, uint64_t rs, uint64_t e2,
                                             uint64_t e3, uint64_t e4, uint32_t &tx, uint32_t &ty, uint32_t &ti,
                                             CellRecord &rec, uint32_t &err) {
    constexpr bool EAGER = DRAWN >= 4;
    if (KIND == kNonSpatial) {
        non_spatial_dispersal_draw(e2, 0, 0, p.width, p.height, p.width_magic, tx, ty);
        ti = coalescence_index(e3, p.deme);
    } else if (KIND == kSpatiallyImplicit) {
        // dispersal_sampler/spatially_implicit.rs:58-86
        const bool local = in_local(p, l.x, l.y);
        const bool to_meta = !local || (e2 >> 11) < p.migration_threshold;
        const uint64_t d_index = local ? e3 : e2;
        const uint64_t d_coal = local ? (EAGER ? e4 : draw_at(rs, 4)) : e3;
        // one draw from the chosen community's extent (selects, not branches)
        const uint32_t ox = to_meta ? p.meta_ox : 0u, oy = to_meta ? p.meta_oy : 0u;
        const uint64_t w = to_meta ? p.meta_width : p.width, h = to_meta ? p.meta_height : p.height;
        const uint64_t magic = to_meta ? p.meta_width_magic : p.width_magic;
        non_spatial_dispersal_draw(d_index, ox, oy, w, h, magic, tx, ty);
        // habitat/spatially_implicit.rs:95-103: local extent first
        ti = coalescence_index(d_coal, in_local(p, tx, ty) ? p.deme : p.meta_deme);
    } else if (KIND == kAlmostInfiniteNormal) {
        // sample e4 is CoalescenceRngSample::new's draw; singleton demes -> index 0
        if (p.clark)
            clark2dt_dispersal_draw(e2, e3, p.clark_shape_u, p.clark_exponent, l.x, l.y, tx, ty);
        else
            normal_dispersal_draw(e2, e3, p.sigma, l.x, l.y, tx, ty);
        ti = 0;
    } else if (KIND == kWrappingNoise) {
        // dispersal_sampler/wrapping_noise.rs:42-87: self-dispersal iff
        // sample 2 is below p_self; otherwise Normal targets from samples
        // (3 + 2c, 4 + 2c) until one is habitable and not the origin.  The
        // coalescence sample then reads habitat 1 at the target: index 0.
        tx = l.x;
        ty = l.y;
        if ((e2 >> 11) >= p.noise.self_threshold) {
            uint64_t d0 = e3, d1 = EAGER ? e4 : draw_at(rs, 4);
            for (uint32_t c = 0;; ++c) {
                normal_dispersal_draw(d0, d1, p.sigma, l.x, l.y, tx, ty);
                if ((tx != l.x || ty != l.y) && noise::habitat_at(p.noise, tx, ty) != 0) break;
                if (c + 1 == kMaxDispersalRejections) {
                    err |= kErrDispersalRejections;
                    return false;
                }
                d0 = draw_at(rs, 5 + 2 * (uint64_t)c);
                d1 = draw_at(rs, 6 + 2 * (uint64_t)c);
            }
        }
        ti = 0;
    } else {
        uint64_t d_coal;
        if (!spatially_explicit_dispersal_draw<EAGER>(e2, e3, e4, rs, p, l.x, l.y, l.rec, tx, ty, d_coal, err))
            return false;
        if (!fetch_cell(p, tx, ty, rec)) {
            err |= kErrCellIndex;
            return false;
        }
        ti = coalescence_index(d_coal, rec.habitat);
    }
    return true;
}

// The event at l.next (event_sampler/independent.rs:112-222) from the
// re-primed state rs: speciation, or dispersal + coalescence index.  The
// event's first DRAWN samples arrive drawn (e1..e4); later ones are drawn
// here only when the branch consumes them.  Only a lane with `emit` writes
// events and counters (all lanes of a cooperative warp hold the same
// lineage).
template <int KIND, int DRAWN>
__device__ __forceinline__ int lineage_event(Lane &l, const SimParams &p, const EventSink &k, uint64_t rs,
                                             uint64_t e1, uint64_t e2, uint64_t e3, uint64_t e4, bool emit) {
    l.steps += 1;
    // speciation iff U[0,1) < nu  <=>  (e1 >> 11) < ceil(nu * 2^53)
    if ((e1 >> 11) < speciation_threshold<KIND>(p, l.x, l.y)) {
        if (emit) emit_speciation(l, k);
        return kStepSpeciated;
    }
    if (DRAWN < 2) e2 = draw_at(rs, 2);
    if (DRAWN < 3) e3 = draw_at(rs, 3);
    uint32_t tx, ty, ti, err = 0;
    CellRecord rec;
    if (!event_target<KIND, DRAWN>(l, p, rs, e2, e3, e4, tx, ty, ti, rec, err)) {
        set_status(k.status, err);
        return kStepDropped;
    }
    if (emit && k.report_dispersal) emit_dispersal(l, k, tx, ty, ti);
    if (KIND == kSpatiallyExplicit) l.rec = rec;
    l.x = tx;
    l.y = ty;
    l.i = ti;
    l.last = l.next;
    l.has_next = false;
    return kStepMoved;
}

// One step of a lineage: peek its next event time (or use the peek kept from
// the previous round) and stop if it is at or beyond the horizon; otherwise
// execute the event.  LAT selects the latency form (two buckets primed at a
// time, all samples drawn ahead) for lanes whose warp has little else to run;
// the throughput form draws only what the reference consumes.  EXP selects
// the exponential event-time sampler (exp.rs) instead of the Poisson one.
template <int KIND, bool LAT, bool EXP = false>
__device__ __forceinline__ int lineage_step(Lane &l, const SimParams &p, const EventSink &k) {
    const uint64_t loc_term = location_term(p.seed, lane_injection<KIND>(l, p));
    uint64_t rs;  // WyHash state re-primed for the event
    if (!l.has_next) {
        const PoissonConsts &pc = poisson_consts<KIND>(l, p);
        // IndependentActiveLineageSampler::pop_active_lineage_and_event_time
        // (active_lineage_sampler/independent/sampler.rs:69-116)
        const double before = l.last > p.min_event_time ? l.last : p.min_event_time;
        double t;
        if (EXP) {
            t = exp_next_event_time(loc_term, before, p, pc, l.reprime);
            rs = primed_state(loc_term, l.reprime);
        } else {
            t = LAT ? poisson_next_event_time_lat(loc_term, before, p, pc, l.reprime, rs)
                    : poisson_next_event_time_ilp(loc_term, before, p, pc, l.reprime, rs);
        }
        l.next = max_after(before, t);
        l.has_next = true;
    } else {
        rs = primed_state(loc_term, l.reprime);
    }
    // the reference's early stop `next_event_time >= level_time`
    // (monolithic/mod.rs:228-239); non-negative doubles order like their bits
    if (__double_as_longlong(l.next) >= __double_as_longlong(l.horizon)) return kStepStop;
    const uint64_t e1 = draw_at(rs, 1);
    if (LAT) {
        return lineage_event<KIND, 4>(l, p, k, rs, e1, draw_at(rs, 2), draw_at(rs, 3), draw_at(rs, 4), true);
    }
    return lineage_event<KIND, 1>(l, p, k, rs, e1, 0, 0, 0, true);
}

// Copies lane 0's lineage registers to every lane of the warp.
__device__ __forceinline__ void broadcast_from_lane0(Lane &l) {
    l.slot = __shfl_sync(kFull, l.slot, 0);
    l.x = __shfl_sync(kFull, l.x, 0);
    l.y = __shfl_sync(kFull, l.y, 0);
    l.i = __shfl_sync(kFull, l.i, 0);
    l.s = __shfl_sync(kFull, l.s, 0);
    l.last = __shfl_sync(kFull, l.last, 0);
    l.next = __shfl_sync(kFull, l.next, 0);
    l.horizon = __shfl_sync(kFull, l.horizon, 0);
    l.reprime = __shfl_sync(kFull, l.reprime, 0);
    l.gref = __shfl_sync(kFull, l.gref, 0);
    l.steps = __shfl_sync(kFull, l.steps, 0);
    l.has_next = __shfl_sync(kFull, l.has_next ? 1 : 0, 0) != 0;
    l.rec.injection = __shfl_sync(kFull, l.rec.injection, 0);
    l.rec.self_dispersal = __shfl_sync(kFull, l.rec.self_dispersal, 0);
    l.rec.atom_start = __shfl_sync(kFull, l.rec.atom_start, 0);
    l.rec.atom_count = __shfl_sync(kFull, l.rec.atom_count, 0);
    l.rec.habitat = __shfl_sync(kFull, l.rec.habitat, 0);
    l.rec.non_self_event = __shfl_sync(kFull, l.rec.non_self_event, 0);
}

constexpr long long kNoEvent = 0x7fffffffffffffffLL;

// The exponential sampler's search (exp.rs:37-83) for a lineage held by all
// 32 lanes of a warp: lanes 8g..8g+7 evaluate samples 1..8 of bucket
// base + g (one logarithm per lane, the costly part, all at once), then
// every lane replays its bucket's running sum in sample order (the
// reference's rounding order) from the shuffled samples.  The first bucket
// that is not empty decides; one whose eight samples pass neither `time`
// nor its end (rare for lambda * delta_t of order one) continues
// sequentially from its ninth sample.  Every lane returns the same result.
// Alongside its logarithm each lane primes the event state its sample would
// select (re-prime index ts + (j + 1) * INV_PHI) and draws the event's four
// samples, so a decided bucket hands the event its samples at once
// (drawn = true); the sequential continuation leaves them undrawn.
__device__ __forceinline__ double exp_search_coop(uint64_t loc_term, double time, const SimParams &p,
                                                  const PoissonConsts &pc, uint64_t &reprime, uint64_t &rs, uint64_t &e1, uint64_t &e2,
                                                  uint64_t &e3, uint64_t &e4, bool &drawn) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned first = lane & ~7u;  // the bucket's first lane
    uint64_t base = time_bucket(p, time);
    for (;;) {
        const uint64_t ts = base + (lane >> 3);
        const uint64_t mine = (uint64_t)(lane & 7u) + 1u;  // this lane's sample of the bucket
        const double e = exp_sample(draw_at(primed_state(loc_term, ts), (uint32_t)mine), pc.lambda);
        const uint64_t sc = primed_state(loc_term, ts + kInvPhi * mine);
        const uint64_t c1 = draw_at(sc, 1), c2 = draw_at(sc, 2), c3 = draw_at(sc, 3), c4 = draw_at(sc, 4);
        const double slice_end = __dmul_rn(__ull2double_rn(ts + 1), p.delta_t);
        double et = __dmul_rn(__ull2double_rn(ts), p.delta_t);
        int state = 0;  // 0: undecided, 1: event after `time` at sample j, 2: empty
        uint32_t j = 0;
#pragma unroll
        for (unsigned q = 0; q < 8u; ++q) {
            const double eq = __shfl_sync(kFull, e, (int)(first + q));
            if (state == 0) {
                et = __dadd_rn(et, eq);
                if (et >= slice_end) {
                    state = 2;
                } else if (et > time) {
                    state = 1;
                    j = q + 1u;
                }
            }
        }
        const unsigned open = __ballot_sync(kFull, (lane & 7u) == 0u && state != 2);
        if (open) {
            const int leader = __ffs(open) - 1;
            const int st = __shfl_sync(kFull, state, leader);
            const double et_l = __shfl_sync(kFull, et, leader);
            const uint32_t j_l = __shfl_sync(kFull, j, leader);
            const uint64_t ts_l = base + ((unsigned)leader >> 3);
            if (st == 1) {
                const int src = leader + (int)j_l - 1;  // the lane of sample j_l
                rs = __shfl_sync(kFull, sc, src);
                e1 = __shfl_sync(kFull, c1, src);
                e2 = __shfl_sync(kFull, c2, src);
                e3 = __shfl_sync(kFull, c3, src);
                e4 = __shfl_sync(kFull, c4, src);
                drawn = true;
                reprime = ts_l + kInvPhi * (uint64_t)j_l;
                return et_l;
            }
            drawn = false;
            return exp_continue(loc_term, time, p, pc, ts_l, 8u, et_l, reprime);
        }
        base += 4;
    }
}

// lineage_step for one lineage held (identically) by all 32 lanes of a warp.
// Every lane computes exactly one prime and one draw per pass, so the
// event's hash work costs the instruction stream of a single prime + draw:
//   lanes  0..15: bucket b = lane / 4 of four consecutive buckets; role
//                 r = lane % 4 draws sample r + 1 of the bucket (r = 0: the
//                 Devroye sample, r = 1..3: the times of events 0..2);
//   lanes 16..31: candidate c = (lane - 16) / 4 = (bucket c / 2, event c % 2)
//                 re-primed as if it came next, drawing the event's sample
//                 lane % 4 + 1.
// The first bucket with an event after `before` (the bucket and event the
// sequential loop of poisson.rs:48-100 stops at) selects the candidate whose
// four lanes hold the event's samples; other events re-prime after the
// selection.  Side effects happen on lane 0 only; every lane returns with
// the same updated lineage.  EXP selects the exponential event-time
// sampler, searched by exp_search_coop.
template <int KIND, bool EXP = false>
__device__ __forceinline__ int lineage_step_coop(Lane &l, const SimParams &p, const EventSink &k) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t loc_term = location_term(p.seed, lane_injection<KIND>(l, p));
    const PoissonConsts &pc = poisson_consts<KIND>(l, p);
    uint64_t rs, e1, e2, e3, e4;
    bool drawn = false;
    if (EXP && !l.has_next) {
        const double before = l.last > p.min_event_time ? l.last : p.min_event_time;
        l.next = max_after(before,
                           exp_search_coop(loc_term, before, p, pc, l.reprime, rs, e1, e2, e3, e4, drawn));
        l.has_next = true;
    }
    if (!l.has_next) {
        const double before = l.last > p.min_event_time ? l.last : p.min_event_time;
        const long long before_bits = __double_as_longlong(before);
        const double q = p.inv_delta_t != 0.0 ? __dmul_rn(before, p.inv_delta_t) : __ddiv_rn(before, p.delta_t);
        const bool bucket_lane = lane < 16u;
        const uint32_t role = lane & 3u;
        const uint32_t grp = (lane >> 2) & 3u;  // bucket (lanes 0..15) or candidate (16..31)
        uint64_t base = f64_to_u64(floor(q));
        long long best_bits = 0;
        uint32_t best_k = 0;
        uint64_t best_ts = 0;
        for (;;) {
            const uint64_t ts = base + (bucket_lane ? grp : (grp >> 1));
            const uint64_t tindex = bucket_lane ? ts : ts + kInvPhi * (uint64_t)((grp & 1u) + 1u);
            const uint64_t s = primed_state(loc_term, tindex);
            const uint64_t d = draw_at(s, role + 1u);
            // bucket lanes: the Devroye count from role 0, shared in the bucket
            const uint32_t n_own = poisson_count(d, pc);
            const uint32_t n_ev = __shfl_sync(kFull, n_own, (int)(lane & ~3u));
            long long mine = kNoEvent;
            uint32_t mine_k = 0xffffffffu;
            if (bucket_lane) {
                const double step_start = __ull2double_rn(ts);
                if (role >= 1u && role - 1u < n_ev) {
                    const long long eb = event_time_bits(step_start, d, p.delta_t);
                    if (eb > before_bits) {
                        mine = eb;
                        mine_k = role - 1u;
                    }
                } else if (role == 0u) {
                    // events 3.. of a bucket with more than three (rare)
                    for (uint32_t kk = 3; kk < n_ev; ++kk) {
                        const long long eb = event_time_bits(step_start, draw_at(s, kk + 2u), p.delta_t);
                        if (eb > before_bits && eb < mine) {  // kk ascending: ties keep the lower index
                            mine = eb;
                            mine_k = kk;
                        }
                    }
                }
            }
            // minimum over the bucket's 4 lanes (ties: lowest event index)
#pragma unroll
            for (int off = 1; off < 4; off <<= 1) {
                const long long ob = __shfl_xor_sync(kFull, mine, off);
                const uint32_t ok = __shfl_xor_sync(kFull, mine_k, off);
                if (ob < mine || (ob == mine && ok < mine_k)) {
                    mine = ob;
                    mine_k = ok;
                }
            }
            // the first of the 4 buckets with an event
            const unsigned found = __ballot_sync(kFull, bucket_lane && role == 0u && mine != kNoEvent);
            if (found) {
                const int leader = __ffs(found) - 1;
                const uint32_t bsel = (uint32_t)leader >> 2;
                best_bits = __shfl_sync(kFull, mine, leader);
                best_k = __shfl_sync(kFull, mine_k, leader);
                best_ts = base + bsel;
                // the candidate lanes of (bsel, best_k), when speculated
                // (bsel and best_k are the same on every lane)
                if (bsel < 2u && best_k < 2u) {
                    const int src = 16 + 4 * (int)(bsel * 2u + best_k);
                    rs = __shfl_sync(kFull, s, src);
                    e1 = __shfl_sync(kFull, d, src);
                    e2 = __shfl_sync(kFull, d, src + 1);
                    e3 = __shfl_sync(kFull, d, src + 2);
                    e4 = __shfl_sync(kFull, d, src + 3);
                    drawn = true;
                }
                break;
            }
            base += 4;
        }
        l.reprime = best_ts + kInvPhi * (uint64_t)(best_k + 1);
        l.next = max_after(before, __longlong_as_double(best_bits));
        l.has_next = true;
    }
    if (!drawn) {
        // a peek kept from the previous round, or an event outside the
        // speculated candidates: re-prime, lanes 0..3 draw samples 1..4
        rs = primed_state(loc_term, l.reprime);
        const uint64_t dk = draw_at(rs, (lane & 3u) + 1u);
        e1 = __shfl_sync(kFull, dk, 0);
        e2 = __shfl_sync(kFull, dk, 1);
        e3 = __shfl_sync(kFull, dk, 2);
        e4 = __shfl_sync(kFull, dk, 3);
    }
    if (__double_as_longlong(l.next) >= __double_as_longlong(l.horizon)) return kStepStop;
    return lineage_event<KIND, 4>(l, p, k, rs, e1, e2, e3, e4, lane == 0);
}

// ---- the cooperative step, speculative form (Poisson sampler) ----
//
// One lineage held by all 32 lanes of a warp, stepped event after event.
// Every lane primes one WyHash state and draws its samples 1..4 per pass:
//   lanes 0..7  (bucket lanes): bucket base + b, b = lane, of the search of
//               poisson.rs:48-100: the Devroye count and the times of
//               events 0..2 (further events draw their samples here);
//   lanes 8..31 (candidate lanes): one (bucket b, event k) pair each,
//               re-primed as if that event came next (time index
//               base + b + INV_PHI (k + 1), poisson.rs:102-106), computing
//               the whole event from its samples: speciation, dispersal
//               target, coalescence index and the target's location term.
// The first bucket with an event after `before` selects (b, k); the
// candidate lane holding that pair hands its event to the warp, so the next
// event's primes start right after the selection.  The pairs are the 24
// likeliest selections for lambda * delta_t = 1 (the reference's defaults,
// 99.7% of events); any other selection is computed after it.  Every
// outcome is a pure function of the lineage and the samples, so the
// speculation changes no result.

constexpr unsigned kCoopBuckets = 8;
// SpatiallyExplicit candidates read an alias atom and the target's record:
// only the likeliest pairs speculate (the others are computed on selection)
constexpr unsigned kCoopSpecLoads = 8;

struct CoopPair {
    uint8_t b, k;
};
// decreasing probability of being the selected (bucket, event) pair
constexpr CoopPair kCoopPairList[32 - kCoopBuckets] = {
    {1, 0}, {0, 0}, {2, 0}, {0, 1}, {1, 1}, {3, 0}, {2, 1}, {0, 2}, {1, 2}, {4, 0}, {3, 1}, {2, 2},
    {5, 0}, {0, 3}, {4, 1}, {1, 3}, {3, 2}, {6, 0}, {5, 1}, {2, 3}, {4, 2}, {7, 0}, {0, 4}, {6, 1}};
// the list as bytes b | k << 4, eight per word, so a lane finds its pair in registers
constexpr uint64_t coop_pair_word(int first) {
    uint64_t w = 0;
    for (int j = 0; j < 8; ++j)
        w |= (uint64_t)(kCoopPairList[first + j].b | (kCoopPairList[first + j].k << 4)) << (8 * j);
    return w;
}
constexpr uint64_t kCoopPairWord0 = coop_pair_word(0), kCoopPairWord1 = coop_pair_word(8),
                   kCoopPairWord2 = coop_pair_word(16);

// An event computed from its samples: what happened and where the lineage went.
struct CoopOutcome {
    uint32_t code;      // kStepMoved, kStepSpeciated or kStepDropped, status bits << 8
    uint32_t tx, ty, ti;
    uint64_t loc_next;  // location term of the target (kStepMoved)
    CellRecord rec;     // record of the target cell (SpatiallyExplicit)
};

// The event of lineage l from the re-primed state rs and its samples 1..4
// (event_sampler/independent.rs:112-222), without side effects.  An inactive
// lane computes nothing (code kStepDropped with no status bits).
template <int KIND>
__device__ __forceinline__ void coop_outcome(const Lane &l, const SimParams &p, uint64_t seed, uint64_t rs,
                                             uint64_t e1, uint64_t e2, uint64_t e3, uint64_t e4, bool active,
                                             CoopOutcome &o) {
    o.code = kStepDropped;
    if (KIND == kNonSpatial || KIND == kSpatiallyImplicit || KIND == kAlmostInfiniteNormal) {
        // no loads and no rejection loop: every lane computes both outcomes
        // without branching, so the warp's instruction stream stays one
        // block that interleaves with the bucket view's
        const bool spec = (e1 >> 11) < speciation_threshold<KIND>(p, l.x, l.y);
        uint32_t err = 0;
        event_target<KIND, 4>(l, p, rs, e2, e3, e4, o.tx, o.ty, o.ti, o.rec, err);
        o.loc_next = location_term(seed, injection_at<KIND>(p, o.tx, o.ty, o.ti, o.rec));
        o.code = !active ? kStepDropped : (spec ? kStepSpeciated : kStepMoved);
        return;
    }
    if (!active) return;
    if ((e1 >> 11) < speciation_threshold<KIND>(p, l.x, l.y)) {
        o.code = kStepSpeciated;
        return;
    }
    uint32_t err = 0;
    if (!event_target<KIND, 4>(l, p, rs, e2, e3, e4, o.tx, o.ty, o.ti, o.rec, err)) {
        o.code = kStepDropped | (err << 8);
        return;
    }
    o.code = kStepMoved;
    o.loc_next = location_term(seed, injection_at<KIND>(p, o.tx, o.ty, o.ti, o.rec));
}

template <int KIND>
__device__ __forceinline__ void shfl_outcome(CoopOutcome &o, int src) {
    o.code = __shfl_sync(kFull, o.code, src);
    o.tx = __shfl_sync(kFull, o.tx, src);
    o.ty = __shfl_sync(kFull, o.ty, src);
    o.ti = __shfl_sync(kFull, o.ti, src);
    o.loc_next = __shfl_sync(kFull, o.loc_next, src);
    if (KIND == kSpatiallyExplicit) {
        o.rec.injection = __shfl_sync(kFull, o.rec.injection, src);
        o.rec.self_dispersal = __shfl_sync(kFull, o.rec.self_dispersal, src);
        o.rec.atom_start = __shfl_sync(kFull, o.rec.atom_start, src);
        o.rec.atom_count = __shfl_sync(kFull, o.rec.atom_count, src);
        o.rec.habitat = __shfl_sync(kFull, o.rec.habitat, src);
        o.rec.non_self_event = __shfl_sync(kFull, o.rec.non_self_event, src);
    }
}

// Steps lineage l (identical on every lane of the warp) until its next event
// is at or beyond l.horizon (kStepStop, the peek kept in l), it speciates
// (kStepSpeciated) or a bound check fails (kStepDropped).  `events` counts
// the executed events; side effects happen on lane 0 only.
// `stop`, when given, interrupts the run at a peek below the horizon once it
// reads zero (checked every 32 events): the lineage keeps that peek and
// continues in a later launch.  Only a simulation with a single lineage may
// be interrupted mid-round (its rounds merge nothing).
template <int KIND>
__device__ __forceinline__ int coop_run(Lane &l, const SimParams &p, const EventSink &k, uint64_t &events,
                                        const volatile unsigned *stop = nullptr) {
    const unsigned lane = threadIdx.x & 31u;
    const bool bucket_lane = lane < kCoopBuckets;
    uint32_t my_b = lane, my_k = 0xffu;
    if (!bucket_lane) {
        const unsigned j = lane - kCoopBuckets;
        const uint64_t w = j < 8u ? kCoopPairWord0 : (j < 16u ? kCoopPairWord1 : kCoopPairWord2);
        const uint32_t pr = (uint32_t)(w >> (8u * (j & 7u))) & 0xffu;
        my_b = pr & 15u;
        my_k = pr >> 4;
    }
    const uint64_t my_tadd = (uint64_t)my_b + (bucket_lane ? 0ULL : kInvPhi * (uint64_t)(my_k + 1u));
    const bool speculate =
        !bucket_lane && (KIND != kSpatiallyExplicit || lane < kCoopBuckets + kCoopSpecLoads);
    const uint64_t seed = p.seed;
    const double delta_t = p.delta_t;
    const long long horizon_bits = __double_as_longlong(l.horizon);
    uint64_t loc_term = location_term(seed, lane_injection<KIND>(l, p));
    const PoissonConsts *pc = &poisson_consts<KIND>(l, p);
    for (;;) {
        CoopOutcome o;
        bool have = false;
        if (l.has_next) {
            // a peek kept from the previous round
            if (__double_as_longlong(l.next) >= horizon_bits) return kStepStop;
        } else {
            // IndependentActiveLineageSampler::pop_active_lineage_and_event_time
            // (active_lineage_sampler/independent/sampler.rs:69-116)
            const double before = l.last > p.min_event_time ? l.last : p.min_event_time;
            const long long before_bits = __double_as_longlong(before);
            uint64_t base = time_bucket(p, before);
            uint32_t b_sel, k_sel;
            long long t_bits;
            for (;;) {
                const uint64_t s = primed_state(loc_term, base + my_tadd);
                const uint64_t d1 = draw_at(s, 1), d2 = draw_at(s, 2), d3 = draw_at(s, 3), d4 = draw_at(s, 4);
                // bucket view: the earliest event of bucket base + b after
                // `before` (ties: lowest index), poisson.rs:50-95
                const uint32_t n_ev = poisson_count(d1, *pc);
                const double step_start = __ull2double_rn(base + my_b);
                const long long t0 = event_time_bits(step_start, d2, delta_t);
                const long long t1 = event_time_bits(step_start, d3, delta_t);
                const long long t2 = event_time_bits(step_start, d4, delta_t);
                long long mine = kNoEvent;
                uint32_t mine_k = 0;
                if (n_ev > 0u && t0 > before_bits) {
                    mine = t0;
                    mine_k = 0;
                }
                if (n_ev > 1u && t1 > before_bits && t1 < mine) {
                    mine = t1;
                    mine_k = 1;
                }
                if (n_ev > 2u && t2 > before_bits && t2 < mine) {
                    mine = t2;
                    mine_k = 2;
                }
                // candidate view: the event this lane's pair would be
                coop_outcome<KIND>(l, p, seed, s, d1, d2, d3, d4, speculate, o);
                // rare: a bucket with more than three events
                if (bucket_lane && n_ev > 3u) {
                    for (uint32_t kk = 3; kk < n_ev; ++kk) {
                        const long long eb = event_time_bits(step_start, draw_at(s, kk + 2u), delta_t);
                        if (eb > before_bits && eb < mine) {
                            mine = eb;
                            mine_k = kk;
                        }
                    }
                }
                const unsigned found = __ballot_sync(kFull, bucket_lane && mine != kNoEvent);
                if (found) {
                    b_sel = (uint32_t)(__ffs(found) - 1);
                    k_sel = __shfl_sync(kFull, mine_k, (int)b_sel);
                    t_bits = __shfl_sync(kFull, mine, (int)b_sel);
                    break;
                }
                base += kCoopBuckets;  // eight empty buckets: the next eight
            }
            l.reprime = base + (uint64_t)b_sel + kInvPhi * (uint64_t)(k_sel + 1u);
            l.next = max_after(before, __longlong_as_double(t_bits));
            l.has_next = true;
            // the reference's early stop `next_event_time >= level_time`
            // (monolithic/mod.rs:228-239); non-negative doubles order like their bits
            if (__double_as_longlong(l.next) >= horizon_bits) return kStepStop;
            if (stop && (events & 31u) == 0u && __shfl_sync(kFull, lane == 0 ? *stop : 1u, 0) == 0u)
                return kStepStop;  // interrupted with the peek kept
            const unsigned hit = __ballot_sync(kFull, speculate && my_b == b_sel && my_k == k_sel);
            if (hit) {
                shfl_outcome<KIND>(o, __ffs(hit) - 1);
                have = true;
            }
        }
        if (!have) {
            // re-prime for the event; lanes 0..3 draw samples 1..4
            const uint64_t rs = primed_state(loc_term, l.reprime);
            const uint64_t dk = draw_at(rs, (lane & 3u) + 1u);
            const uint64_t e1 = __shfl_sync(kFull, dk, 0), e2 = __shfl_sync(kFull, dk, 1);
            const uint64_t e3 = __shfl_sync(kFull, dk, 2), e4 = __shfl_sync(kFull, dk, 3);
            coop_outcome<KIND>(l, p, seed, rs, e1, e2, e3, e4, true, o);
        }
        l.steps += 1;
        const uint32_t code = o.code & 0xffu;
        if (code == kStepSpeciated) {
            events += 1;
            if (lane == 0) emit_speciation(l, k);
            return kStepSpeciated;
        }
        if (code != kStepMoved) {
            if (lane == 0) set_status(k.status, o.code >> 8);
            return kStepDropped;
        }
        events += 1;
        if (lane == 0 && k.report_dispersal) emit_dispersal(l, k, o.tx, o.ty, o.ti);
        l.x = o.tx;
        l.y = o.ty;
        l.i = o.ti;
        l.last = l.next;
        l.has_next = false;
        if (KIND == kSpatiallyExplicit) {
            l.rec = o.rec;
            pc = &poisson_consts<KIND>(l, p);
        }
        loc_term = o.loc_next;
    }
}

__device__ __forceinline__ EventSink sink_of(const StepArgs &a) {
    EventSink k;
    k.spec = a.spec;
    k.n_spec_total = a.n_spec_total;
    k.spec_cap = a.spec_cap;
    k.disp = a.disp;
    k.n_disp_total = a.n_disp_total;
    k.disp_cap = a.disp_cap;
    k.report_dispersal = a.report_dispersal;
    k.status = a.status;
    k.counters = a.counters;
    k.trace = a.trace;
    return k;
}

// Loads queue position k's lineage into the lane (false: simulation idle or
// a failed bound check).
template <int KIND, bool SINGLE>
__device__ __forceinline__ bool take_lineage(const StepArgs &a, const SimParams *P, unsigned long long k,
                                             Lane &l, bool ordered = true) {
    const uint32_t slot = (ordered && a.order) ? a.order[k] : (uint32_t)k;
    const uint32_t s = a.in.sim[slot];
    const SimParams &p = P[SINGLE ? 0 : s];
    if (!p.active) return false;
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
    if (KIND == kSpatiallyExplicit) return load_cell(p, l.x, l.y, l.rec, a.status);
    return true;
}

// Keeps a lineage that reached the horizon (with its peeked next event).
__device__ __forceinline__ void store_stopped(const StepArgs &a, const Lane &l) {
    a.in.x[l.slot] = l.x;
    a.in.y[l.slot] = l.y;
    a.in.idx[l.slot] = l.i;
    a.in.last[l.slot] = l.last;
    a.in.next[l.slot] = l.next;
    a.in.reprime[l.slot] = l.reprime;
    a.in.steps[l.slot] = l.steps;
    a.in.has_next[l.slot] = 1;
}

// A lane's lineage in converged passes: the pass kind, the current Poisson
// bucket, the time the search starts after, and the location term.
struct Pass {
    bool searching;
    uint64_t ts, loc_term;
    double before;
};

// Result of one converged pass besides those of lineage_step.
constexpr int kPassSearch = 4;

// Prepares the passes of a lineage; false when its peeked next event is
// already at or beyond the horizon (nothing to do this round).
template <int KIND>
__device__ __forceinline__ bool pass_begin(Lane &l, const SimParams &p, Pass &ps) {
    ps.loc_term = location_term(p.seed, lane_injection<KIND>(l, p));
    if (l.has_next) {
        ps.searching = false;
        return __double_as_longlong(l.next) < __double_as_longlong(l.horizon);
    }
    // IndependentActiveLineageSampler::pop_active_lineage_and_event_time
    // (active_lineage_sampler/independent/sampler.rs:69-116)
    ps.searching = true;
    ps.before = l.last > p.min_event_time ? l.last : p.min_event_time;
    ps.ts = time_bucket(p, ps.before);
    return true;
}

// One converged pass: prime the WyHash state for the current bucket or the
// current event and draw samples 1..3 (the same instructions on every lane
// whatever the pass is), then the short branch of that pass.  Returns
// kPassSearch (the search goes on), kStepMoved (event executed, searching
// again), kStepStop (next event at or beyond the horizon, peek kept),
// kStepSpeciated or kStepDropped.
template <int KIND>
__device__ __forceinline__ int pass_run(Lane &l, const SimParams &p, const EventSink &k, Pass &ps) {
    const uint64_t st = primed_state(ps.loc_term, ps.searching ? ps.ts : l.reprime);
    const uint64_t d1 = draw_at(st, 1), d2 = draw_at(st, 2), d3 = draw_at(st, 3);
    if (ps.searching) {
        // poisson.rs:48-100: the first bucket with an event after `before`
        long long bits = 0;
        const int kk = poisson_bucket_drawn(st, d1, d2, d3, ps.ts, __double_as_longlong(ps.before), p,
                                            poisson_consts<KIND>(l, p), bits);
        if (kk < 0) {
            ps.ts += 1;
            return kPassSearch;
        }
        l.reprime = ps.ts + kInvPhi * (uint64_t)(kk + 1);
        l.next = max_after(ps.before, __longlong_as_double(bits));
        l.has_next = true;
        ps.searching = false;
        // the reference's early stop `next_event_time >= level_time`
        // (monolithic/mod.rs:228-239); non-negative doubles order like their bits
        if (__double_as_longlong(l.next) >= __double_as_longlong(l.horizon)) return kStepStop;
        return kPassSearch;
    }
    const int r = lineage_event<KIND, 3>(l, p, k, st, d1, d2, d3, 0, true);
    if (r == kStepMoved) {
        ps.searching = true;
        ps.loc_term = location_term(p.seed, lane_injection<KIND>(l, p));
        ps.before = l.last;  // the event time, already after min_event_time
        ps.ts = time_bucket(p, ps.before);
    }
    return r;
}

// One lane per lineage at a time; a lane whose lineage reaches the horizon
// (or speciates) takes the next lineage of the queue, so warps stay full
// while lineages of very different event counts drain.
//
// With many lineages per lane (throughput) every lane runs the same pass
// each iteration: prime the WyHash state for either its current Poisson
// bucket or its current event, draw samples 1..3, then take the short
// branch for what the pass was (bucket search or event).  Lanes at
// different points of their lineages thus execute the same instructions
// for the hash work instead of diverging through the bucket loop, the
// event and the refill.  With few lineages per lane (latency) each lane
// runs lineage_step's latency form.  EXP: the exponential event-time
// sampler, one event at a time per lane (no converged-pass form).
// Copies one simulation's parameters to shared memory (single-simulation
// launches); returns the parameters the kernel reads.
template <bool SINGLE>
__device__ __forceinline__ const SimParams *stage_params(const StepArgs &a, unsigned char *smem) {
    if (!SINGLE) return a.params;
    const uint4 *src = reinterpret_cast<const uint4 *>(a.params);
    uint4 *dst = reinterpret_cast<uint4 *>(smem);
    for (unsigned w = threadIdx.x; w < sizeof(SimParams) / 16; w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    return reinterpret_cast<const SimParams *>(smem);
}

// Per-simulation horizon rule (canonical schedule):
// H' = min(H + clamp(ceil(min_round_events / n), step_slice, step_slice_max) / lambda, pause),
// or no further round when n == 0 or H has reached pause_before.
__device__ __forceinline__ bool next_horizon(const SimParams &p, unsigned long long live, double &h) {
    const bool paused = p.pause_before >= 0.0 && !(p.horizon < p.pause_before);
    if (live == 0 || paused) return false;
    const unsigned long long step_slice = p.step_slice ? p.step_slice : 1ULL;
    unsigned long long per = (p.min_round_events + live - 1) / live;
    if (p.step_slice_max && per > p.step_slice_max) per = p.step_slice_max;
    if (per < step_slice) per = step_slice;
    h = __dadd_rn(p.horizon, __ddiv_rn(__ull2double_rn(per), p.lambda));
    if (p.pause_before >= 0.0 && p.pause_before < h) h = p.pause_before;
    return true;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The SM reservation (SmGate): true when the calling block's SM is one its
// engine must leave while the reservation is on.
__device__ __forceinline__ bool gate_leaves(const SmGate *g, uint32_t role) {
    if (*(volatile const uint32_t *)&g->on == 0u) return false;
    uint32_t smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    const bool reserved = smid < 256u && ((g->mask[smid >> 5] >> (smid & 31u)) & 1u) != 0u;
    return role == kGateAvoid ? reserved : !reserved;
}

// Block-uniform.  Every block of a gated launch arrives once at `done`: a
// block that leaves arrives at once, one that works arrives when its first
// warp has found the queue empty.  A leaving block that arrives last stays
// and takes whatever is left, so the launch's work is done wherever its
// blocks landed (when any working block arrives, every item is claimed).
__device__ __forceinline__ bool block_leaves(const SmGate *g, uint32_t role, unsigned int *done) {
    if (g == nullptr || role == kGateNone) return false;
    __shared__ int s_leave;
    if (threadIdx.x == 0) {
        int leave = gate_leaves(g, role) ? 1 : 0;
        if (leave) leave = (atomicAdd(done, 1u) + 1u < gridDim.x) ? 1 : 0;
        s_leave = leave;
    }
    __syncthreads();
    return s_leave != 0;
}

__device__ __forceinline__ void block_arrives(const SmGate *g, uint32_t role, unsigned int *done) {
    if (g != nullptr && role != kGateNone && threadIdx.x == 0) atomicAdd(done, 1u);
}

// At most one lineage per warp: each warp takes lineages from the queue and
// steps each one with all its lanes (a lineage's events at warp latency,
// lineages on all SMs).  Every lineage gets a warp at once, so the queue
// order is moot (and not computed for such rounds).
template <int KIND, bool SINGLE, bool EXP>
__device__ __forceinline__ void coop_body(const StepArgs &a, const SimParams *P, uint64_t n) {
    const EventSink sink = sink_of(a);
    const unsigned lane_id = threadIdx.x & 31u;
    uint64_t warp_steps = 0;
    for (;;) {
        unsigned long long k = 0;
        if (lane_id == 0) {
            k = atomicAdd(a.work, 1ULL);
            if (a.busy && k < n) atomicAdd(a.busy, 1u);
        }
        k = __shfl_sync(kFull, k, 0);
        if (k >= n) break;
        Lane c;
        if (!take_lineage<KIND, SINGLE>(a, P, k, c, false)) {
            if (a.busy && lane_id == 0) atomicSub(a.busy, 1u);
            continue;
        }
        const SimParams &p = P[SINGLE ? 0 : c.s];
        int r;
        if constexpr (EXP) {
            for (;;) {
                r = lineage_step_coop<KIND, true>(c, p, sink);
                if (r != kStepMoved) break;
                warp_steps += 1;
            }
            if (r == kStepSpeciated) warp_steps += 1;
        } else {
            if constexpr (KIND == kSpatiallyExplicit) {
                // the speculative candidates' alias and record reads cost more
                // than they save here: select first, then read (measured)
                for (;;) {
                    r = lineage_step_coop<KIND, false>(c, p, sink);
                    if (r != kStepMoved) break;
                    warp_steps += 1;
                }
                if (r == kStepSpeciated) warp_steps += 1;
            } else {
                r = coop_run<KIND>(c, p, sink, warp_steps);
            }
            // the lineage's own round is done: it no longer holds the launch
            if (a.busy && lane_id == 0) atomicSub(a.busy, 1u);
            // A simulation that started the round with one live lineage has
            // nothing to merge: while other lineages of the launch are still
            // in their own round (or the launch has this simulation alone),
            // its warp runs the simulation's next rounds itself, each to the
            // horizon the scheduler would set (next_horizon) and counted as a
            // round.  Free-running warps do not keep one another going.
            if (KIND != kSpatiallyExplicit && a.free_rounds && r == kStepStop && a.counters[c.s].n_live == 1) {
                SimParams &pg = const_cast<SimParams *>(a.params)[SINGLE ? 0 : c.s];
                for (uint32_t extra = 0; extra < a.free_rounds; ++extra) {
                    const bool others = SINGLE || *(volatile const unsigned *)a.busy > 0u;
                    if (!__shfl_sync(kFull, others ? 1 : 0, 0)) break;
                    double h;
                    if (!next_horizon(pg, 1, h)) break;  // paused
                    const double h_prev = pg.horizon;
                    __syncwarp();
                    if (lane_id == 0) {
                        pg.horizon = h;
                        a.counters[c.s].n_rounds += 1;
                    }
                    __syncwarp();
                    c.horizon = h;
                    // interrupted at a peek once the launch's regular work is done
                    r = coop_run<KIND>(c, p, sink, warp_steps, SINGLE ? nullptr : a.busy);
                    if (r == kStepStop && __double_as_longlong(c.next) < __double_as_longlong(h)) {
                        // the round is not finished: give it back, so the
                        // scheduler sets (and counts) the same horizon again
                        __syncwarp();
                        if (lane_id == 0) {
                            pg.horizon = h_prev;
                            a.counters[c.s].n_rounds -= 1;
                        }
                        __syncwarp();
                        break;
                    }
                    if (r != kStepStop) break;
                }
            }
        }
        if (EXP && a.busy && lane_id == 0) atomicSub(a.busy, 1u);
        if (lane_id == 0) {
            if (r == kStepStop)
                store_stopped(a, c);
            else
                a.state[c.slot] = (r == kStepSpeciated) ? 1 : 2;
        }
    }
    if (a.steps_total && lane_id == 0 && warp_steps) atomicAdd(a.steps_total, (unsigned long long)warp_steps);
}

template <int KIND, bool SINGLE, bool EXP>
__device__ __forceinline__ void step_body(const StepArgs &a) {
    // one simulation: its parameters live in shared memory for the launch
    __shared__ __align__(16) unsigned char params_smem[SINGLE ? sizeof(SimParams) : 16];
    const uint64_t n = *a.n_cur;
    // the Poisson sampler's cooperative rounds run in coop_kernel
    if (!EXP && n <= a.coop_max) return;
    if (block_leaves(a.gate, a.gate_role, a.blocks_done)) return;
    const SimParams *P = stage_params<SINGLE>(a, params_smem);
    const EventSink sink = sink_of(a);
    const unsigned lane_id = threadIdx.x & 31u;
    if (EXP && n <= (uint64_t)gridDim.x * (blockDim.x / 32u)) {
        coop_body<KIND, SINGLE, true>(a, P, n);
        block_arrives(a.gate, a.gate_role, a.blocks_done);
        return;
    }
    const bool lat = n * 4 <= (uint64_t)gridDim.x * blockDim.x;
    const unsigned lanemask_lt = (1u << lane_id) - 1u;
    bool have = false;
    bool exhausted = (n == 0);
    Lane l;
    uint64_t local_steps = 0;
    Pass ps;  // converged form

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
                    have = take_lineage<KIND, SINGLE>(a, P, k, l);
                    if (have && !EXP && !lat && !pass_begin<KIND>(l, P[SINGLE ? 0 : l.s], ps)) {
                        store_stopped(a, l);  // nothing to do before this horizon
                        have = false;
                    }
                } else {
                    exhausted = true;
                }
            }
        }
        // a warp leaves only when the queue is empty for all its lanes (a
        // lineage of an inactive simulation, or one with nothing to do before
        // the horizon, leaves its lane free to take the next)
        if (!__any_sync(kFull, have || !exhausted)) break;
        if (!have) continue;
        const SimParams &p = P[SINGLE ? 0 : l.s];

        // few lineages for the grid's lanes: latency form (uniform branch);
        // the exponential sampler steps lineages one event at a time
        const int r = EXP ? (lat ? lineage_step<KIND, true, true>(l, p, sink)
                                 : lineage_step<KIND, false, true>(l, p, sink))
                          : (lat ? lineage_step<KIND, true>(l, p, sink) : pass_run<KIND>(l, p, sink, ps));
        if (r == kPassSearch) continue;
        if (r == kStepMoved) {
            local_steps += 1;
            continue;
        }
        if (r == kStepStop) {
            store_stopped(a, l);  // keep the peeked time for the next round
        } else {
            if (r == kStepSpeciated) local_steps += 1;
            a.state[l.slot] = (r == kStepSpeciated) ? 1 : 2;  // 2: dropped by a failed bound check
        }
        have = false;
    }
    if (a.steps_total) {
        // one atomic per warp for the launch's event count
        unsigned long long w = local_steps;
        for (int off = 16; off > 0; off >>= 1) w += __shfl_down_sync(kFull, w, off);
        if (lane_id == 0 && w) atomicAdd(a.steps_total, w);
    }
    block_arrives(a.gate, a.gate_role, a.blocks_done);
}

// The step kernel with the Poisson sampler, and with the exponential one:
// the latter's logarithm needs more registers than the allocation ptxas
// picks by default (which spills), so it asks for one block per SM at least
// instead; the Poisson kernel keeps its allocation.
template <int KIND, bool SINGLE>
__global__ void __launch_bounds__(kStepBlockMax) step_kernel(StepArgs a) {
    step_body<KIND, SINGLE, false>(a);
}
template <int KIND, bool SINGLE>
__global__ void __launch_bounds__(kStepBlockMax, 1) step_kernel_exp(StepArgs a) {
    step_body<KIND, SINGLE, true>(a);
}

// The Poisson sampler's rounds with at most coop_max live lineages, one warp
// per lineage (coop_run); the step kernel takes the other rounds.  Its own
// kernel, so that the speculative form's registers do not lower the step
// kernel's occupancy.
template <int KIND, bool SINGLE>
__global__ void __launch_bounds__(kCoopBlock) coop_kernel(StepArgs a) {
    __shared__ __align__(16) unsigned char params_smem[SINGLE ? sizeof(SimParams) : 16];
    const uint64_t n = *a.n_cur;
    if (n > a.coop_max) return;
    if (block_leaves(a.gate, a.gate_role, a.blocks_done)) return;
    const SimParams *P = stage_params<SINGLE>(a, params_smem);
    coop_body<KIND, SINGLE, false>(a, P, n);
    block_arrives(a.gate, a.gate_role, a.blocks_done);
}

// A simulation with at most kResidentMax live lineages is advanced by one
// thread block on its own: the block runs the simulation's rounds (the same
// horizons and the same smallest-global-reference dedup as the global
// kernels) with its lineages in registers and the dedup in shared memory,
// so small simulations progress at their own pace instead of waiting for
// the whole batch at every round.  A launch runs at most `budget` rounds per
// simulation; lineages are kept in the simulation's segment of the resident
// arena between launches.
//
// Lineage slot j lives on warp j % 8, lane j / 8: a simulation with few
// lineages gets one lineage per warp, so lineages never share (and diverge
// within) a warp until there are more than eight of them.
template <int KIND, int THREADS, bool EXP>
__global__ void __launch_bounds__(THREADS, 1) resident_kernel(ResidentArgs a) {
    constexpr unsigned kWarps = THREADS / 32;
    constexpr unsigned kSlots = THREADS;  // lineage slots (>= kResidentMax)
    __shared__ uint32_t sx[kSlots], sy[kSlots], si[kSlots];
    __shared__ unsigned long long slast[kSlots], sgref[kSlots];
    __shared__ unsigned char salive[kSlots];
    __shared__ unsigned int sscan[kSlots];
    __shared__ unsigned int s_n;
    __shared__ int s_go;
    __shared__ double s_h;
    // staging of surviving lineages during the block's compaction
    __shared__ uint32_t tx_[kSlots], ty_[kSlots], ti_[kSlots];
    __shared__ double tlast[kSlots], tnext[kSlots];
    __shared__ unsigned long long trep[kSlots], tgref[kSlots], tsteps[kSlots];
    __shared__ unsigned char thas[kSlots];

    const unsigned t = threadIdx.x;
    const unsigned j = (t & 31u) * kWarps + (t >> 5);  // this thread's lineage slot
    EventSink sink;
    sink.spec = a.spec;
    sink.n_spec_total = a.n_spec_total;
    sink.spec_cap = a.spec_cap;
    sink.disp = nullptr;
    sink.n_disp_total = nullptr;
    sink.disp_cap = 0;
    sink.report_dispersal = 0;
    sink.status = a.status;
    sink.counters = a.counters;
    sink.trace.deaths = nullptr;
    sink.trace.n_deaths = nullptr;
    sink.trace.cap = 0;

    // with an SM gate the blocks claim simulations one at a time (a block
    // may leave its SM), else block b takes simulations b, b + grid, ...
    const bool claiming = a.gate != nullptr && a.gate_role != kGateNone;
    if (block_leaves(a.gate, a.gate_role, a.blocks_done)) return;
    __shared__ uint32_t s_claim;
    auto next_sim = [&](uint32_t prev) -> uint32_t {
        if (!claiming) return prev + gridDim.x;
        __syncthreads();  // every thread has read the previous claim
        if (t == 0) s_claim = atomicAdd(a.claim, 1u);
        __syncthreads();
        return s_claim;
    };
    for (uint32_t s = claiming ? next_sim(0) : blockIdx.x; s < a.n_sims; s = next_sim(s)) {
        SimParams &pm = a.params[s];
        if (t == 0) {
            // resident == 2: owned by this kernel (1: routed, handed over at
            // the next launch boundary)
            s_go = (pm.resident == 2 && pm.active) ? 1 : 0;
            s_n = (unsigned)a.counters[s].n_live;
            s_h = pm.horizon;
        }
        __syncthreads();
        if (!s_go) {
            __syncthreads();
            continue;
        }
        const SimParams &p = pm;
        const uint64_t seg = p.lineage_offset;
        unsigned n = s_n;
        if (n > (unsigned)kResidentMax) {  // never routed with more: guard the block's arrays
            if (t == 0) set_status(a.status, kErrResident);
            n = kResidentMax;
        }
        Lane l;
        bool alive = j < n;
        if (alive) {
            const uint64_t g = seg + j;
            l.slot = (uint32_t)g;
            l.s = s;
            l.x = a.arena.x[g];
            l.y = a.arena.y[g];
            l.i = a.arena.idx[g];
            l.last = a.arena.last[g];
            l.next = a.arena.next[g];
            l.reprime = a.arena.reprime[g];
            l.gref = a.arena.gref[g];
            l.steps = a.arena.steps[g];
            l.has_next = a.arena.has_next[g] != 0;
            if (KIND == kSpatiallyExplicit) alive = load_cell(p, l.x, l.y, l.rec, a.status);
        }
        for (uint32_t round = 0; round < a.budget; ++round) {
            // advance every lineage to the round's horizon
            l.horizon = s_h;
            unsigned long long my_events = 0;
            if (n <= kWarps) {
                // at most one lineage per warp (slot w on lane 0 of warp w):
                // the whole warp steps it cooperatively
                Lane c = l;
                broadcast_from_lane0(c);
                const bool c_alive = __shfl_sync(kFull, alive ? 1 : 0, 0) != 0;
                if (c_alive) {
                    bool c_live = true;
                    if constexpr (EXP) {
                        for (;;) {
                            const int r = lineage_step_coop<KIND, true>(c, p, sink);
                            if (r == kStepMoved) {
                                ++my_events;
                                continue;
                            }
                            if (r == kStepSpeciated) {
                                ++my_events;
                                c_live = false;
                            } else if (r == kStepDropped) {
                                c_live = false;
                            }
                            break;
                        }
                    } else {
                        uint64_t ev = 0;
                        c_live = coop_run<KIND>(c, p, sink, ev) == kStepStop;
                        my_events += ev;
                    }
                    if ((t & 31u) == 0) {
                        l = c;
                        alive = c_live;
                    } else {
                        my_events = 0;
                    }
                }
            } else if (alive) {
                // up to 8 lineages per warp: latency form
                const bool lat = n <= 8 * kWarps;
                for (;;) {
                    const int r = lat ? lineage_step<KIND, true, EXP>(l, p, sink)
                                      : lineage_step<KIND, false, EXP>(l, p, sink);
                    if (r == kStepMoved) {
                        ++my_events;
                        continue;
                    }
                    if (r == kStepSpeciated) {
                        ++my_events;
                        alive = false;
                    } else if (r == kStepDropped) {
                        alive = false;
                    }
                    break;
                }
            }
            if (a.steps_total && my_events) atomicAdd(a.steps_total, my_events);
            // dedup: a live lineage survives unless another live lineage in
            // the same state (location, index, last event time) has a smaller
            // global reference
            if (j < n) {
                sx[j] = l.x;
                sy[j] = l.y;
                si[j] = l.i;
                slast[j] = (unsigned long long)__double_as_longlong(l.last);
                sgref[j] = l.gref;
                salive[j] = alive ? 1 : 0;
            }
            __syncthreads();
            bool survivor = alive;
            if (alive) {
                const unsigned long long lb = (unsigned long long)__double_as_longlong(l.last);
                for (unsigned k2 = 0; k2 < n; ++k2) {
                    if (salive[k2] && sgref[k2] < l.gref && sx[k2] == l.x && sy[k2] == l.y &&
                        si[k2] == l.i && slast[k2] == lb) {
                        survivor = false;
                        break;
                    }
                }
                if (!survivor) {
                    SimCounters &c = a.counters[s];
                    atomicAdd(&c.steps, (unsigned long long)l.steps);
                    atomicMax(&c.max_time_bits, f64_bits(l.last));
                    atomicAdd(&c.n_dedup, 1ULL);
                }
            }
            // inclusive scan of the survivor flags in slot order
            sscan[j] = survivor ? 1u : 0u;
            __syncthreads();
            for (unsigned d = 1; d < kSlots; d <<= 1) {
                const unsigned add = (j >= d) ? sscan[j - d] : 0u;
                __syncthreads();
                sscan[j] += add;
                __syncthreads();
            }
            const unsigned total = sscan[kSlots - 1];
            if (survivor) {
                const unsigned d = sscan[j] - 1u;
                tx_[d] = l.x;
                ty_[d] = l.y;
                ti_[d] = l.i;
                tlast[d] = l.last;
                tnext[d] = l.next;
                trep[d] = l.reprime;
                tgref[d] = l.gref;
                tsteps[d] = l.steps;
                thas[d] = l.has_next ? 1 : 0;
            }
            __syncthreads();
            const unsigned n_prev = n;
            n = total;
            alive = j < n;
            if (alive) {
                l.x = tx_[j];
                l.y = ty_[j];
                l.i = ti_[j];
                l.last = tlast[j];
                l.next = tnext[j];
                l.reprime = trep[j];
                l.gref = tgref[j];
                l.steps = tsteps[j];
                l.has_next = thas[j] != 0;
                if (KIND == kSpatiallyExplicit) alive = load_cell(p, l.x, l.y, l.rec, a.status);
            }
            // the simulation's schedule, as the global scheduler would do it
            if (t == 0) {
                SimCounters &c = a.counters[s];
                atomicAdd(a.visits, (unsigned long long)n_prev);
                c.n_live = n;
                double h;
                if (next_horizon(pm, n, h)) {
                    pm.horizon = h;
                    c.n_rounds += 1;
                    s_h = h;
                    s_go = 1;
                    // the global rounds running beside this launch have
                    // finished: hand control back (the state is consistent)
                    if (a.stop_flag && *(volatile const int *)a.stop_flag) s_go = 2;
                } else {
                    pm.active = 0;
                    c.end_ns = global_ns();
                    atomicSub(a.n_resident, 1u);
                    s_go = 0;
                }
            }
            __syncthreads();
            if (s_go != 1) break;
        }
        // keep the survivors (and their peeked next events) in the arena
        if (j < n) {
            const uint64_t g = seg + j;
            a.arena.x[g] = l.x;
            a.arena.y[g] = l.y;
            a.arena.idx[g] = l.i;
            a.arena.last[g] = l.last;
            a.arena.next[g] = l.next;
            a.arena.reprime[g] = l.reprime;
            a.arena.gref[g] = l.gref;
            a.arena.steps[g] = l.steps;
            a.arena.has_next[g] = l.has_next ? 1 : 0;
        }
        __syncthreads();
    }
    block_arrives(a.gate, a.gate_role, a.blocks_done);
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
        // survivors of a simulation that started the round with at most
        // kResidentMax lineages move to its segment of the resident arena
        // (the resident kernel owns the simulation from the next round on)
        const bool to_arena = survivor && a.arena.x != nullptr &&
                              a.counters[s].n_live <= (unsigned long long)a.resident_max;
        const bool to_out = survivor && !to_arena;
        const unsigned sv = __ballot_sync(kFull, to_out);
        unsigned long long dst_base = 0;
        if (sv) {
            const int leader = __ffs(sv) - 1;
            if ((int)lane_id == leader) dst_base = atomicAdd(a.out_count, (unsigned long long)__popc(sv));
            dst_base = __shfl_sync(kFull, dst_base, leader);
        }
        if (to_out) {
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
            if (a.out.pred_end) a.out.pred_end[d] = a.in.pred_end[j];
            a.state_out[d] = 0;
        }
        // per-simulation live counts, aggregated over lanes of the same
        // simulation (the count doubles as the arena slot of a moved lineage)
        const unsigned same = __match_any_sync(kFull, to_out ? s : 0xffffffffu);
        if (to_out && (__ffs(same) - 1) == (int)lane_id)
            atomicAdd(&a.counters[s].n_live_next, (unsigned long long)__popc(same));
        if (to_arena) {
            SimCounters &c = a.counters[s];
            const uint64_t d = a.params[s].lineage_offset + atomicAdd(&c.n_live_next, 1ULL);
            c.routed = 1;
            a.arena.x[d] = a.in.x[j];
            a.arena.y[d] = a.in.y[j];
            a.arena.idx[d] = a.in.idx[j];
            a.arena.sim[d] = s;
            a.arena.last[d] = a.in.last[j];
            a.arena.next[d] = a.in.next[j];
            a.arena.reprime[d] = a.in.reprime[j];
            a.arena.gref[d] = a.in.gref[j];
            a.arena.steps[d] = a.in.steps[j];
            a.arena.has_next[d] = a.in.has_next[j];
        }
        if (dup) {
            SimCounters &c = a.counters[s];
            atomicAdd(&c.steps, (unsigned long long)a.in.steps[j]);
            atomicMax(&c.max_time_bits, f64_bits(a.in.last[j]));
            atomicAdd(&c.n_dedup, 1ULL);
            record_death(a.trace, a.in.gref[j], a.in.steps[j], s);
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
        if (p.resident) continue;  // the resident kernel schedules it
        const unsigned long long live = c.n_live_next;
        c.n_live = live;
        c.n_live_next = 0;
        double h;
        const bool more = next_horizon(p, live, h);
        const unsigned long long now = global_ns();
        if (c.start_ns == 0) c.start_ns = now;
        // the end: the round in which it stops (or, never started, now)
        if (!more && (p.active || c.end_ns == 0)) c.end_ns = now;
        if (more) {
            p.horizon = h;
            c.n_rounds += 1;
        }
        p.active = more ? 1 : 0;
        if (c.routed) {
            // its survivors are in the resident arena
            if (c.routed_ns == 0) c.routed_ns = now;
            p.resident = 1;
            if (more) atomicAdd(a.n_resident, 1u);
        } else if (more) {
            my_active += 1;
        }
    }
    atomicAdd(&active_sum, my_active);
    __syncthreads();
    if (threadIdx.x == 0) {
        *a.n_active = active_sum;
        if (active_sum > 0) atomicAdd(a.visits, *a.out_count);  // shared with the resident kernel
        const unsigned long long n = *a.out_count;
        *a.n_cur = n;
        *a.out_count = 0;
        *a.work = 0;
        if (a.blocks_done) *a.blocks_done = 0;
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
static cudaError_t launch_step_t(const StepArgs &a, unsigned grid, unsigned block, unsigned coop_grid,
                                 cudaStream_t st) {
    if (a.exp_sampler) {
        if (a.n_sims == 1)
            step_kernel_exp<KIND, true><<<grid, block, 0, st>>>(a);
        else
            step_kernel_exp<KIND, false><<<grid, block, 0, st>>>(a);
        return cudaGetLastError();
    }
    if (a.coop_max) {
        if (a.n_sims == 1)
            coop_kernel<KIND, true><<<coop_grid, kCoopBlock, 0, st>>>(a);
        else
            coop_kernel<KIND, false><<<coop_grid, kCoopBlock, 0, st>>>(a);
    }
    if (a.n_sims == 1)
        step_kernel<KIND, true><<<grid, block, 0, st>>>(a);
    else
        step_kernel<KIND, false><<<grid, block, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_step(int kind, const StepArgs &a, unsigned grid, unsigned block, unsigned coop_grid,
                        cudaStream_t st) {
    if (!a.exp_sampler && a.coop_max > (uint64_t)coop_grid * (kCoopBlock / 32)) return cudaErrorInvalidValue;
    switch (kind) {
    case kNonSpatial: return launch_step_t<kNonSpatial>(a, grid, block, coop_grid, st);
    case kSpatiallyImplicit: return launch_step_t<kSpatiallyImplicit>(a, grid, block, coop_grid, st);
    case kAlmostInfiniteNormal: return launch_step_t<kAlmostInfiniteNormal>(a, grid, block, coop_grid, st);
    case kSpatiallyExplicit: return launch_step_t<kSpatiallyExplicit>(a, grid, block, coop_grid, st);
    case kWrappingNoise: return launch_step_t<kWrappingNoise>(a, grid, block, coop_grid, st);
    default: return cudaErrorInvalidValue;
    }
}

template <int KIND>
static cudaError_t coop_occupancy_t(int *blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, coop_kernel<KIND, false>, kCoopBlock, 0);
}

cudaError_t coop_kernel_occupancy(int kind, int *blocks_per_sm) {
    switch (kind) {
    case kNonSpatial: return coop_occupancy_t<kNonSpatial>(blocks_per_sm);
    case kSpatiallyImplicit: return coop_occupancy_t<kSpatiallyImplicit>(blocks_per_sm);
    case kAlmostInfiniteNormal: return coop_occupancy_t<kAlmostInfiniteNormal>(blocks_per_sm);
    case kSpatiallyExplicit: return coop_occupancy_t<kSpatiallyExplicit>(blocks_per_sm);
    case kWrappingNoise: return coop_occupancy_t<kWrappingNoise>(blocks_per_sm);
    default: return cudaErrorInvalidValue;
    }
}

template <int KIND>
static cudaError_t step_occupancy_t(bool exp_sampler, int block, int *blocks_per_sm) {
    if (exp_sampler)
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, step_kernel_exp<KIND, false>, block, 0);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, step_kernel<KIND, false>, block, 0);
}

cudaError_t step_kernel_occupancy(int kind, bool exp_sampler, int block, int *blocks_per_sm) {
    switch (kind) {
    case kNonSpatial: return step_occupancy_t<kNonSpatial>(exp_sampler, block, blocks_per_sm);
    case kSpatiallyImplicit: return step_occupancy_t<kSpatiallyImplicit>(exp_sampler, block, blocks_per_sm);
    case kAlmostInfiniteNormal: return step_occupancy_t<kAlmostInfiniteNormal>(exp_sampler, block, blocks_per_sm);
    case kSpatiallyExplicit: return step_occupancy_t<kSpatiallyExplicit>(exp_sampler, block, blocks_per_sm);
    case kWrappingNoise: return step_occupancy_t<kWrappingNoise>(exp_sampler, block, blocks_per_sm);
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

__global__ void sm_census_kernel(uint32_t *mask) {
    if (threadIdx.x != 0) return;
    uint32_t smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    if (smid < 256u) atomicOr(&mask[smid >> 5], 1u << (smid & 31u));
}

cudaError_t launch_sm_census(uint32_t *mask, unsigned grid, cudaStream_t st) {
    sm_census_kernel<<<grid, 32, 0, st>>>(mask);
    return cudaGetLastError();
}

// Hands simulations routed to the resident arena (resident == 1) over to the
// resident kernel (resident == 2); runs while no kernel of either kind does.
__global__ void promote_kernel(SimParams *params, uint32_t n_sims) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n_sims; s += gridDim.x * blockDim.x)
        if (params[s].resident == 1) params[s].resident = 2;
}

// The integer-issue ceiling of the hash work: eight independent chains of
// wymum (64x64 -> 128-bit multiply, halves xor-folded) per thread on every
// SM; the step kernel's algorithmic wymum rate is measured against it.
__global__ void __launch_bounds__(256) hash_peak_kernel(uint64_t seed, uint32_t iters, unsigned long long *sink) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = seahash_diffuse(seed + t * 8 + (uint64_t)j);
    const uint64_t b = kWyP1 ^ seed;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = wymum(a[j], b);
    }
    uint64_t x = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) x ^= a[j];
    if (x == 0) atomicAdd(sink, 1ULL);  // keeps every chain live
}

cudaError_t launch_hash_peak(unsigned grid, uint64_t seed, uint32_t iters, unsigned long long *sink,
                             cudaStream_t st) {
    hash_peak_kernel<<<grid, 256, 0, st>>>(seed, iters, sink);
    return cudaGetLastError();
}

// The AlmostInfinite displacements (dx, dy) before rounding for n pairs of
// samples: Normal (kind kAlmostInfiniteNormal, a = sigma) or Clark2Dt (any
// other kind, a = shape u, b = 1 / p), exactly as the step kernels compute them.
__global__ void displacement_kernel(int32_t kind, const uint64_t *draws, uint64_t n, double a, double b,
                                    double *dx, double *dy) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x * blockDim.x) {
        double x, y;
        if (kind == kAlmostInfiniteNormal)
            normal_displacement(draws[2 * j], draws[2 * j + 1], a, x, y);
        else
            clark2dt_displacement(draws[2 * j], draws[2 * j + 1], a, b, x, y);
        dx[j] = x;
        dy[j] = y;
    }
}

cudaError_t launch_displacements(int32_t kind, const uint64_t *draws, uint64_t n, double a, double b, double *dx,
                                 double *dy, unsigned grid, cudaStream_t st) {
    displacement_kernel<<<grid, 256, 0, st>>>(kind, draws, n, a, b, dx, dy);
    return cudaGetLastError();
}

cudaError_t launch_promote(SimParams *params, uint32_t n_sims, cudaStream_t st) {
    promote_kernel<<<1, 256, 0, st>>>(params, n_sims);
    return cudaGetLastError();
}

template <int KIND>
static void launch_resident_t(const ResidentArgs &a, unsigned grid, cudaStream_t st) {
    if (a.exp_sampler)
        resident_kernel<KIND, kResidentMax, true><<<grid, kResidentMax, 0, st>>>(a);
    else
        resident_kernel<KIND, kResidentMax, false><<<grid, kResidentMax, 0, st>>>(a);
}

cudaError_t launch_resident(int kind, const ResidentArgs &a, unsigned grid, cudaStream_t st) {
    switch (kind) {
    case kNonSpatial: launch_resident_t<kNonSpatial>(a, grid, st); break;
    case kSpatiallyImplicit: launch_resident_t<kSpatiallyImplicit>(a, grid, st); break;
    case kAlmostInfiniteNormal: launch_resident_t<kAlmostInfiniteNormal>(a, grid, st); break;
    case kSpatiallyExplicit: launch_resident_t<kSpatiallyExplicit>(a, grid, st); break;
    case kWrappingNoise: launch_resident_t<kWrappingNoise>(a, grid, st); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace necsim
