// layout.h -- data layout shared by the host driver and the sm_100a kernels.
//
// HBM layout (one simulation or a batch of simulations of one scenario kind):
//  * lineages: structure of arrays, double-buffered (round r reads A, writes
//    the survivors to B), one slot per live lineage, coalesced per field;
//  * SpatiallyExplicit tables: one 32-byte CellRecord per habitat cell (one
//    DRAM sector: injection base, habitat, alias range, self-dispersal) and
//    one 16-byte AliasAtom per alias bucket, so an event reads 2 sectors;
//  * per-simulation SimParams (scenario scalars + the round horizon) and
//    SimCounters (steps, time, event counts), indexed by the lineage's sim id;
//  * dedup table: open-addressed slots (owner lineage, min global reference).
#pragma once

#include <cstdint>

namespace necsim {

enum Kind : int32_t {
    kNonSpatial = 0,
    kSpatiallyImplicit = 1,
    kAlmostInfiniteNormal = 2,
    kSpatiallyExplicit = 3,
    kWrappingNoise = 5,
};

// A WrappingNoise dispersal that rejects this many Normal targets in a row
// fails (kErrDispersalRejections) where the reference keeps drawing: it
// bounds the time one event can take on the device.
constexpr uint32_t kMaxDispersalRejections = 1u << 20;

// The WrappingNoise habitat (habitat/wrapping_noise/mod.rs) and its
// approximate Normal dispersal (dispersal_sampler/wrapping_noise.rs).
struct alignas(16) NoiseHabitat {
    // low bytes of the OpenSimplex permutation's first 256 entries
    // (opensimplex_noise/mod.rs:76-96): the lattice hash reads no others
    uint8_t perm[256];
    double threshold;         // habitable iff the octave noise <= threshold
    double scale, persistence;
    double coverage;          // <= 0: nothing habitable; >= 1: everything
    uint64_t octaves;
    uint64_t self_threshold;  // ceil(p_self * 2^53): self-dispersal iff X < this
};
static_assert(sizeof(NoiseHabitat) % 16 == 0, "NoiseHabitat must be whole 16-byte words");

// One habitat cell of a SpatiallyExplicit map, 32 bytes (one DRAM sector).
// Restates InMemoryHabitat's u64 injection prefix (habitat/in_memory.rs:143-163),
// the cell's habitat, AliasSamplerRange and SeparableAliasSelfDispersal
// (dispersal_sampler/in_memory/packed_separable_alias/mod.rs:22-42).
struct alignas(32) CellRecord {
    uint64_t injection;      // prefix sum of habitat over preceding cells
    double self_dispersal;   // probability of self-dispersal
    uint32_t atom_start;     // first alias atom of the cell
    uint32_t atom_count;     // number of alias atoms
    uint32_t habitat;        // deme capacity
    uint32_t non_self_event; // == own cell index iff self-dispersal is not in the atoms
};
static_assert(sizeof(CellRecord) == 32, "CellRecord must fill one sector");

// AliasMethodSamplerAtom<usize> (alias/packed.rs:10-15) with u32 events, 16 bytes.
struct alignas(16) AliasAtom {
    double u;
    uint32_t e;
    uint32_t k;
};
static_assert(sizeof(AliasAtom) == 16, "AliasAtom must be 16 bytes");

constexpr int kPoissonTable = 16;
constexpr int kPoissonThresholds = 8;

// The event-time samplers' constants for one turnover rate lambda: the
// exponential sampler's lambda and the Poisson sampler's Devroye sequence.
//
// Comparisons of a uniform u = X * 2^-53 (X the 53-bit integer of a draw)
// with a constant c are done on integers: u > c  <=>  X > floor(c * 2^53) and
// u < c  <=>  X < ceil(c * 2^53), both exact (scaling by 2^53 is exact).
struct alignas(16) PoissonConsts {
    // Devroye's loop (poisson.rs:51-65) visits the constant sequence
    // acc_n = acc_{n-1} + prod_n, prod_n = prod_{n-1} * (lambda_dt / n); the
    // draw continues past rank n iff X > threshold[n] (and prod_n > 0)
    uint64_t threshold[kPoissonThresholds];  // floor(acc_n * 2^53)
    uint32_t alive;           // bit n: prod_n > 0
    uint32_t pad;
    double prod_k;            // prod_n and acc_n at n = kPoissonThresholds
    double acc_k;
    double lambda;            // turnover rate
    double lambda_dt;         // lambda * delta_t   (poisson.rs:40)
    double lambda_dt_over_k[kPoissonTable];  // lambda_dt / k, k = 1..16
};
static_assert(sizeof(PoissonConsts) % 16 == 0, "PoissonConsts must be whole 16-byte words");

// Per-simulation scalars, read by every lineage of the simulation.
struct alignas(16) SimParams {
    PoissonConsts pois;       // the samplers' constants under uniform turnover
    // SpatiallyExplicit with a turnover map (turnover_rate/in_memory.rs): the
    // constants of every cell, row-major (nullptr: uniform turnover, `pois`)
    const PoissonConsts *turnover_cells;
    uint64_t pad4;
    uint64_t nu_threshold;    // ceil(nu * 2^53): speciation iff X < this
    uint64_t migration_threshold;  // ceil(migration * 2^53)
    // ceil(2^64 / d) for d = width and d = meta_width (0 when d == 1): a
    // 32-bit n divides as n / d = mulhi64(magic, n) (Lemire, Kaser & Kurz,
    // "Faster remainder by direct computation", 2019, Theorem 1 with F = 64)
    uint64_t width_magic;
    uint64_t meta_width_magic;
    double inv_delta_t;       // 1 / delta_t if delta_t is a power of two, else 0
    uint64_t seed;            // WyHash seed word
    double nu;                // speciation probability
    double lambda;            // the rounds' rate: the turnover rate, or the largest habitable one of a map
    double delta_t;
    double lambda_dt;         // lambda * delta_t (uniform turnover)
    double p0;                // exp(-lambda * delta_t), host libm (uniform turnover)
    double migration;         // SI
    double sigma;             // AlmostInfinite
    double min_event_time;    // resume time (0 for a fresh start)
    double pause_before;      // < 0: none
    double horizon;           // current round's horizon (schedule kernel)
    uint32_t width, height, deme;             // NS / SI local / SE map width
    uint32_t meta_ox, meta_oy, meta_width, meta_height, meta_deme;
    const CellRecord *cells;  // SE
    const AliasAtom *atoms;   // SE
    const float *cell_entropy;  // SE: per-cell dispersal entropy (learned-model feature), nullable
    uint64_t pad2;
    // AlmostInfinite with Clark2Dt dispersal (clark != 0): shape u and the
    // exponent 1 / p (almost_infinite_clark2dt.rs, clark2dt::cdf_inverse)
    double clark_shape_u;
    double clark_exponent;
    uint32_t clark;
    uint32_t pad3[3];
    NoiseHabitat noise;       // WrappingNoise
    uint64_t n_cells;
    uint64_t n_atoms;
    uint64_t step_slice;
    uint64_t min_round_events;
    uint64_t step_slice_max;
    uint64_t lineage_offset;  // first slot of the simulation's resident-arena segment
    int32_t resident;         // 1 once the resident kernel owns the simulation
    int32_t pad1;
    int32_t active;           // 1 while the simulation still advances
    int32_t pad;
};

// the step kernel copies one SimParams into shared memory in 16-byte words
static_assert(sizeof(SimParams) % 16 == 0, "SimParams must be whole 16-byte words");

// Per-simulation counters (device), accumulated as lineages leave.
struct SimCounters {
    unsigned long long steps;          // events of removed lineages
    unsigned long long max_time_bits;  // max event time (non-negative f64 bits)
    unsigned long long n_speciation;
    unsigned long long n_dedup;
    unsigned long long n_rounds;
    unsigned long long n_live;         // live lineages at the round start
    unsigned long long n_live_next;    // survivors of the current round
    unsigned long long n_dispersal;
    unsigned long long routed;         // survivors were moved to the resident arena
    // device clock (%globaltimer, ns): the simulation's first schedule, its
    // hand-over to the resident kernel (0: never) and its end or pause
    unsigned long long start_ns, routed_ns, end_ns;
};

// Lineage state, structure of arrays.
struct LineageSoA {
    uint32_t *x, *y, *idx, *sim;
    double *last;        // last event time
    double *next;        // peeked next event time (valid iff has_next)
    uint64_t *reprime;   // time index the RNG is primed with after the peek
    uint64_t *gref;      // global lineage reference
    uint64_t *steps;     // events executed by this lineage
    uint8_t *has_next;
    // learned schedule: predicted step count at which the lineage leaves the
    // simulation (0: not predicted yet); nullptr when no model is used
    float *pred_end = nullptr;
};

// Speciation event record written by the kernel (SpeciationEvent plus the
// simulation id), 40 bytes.
struct DevSpeciationEvent {
    uint64_t gref;
    double prior_time;
    double event_time;
    uint32_t x, y, idx, sim;
};

// Dispersal event record (DispersalEvent payload plus simulation id), 56 bytes.
struct DevDispersalEvent {
    uint64_t gref;
    double prior_time;
    double event_time;
    uint32_t x, y, idx;
    uint32_t tx, ty, tidx;
    uint32_t sim, pad;
};

// Device status word bits (set instead of trapping).
enum : uint32_t {
    kErrCellIndex = 1u << 0,     // a SpatiallyExplicit cell index out of range
    kErrAtomIndex = 1u << 1,     // an alias atom index out of range
    kErrEventOverflow = 1u << 2, // speciation event buffer full
    kErrDedupFull = 1u << 3,     // dedup probe sequence exhausted
    kErrDispersalOverflow = 1u << 4,
    kErrResident = 1u << 5,      // a resident simulation exceeded the block's capacity
    kErrDispersalRejections = 1u << 6,  // a WrappingNoise dispersal hit kMaxDispersalRejections
};

}  // namespace necsim
