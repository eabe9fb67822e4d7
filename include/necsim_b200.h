/*
 * necsim_b200.h -- C ABI of the B200 (sm_100a) backend for necsim-rust's
 * Independent coalescence algorithm.
 *
 * The backend is a drop-in for the reference's `algorithm: CUDA(...)` /
 * `Independent(...)` path: it takes a scenario (NonSpatial,
 * SpatiallyImplicit, AlmostInfinite with Normal or Clark2Dt dispersal,
 * SpatiallyExplicit with uniform turnover or a turnover map, WrappingNoise), a seeded
 * WyHash RNG and the
 * algorithm arguments, simulates every lineage on the GPU and hands the
 * events to reporters in the reference's reporting order.
 *
 * Conventions: every entry point returns 0 on success and a negative
 * NECSIM_E_* code on failure (never aborts or throws across the ABI); the
 * message of the last failure on a context is returned by
 * necsim_gpu_last_error().  All pointers are host pointers owned by the
 * caller; the backend copies what it needs.  A context is used by one host
 * thread at a time.
 */
#ifndef NECSIM_B200_H
#define NECSIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NECSIM_B200_ABI_VERSION 3

/* ---- error codes ---- */
#define NECSIM_OK 0
#define NECSIM_E_INVALID_ARGUMENT (-1)   /* bad scenario / argument values     */
#define NECSIM_E_CUDA (-2)               /* a CUDA runtime call failed          */
#define NECSIM_E_OUT_OF_MEMORY (-3)      /* device or host allocation failed    */
#define NECSIM_E_DEVICE_CHECK (-4)       /* a device-side bound check tripped   */
#define NECSIM_E_TIMEOUT (-5)            /* a bounded device wait gave up       */
#define NECSIM_E_DISPERSAL_MAP (-6)      /* dispersal map breaks the contract   */
#define NECSIM_E_EMPTY_HABITAT (-7)      /* habitat map has no habitable cell   */
#define NECSIM_E_UNSUPPORTED (-8)        /* valid in the reference, not here    */
#define NECSIM_E_CALLBACK (-9)           /* a reporter callback asked to stop   */
#define NECSIM_E_TOO_LARGE (-10)         /* exceeds a documented size limit     */
#define NECSIM_E_DISPERSAL_REJECTED (-11) /* a WrappingNoise dispersal rejected
                                            2^20 targets in a row (the reference
                                            keeps drawing)                      */

/* ---- scenarios ---- */
enum necsim_scenario_kind {
    NECSIM_NON_SPATIAL = 0,            /* rustcoalescence/scenarios/src/non_spatial.rs               */
    NECSIM_SPATIALLY_IMPLICIT = 1,     /* rustcoalescence/scenarios/src/spatially_implicit.rs        */
    NECSIM_ALMOST_INFINITE_NORMAL = 2, /* rustcoalescence/scenarios/src/almost_infinite/normal.rs    */
    NECSIM_SPATIALLY_EXPLICIT = 3,     /* rustcoalescence/scenarios/src/spatially_explicit/turnover/{uniform,map}.rs */
    NECSIM_ALMOST_INFINITE_CLARK2DT = 4, /* rustcoalescence/scenarios/src/almost_infinite/clark2dt.rs */
    NECSIM_WRAPPING_NOISE = 5,         /* rustcoalescence/scenarios/src/wrapping_noise.rs            */
};

/* Replaces the reference's `ScenarioCogs` as produced by `Scenario::new`
 * (rustcoalescence/scenarios/src/lib.rs:39-109) plus the
 * `speciation_probability_per_generation` argument. */
typedef struct necsim_scenario {
    int32_t kind;                    /* enum necsim_scenario_kind */
    uint32_t reserved0;
    double speciation_probability;   /* (0, 1] per generation */
    double turnover_rate;            /* uniform turnover lambda, reference default 0.5 */
    uint32_t width, height, deme;    /* NonSpatial area + deme; SI local area + deme;
                                        SpatiallyExplicit habitat map size */
    uint32_t meta_width, meta_height, meta_deme; /* SI metacommunity */
    double migration_probability;    /* SI migration probability per generation */
    double sigma;                    /* AlmostInfinite Normal dispersal sigma */
    uint32_t centre_x, centre_y, radius, reserved1; /* AlmostInfinite Circle sample */
    const uint32_t *habitat;         /* SpatiallyExplicit: width*height u32, row-major */
    const double *dispersal;         /* SpatiallyExplicit: (w*h) x (w*h) f64, row-major */
    double shape_u, tail_p;          /* AlmostInfinite Clark2Dt dispersal (u > 0, p > 0); the
                                        Circle sample fields as for Normal */
    const double *turnover_map;      /* SpatiallyExplicit: width*height f64 turnover rates, row-major
                                        (spatially_explicit/turnover/map.rs, InMemoryTurnoverRate); NULL:
                                        uniform `turnover_rate`.  Rates >= 0, > 0 on habitable cells */
    /* WrappingNoise (WrappingNoiseArguments, wrapping_noise.rs:36-48): habitable where the
       OpenSimplex octave noise is at most its coverage quantile; `sigma` is the approximate
       Normal dispersal; origins are the habitable cells of the Rectangle sample.
       AlmostInfinite: sample_width > 0 selects the Rectangle sample (sample_x, sample_y,
       sample_width, sample_height) instead of the Circle (almost_infinite/mod.rs:92-122) */
    int64_t noise_seed;
    double coverage;                 /* [0, 1] */
    double scale, persistence;       /* (0, 1] */
    uint64_t octaves;                /* >= 1 */
    uint32_t sample_x, sample_y;     /* Rectangle sample: LandscapeExtent origin */
    uint64_t sample_width, sample_height; /* 1 ..= 2^32 (OffByOneU32) */
    /* SpatiallyExplicit: device tables built before (necsim_build_tables), used instead of
       building them from `dispersal` (which may then be NULL; the learned model's dispersal
       entropy feature is 0 without it): width*height cell records and n_atoms alias atoms,
       read during the call only.  The host does not check the ranges they hold: the kernels
       bound-check every cell and atom index before reading it, and a record or atom that
       points outside the tables fails the run with NECSIM_E_DEVICE_CHECK.  NULL: build
       the tables from the maps. */
    const struct necsim_cell_record *cells;
    const struct necsim_alias_atom *atoms;
    uint64_t n_atoms;
} necsim_scenario;

/* necsim_args.event_time_sampler: which EventTimeSampler
 * (necsim/impls/no-std/src/cogs/active_lineage_sampler/independent/event_time_sampler/)
 * draws each lineage's next event time */
#define NECSIM_SAMPLER_POISSON 0u /* poisson.rs, the Independent algorithm's (launch.rs:86) */
#define NECSIM_SAMPLER_EXP 1u     /* exp.rs, the CUDA algorithm's (cuda/src/launch.rs:121) */

/* Replaces `CudaArguments` / `IndependentArguments`
 * (rustcoalescence/algorithms/cuda/src/arguments.rs:61-138,
 *  rustcoalescence/algorithms/independent/src/arguments.rs:79-146).
 * Zero fields take the documented defaults. */
typedef struct necsim_args {
    double delta_t;            /* Poisson re-priming interval; default 2.0 (Independent) */
    uint64_t step_slice;       /* expected events per lineage between dedup passes; default 10 */
    uint64_t min_round_events; /* a round runs at least this many expected events in total
                                  (widens rounds when few lineages are left); default 2^20 */
    uint64_t step_slice_max;   /* cap on expected events per lineage per round; default 1024 */
    uint32_t block_size;       /* threads per block of the step kernel; 0 = autotuned */
    uint32_t grid_size;        /* blocks of the step kernel; 0 = autotuned */
    uint32_t dedup_factor_pct; /* dedup hash table load: slots = next_pow2(n*pct/100); default 200 */
    uint32_t schedule;         /* 0 = plain (unsorted) kernel, 1 = learned lifetime buckets */
    int32_t report_dispersal;  /* reporters consume dispersal events (ReportDispersal): events
                                  leave the device after every round and reach the reporter
                                  as one stream per simulation in PackedEvent order; every
                                  lineage stays in the global rounds (no CUDA graphs, no
                                  resident kernel); NECSIM_E_TOO_LARGE if one round's events
                                  would exceed the buffer (2x the round's expected events) */
    int32_t device;            /* CUDA device ordinal; default 0 */
    uint32_t rounds_per_graph; /* rounds captured per CUDA graph launch; 0 = default (16) */
    uint32_t resident;         /* in a batch, simulations that start a round with few live lineages
                                  leave the global rounds for the per-simulation resident kernel (one
                                  block each, running its own rounds beside the global ones): 1 routes
                                  at 8 lineages (one warp of the block per lineage, each stepped
                                  cooperatively), 2..256 at that many; default 0: every simulation
                                  stays in the global rounds; same results either way; a run of one
                                  simulation always stays global */
    uint32_t event_time_sampler; /* NECSIM_SAMPLER_POISSON (0, default): PoissonEventTimeSampler,
                                    the Independent algorithm's (event_time_sampler/poisson.rs);
                                    NECSIM_SAMPLER_EXP (1): ExpEventTimeSampler, the CUDA
                                    algorithm's (event_time_sampler/exp.rs), -ln(U(0,1]) / lambda
                                    per event with a correctly rounded f64 ln */
    struct necsim_model *model; /* schedule == 1: the lifetime model ordering the step queue
                                   (must stay alive during the call; same device) */
    uint64_t max_rounds;       /* watchdog: a run that needs more rounds fails with
                                  NECSIM_E_TIMEOUT; 0 = default 2^26.  Every round advances each
                                  live lineage by >= step_slice expected events, so a valid run
                                  only meets a limit chosen below its round count */
    uint32_t priority_sims;    /* batches: this many simulations run in one priority engine (own
                                  rounds, stream and host thread) beside the others, so the others'
                                  rounds never hold them back: those in priority_list, else (schedule
                                  1) the ones the lifetime model scores as longest-lived; 0 = none,
                                  or 8 with schedule 1.  Results are identical either way */
    uint32_t priority_groups;  /* batches: the simulations outside the priority engine split into
                                  this many engines (0 or 1: one), contiguous runs of the priority order
                                  (schedule 1: the lifetime model's longest-lived first, else batch
                                  order) whose streams have decreasing CUDA stream priority, so the
                                  first groups' rounds go first and their tails start early.
                                  Results are identical either way */
    const uint32_t *priority_list; /* batch indices of the priority simulations (NULL: the model's
                                      choice); at most priority_sims are used */
    uint32_t reserve_sms;      /* batches with a priority engine: once the priority engine's live
                                  lineages fit this many SMs (its cooperative kernel's warps there),
                                  its kernels run on these SMs alone and the other engines' kernels
                                  leave them, so the priority tails' dependent event chains do not
                                  share issue slots with bulk warps; at most half the SMs; 0 = off;
                                  only with one priority engine.  Results are identical either way */
    uint32_t priority_engines; /* batches: the priority simulations split into this many engines,
                                  contiguous runs of the priority order, so that a long tail waits in
                                  lockstep rounds for fewer other priority simulations' bulk; 0 = one
                                  engine.  An engine of one simulation runs it without the resident
                                  kernel.  Results are identical either way */
} necsim_args;

/* ---- events and lineages (reference layouts) ---- */
/* SpeciationEvent (necsim/core/src/event.rs:57-66), 40 bytes */
typedef struct necsim_speciation_event {
    uint64_t global_lineage_reference;
    double prior_time;
    double event_time;
    uint32_t x, y, index, pad;
} necsim_speciation_event;

/* DispersalEvent (necsim/core/src/event.rs:74-82) without the interaction
 * (always LineageInteraction::Maybe on the Independent path), 56 bytes */
typedef struct necsim_dispersal_event {
    uint64_t global_lineage_reference;
    double prior_time;
    double event_time;
    uint32_t x, y, index;
    uint32_t target_x, target_y, target_index;
    uint32_t pad, pad2;
} necsim_dispersal_event;

/* Lineage (necsim/core/src/lineage.rs:91-106), 32 bytes */
typedef struct necsim_lineage {
    uint64_t global_reference;
    double last_event_time;
    uint32_t x, y, index, pad;
} necsim_lineage;

/* Reporter sink, replaces `Reporter::report_speciation` /
 * `report_dispersal` (necsim/core/src/reporter/mod.rs:22-58).  Events are
 * delivered in batches, each batch in the reference's PackedEvent order
 * (event.rs:256-280), batches in increasing time.  A callback returning
 * non-zero stops the delivery with NECSIM_E_CALLBACK. */
typedef struct necsim_reporter {
    void *user;
    int (*report_speciation)(void *user, const necsim_speciation_event *events, uint64_t n);
    int (*report_dispersal)(void *user, const necsim_dispersal_event *events, uint64_t n);
} necsim_reporter;

/* Replaces `SimulationOutcome` (rustcoalescence/algorithms/src/result.rs):
 * Done{time, steps} or Paused{time, steps, lineages, rng}. */
typedef struct necsim_outcome {
    int32_t paused;            /* 0 = Done, 1 = Paused (remaining lineages available) */
    int32_t pad;
    double time;               /* time of the last executed event */
    uint64_t steps;            /* executed events (lineage steps) */
    uint64_t n_initial;        /* lineages simulated */
    uint64_t n_remaining;      /* lineages left when paused */
    uint64_t n_speciation;     /* speciation events reported (with duplicates) */
    uint64_t biodiversity;     /* BiodiversityReporter count of distinct species */
    uint64_t n_dispersal;      /* dispersal events reported */
    uint64_t n_rounds;         /* synchronised rounds executed */
    uint64_t n_dedup;          /* duplicate lineages removed */
    uint64_t n_launches;       /* kernels launched by this call */
    double kernel_ms;          /* device time of the step kernel (CUDA events) */
    double total_ms;           /* device time of the whole simulation (CUDA events) */
    uint64_t h2d_bytes;        /* host-to-device bytes copied by the call */
    uint64_t d2h_bytes;        /* device-to-host bytes copied by the call */
    uint64_t n_step_launches;  /* step-kernel launches (one per round) */
    uint64_t lineage_visits;   /* lineage slots the step kernels processed */
    double resident_ms;        /* device time of the per-simulation resident kernel (CUDA
                                  events; overlaps the global rounds) */
    double end_ms;             /* when this simulation ended (or paused), in ms of the device
                                  clock after the run (batch: the batch) began its rounds */
    double routed_ms;          /* batches: when the resident kernel took the simulation over
                                  (same clock), -1 if it stayed in the global rounds */
} necsim_outcome;

typedef struct necsim_ctx necsim_ctx;

/* Create a context: validates the scenario, builds the dispersal tables
 * (SpatiallyExplicit: packed separable alias, packed_separable_alias/mod.rs:64-203),
 * uploads them to the device and enumerates the origin lineages
 * (OriginPreSampler::all() and the origin samplers).  Replaces the set-up half of
 * `Algorithm::initialise_and_simulate` (rustcoalescence/algorithms/src/lib.rs:81-93). */
int necsim_gpu_create(const necsim_scenario *scenario, const necsim_args *args,
                      necsim_ctx **out_ctx);
/* On failure *out_ctx may still receive a context that only carries the
 * error message (necsim_gpu_last_error); destroy it with necsim_gpu_destroy. */

/* Simulate all origin lineages of the context's scenario to completion or
 * until `pause_before` (< 0: no pause).  `wyhash_seed` is the WyHash seed
 * word (necsim/impls/no-std/src/cogs/rng/wyhash.rs:41-49); use
 * necsim_seed_from_u64() for the reference's `rng: Seed(u64)`.
 * Replaces `Algorithm::initialise_and_simulate` (algorithms/src/lib.rs:81-93). */
int necsim_gpu_simulate(necsim_ctx *ctx, uint64_t wyhash_seed, double pause_before,
                        const necsim_reporter *reporter, necsim_outcome *outcome);

/* Simulate caller-provided lineages (resume), with min_event_time =
 * resume_time.  Replaces `Algorithm::resume_and_simulate`
 * (algorithms/src/lib.rs:95-107).  A lineage outside the habitat (its
 * location off the landscape or of habitat 0) or outside its deme (index >=
 * habitat) fails the call with NECSIM_E_INVALID_ARGUMENT, as the reference's
 * ResumeError::Sample does (algorithms/src/result.rs:29-31). */
int necsim_gpu_simulate_lineages(necsim_ctx *ctx, const necsim_lineage *lineages, uint64_t n,
                                 double resume_time, uint64_t wyhash_seed, double pause_before,
                                 const necsim_reporter *reporter, necsim_outcome *outcome);

/* Lineages left after a paused simulation (SimulationOutcome::Paused.lineages),
 * in ascending global reference order.  *n_out receives the count; at most
 * `cap` are written. */
int necsim_gpu_remaining_lineages(necsim_ctx *ctx, necsim_lineage *out, uint64_t cap,
                                  uint64_t *n_out);

/* Batched sweep: simulate `n_sims` independent simulations (scenarios may
 * differ in every parameter, seeds per simulation) in one persistent launch
 * per round.  No reference counterpart as a single call: it replaces
 * `n_sims` calls of `Algorithm::initialise_and_simulate`.  outcomes[s]
 * receives simulation s's outcome; reporters may be NULL or an array of
 * n_sims sinks. */
int necsim_gpu_simulate_batch(const necsim_scenario *scenarios, const uint64_t *wyhash_seeds,
                              uint32_t n_sims, const necsim_args *args, double pause_before,
                              const necsim_reporter *reporters, necsim_outcome *outcomes,
                              char *error, size_t error_cap);

/* Resident batch: the same batch as necsim_gpu_simulate_batch split into a
 * set-up call (validation, tables, origin lineages uploaded once and kept
 * in device memory, CUDA graph captured) and runs that restart from the
 * resident origins with no host-to-device lineage copy.  Each run simulates
 * every simulation from its origins with its seed; runs are identical.
 * No reference counterpart: it is `n_sims` calls of
 * `Algorithm::initialise_and_simulate` with the set-up hoisted out.
 * On failure *out may still receive an object carrying the message
 * (necsim_gpu_batch_last_error); destroy it with necsim_gpu_batch_destroy. */
typedef struct necsim_batch necsim_batch;
int necsim_gpu_batch_create(const necsim_scenario *scenarios, const uint64_t *wyhash_seeds,
                            uint32_t n_sims, const necsim_args *args, double pause_before,
                            necsim_batch **out);
int necsim_gpu_batch_run(necsim_batch *batch, const necsim_reporter *reporters,
                         necsim_outcome *outcomes);
/* The batch indices of the simulations in the priority engine
 * (necsim_args.priority_sims), in priority order: up to `cap` into `ids`,
 * their count in *n.  No reference counterpart. */
int necsim_gpu_batch_priority(const necsim_batch *batch, uint32_t *ids, uint32_t cap, uint32_t *n);
const char *necsim_gpu_batch_last_error(const necsim_batch *batch);
void necsim_gpu_batch_destroy(necsim_batch *batch);

/* ---- allocation-free round ----
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory themselves or through us (a host whose allocator owns the GPU, a
 * plugin handed a fixed arena, a service that forbids cudaMalloc/cudaFree
 * and the device synchronisation they can cause after start-up): one round
 * -- every lineage advanced through all its events before `horizon`, then
 * lineages in identical state merged into the one with the smallest global
 * reference -- computed in a working area that lives in the library as a
 * static device array (about 9.5 MB per GPU, kept until the process exits).
 *
 * d_lineages (n entries), d_out (n entries) and d_events (events_cap
 * entries) are DEVICE pointers owned by the caller; n may not exceed
 * NECSIM_NOALLOC_MAX_LINEAGES (NECSIM_E_TOO_LARGE otherwise).  Scenario
 * kinds without tables only (NonSpatial, SpatiallyImplicit, AlmostInfinite);
 * SpatiallyExplicit returns NECSIM_E_UNSUPPORTED.  resume_time is the
 * min_event_time of the lineages.  `args` (NULL: defaults) selects the
 * event-time sampler (event_time_sampler; other values are
 * NECSIM_E_INVALID_ARGUMENT) and delta_t; the launch shape follows the
 * device's SM count.  Surviving lineages and speciation events are written
 * in no particular order; *n_out, *n_events and *steps (events executed)
 * are set on return.  Work is queued on `stream` (a cudaStream_t, NULL =
 * default stream) and the call waits for it.
 *
 * The first call on a device looks up the device address of the working
 * area and the device's SM count; make that first call before capturing any
 * stream into a CUDA graph.
 * Every call shares the one working area and clears it before use, so calls
 * whose GPU work overlaps (other streams or host threads) race. */
#define NECSIM_NOALLOC_MAX_LINEAGES 65536
int necsim_gpu_round_noalloc(const necsim_scenario *scenario, const necsim_args *args,
                             uint64_t wyhash_seed, const necsim_lineage *d_lineages, uint64_t n,
                             double resume_time, double horizon, necsim_lineage *d_out,
                             uint64_t *n_out, necsim_speciation_event *d_events,
                             uint64_t events_cap, uint64_t *n_events, uint64_t *steps,
                             void *stream);

const char *necsim_gpu_last_error(const necsim_ctx *ctx);
void necsim_gpu_destroy(necsim_ctx *ctx);

/* SeedableRng::seed_from_u64 (necsim/core/src/cogs/rng.rs:33-63) followed by
 * WyHash::from_seed (wyhash.rs:41-49): the WyHash seed word for `Seed(seed)`. */
uint64_t necsim_seed_from_u64(uint64_t seed);

/* ABI version, for bindings to check. */
int necsim_abi_version(void);

/* ---- host-side table construction (no GPU needed) ---- */
/* One cell of the SpatiallyExplicit device tables, 32 bytes: the habitat
 * injection prefix (habitat/in_memory.rs:143-163), the self-dispersal
 * probability and non-self event (SeparableAliasSelfDispersal) and the
 * cell's alias range (AliasSamplerRange), packed_separable_alias/mod.rs:22-42. */
typedef struct necsim_cell_record {
    uint64_t injection;
    double self_dispersal;
    uint32_t atom_start, atom_count, habitat, non_self_event;
} necsim_cell_record;

/* AliasMethodSamplerAtom (alias/packed.rs:10-15) with u32 events, 16 bytes. */
typedef struct necsim_alias_atom {
    double u;
    uint32_t e, k;
} necsim_alias_atom;

/* Builds the tables InMemoryPackedSeparableAliasDispersalSampler::new
 * (packed_separable_alias/mod.rs:64-203) builds, into caller buffers:
 * `cells` needs width*height records, `atoms` up to `atom_cap` atoms;
 * *n_atoms receives the atom count (call with atoms == NULL to size). */
int necsim_build_tables(const necsim_scenario *scenario, necsim_cell_record *cells,
                        necsim_alias_atom *atoms, uint64_t atom_cap, uint64_t *n_atoms);

/* The scenario's origin lineages in the reference's origin-sampler order
 * (OriginPreSampler::all() through origin_sampler/{non_spatial,in_memory,
 * spatially_implicit,singleton_demes/{circle,rectangle}}.rs, Lineage::new gives the
 * global reference = the location's u64 injection).  *n_out receives the
 * count; at most `cap` are written (out may be NULL to size). */
int necsim_enumerate_origins(const necsim_scenario *scenario, necsim_lineage *out, uint64_t cap,
                             uint64_t *n_out);

/* IsolatedLandscape parallelism (rustcoalescence/algorithms/independent/src/launch.rs:101-110,
 * algorithms/cuda/src/launch.rs:135-140): the subdomain rank of each lineage's location under the
 * scenario's decomposition into `size` subdomains; origin_sampler/decomposition.rs keeps an origin iff
 * its rank is the partition's.  The decompositions are the scenarios' `decompose`:
 * ModuloDecomposition (NonSpatial, SpatiallyImplicit), RadialDecomposition (AlmostInfinite,
 * WrappingNoise) and EqualDecomposition::weight (SpatiallyExplicit), decomposition/{modulo,radial,
 * equal/{mod,weight}}.rs.  `exact` (may be NULL) receives 0 when the weight decomposition could not
 * split the habitat into `size` parts (the reference warns and uses the ranks it found), else 1. */
int necsim_subdomain_ranks(const necsim_scenario *scenario, uint32_t size, const necsim_lineage *lineages,
                           uint64_t n, uint32_t *ranks, int32_t *exact);

/* Origin pre-sampling: positions, in the order of necsim_enumerate_origins,
 * of the origins that OriginPreSampler::all().percentage(percentage)
 * .partition(rank, size) selects among the first n
 * (necsim/impls/no-std/src/cogs/origin_sampler/pre_sampler.rs:48-112: a
 * golden-ratio quasi-random geometric skip sequence evaluated with the
 * system libm's log, then every size-th starting at rank).  Simulate the
 * selected origins with necsim_gpu_simulate_lineages (resume_time 0).
 * *n_out receives the count; at most `cap` are written (out may be NULL). */
int necsim_presample_origins(uint64_t n, double percentage, uint32_t rank, uint32_t size, uint64_t *out,
                             uint64_t cap, uint64_t *n_out);

/* ---- SpatiallyExplicit maps ----
 * Replaces load_map_from_tiff (rustcoalescence/scenarios/src/spatially_explicit/
 * maps/tiff/mod.rs:27-127): loads the first image of a one-band (Geo)TIFF --
 * classic or BigTIFF, either byte order, strips or tiles, uncompressed, LZW,
 * PackBits or Deflate, predictor 1, 2 or 3 -- as row-major samples:
 * NECSIM_MAP_U32 (habitat: 32-bit, SampleFormat Uint or absent) or
 * NECSIM_MAP_F64 (dispersal, turnover: 64-bit IEEEFP).  Unless `strict`,
 * samples equal to the GDAL no-data value (tag 42113, parsed like Rust's
 * `str::parse`) become 0.  *data is allocated here: release it with
 * necsim_map_free.  Errors name the file in `error`. */
#define NECSIM_MAP_U32 0
#define NECSIM_MAP_F64 1
int necsim_map_load(const char *path, int32_t sample, int32_t strict, void **data, uint32_t *width,
                    uint32_t *height, char *error, size_t error_cap);
void necsim_map_free(void *data);

/* Map loading modes (maps/mod.rs:79-89, MapLoadingMode) and their fix-ups
 * (maps/mod.rs:56-77, 90-215), applied in place:
 *   OFF_BY_ONE (the reference's default): habitat values 0/1 become 1 where
 *     any dispersal leaves the cell, else 0 (0 where turnover is 0);
 *   FIX_ME: that, then habitat 0 where turnover is 0, then dispersal to and
 *     from non-habitat removed and self-dispersal 1 added to habitat cells
 *     with none left (the dispersal map must be (w*h) x (w*h));
 *   STRICT: no change (maps load with `strict`).
 * Every mode first rejects negative dispersal weights
 * (NECSIM_E_DISPERSAL_MAP) and turnover rates.  `turnover` (w*h rates) may
 * be NULL (uniform turnover). */
#define NECSIM_MAPS_OFF_BY_ONE 0
#define NECSIM_MAPS_FIX_ME 1
#define NECSIM_MAPS_STRICT 2
int necsim_maps_fix(uint32_t *habitat, uint32_t width, uint32_t height, double *dispersal, uint64_t dispersal_rows,
                    uint64_t dispersal_cols, const double *turnover, int32_t mode, char *error, size_t error_cap);

/* ---- event log ----
 * The reference's on-disk event log (EventLogRecorder,
 * necsim/impls/std/src/event_log/recorder.rs): a reporter that buffers
 * events as PackedEvents and writes segments of `segment_capacity` events,
 * each sorted by PackedEvent::cmp, as files 0, 1, ... of `directory` in
 * bincode 1.3 encoding (a 26-byte EventLogHeader, then 56-byte PackedEvents;
 * dispersal events carry LineageInteraction::Maybe, as the Independent
 * algorithm reports them), readable by the reference's replay.  `directory`
 * must not exist (its parents are created).  Pass the reporter to any
 * simulate call; close to write the last segment. */
typedef struct necsim_event_log necsim_event_log;
int necsim_event_log_create(const char *directory, uint64_t segment_capacity, int32_t record_speciation,
                            int32_t record_dispersal, necsim_event_log **out);
necsim_reporter necsim_event_log_reporter(necsim_event_log *log);
int necsim_event_log_close(necsim_event_log *log);

/* Replays event-log segments (EventLogReplay, necsim/impls/std/src/
 * event_log/replay/mod.rs; rustcoalescence replay): reads the segment files
 * `segments[0..n)` -- `capacity` events at a time per segment -- and hands
 * every event to `reporter` as one stream in PackedEvent order, speciation
 * and dispersal batches interleaved as the stream requires.  Segments must
 * agree on the kinds they record.  The reporters' needs (need_speciation,
 * need_dispersal) are checked against the log as the replay's `mode` does:
 * an unmet need fails when `strict` (ReplayMode::Strict) and is returned as
 * a warning in `error` with NECSIM_OK otherwise (WarnOnly).  *n_events
 * receives the number of events replayed. */
int necsim_event_log_replay(const char *const *segments, uint64_t n_segments, uint64_t capacity,
                            int32_t need_speciation, int32_t need_dispersal, int32_t strict,
                            const necsim_reporter *reporter, uint64_t *n_events, char *error, size_t error_cap);

/* The integer-issue ceiling of the path's hash work, measured on `device`:
 * the rate of wymum (64x64 -> 128-bit multiply, WyHash's mixing step,
 * wyhash.rs:85-96) over independent chains filling every SM.  No reference
 * counterpart: the denominator of the benchmark's integer-issue roofline. */
int necsim_gpu_hash_peak(int32_t device, double *wymum_per_second);

/* The AlmostInfinite dispersal displacements (dx, dy), before
 * clamp_round_dispersal (habitat/almost_infinite.rs:100-114) rounds them onto
 * the plane, that the kernels compute for n pairs of WyHash samples
 * (draws[2j], draws[2j + 1]): Normal (kind NECSIM_ALMOST_INFINITE_NORMAL, a =
 * sigma; Box-Muller of rng.rs:180-197 scaled as almost_infinite_normal.rs:58-68)
 * or Clark2Dt (NECSIM_ALMOST_INFINITE_CLARK2DT, a = shape u, b = tail p;
 * almost_infinite_clark2dt.rs:96-107).  The device evaluates ln/sin/cos/pow
 * with CUDA's f64 library where the reference calls the system libm; this
 * entry point lets a caller measure where the two disagree.  No reference
 * counterpart. */
int necsim_gpu_displacements(int32_t device, int32_t kind, const uint64_t *draws, uint64_t n, double a, double b,
                             double *dx, double *dy);

/* ---- launch autotuner ----
 * Times a bounded sample of a batch -- every k-th simulation so that the
 * sample holds at most `max_sample_lineages` origins, each paused at
 * `sample_pause` -- under every combination of block size {64, 128, 256},
 * step_slice {s, 2s, 4s} (s = args->step_slice) and dedup table factor
 * {200, 400} %, on the device of `args`, and returns in *best the argument
 * set with the shortest time to the pause (best of two runs after a
 * warm-up run).  Every candidate yields the same species and speciation
 * events; only steps (duplicate work) and time differ.  `results` (nullable)
 * receives one record per candidate, at most `results_cap`; *n_results the
 * count.  No counterpart in the reference (its arguments are set by hand). */
typedef struct necsim_autotune_result {
    uint32_t block_size;
    uint32_t dedup_factor_pct;
    uint64_t step_slice;
    double ms;      /* best device time of the sample (CUDA events) */
    uint64_t steps; /* events of the sample */
} necsim_autotune_result;

int necsim_gpu_autotune(const necsim_scenario *scenarios, const uint64_t *wyhash_seeds, uint32_t n_sims,
                        const necsim_args *args, double sample_pause, uint64_t max_sample_lineages,
                        necsim_args *best, necsim_autotune_result *results, uint32_t results_cap,
                        uint32_t *n_results, char *error, size_t error_cap);

/* ---- learned lifetime scheduler ----
 * A small MLP (8 -> 64 -> 64 -> 1, ReLU, bf16 weights, fp32 accumulation)
 * predicting, from one lineage's 8 features (position in the extent,
 * habitat, dispersal entropy, time, speciation probability, live lineages of
 * its simulation, events executed), log(1 + remaining events) of its
 * simulation's longest-lived lineage: the simulation's remaining life.  With
 * necsim_args.schedule = 1 and .model set, a batch's simulations with the
 * longest predicted lives run in a priority engine of their own
 * (necsim_args.priority_sims) and every round's step queue is bucketed by
 * expected work (min(events per round, prediction)), largest first.  The
 * model only reorders work: events, species counts and step counts are the
 * same as with schedule = 0.  There is no reference interface for this part
 * (it is new in this backend). */
#define NECSIM_MODEL_FEATURES 8
#define NECSIM_MODEL_PARAMS 4801 /* W1[64][8], b1[64], W2[64][64], b2[64], W3[64], b3 */

typedef struct necsim_model necsim_model;

/* He-initialised weights from `seed`, on CUDA device `device`. */
int necsim_model_create(int32_t device, uint64_t seed, necsim_model **out);
void necsim_model_destroy(necsim_model *model);
const char *necsim_model_last_error(const necsim_model *model);
/* The bf16 weights (as fp32) / set the weights (fp32 master copy, rounded
 * to bf16 for use; resets the optimiser state). */
int necsim_model_get_weights(necsim_model *model, float *out);
int necsim_model_set_weights(necsim_model *model, const float *weights);
/* y[i] = MLP(X[i * 8 .. i * 8 + 8]) for n rows (host buffers). */
int necsim_model_predict(necsim_model *model, const float *X, uint64_t n, float *y);
/* Gradient of L = sum_i 0.5 * (MLP(X_i) - T_i)^2 / n with respect to the
 * NECSIM_MODEL_PARAMS parameters (evaluated at the bf16 weights), and L. */
int necsim_model_gradients(necsim_model *model, const float *X, const float *T, uint64_t n, float *grads,
                           double *loss);
/* Adam on the device: `epochs` passes over the n rows in a fresh random
 * order each (from `seed`), mini-batches of `batch` rows, learning rate
 * `lr`; epoch_loss (nullable) receives the mean loss of each epoch. */
int necsim_model_train(necsim_model *model, const float *X, const float *T, uint64_t n, uint32_t epochs,
                       uint32_t batch, float lr, uint64_t seed, double *epoch_loss);

/* Training traces: runs the batch (global rounds only) and every
 * `snapshot_rounds` rounds (even, >= 2) records the features of the live
 * lineages; a recorded lineage's label is log(1 + events it executed after
 * the snapshot until it speciated or was removed as a duplicate).  Rows
 * whose lineage outlives the run are dropped.  At most `max_rows` rows are
 * returned, evenly subsampled; `features` holds max_rows * 8 floats,
 * `labels` max_rows; *n_rows receives the count. */
int necsim_gpu_trace_batch(const necsim_scenario *scenarios, const uint64_t *wyhash_seeds, uint32_t n_sims,
                           const necsim_args *args, double pause_before, uint32_t snapshot_rounds,
                           uint64_t max_rows, float *features, float *labels, uint64_t *n_rows,
                           char *error, size_t error_cap);

#ifdef __cplusplus
}
#endif

#endif /* NECSIM_B200_H */
