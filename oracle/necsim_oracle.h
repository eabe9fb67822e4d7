/*
 * necsim_oracle.h -- CPU restatement of necsim-rust's Independent algorithm.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * GPU backend and the timed CPU baseline.  Only the tests, the smoke check
 * and the CPU-baseline leg of the benchmark may load it; the product never
 * links or calls it.
 *
 * Parity status: the reference (Rust, needs cargo + crates.io + a git
 * dependency) cannot be built in this environment and its own tests hold no
 * golden vectors for this path, so this restatement is pinned by
 * hand-derived known-answer values (tests/golden) and by code equivalence
 * with the cited reference lines ("parity unpinned" at the reference
 * boundary itself).
 *
 * Struct layouts below are plain C, identical to the product's C-ABI
 * structs of the same name so that one ctypes definition serves both.
 */
#ifndef NECSIM_ORACLE_H
#define NECSIM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORACLE_NON_SPATIAL = 0,
    ORACLE_SPATIALLY_IMPLICIT = 1,
    ORACLE_ALMOST_INFINITE_NORMAL = 2,
    ORACLE_SPATIALLY_EXPLICIT = 3,
    ORACLE_ALMOST_INFINITE_CLARK2DT = 4,
    ORACLE_WRAPPING_NOISE = 5,
};

/* Scenario description (same layout as the product's necsim_scenario). */
typedef struct oracle_scenario {
    int32_t kind;
    uint32_t reserved0;
    double speciation_probability;
    double turnover_rate;
    uint32_t width, height, deme;             /* NonSpatial area/deme; SI local area/deme; SE map size */
    uint32_t meta_width, meta_height, meta_deme;
    double migration_probability;
    double sigma;                             /* AlmostInfinite Normal dispersal */
    uint32_t centre_x, centre_y, radius, reserved1;
    const uint32_t *habitat;                  /* SE: width*height row-major */
    const double *dispersal;                  /* SE: (w*h) x (w*h) row-major */
    double shape_u, tail_p;                   /* AlmostInfinite Clark2Dt dispersal */
    const double *turnover;                   /* SE turnover map, width*height row-major (NULL: uniform) */
    /* WrappingNoise (rustcoalescence/scenarios/src/wrapping_noise.rs); `sigma` is its
     * Normal dispersal.  The sample fields also serve AlmostInfinite, where
     * sample_width > 0 selects the Rectangle sample over the Circle */
    int64_t noise_seed;
    double coverage;                          /* [0, 1] */
    double scale, persistence;                /* (0, 1] */
    uint64_t octaves;                         /* >= 1 */
    uint32_t sample_x, sample_y;              /* Rectangle sample: LandscapeExtent origin */
    uint64_t sample_width, sample_height;     /* 1 ..= 2^32 */
} oracle_scenario;

enum { ORACLE_MODE_REFERENCE = 0, ORACLE_MODE_CANONICAL = 1 };

typedef struct oracle_args {
    double delta_t;             /* Independent default 2.0 */
    uint64_t step_slice;        /* Independent default 10 */
    double dedup_factor;        /* DedupCache::Relative(factor); <= 0 means DedupCache::None */
    double event_slice_factor;  /* EventSlice::Relative(factor), default 2.0 */
    uint64_t min_round_events;  /* canonical schedule only */
    int32_t report_dispersal;   /* 1 if a reporter consumes dispersal events */
    int32_t mode;               /* ORACLE_MODE_* */
    uint32_t partition_rank;    /* IsolatedIndividuals partition (size 1 = monolithic) */
    uint32_t partition_size;
    uint64_t step_slice_max;    /* canonical schedule: cap on events per lineage per round (0: none) */
    int32_t event_time_sampler; /* ORACLE_SAMPLER_POISSON (default) or ORACLE_SAMPLER_EXP */
    int32_t pad;
} oracle_args;

#define ORACLE_SAMPLER_POISSON 0 /* event_time_sampler/poisson.rs */
#define ORACLE_SAMPLER_EXP 1     /* event_time_sampler/exp.rs */

typedef struct oracle_speciation_event {   /* SpeciationEvent, 40 bytes */
    uint64_t gref;
    double prior_time;
    double event_time;
    uint32_t x, y, index, pad;
} oracle_speciation_event;

typedef struct oracle_dispersal_event {    /* DispersalEvent payload, 56 bytes */
    uint64_t gref;
    double prior_time;
    double event_time;
    uint32_t x, y, index;
    uint32_t tx, ty, tindex;
    uint32_t pad, pad2;
} oracle_dispersal_event;

typedef struct oracle_lineage {            /* Lineage, 32 bytes */
    uint64_t gref;
    double last_event_time;
    uint32_t x, y, index, pad;
} oracle_lineage;

typedef struct oracle_result {
    int32_t status;             /* 0 done, 1 paused, < 0 error */
    int32_t pad;
    double time;                /* max event time */
    uint64_t steps;             /* executed events */
    uint64_t n_initial;         /* initial lineages */
    uint64_t n_remaining;       /* lineages left when paused */
    uint64_t n_speciation;      /* speciation events reported (with duplicates) */
    uint64_t biodiversity;      /* BiodiversityReporter count */
    uint64_t n_dispersal;       /* dispersal events reported */
    uint64_t n_primes;          /* WyHash prime_with calls (instrumentation) */
    uint64_t n_draws;           /* WyHash sample_u64 calls (instrumentation) */
    uint64_t n_rounds;          /* water-level windows (reference) / rounds (canonical) */
    uint64_t n_dedup;           /* lineages removed as duplicates */
} oracle_result;

/* Full simulation.  Speciation events are written in delivery order (the
 * order the reporters receive them), up to spec_cap; dispersal events up
 * to disp_cap (NULL/0 to skip); remaining lineages (paused runs) up to
 * lin_cap.  pause_before < 0 means no pause. */
int oracle_simulate(const oracle_scenario *sc, const oracle_args *args, uint64_t seed,
                    double pause_before, oracle_result *out,
                    oracle_speciation_event *spec, uint64_t spec_cap,
                    oracle_dispersal_event *disp, uint64_t disp_cap,
                    oracle_lineage *lin, uint64_t lin_cap);

/* Same as oracle_simulate but starting from caller-provided lineages
 * (resume), with min_event_time = resume_time. */
/* resume the given lineages; -5 when one is off the habitat or its deme
 * (the reference's ResumeError::Sample).  Both entry points return -6 when a
 * WrappingNoise dispersal rejects ORACLE_MAX_DISPERSAL_REJECTIONS targets in
 * a row, where the reference keeps drawing. */
#define ORACLE_MAX_DISPERSAL_REJECTIONS (1u << 20)
int oracle_simulate_lineages(const oracle_scenario *sc, const oracle_args *args, uint64_t seed,
                             const oracle_lineage *lineages, uint64_t n_lineages,
                             double resume_time, double pause_before, oracle_result *out,
                             oracle_speciation_event *spec, uint64_t spec_cap,
                             oracle_dispersal_event *disp, uint64_t disp_cap,
                             oracle_lineage *lin, uint64_t lin_cap);

/* ---- known-answer helpers ---- */
uint64_t oracle_seed_from_u64(uint64_t seed);
void oracle_wyhash_sequence(uint64_t seed, uint64_t location, uint64_t time_index,
                            uint64_t *out, uint64_t n);
uint64_t oracle_seahash_diffuse(uint64_t x);
uint64_t oracle_wymum(uint64_t a, uint64_t b);
/* next event time of the Poisson sampler at `injection` weakly after t; also
 * returns the re-prime time index in *reprime */
double oracle_poisson_next_event_time(uint64_t seed, uint64_t injection, double t,
                                      double lambda, double delta_t, uint64_t *reprime);
/* the same for the exponential sampler (exp.rs) */
double oracle_exp_next_event_time(uint64_t seed, uint64_t injection, double t,
                                  double lambda, double delta_t, uint64_t *reprime);
/* the shared correctly rounded logarithm (ln_dd.h) of n values in (0, 1] */
void oracle_ln(const double *x, double *out, uint64_t n);
/* number of origins the scenario's origin sampler yields (100% sample) */
int64_t oracle_count_origins(const oracle_scenario *sc);
int64_t oracle_enumerate_origins(const oracle_scenario *sc, oracle_lineage *out, uint64_t cap);

/* packed separable alias tables (reference layout, u32 events) */
typedef struct oracle_alias_tables {
    uint64_t n_cells;
    uint64_t n_atoms;
    uint64_t *range_start, *range_end;      /* per cell */
    double *self_dispersal;                 /* per cell */
    uint64_t *non_self_event;               /* per cell */
    double *atom_u;
    uint32_t *atom_e, *atom_k;
} oracle_alias_tables;
int oracle_build_alias(const oracle_scenario *sc, oracle_alias_tables *out);
void oracle_free_alias(oracle_alias_tables *t);
/* check_in_memory_dispersal_contract: 0 ok, 1 size mismatch, 2 dispersal to
 * non-habitat, 3 no dispersal from habitat, 4 dispersal from non-habitat */
int oracle_check_dispersal_contract(const oracle_scenario *sc);

/* Box-Muller + clamp_round_dispersal for given raw u64 draws (AlmostInfinite). */
/* clark2dt::cdf_inverse(u01, shape_u, tail_p): the Clark2Dt jump distance. */
double oracle_clark2dt_cdf_inverse(double u01, double shape_u, double tail_p);
/* Clark2Dt cdf_inverse + clamp_round_dispersal for given raw u64 draws. */
void oracle_clark2dt_dispersal(uint64_t draw0, uint64_t draw1, double shape_u, double tail_p, uint32_t x,
                               uint32_t y, uint32_t *tx, uint32_t *ty);
void oracle_normal_dispersal(uint64_t draw0, uint64_t draw1, double sigma, uint32_t x, uint32_t y,
                             uint32_t *tx, uint32_t *ty);
/* The raw displacements (dx, dy) before rounding, from n draw pairs: kind
 * ORACLE_ALMOST_INFINITE_NORMAL (a = sigma) or ORACLE_ALMOST_INFINITE_CLARK2DT
 * (a = shape u, b = tail p), with the C library's log/sin/cos/pow. */
void oracle_displacements(int32_t kind, const uint64_t *draws, uint64_t n, double a, double b, double *dx,
                          double *dy);

/* WrappingNoise: the octave noise at (x, y) (sum_noise_octaves), the
 * habitat threshold of WrappingNoiseHabitat::new, and the self-dispersal
 * probability of the approximate Normal dispersal */
double oracle_wrapping_noise(int64_t seed, double scale, double persistence, uint64_t octaves, uint32_t x,
                             uint32_t y);
double oracle_wrapping_noise_threshold(int64_t seed, double coverage, double scale, double persistence,
                                       uint64_t octaves);
double oracle_wrapping_noise_self_dispersal(double sigma, double coverage);

#ifdef __cplusplus
}
#endif

#endif
