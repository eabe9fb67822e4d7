/*
 * necsim_oracle.c -- CPU restatement of necsim-rust's Independent algorithm
 * (Monolithic parallelisation, Poisson event-time sampler, WyHash RNG,
 * IntrinsicsMathsCore = the system libm), with the CUDA algorithm's
 * exponential event-time sampler as an option (its logarithm is the
 * product's correctly rounded ln_dd.h, shared source, so event times agree
 * bit for bit; glibc's log differs from it by one ulp on ~0.08% of inputs).
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for the GPU backend and the
 * timed CPU baseline.  The product never links or calls this file.
 *
 * Two modes:
 *   ORACLE_MODE_REFERENCE  -- the reference's own schedule: VecDeque slow/fast
 *       queues, step_slice early stops, a lossy FNV-hashed direct-mapped
 *       dedup cache and the live water-level reporter (sort per window).
 *   ORACLE_MODE_CANONICAL  -- the GPU backend's deterministic schedule: all
 *       lineages advance to a common time horizon per round, then lineages in
 *       identical state are deduplicated keeping the smallest global
 *       reference.  Same per-lineage arithmetic as the reference mode.
 * Both modes yield the same species count and the same set of distinct
 * speciation events (event time, origin); only which duplicate lineages are
 * simulated (and hence `steps` and duplicate events) differs.
 *
 * Compiled with -ffp-contract=off -fno-fast-math: every f64 operation is a
 * single IEEE-754 round-to-nearest operation in the order written, as in the
 * Rust reference (LLVM does not contract f64 mul/add without fast-math).
 *
 * Parity unpinned at the reference boundary: the Rust reference cannot be
 * built here and its tests hold no golden vectors for this path.
 */
#include "necsim_oracle.h"
#include "../necsim-rust_b200/csrc/ln_dd.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* WyHash PrimeableRng                                                       */
/* necsim/impls/no-std/src/cogs/rng/wyhash.rs:9-12 (constants)               */
/* ------------------------------------------------------------------------ */
#define WY_P0 0xa0761d6478bd642fULL
#define WY_P1 0xe7037ed1a0b428dbULL
#define WY_P2 0x8ebc6af09c88c6e3ULL
#define WY_P5 0xeb44accab455d165ULL
#define SEAHASH_K 0x6eed0e9da4d94a4fULL
/* event_time_sampler/poisson.rs:10 -- 2^64 / PHI */
#define INV_PHI_U64 0x9e3779b97f4a7c15ULL

typedef struct rng_t {
    uint64_t seed;
    uint64_t state;
    uint64_t n_primes;
    uint64_t n_draws;
} rng_t;

/* wyhash.rs:85-96 -- 64x64->128 multiply, xor-folded ("condom") */
static inline uint64_t wymum(uint64_t a, uint64_t b) {
    unsigned __int128 r = (unsigned __int128)a * (unsigned __int128)b;
    a ^= (uint64_t)r;
    b ^= (uint64_t)(r >> 64);
    return a ^ b;
}

/* wyhash.rs:99-119 -- SeaHash diffusion */
static inline uint64_t seahash_diffuse(uint64_t x) {
    x *= SEAHASH_K;
    uint64_t a = x >> 32;
    uint64_t b = x >> 60;
    x ^= a >> b;
    x *= SEAHASH_K;
    return x;
}

/* wyhash.rs:53-63 */
static inline uint64_t rng_sample_u64(rng_t *g) {
    g->n_draws++;
    g->state += WY_P0;
    uint64_t wyrng = wymum(g->state ^ WY_P1, g->state);
    return seahash_diffuse(wyrng);
}

static inline uint64_t swap_halves(uint64_t v) { return (v << 32) | (v >> 32); }

/* wyhash.rs:68-80 */
static inline void rng_prime(rng_t *g, uint64_t location_index, uint64_t time_index) {
    g->n_primes++;
    uint64_t l = seahash_diffuse(location_index);
    uint64_t t = seahash_diffuse(time_index);
    uint64_t hash = wymum(swap_halves(l) ^ (g->seed ^ WY_P0), swap_halves(t) ^ WY_P2);
    g->state = wymum(hash, 16ULL ^ WY_P5);
}

/* necsim/core/src/cogs/rng.rs:33-63 -- SeedableRng::seed_from_u64 (PCG32
 * expansion into the 8 seed bytes), then wyhash.rs:41-49 from_seed (LE). */
uint64_t oracle_seed_from_u64(uint64_t state) {
    const uint64_t MUL = 6364136223846793005ULL;
    const uint64_t INC = 11634580027462260723ULL;
    uint64_t seed = 0;
    for (int chunk = 0; chunk < 2; ++chunk) {
        state = state * MUL + INC;
        uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
        uint32_t rot = (uint32_t)(state >> 59);
        uint32_t x = (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
        seed |= ((uint64_t)x) << (32 * chunk);
    }
    return seed;
}

/* rng.rs:75-82 sample_uniform_closed_open: (u64 >> 11) * 2^-53 */
static inline double u01_closed_open(rng_t *g) {
    return (double)(rng_sample_u64(g) >> 11) * 0x1.0p-53;
}

/* rng.rs:84-93 sample_uniform_open_closed: ((u64 >> 11) + 1) * 2^-53 */
static inline double u01_open_closed(rng_t *g) {
    return (double)((rng_sample_u64(g) >> 11) + 1) * 0x1.0p-53;
}

/* Rust `f64 as u64` / `as u32` / `as i64`: truncate, saturate, NaN -> 0 */
static inline uint64_t f64_as_u64(double v) {
    if (!(v > 0.0)) return 0;
    if (v >= 18446744073709551616.0) return UINT64_MAX;
    return (uint64_t)v;
}
static inline uint32_t f64_as_u32(double v) {
    if (!(v > 0.0)) return 0;
    if (v >= 4294967296.0) return UINT32_MAX;
    return (uint32_t)v;
}
static inline int64_t f64_as_i64(double v) {
    if (v != v) return 0;
    if (v >= 9223372036854775808.0) return INT64_MAX;
    if (v < -9223372036854775808.0) return INT64_MIN;
    return (int64_t)v;
}

/* rng.rs:133-145 sample_index_u64 */
static inline uint64_t sample_index_u64(rng_t *g, uint64_t length) {
    uint64_t index = f64_as_u64(floor(u01_closed_open(g) * (double)length));
    return index < length - 1 ? index : length - 1;
}

/* positive_f64.rs:103-113 PositiveF64::max_after */
static inline double max_after(double before, double value) {
    if (value > before || isnan(before)) return value;
    if (isinf(before)) return INFINITY;
    uint64_t bits;
    memcpy(&bits, &before, 8);
    bits += 1;
    double r;
    memcpy(&r, &bits, 8);
    return r;
}

static inline uint64_t f64_bits(double v) {
    uint64_t b;
    memcpy(&b, &v, 8);
    return b;
}

/* ------------------------------------------------------------------------ */
/* Scenario cogs                                                             */
/* ------------------------------------------------------------------------ */
typedef struct extent_t {
    uint32_t ox, oy;
    uint64_t w, h;  /* OffByOneU32::get() values (>= 1) */
} extent_t;

/* necsim/core/src/landscape/extent.rs:44-49 LandscapeExtent::contains */
static inline int extent_contains(const extent_t *e, uint32_t x, uint32_t y) {
    uint32_t x_hi = e->ox + (uint32_t)(e->w - 1);  /* add_incl, wrapping */
    uint32_t y_hi = e->oy + (uint32_t)(e->h - 1);
    return x >= e->ox && x <= x_hi && y >= e->oy && y <= y_hi;
}

typedef struct alias_t {
    uint64_t n_cells, n_atoms;
    uint64_t *range_start, *range_end;
    double *self_dispersal;
    uint64_t *non_self_event;
    double *atom_u;
    uint32_t *atom_e, *atom_k;
} alias_t;

typedef struct sim_t {
    int kind;
    double nu;          /* speciation probability */
    double lambda;      /* uniform turnover rate */
    double delta_t;
    double lambda_dt;   /* lambda * delta_t   (poisson.rs:40) */
    double p0;          /* exp(-lambda * delta_t) (poisson.rs:42) */
    double migration;
    double sigma;
    int clark;          /* AlmostInfinite with Clark2Dt dispersal */
    int exp_sampler;    /* ExpEventTimeSampler instead of the Poisson one */
    const double *turnover;  /* SE turnover map (InMemoryTurnoverRate), NULL: uniform lambda */
    double shape_u, tail_p;
    extent_t local;     /* NonSpatial / SI local / SE map extent */
    uint32_t deme;
    extent_t meta;      /* SI meta */
    uint32_t meta_deme;
    /* SE */
    const uint32_t *habitat;
    uint64_t *injection;  /* prefix sums, n_cells + 1 */
    alias_t alias;
    /* WrappingNoise */
    int64_t perm[2048];   /* OpenSimplexNoise permutation */
    double coverage, scale, persistence, threshold, p_self;
    uint64_t octaves;
    int fault;            /* -6 once a dispersal ran out of rejections */
    rng_t rng;
} sim_t;

/* habitat/non_spatial.rs:88-105 map_indexed_location_to_u64_injective */
static inline uint64_t non_spatial_injection(const extent_t *e, uint32_t deme, uint32_t x,
                                             uint32_t y, uint32_t i) {
    return ((uint64_t)(y - e->oy) * e->w + (uint64_t)(x - e->ox)) * (uint64_t)deme + (uint64_t)i;
}

static inline uint64_t injection(const sim_t *s, uint32_t x, uint32_t y, uint32_t i) {
    switch (s->kind) {
    case ORACLE_NON_SPATIAL:
        return non_spatial_injection(&s->local, s->deme, x, y, i);
    case ORACLE_SPATIALLY_IMPLICIT:
        /* habitat/spatially_implicit.rs:106-120 (overlapping codomains) */
        if (extent_contains(&s->local, x, y))
            return non_spatial_injection(&s->local, s->deme, x, y, i);
        return non_spatial_injection(&s->meta, s->meta_deme, x, y, i);
    case ORACLE_ALMOST_INFINITE_NORMAL:
    case ORACLE_WRAPPING_NOISE:
        /* habitat/almost_infinite.rs:66-70 (WrappingNoise defers to it,
         * habitat/wrapping_noise/mod.rs:170-175) */
        return ((uint64_t)y << 32) | (uint64_t)x;
    default: {
        /* habitat/in_memory.rs:70-80 */
        uint64_t cell = (uint64_t)y * s->local.w + (uint64_t)x;
        uint64_t n = s->local.w * s->local.h;
        return (cell < n ? s->injection[cell] : 0) + (uint64_t)i;
    }
    }
}

static double noise_octaves(const sim_t *s, uint32_t x, uint32_t y);

static inline uint32_t habitat_at(const sim_t *s, uint32_t x, uint32_t y) {
    switch (s->kind) {
    case ORACLE_NON_SPATIAL:
        return s->deme;
    case ORACLE_SPATIALLY_IMPLICIT:
        /* habitat/spatially_implicit.rs:95-103 */
        if (extent_contains(&s->local, x, y)) return s->deme;
        if (extent_contains(&s->meta, x, y)) return s->meta_deme;
        return 0;
    case ORACLE_ALMOST_INFINITE_NORMAL:
        return 1;
    case ORACLE_WRAPPING_NOISE:
        /* habitat/wrapping_noise/mod.rs:148-168 */
        if (s->coverage <= 0.0) return 0;
        if (s->coverage >= 1.0) return 1;
        return noise_octaves(s, x, y) <= s->threshold ? 1u : 0u;
    default: {
        uint64_t cell = (uint64_t)y * s->local.w + (uint64_t)x;
        return cell < s->local.w * s->local.h ? s->habitat[cell] : 0;
    }
    }
}

/* speciation_probability/uniform.rs; spatially_implicit.rs:31-44 */
static inline double speciation_probability(const sim_t *s, uint32_t x, uint32_t y) {
    if (s->kind == ORACLE_SPATIALLY_IMPLICIT && extent_contains(&s->local, x, y)) return 0.0;
    return s->nu;
}

/* turnover_rate/uniform.rs, turnover_rate/in_memory.rs:22-40 (a cell
 * outside the map has rate 0) */
static inline double turnover_at(const sim_t *s, uint32_t x, uint32_t y) {
    if (!s->turnover) return s->lambda;
    uint64_t cell = (uint64_t)y * s->local.w + (uint64_t)x;
    return cell < s->local.w * s->local.h ? s->turnover[cell] : 0.0;
}

/* event_time_sampler/poisson.rs:30-109, at a location with turnover rate lam */
static double poisson_next_event_time(sim_t *s, uint64_t inj, double time, uint64_t *reprime_out, double lam) {
    rng_t *g = &s->rng;
    const double lambda_dt = s->turnover ? lam * s->delta_t : s->lambda_dt;  /* poisson.rs:40 */
    const double p0 = s->turnover ? exp(-lambda_dt) : s->p0;                  /* poisson.rs:42 */
    uint64_t time_step = f64_as_u64(floor(time / s->delta_t));
    double event_time;
    uint32_t event_index;
    for (;;) {
        rng_prime(g, inj, time_step);
        uint32_t n_events;
        if (p0 > 0.0) {
            /* Devroye inversion of Poisson(lambda * delta_t) */
            uint32_t poisson = 0;
            double prod = p0;
            double acc = p0;
            double u = u01_closed_open(g);
            while (u > acc && prod > 0.0) {
                poisson += 1;
                prod *= lambda_dt / (double)poisson;
                acc += prod;
            }
            n_events = poisson;
        } else {
            /* normal approximation fallback (poisson.rs:66-75) */
            double u0 = u01_open_closed(g);
            double u1 = u01_closed_open(g);
            double r = sqrt(-2.0 * log(u0));
            double theta = -6.283185307179586 * u1;
            double z0 = r * sin(theta);
            double v = z0 * sqrt(lambda_dt) + lambda_dt;
            n_events = f64_as_u32(v > 0.0 ? v : 0.0);
        }
        int found = 0;
        double best = 0.0;
        uint32_t best_k = 0;
        for (uint32_t k = 0; k < n_events; ++k) {
            double et = ((double)time_step + u01_closed_open(g)) * s->delta_t;
            if (et > time) {
                if (!found || best > et) {
                    best = et;
                    best_k = k;
                    found = 1;
                }
            }
        }
        if (found) {
            event_time = best;
            event_index = best_k;
            break;
        }
        time_step += 1;
    }
    uint64_t reprime = time_step + INV_PHI_U64 * (uint64_t)(event_index + 1);
    rng_prime(g, inj, reprime);
    if (reprime_out) *reprime_out = reprime;
    return event_time;
}

/* event_time_sampler/exp.rs:37-83 ExpEventTimeSampler, with
 * rng.rs:163-167 sample_exponential = -ln(U(0,1]) / lambda */
static double exp_next_event_time(sim_t *s, uint64_t inj, double time, uint64_t *reprime_out, double lam) {
    rng_t *g = &s->rng;
    uint64_t time_step = f64_as_u64(floor(time / s->delta_t));
    double event_time = (double)time_step * s->delta_t;
    double time_slice_end = (double)(time_step + 1) * s->delta_t;
    uint64_t sub_index = 0;
    rng_prime(g, inj, time_step);
    for (;;) {
        event_time += -necsim_ln(u01_open_closed(g)) / lam;
        sub_index += INV_PHI_U64;
        /* the time slice is exclusive at time_slice_end */
        if (event_time >= time_slice_end) {
            time_step += 1;
            sub_index = 0;
            event_time = time_slice_end;
            time_slice_end = (double)(time_step + 1) * s->delta_t;
            rng_prime(g, inj, time_step);
        } else if (event_time > time) {
            break;
        }
    }
    uint64_t reprime = time_step + sub_index;
    rng_prime(g, inj, reprime);
    if (reprime_out) *reprime_out = reprime;
    return event_time;
}

static double next_event_time(sim_t *s, uint64_t inj, double time, uint64_t *reprime_out, double lam) {
    return s->exp_sampler ? exp_next_event_time(s, inj, time, reprime_out, lam)
                          : poisson_next_event_time(s, inj, time, reprime_out, lam);
}

/* dispersal_sampler/non_spatial.rs:42-66 */
static inline void non_spatial_disperse(rng_t *g, const extent_t *e, uint32_t *tx, uint32_t *ty) {
    uint64_t n = e->w * e->h;
    uint64_t idx = sample_index_u64(g, n);
    *tx = e->ox + (uint32_t)(idx % e->w);
    *ty = e->oy + (uint32_t)(idx / e->w);
}

/* habitat/almost_infinite.rs:100-114 clamp_round_dispersal */
static inline void clamp_round_dispersal(uint32_t x, uint32_t y, double dx, double dy,
                                         uint32_t *tx, uint32_t *ty) {
    const int64_t WRAP = (int64_t)1 << 32;
    int64_t ix = f64_as_i64(round(dx));
    int64_t iy = f64_as_i64(round(dy));
    int64_t nx = ((int64_t)x + ix) % WRAP;
    int64_t ny = ((int64_t)y + iy) % WRAP;
    *tx = (uint32_t)((nx + WRAP) % WRAP);
    *ty = (uint32_t)((ny + WRAP) % WRAP);
}

/* rng.rs:180-197 sample_2d_normal via Box-Muller; almost_infinite_normal.rs:58-68 */
static inline void normal_displacement(uint64_t d0, uint64_t d1, double sigma, double *dx, double *dy) {
    double u0 = (double)((d0 >> 11) + 1) * 0x1.0p-53;
    double u1 = (double)(d1 >> 11) * 0x1.0p-53;
    double r = sqrt(-2.0 * log(u0));
    double theta = -6.283185307179586 * u1;
    double z0 = r * sin(theta);
    double z1 = r * cos(theta);
    *dx = z0 * sigma + 0.0;
    *dy = z1 * sigma + 0.0;
}

static inline void normal_disperse_from_draws(uint64_t d0, uint64_t d1, double sigma, uint32_t x,
                                              uint32_t y, uint32_t *tx, uint32_t *ty) {
    double dx, dy;
    normal_displacement(d0, d1, sigma, &dx, &dy);
    clamp_round_dispersal(x, y, dx, dy, tx, ty);
}

/* clark2dt::cdf_inverse with pow_fast_one (almost_infinite_clark2dt.rs:167-189):
 * jump = sqrt(u * (pow(1 / (1 - u01), 1 / p) - 1)), the power skipped for an
 * exponent of exactly 1 */
static inline double clark2dt_cdf_inverse(double u01, double shape_u, double tail_p) {
    double expo = 1.0 / tail_p;
    double base = 1.0 / (1.0 - u01);
    double powed = (expo == 1.0) ? base : pow(base, expo);
    return sqrt(shape_u * (powed - 1.0));
}

double oracle_clark2dt_cdf_inverse(double u01, double shape_u, double tail_p) {
    return clark2dt_cdf_inverse(u01, shape_u, tail_p);
}

/* almost_infinite_clark2dt.rs:96-107: the jump from cdf_inverse,
 * theta = u2 * 2 * pi, (dx, dy) = (cos(theta) * jump, sin(theta) * jump) */
static inline void clark2dt_displacement(uint64_t d0, uint64_t d1, double shape_u, double tail_p, double *dx,
                                         double *dy) {
    double u01 = (double)(d0 >> 11) * 0x1.0p-53;
    double u2 = (double)((d1 >> 11) + 1) * 0x1.0p-53;
    double jump = clark2dt_cdf_inverse(u01, shape_u, tail_p);
    double theta = u2 * 2.0 * 3.141592653589793;
    *dx = cos(theta) * jump;
    *dy = sin(theta) * jump;
}

static inline void clark2dt_disperse_from_draws(uint64_t d0, uint64_t d1, double shape_u, double tail_p,
                                                uint32_t x, uint32_t y, uint32_t *tx, uint32_t *ty) {
    double dx, dy;
    clark2dt_displacement(d0, d1, shape_u, tail_p, &dx, &dy);
    clamp_round_dispersal(x, y, dx, dy, tx, ty);
}

void oracle_clark2dt_dispersal(uint64_t draw0, uint64_t draw1, double shape_u, double tail_p, uint32_t x,
                               uint32_t y, uint32_t *tx, uint32_t *ty) {
    clark2dt_disperse_from_draws(draw0, draw1, shape_u, tail_p, x, y, tx, ty);
}

void oracle_normal_dispersal(uint64_t draw0, uint64_t draw1, double sigma, uint32_t x, uint32_t y,
                             uint32_t *tx, uint32_t *ty) {
    normal_disperse_from_draws(draw0, draw1, sigma, x, y, tx, ty);
}

void oracle_displacements(int32_t kind, const uint64_t *draws, uint64_t n, double a, double b, double *dx,
                          double *dy) {
    for (uint64_t j = 0; j < n; ++j) {
        if (kind == ORACLE_ALMOST_INFINITE_CLARK2DT)
            clark2dt_displacement(draws[2 * j], draws[2 * j + 1], a, b, &dx[j], &dy[j]);
        else
            normal_displacement(draws[2 * j], draws[2 * j + 1], a, &dx[j], &dy[j]);
    }
}

/* ------------------------------------------------------------------------ */
/* WrappingNoise: OpenSimplex 2D noise with wrapping                        */
/* habitat/wrapping_noise/{mod.rs, opensimplex_noise/{mod.rs,               */
/*                         open_simplex_noise_2d.rs,utils.rs}}              */
/* ------------------------------------------------------------------------ */
#define OS_STRETCH (-0.211324865405187) /* open_simplex_noise_2d.rs:9, as written there */
#define OS_SQUISH 0.366025403784439     /* open_simplex_noise_2d.rs:10 */
#define NOISE_2_32 4294967296.0         /* (u32::MAX as f64) + 1.0 */
#define NOISE_FRAC_1_PI 0.318309886183790671537767526745028724
#define NOISE_SQRT_2 1.41421356237309504880168872420969808

/* Rust's `v as i64`: truncating, saturating, NaN -> 0 */
static inline int64_t sat_i64(double v) {
    if (v != v) return 0;
    if (v >= 9223372036854775808.0) return INT64_MAX;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)v;
}

/* opensimplex_noise/mod.rs:76-96 generate_perm_array: the i128 seed is
 * never advanced, so every swap index comes from the same value */
static void opensimplex_perm(int64_t seed, int64_t *perm) {
    int64_t source[2048];
    __int128 a = (__int128)seed * (__int128)6364136223846793005LL + (__int128)1442695040888963407LL;
    for (int64_t i = 0; i < 2048; ++i) source[i] = i;
    for (int64_t i = 2047; i >= 0; --i) {
        int64_t r = (int64_t)((a + 31) % (__int128)(i + 1)); /* C's % truncates, like Rust's */
        if (r < 0) r += i + 1;
        perm[i] = source[r];
        source[r] = source[i];
    }
}

/* open_simplex_noise_2d.rs:21-59 extrapolate: wrap the lattice point into
 * [0, wrap), then the gradient (+-5, +-2) or (+-2, +-5) from two perm reads */
static double os_extrapolate(const int64_t *perm, double gx, double gy, double dx, double dy,
                             double wrap) {
    gx = floor(gx - floor(gx / wrap) * wrap);
    gy = floor(gy - floor(gy / wrap) * wrap);
    /* i64 arithmetic (wrapping), masked to the low byte */
    uint64_t i0 = ((uint64_t)perm[(uint64_t)sat_i64(gx) & 0xFF] + (uint64_t)sat_i64(gy)) & 0xFF;
    uint64_t idx = ((uint64_t)perm[i0] & 0x0E) >> 1;
    double px = (idx & 1) == 0 ? 5.0 : 2.0;
    double py = (idx & 1) == 0 ? 2.0 : 5.0;
    if (idx & 2) px *= -1.0;
    if (idx & 4) py *= -1.0;
    return px * dx + py * dy;
}

/* opensimplex_noise/utils.rs:5-23 contribute */
static double os_contribute(const int64_t *perm, double dx, double dy, double ox, double oy, double gx,
                            double gy, double wrap) {
    double ds = dx + dy;
    double sx = (ox - dx) - OS_SQUISH * ds;
    double sy = (oy - dy) - OS_SQUISH * ds;
    double attn = 2.0 - (sx * sx + sy * sy);
    if (attn <= 0.0) return 0.0;
    double a2 = attn * attn;
    double a4 = a2 * a2;
    return a4 * os_extrapolate(perm, gx + dx, gy + dy, sx, sy, wrap);
}

/* open_simplex_noise_2d.rs:61-128 eval, get_value, evaluate_inside_triangle */
static double os_eval(const int64_t *perm, double x, double y, double wrap) {
    double s = x + y;
    double ix = x + OS_SQUISH * s, iy = y + OS_SQUISH * s; /* pre-squished input */
    double s2 = ix + iy;
    double stx = ix + OS_STRETCH * s2, sty = iy + OS_STRETCH * s2;
    double gx = floor(stx), gy = floor(sty);
    double gs = gx + gy;
    double sqx = gx + OS_SQUISH * gs, sqy = gy + OS_SQUISH * gs;
    double insx = stx - gx, insy = sty - gy;
    double ox = ix - sqx, oy = iy - sqy;
    double value = os_contribute(perm, 1.0, 0.0, ox, oy, gx, gy, wrap) +
                   os_contribute(perm, 0.0, 1.0, ox, oy, gx, gy, wrap);
    double in_sum = insx + insy;
    double f = in_sum <= 1.0 ? 0.0 : 1.0;
    double z = 1.0 + f - in_sum;
    double px, py;
    if (z > insx || z > insy) {
        if (insx > insy) {
            px = 1.0 + f;
            py = -1.0 + f;
        } else {
            px = -1.0 + f;
            py = 1.0 + f;
        }
    } else {
        px = 1.0 - f;
        py = 1.0 - f;
    }
    double tri = os_contribute(perm, 0.0 + f, 0.0 + f, ox, oy, gx, gy, wrap) +
                 os_contribute(perm, px, py, ox, oy, gx, gy, wrap);
    return (value + tri) / 47.0;
}

/* habitat/wrapping_noise/mod.rs:216-249 sum_noise_octaves */
static double noise_sum(const int64_t *perm, double persistence, double scale, uint64_t octaves, uint32_t x,
                        uint32_t y) {
    double max_amplitude = 0.0, amplitude = 1.0;
    double frequency = scale * NOISE_FRAC_1_PI * 3.0;
    double result = 0.0;
    for (uint64_t o = 0; o < octaves; ++o) {
        double wrap = round(NOISE_2_32 * frequency);
        double fixed = wrap / NOISE_2_32;
        result += os_eval(perm, (double)x * fixed, (double)y * fixed, wrap) * amplitude;
        max_amplitude += amplitude;
        amplitude *= persistence;
        frequency *= 2.0;
    }
    return result / max_amplitude;
}

static double noise_octaves(const sim_t *s, uint32_t x, uint32_t y) {
    return noise_sum(s->perm, s->persistence, s->scale, s->octaves, x, y);
}

/* f64::total_cmp */
static int total_cmp(const void *pa, const void *pb) {
    int64_t a, b;
    memcpy(&a, pa, 8);
    memcpy(&b, pb, 8);
    a ^= (int64_t)((uint64_t)(a >> 63) >> 1);
    b ^= (int64_t)((uint64_t)(b >> 63) >> 1);
    return a < b ? -1 : (a > b ? 1 : 0);
}

/* habitat/wrapping_noise/mod.rs:47-99: the noise at 2^16 locations drawn by
 * WyHash::from_seed(seed.to_le_bytes()), sorted, read at the coverage */
static int noise_threshold(const int64_t *perm, int64_t seed, double coverage, double scale, double persistence,
                           uint64_t octaves, double *out) {
    enum { N = 1 << 16 };
    double *samples = (double *)malloc(N * sizeof(double));
    if (!samples) return -1;
    rng_t g = {(uint64_t)seed, (uint64_t)seed, 0, 0};
    for (int j = 0; j < N; ++j) {
        uint64_t loc = rng_sample_u64(&g);
        samples[j] = noise_sum(perm, persistence, scale, octaves, (uint32_t)loc, (uint32_t)(loc >> 32));
    }
    qsort(samples, N, sizeof(double), total_cmp);
    double k = floor((double)N * coverage);
    uint64_t at = k >= (double)(N - 1) ? (uint64_t)(N - 1) : (uint64_t)k;
    *out = samples[at];
    free(samples);
    return 0;
}

/* dispersal_sampler/wrapping_noise.rs:89-110 with almost_infinite_normal.rs:22-37:
 * ps = erf(0.5 / (sigma * sqrt 2))^2 (libm's erf; the C library's here),
 * self-dispersal ps / (ps + (1 - ps) * coverage) */
static double noise_self_dispersal(double sigma, double coverage) {
    double p1 = sigma > 0.0 ? erf(0.5 / (sigma * NOISE_SQRT_2)) : 1.0;
    double ps = p1 * p1;
    double pout = (1.0 - ps) * coverage;
    return ps / (ps + pout);
}

double oracle_wrapping_noise(int64_t seed, double scale, double persistence, uint64_t octaves, uint32_t x,
                             uint32_t y) {
    int64_t perm[2048];
    opensimplex_perm(seed, perm);
    return noise_sum(perm, persistence, scale, octaves, x, y);
}

double oracle_wrapping_noise_threshold(int64_t seed, double coverage, double scale, double persistence,
                                       uint64_t octaves) {
    int64_t perm[2048];
    double t = NAN;
    opensimplex_perm(seed, perm);
    if (noise_threshold(perm, seed, coverage, scale, persistence, octaves, &t)) return NAN;
    return t;
}

double oracle_wrapping_noise_self_dispersal(double sigma, double coverage) {
    return noise_self_dispersal(sigma, coverage);
}

/* alias/packed.rs:135-163 sample_event_with_cdf_limit (limit = 1) */
static inline uint32_t alias_sample(const alias_t *a, uint64_t start, uint64_t end, rng_t *g) {
    uint64_t len = end - start;
    double f = u01_closed_open(g) * 1.0 * (double)len;
    uint64_t i = f64_as_u64(floor(f));
    double y = f - (double)i;
    uint64_t at = start + i;
    return (y < a->atom_u[at]) ? a->atom_e[at] : a->atom_k[at];
}

/* packed_separable_alias/dispersal.rs:16-77 */
static inline void spatially_explicit_disperse(const sim_t *s, rng_t *g, uint32_t x, uint32_t y,
                                               uint32_t *tx, uint32_t *ty) {
    const alias_t *a = &s->alias;
    uint64_t w = s->local.w;
    uint64_t cell = (uint64_t)(y - s->local.oy) * w + (uint64_t)(x - s->local.ox);
    double sd = a->self_dispersal[cell];
    uint64_t target;
    if (sd == 1.0) {
        target = cell;
    } else if (sd == 0.0 || a->non_self_event[cell] != cell || u01_closed_open(g) >= sd) {
        target = alias_sample(a, a->range_start[cell], a->range_end[cell], g);
    } else {
        target = cell;
    }
    *tx = s->local.ox + (uint32_t)(target % w);
    *ty = s->local.oy + (uint32_t)(target / w);
}

static inline void disperse(sim_t *s, uint32_t x, uint32_t y, uint32_t *tx, uint32_t *ty) {
    rng_t *g = &s->rng;
    switch (s->kind) {
    case ORACLE_NON_SPATIAL:
        non_spatial_disperse(g, &s->local, tx, ty);
        break;
    case ORACLE_SPATIALLY_IMPLICIT:
        /* dispersal_sampler/spatially_implicit.rs:58-86 */
        if (extent_contains(&s->local, x, y)) {
            if (u01_closed_open(g) < s->migration)
                non_spatial_disperse(g, &s->meta, tx, ty);
            else
                non_spatial_disperse(g, &s->local, tx, ty);
        } else {
            non_spatial_disperse(g, &s->meta, tx, ty);
        }
        break;
    case ORACLE_ALMOST_INFINITE_NORMAL: {
        uint64_t d0 = rng_sample_u64(g);
        uint64_t d1 = rng_sample_u64(g);
        if (s->clark)
            clark2dt_disperse_from_draws(d0, d1, s->shape_u, s->tail_p, x, y, tx, ty);
        else
            normal_disperse_from_draws(d0, d1, s->sigma, x, y, tx, ty);
        break;
    }
    case ORACLE_WRAPPING_NOISE:
        /* dispersal_sampler/wrapping_noise.rs:42-87: sample_event(p_self)
         * (rng.rs:97-102), else Normal draws until the target is habitable
         * and not the origin (bounded here, unbounded in the reference) */
        if (u01_closed_open(g) < s->p_self) {
            *tx = x;
            *ty = y;
            break;
        }
        for (uint32_t k = 0;; ++k) {
            if (k == ORACLE_MAX_DISPERSAL_REJECTIONS) {
                s->fault = -6;
                *tx = x;
                *ty = y;
                break;
            }
            uint64_t d0 = rng_sample_u64(g);
            uint64_t d1 = rng_sample_u64(g);
            normal_disperse_from_draws(d0, d1, s->sigma, x, y, tx, ty);
            if (habitat_at(s, *tx, *ty) != 0 && !(*tx == x && *ty == y)) break;
        }
        break;
    default:
        spatially_explicit_disperse(s, g, x, y, tx, ty);
        break;
    }
}

/* coalescence_sampler.rs:59-78 (+ independent.rs:59-76 singleton demes) */
static inline uint32_t coalescence_index(sim_t *s, uint32_t tx, uint32_t ty) {
    double u = u01_closed_open(&s->rng);
    if (s->kind == ORACLE_ALMOST_INFINITE_NORMAL) return 0;
    return f64_as_u32(floor(u * (double)habitat_at(s, tx, ty)));
}

/* ------------------------------------------------------------------------ */
/* Packed separable alias builder                                            */
/* packed_separable_alias/mod.rs:64-203, alias/packed.rs:59-121              */
/* ------------------------------------------------------------------------ */
typedef struct weight_t {
    uint64_t event;
    double w;
} weight_t;

/* alias/packed.rs:59-121 AliasMethodSamplerAtom::create */
static void alias_create(const weight_t *ew, uint64_t n, double *u, uint32_t *e, uint32_t *k,
                         uint64_t *over, uint64_t *under) {
    double total = 0.0;
    for (uint64_t i = 0; i < n; ++i) total = total + ew[i].w;
    double nf = (double)n;
    for (uint64_t i = 0; i < n; ++i) {
        u[i] = ew[i].w * nf / total;
        e[i] = (uint32_t)ew[i].event;
        k[i] = (uint32_t)ew[i].event;
    }
    uint64_t n_over = 0, n_under = 0;
    for (uint64_t i = 0; i < n; ++i)
        if (u[i] > 1.0) over[n_over++] = i;
    for (uint64_t i = 0; i < n; ++i)
        if (u[i] < 1.0) under[n_under++] = i;
    while (n_over > 0 && n_under > 0) {
        uint64_t o = over[--n_over];
        uint64_t un = under[--n_under];
        u[o] = u[o] + u[un] - 1.0;
        k[un] = e[o];
        if (u[o] < 1.0)
            under[n_under++] = o;
        else if (u[o] > 1.0)
            over[n_over++] = o;
    }
    for (uint64_t i = 0; i < n_over; ++i) u[over[i]] = 1.0;
    for (uint64_t i = 0; i < n_under; ++i) u[under[i]] = 1.0;
}

int oracle_check_dispersal_contract(const oracle_scenario *sc) {
    /* dispersal_sampler/in_memory/contract.rs:13-69 */
    uint64_t w = sc->width, h = sc->height, n = w * h;
    for (uint64_t row = 0; row < n; ++row) {
        const double *r = sc->dispersal + row * n;
        if (sc->habitat[row] > 0) {
            int any = 0;
            for (uint64_t c = 0; c < n; ++c) {
                if (r[c] > 0.0) {
                    if (sc->habitat[c] == 0) return 2;
                    any = 1;
                }
            }
            if (!any) return 3;
        } else {
            for (uint64_t c = 0; c < n; ++c)
                if (r[c] != 0.0) return 4;
        }
    }
    return 0;
}

static int build_alias(const oracle_scenario *sc, alias_t *a) {
    uint64_t w = sc->width, h = sc->height, n = w * h;
    memset(a, 0, sizeof(*a));
    a->n_cells = n;
    a->range_start = (uint64_t *)calloc(n, sizeof(uint64_t));
    a->range_end = (uint64_t *)calloc(n, sizeof(uint64_t));
    a->self_dispersal = (double *)calloc(n, sizeof(double));
    a->non_self_event = (uint64_t *)calloc(n, sizeof(uint64_t));
    weight_t *ew = (weight_t *)malloc(n * sizeof(weight_t));
    uint64_t *over = (uint64_t *)malloc(n * sizeof(uint64_t));
    uint64_t *under = (uint64_t *)malloc(n * sizeof(uint64_t));
    if (!a->range_start || !a->range_end || !a->self_dispersal || !a->non_self_event || !ew ||
        !over || !under)
        return -1;
    /* first pass: count atoms per row to size the buffer exactly */
    uint64_t total_atoms = 0;
    for (uint64_t row = 0; row < n; ++row) {
        const double *r = sc->dispersal + row * n;
        uint64_t cnt = 0;
        for (uint64_t c = 0; c < n; ++c)
            if (r[c] * (double)sc->habitat[c] > 0.0) cnt++;
        total_atoms += cnt;
    }
    a->atom_u = (double *)malloc((total_atoms ? total_atoms : 1) * sizeof(double));
    a->atom_e = (uint32_t *)malloc((total_atoms ? total_atoms : 1) * sizeof(uint32_t));
    a->atom_k = (uint32_t *)malloc((total_atoms ? total_atoms : 1) * sizeof(uint32_t));
    if (!a->atom_u || !a->atom_e || !a->atom_k) return -1;

    uint64_t len = 0;
    for (uint64_t row = 0; row < n; ++row) {
        /* default: no self-dispersal, non_self_dispersal_event = own index */
        a->self_dispersal[row] = 0.0;
        a->non_self_event[row] = row;
        const double *r = sc->dispersal + row * n;
        uint64_t n_ew = 0;
        double self_w = 0.0;
        for (uint64_t c = 0; c < n; ++c) {
            /* weight = p * habitat(target) (mod.rs:95-97) */
            double weight = r[c] * (double)sc->habitat[c];
            if (weight > 0.0) {
                ew[n_ew].event = c;
                ew[n_ew].w = weight;
                n_ew++;
                if (c == row) self_w = weight;
            }
        }
        uint64_t from = len;
        if (n_ew == 0) {
            a->range_start[row] = from;
            a->range_end[row] = from;
            continue;
        }
        double total = 0.0;
        for (uint64_t i = 0; i < n_ew; ++i) total = total + ew[i].w;
        double sd_prob = self_w / total;
        double sd_u = self_w * (double)n_ew / total;
        uint64_t non_self = row;
        double *u = a->atom_u + from;
        uint32_t *e = a->atom_e + from;
        uint32_t *k = a->atom_k + from;
        uint64_t n_atoms;
        if (sd_u < 1.0) {
            alias_create(ew, n_ew, u, e, k, over, under);
            n_atoms = n_ew;
            for (uint64_t i = 0; i < n_atoms; ++i) {
                if (e[i] == (uint32_t)row || k[i] == (uint32_t)row) {
                    if (e[i] == (uint32_t)row) {
                        /* flip(): swap e/k, u = 1 - u */
                        uint32_t t = e[i];
                        e[i] = k[i];
                        k[i] = t;
                        u[i] = 1.0 - u[i];
                    }
                    non_self = e[i];
                    uint64_t last = n_atoms - 1;
                    double tu = u[i];
                    uint32_t te = e[i], tk = k[i];
                    u[i] = u[last];
                    e[i] = e[last];
                    k[i] = k[last];
                    u[last] = tu;
                    e[last] = te;
                    k[last] = tk;
                    break;
                }
            }
        } else {
            /* retain: drop self-dispersal from the alias sampler */
            uint64_t m = 0;
            for (uint64_t i = 0; i < n_ew; ++i)
                if (ew[i].event != row) ew[m++] = ew[i];
            alias_create(ew, m, u, e, k, over, under);
            n_atoms = m;
        }
        a->self_dispersal[row] = sd_prob;
        a->non_self_event[row] = non_self;
        len += n_atoms;
        a->range_start[row] = from;
        a->range_end[row] = len;
    }
    a->n_atoms = len;
    free(ew);
    free(over);
    free(under);
    return 0;
}

static void free_alias(alias_t *a) {
    free(a->range_start);
    free(a->range_end);
    free(a->self_dispersal);
    free(a->non_self_event);
    free(a->atom_u);
    free(a->atom_e);
    free(a->atom_k);
    memset(a, 0, sizeof(*a));
}

int oracle_build_alias(const oracle_scenario *sc, oracle_alias_tables *out) {
    alias_t a;
    int rc = build_alias(sc, &a);
    if (rc) {
        free_alias(&a);
        return rc;
    }
    out->n_cells = a.n_cells;
    out->n_atoms = a.n_atoms;
    out->range_start = a.range_start;
    out->range_end = a.range_end;
    out->self_dispersal = a.self_dispersal;
    out->non_self_event = a.non_self_event;
    out->atom_u = a.atom_u;
    out->atom_e = a.atom_e;
    out->atom_k = a.atom_k;
    return 0;
}

void oracle_free_alias(oracle_alias_tables *t) {
    free(t->range_start);
    free(t->range_end);
    free(t->self_dispersal);
    free(t->non_self_event);
    free(t->atom_u);
    free(t->atom_e);
    free(t->atom_k);
    memset(t, 0, sizeof(*t));
}

/* ------------------------------------------------------------------------ */
/* Scenario set-up                                                           */
/* ------------------------------------------------------------------------ */
static int sim_init(sim_t *s, const oracle_scenario *sc, const oracle_args *args, uint64_t seed) {
    memset(s, 0, sizeof(*s));
    s->kind = sc->kind;
    s->nu = sc->speciation_probability;
    s->lambda = sc->turnover_rate;
    s->delta_t = args->delta_t;
    s->lambda_dt = s->lambda * s->delta_t;
    s->p0 = exp(-s->lambda_dt);
    s->exp_sampler = args->event_time_sampler == ORACLE_SAMPLER_EXP;
    if (args->event_time_sampler != ORACLE_SAMPLER_POISSON && !s->exp_sampler) return -2;
    s->migration = sc->migration_probability;
    s->sigma = sc->sigma;
    if (sc->kind == ORACLE_ALMOST_INFINITE_CLARK2DT) {
        /* the same habitat, origins and coalescence as AlmostInfinite Normal */
        s->kind = ORACLE_ALMOST_INFINITE_NORMAL;
        s->clark = 1;
        s->shape_u = sc->shape_u;
        s->tail_p = sc->tail_p;
        if (!(sc->shape_u > 0.0) || !(sc->tail_p > 0.0)) return -2;
    }
    s->rng.seed = oracle_seed_from_u64(seed);
    s->rng.state = s->rng.seed;
    if (sc->turnover) {
        /* turnover/map.rs: SpatiallyExplicit only; rates >= 0 (maps/mod.rs:34-53),
         * > 0 on habitable cells (turnover_rate/in_memory.rs:50-72); the canonical
         * rounds advance at the largest habitable rate */
        if (sc->kind != ORACLE_SPATIALLY_EXPLICIT || !sc->habitat) return -2;
        uint64_t cells = (uint64_t)sc->width * sc->height;
        double top = 0.0;
        for (uint64_t c = 0; c < cells; ++c) {
            double t = sc->turnover[c];
            if (!(t >= 0.0) || !isfinite(t)) return -2;
            if (t == 0.0 && sc->habitat[c] != 0) return -2;
            if (sc->habitat[c] != 0 && t > top) top = t;
        }
        s->turnover = sc->turnover;
        s->lambda = top;
        s->lambda_dt = s->lambda * s->delta_t;
        s->p0 = exp(-s->lambda_dt);
    }
    if (!(s->lambda > 0.0) || !(s->delta_t > 0.0)) return -2;
    switch (sc->kind) {
    case ORACLE_NON_SPATIAL:
        if (!sc->width || !sc->height || !sc->deme) return -2;
        s->local = (extent_t){0, 0, sc->width, sc->height};
        s->deme = sc->deme;
        break;
    case ORACLE_SPATIALLY_IMPLICIT:
        if (!sc->width || !sc->height || !sc->deme || !sc->meta_width || !sc->meta_height ||
            !sc->meta_deme)
            return -2;
        s->local = (extent_t){0, 0, sc->width, sc->height};
        s->deme = sc->deme;
        /* habitat/spatially_implicit.rs:45-49: meta offset = (inv(w), inv(h)) */
        s->meta = (extent_t){UINT32_MAX - (sc->meta_width - 1), UINT32_MAX - (sc->meta_height - 1),
                             sc->meta_width, sc->meta_height};
        s->meta_deme = sc->meta_deme;
        break;
    case ORACLE_ALMOST_INFINITE_NORMAL:
    case ORACLE_ALMOST_INFINITE_CLARK2DT:
        s->local = (extent_t){0, 0, 1ULL << 32, 1ULL << 32};
        break;
    case ORACLE_WRAPPING_NOISE:
        /* WrappingNoiseArguments (wrapping_noise.rs:39-48): coverage in [0, 1],
         * scale and persistence in (0, 1], octaves >= 1, sigma >= 0 */
        if (!(sc->coverage >= 0.0 && sc->coverage <= 1.0) || !(sc->scale > 0.0 && sc->scale <= 1.0) ||
            !(sc->persistence > 0.0 && sc->persistence <= 1.0) || sc->octaves == 0 ||
            !(sc->sigma >= 0.0) || !isfinite(sc->sigma) || sc->sample_width == 0 || sc->sample_height == 0 ||
            sc->sample_width > (1ULL << 32) || sc->sample_height > (1ULL << 32))
            return -2;
        s->local = (extent_t){0, 0, 1ULL << 32, 1ULL << 32};
        s->coverage = sc->coverage;
        s->scale = sc->scale;
        s->persistence = sc->persistence;
        s->octaves = sc->octaves;
        opensimplex_perm(sc->noise_seed, s->perm);
        if (noise_threshold(s->perm, sc->noise_seed, sc->coverage, sc->scale, sc->persistence, sc->octaves,
                            &s->threshold))
            return -1;
        s->p_self = noise_self_dispersal(sc->sigma, sc->coverage);
        break;
    case ORACLE_SPATIALLY_EXPLICIT: {
        if (!sc->width || !sc->height || !sc->habitat || !sc->dispersal) return -2;
        s->local = (extent_t){0, 0, sc->width, sc->height};
        s->habitat = sc->habitat;
        uint64_t n = (uint64_t)sc->width * sc->height;
        s->injection = (uint64_t *)malloc((n + 1) * sizeof(uint64_t));
        if (!s->injection) return -1;
        /* habitat/in_memory.rs:143-163 prefix sums */
        uint64_t acc = 0;
        for (uint64_t c = 0; c < n; ++c) {
            s->injection[c] = acc;
            acc += sc->habitat[c];
        }
        s->injection[n] = acc;
        if (acc == 0) return -3;
        if (oracle_check_dispersal_contract(sc)) return -4;
        if (build_alias(sc, &s->alias)) return -1;
        break;
    }
    default:
        return -2;
    }
    return 0;
}

static void sim_free(sim_t *s) {
    free(s->injection);
    free_alias(&s->alias);
}

/* ------------------------------------------------------------------------ */
/* Origin enumeration (100% sample)                                          */
/* origin_sampler/{non_spatial,in_memory,spatially_implicit,                 */
/*                 singleton_demes/circle}.rs, landscape/extent.rs:80-100    */
/* ------------------------------------------------------------------------ */
typedef struct lineage_t {
    uint64_t gref;
    double last;
    uint32_t x, y, i;
} lineage_t;

static int64_t enumerate_origins(const oracle_scenario *sc, const sim_t *s, lineage_t *out,
                                 uint64_t cap) {
    uint64_t n = 0;
    switch (sc->kind) {
    case ORACLE_NON_SPATIAL:
    case ORACLE_SPATIALLY_IMPLICIT:
        /* row-major over the (local) extent, x fastest, then deme index */
        for (uint64_t y = 0; y < sc->height; ++y)
            for (uint64_t x = 0; x < sc->width; ++x)
                for (uint32_t i = 0; i < sc->deme; ++i) {
                    if (out && n < cap) {
                        out[n].x = (uint32_t)x;
                        out[n].y = (uint32_t)y;
                        out[n].i = i;
                        out[n].last = 0.0;
                        out[n].gref = injection(s, (uint32_t)x, (uint32_t)y, i);
                    }
                    n++;
                }
        break;
    case ORACLE_ALMOST_INFINITE_NORMAL:
    case ORACLE_ALMOST_INFINITE_CLARK2DT: {
        if (sc->sample_width) {
            /* almost_infinite/mod.rs:98, 118-120: the Rectangle sample,
             * singleton_demes/rectangle.rs:93-120 (every location habitable) */
            for (uint64_t yy = 0; yy < sc->sample_height; ++yy)
                for (uint64_t xx = 0; xx < sc->sample_width; ++xx) {
                    uint32_t x = sc->sample_x + (uint32_t)xx, y = sc->sample_y + (uint32_t)yy;
                    if (out && n < cap) {
                        out[n].x = x;
                        out[n].y = y;
                        out[n].i = 0;
                        out[n].last = 0.0;
                        out[n].gref = ((uint64_t)y << 32) | x;
                    }
                    n++;
                }
            break;
        }
        /* singleton_demes/circle.rs:36-70, 100-140 */
        uint32_t r = sc->radius;
        uint64_t d = (uint64_t)r * 2 + 1;
        uint32_t ox = sc->centre_x - r, oy = sc->centre_y - r;
        uint64_t r2 = (uint64_t)r * r;
        for (uint64_t yy = 0; yy < d; ++yy)
            for (uint64_t xx = 0; xx < d; ++xx) {
                uint32_t x = ox + (uint32_t)xx, y = oy + (uint32_t)yy;
                uint32_t dx1 = x - sc->centre_x, dx2 = sc->centre_x - x;
                uint32_t dy1 = y - sc->centre_y, dy2 = sc->centre_y - y;
                uint64_t dx = dx1 < dx2 ? dx1 : dx2;
                uint64_t dy = dy1 < dy2 ? dy1 : dy2;
                if (dx * dx + dy * dy <= r2) {
                    if (out && n < cap) {
                        out[n].x = x;
                        out[n].y = y;
                        out[n].i = 0;
                        out[n].last = 0.0;
                        out[n].gref = ((uint64_t)y << 32) | x;
                    }
                    n++;
                }
            }
        break;
    }
    case ORACLE_WRAPPING_NOISE:
        /* singleton_demes/rectangle.rs:93-120: the habitable locations of the
         * sample extent in its row-major order (extent.rs:80-100, wrapping) */
        for (uint64_t yy = 0; yy < sc->sample_height; ++yy)
            for (uint64_t xx = 0; xx < sc->sample_width; ++xx) {
                uint32_t x = sc->sample_x + (uint32_t)xx, y = sc->sample_y + (uint32_t)yy;
                if (habitat_at(s, x, y) == 0) continue;
                if (out && n < cap) {
                    out[n].x = x;
                    out[n].y = y;
                    out[n].i = 0;
                    out[n].last = 0.0;
                    out[n].gref = ((uint64_t)y << 32) | x;
                }
                n++;
            }
        break;
    default:
        for (uint64_t y = 0; y < sc->height; ++y)
            for (uint64_t x = 0; x < sc->width; ++x) {
                uint32_t hcap = sc->habitat[y * sc->width + x];
                for (uint32_t i = 0; i < hcap; ++i) {
                    if (out && n < cap) {
                        out[n].x = (uint32_t)x;
                        out[n].y = (uint32_t)y;
                        out[n].i = i;
                        out[n].last = 0.0;
                        out[n].gref = s->injection[y * sc->width + x] + i;
                    }
                    n++;
                }
            }
        break;
    }
    return (int64_t)n;
}

int64_t oracle_count_origins(const oracle_scenario *sc) {
    oracle_args a = {2.0, 10, 1.0, 2.0, 0, 0, 0, 0, 1, 0, 0, 0};
    sim_t s;
    oracle_scenario tmp = *sc;
    int rc;
    if (sc->kind == ORACLE_SPATIALLY_EXPLICIT) {
        uint64_t n = 0;
        for (uint64_t c = 0; c < (uint64_t)sc->width * sc->height; ++c) n += sc->habitat[c];
        return (int64_t)n;
    }
    rc = sim_init(&s, &tmp, &a, 0);
    if (rc) return rc;
    int64_t n = enumerate_origins(sc, &s, NULL, 0);
    sim_free(&s);
    return n;
}

int64_t oracle_enumerate_origins(const oracle_scenario *sc, oracle_lineage *out, uint64_t cap) {
    oracle_args a = {2.0, 10, 1.0, 2.0, 0, 0, 0, 0, 1, 0, 0, 0};
    sim_t s;
    int rc;
    if (sc->kind == ORACLE_SPATIALLY_EXPLICIT) {
        /* the injection table is enough; skip the alias build */
        memset(&s, 0, sizeof(s));
        s.kind = sc->kind;
        s.local = (extent_t){0, 0, sc->width, sc->height};
        s.habitat = sc->habitat;
        uint64_t n = (uint64_t)sc->width * sc->height;
        s.injection = (uint64_t *)malloc((n + 1) * sizeof(uint64_t));
        uint64_t acc = 0;
        for (uint64_t c = 0; c < n; ++c) {
            s.injection[c] = acc;
            acc += sc->habitat[c];
        }
        s.injection[n] = acc;
    } else {
        rc = sim_init(&s, sc, &a, 0);
        if (rc) return rc;
    }
    lineage_t *tmp = (lineage_t *)malloc((cap ? cap : 1) * sizeof(lineage_t));
    int64_t n = enumerate_origins(sc, &s, tmp, cap);
    for (uint64_t j = 0; j < cap && (int64_t)j < n; ++j) {
        out[j].gref = tmp[j].gref;
        out[j].last_event_time = tmp[j].last;
        out[j].x = tmp[j].x;
        out[j].y = tmp[j].y;
        out[j].index = tmp[j].i;
        out[j].pad = 0;
    }
    free(tmp);
    sim_free(&s);
    return n;
}

/* ------------------------------------------------------------------------ */
/* Events, ordering and reporters                                            */
/* ------------------------------------------------------------------------ */
typedef struct event_t {
    uint64_t gref;
    double prior;
    double time;
    uint32_t x, y, i;
    uint32_t tx, ty, ti;
    int speciation;
} event_t;

typedef struct evbuf_t {
    event_t *v;
    uint64_t n, cap;
} evbuf_t;

static int evbuf_push(evbuf_t *b, const event_t *e) {
    if (b->n == b->cap) {
        uint64_t nc = b->cap ? b->cap * 2 : 1024;
        event_t *nv = (event_t *)realloc(b->v, nc * sizeof(event_t));
        if (!nv) return -1;
        b->v = nv;
        b->cap = nc;
    }
    b->v[b->n++] = *e;
    return 0;
}

static inline int cmp_u64(uint64_t a, uint64_t b) { return a < b ? -1 : (a > b ? 1 : 0); }
static inline int cmp_u32(uint32_t a, uint32_t b) { return a < b ? -1 : (a > b ? 1 : 0); }

/* event.rs:256-280 PackedEvent::cmp: (event_time, origin, target,
 * prior_time, global_lineage_reference); times are non-negative so their
 * bit patterns order like total_cmp */
static int event_cmp(const void *pa, const void *pb) {
    const event_t *a = (const event_t *)pa, *b = (const event_t *)pb;
    int c;
    if ((c = cmp_u64(f64_bits(a->time), f64_bits(b->time)))) return c;
    if ((c = cmp_u32(a->x, b->x))) return c;
    if ((c = cmp_u32(a->y, b->y))) return c;
    if ((c = cmp_u32(a->i, b->i))) return c;
    if ((c = cmp_u32(a->tx, b->tx))) return c;
    if ((c = cmp_u32(a->ty, b->ty))) return c;
    if ((c = cmp_u32(a->ti, b->ti))) return c;
    if ((c = cmp_u64(f64_bits(a->prior), f64_bits(b->prior)))) return c;
    return cmp_u64(a->gref, b->gref);
}

typedef struct sink_t {
    oracle_result *out;
    oracle_speciation_event *spec;
    uint64_t spec_cap;
    oracle_dispersal_event *disp;
    uint64_t disp_cap;
    int has_last;
    event_t last;   /* BiodiversityReporter::last_event */
} sink_t;

/* the downstream reporters: BiodiversityReporter (plugins/common/src/
 * biodiversity.rs:32-45) + event capture */
static void deliver(sink_t *k, const event_t *e) {
    if (e->speciation) {
        uint64_t j = k->out->n_speciation++;
        if (k->spec && j < k->spec_cap) {
            k->spec[j].gref = e->gref;
            k->spec[j].prior_time = e->prior;
            k->spec[j].event_time = e->time;
            k->spec[j].x = e->x;
            k->spec[j].y = e->y;
            k->spec[j].index = e->i;
            k->spec[j].pad = 0;
        }
        /* SpeciationEvent equality: origin and event_time (event.rs:299-307) */
        if (k->has_last && k->last.x == e->x && k->last.y == e->y && k->last.i == e->i &&
            k->last.time == e->time)
            return;
        k->last = *e;
        k->has_last = 1;
        k->out->biodiversity++;
    } else {
        uint64_t j = k->out->n_dispersal++;
        if (k->disp && j < k->disp_cap) {
            oracle_dispersal_event *d = &k->disp[j];
            d->gref = e->gref;
            d->prior_time = e->prior;
            d->event_time = e->time;
            d->x = e->x;
            d->y = e->y;
            d->index = e->i;
            d->tx = e->tx;
            d->ty = e->ty;
            d->tindex = e->ti;
            d->pad = 0;
            d->pad2 = 0;
        }
    }
}

static void flush_sorted(sink_t *k, evbuf_t *b) {
    qsort(b->v, b->n, sizeof(event_t), event_cmp);
    for (uint64_t j = 0; j < b->n; ++j) deliver(k, &b->v[j]);
    b->n = 0;
}

/* ------------------------------------------------------------------------ */
/* One lineage slice: Simulation::simulate_incremental_early_stop            */
/* (core/src/simulation/mod.rs:53-134, process/local.rs:33-105,              */
/*  independent/sampler.rs:69-116, event_sampler/independent.rs:112-222)     */
/* ------------------------------------------------------------------------ */
typedef struct spec_sample_t {   /* event_sampler/tracking.rs:29-56 */
    double u;
    double t;
    uint32_t x, y, i;
} spec_sample_t;

typedef struct slice_out_t {
    uint64_t steps;
    int alive;            /* 0 if the lineage speciated */
    int peeked;           /* early_peek_stop was called at least once */
    double next;          /* last peeked next event time */
    double new_time;      /* active_lineage_sampler.get_last_event_time() */
    int has_sample;
    spec_sample_t sample; /* min speciation sample over the slice */
} slice_out_t;

/* Called with a live lineage; `report` receives events with
 * `event_time < water` to `slow` else `fast` (live.rs:48-62). */
static int run_slice(sim_t *s, lineage_t *lin, double min_event_time, uint64_t step_slice,
                     double level, int report_dispersal, evbuf_t *slow, evbuf_t *fast,
                     double water, slice_out_t *o) {
    o->steps = 0;
    o->alive = 1;
    o->peeked = 0;
    o->has_sample = 0;
    o->new_time = lin->last > min_event_time ? lin->last : min_event_time;
    for (;;) {
        double before = lin->last > min_event_time ? lin->last : min_event_time;
        uint64_t inj = injection(s, lin->x, lin->y, lin->i);
        rng_t saved = s->rng;
        double t = next_event_time(s, inj, before, NULL, turnover_at(s, lin->x, lin->y));
        double next = max_after(before, t);
        o->peeked = 1;
        o->next = next;
        if (o->steps >= step_slice || next >= level) {
            /* early stop: restore the RNG (simulation/mod.rs:111-115) */
            uint64_t np = s->rng.n_primes, nd = s->rng.n_draws;
            s->rng = saved;
            s->rng.n_primes = np;
            s->rng.n_draws = nd;
            return 0;
        }
        o->new_time = next;
        /* speciation sample + min tracking */
        double us = u01_closed_open(&s->rng);
        if (!o->has_sample || !(o->sample.u <= us)) {
            o->sample.u = us;
            o->sample.t = next;
            o->sample.x = lin->x;
            o->sample.y = lin->y;
            o->sample.i = lin->i;
            o->has_sample = 1;
        }
        o->steps++;
        if (us < speciation_probability(s, lin->x, lin->y)) {
            event_t e = {lin->gref, lin->last, next, lin->x, lin->y, lin->i,
                         lin->x, lin->y, lin->i, 1};
            if (evbuf_push(next < water ? slow : fast, &e)) return -1;
            o->alive = 0;
            return 0;
        }
        uint32_t tx, ty;
        disperse(s, lin->x, lin->y, &tx, &ty);
        if (s->fault) return s->fault;
        uint32_t ti = coalescence_index(s, tx, ty);
        if (report_dispersal) {
            event_t e = {lin->gref, lin->last, next, lin->x, lin->y, lin->i, tx, ty, ti, 0};
            if (evbuf_push(next < water ? slow : fast, &e)) return -1;
        }
        lin->x = tx;
        lin->y = ty;
        lin->i = ti;
        lin->last = next;
    }
}

/* ------------------------------------------------------------------------ */
/* DirectMappedCache with FNV-1a 64 (cache.rs:39-54, fnv 1.0.7)              */
/* ------------------------------------------------------------------------ */
typedef struct cache_t {
    spec_sample_t *slot;
    unsigned char *used;
    uint64_t cap;
} cache_t;

static inline uint64_t fnv_bytes(uint64_t h, const unsigned char *b, int n) {
    for (int j = 0; j < n; ++j) {
        h ^= (uint64_t)b[j];
        h *= 0x100000001b3ULL;
    }
    return h;
}

/* Hash for SpeciationSample (tracking.rs:69-75): location (x, y u32 LE),
 * index (u32 LE), sample_time bits (u64 LE), speciation_sample bits (u64 LE) */
static inline uint64_t spec_sample_hash(const spec_sample_t *v) {
    unsigned char buf[28];
    uint64_t tb = f64_bits(v->t), ub = f64_bits(v->u);
    memcpy(buf + 0, &v->x, 4);
    memcpy(buf + 4, &v->y, 4);
    memcpy(buf + 8, &v->i, 4);
    memcpy(buf + 12, &tb, 8);
    memcpy(buf + 20, &ub, 8);
    return fnv_bytes(0xcbf29ce484222325ULL, buf, 28);
}

/* returns 1 if inserted as new (not a duplicate) */
static inline int cache_insert(cache_t *c, const spec_sample_t *v) {
    if (c->cap == 0) return 1;
    uint64_t idx = spec_sample_hash(v) % c->cap;
    int insert = 1;
    if (c->used[idx]) {
        const spec_sample_t *o = &c->slot[idx];
        if (o->u == v->u && o->t == v->t && o->x == v->x && o->y == v->y && o->i == v->i)
            insert = 0;
    }
    c->slot[idx] = *v;
    c->used[idx] = 1;
    return insert;
}

/* ------------------------------------------------------------------------ */
/* Deque of (lineage, pessimistic next event time)                           */
/* ------------------------------------------------------------------------ */
typedef struct qitem_t {
    lineage_t lin;
    double next;
} qitem_t;

typedef struct deque_t {
    qitem_t *v;
    uint64_t head, n, cap;
} deque_t;

static int dq_push_back(deque_t *d, const qitem_t *it) {
    if (d->n == d->cap) {
        uint64_t nc = d->cap ? d->cap * 2 : 1024;
        qitem_t *nv = (qitem_t *)malloc(nc * sizeof(qitem_t));
        if (!nv) return -1;
        for (uint64_t j = 0; j < d->n; ++j) nv[j] = d->v[(d->head + j) % d->cap];
        free(d->v);
        d->v = nv;
        d->head = 0;
        d->cap = nc;
    }
    d->v[(d->head + d->n) % d->cap] = *it;
    d->n++;
    return 0;
}

static int dq_pop_front(deque_t *d, qitem_t *it) {
    if (d->n == 0) return 0;
    *it = d->v[d->head];
    d->head = (d->head + 1) % d->cap;
    d->n--;
    return 1;
}

/* ------------------------------------------------------------------------ */
/* Reference-faithful Monolithic water-level loop                            */
/* parallelisation/independent/monolithic/mod.rs:43-270 + reporter/live.rs  */
/* ------------------------------------------------------------------------ */
static int simulate_reference(sim_t *s, const oracle_args *args, lineage_t *init, uint64_t n_init,
                              double min_event_time, double pause_before, sink_t *k,
                              oracle_lineage *lin_out, uint64_t lin_cap) {
    oracle_result *out = k->out;
    deque_t slow = {0}, fast = {0};
    for (uint64_t j = 0; j < n_init; ++j) {
        qitem_t it = {init[j], init[j].last};
        if (dq_push_back(&slow, &it)) return -1;
    }
    /* EventSlice::capacity (independent/mod.rs:64-82) */
    uint64_t event_slice = (uint64_t)((double)n_init * args->event_slice_factor);
    if (event_slice < 1) event_slice = 1;
    /* DedupCache::construct (independent/mod.rs:38-58) */
    cache_t cache = {0};
    if (args->dedup_factor > 0.0) {
        cache.cap = (uint64_t)((double)n_init * args->dedup_factor);
        cache.slot = (spec_sample_t *)calloc(cache.cap ? cache.cap : 1, sizeof(spec_sample_t));
        cache.used = (unsigned char *)calloc(cache.cap ? cache.cap : 1, 1);
    }
    evbuf_t slow_ev = {0}, fast_ev = {0};
    double water = 0.0;
    uint64_t total_steps = 0;
    double max_time = 0.0, level = 0.0;
    for (uint64_t j = 0; j < n_init; ++j) {
        if (j == 0 || init[j].last > max_time) max_time = init[j].last;
        if (j == 0 || init[j].last < level) level = init[j].last;
    }
    int has_pause = pause_before >= 0.0;

    while (slow.n > 0 && (!has_pause || level < pause_before)) {
        /* total event rate: left fold over the slow queue in queue order */
        double rate = 0.0;
        for (uint64_t j = 0; j < slow.n; ++j) {
            const lineage_t *l = &slow.v[(slow.head + j) % slow.cap].lin;
            if (args->report_dispersal)
                rate = rate + turnover_at(s, l->x, l->y);
            else
                rate = rate + turnover_at(s, l->x, l->y) * speciation_probability(s, l->x, l->y);
        }
        level = level + (double)event_slice / rate;
        if (has_pause && pause_before < level) level = pause_before;
        /* proxy.advance_water_level (live.rs:88-115) */
        flush_sorted(k, &slow_ev);
        water = level;
        {
            uint64_t m = 0;
            for (uint64_t j = 0; j < fast_ev.n; ++j) {
                if (fast_ev.v[j].time < water) {
                    if (evbuf_push(&slow_ev, &fast_ev.v[j])) return -1;
                } else {
                    fast_ev.v[m++] = fast_ev.v[j];
                }
            }
            fast_ev.n = m;
        }
        out->n_rounds++;

        int has_active = 0;
        lineage_t active;
        int has_prev_next = 0;
        double prev_next = 0.0;
        int has_prev_sample = 0;
        spec_sample_t prev_sample;
        slice_out_t so;
        memset(&so, 0, sizeof(so));

        while (slow.n > 0 || has_active) {
            int has_next_slow = 0;
            lineage_t next_slow;
            qitem_t it;
            while (dq_pop_front(&slow, &it)) {
                if (it.next < level) {
                    next_slow = it.lin;
                    has_next_slow = 1;
                    break;
                }
                if (dq_push_back(&fast, &it)) return -1;
            }
            /* replace_active_lineage + replace_min_speciation(None) */
            int has_prev_task = has_active;
            lineage_t prev_task = active;
            has_active = has_next_slow;
            if (has_next_slow) active = next_slow;
            int had_sample = has_prev_sample;
            spec_sample_t sample = prev_sample;
            has_prev_sample = 0;

            if (has_prev_task && has_prev_next) {
                int dup = had_sample ? !cache_insert(&cache, &sample) : 0;
                if (!dup) {
                    qitem_t q = {prev_task, prev_next};
                    if (dq_push_back(prev_next < level ? &slow : &fast, &q)) return -1;
                } else {
                    out->n_dedup++;
                }
            }
            has_prev_next = 0;

            uint64_t new_steps = 0;
            double new_time = min_event_time;
            if (has_active) {
                if (run_slice(s, &active, min_event_time, args->step_slice, level,
                              args->report_dispersal, &slow_ev, &fast_ev, water, &so))
                    return s->fault ? s->fault : -1;
                new_steps = so.steps;
                new_time = so.new_time;
                if (so.peeked) {
                    has_prev_next = 1;
                    prev_next = so.next;
                }
                has_prev_sample = so.has_sample;
                prev_sample = so.sample;
                if (!so.alive) has_active = 0;
            }
            total_steps += new_steps;
            if (new_time > max_time) max_time = new_time;
        }
        /* fast lineages are now slow again */
        deque_t tmp = slow;
        slow = fast;
        fast = tmp;
    }
    /* proxy.finalise(): slow events sorted, then fast events sorted */
    flush_sorted(k, &slow_ev);
    flush_sorted(k, &fast_ev);

    out->steps = total_steps;
    out->time = max_time;
    out->n_remaining = slow.n;
    out->status = slow.n > 0 ? 1 : 0;
    for (uint64_t j = 0; j < slow.n && j < lin_cap; ++j) {
        const lineage_t *l = &slow.v[(slow.head + j) % slow.cap].lin;
        lin_out[j].gref = l->gref;
        lin_out[j].last_event_time = l->last;
        lin_out[j].x = l->x;
        lin_out[j].y = l->y;
        lin_out[j].index = l->i;
        lin_out[j].pad = 0;
    }
    free(slow.v);
    free(fast.v);
    free(cache.slot);
    free(cache.used);
    free(slow_ev.v);
    free(fast_ev.v);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Canonical schedule (the GPU backend's): common time horizons per round,   */
/* state-equality dedup keeping the smallest global reference.               */
/* ------------------------------------------------------------------------ */
static int lineage_key_cmp(const void *pa, const void *pb) {
    const lineage_t *a = (const lineage_t *)pa, *b = (const lineage_t *)pb;
    int c;
    if ((c = cmp_u32(a->x, b->x))) return c;
    if ((c = cmp_u32(a->y, b->y))) return c;
    if ((c = cmp_u32(a->i, b->i))) return c;
    if ((c = cmp_u64(f64_bits(a->last), f64_bits(b->last)))) return c;
    return cmp_u64(a->gref, b->gref);
}

static int simulate_canonical(sim_t *s, const oracle_args *args, lineage_t *lins, uint64_t n,
                              double min_event_time, double pause_before, sink_t *k,
                              oracle_lineage *lin_out, uint64_t lin_cap) {
    oracle_result *out = k->out;
    evbuf_t ev = {0}, none = {0};
    uint64_t total_steps = 0;
    double max_time = 0.0, horizon = 0.0;
    for (uint64_t j = 0; j < n; ++j) {
        if (j == 0 || lins[j].last > max_time) max_time = lins[j].last;
        if (j == 0 || lins[j].last < horizon) horizon = lins[j].last;
    }
    int has_pause = pause_before >= 0.0;
    uint64_t step_slice = args->step_slice ? args->step_slice : 1;
    while (n > 0 && (!has_pause || horizon < pause_before)) {
        /* events per lineage this round:
         * clamp(ceil(min_round_events / n), step_slice, max(step_slice, step_slice_max)) */
        uint64_t per = (args->min_round_events + n - 1) / n;
        if (args->step_slice_max && per > args->step_slice_max) per = args->step_slice_max;
        if (per < step_slice) per = step_slice;
        double next_horizon = horizon + (double)per / s->lambda;
        if (has_pause && pause_before < next_horizon) next_horizon = pause_before;
        out->n_rounds++;
        uint64_t m = 0;
        for (uint64_t j = 0; j < n; ++j) {
            slice_out_t so;
            if (run_slice(s, &lins[j], min_event_time, UINT64_MAX, next_horizon,
                          args->report_dispersal, &ev, &none, INFINITY, &so))
                return s->fault ? s->fault : -1;
            total_steps += so.steps;
            if (so.new_time > max_time) max_time = so.new_time;
            if (so.alive) lins[m++] = lins[j];
        }
        n = m;
        /* dedup: identical (x, y, i, last_event_time) => identical future */
        qsort(lins, n, sizeof(lineage_t), lineage_key_cmp);
        m = 0;
        for (uint64_t j = 0; j < n; ++j) {
            if (m > 0 && lins[m - 1].x == lins[j].x && lins[m - 1].y == lins[j].y &&
                lins[m - 1].i == lins[j].i && f64_bits(lins[m - 1].last) == f64_bits(lins[j].last)) {
                out->n_dedup++;
                continue;
            }
            lins[m++] = lins[j];
        }
        n = m;
        horizon = next_horizon;
    }
    flush_sorted(k, &ev);
    out->steps = total_steps;
    out->time = max_time;
    out->n_remaining = n;
    out->status = n > 0 ? 1 : 0;
    for (uint64_t j = 0; j < n && j < lin_cap; ++j) {
        lin_out[j].gref = lins[j].gref;
        lin_out[j].last_event_time = lins[j].last;
        lin_out[j].x = lins[j].x;
        lin_out[j].y = lins[j].y;
        lin_out[j].index = lins[j].i;
        lin_out[j].pad = 0;
    }
    free(ev.v);
    free(none.v);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Entry points                                                              */
/* ------------------------------------------------------------------------ */
static int run_common(sim_t *s, const oracle_args *args, lineage_t *lins, uint64_t n,
                      double min_event_time, double pause_before, oracle_result *out,
                      oracle_speciation_event *spec, uint64_t spec_cap,
                      oracle_dispersal_event *disp, uint64_t disp_cap, oracle_lineage *lin,
                      uint64_t lin_cap) {
    /* IsolatedIndividuals partitioning (pre_sampler.rs:103-112): rank r of P
     * keeps every P-th origin starting at r */
    uint32_t P = args->partition_size ? args->partition_size : 1;
    uint32_t r = args->partition_rank;
    if (P > 1) {
        uint64_t m = 0;
        for (uint64_t j = r; j < n; j += P) lins[m++] = lins[j];
        n = m;
    }
    out->n_initial = n;
    sink_t k;
    memset(&k, 0, sizeof(k));
    k.out = out;
    k.spec = spec;
    k.spec_cap = spec_cap;
    k.disp = disp;
    k.disp_cap = disp_cap;
    int rc;
    if (args->mode == ORACLE_MODE_CANONICAL)
        rc = simulate_canonical(s, args, lins, n, min_event_time, pause_before, &k, lin, lin_cap);
    else
        rc = simulate_reference(s, args, lins, n, min_event_time, pause_before, &k, lin, lin_cap);
    out->n_primes = s->rng.n_primes;
    out->n_draws = s->rng.n_draws;
    if (rc) out->status = rc;
    return rc;
}

int oracle_simulate(const oracle_scenario *sc, const oracle_args *args, uint64_t seed,
                    double pause_before, oracle_result *out, oracle_speciation_event *spec,
                    uint64_t spec_cap, oracle_dispersal_event *disp, uint64_t disp_cap,
                    oracle_lineage *lin, uint64_t lin_cap) {
    memset(out, 0, sizeof(*out));
    sim_t s;
    int rc = sim_init(&s, sc, args, seed);
    if (rc) {
        sim_free(&s);
        out->status = rc;
        return rc;
    }
    int64_t n = enumerate_origins(sc, &s, NULL, 0);
    lineage_t *lins = (lineage_t *)malloc((n > 0 ? n : 1) * sizeof(lineage_t));
    if (!lins) {
        sim_free(&s);
        out->status = -1;
        return -1;
    }
    enumerate_origins(sc, &s, lins, (uint64_t)n);
    rc = run_common(&s, args, lins, (uint64_t)n, 0.0, pause_before, out, spec, spec_cap, disp,
                    disp_cap, lin, lin_cap);
    free(lins);
    sim_free(&s);
    return rc;
}

int oracle_simulate_lineages(const oracle_scenario *sc, const oracle_args *args, uint64_t seed,
                             const oracle_lineage *lineages, uint64_t n_lineages,
                             double resume_time, double pause_before, oracle_result *out,
                             oracle_speciation_event *spec, uint64_t spec_cap,
                             oracle_dispersal_event *disp, uint64_t disp_cap, oracle_lineage *lin,
                             uint64_t lin_cap) {
    memset(out, 0, sizeof(*out));
    sim_t s;
    int rc = sim_init(&s, sc, args, seed);
    if (rc) {
        sim_free(&s);
        out->status = rc;
        return rc;
    }
    lineage_t *lins = (lineage_t *)malloc((n_lineages ? n_lineages : 1) * sizeof(lineage_t));
    uint64_t n = 0;
    for (uint64_t j = 0; j < n_lineages; ++j) {
        const oracle_lineage *l = &lineages[j];
        /* independent/mod.rs:98-117: a lineage off the habitat (Habitat::
         * is_location_habitable = extent contains it and habitat > 0) or off
         * its deme is exceptional, and initialiser/resume.rs:79-85 then fails */
        int on_map = 1;
        if (s.kind == ORACLE_NON_SPATIAL || s.kind == ORACLE_SPATIALLY_EXPLICIT)
            on_map = extent_contains(&s.local, l->x, l->y);
        uint32_t h = on_map ? habitat_at(&s, l->x, l->y) : 0;
        if (h == 0 || l->index >= h) {
            free(lins);
            sim_free(&s);
            out->status = -5;
            return -5;
        }
        lins[n].gref = l->gref;
        lins[n].last = l->last_event_time;
        lins[n].x = l->x;
        lins[n].y = l->y;
        lins[n].i = l->index;
        n++;
    }
    rc = run_common(&s, args, lins, n, resume_time, pause_before, out, spec, spec_cap, disp,
                    disp_cap, lin, lin_cap);
    free(lins);
    sim_free(&s);
    return rc;
}

/* ---- known-answer helpers ---- */
void oracle_wyhash_sequence(uint64_t seed, uint64_t location, uint64_t time_index, uint64_t *out,
                            uint64_t n) {
    rng_t g = {seed, seed, 0, 0};
    rng_prime(&g, location, time_index);
    for (uint64_t j = 0; j < n; ++j) out[j] = rng_sample_u64(&g);
}

uint64_t oracle_seahash_diffuse(uint64_t x) { return seahash_diffuse(x); }
uint64_t oracle_wymum(uint64_t a, uint64_t b) { return wymum(a, b); }

double oracle_poisson_next_event_time(uint64_t seed, uint64_t inj, double t, double lambda,
                                      double delta_t, uint64_t *reprime) {
    sim_t s;
    memset(&s, 0, sizeof(s));
    s.rng.seed = seed;
    s.rng.state = seed;
    s.lambda = lambda;
    s.delta_t = delta_t;
    s.lambda_dt = lambda * delta_t;
    s.p0 = exp(-s.lambda_dt);
    return poisson_next_event_time(&s, inj, t, reprime, lambda);
}

double oracle_exp_next_event_time(uint64_t seed, uint64_t inj, double t, double lambda,
                                  double delta_t, uint64_t *reprime) {
    sim_t s;
    memset(&s, 0, sizeof(s));
    s.rng.seed = seed;
    s.rng.state = seed;
    s.lambda = lambda;
    s.delta_t = delta_t;
    return exp_next_event_time(&s, inj, t, reprime, lambda);
}

void oracle_ln(const double *x, double *out, uint64_t n) {
    for (uint64_t j = 0; j < n; ++j) out[j] = necsim_ln(x[j]);
}
