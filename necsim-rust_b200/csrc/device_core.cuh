// device_core.cuh -- per-lineage arithmetic of the Independent algorithm on
// sm_100a: WyHash priming/sampling, the Poisson and exponential event-time
// samplers, the speciation test, the four dispersal samplers and the coalescence index.
//
// Every f64 expression is evaluated as one IEEE-754 round-to-nearest
// operation per source operator in the reference's order (the file is
// compiled with --fmad=false so no multiply-add is contracted), and every
// integer operation wraps like Rust's, so a lineage's trajectory is the
// reference's bit for bit.
#pragma once

#include <cstdint>

#include "layout.h"
#include "ln_dd.h"

namespace necsim {

// necsim/impls/no-std/src/cogs/rng/wyhash.rs:9-12
constexpr uint64_t kWyP0 = 0xa0761d6478bd642fULL;
constexpr uint64_t kWyP1 = 0xe7037ed1a0b428dbULL;
constexpr uint64_t kWyP2 = 0x8ebc6af09c88c6e3ULL;
constexpr uint64_t kWyP5 = 0xeb44accab455d165ULL;
// wyhash.rs:99-119 SeaHash diffusion multiplier
constexpr uint64_t kSeaHashK = 0x6eed0e9da4d94a4fULL;
// event_time_sampler/poisson.rs:10: 2^64 / phi
constexpr uint64_t kInvPhi = 0x9e3779b97f4a7c15ULL;
// core::f64::consts::TAU
constexpr double kTau = 6.283185307179586;

// wyhash.rs:85-96: 64x64 -> 128 multiply, low and high halves xor-folded
__device__ __forceinline__ uint64_t wymum(uint64_t a, uint64_t b) {
    const uint64_t lo = a * b;
    const uint64_t hi = __umul64hi(a, b);
    return (a ^ lo) ^ (b ^ hi);
}

// wyhash.rs:99-119
__device__ __forceinline__ uint64_t seahash_diffuse(uint64_t x) {
    x *= kSeaHashK;
    const uint64_t a = x >> 32;
    const uint64_t b = x >> 60;
    x ^= a >> b;
    x *= kSeaHashK;
    return x;
}

__device__ __forceinline__ uint64_t swap_halves(uint64_t v) { return (v << 32) | (v >> 32); }

struct Rng {
    uint64_t seed;
    uint64_t state;

    // wyhash.rs:68-80 PrimeableRng::prime_with
    __device__ __forceinline__ void prime(uint64_t location_index, uint64_t time_index) {
        const uint64_t l = seahash_diffuse(location_index);
        const uint64_t t = seahash_diffuse(time_index);
        const uint64_t h = wymum(swap_halves(l) ^ (seed ^ kWyP0), swap_halves(t) ^ kWyP2);
        state = wymum(h, 16ULL ^ kWyP5);
    }

    // wyhash.rs:53-63 RngCore::sample_u64
    __device__ __forceinline__ uint64_t next_u64() {
        state += kWyP0;
        return seahash_diffuse(wymum(state ^ kWyP1, state));
    }

    // necsim/core/src/cogs/rng.rs:75-82 -- [0, 1)
    __device__ __forceinline__ double closed_open() {
        return __dmul_rn(__ull2double_rn(next_u64() >> 11), 0x1.0p-53);
    }

    // rng.rs:84-93 -- (0, 1]
    __device__ __forceinline__ double open_closed() {
        return __dmul_rn(__ull2double_rn((next_u64() >> 11) + 1ULL), 0x1.0p-53);
    }
};

// ---- counter form of the same generator ----
// After prime_with the k-th sample_u64 (k = 1, 2, ...) only depends on the
// primed state s0: state_k = s0 + k * P0 (wrapping).  Computing the samples
// of one event from s0 independently, instead of one after the other, gives
// the same values with the 64-bit multiply chains overlapped.

// the location half of prime_with: rotate(diffuse(location)) ^ seed ^ P0
__device__ __forceinline__ uint64_t location_term(uint64_t seed, uint64_t location_index) {
    return swap_halves(seahash_diffuse(location_index)) ^ (seed ^ kWyP0);
}

// WyHash state after prime_with(location, time_index), from the location term
__device__ __forceinline__ uint64_t primed_state(uint64_t loc_term, uint64_t time_index) {
    const uint64_t h = wymum(loc_term, swap_halves(seahash_diffuse(time_index)) ^ kWyP2);
    return wymum(h, 16ULL ^ kWyP5);
}

// the k-th sample_u64 after priming to s0
__device__ __forceinline__ uint64_t draw_at(uint64_t s0, uint32_t k) {
    const uint64_t s = s0 + (uint64_t)k * kWyP0;
    return seahash_diffuse(wymum(s ^ kWyP1, s));
}

__device__ __forceinline__ double unit_closed_open(uint64_t v) {
    return __dmul_rn(__ull2double_rn(v >> 11), 0x1.0p-53);
}
__device__ __forceinline__ double unit_open_closed(uint64_t v) {
    return __dmul_rn(__ull2double_rn((v >> 11) + 1ULL), 0x1.0p-53);
}

// Rust `f64 as u64` for the non-negative finite values these call sites see
// (floor of a product of a unit sample and a table length, or of t / dt);
// saturates like Rust above range.
__device__ __forceinline__ uint64_t f64_to_u64(double v) {
    if (!(v > 0.0)) return 0;
    if (v >= 18446744073709551616.0) return ~0ULL;
    return __double2ull_rz(v);
}
__device__ __forceinline__ uint32_t f64_to_u32(double v) {
    if (!(v > 0.0)) return 0;
    if (v >= 4294967296.0) return 0xffffffffu;
    return __double2uint_rz(v);
}
__device__ __forceinline__ int64_t f64_to_i64(double v) {
    if (v != v) return 0;
    if (v >= 9223372036854775808.0) return INT64_MAX;
    if (v < -9223372036854775808.0) return INT64_MIN;
    return __double2ll_rz(v);
}

// necsim/core/bond/src/positive_f64.rs:103-113 PositiveF64::max_after
__device__ __forceinline__ double max_after(double before, double value) {
    if (value > before || before != before) return value;
    if (isinf(before)) return before;
    return __longlong_as_double(__double_as_longlong(before) + 1);
}

// Devroye's Poisson(lambda * delta_t) count (poisson.rs:51-65) from the
// bucket's first sample d1: the loop passes rank n while
// X > floor(acc_n * 2^53) and prod_n > 0.  The thresholds are
// non-decreasing and a rank with prod_n == 0 carries the threshold ~0, so
// the stopping rank is the number of thresholds X exceeds: eight independent
// compares instead of a loop of dependent loads.  Beyond the tabulated ranks
// the reference loop continues in f64.
__device__ __forceinline__ uint32_t poisson_count(uint64_t d1, const PoissonConsts &pc) {
    const uint64_t X = d1 >> 11;
    uint32_t n_events = 0;
#pragma unroll
    for (int r = 0; r < kPoissonThresholds; ++r) n_events += X > pc.threshold[r] ? 1u : 0u;
    if (n_events == (uint32_t)kPoissonThresholds) {
        const double u = unit_closed_open(d1);
        double prod = pc.prod_k;
        double acc = pc.acc_k;
        while (u > acc && prod > 0.0) {
            n_events += 1;
            const double ratio = n_events <= (uint32_t)kPoissonTable
                                     ? pc.lambda_dt_over_k[n_events - 1]
                                     : __ddiv_rn(pc.lambda_dt, __uint2double_rn(n_events));
            prod = __dmul_rn(prod, ratio);
            acc = __dadd_rn(acc, prod);
        }
    }
    return n_events;
}

// event time (t_s + u) * delta_t of a bucket's sample, as its bit pattern
// (non-negative doubles order like their bits)
__device__ __forceinline__ long long event_time_bits(double step_start, uint64_t d, double delta_t) {
    return __double_as_longlong(__dmul_rn(__dadd_rn(step_start, unit_closed_open(d)), delta_t));
}

// One bucket of the Poisson sampler (poisson.rs:50-95) primed to s0: the
// earliest event strictly after `time` (ties: lowest index), or -1.  Samples
// are drawn only as the reference consumes them (throughput form).
__device__ __forceinline__ int poisson_bucket(uint64_t s0, uint64_t time_step, double time,
                                              const SimParams &p, const PoissonConsts &pc, double &best) {
    const uint32_t n_events = poisson_count(draw_at(s0, 1), pc);
    if (n_events == 0) return -1;
    const double step_start = __ull2double_rn(time_step);
    const long long time_bits = __double_as_longlong(time);
    int best_k = -1;
    long long best_bits = 0;
    for (uint32_t k = 0; k < n_events; ++k) {
        const long long eb = event_time_bits(step_start, draw_at(s0, k + 2), p.delta_t);
        if (eb > time_bits && (best_k < 0 || best_bits > eb)) {
            best_bits = eb;
            best_k = (int)k;
        }
    }
    best = __longlong_as_double(best_bits);
    return best_k;
}

// The same bucket from its first three samples drawn ahead (latency form):
// events 0 and 1 use d2 and d3, further events draw their samples here.
__device__ __forceinline__ int poisson_bucket_drawn(uint64_t s0, uint64_t d1, uint64_t d2, uint64_t d3,
                                                    uint64_t time_step, long long time_bits,
                                                    const SimParams &p, const PoissonConsts &pc,
                                                    long long &best_bits) {
    const double step_start = __ull2double_rn(time_step);
    const long long e0 = event_time_bits(step_start, d2, p.delta_t);
    const long long e1 = event_time_bits(step_start, d3, p.delta_t);
    const uint32_t n_events = poisson_count(d1, pc);
    int best_k = -1;
    long long bb = 0;
    if (n_events >= 1 && e0 > time_bits) {
        bb = e0;
        best_k = 0;
    }
    if (n_events >= 2 && e1 > time_bits && (best_k < 0 || bb > e1)) {
        bb = e1;
        best_k = 1;
    }
    for (uint32_t k = 2; k < n_events; ++k) {
        const long long eb = event_time_bits(step_start, draw_at(s0, k + 2), p.delta_t);
        if (eb > time_bits && (best_k < 0 || bb > eb)) {
            bb = eb;
            best_k = (int)k;
        }
    }
    best_bits = bb;
    return best_k;
}

// poisson_next_event_time in counter form: buckets are primed two at a time
// (the second speculatively) from the shared location term.  Returns the
// event time, the re-prime time index and the re-primed state.
__device__ __forceinline__ double poisson_next_event_time_ilp(uint64_t loc_term, double time,
                                                              const SimParams &p, const PoissonConsts &pc,
                                                              uint64_t &reprime,
                                                              uint64_t &reprimed_state) {
    const double q = p.inv_delta_t != 0.0 ? __dmul_rn(time, p.inv_delta_t) : __ddiv_rn(time, p.delta_t);
    uint64_t time_step = f64_to_u64(floor(q));
    for (;;) {
        double best = 0.0;
        const int k = poisson_bucket(primed_state(loc_term, time_step), time_step, time, p, pc, best);
        if (k >= 0) {
            reprime = time_step + kInvPhi * (uint64_t)(k + 1);
            reprimed_state = primed_state(loc_term, reprime);
            return best;
        }
        time_step += 1;
    }
}

// poisson_next_event_time for a lineage whose warp has few others to run
// (latency form): buckets are primed two at a time, the second
// speculatively, with each bucket's first three samples drawn at once, so
// the dependent chain per event is one prime, one draw and the compares.
__device__ __forceinline__ double poisson_next_event_time_lat(uint64_t loc_term, double time,
                                                              const SimParams &p, const PoissonConsts &pc,
                                                              uint64_t &reprime,
                                                              uint64_t &reprimed_state) {
    const double q = p.inv_delta_t != 0.0 ? __dmul_rn(time, p.inv_delta_t) : __ddiv_rn(time, p.delta_t);
    uint64_t time_step = f64_to_u64(floor(q));
    const long long time_bits = __double_as_longlong(time);
    for (;;) {
        const uint64_t s0 = primed_state(loc_term, time_step);
        const uint64_t s1 = primed_state(loc_term, time_step + 1);
        const uint64_t a1 = draw_at(s0, 1), a2 = draw_at(s0, 2), a3 = draw_at(s0, 3);
        const uint64_t b1 = draw_at(s1, 1), b2 = draw_at(s1, 2), b3 = draw_at(s1, 3);
        long long bits = 0;
        uint64_t chosen = time_step;
        int k = poisson_bucket_drawn(s0, a1, a2, a3, time_step, time_bits, p, pc, bits);
        if (k < 0) {
            chosen = time_step + 1;
            k = poisson_bucket_drawn(s1, b1, b2, b3, chosen, time_bits, p, pc, bits);
        }
        if (k >= 0) {
            reprime = chosen + kInvPhi * (uint64_t)(k + 1);
            reprimed_state = primed_state(loc_term, reprime);
            return __longlong_as_double(bits);
        }
        time_step += 2;
    }
}

// ---- the exponential event-time sampler ----

// rng.rs:163-167 sample_exponential of one sample: -ln(U(0,1]) / lambda,
// with the logarithm shared bit for bit with the host (ln_dd.h)
__device__ __forceinline__ double exp_sample(uint64_t d, double lambda) {
    return __ddiv_rn(-necsim_ln(unit_open_closed(d)), lambda);
}

// floor(time / delta_t) as u64 (poisson.rs:44, exp.rs:52)
__device__ __forceinline__ uint64_t time_bucket(const SimParams &p, double time) {
    const double q = p.inv_delta_t != 0.0 ? __dmul_rn(time, p.inv_delta_t) : __ddiv_rn(time, p.delta_t);
    return f64_to_u64(floor(q));
}

// The loop of ExpEventTimeSampler (event_time_sampler/exp.rs:37-83) from
// the state after sample j of bucket ts (running event time et, bucket
// start ts * delta_t when j == 0): sample j + 1 of the bucket primed at ts
// is draw_at(s0, j + 1) and its sub-index (j + 1) * INV_PHI, and a sum at
// or past the bucket's end moves to the next bucket.  Returns the first
// event time after `time` and its re-prime time index ts + j * INV_PHI.
__device__ __forceinline__ double exp_continue(uint64_t loc_term, double time, const SimParams &p,
                                               const PoissonConsts &pc, uint64_t ts, uint32_t j, double et,
                                               uint64_t &reprime) {
    uint64_t s0 = primed_state(loc_term, ts);
    double slice_end = __dmul_rn(__ull2double_rn(ts + 1), p.delta_t);
    for (;;) {
        j += 1;
        et = __dadd_rn(et, exp_sample(draw_at(s0, j), pc.lambda));
        if (et >= slice_end) {
            ts += 1;
            j = 0;
            et = slice_end;
            slice_end = __dmul_rn(__ull2double_rn(ts + 1), p.delta_t);
            s0 = primed_state(loc_term, ts);
        } else if (et > time) {
            break;
        }
    }
    reprime = ts + kInvPhi * (uint64_t)j;
    return et;
}

// exp.rs:37-83 ExpEventTimeSampler::next_event_time_at_indexed_location_weakly_after
__device__ __forceinline__ double exp_next_event_time(uint64_t loc_term, double time, const SimParams &p,
                                                      const PoissonConsts &pc, uint64_t &reprime) {
    const uint64_t ts = time_bucket(p, time);
    return exp_continue(loc_term, time, p, pc, ts, 0, __dmul_rn(__ull2double_rn(ts), p.delta_t), reprime);
}

// ---- the samplers fed with pre-drawn samples ----

// rng.rs:133-145 sample_index_u64 of one sample
__device__ __forceinline__ uint64_t index_from_draw(uint64_t d, uint64_t length) {
    const uint64_t index = f64_to_u64(floor(__dmul_rn(unit_closed_open(d), __ull2double_rn(length))));
    return index < length - 1 ? index : length - 1;
}

// n / d for n, d < 2^32 from magic = ceil(2^64 / d) (0 when d == 1)
__device__ __forceinline__ uint32_t div_by_magic(uint32_t n, uint64_t magic) {
    return magic ? (uint32_t)__umul64hi(magic, (uint64_t)n) : n;
}

// dispersal_sampler/non_spatial.rs:42-66
__device__ __forceinline__ void non_spatial_dispersal_draw(uint64_t d, uint32_t ox, uint32_t oy,
                                                           uint64_t w, uint64_t h, uint64_t w_magic,
                                                           uint32_t &tx, uint32_t &ty) {
    const uint64_t n = w * h;
    const uint64_t idx = index_from_draw(d, n);
    if (h == 1) {  // idx < w: quotient 0
        tx = ox + (uint32_t)idx;
        ty = oy;
    } else if (n <= 0xffffffffULL) {  // 32-bit quotient by the width's magic
        const uint32_t i32 = (uint32_t)idx;
        const uint32_t q = div_by_magic(i32, w_magic);
        tx = ox + (i32 - q * (uint32_t)w);
        ty = oy + q;
    } else {
        tx = ox + (uint32_t)(idx % w);
        ty = oy + (uint32_t)(idx / w);
    }
}

// core/src/cogs/coalescence_sampler.rs:59-78: floor(u * habitat) as u32
__device__ __forceinline__ uint32_t coalescence_index(uint64_t d, uint32_t habitat) {
    return f64_to_u32(floor(__dmul_rn(unit_closed_open(d), __uint2double_rn(habitat))));
}

// habitat/almost_infinite.rs:100-114 clamp_round_dispersal
__device__ __forceinline__ void clamp_round_dispersal(uint32_t x, uint32_t y, double dx, double dy,
                                                      uint32_t &tx, uint32_t &ty) {
    const int64_t wrap = (int64_t)1 << 32;
    const int64_t nx = ((int64_t)x + f64_to_i64(round(dx))) % wrap;
    const int64_t ny = ((int64_t)y + f64_to_i64(round(dy))) % wrap;
    tx = (uint32_t)((nx + wrap) % wrap);
    ty = (uint32_t)((ny + wrap) % wrap);
}

// almost_infinite_clark2dt.rs:96-107 with clark2dt::cdf_inverse and
// pow_fast_one (:167-189) from samples 2 (u01, [0, 1)) and 3 (angle, (0, 1]):
// jump = sqrt(u * (pow(1 / (1 - u01), 1 / p) - 1)), theta = u2 * 2 * pi,
// displacement (cos(theta) * jump, sin(theta) * jump).  The transcendental
// calls are CUDA's f64 pow/cos/sin; their results only pass through
// round(), like the Normal sampler's.
__device__ __forceinline__ void clark2dt_displacement(uint64_t d0, uint64_t d1, double shape_u, double exponent,
                                                      double &dx, double &dy) {
    const double u01 = unit_closed_open(d0);
    const double u2 = unit_open_closed(d1);
    const double base = __ddiv_rn(1.0, __dsub_rn(1.0, u01));
    const double powed = exponent == 1.0 ? base : pow(base, exponent);
    const double jump = __dsqrt_rn(__dmul_rn(shape_u, __dsub_rn(powed, 1.0)));
    const double theta = __dmul_rn(__dmul_rn(u2, 2.0), 3.141592653589793);
    dx = __dmul_rn(cos(theta), jump);
    dy = __dmul_rn(sin(theta), jump);
}

__device__ __forceinline__ void clark2dt_dispersal_draw(uint64_t d0, uint64_t d1, double shape_u,
                                                        double exponent, uint32_t x, uint32_t y, uint32_t &tx,
                                                        uint32_t &ty) {
    double dx, dy;
    clark2dt_displacement(d0, d1, shape_u, exponent, dx, dy);
    clamp_round_dispersal(x, y, dx, dy, tx, ty);
}

// rng.rs:180-197 sample_2d_normal (Box-Muller) scaled by sigma
// (almost_infinite_normal.rs:58-68) from the two samples, with CUDA's f64
// log/sin/cos
__device__ __forceinline__ void normal_displacement(uint64_t d0, uint64_t d1, double sigma, double &dx,
                                                    double &dy) {
    const double u0 = unit_open_closed(d0);
    const double u1 = unit_closed_open(d1);
    const double r = __dsqrt_rn(__dmul_rn(-2.0, log(u0)));
    const double theta = __dmul_rn(-kTau, u1);
    const double z0 = __dmul_rn(r, sin(theta));
    const double z1 = __dmul_rn(r, cos(theta));
    dx = __dadd_rn(__dmul_rn(z0, sigma), 0.0);
    dy = __dadd_rn(__dmul_rn(z1, sigma), 0.0);
}

// the Normal displacement rounded onto the plane (almost_infinite.rs:100-114)
__device__ __forceinline__ void normal_dispersal_draw(uint64_t d0, uint64_t d1, double sigma,
                                                      uint32_t x, uint32_t y, uint32_t &tx,
                                                      uint32_t &ty) {
    double dx, dy;
    normal_displacement(d0, d1, sigma, dx, dy);
    clamp_round_dispersal(x, y, dx, dy, tx, ty);
}

// landscape/extent.rs:44-49 LandscapeExtent::contains for the SI local
// extent, whose origin is (0, 0)
__device__ __forceinline__ bool in_local(const SimParams &p, uint32_t x, uint32_t y) {
    return x <= p.width - 1 && y <= p.height - 1;
}

// habitat/non_spatial.rs:88-105 map_indexed_location_to_u64_injective
__device__ __forceinline__ uint64_t non_spatial_injection(uint32_t ox, uint32_t oy, uint64_t w,
                                                          uint32_t deme, uint32_t x, uint32_t y,
                                                          uint32_t i) {
    return ((uint64_t)(y - oy) * w + (uint64_t)(x - ox)) * (uint64_t)deme + (uint64_t)i;
}

}  // namespace necsim
