// wrapping_noise.h -- the WrappingNoise habitat, shared by the host (habitat
// threshold, origins, resume checks) and the kernels (dispersal targets).
//
// WrappingNoiseHabitat (necsim/impls/no-std/src/cogs/habitat/wrapping_noise/
// mod.rs) marks a location habitable when its octave sum of 2D OpenSimplex
// noise (opensimplex_noise/open_simplex_noise_2d.rs, utils.rs) is at most a
// threshold, the coverage quantile of the noise at 2^16 pseudo-random
// locations.  Every octave wraps at an integer lattice period, so the plane
// of 2^32 x 2^32 locations tiles seamlessly.
//
// Each f64 operation rounds once, in the reference's order: the device uses
// the explicit round-to-nearest intrinsics (never contracted into a fused
// multiply-add), the host is compiled without contraction; floor and round
// are exact in both.  Host and device therefore compute identical bits.
#pragma once

#include <cmath>
#include <cstdint>

#include "layout.h"

#if defined(__CUDACC__)
#define NECSIM_NOISE_FN __host__ __device__ __forceinline__
#else
#define NECSIM_NOISE_FN inline
#endif

namespace necsim {
namespace noise {

NECSIM_NOISE_FN double add(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}

NECSIM_NOISE_FN double sub(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}

NECSIM_NOISE_FN double mul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}

NECSIM_NOISE_FN double div(double a, double b) {
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}

NECSIM_NOISE_FN double flr(double v) {
#ifdef __CUDA_ARCH__
    return ::floor(v);
#else
    return std::floor(v);
#endif
}

// f64::round: half away from zero
NECSIM_NOISE_FN double rnd(double v) {
#ifdef __CUDA_ARCH__
    return ::round(v);
#else
    return std::round(v);
#endif
}

// the low byte of Rust's `v as i64` (truncating, saturating, NaN -> 0)
NECSIM_NOISE_FN uint32_t low_byte_of_i64(double v) {
    if (v != v) return 0u;
    if (v >= 9223372036854775808.0) return 0xffu;  // i64::MAX
    if (v <= -9223372036854775808.0) return 0u;    // i64::MIN
    return (uint32_t)((uint64_t)(int64_t)v & 0xffu);
}

constexpr double kStretch = -0.211324865405187;  // open_simplex_noise_2d.rs:9, as written there
constexpr double kSquish = 0.366025403784439;    // open_simplex_noise_2d.rs:10
constexpr double kTwo32 = 4294967296.0;          // (u32::MAX as f64) + 1.0
constexpr double kTwoM32 = 1.0 / 4294967296.0;   // exact: x / 2^32 == x * 2^-32
constexpr double kFrac1Pi = 0.318309886183790671537767526745028724;  // core::f64::consts::FRAC_1_PI

// open_simplex_noise_2d.rs:21-59 extrapolate: the lattice point wrapped into
// [0, wrap), its gradient (+-5, +-2) or (+-2, +-5) from two permutation
// reads.  The hash reads perm[0..256) and only their low bytes:
// (perm[a] + b) & 0xff and (perm[c] & 0x0e) >> 1 depend on nothing else.
NECSIM_NOISE_FN double extrapolate(const uint8_t *perm, double gx, double gy, double dx, double dy, double wrap) {
    gx = flr(sub(gx, mul(flr(div(gx, wrap)), wrap)));
    gy = flr(sub(gy, mul(flr(div(gy, wrap)), wrap)));
    const uint32_t i0 = ((uint32_t)perm[low_byte_of_i64(gx)] + low_byte_of_i64(gy)) & 0xffu;
    const uint32_t idx = ((uint32_t)perm[i0] & 0x0eu) >> 1;
    double px = (idx & 1u) == 0 ? 5.0 : 2.0;
    double py = (idx & 1u) == 0 ? 2.0 : 5.0;
    if (idx & 2u) px = -px;
    if (idx & 4u) py = -py;
    return add(mul(px, dx), mul(py, dy));
}

// opensimplex_noise/utils.rs:5-23 contribute
NECSIM_NOISE_FN double contribute(const uint8_t *perm, double dx, double dy, double ox, double oy, double gx,
                                  double gy, double wrap) {
    const double ds = add(dx, dy);
    const double sx = sub(sub(ox, dx), mul(kSquish, ds));
    const double sy = sub(sub(oy, dy), mul(kSquish, ds));
    const double attn = sub(2.0, add(mul(sx, sx), mul(sy, sy)));
    if (attn <= 0.0) return 0.0;
    const double a2 = mul(attn, attn);
    const double a4 = mul(a2, a2);
    return mul(a4, extrapolate(perm, add(gx, dx), add(gy, dy), sx, sy, wrap));
}

// open_simplex_noise_2d.rs:61-128 eval, get_value, evaluate_inside_triangle
NECSIM_NOISE_FN double eval2d(const uint8_t *perm, double x, double y, double wrap) {
    const double s = add(x, y);
    const double ix = add(x, mul(kSquish, s)), iy = add(y, mul(kSquish, s));  // pre-squished input
    const double s2 = add(ix, iy);
    const double stx = add(ix, mul(kStretch, s2)), sty = add(iy, mul(kStretch, s2));
    const double gx = flr(stx), gy = flr(sty);
    const double gs = add(gx, gy);
    const double ox = sub(ix, add(gx, mul(kSquish, gs)));
    const double oy = sub(iy, add(gy, mul(kSquish, gs)));
    const double insx = sub(stx, gx), insy = sub(sty, gy);
    const double value =
        add(contribute(perm, 1.0, 0.0, ox, oy, gx, gy, wrap), contribute(perm, 0.0, 1.0, ox, oy, gx, gy, wrap));
    const double in_sum = add(insx, insy);
    const double f = in_sum <= 1.0 ? 0.0 : 1.0;
    const double z = sub(add(1.0, f), in_sum);
    double px, py;
    if (z > insx || z > insy) {
        // (0, 0) is one of the two closest triangle vertices
        px = insx > insy ? add(1.0, f) : add(-1.0, f);
        py = insx > insy ? add(-1.0, f) : add(1.0, f);
    } else {
        px = sub(1.0, f);
        py = sub(1.0, f);
    }
    const double tri = add(contribute(perm, f, f, ox, oy, gx, gy, wrap), contribute(perm, px, py, ox, oy, gx, gy, wrap));
    return div(add(value, tri), 47.0);
}

// habitat/wrapping_noise/mod.rs:216-249 sum_noise_octaves
NECSIM_NOISE_FN double octave_sum(const NoiseHabitat &h, uint32_t x, uint32_t y) {
    double max_amplitude = 0.0, amplitude = 1.0;
    double frequency = mul(mul(h.scale, kFrac1Pi), 3.0);
    double result = 0.0;
    for (uint64_t o = 0; o < h.octaves; ++o) {
        const double wrap = rnd(mul(kTwo32, frequency));  // an integer period
        const double fixed = mul(wrap, kTwoM32);
        result = add(result, mul(eval2d(h.perm, mul((double)x, fixed), mul((double)y, fixed), wrap), amplitude));
        max_amplitude = add(max_amplitude, amplitude);
        amplitude = mul(amplitude, h.persistence);
        frequency = mul(frequency, 2.0);
    }
    return div(result, max_amplitude);
}

// habitat/wrapping_noise/mod.rs:148-168 get_habitat_at_location
NECSIM_NOISE_FN uint32_t habitat_at(const NoiseHabitat &h, uint32_t x, uint32_t y) {
    if (h.coverage <= 0.0) return 0u;
    if (h.coverage >= 1.0) return 1u;
    return octave_sum(h, x, y) <= h.threshold ? 1u : 0u;
}

}  // namespace noise
}  // namespace necsim
