// ix_device.cuh -- device-side building blocks of the spectral transport (sm_100a).
//
// Every function here is the GPU form of one step of the reference's per-sample
// estimator; the comment on each names the reference file:line whose arithmetic it
// reproduces.  The operation order follows the reference's scalar code (glam's
// left-associated dot products, separate multiply and add, `fmaf` exactly where the
// reference calls `mul_add`).  The library builds this code twice:
//   * IX_EXACT=1 with -fmad=false: no multiply-add contraction, so every step that has
//     no transcendental rounds exactly as the CPU tracer does;
//   * IX_EXACT=0 with contraction, approximate division and square root
//     (-prec-div=false -prec-sqrt=false) and denormal flushing: the fast build, held to
//     the reference's per-function ULP budgets and the statistical image tests.
// Explicit __fdiv_rn (the slab scan's t) is IEEE round-to-nearest in both builds.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/ix_cie_tables.h"
#include "../../include/ix_scene.h"

#ifndef IX_EXACT
#define IX_EXACT 0
#endif

#define IX_DEV __device__ __forceinline__

namespace ix {

// ------------------------------------------------------------------------------------
// Vector type (glam Vec3 scalar order).
// ------------------------------------------------------------------------------------
struct V3 {
    float x, y, z;
};
IX_DEV V3 v3(float x, float y, float z) { return V3{x, y, z}; }
IX_DEV V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
IX_DEV V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
IX_DEV V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
IX_DEV V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
IX_DEV V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
IX_DEV float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
IX_DEV V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
// glam's cross product with each product rounded before the subtraction in both builds
// (no multiply-add contraction): parallel inputs give exactly the zero vector, as on the
// CPU.  For the sites that normalise a cross product or test its length for a degenerate
// frame (a contracted product leaves the other's rounding residual: a nonzero vector in
// an arbitrary direction).
IX_DEV V3 cross_rn(V3 a, V3 b) {
    return v3(__fmul_rn(a.y, b.z) - __fmul_rn(b.y, a.z), __fmul_rn(a.z, b.x) - __fmul_rn(b.z, a.x),
              __fmul_rn(a.x, b.y) - __fmul_rn(b.x, a.y));
}
IX_DEV float length_squared(V3 a) { return dot(a, a); }
// glam normalize: v * (1 / sqrt(dot(v, v))), IEEE divide and sqrt.
IX_DEV V3 normalize(V3 a) {
    float rcp = 1.0f / sqrtf(dot(a, a));
    return a * rcp;
}
// normalize for the refracted directions the companion-termination test compares against
// 1 - 1e-6, with an IEEE square root and divide in both builds (glam's two roundings).
// For two nearly parallel unit vectors that test reads the vectors' lengths more than
// their directions, and an approximate reciprocal square root -- bare, or refined by a
// Newton step -- rounds the length differently often enough to flip ~5 % of the
// reference's match decisions (measured per path); the IEEE form keeps the fast build's
// decisions with the reference's.
IX_DEV V3 normalize_dir(V3 a) {
    const float rcp = __fdiv_rn(1.0f, __fsqrt_rn(dot(a, a)));
    return a * rcp;
}
IX_DEV V3 normalize_or_zero(V3 a) {
    float rcp = 1.0f / sqrtf(dot(a, a));
    if (isfinite(rcp) && rcp > 0.0f) return a * rcp;
    return v3(0.0f, 0.0f, 0.0f);
}
IX_DEV V3 load3(const float* p) { return v3(p[0], p[1], p[2]); }
// f32::clamp: `if x < lo {lo}`, then `if x > hi {hi}`.
IX_DEV float clampf_(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
// f32::midpoint on x86_64 rounds (a + b) / 2 once; for finite operands whose sum is a
// normal number (every use here: squared amplitudes in [0, 4]) halving a correctly
// rounded sum is that same value.
IX_DEV float midpointf_(float a, float b) { return (a + b) * 0.5f; }

// ------------------------------------------------------------------------------------
// Stokes vectors and the Mueller matrices the transport applies
// (optics/polarization.rs:117-191).  The matrices are sparse; only their non-zero
// entries are multiplied, in glam's Mat4 * Vec4 column order.
// ------------------------------------------------------------------------------------
struct Stokes {
    float i, q, u, v;
};
IX_DEV float intensity(const Stokes& s) { return fmaxf(s.i, 0.0f); }
IX_DEV Stokes scale(const Stokes& s, float k) {
    return Stokes{s.i * k, s.q * k, s.u * k, s.v * k};
}
// frame_rotation(psi): cols (1,0,0,0), (0,c2,-s2,0), (0,s2,c2,0), (0,0,0,1).
IX_DEV Stokes rotate(const Stokes& s, float c2, float s2) {
    return Stokes{s.i, c2 * s.q + s2 * s.u, (-s2) * s.q + c2 * s.u, s.v};
}
// fresnel_reflection / fresnel_transmission share the (a, b, c) form
// cols (a,b,0,0), (b,a,0,0), (0,0,c,0), (0,0,0,c).
IX_DEV Stokes apply_abc(const Stokes& s, float a, float b, float c) {
    return Stokes{a * s.i + b * s.q, b * s.i + a * s.q, c * s.u, c * s.v};
}
// MuellerMatrix::fresnel_reflection (polarization.rs:148).
IX_DEV Stokes fresnel_reflect_apply(const Stokes& s, float r_s, float r_p) {
    float rs2 = r_s * r_s;
    float rp2 = r_p * r_p;
    float a = midpointf_(rs2, rp2);
    float b = 0.5f * (rs2 - rp2);
    float c = r_s * r_p;
    return apply_abc(s, a, b, c);
}
// MuellerMatrix::fresnel_transmission (polarization.rs:162).
IX_DEV Stokes fresnel_transmit_apply(const Stokes& s, float n1, float n2, float cos_i,
                                     float cos_t, float t_s, float t_p) {
    float factor = (n2 * cos_t) / fmaxf(n1 * cos_i, 1e-6f);
    float ts2 = t_s * t_s * factor;
    float tp2 = t_p * t_p * factor;
    float a = midpointf_(ts2, tp2);
    float b = 0.5f * (ts2 - tp2);
    float c = t_s * t_p * factor;
    return apply_abc(s, a, b, c);
}
// MuellerMatrix::tir_retardation (polarization.rs:184):
// cols (1,0,0,0), (0,1,0,0), (0,0,cd,-sd), (0,0,sd,cd).
// sin and cos of an f32 angle, each rounded to f32 from a double evaluation: the
// correctly rounded values in all but the rarest cases, which is what a correctly
// rounding host libm returns.
IX_DEV void sincos_f32_rounded(float x, float* s, float* c) {
    double sd, cd;
    sincos((double)x, &sd, &cd);
    *s = (float)sd;
    *c = (float)cd;
}
IX_DEV Stokes tir_retard_apply(const Stokes& s, float delta) {
    float sd, cd;
    sincos_f32_rounded(delta, &sd, &cd);
    return Stokes{s.i, s.q, cd * s.u + sd * s.v, (-sd) * s.u + cd * s.v};
}
// cos 2psi and sin 2psi of the frame-rotation angle psi = atan2(s, c)
// (raytracer/absorption.rs:47, polarization.rs:138).  The exact build forms psi and its
// sincos as the reference does, each step rounded to f32 from double as a correctly
// rounding libm would; the fast build uses the double-angle identities
// cos 2psi = (c^2 - s^2) / (c^2 + s^2), sin 2psi = 2cs / (c^2 + s^2), which need no
// transcendental (and give psi = 0 for c = s = 0, as atan2 does).
IX_DEV void rotation_2psi(float sin_psi, float cos_psi, float& c2, float& s2) {
#if IX_EXACT
    // psi and sin / cos of 2 psi, each rounded to f32 from double (see sincos_f32_rounded).
    const float psi = (float)atan2((double)sin_psi, (double)cos_psi);
    sincos_f32_rounded(2.0f * psi, &s2, &c2);
#else
    const float nn = fmaf(cos_psi, cos_psi, sin_psi * sin_psi);
    if (nn > 0.0f) {
        const float inv = 1.0f / nn;
        c2 = fmaf(cos_psi, cos_psi, -(sin_psi * sin_psi)) * inv;
        s2 = ((2.0f * cos_psi) * sin_psi) * inv;
    } else {
        c2 = 1.0f;
        s2 = 0.0f;
    }
#endif
}

// ------------------------------------------------------------------------------------
// Sampler (optics/raytracer/sampling.rs).
// ------------------------------------------------------------------------------------
constexpr uint32_t FRESNEL_BRANCH_STREAM = 0x9E3779B1u;            // sampling.rs:13
constexpr uint32_t RUSSIAN_ROULETTE_STREAM = 0x517CC1B7u;          // sampling.rs:14
constexpr uint32_t PIXEL_JITTER_X_ROTATION_STREAM = 0xA511E9B3u;   // sampling.rs:95
constexpr uint32_t PIXEL_JITTER_Y_ROTATION_STREAM = 0x63D81B23u;   // sampling.rs:97
constexpr uint32_t HERO_WAVELENGTH_ROTATION_STREAM = 0x1B873593u;  // sampling.rs:99

// hash_u32 (sampling.rs:66).
IX_DEV uint32_t hash_u32(uint32_t x) {
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    x *= 0xC2B2AE35u;
    x ^= x >> 16;
    return x;
}
// `(h as f32) / 4_294_967_295.0` -- the divisor rounds to 2^32, so the quotient is the
// exact scaling of the round-to-nearest conversion.
IX_DEV float unit_from_hash(uint32_t h) { return __uint2float_rn(h) * 2.3283064365386963e-10f; }
IX_DEV float unit_draw(uint32_t seed, uint32_t bounce, uint32_t stream) {
    return unit_from_hash(hash_u32(seed ^ hash_u32(bounce ^ stream)));
}
// low_discrepancy_base2 (sampling.rs:110).
IX_DEV float low_discrepancy_base2(uint32_t n) {
    return __uint2float_rn(__brev(n)) * 2.3283064365386963e-10f;
}
// radical_inverse_base (sampling.rs:127) accumulates digit * inv_base with a fused
// multiply-add and divides inv_base by the base after every digit.  Those weights,
// w_0 = 1/B and w_{k+1} = w_k / B, each an IEEE round-to-nearest quotient, depend on the
// base alone: they are evaluated once, at compile time, for the bases the sampler uses
// (N covers every digit of a u32: 21 in base 3, 14 in base 5).
template <uint32_t B, int N>
struct DigitWeights {
    float w[N];
    constexpr DigitWeights() : w() {
        float x = 1.0f / (float)B;
        for (int k = 0; k < N; ++k) {
            w[k] = x;
            x = x / (float)B;
        }
    }
};
static __constant__ DigitWeights<3, 21> c_weights3;
static __constant__ DigitWeights<5, 14> c_weights5;
// radical_inverse_base for base 3 or 5: the same fused accumulation with the weights read
// from the table instead of a division per digit (bit-identical).  The digit index
// advances in step across a warp, so the constant-cache reads broadcast.
template <uint32_t B>
IX_DEV float radical_inverse_table(uint32_t n) {
    const float* w = (B == 3) ? c_weights3.w : c_weights5.w;
    uint32_t remaining = n;
    float val = 0.0f;
    for (int k = 0; remaining > 0; ++k) {
        const uint32_t digit = remaining % B;
        val = fmaf(__uint2float_rn(digit), w[k], val);
        remaining /= B;
    }
    return val;
}
// cranley_patterson_rotate (sampling.rs:148).
IX_DEV float cranley_patterson_rotate(float x, float offset) {
    float sum = x + offset;
    return sum - floorf(sum);
}
struct Draws {
    uint32_t seed;
    float jx, jy, hero;
};
// pixel_rotations (sampling.rs:176) + sample_draws (sampling.rs:206).
IX_DEV Draws sample_draws(uint32_t pixel, uint32_t sample) {
    float rx = low_discrepancy_base2(hash_u32(pixel ^ PIXEL_JITTER_X_ROTATION_STREAM));
    float ry = low_discrepancy_base2(hash_u32(pixel ^ PIXEL_JITTER_Y_ROTATION_STREAM));
    float rh = low_discrepancy_base2(hash_u32(pixel ^ HERO_WAVELENGTH_ROTATION_STREAM));
    Draws d;
    d.seed = hash_u32((pixel * 0x9E3779B9u) ^ (sample * 0x85EBCA6Bu));
    d.jx = cranley_patterson_rotate(low_discrepancy_base2(sample), rx) - 0.5f;
    d.jy = cranley_patterson_rotate(radical_inverse_table<3>(sample), ry) - 0.5f;
    d.hero = cranley_patterson_rotate(radical_inverse_table<5>(sample), rh);
    return d;
}

// ------------------------------------------------------------------------------------
// Camera (camera.rs:149) and the hero comb (transport/mod.rs:58).
// ------------------------------------------------------------------------------------
struct Ray {
    V3 origin, dir;
};
// IEEE divides and square root in both builds (once per path; the camera ray is held to
// the reference's bits in the exact build and its 64-ULP budget in the fast one).
IX_DEV Ray generate_ray(const ix_camera& c, float sx, float sy, float w, float h, float jx,
                        float jy) {
    float aspect = __fdiv_rn(w, h);
    float u = (__fdiv_rn(sx + jx, w) - 0.5f) * 2.0f * aspect * c.fov_tan;
    float v = (0.5f - __fdiv_rn(sy + jy, h)) * 2.0f * c.fov_tan;
    V3 d = load3(c.forward) + load3(c.right) * u + load3(c.up) * v;
    V3 dir = d * __fdiv_rn(1.0f, __fsqrt_rn(dot(d, d)));
    return Ray{load3(c.origin), dir};
}
// f32::rem_euclid(a, 400).  The remainder is exact; for 0 <= a < 800 it is a or a - 400
// (exact by Sterbenz's lemma), which covers every offset of the hero comb, so fmodf runs
// only for inputs outside that range.
IX_DEV float rem_euclid_400(float a) {
    if (a >= 0.0f && a < 800.0f) return a < 400.0f ? a : a - 400.0f;
    float r = fmodf(a, 400.0f);
    return (r < 0.0f) ? r + 400.0f : r;
}
IX_DEV void hero_wavelengths(float hero_rand, float out[8]) {
    float lambda_hero = fmaf(hero_rand, 400.0f, 380.0f);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float offset = fmaf((float)k, 50.0f, lambda_hero - 380.0f);
        out[k] = 380.0f + rem_euclid_400(offset);
    }
}

// ------------------------------------------------------------------------------------
// Dispersion (optics/dispersion.rs:149-210).
// ------------------------------------------------------------------------------------
IX_DEV float dispersion_unclamped(const ix_dispersion& d, float lambda_nm) {
    float um = lambda_nm * 1e-3f;
    float l2 = um * um;
    if (d.kind == IX_DISP_SELLMEIER1) {
        float n2 = 1.0f + (d.b[0] * l2) / (l2 - d.c[0]);
        return sqrtf(fmaxf(n2, 1.0f));
    }
    if (d.kind == IX_DISP_SELLMEIER3) {
        float n2 = 1.0f;
        n2 += (d.b[0] * l2) / (l2 - d.c[0]);
        n2 += (d.b[1] * l2) / (l2 - d.c[1]);
        n2 += (d.b[2] * l2) / (l2 - d.c[2]);
        return sqrtf(fmaxf(n2, 1.0f));
    }
    float l4 = l2 * l2;
    return fmaxf((d.b[0] + d.b[1] / l2) + d.b[2] / l4, 1.0f);
}
IX_DEV float dispersion_min_valid_nm(const ix_dispersion& d) {
    if (d.kind == IX_DISP_CAUCHY) return 380.0f;
    int n = (d.kind == IX_DISP_SELLMEIER1) ? 1 : 3;
    float floor_nm = 300.0f;
    for (int i = 0; i < n; ++i) {
        float c = d.c[i];
        if (c > 0.0f) {
            float pole = sqrtf(c) * 1e3f;
            if (pole < 380.0f) floor_nm = fmaxf(floor_nm, pole * 1.05f);
        }
    }
    return fminf(floor_nm, 380.0f);
}
IX_DEV float dispersion_eval(const ix_dispersion& d, float lambda_nm) {
    if (lambda_nm < 380.0f)
        return dispersion_unclamped(d, fmaxf(lambda_nm, dispersion_min_valid_nm(d)));
    return dispersion_unclamped(d, lambda_nm);
}

// ------------------------------------------------------------------------------------
// Absorption alpha(lambda): Gaussian bands (optics/absorption.rs:108) plus the uniform
// Catmull-Rom knot table (ix_scene.h), and the Cephes-style exponential the reference
// applies per channel (simd/exp_poly.rs:37, its own constants).
// ------------------------------------------------------------------------------------
IX_DEV float band_eval(const ix_band& b, float lambda_nm) {
    if (b.shape == IX_BAND_GAUSS_WAVELENGTH) {
        float t = (lambda_nm - b.center_nm) / b.width_nm;
        return b.peak * expf(-0.5f * t * t);
    }
    float delta_nm = b.center_nm - lambda_nm;
    float nu_diff = 1.0e7f * delta_nm / (lambda_nm * b.center_nm);
    float t = nu_diff / b.width_nm;
    return b.peak * expf(-0.5f * t * t);
}
IX_DEV float spline_eval(const float* knots, float lambda_nm) {
    const int n = IX_SPLINE_KNOTS;
    float pos = (clampf_(lambda_nm, 380.0f, 780.0f) - 380.0f) * ((float)(n - 1) / 400.0f);
    int s = (int)floorf(pos);
    s = s > n - 2 ? n - 2 : (s < 0 ? 0 : s);
    float t = pos - (float)s;
    float p0 = knots[s > 0 ? s - 1 : 0];
    float p1 = knots[s];
    float p2 = knots[s + 1];
    float p3 = knots[s + 2 < n ? s + 2 : n - 1];
    float a = 3.0f * p1 - p0 - 3.0f * p2 + p3;
    float b = 2.0f * p0 - 5.0f * p1 + 4.0f * p2 - p3;
    float c = p2 - p0;
    float poly = fmaf(fmaf(fmaf(a, t, b), t, c), t, 2.0f * p1);
    return fmaxf(0.5f * poly, 0.0f);
}
IX_DEV float spectral_absorption(const ix_absorption& a, float lambda_nm) {
    float sum = 0.0f;
    bool first = true;
    for (uint32_t i = 0; i < a.n_bands && i < IX_MAX_BANDS; ++i) {
        float v = band_eval(a.bands[i], lambda_nm);
        sum = first ? v : sum + v;
        first = false;
    }
    if (a.has_spline) {
        float v = spline_eval(a.spline, lambda_nm);
        sum = first ? v : sum + v;
    }
    return sum;
}
IX_DEV float exp_lane(float x) {
    const float LOG2E = 1.44269504088896340736f;
    const float C1 = __uint_as_float(0x3F318000u);
    const float C2 = -2.1219444e-4f;
    float upper = (x < 88.02875f) ? x : 88.02875f;
    x = (upper > -87.33654f) ? upper : -87.33654f;
    float n = floorf(fmaf(x, LOG2E, 0.5f));
    x = fmaf(n, -C1, x);
    x = fmaf(n, -C2, x);
    float z = x * x;
    float p = 1.9875691e-4f;
    p = fmaf(p, x, 1.3981999e-3f);
    p = fmaf(p, x, 8.333452e-3f);
    p = fmaf(p, x, 4.1665796e-2f);
    p = fmaf(p, x, 1.6666665e-1f);
    p = fmaf(p, x, 5.0000003e-1f);
    p = fmaf(p, z, x) + 1.0f;
    int e = (int)n;
    return p * __int_as_float((e + 127) << 23);
}

// ------------------------------------------------------------------------------------
// Colour tables and spectral integration (color/cie1931.rs:157; environment/spectral.rs:28).
// ------------------------------------------------------------------------------------
// In global memory, read through the read-only data cache: the 8 channels of a path look
// up 8 different wavelengths, which the constant cache would serialise.
static __device__ const float c_cmf[81][3] = IX_CIE1931_CMF_INIT;
static __device__ const float c_d65[41] = IX_CIE_D65_SPD_INIT;
static __device__ const float c_d65_uv[9] = IX_CIE_D65_UV_SPD_INIT;

IX_DEV V3 cmf(float lambda_nm) {
    if (!(lambda_nm >= 380.0f && lambda_nm <= 780.0f)) return v3(0.0f, 0.0f, 0.0f);
    float position = (lambda_nm - 380.0f) / 5.0f;
    int i0 = (int)floorf(position);
    i0 = i0 > 79 ? 79 : i0;
    float t = position - (float)i0;
    float l0 = __ldg(&c_cmf[i0][0]), l1 = __ldg(&c_cmf[i0][1]), l2 = __ldg(&c_cmf[i0][2]);
    float h0 = __ldg(&c_cmf[i0 + 1][0]), h1 = __ldg(&c_cmf[i0 + 1][1]), h2 = __ldg(&c_cmf[i0 + 1][2]);
    return v3(l0 + (h0 - l0) * t, l1 + (h1 - l1) * t, l2 + (h2 - l2) * t);
}
IX_DEV float d65(float lambda_nm) {
    if (lambda_nm < 380.0f) {
        float clamped = fmaxf(lambda_nm, 300.0f);
        float position = (clamped - 300.0f) / 10.0f;
        int i0 = (int)floorf(position);
        i0 = i0 > 7 ? 7 : i0;
        float frac = position - (float)i0;
        float v0 = __ldg(&c_d65_uv[i0]), v1 = __ldg(&c_d65_uv[i0 + 1]);
        return fmaf(frac, v1 - v0, v0) / 100.0f;
    }
    float clamped = clampf_(lambda_nm, 380.0f, 780.0f);
    float position = (clamped - 380.0f) / 10.0f;
    int i0 = (int)floorf(position);
    i0 = i0 > 39 ? 39 : i0;
    float frac = position - (float)i0;
    float v0 = __ldg(&c_d65[i0]), v1 = __ldg(&c_d65[i0 + 1]);
    return fmaf(frac, v1 - v0, v0) / 100.0f;
}
// powi with a constant exponent: x^(2^i) factors multiplied in ascending bit order.
IX_DEV float powi5(float x) {
    float x2 = x * x;
    return x * (x2 * x2);
}
IX_DEV float powi6(float x) {
    float x2 = x * x;
    return x2 * (x2 * x2);
}
IX_DEV float powi18(float x) {
    float x2 = x * x, x4 = x2 * x2, x8 = x4 * x4, x16 = x8 * x8;
    return x2 * x16;
}
IX_DEV float powi28(float x) {
    float x2 = x * x, x4 = x2 * x2, x8 = x4 * x4, x16 = x8 * x8;
    return (x4 * x8) * x16;
}
// blackbody_spectrum_with (environment/spectral.rs:62).
IX_DEV float blackbody(float t_k, float denom_560, float lambda_nm) {
    float exp_val = expf(fminf(14388000.0f / (lambda_nm * t_k), 80.0f));
    float denom = fmaxf(exp_val - 1.0f, 1e-6f);
    float ratio = denom_560 / denom;
    return clampf_(powi5(560.0f / lambda_nm) * ratio, 0.01f, 20.0f);
}
IX_DEV float spectral_power(const ix_environment& env, float lambda_nm) {
    if (env.spectrum == IX_SPEC_D65) return d65(lambda_nm);
    if (env.spectrum == IX_SPEC_BLACKBODY) return blackbody(env.bb_t_k, env.bb_denom_560, lambda_nm);
    return 1.0f;
}
// ... with the UV lamps' line and the ASET view's wavelength input (spectral.rs:137,
// rig.rs:165): the extended lookup's.
IX_DEV float spectral_power_ext(const ix_environment& env, float lambda_nm) {
    if (env.spectrum == IX_SPEC_GAUSSIAN) {
        const float z = (lambda_nm - env.line_centre_nm) / env.line_sigma_nm;
        return expf((-0.5f * z) * z);
    }
    if (env.spectrum == IX_SPEC_WAVELENGTH) return lambda_nm;
    return spectral_power(env, lambda_nm);
}

// ------------------------------------------------------------------------------------
// Environment (environment/rig.rs:67-377): the direction-only lighting, then the
// per-wavelength radiance built from it.
// ------------------------------------------------------------------------------------
IX_DEV float smoothstep_(float e0, float e1, float x) {
    float t = clampf_((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * fmaf(-2.0f, t, 3.0f);
}
struct Lighting {
    float factor;  // scaled models: radiance = factor * (spec * exposure)
    float bg, softbox, fill, ground, horizon;
    float ring[4];
    int ring_len;  // ring emitters lit for this direction (at most 4 overlap)
    bool has_softbox, has_fill, has_ground;
};
// The tent, dome, sun and ASET constants (rig.rs:67-85, :120-135, sun.rs:10-20).
constexpr float TENT_KEY_OUTER_COS = 0.7660444f, TENT_KEY_INNER_COS = 0.9396926f;
constexpr float SPARK_OUTER_COS = 0.9961947f, SPARK_INNER_COS = 0.9993908f;
constexpr float CARD_OUTER_COS = 0.898794f, CARD_INNER_COS = 0.9612617f;
constexpr float ASET_SIGMA_NM = 8.493218f;
constexpr float ASET_EDGE_45_LO = 0.6871068f, ASET_EDGE_45_HI = 0.7271068f;
constexpr float ASET_EDGE_75_LO = 0.9459258f, ASET_EDGE_75_HI = 0.9859258f;
constexpr float SUN_DISC_COS = 0.9999889f;
IX_DEV float aset_band(float lambda_nm, float centre_nm) {
    const float z = (lambda_nm - centre_nm) / ASET_SIGMA_NM;
    return expf((-0.5f * z) * z);
}
// The scaled and banded models other than the iso-hemisphere (rig.rs:254-310, :439-500):
// returns the Scaled factor for the tent, dome and sun; for the ASET view the three zone
// weights and the tray's ground in *bands (the radiance is banded at lookup time).
IX_DEV float other_model_lighting(const ix_environment& env, V3 d, V3 observer, float* bands) {
    const float tray = env.backdrop;
    const float horizon = smoothstep_(-0.05f, 0.05f, d.y);
    const float vis = 1.0f - smoothstep_(env.shadow_cos[0], env.shadow_cos[1], dot(d, observer));
    auto lit_ground = [&](float own) {
        return tray > 0.0f ? ((1.0f - horizon) * vis) * tray : own * (1.0f - horizon);
    };
    if (env.model == IX_ENV_LIGHT_TENT) {
        float walls = fmaf(0.08f, fmaxf(d.y, 0.0f), 0.14f) * env.tent_walls;
        if (env.tent_flat > 0.0f) walls = fmaf(0.18f * env.tent_walls, env.tent_flat, walls * (1.0f - env.tent_flat));
        float card = 0.0f;
#pragma unroll
        for (int slot = 4; slot <= 12; slot += 4)
            card = fmaxf(card, smoothstep_(CARD_OUTER_COS, CARD_INNER_COS, dot(d, load3(env.ring_dirs[slot]))));
        walls = walls * fmaf(card * env.tent_cards, -0.9f, 1.0f);
        const float key = smoothstep_(TENT_KEY_OUTER_COS, TENT_KEY_INNER_COS, dot(d, load3(env.key_dir))) *
                          (1.4f * env.spot_mult);
        const float spark = (smoothstep_(SPARK_OUTER_COS, SPARK_INNER_COS, dot(d, load3(env.fill_dir))) *
                             (5.0f * env.spot_mult)) * env.tent_spark;
        return ((walls + key) + spark) * (horizon * vis) + lit_ground(env.tent_ground);
    }
    if (env.model == IX_ENV_ASET) {
        const float s45 = smoothstep_(ASET_EDGE_45_LO, ASET_EDGE_45_HI, d.y);
        const float s75 = smoothstep_(ASET_EDGE_75_LO, ASET_EDGE_75_HI, d.y);
        bands[0] = (s45 * (1.0f - s75)) * horizon;
        bands[1] = (1.0f - s45) * horizon;
        bands[2] = s75 * horizon;
        bands[3] = tray > 0.0f ? (1.0f - horizon) * tray : 0.0f;
        return 0.0f;
    }
    // DaylightDome and DaylightSun: the sky, its aureole about the sun, and the sun's disc.
    const float sun_dot = dot(d, load3(env.key_dir));
    const float sky = fmaf(0.08f, 1.0f - fmaxf(d.y, 0.0f), 0.10f);
    const float glow = fmaxf(sun_dot, 0.0f);
    const float glow2 = glow * glow;
    const float glow4 = glow2 * glow2;
    const float aureole = (glow4 * glow4) * 0.30f;
    const float sum = (sky + aureole) * (horizon * vis) + lit_ground(0.04f);
    if (env.model == IX_ENV_DAYLIGHT_DOME) return sum;
    return sum + (sun_dot >= SUN_DISC_COS ? env.sun_factor : 0.0f);
}
IX_DEV Lighting direction_lighting(const ix_environment& env, V3 dir, V3 observer) {
    Lighting L;
    L.factor = 0.0f;
    L.ring_len = 0;
    L.has_softbox = L.has_fill = L.has_ground = false;
    L.bg = L.softbox = L.fill = L.ground = L.horizon = 0.0f;
    if (env.model == IX_ENV_UNIFORM) return L;
    V3 d = normalize(dir);
    float tray = env.backdrop;
    if (env.model == IX_ENV_ISO_HEMISPHERE) {
        float horizon = smoothstep_(-0.05f, 0.05f, d.y);
        float vis = 1.0f - smoothstep_(env.shadow_cos[0], env.shadow_cos[1], dot(d, observer));
        L.factor = (tray > 0.0f) ? fmaf((1.0f - horizon) * vis, tray, horizon * vis) : horizon * vis;
        return L;
    }

    float exposure = env.exposure;
    float spot = env.spot_mult;
    L.bg = env.ambient_fill ? fmaxf(fmaf(0.012f, fmaf(d.y, 0.5f, 0.5f), 0.015f), 0.005f) * exposure
                            : 0.0f;
    float key_dot = fmaxf(dot(d, load3(env.key_dir)), 0.0f);
    if (key_dot > 0.0f) {
        L.has_softbox = true;
        L.softbox = powi28(key_dot) * 12.0f * spot * exposure;
    }
    float fill_dot = fmaxf(dot(d, load3(env.fill_dir)), 0.0f);
    if (fill_dot > 0.0f) {
        L.has_fill = true;
        L.fill = powi18(fill_dot) * 4.5f * exposure;
    }
    for (int i = 0; i < IX_RING_LIGHTS; ++i) {
        float ring_dot = fmaxf(dot(d, load3(env.ring_dirs[i])), 0.0f);
        if (ring_dot > 0.96f && L.ring_len < 4) {
            float spark = (ring_dot - 0.96f) / 0.04f;
            L.ring[L.ring_len++] = powi6(spark) * 22.0f * spot * exposure;
        }
    }
    if (tray > 0.0f) {
        L.has_ground = true;
        L.horizon = smoothstep_(-0.05f, 0.05f, d.y);
        L.ground = ((1.0f - L.horizon) * tray) * exposure;
    }
    return L;
}
IX_DEV float lighting_radiance(const Lighting& L, const ix_environment& env, float spec) {
    if (env.model == IX_ENV_UNIFORM) return env.uniform_radiance * spec;
    if (env.model != IX_ENV_STUDIO) return L.factor * (spec * env.exposure);
    float r = L.bg * spec;
    if (L.has_softbox) r = fmaf(L.softbox, spec, r);
    if (L.has_fill) r = fmaf(L.fill, spec, r);
    for (int i = 0; i < L.ring_len; ++i) r = fmaf(L.ring[i], spec, r);
    if (L.has_ground) return fmaf(L.horizon, r, L.ground * spec);
    return r;
}

// The escape radiance for every lighting model (sample_studio_environment_channels,
// rig.rs:701): the studio rig, iso-hemisphere and uniform dome as direction_lighting /
// lighting_radiance form them, the tent, dome, sun and ASET models beside them.  Only the
// extended transport instantiation calls it, so the other instantiations' escape lookup
// (and, through the interprocedural register allocation, their kernels) is unchanged.
IX_DEV float environment_radiance_ext(const ix_environment& env, V3 dir, V3 observer, float lambda) {
    const float spec = spectral_power_ext(env, lambda);
    if (env.model == IX_ENV_STUDIO || env.model == IX_ENV_ISO_HEMISPHERE || env.model == IX_ENV_UNIFORM)
        return lighting_radiance(direction_lighting(env, dir, observer), env, spec);
    float bands[4];
    const float factor = other_model_lighting(env, normalize(dir), observer, bands);
    if (env.model != IX_ENV_ASET) return factor * (spec * env.exposure);
    // DirectionLighting::Banded (rig.rs:140): `spec` is the wavelength.
    const float r = (bands[0] * aset_band(spec, 610.0f)) * 8.0f;
    const float g = (bands[1] * aset_band(spec, 540.0f)) * 5.0f;
    const float b = (bands[2] * aset_band(spec, 460.0f)) * 16.0f;
    const float zones = ((r + g) + b) * env.exposure;
    return bands[3] > 0.0f ? fmaf(bands[3] * d65(spec), env.exposure, zones) : zones;
}

// RadianceSource::radiance (color/metrics/lighting.rs:93) of the models past the studio rig
// and the iso-hemisphere (tent, dome, sun): the extended lookup at 550 nm with no observer.
// Out of line: the kernels that may meet either kind of model call it from a branch.
static __device__ __noinline__ float exit_radiance_ext(const ix_environment& env, V3 dir) {
    return environment_radiance_ext(env, dir, v3(0.0f, 0.0f, 0.0f), 550.0f);
}
// The scoring radiance along `dir`: the rig's direction lighting at the host's 550 nm
// power `spec` (SCORE_RIG: the studio rigs and the iso-hemisphere), the extended lookup
// (SCORE_EXT: every other model), or either by the environment's model (SCORE_ANY).  The
// metrics kernel is built for the first two, so the rig's instantiation compiles as it
// does without the extended lookup.
enum ScoreKind { SCORE_RIG = 0, SCORE_EXT = 1, SCORE_ANY = 2 };
__host__ __device__ __forceinline__ bool rig_scored(const ix_environment& env) {
    return env.model == IX_ENV_STUDIO || env.model == IX_ENV_ISO_HEMISPHERE;
}
template <int SCORE>
IX_DEV float exit_radiance(const ix_environment& env, float spec, V3 dir) {
    if constexpr (SCORE == SCORE_EXT) {
        return exit_radiance_ext(env, dir);
    } else {
        if constexpr (SCORE == SCORE_ANY)
            if (!rig_scored(env)) return exit_radiance_ext(env, dir);
        return lighting_radiance(direction_lighting(env, dir, v3(0.0f, 0.0f, 0.0f)), env, spec);
    }
}

// ExitLighting (color/metrics/lighting.rs:137-209) and returned_or_reason
// (visibility.rs:55): the metrics' verdict on a direction leaving the stone.  `env` is the
// scoring environment (the preset at exposure 1, no tray), `spec` its 550 nm power.
template <int SCORE>
struct ExitScorerT {
    const ix_environment& env;
    float spec, threshold, head_shadow_cos;
    // is_illuminated (lighting.rs:207): the scoring light's radiance along `dir`.
    IX_DEV bool lit(V3 dir) const { return exit_radiance<SCORE>(env, spec, dir) > threshold; }
    // Exits closer to the eye than the head-shadow cone are lost to the observer.
    IX_DEV bool shadowed(V3 exit_dir, V3 observer) const { return dot(exit_dir, observer) > head_shadow_cos; }
    // ray_is_visibly_returned (visibility.rs:78) for an observer at -forward.
    IX_DEV bool returned(V3 exit_dir, V3 forward) const {
        if (shadowed(exit_dir, -forward)) return false;
        return lit(exit_dir);
    }
};
using ExitScorer = ExitScorerT<SCORE_ANY>;

// ambient_level (lighting.rs:101) scaled by SOURCE_OVER_AMBIENT or
// UNIFORM_FRACTION_OF_AMBIENT (`factor`) and floored at the least positive normal
// (lighting.rs:186): the median of the radiances along the 96 hemisphere directions.
// Block-wide: every thread of the block calls it; `s_rad` is 96 floats of shared memory.
template <int SCORE>
IX_DEV float exit_lighting_threshold(const ix_environment& env, float spec, float factor, const float (*dirs)[3],
                                     float* s_rad, float* s_threshold) {
    for (int i = threadIdx.x; i < 96; i += blockDim.x) {
        const V3 d = v3(dirs[i][0], dirs[i][1], dirs[i][2]);
        s_rad[i] = exit_radiance<SCORE>(env, spec, d);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < 96; ++i) {  // insertion sort, ascending
            const float v = s_rad[i];
            int j = i - 1;
            while (j >= 0 && s_rad[j] > v) {
                s_rad[j + 1] = s_rad[j];
                --j;
            }
            s_rad[j + 1] = v;
        }
        *s_threshold = fmaxf(s_rad[48] * factor, 1.17549435e-38f);
    }
    __syncthreads();
    return *s_threshold;
}

// ------------------------------------------------------------------------------------
// Convex slab intersection over the CTA's shared-memory plane cache
// (simd/slab.rs:120-160; intersect.rs:101-127).
// ------------------------------------------------------------------------------------
struct Hit {
    float t;
    int facet;  // -1: no hit
};
//
// The reference divides t = -side / denom for every plane.  Here the IEEE quotient is
// formed only for candidate planes, with no change to any result: for an entering
// plane (denom < 0) the update `RN(q) > t_near` (q = -side / denom exactly) needs
// q > t_near, i.e. t_near * denom + side > 0; for an exiting plane (denom > 0)
// `RN(q) < t_far` needs t_far * denom + side > 0.  One fused multiply-add rounds that
// expression once, which keeps its sign (a positive value can only round to +0, so the
// test is `>= 0`), so every plane the reference would select passes the filter, and the
// exact division and comparison then decide exactly as the reference does.
IX_DEV Hit intersect_planes(const float4* __restrict__ planes, int n, V3 o, V3 d) {
    float t_near = -1e30f, t_far = 1e30f;
    int near_idx = -1, far_idx = -1;
    bool outside = false;
#pragma unroll 4
    for (int i = 0; i < n; ++i) {
        float4 p = planes[i];
        float denom = (p.x * d.x + p.y * d.y) + p.z * d.z;
        float side = p.w + ((p.x * o.x + p.y * o.y) + p.z * o.z);
        if (fabsf(denom) > 1e-7f) {
            // An entering plane the origin is not outside of cannot make the entry (t <= 0)
            // and an exiting plane the origin is outside of makes the scan a miss: neither
            // needs its division (the argument is spelled out at group_intersect).
            const bool entering = denom < 0.0f;
            if (!entering && side > 0.0f) {
                outside = true;
                break;
            }
            const float bound = entering ? t_near : t_far;
            if ((side > 0.0f || !entering) && fmaf(bound, denom, side) >= 0.0f) {
                const float t = __fdiv_rn(-side, denom);
                if (entering) {
                    if (t > t_near) {
                        t_near = t;
                        near_idx = i;
                    }
                } else if (t < t_far) {
                    t_far = t;
                    far_idx = i;
                }
            }
        } else if (side > 0.0f) {
            outside = true;
            break;
        }
    }
    Hit h;
    h.facet = -1;
    h.t = 0.0f;
    if (outside || t_near > t_far) return h;
    if (t_near > 1e-4f) {
        h.t = t_near;
        h.facet = near_idx >= 0 ? near_idx : 0;
    } else if (t_far > 1e-4f) {
        h.t = t_far;
        h.facet = far_idx >= 0 ? far_idx : 0;
    }
    return h;
}

}  // namespace ix
