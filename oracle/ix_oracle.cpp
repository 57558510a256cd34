// ix_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the CPU oracle.
//
// A C++ restatement of the reference's CPU spectral tracer, used by the test suite as
// the parity checker and by the benchmark as the reported CPU baseline.  It is never
// linked into, loaded by or called from the CUDA backend.
//
// Rounding discipline (the reference's determinism contract, simd/mod.rs:1-27):
//   * built with -ffp-contract=off, so `a * b + c` rounds twice exactly like the Rust
//     source; std::fma is used exactly where the reference calls `mul_add`;
//   * glam's scalar operation order (glam =0.34.1, not vendored): left-associated dot
//     products `(x*x' + y*y') + z*z'`, cross `(y*z' - y'*z, ...)`, normalize as
//     `v * (1 / sqrt(dot(v, v)))`, Mat4 * Vec4 as `((c0*x + c1*y) + c2*z) + c3*w`;
//   * the same libm calls (sinf, cosf, atan2f, atanf, acosf, tanf, expf) that Rust's
//     std makes on Linux;  f32::midpoint through f64 as Rust's core does on x86_64.
// Every function names the reference file:line it restates.
//
// Built twice: normally (F = float) and with -DIX_COUNT_FLOPS, where F is a wrapper
// that tallies every floating-point operation so the algorithmic FLOPs per path can be
// counted on the same inputs the GPU runs.

#include "ix_oracle.h"
#include "../include/ix_cie_tables.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#if defined(IX_ORACLE_AVX2) && !defined(IX_COUNT_FLOPS)
#include <immintrin.h>
#endif
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace ixo {

// ------------------------------------------------------------------------------------
// The scalar type.
// ------------------------------------------------------------------------------------
#ifdef IX_COUNT_FLOPS
struct Counters {
    uint64_t add = 0, mul = 0, fma = 0, div = 0, sqrt = 0, transc = 0;
};
thread_local Counters g_cnt;
struct F {
    float v;
    F() = default;
    F(float x) : v(x) {}  // NOLINT: implicit by design so literals mix freely
};
static inline F operator+(F a, F b) { g_cnt.add++; return F(a.v + b.v); }
static inline F operator-(F a, F b) { g_cnt.add++; return F(a.v - b.v); }
static inline F operator*(F a, F b) { g_cnt.mul++; return F(a.v * b.v); }
static inline F operator/(F a, F b) { g_cnt.div++; return F(a.v / b.v); }
static inline F operator-(F a) { return F(-a.v); }
static inline F& operator+=(F& a, F b) { a = a + b; return a; }
static inline F& operator*=(F& a, F b) { a = a * b; return a; }
static inline F& operator/=(F& a, F b) { a = a / b; return a; }
static inline bool operator<(F a, F b) { return a.v < b.v; }
static inline bool operator>(F a, F b) { return a.v > b.v; }
static inline bool operator<=(F a, F b) { return a.v <= b.v; }
static inline bool operator>=(F a, F b) { return a.v >= b.v; }
static inline bool operator==(F a, F b) { return a.v == b.v; }
static inline bool operator!=(F a, F b) { return a.v != b.v; }
static inline float raw(F x) { return x.v; }
static inline F fma_(F a, F b, F c) { g_cnt.fma++; return F(std::fma(a.v, b.v, c.v)); }
static inline F sqrt_(F a) { g_cnt.sqrt++; return F(std::sqrt(a.v)); }
static inline F sin_(F a) { g_cnt.transc++; return F(sinf(a.v)); }
static inline F cos_(F a) { g_cnt.transc++; return F(cosf(a.v)); }
static inline F tan_(F a) { g_cnt.transc++; return F(tanf(a.v)); }
static inline F atan_(F a) { g_cnt.transc++; return F(atanf(a.v)); }
static inline F atan2_(F a, F b) { g_cnt.transc++; return F(atan2f(a.v, b.v)); }
static inline F acos_(F a) { g_cnt.transc++; return F(acosf(a.v)); }
static inline F exp_(F a) { g_cnt.transc++; return F(expf(a.v)); }
static inline F ln_(F a) { g_cnt.transc++; return F(logf(a.v)); }
static inline F midpoint_(F a, F b) {
    g_cnt.add++; g_cnt.mul++;
    return F((float)(((double)a.v + (double)b.v) / 2.0));
}
#else
using F = float;
static inline float raw(F x) { return x; }
static inline F fma_(F a, F b, F c) { return std::fma(a, b, c); }
static inline F sqrt_(F a) { return std::sqrt(a); }
static inline F sin_(F a) { return sinf(a); }
static inline F cos_(F a) { return cosf(a); }
static inline F tan_(F a) { return tanf(a); }
static inline F atan_(F a) { return atanf(a); }
static inline F atan2_(F a, F b) { return atan2f(a, b); }
static inline F acos_(F a) { return acosf(a); }
static inline F exp_(F a) { return expf(a); }
static inline F ln_(F a) { return logf(a); }
// f32::midpoint on x86_64: ((a as f64 + b as f64) / 2.0) as f32.
static inline F midpoint_(F a, F b) { return (float)(((double)a + (double)b) / 2.0); }
#endif

// f32::max / f32::min are IEEE maxNum/minNum (a NaN operand yields the other one).
static inline F max_(F a, F b) { return F(fmaxf(raw(a), raw(b))); }
static inline F min_(F a, F b) { return F(fminf(raw(a), raw(b))); }
static inline F abs_(F a) { return F(fabsf(raw(a))); }
static inline F floor_(F a) { return F(floorf(raw(a))); }
// f32::clamp: `if x < lo { lo }` then `if x > hi { hi }` (NaN passes through).
static inline F clamp_(F x, F lo, F hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
static inline bool is_finite_(F x) { return std::isfinite(raw(x)); }
static inline F fromu(uint32_t u) { return F((float)u); }

// ------------------------------------------------------------------------------------
// glam Vec3 (scalar operation order).
// ------------------------------------------------------------------------------------
struct V3 {
    F x, y, z;
};
static inline V3 v3(F x, F y, F z) { return V3{x, y, z}; }
static inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
static inline V3 operator*(V3 a, F s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 operator*(F s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
static inline V3 mulv(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline F dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
static inline F length_squared(V3 a) { return dot(a, a); }
static inline V3 normalize(V3 a) {
    F rcp = F(1.0f) / sqrt_(dot(a, a));
    return a * rcp;
}
static inline V3 normalize_or_zero(V3 a) {
    F rcp = F(1.0f) / sqrt_(dot(a, a));
    if (is_finite_(rcp) && rcp > F(0.0f)) return a * rcp;
    return v3(0.0f, 0.0f, 0.0f);
}
static inline V3 vmax0(V3 a) {
    return v3(max_(a.x, 0.0f), max_(a.y, 0.0f), max_(a.z, 0.0f));
}
static inline V3 load3(const float* p) { return v3(p[0], p[1], p[2]); }
static inline void store3(float* p, V3 v) {
    p[0] = raw(v.x);
    p[1] = raw(v.y);
    p[2] = raw(v.z);
}

// ------------------------------------------------------------------------------------
// Stokes vector and the Mueller matrices (optics/polarization.rs:9-191).
// A 4x4 is stored column-major as glam's Mat4 (from_cols_array).
// ------------------------------------------------------------------------------------
struct Stokes {
    F i, q, u, v;
};
struct M4 {
    F c[16];
};
static inline Stokes unpolarized(F i) { return Stokes{i, 0.0f, 0.0f, 0.0f}; }
static inline F intensity(const Stokes& s) { return max_(s.i, 0.0f); }
static inline Stokes scale(const Stokes& s, F k) {
    return Stokes{s.i * k, s.q * k, s.u * k, s.v * k};
}
// glam Mat4::mul_vec4: ((col0*x + col1*y) + col2*z) + col3*w, element-wise.
static inline Stokes apply(const M4& m, const Stokes& s) {
    Stokes o;
    o.i = ((m.c[0] * s.i + m.c[4] * s.q) + m.c[8] * s.u) + m.c[12] * s.v;
    o.q = ((m.c[1] * s.i + m.c[5] * s.q) + m.c[9] * s.u) + m.c[13] * s.v;
    o.u = ((m.c[2] * s.i + m.c[6] * s.q) + m.c[10] * s.u) + m.c[14] * s.v;
    o.v = ((m.c[3] * s.i + m.c[7] * s.q) + m.c[11] * s.u) + m.c[15] * s.v;
    return o;
}
// MuellerMatrix::frame_rotation (polarization.rs:138).
static M4 frame_rotation(F psi) {
    F c2 = cos_(F(2.0f) * psi);
    F s2 = sin_(F(2.0f) * psi);
    return M4{{1.0f, 0.0f, 0.0f, 0.0f, 0.0f, c2, -s2, 0.0f, 0.0f, s2, c2, 0.0f, 0.0f, 0.0f,
               0.0f, 1.0f}};
}
// MuellerMatrix::fresnel_reflection (polarization.rs:148).
static M4 fresnel_reflection(F r_s, F r_p) {
    F rs2 = r_s * r_s;
    F rp2 = r_p * r_p;
    F a = midpoint_(rs2, rp2);
    F b = F(0.5f) * (rs2 - rp2);
    F c = r_s * r_p;
    return M4{{a, b, 0.0f, 0.0f, b, a, 0.0f, 0.0f, 0.0f, 0.0f, c, 0.0f, 0.0f, 0.0f, 0.0f, c}};
}
// MuellerMatrix::fresnel_transmission (polarization.rs:162).
static M4 fresnel_transmission(F n1, F n2, F cos_i, F cos_t, F t_s, F t_p) {
    F factor = (n2 * cos_t) / max_(n1 * cos_i, 1e-6f);
    F ts2 = t_s * t_s * factor;
    F tp2 = t_p * t_p * factor;
    F a = midpoint_(ts2, tp2);
    F b = F(0.5f) * (ts2 - tp2);
    F c = t_s * t_p * factor;
    return M4{{a, b, 0.0f, 0.0f, b, a, 0.0f, 0.0f, 0.0f, 0.0f, c, 0.0f, 0.0f, 0.0f, 0.0f, c}};
}
// MuellerMatrix::tir_retardation (polarization.rs:184).
static M4 tir_retardation(F delta) {
    F cd = cos_(delta);
    F sd = sin_(delta);
    return M4{{1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, cd, -sd, 0.0f, 0.0f,
               sd, cd}};
}

// ------------------------------------------------------------------------------------
// sampling.rs
// ------------------------------------------------------------------------------------
static const uint32_t FRESNEL_BRANCH_STREAM = 0x9E3779B1u;     // sampling.rs:13
static const uint32_t RUSSIAN_ROULETTE_STREAM = 0x517CC1B7u;   // sampling.rs:14
static const uint32_t PIXEL_JITTER_X_ROTATION_STREAM = 0xA511E9B3u;  // sampling.rs:95
static const uint32_t PIXEL_JITTER_Y_ROTATION_STREAM = 0x63D81B23u;  // sampling.rs:97
static const uint32_t HERO_WAVELENGTH_ROTATION_STREAM = 0x1B873593u; // sampling.rs:99

// hash_u32 (sampling.rs:66).
static inline uint32_t hash_u32(uint32_t x) {
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    x *= 0xC2B2AE35u;
    x ^= x >> 16;
    return x;
}
static inline uint32_t reverse_bits(uint32_t v) {
    uint32_t r = 0;
    for (int i = 0; i < 32; ++i) {
        r = (r << 1) | (v & 1u);
        v >>= 1;
    }
    return r;
}
// `(x as f32) / 4_294_967_295.0`: the literal rounds to 2^32 in f32.
static inline F unit_from_hash(uint32_t h) { return fromu(h) / F(4294967296.0f); }
// unit_draw (transport/inner/bounce_body.rs:71-73), the per-bounce stream draw.
constexpr uint32_t FROSTED_NEE_ENV_DIR_U_STREAM = 0x6A09E667u;  // sampling.rs:52
constexpr uint32_t FROSTED_NEE_ENV_DIR_V_STREAM = 0xBB67AE85u;  // sampling.rs:53
static inline F unit_draw(uint32_t seed, uint32_t bounce, uint32_t stream) {
    return unit_from_hash(hash_u32(seed ^ hash_u32(bounce ^ stream)));
}
// low_discrepancy_base2 (sampling.rs:110).
static inline F low_discrepancy_base2(uint32_t n) {
    return fromu(reverse_bits(n)) / F(4294967296.0f);
}
// radical_inverse_base (sampling.rs:127).
static inline F radical_inverse_base(uint32_t n, uint32_t base) {
    uint32_t remaining = n;
    F val = 0.0f;
    F inv_base = F(1.0f) / fromu(base);
    while (remaining > 0) {
        uint32_t digit = remaining % base;
        val = fma_(fromu(digit), inv_base, val);
        inv_base = inv_base / fromu(base);
        remaining /= base;
    }
    return val;
}
// cranley_patterson_rotate (sampling.rs:148).
static inline F cranley_patterson_rotate(F x, F offset) {
    F sum = x + offset;
    return sum - floor_(sum);
}
struct Rot {
    F jx, jy, hero;
};
// pixel_rotations (sampling.rs:176).
static inline Rot pixel_rotations(uint32_t pixel) {
    return Rot{low_discrepancy_base2(hash_u32(pixel ^ PIXEL_JITTER_X_ROTATION_STREAM)),
               low_discrepancy_base2(hash_u32(pixel ^ PIXEL_JITTER_Y_ROTATION_STREAM)),
               low_discrepancy_base2(hash_u32(pixel ^ HERO_WAVELENGTH_ROTATION_STREAM))};
}
struct Draws {
    uint32_t seed;
    F jx, jy, hero;
};
// sample_draws (sampling.rs:206).
static inline Draws sample_draws(uint32_t pixel, uint32_t sample, const Rot& rot) {
    Draws d;
    d.seed = hash_u32((pixel * 0x9E3779B9u) ^ (sample * 0x85EBCA6Bu));
    d.jx = cranley_patterson_rotate(low_discrepancy_base2(sample), rot.jx) - F(0.5f);
    d.jy = cranley_patterson_rotate(radical_inverse_base(sample, 3), rot.jy) - F(0.5f);
    d.hero = cranley_patterson_rotate(radical_inverse_base(sample, 5), rot.hero);
    return d;
}

// ------------------------------------------------------------------------------------
// camera.rs
// ------------------------------------------------------------------------------------
struct Ray {
    V3 origin, dir;
};
// f32::to_radians: self * (PI / 180.0) with the constant rounded to f32.
static inline F to_radians(F deg) {
    return deg * (F(3.14159265358979323846f) / F(180.0f));
}

// Camera::new (camera.rs:108).
static void camera_new(F yaw, F pitch, F distance, F fov_deg, ix_camera* out) {
    F cos_p = cos_(pitch), sin_p = sin_(pitch), cos_y = cos_(yaw), sin_y = sin_(yaw);
    V3 origin = v3(distance * cos_p * sin_y, distance * sin_p, distance * cos_p * cos_y);
    V3 forward = normalize(-origin);
    V3 world_up;
    if (abs_(cos_p) < F(1e-4f))
        world_up = v3(0.0f, 0.0f, -1.0f);
    else if (cos_p < F(0.0f))
        world_up = v3(0.0f, -1.0f, 0.0f);
    else
        world_up = v3(0.0f, 1.0f, 0.0f);
    V3 right = normalize(cross(forward, world_up));
    V3 up = normalize(cross(right, forward));
    F fov_tan = tan_(to_radians(fov_deg) * F(0.5f));
    store3(out->origin, origin);
    store3(out->forward, forward);
    store3(out->right, right);
    store3(out->up, up);
    out->fov_tan = raw(fov_tan);
}
// Camera::generate_ray (camera.rs:149).
static inline Ray generate_ray(const ix_camera& c, F sx, F sy, F w, F h, F jx, F jy) {
    F aspect = w / h;
    F fov_tan = c.fov_tan;
    F u = ((sx + jx) / w - F(0.5f)) * F(2.0f) * aspect * fov_tan;
    F v = (F(0.5f) - (sy + jy) / h) * F(2.0f) * fov_tan;
    V3 dir = normalize(load3(c.forward) + load3(c.right) * u + load3(c.up) * v);
    return Ray{load3(c.origin), dir};
}

// ------------------------------------------------------------------------------------
// transport/mod.rs:58 -- the wrapped hero comb.
// ------------------------------------------------------------------------------------
static inline F rem_euclid(F a, F b) {
    F r = F(fmodf(raw(a), raw(b)));
    return (r < F(0.0f)) ? r + abs_(b) : r;
}
static inline void hero_wavelengths(F hero_rand, F out[8]) {
    const F span = 400.0f;
    const F width = 50.0f;  // 400 / 8
    F lambda_hero = fma_(hero_rand, span, 380.0f);
    for (int k = 0; k < 8; ++k) {
        F offset = fma_(F((float)k), width, lambda_hero - F(380.0f));
        out[k] = F(380.0f) + rem_euclid(offset, span);
    }
}

// ------------------------------------------------------------------------------------
// dispersion.rs:170-210
// ------------------------------------------------------------------------------------
static F dispersion_unclamped(const ix_dispersion& d, F lambda_nm) {
    F um = lambda_nm * F(1e-3f);
    F l2 = um * um;
    switch (d.kind) {
        case IX_DISP_SELLMEIER1: {
            F n2 = F(1.0f) + (F(d.b[0]) * l2) / (l2 - F(d.c[0]));
            return sqrt_(max_(n2, 1.0f));
        }
        case IX_DISP_SELLMEIER3: {
            F n2 = 1.0f;
            n2 += (F(d.b[0]) * l2) / (l2 - F(d.c[0]));
            n2 += (F(d.b[1]) * l2) / (l2 - F(d.c[1]));
            n2 += (F(d.b[2]) * l2) / (l2 - F(d.c[2]));
            return sqrt_(max_(n2, 1.0f));
        }
        default: {
            F l4 = l2 * l2;
            return max_((F(d.b[0]) + F(d.b[1]) / l2) + F(d.b[2]) / l4, 1.0f);
        }
    }
}
// DispersionModel::min_valid_nm (dispersion.rs:149).
static F dispersion_min_valid_nm(const ix_dispersion& d) {
    if (d.kind == IX_DISP_CAUCHY) return 380.0f;
    int n = (d.kind == IX_DISP_SELLMEIER1) ? 1 : 3;
    F floor_nm = 300.0f;
    for (int i = 0; i < n; ++i) {
        F c = d.c[i];
        if (c > F(0.0f)) {
            F pole_nm = sqrt_(c) * F(1e3f);
            if (pole_nm < F(380.0f)) floor_nm = max_(floor_nm, pole_nm * F(1.05f));
        }
    }
    return min_(floor_nm, 380.0f);
}
static F dispersion_eval(const ix_dispersion& d, F lambda_nm) {
    if (lambda_nm < F(380.0f))
        return dispersion_unclamped(d, max_(lambda_nm, dispersion_min_valid_nm(d)));
    return dispersion_unclamped(d, lambda_nm);
}

// ------------------------------------------------------------------------------------
// Absorption alpha(lambda) (optics/absorption.rs:108; raytracer/absorption.rs:32) plus
// the tabulated spline this library adds (ix_scene.h, ix_absorption).
// ------------------------------------------------------------------------------------
static F band_eval(const ix_band& b, F lambda_nm) {
    if (b.shape == IX_BAND_GAUSS_WAVELENGTH) {
        F t = (lambda_nm - F(b.center_nm)) / F(b.width_nm);
        return F(b.peak) * exp_(F(-0.5f) * t * t);
    }
    F delta_nm = F(b.center_nm) - lambda_nm;
    F nu_diff = F(1.0e7f) * delta_nm / (lambda_nm * F(b.center_nm));
    F t = nu_diff / F(b.width_nm);
    return F(b.peak) * exp_(F(-0.5f) * t * t);
}
// Uniform Catmull-Rom through IX_SPLINE_KNOTS knots over [380, 780] nm, end knots
// repeated, floored at zero.  Segment s covers [380 + s*h, 380 + (s+1)*h], h = 400/15.
static F spline_eval(const float* knots, F lambda_nm) {
    const int n = IX_SPLINE_KNOTS;
    F pos = (clamp_(lambda_nm, 380.0f, 780.0f) - F(380.0f)) * F((float)(n - 1) / 400.0f);
    int s = (int)raw(floor_(pos));
    if (s > n - 2) s = n - 2;
    if (s < 0) s = 0;
    F t = pos - F((float)s);
    F p0 = knots[s > 0 ? s - 1 : 0];
    F p1 = knots[s];
    F p2 = knots[s + 1];
    F p3 = knots[s + 2 < n ? s + 2 : n - 1];
    // 0.5 * (2 p1 + (p2 - p0) t + (2 p0 - 5 p1 + 4 p2 - p3) t^2 + (3 p1 - p0 - 3 p2 + p3) t^3)
    F a = F(3.0f) * p1 - p0 - F(3.0f) * p2 + p3;
    F b = F(2.0f) * p0 - F(5.0f) * p1 + F(4.0f) * p2 - p3;
    F c = p2 - p0;
    F poly = fma_(fma_(fma_(a, t, b), t, c), t, F(2.0f) * p1);
    return max_(F(0.5f) * poly, 0.0f);
}
static F spectral_absorption(const ix_absorption& a, F lambda_nm) {
    F sum = 0.0f;
    bool first = true;
    for (uint32_t i = 0; i < a.n_bands && i < IX_MAX_BANDS; ++i) {
        F v = band_eval(a.bands[i], lambda_nm);
        sum = first ? v : sum + v;
        first = false;
    }
    if (a.has_spline) sum = first ? spline_eval(a.spline, lambda_nm) : sum + spline_eval(a.spline, lambda_nm);
    return sum;
}
static bool absorption_present(const ix_absorption& a) {
    if (a.has_spline) return true;
    for (uint32_t i = 0; i < a.n_bands && i < IX_MAX_BANDS; ++i)
        if (a.bands[i].peak != 0.0f) return true;
    return false;
}

// simd/exp_poly.rs:37 -- the Cephes-style polynomial exponential (Moshier), with the
// reference's own constants and its AVX2 min/max clamp semantics.
static F exp_lane(F x) {
    const F LOG2E = 1.44269504088896340736f;
    uint32_t c1bits = 0x3F318000u;
    float c1f;
    std::memcpy(&c1f, &c1bits, 4);
    const F C1 = c1f;
    const F C2 = -2.1219444e-4f;
    const F P0 = 1.9875691e-4f, P1 = 1.3981999e-3f, P2 = 8.333452e-3f, P3 = 4.1665796e-2f,
            P4 = 1.6666665e-1f, P5 = 5.0000003e-1f;
    const F HI = 88.02875f, LO = -87.33654f;
    F upper = (x < HI) ? x : HI;
    x = (upper > LO) ? upper : LO;
    F n = floor_(fma_(x, LOG2E, 0.5f));
    x = fma_(n, -C1, x);
    x = fma_(n, -C2, x);
    F z = x * x;
    F p = P0;
    p = fma_(p, x, P1);
    p = fma_(p, x, P2);
    p = fma_(p, x, P3);
    p = fma_(p, x, P4);
    p = fma_(p, x, P5);
    p = fma_(p, z, x) + F(1.0f);
    int32_t e = (int32_t)raw(n);
    uint32_t bits = (uint32_t)((e + 127) << 23);
    float pow2n;
    std::memcpy(&pow2n, &bits, 4);
    return p * F(pow2n);
}

// ------------------------------------------------------------------------------------
// Colour (color/cie1931.rs:157-199; optics/raytracer/color.rs:85-180, 219-329).
// ------------------------------------------------------------------------------------
static const float CMF[81][3] = IX_CIE1931_CMF_INIT;
static const float D65[41] = IX_CIE_D65_SPD_INIT;
static const float D65_UV[9] = IX_CIE_D65_UV_SPD_INIT;

static V3 cmf(F lambda_nm) {
    if (!(lambda_nm >= F(380.0f) && lambda_nm <= F(780.0f))) return v3(0.0f, 0.0f, 0.0f);
    F position = (lambda_nm - F(380.0f)) / F(5.0f);
    int i0 = (int)raw(floor_(position));
    if (i0 > 79) i0 = 79;
    F t = position - F((float)i0);
    const float* lo = CMF[i0];
    const float* hi = CMF[i0 + 1];
    return v3(F(lo[0]) + (F(hi[0]) - F(lo[0])) * t, F(lo[1]) + (F(hi[1]) - F(lo[1])) * t,
              F(lo[2]) + (F(hi[2]) - F(lo[2])) * t);
}
// d65_relative_spectral_power (environment/spectral.rs:28).
static F d65(F lambda_nm) {
    if (lambda_nm < F(380.0f)) {
        F clamped = max_(lambda_nm, 300.0f);
        F position = (clamped - F(300.0f)) / F(10.0f);
        int i0 = (int)raw(floor_(position));
        if (i0 > 7) i0 = 7;
        F frac = position - F((float)i0);
        F v0 = D65_UV[i0], v1 = D65_UV[i0 + 1];
        return fma_(frac, v1 - v0, v0) / F(100.0f);
    }
    F clamped = clamp_(lambda_nm, 380.0f, fma_(10.0f, 40.0f, 380.0f));
    F position = (clamped - F(380.0f)) / F(10.0f);
    int i0 = (int)raw(floor_(position));
    if (i0 > 39) i0 = 39;
    F frac = position - F((float)i0);
    F v0 = D65[i0], v1 = D65[i0 + 1];
    return fma_(frac, v1 - v0, v0) / F(100.0f);
}
// powi with a constant exponent: LLVM's binary decomposition (and compiler-rt's
// __powisf2), `res *= x^(2^i)` for the set bits in ascending order.
static F powi_(F x, unsigned n) {
    bool have = false;
    F res = 1.0f;
    F sq = x;
    while (n) {
        if (n & 1u) {
            res = have ? res * sq : sq;
            have = true;
        }
        n >>= 1;
        if (n) sq = sq * sq;
    }
    return res;
}
// blackbody_spectrum_with (environment/spectral.rs:62-82).
static F blackbody(F t_k, F denom_560, F lambda_nm) {
    F exp_val = exp_(min_(F(14388000.0f) / (lambda_nm * t_k), 80.0f));
    F denom = max_(exp_val - F(1.0f), 1e-6f);
    F ratio = denom_560 / denom;
    return clamp_(powi_(F(560.0f) / lambda_nm, 5) * ratio, 0.01f, 20.0f);
}
static void blackbody_norm(F temp_k, F* t_k, F* denom_560) {
    *t_k = max_(temp_k, 1000.0f);
    F exp_560 = exp_(min_(F(14388000.0f) / (F(560.0f) * *t_k), 80.0f));
    *denom_560 = max_(exp_560 - F(1.0f), 1e-6f);
}
static const float BRADFORD_XYZ_TO_LMS[3][3] = {
    {0.8951f, 0.2664f, -0.1614f}, {-0.7502f, 1.7135f, 0.0367f}, {0.0389f, -0.0685f, 1.0296f}};
static const float BRADFORD_LMS_TO_XYZ[3][3] = {{0.986993f, -0.147054f, 0.159963f},
                                                {0.432305f, 0.518360f, 0.049291f},
                                                {-0.008529f, 0.040043f, 0.968487f}};
static V3 mat3_fma(const float m[3][3], V3 v) {
    return v3(fma_(m[0][0], v.x, fma_(m[0][1], v.y, F(m[0][2]) * v.z)),
              fma_(m[1][0], v.x, fma_(m[1][1], v.y, F(m[1][2]) * v.z)),
              fma_(m[2][0], v.x, fma_(m[2][1], v.y, F(m[2][2]) * v.z)));
}
// compute_illuminant_white_balance (color.rs:277).
static V3 illuminant_white_balance(F temp_k) {
    F t_k, den;
    blackbody_norm(temp_k, &t_k, &den);
    V3 xyz_w = v3(0.0f, 0.0f, 0.0f);
    for (int step = 0; step <= 400; ++step) {
        F lambda = F(380.0f) + F((float)step);
        xyz_w = xyz_w + cmf(lambda) * blackbody(t_k, den, lambda);
    }
    F target_y = max_(xyz_w.y, 1e-6f);
    const F wx = 0.3127f, wy = 0.3290f;
    V3 target = v3((wx / wy) * target_y, target_y, ((F(1.0f) - wx - wy) / wy) * target_y);
    V3 src = mat3_fma(BRADFORD_XYZ_TO_LMS, xyz_w);
    V3 tgt = mat3_fma(BRADFORD_XYZ_TO_LMS, target);
    return v3(src.x > F(1e-6f) ? tgt.x / src.x : F(1.0f),
              src.y > F(1e-6f) ? tgt.y / src.y : F(1.0f),
              src.z > F(1e-6f) ? tgt.z / src.z : F(1.0f));
}

// ------------------------------------------------------------------------------------
// Environment (environment/rig.rs, environment/mod.rs:128-143, optics/studio_rig.rs).
// ------------------------------------------------------------------------------------
static inline F smoothstep(F e0, F e1, F x) {
    F t = clamp_((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * fma_(-2.0f, t, 3.0f);
}
static F spectral_power(const ix_environment& env, F lambda_nm) {
    switch (env.spectrum) {
        case IX_SPEC_D65: return d65(lambda_nm);
        case IX_SPEC_BLACKBODY: return blackbody(env.bb_t_k, env.bb_denom_560, lambda_nm);
        case IX_SPEC_GAUSSIAN: {  // IlluminantSpectrum::Gaussian (spectral.rs:137)
            const F z = (lambda_nm - F(env.line_centre_nm)) / F(env.line_sigma_nm);
            return exp_((F(-0.5f) * z) * z);
        }
        case IX_SPEC_WAVELENGTH: return lambda_nm;  // aset_spec_input (rig.rs:165)
        default: return 1.0f;
    }
}
// The tent, dome and ASET constants (rig.rs:67-85, :120-135, sun.rs:10-20).
constexpr float TENT_KEY_OUTER_COS = 0.7660444f, TENT_KEY_INNER_COS = 0.9396926f;
constexpr float SPARK_OUTER_COS = 0.9961947f, SPARK_INNER_COS = 0.9993908f;
constexpr float CARD_OUTER_COS = 0.898794f, CARD_INNER_COS = 0.9612617f;
constexpr int CARD_RING_SLOTS[3] = {4, 8, 12};
constexpr float ASET_SIGMA_NM = 8.493218f;
constexpr float ASET_EDGE_45_LO = 0.6871068f, ASET_EDGE_45_HI = 0.7271068f;
constexpr float ASET_EDGE_75_LO = 0.9459258f, ASET_EDGE_75_HI = 0.9859258f;
constexpr float SUN_DISC_COS = 0.9999889f;
constexpr float SUN_RADIANCE = 40000.0f;
constexpr float SUN_ONE_MINUS_COS = 1.1086464e-5f;  // 186 x 2^-24
constexpr float SUN_SOLID_ANGLE = 6.965831e-5f;
// The direction-only part of the lighting (rig.rs:67-96, 157-170, 320-377), reduced to
// how radiance(spec_power) is formed from it.
struct Lighting {
    int kind;  // 0 scaled, 1 rig, 2 uniform, 3 banded (ASET)
    F factor;
    F red, green, blue, tray_ground;  // banded
    F bg, softbox, fill;
    bool has_softbox, has_fill;
    F ring[IX_RING_LIGHTS];
    int ring_len;
    bool has_ground;
    F horizon, ground;
};
static Lighting direction_lighting(const ix_environment& env, V3 dir, V3 observer) {
    Lighting L;
    L.kind = 0;
    L.has_softbox = L.has_fill = L.has_ground = false;
    L.ring_len = 0;
    if (env.model == IX_ENV_UNIFORM) {
        L.kind = 2;
        return L;
    }
    V3 d = normalize(dir);
    F tray = env.backdrop;
    if (env.model == IX_ENV_ISO_HEMISPHERE) {
        F horizon = smoothstep(-0.05f, 0.05f, d.y);
        F vis = F(1.0f) - smoothstep(env.shadow_cos[0], env.shadow_cos[1], dot(d, observer));
        if (tray > F(0.0f))
            L.factor = fma_((F(1.0f) - horizon) * vis, tray, horizon * vis);
        else
            L.factor = horizon * vis;
        return L;
    }
    // lit_ground (rig.rs:230): the tray below the horizon, else the model's own ground.
    auto lit_ground = [&](F horizon, F vis, F own) {
        return tray > F(0.0f) ? ((F(1.0f) - horizon) * vis) * tray : own * (F(1.0f) - horizon);
    };
    if (env.model == IX_ENV_LIGHT_TENT) {
        // light_tent_lighting (rig.rs:254).
        const F horizon = smoothstep(-0.05f, 0.05f, d.y);
        F walls = fma_(0.08f, max_(d.y, 0.0f), 0.14f) * F(env.tent_walls);
        if (F(env.tent_flat) > F(0.0f))
            walls = fma_(F(0.18f) * F(env.tent_walls), env.tent_flat, walls * (F(1.0f) - F(env.tent_flat)));
        F card = 0.0f;
        for (int slot : CARD_RING_SLOTS)
            card = max_(card, smoothstep(CARD_OUTER_COS, CARD_INNER_COS, dot(d, load3(env.ring_dirs[slot]))));
        walls = walls * fma_(card * F(env.tent_cards), -0.9f, 1.0f);
        const F key = smoothstep(TENT_KEY_OUTER_COS, TENT_KEY_INNER_COS, dot(d, load3(env.key_dir))) *
                      (F(1.4f) * F(env.spot_mult));
        const F spark = (smoothstep(SPARK_OUTER_COS, SPARK_INNER_COS, dot(d, load3(env.fill_dir))) *
                         (F(5.0f) * F(env.spot_mult))) * F(env.tent_spark);
        const F vis = F(1.0f) - smoothstep(env.shadow_cos[0], env.shadow_cos[1], dot(d, observer));
        const F above = ((walls + key) + spark) * (horizon * vis);
        L.factor = above + lit_ground(horizon, vis, env.tent_ground);
        return L;
    }
    if (env.model == IX_ENV_DAYLIGHT_DOME || env.model == IX_ENV_DAYLIGHT_SUN) {
        // daylight_dome_lighting (rig.rs:297) and daylight_sun_radiance (rig.rs:466): the
        // sky, its aureole about the sun, and for DaylightSun the 0.27 degree disc.
        const F horizon = smoothstep(-0.05f, 0.05f, d.y);
        const F sun_dot = dot(d, load3(env.key_dir));
        const F sky = fma_(0.08f, F(1.0f) - max_(d.y, 0.0f), 0.10f);
        const F glow = max_(sun_dot, 0.0f);
        const F glow2 = glow * glow;
        const F glow4 = glow2 * glow2;
        const F aureole = (glow4 * glow4) * F(0.30f);
        const F vis = F(1.0f) - smoothstep(env.shadow_cos[0], env.shadow_cos[1], dot(d, observer));
        const F above = (sky + aureole) * (horizon * vis);
        const F ground = lit_ground(horizon, vis, 0.04f);
        if (env.model == IX_ENV_DAYLIGHT_DOME) {
            L.factor = above + ground;
        } else {
            const F sun = sun_dot >= F(SUN_DISC_COS) ? F(env.sun_factor) : F(0.0f);
            L.factor = (above + ground) + sun;
        }
        return L;
    }
    if (env.model == IX_ENV_ASET) {
        // aset_radiance (rig.rs:439): three elevation zones, banded at radiance time.
        const F horizon = smoothstep(-0.05f, 0.05f, d.y);
        const F s45 = smoothstep(ASET_EDGE_45_LO, ASET_EDGE_45_HI, d.y);
        const F s75 = smoothstep(ASET_EDGE_75_LO, ASET_EDGE_75_HI, d.y);
        L.kind = 3;
        L.red = (s45 * (F(1.0f) - s75)) * horizon;
        L.green = (F(1.0f) - s45) * horizon;
        L.blue = s75 * horizon;
        L.tray_ground = tray > F(0.0f) ? (F(1.0f) - horizon) * tray : F(0.0f);
        return L;
    }
    // Studio rig (rig.rs:320-377).
    L.kind = 1;
    F exposure = env.exposure;
    F spot = env.spot_mult;
    L.bg = env.ambient_fill
               ? max_(fma_(0.012f, fma_(d.y, 0.5f, 0.5f), 0.015f), 0.005f) * exposure
               : F(0.0f);
    F key_dot = max_(dot(d, load3(env.key_dir)), 0.0f);
    if (key_dot > F(0.0f)) {
        L.has_softbox = true;
        L.softbox = powi_(key_dot, 28) * F(12.0f) * spot * exposure;
    }
    F fill_dot = max_(dot(d, load3(env.fill_dir)), 0.0f);
    if (fill_dot > F(0.0f)) {
        L.has_fill = true;
        L.fill = powi_(fill_dot, 18) * F(4.5f) * exposure;
    }
    for (int i = 0; i < IX_RING_LIGHTS; ++i) {
        F ring_dot = max_(dot(d, load3(env.ring_dirs[i])), 0.0f);
        if (ring_dot > F(0.96f)) {
            F spark = (ring_dot - F(0.96f)) / F(0.04f);
            L.ring[L.ring_len++] = powi_(spark, 6) * F(22.0f) * spot * exposure;
        }
    }
    if (tray > F(0.0f)) {
        L.has_ground = true;
        L.horizon = smoothstep(-0.05f, 0.05f, d.y);
        L.ground = ((F(1.0f) - L.horizon) * tray) * exposure;
    }
    return L;
}
// DirectionLighting::radiance (rig.rs:112-155).
static F aset_band(F lambda_nm, F centre_nm) {
    const F z = (lambda_nm - centre_nm) / F(ASET_SIGMA_NM);
    return exp_((F(-0.5f) * z) * z);
}
static F lighting_radiance(const Lighting& L, const ix_environment& env, F spec) {
    if (L.kind == 2) return F(env.uniform_radiance) * spec;
    if (L.kind == 0) return L.factor * (spec * F(env.exposure));
    if (L.kind == 3) {
        // DirectionLighting::Banded (rig.rs:140): `spec` is the wavelength.
        const F r = (L.red * aset_band(spec, 610.0f)) * F(8.0f);
        const F g = (L.green * aset_band(spec, 540.0f)) * F(5.0f);
        const F b = (L.blue * aset_band(spec, 460.0f)) * F(16.0f);
        const F zones = ((r + g) + b) * F(env.exposure);
        if (L.tray_ground > F(0.0f)) return fma_(L.tray_ground * d65(spec), env.exposure, zones);
        return zones;
    }
    F r = L.bg * spec;
    if (L.has_softbox) r = fma_(L.softbox, spec, r);
    if (L.has_fill) r = fma_(L.fill, spec, r);
    for (int i = 0; i < L.ring_len; ++i) r = fma_(L.ring[i], spec, r);
    if (L.has_ground) return fma_(L.horizon, r, L.ground * spec);
    return r;
}
static void environment_channels(const ix_environment& env, V3 dir, const F lambdas[8],
                                 V3 observer, F out[8]) {
    Lighting L = direction_lighting(env, dir, observer);
    for (int k = 0; k < 8; ++k) out[k] = lighting_radiance(L, env, spectral_power(env, lambdas[k]));
}
static F environment_channel(const ix_environment& env, V3 dir, F lambda, V3 observer) {
    Lighting L = direction_lighting(env, dir, observer);
    return lighting_radiance(L, env, spectral_power(env, lambda));
}

// ------------------------------------------------------------------------------------
// Intersection (simd/slab.rs:120-160, intersect.rs:101-127).
// ------------------------------------------------------------------------------------
struct Hit {
    F t;
    V3 normal;
    int facet;
};
#if defined(IX_ORACLE_AVX2) && !defined(IX_COUNT_FLOPS)
// The AVX2 twin of the slab scan (simd/slab.rs:200-290, slab_scan_avx2): 8 planes per
// block with the scalar operation order (left-associated dot products, separate
// multiply and add, an IEEE division), the block's entering max / exiting min checked
// against the running state, and only blocks that could change it replayed through the
// scalar step in ascending plane order -- bit-identical to the scalar scan.  Planes are
// read in this library's {nx, ny, nz, d} rows and transposed in registers.
static inline float hmax8(__m256 v) {
    __m128 m = _mm_max_ps(_mm256_castps256_ps128(v), _mm256_extractf128_ps(v, 1));
    m = _mm_max_ps(m, _mm_movehl_ps(m, m));
    m = _mm_max_ps(m, _mm_shuffle_ps(m, m, 0x01));
    return _mm_cvtss_f32(m);
}
static inline float hmin8(__m256 v) {
    __m128 m = _mm_min_ps(_mm256_castps256_ps128(v), _mm256_extractf128_ps(v, 1));
    m = _mm_min_ps(m, _mm_movehl_ps(m, m));
    m = _mm_min_ps(m, _mm_shuffle_ps(m, m, 0x01));
    return _mm_cvtss_f32(m);
}
#endif

// The slab scan proper (simd/slab.rs slab_scan): the entering planes' largest t and the
// first plane attaining it, the exiting planes' smallest t and its plane; false for a
// parallel plane the origin is outside of.
static bool slab_scan_raw(const float* planes, uint32_t n, const Ray& ray, F* tn_out, int* ni_out, F* tf_out,
                          int* fi_out) {
    F t_near = -1e30f, t_far = 1e30f;
    int near_idx = -1, far_idx = -1;
    uint32_t i0 = 0;
#if defined(IX_ORACLE_AVX2) && !defined(IX_COUNT_FLOPS)
    {
        const __m256 dx = _mm256_set1_ps(ray.dir.x), dy = _mm256_set1_ps(ray.dir.y), dz = _mm256_set1_ps(ray.dir.z);
        const __m256 ox = _mm256_set1_ps(ray.origin.x), oy = _mm256_set1_ps(ray.origin.y),
                     oz = _mm256_set1_ps(ray.origin.z);
        const __m256 thr = _mm256_set1_ps(1e-7f), sign = _mm256_set1_ps(-0.0f), zero = _mm256_setzero_ps();
        const __m256 neg_inf = _mm256_set1_ps(-INFINITY), pos_inf = _mm256_set1_ps(INFINITY);
        alignas(32) float den_l[8], side_l[8], t_l[8];
        for (; i0 + 8 <= n; i0 += 8) {
            const float* b = planes + 4 * (size_t)i0;
            const __m256 r0 = _mm256_insertf128_ps(_mm256_castps128_ps256(_mm_loadu_ps(b)), _mm_loadu_ps(b + 16), 1);
            const __m256 r1 = _mm256_insertf128_ps(_mm256_castps128_ps256(_mm_loadu_ps(b + 4)), _mm_loadu_ps(b + 20), 1);
            const __m256 r2 = _mm256_insertf128_ps(_mm256_castps128_ps256(_mm_loadu_ps(b + 8)), _mm_loadu_ps(b + 24), 1);
            const __m256 r3 = _mm256_insertf128_ps(_mm256_castps128_ps256(_mm_loadu_ps(b + 12)), _mm_loadu_ps(b + 28), 1);
            const __m256 t0 = _mm256_unpacklo_ps(r0, r1), t1 = _mm256_unpackhi_ps(r0, r1);
            const __m256 t2 = _mm256_unpacklo_ps(r2, r3), t3 = _mm256_unpackhi_ps(r2, r3);
            const __m256 nx = _mm256_shuffle_ps(t0, t2, 0x44), ny = _mm256_shuffle_ps(t0, t2, 0xEE);
            const __m256 nz = _mm256_shuffle_ps(t1, t3, 0x44), d = _mm256_shuffle_ps(t1, t3, 0xEE);
            const __m256 denom =
                _mm256_add_ps(_mm256_add_ps(_mm256_mul_ps(nx, dx), _mm256_mul_ps(ny, dy)), _mm256_mul_ps(nz, dz));
            const __m256 dot_o =
                _mm256_add_ps(_mm256_add_ps(_mm256_mul_ps(nx, ox), _mm256_mul_ps(ny, oy)), _mm256_mul_ps(nz, oz));
            const __m256 side = _mm256_add_ps(d, dot_o);
            const __m256 t = _mm256_div_ps(_mm256_xor_ps(side, sign), denom);  // (-side) / denom
            const __m256 absd = _mm256_andnot_ps(sign, denom);
            const __m256 valid = _mm256_cmp_ps(absd, thr, _CMP_GT_OQ);
            const __m256 par_out =
                _mm256_and_ps(_mm256_cmp_ps(absd, thr, _CMP_LE_OQ), _mm256_cmp_ps(side, zero, _CMP_GT_OQ));
            if (_mm256_movemask_ps(par_out) != 0) return false;  // parallel plane, origin outside
            const __m256 entering = _mm256_and_ps(valid, _mm256_cmp_ps(denom, zero, _CMP_LT_OQ));
            const __m256 exiting = _mm256_andnot_ps(entering, valid);
            const float ent_max = hmax8(_mm256_blendv_ps(neg_inf, t, entering));
            const float ex_min = hmin8(_mm256_blendv_ps(pos_inf, t, exiting));
            if (!(ent_max > t_near || ex_min < t_far)) continue;  // the block changes nothing
            _mm256_store_ps(den_l, denom);
            _mm256_store_ps(side_l, side);
            _mm256_store_ps(t_l, t);
            for (int k = 0; k < 8; ++k) {
                const F denom_k = den_l[k];
                if (abs_(denom_k) > F(1e-7f)) {
                    if (denom_k < F(0.0f)) {
                        if (F(t_l[k]) > t_near) {
                            t_near = t_l[k];
                            near_idx = (int)(i0 + k);
                        }
                    } else if (F(t_l[k]) < t_far) {
                        t_far = t_l[k];
                        far_idx = (int)(i0 + k);
                    }
                } else if (F(side_l[k]) > F(0.0f)) {
                    return false;
                }
            }
        }
    }
#endif
    for (uint32_t i = i0; i < n; ++i) {
        V3 nrm = load3(planes + 4 * i);
        F denom = dot(nrm, ray.dir);
        F side = F(planes[4 * i + 3]) + dot(nrm, ray.origin);
        F t = (-side) / denom;
        if (abs_(denom) > F(1e-7f)) {
            if (denom < F(0.0f)) {
                if (t > t_near) {
                    t_near = t;
                    near_idx = (int)i;
                }
            } else if (t < t_far) {
                t_far = t;
                far_idx = (int)i;
            }
        } else if (side > F(0.0f)) {
            return false;
        }
    }
    *tn_out = t_near;
    *ni_out = near_idx;
    *tf_out = t_far;
    *fi_out = far_idx;
    return true;
}

// intersect_polyhedron (intersect.rs:101-127): the slab, then the first boundary past
// the 1e-4 restart epsilon.
static bool intersect(const float* planes, uint32_t n, const Ray& ray, Hit* hit) {
    F t_near, t_far;
    int near_idx, far_idx;
    if (!slab_scan_raw(planes, n, ray, &t_near, &near_idx, &t_far, &far_idx)) return false;
    if (t_near > t_far) return false;
    if (t_near > F(1e-4f)) {
        hit->t = t_near;
        hit->normal = near_idx >= 0 ? load3(planes + 4 * near_idx) : v3(0.0f, 0.0f, 0.0f);
        hit->facet = near_idx >= 0 ? near_idx : 0;
        return true;
    }
    if (t_far > F(1e-4f)) {
        hit->t = t_far;
        hit->normal = far_idx >= 0 ? load3(planes + 4 * far_idx) : v3(0.0f, 0.0f, 0.0f);
        hit->facet = far_idx >= 0 ? far_idx : 0;
        return true;
    }
    return false;
}

// ------------------------------------------------------------------------------------
// Concave tools (geometry/tool.rs, geometry/tool/interval.rs) and the carved stone
// (optics/raytracer/intersect_stone.rs): each tool is the convex hull interval of the
// pieces it decomposes into (balls, frusta, and the wedges of an across-axis sweep); the
// stone is the slab minus the tools, walked in sorted boundary order.
// ------------------------------------------------------------------------------------
enum { TOOL_BALL = 0, TOOL_CYLINDER = 1, TOOL_FRUSTUM = 2, TOOL_BICONE = 3 };
enum { SWEEP_NONE = 0, SWEEP_ALONG = 1, SWEEP_ACROSS = 2 };
enum { PIECE_BALL = 0, PIECE_FRUSTUM = 1, PIECE_WEDGE = 2 };
struct Piece {
    int kind;
    V3 c, a, d;
    F r, hl, s, r0, r1;
};
static Piece ball_piece(V3 c, F r) {
    Piece p{};
    p.kind = PIECE_BALL;
    p.c = c;
    p.r = r;
    return p;
}
static Piece frustum_piece(V3 c, V3 a, F hl, F r0, F r1) {
    Piece p{};
    p.kind = PIECE_FRUSTUM;
    p.c = c;
    p.a = a;
    p.hl = hl;
    p.r0 = r0;
    p.r1 = r1;
    return p;
}
static inline V3 tool_vec(const float* v) { return v3(v[0], v[1], v[2]); }
// ToolPrimitive::pieces (tool.rs:470): at most 6.
static int tool_pieces(const ix_tool& t, Piece out[6]) {
    if (t.kind > TOOL_BICONE || t.sweep_kind > SWEEP_ACROSS) return 0;
    const V3 c = tool_vec(t.origin), a = tool_vec(t.axis);
    const F stroke = t.profile[2];
    const bool swept = t.sweep_kind != SWEEP_NONE && stroke > F(0.0f);
    int n = 0;
    if (t.kind == TOOL_BALL) {
        const F r = t.origin[3];
        if (swept) {
            const V3 dir = t.sweep_kind == SWEEP_ALONG ? a : tool_vec(t.sweep_dir);
            out[n++] = ball_piece(c - dir * stroke, r);
            out[n++] = ball_piece(c + dir * stroke, r);
            out[n++] = frustum_piece(c, dir, stroke, r, r);
        } else {
            out[n++] = ball_piece(c, r);
        }
        return n;
    }
    // segments (tool.rs:430): (z_lo, z_hi, r_lo, r_hi) along the axis, and the peak.
    const F hl = t.axis[3], rim = t.origin[3], rn = t.profile[0], rp = t.profile[1];
    F seg[2][4];
    int ns = 1;
    F peak_z, peak_r;
    if (t.kind == TOOL_CYLINDER) {
        seg[0][0] = -hl; seg[0][1] = hl; seg[0][2] = rim; seg[0][3] = rim;
        peak_z = hl;
        peak_r = rim;
    } else if (t.kind == TOOL_FRUSTUM) {
        seg[0][0] = -hl; seg[0][1] = hl; seg[0][2] = rn; seg[0][3] = rp;
        peak_z = rp >= rn ? hl : -hl;
        peak_r = rp >= rn ? rp : rn;
    } else {
        seg[0][0] = -hl; seg[0][1] = 0.0f; seg[0][2] = rn; seg[0][3] = rim;
        seg[1][0] = 0.0f; seg[1][1] = hl; seg[1][2] = rim; seg[1][3] = rp;
        ns = 2;
        peak_z = 0.0f;
        peak_r = rim;
    }
    auto seg_piece = [&](const F* sg, V3 shift) {
        return frustum_piece((c + a * (F(0.5f) * (sg[0] + sg[1]))) + shift, a, F(0.5f) * (sg[1] - sg[0]), sg[2], sg[3]);
    };
    for (int i = 0; i < ns; ++i) {
        const F* sg = seg[i];
        if (!swept) {
            out[n++] = seg_piece(sg, v3(0.0f, 0.0f, 0.0f));
        } else if (t.sweep_kind == SWEEP_ALONG) {
            out[n++] = seg_piece(sg, sg[3] >= sg[2] ? (-a) * stroke : a * stroke);
        } else {
            const V3 dir = tool_vec(t.sweep_dir);
            out[n++] = seg_piece(sg, (-dir) * stroke);
            out[n++] = seg_piece(sg, dir * stroke);
            Piece w{};
            w.kind = PIECE_WEDGE;
            w.c = c + a * (F(0.5f) * (sg[0] + sg[1]));
            w.a = a;
            w.d = dir;
            w.hl = F(0.5f) * (sg[1] - sg[0]);
            w.s = stroke;
            w.r0 = sg[2];
            w.r1 = sg[3];
            out[n++] = w;
        }
    }
    if (swept && t.sweep_kind == SWEEP_ALONG) out[n++] = frustum_piece(c + a * peak_z, a, stroke, peak_r, peak_r);
    return n;
}
// quadratic_roots (interval.rs:8): a t^2 + 2 b t + c = 0, the stable form.
static bool quadratic_roots(F a, F b, F c, F* lo, F* hi) {
    const F disc = fma_(b, b, -(a * c));
    if (disc <= F(1e-7f) * fma_(b, b, abs_(a * c))) return false;
    const F sq = sqrt_(disc);
    const F q = -(b + F(std::copysign(raw(sq), raw(b))));
    const F r1 = q / a, r2 = c / q;
    *lo = r1 <= r2 ? r1 : r2;
    *hi = r1 <= r2 ? r2 : r1;
    return true;
}
static bool ball_interval(const Ray& ray, V3 c, F r, F* lo, F* hi) {
    const V3 o = ray.origin - c;
    return quadratic_roots(dot(ray.dir, ray.dir), dot(o, ray.dir), fma_(r, -r, dot(o, o)), lo, hi);
}
static bool cap_range(F z0, F dz, F hl, F* s0, F* s1) {
    if (abs_(dz) > F(1e-7f)) {
        const F t1 = (-hl - z0) / dz, t2 = (hl - z0) / dz;
        *s0 = t1 <= t2 ? t1 : t2;
        *s1 = t1 <= t2 ? t2 : t1;
        return true;
    }
    if (abs_(z0) <= hl) {
        *s0 = -1e30f;
        *s1 = 1e30f;
        return true;
    }
    return false;
}
static bool clip_range(F lo, F hi, F s0, F s1, F* l, F* h) {
    *l = max_(lo, s0);
    *h = min_(hi, s1);
    return *l <= *h;
}
// frustum_interval (interval.rs:52): the cone's quadratic clipped to the caps.
static bool frustum_interval(const Ray& ray, V3 c, V3 a, F hl, F r0, F r1, F* lo_out, F* hi_out) {
    const V3 o = ray.origin - c;
    const F z0 = dot(o, a), dz = dot(ray.dir, a);
    F s0, s1;
    if (!cap_range(z0, dz, hl, &s0, &s1)) return false;
    const F rm = F(0.5f) * (r0 + r1);
    const F k = (r1 - r0) / (F(2.0f) * hl);
    const V3 p = o - a * z0, q = ray.dir - a * dz;
    const F rz0 = fma_(k, z0, rm);
    const F rate = k * dz;
    const F qa = fma_(rate, -rate, dot(q, q));
    const F qb = fma_(-rate, rz0, dot(p, q));
    const F qc = fma_(rz0, -rz0, dot(p, p));
    if (abs_(qa) <= F(1e-7f)) {
        if (abs_(qb) <= F(1e-7f)) {
            if (!(qc <= F(0.0f))) return false;
            *lo_out = s0;
            *hi_out = s1;
            return true;
        }
        const F t = -qc / (F(2.0f) * qb);
        return qb > F(0.0f) ? clip_range(-1e30f, t, s0, s1, lo_out, hi_out)
                            : clip_range(t, 1e30f, s0, s1, lo_out, hi_out);
    }
    F lo, hi;
    if (!quadratic_roots(qa, qb, qc, &lo, &hi)) return false;
    if (qa > F(0.0f)) return clip_range(lo, hi, s0, s1, lo_out, hi_out);
    F xl, xh, yl, yh;
    const bool x = clip_range(-1e30f, lo, s0, s1, &xl, &xh);
    const bool y = clip_range(hi, 1e30f, s0, s1, &yl, &yh);
    if (x && y) {
        *lo_out = min_(xl, yl);
        *hi_out = max_(xh, yh);
        return true;
    }
    if (x) {
        *lo_out = xl;
        *hi_out = xh;
        return true;
    }
    if (y) {
        *lo_out = yl;
        *hi_out = yh;
        return true;
    }
    return false;
}
// wedge_interval (interval.rs:112): a slab of six planes.
static bool wedge_interval(const Ray& ray, V3 c, V3 a, V3 d, F hl, F s, F r0, F r1, F* lo, F* hi) {
    const V3 w = cross(a, d);
    const F k = (r1 - r0) / (F(2.0f) * hl);
    const F rm = F(0.5f) * (r0 + r1);
    const V3 fn[6] = {a, -a, d, -d, w - a * k, (-w) - a * k};
    const F fe[6] = {-hl, -hl, -s, -s, -rm, -rm};
    const V3 o = ray.origin - c;
    F t_near = -1e30f, t_far = 1e30f;
    for (int i = 0; i < 6; ++i) {
        const F denom = dot(fn[i], ray.dir);
        const F side = dot(fn[i], o) + fe[i];
        if (abs_(denom) > F(1e-7f)) {
            const F t = -side / denom;
            if (denom < F(0.0f))
                t_near = max_(t_near, t);
            else
                t_far = min_(t_far, t);
        } else if (side > F(0.0f)) {
            return false;
        }
    }
    if (!(t_near <= t_far)) return false;
    *lo = t_near;
    *hi = t_far;
    return true;
}
static bool piece_interval(const Piece& pc, const Ray& ray, F* lo, F* hi) {
    if (pc.kind == PIECE_BALL) return ball_interval(ray, pc.c, pc.r, lo, hi);
    if (pc.kind == PIECE_FRUSTUM) return frustum_interval(ray, pc.c, pc.a, pc.hl, pc.r0, pc.r1, lo, hi);
    return wedge_interval(ray, pc.c, pc.a, pc.d, pc.hl, pc.s, pc.r0, pc.r1, lo, hi);
}
// Vec3::any_orthonormal_vector (glam; Duff et al., "Building an Orthonormal Basis,
// Revisited", JCGT 2017).
static V3 any_orthonormal_vector(V3 n) {
    const F sign = std::signbit(raw(n.z)) ? F(-1.0f) : F(1.0f);
    const F a = F(-1.0f) / (sign + n.z);
    const F b = (n.x * n.y) * a;
    return v3(b, sign + (n.y * n.y) * a, -n.y);
}
// Piece::sd_normal (tool.rs:228): signed distance and outward normal.
static F piece_sd_normal(const Piece& pc, V3 p, V3* n_out) {
    if (pc.kind == PIECE_BALL) {
        const V3 q = p - pc.c;
        const F len = sqrt_(dot(q, q));
        *n_out = len > F(1e-12f) ? v3(q.x / len, q.y / len, q.z / len) : v3(0.0f, 0.0f, 1.0f);
        return len - pc.r;
    }
    if (pc.kind == PIECE_FRUSTUM) {
        const V3 q = p - pc.c;
        const F z = dot(q, pc.a);
        const V3 perp = q - pc.a * z;
        const F rho = sqrt_(dot(perp, perp));
        const V3 rho_hat = rho > F(1e-12f) ? v3(perp.x / rho, perp.y / rho, perp.z / rho) : any_orthonormal_vector(pc.a);
        const F cap_sd = z >= F(0.0f) ? z - pc.hl : -z - pc.hl;
        const V3 cap_n = z >= F(0.0f) ? pc.a : -pc.a;
        const F dr = pc.r1 - pc.r0;
        const F len = sqrt_(fma_(F(4.0f) * pc.hl, pc.hl, dr * dr));
        const F rm = F(0.5f) * (pc.r0 + pc.r1);
        const F side_sd = fma_(z, -dr, ((rho - rm) * F(2.0f)) * pc.hl) / len;
        const V3 side_n = rho_hat * ((F(2.0f) * pc.hl) / len) - pc.a * (dr / len);
        if (side_sd > cap_sd) {
            *n_out = side_n;
            return side_sd;
        }
        *n_out = cap_n;
        return cap_sd;
    }
    const V3 q = p - pc.c;
    const V3 w = cross(pc.a, pc.d);
    const F z = dot(q, pc.a), x = dot(q, pc.d), y = dot(q, w);
    const F k = (pc.r1 - pc.r0) / (F(2.0f) * pc.hl);
    const F rm = F(0.5f) * (pc.r0 + pc.r1);
    const F kappa = F(1.0f) / sqrt_(fma_(k, k, 1.0f));
    F best = z >= F(0.0f) ? z - pc.hl : -z - pc.hl;
    V3 best_n = z >= F(0.0f) ? pc.a : -pc.a;
    const F along = x >= F(0.0f) ? x - pc.s : -x - pc.s;
    if (along > best) {
        best = along;
        best_n = x >= F(0.0f) ? pc.d : -pc.d;
    }
    const F sp = ((y - rm) - k * z) * kappa;
    if (sp > best) {
        best = sp;
        best_n = (w - pc.a * k) * kappa;
    }
    const F sn = ((-y - rm) - k * z) * kappa;
    if (sn > best) {
        best = sn;
        best_n = ((-w) - pc.a * k) * kappa;
    }
    *n_out = best_n;
    return best;
}
// ToolPrimitive::ray_interval (tool.rs:580): the hull of the pieces' intervals.
static bool tool_ray_interval(const ix_tool& t, const Ray& ray, F* lo, F* hi) {
    Piece ps[6];
    const int n = tool_pieces(t, ps);
    bool any = false;
    for (int i = 0; i < n; ++i) {
        F c, d;
        if (!piece_interval(ps[i], ray, &c, &d)) continue;
        if (!any) {
            *lo = c;
            *hi = d;
            any = true;
        } else {
            *lo = min_(*lo, c);
            *hi = max_(*hi, d);
        }
    }
    return any;
}
// outward_normal (tool.rs:560): the normal of the piece whose surface is nearest.
static V3 tool_outward_normal(const ix_tool& t, V3 p) {
    Piece ps[6];
    const int n = tool_pieces(t, ps);
    if (n == 0) return v3(0.0f, 0.0f, 1.0f);
    F best = INFINITY;
    V3 best_n = v3(0.0f, 0.0f, 1.0f);
    for (int i = 0; i < n; ++i) {
        V3 nn;
        const F sd = piece_sd_normal(ps[i], p, &nn);
        if (abs_(sd) < best) {
            best = abs_(sd);
            best_n = nn;
        }
    }
    return best_n;
}
// contains (tool.rs:545).
static bool tool_contains(const ix_tool& t, V3 p) {
    Piece ps[6];
    const int n = tool_pieces(t, ps);
    for (int i = 0; i < n; ++i) {
        V3 nn;
        if (piece_sd_normal(ps[i], p, &nn) <= F(0.0f)) return true;
    }
    return false;
}
// f32::total_cmp's key: the bits, negatives' magnitude bits flipped, compared signed.
static inline int32_t total_order_key(F t) {
    int32_t b;
    const float f = raw(t);
    std::memcpy(&b, &f, 4);
    return b ^ (int32_t)(((uint32_t)(b >> 31)) >> 1);
}
// carve + intersect_stone_soa_side (intersect_stone.rs:62-170): the first boundary past
// 1e-4 where the ray's in-material state changes; *entering is the state after it.
static bool intersect_carved(const float* planes, uint32_t n_planes, const ix_tool* tools, uint32_t n_tools,
                             const Ray& ray, Hit* hit, bool* entering) {
    F t_near, t_far;
    int near_idx, far_idx;
    if (!slab_scan_raw(planes, n_planes, ray, &t_near, &near_idx, &t_far, &far_idx)) return false;
    if (t_near > t_far) return false;
    struct Ev {
        F t;
        uint32_t key;
    };
    std::vector<Ev> ev;
    ev.reserve(2 * n_tools + 2);
    ev.push_back({t_near, 0u});
    ev.push_back({t_far, 1u});
    for (uint32_t k = 0; k < n_tools && k < IX_MAX_TOOLS; ++k) {
        F c, d;
        if (tool_ray_interval(tools[k], ray, &c, &d)) {
            ev.push_back({c, 2u + 2u * k});
            ev.push_back({d, 3u + 2u * k});
        }
    }
    std::sort(ev.begin(), ev.end(), [](const Ev& x, const Ev& y) {
        const int32_t a = total_order_key(x.t), b = total_order_key(y.t);
        return a != b ? a < b : x.key < y.key;
    });
    int plane_depth = 0, tool_depth = 0;
    bool inside = false;
    for (const Ev& e : ev) {
        if (e.key == 0)
            ++plane_depth;
        else if (e.key == 1)
            --plane_depth;
        else if (e.key % 2 == 0)
            ++tool_depth;
        else
            --tool_depth;
        const bool now_inside = plane_depth > 0 && tool_depth <= 0;
        if (now_inside == inside) continue;
        inside = now_inside;
        if (e.t <= F(1e-4f)) continue;
        hit->t = e.t;
        if (e.key <= 1) {
            const int idx = e.key == 0 ? near_idx : far_idx;
            hit->normal = idx >= 0 ? load3(planes + 4 * idx) : v3(0.0f, 0.0f, 0.0f);
            hit->facet = idx >= 0 ? idx : 0;
        } else {
            const uint32_t ti = (e.key - 2u) / 2u;
            const V3 point = ray.origin + ray.dir * e.t;
            hit->normal = -tool_outward_normal(tools[ti], point);
            hit->facet = (int)(n_planes + ti);
        }
        *entering = now_inside;
        return true;
    }
    return false;
}
// intersect_stone_soa (intersect_stone.rs:136) for a scene: the slab alone for a convex
// stone.  *carved tells whether *entering was set.
static bool intersect_scene(const ix_scene* sc, const Ray& ray, Hit* hit, bool* carved, bool* entering) {
    *carved = sc->n_tools > 0 && sc->tools;
    if (!*carved) return intersect(sc->planes, sc->n_planes, ray, hit);
    return intersect_carved(sc->planes, sc->n_planes, sc->tools, sc->n_tools, ray, hit, entering);
}

// shading_normal_near_edge (intersect.rs:196).
static V3 shading_normal_near_edge(const float* planes, uint32_t n, V3 hit_point, int facet,
                                   V3 hit_normal, F radius) {
    if (radius <= F(0.0f)) return hit_normal;
    F nearest = INFINITY;
    V3 nearest_normal = hit_normal;
    for (uint32_t i = 0; i < n; ++i) {
        if ((int)i == facet) continue;
        V3 nrm = load3(planes + 4 * i);
        F dist = -(F(planes[4 * i + 3]) + dot(nrm, hit_point));
        if (dist < nearest) {
            nearest = dist;
            nearest_normal = nrm;
        }
    }
    if (nearest >= radius) return hit_normal;
    F t = clamp_(F(1.0f) - nearest / radius, 0.0f, 1.0f);
    F smooth_t = t * t * fma_(2.0f, -t, 3.0f);
    V3 bis = normalize_or_zero(hit_normal + nearest_normal);
    return normalize_or_zero(hit_normal * (F(1.0f) - smooth_t) + bis * smooth_t);
}

// ------------------------------------------------------------------------------------
// Refraction helpers (refraction/{tir,dispatch,reflect_refract,exit_split}.rs).
// ------------------------------------------------------------------------------------
static const F DIRECTION_MATCH_COS_TOL = 1.0f - 1e-6f;  // refraction/mod.rs:137
static const F R_UNPOL_PDF_MIN = 1e-4f;                  // refraction/mod.rs:143
static const F R_UNPOL_PDF_MAX = 1.0f - 1e-4f;           // refraction/mod.rs:146
static const F R_UNPOL_SELECT_MIN = 0.02f;               // refraction/mod.rs:153
static const F R_UNPOL_SELECT_MAX = 0.98f;               // refraction/mod.rs:156

// tir_phase_delta (refraction/tir.rs:33).
static inline F tir_phase_delta(F n1k, F cos_i, F sin_i) {
    F tan_half = (cos_i * sqrt_(max_(fma_(n1k * n1k * sin_i, sin_i, -1.0f), 0.0f))) /
                 max_(n1k * sin_i * sin_i, 1e-6f);
    return F(2.0f) * atan_(tan_half);
}
static inline void fresnel_rs_rp(F n1, F n2, F cos_i, F cos_t, F* r_s, F* r_p) {
    *r_s = fma_(n2, -cos_t, n1 * cos_i) / fma_(n2, cos_t, n1 * cos_i);
    *r_p = fma_(n1, -cos_t, n2 * cos_i) / fma_(n1, cos_t, n2 * cos_i);
}
static inline F r_unpol_of(F r_s, F r_p) { return F(0.5f) * fma_(r_p, r_p, r_s * r_s); }
static inline V3 reflect(V3 k, V3 n) { return k - F(2.0f) * dot(k, n) * n; }

// ------------------------------------------------------------------------------------
// Uniaxial birefringence helpers (optics/birefringence/uniaxial.rs, helpers.rs,
// absorption_tensor.rs; materials/optics.rs:42).
// ------------------------------------------------------------------------------------
static const uint32_t BIREFRINGENT_SPLIT_STREAM = 0x2545F491u;  // sampling.rs:17
static const uint32_t MODE_COUPLING_STREAM = 0xCC9E2D51u;       // sampling.rs:21

// extraordinary_index_at (materials/optics.rs:42).
static F extraordinary_index_at(const ix_material& m, F lambda_nm, F n_o) {
    if (m.has_e_dispersion) return dispersion_eval(m.e_dispersion, lambda_nm);
    return n_o + F(m.birefringence_delta);
}
// stable_orthonormal_basis (birefringence/helpers.rs:13).
static void stable_orthonormal_basis(V3 n, V3* t_out, V3* b_out) {
    V3 a = (abs_(n.x) > F(0.9f)) ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    V3 t = normalize_or_zero(a - n * dot(n, a));
    *t_out = t;
    if (b_out) *b_out = cross(n, t);
}
// effective_extraordinary_index (birefringence/uniaxial.rs:33).
static F effective_extraordinary_index(F n_o, F n_e, F theta) {
    if (abs_(n_o - n_e) < F(1e-5f)) return n_o;
    F sin_t = sin_(theta);
    F cos_t = cos_(theta);
    F ns = n_o * sin_t;
    F denom_sq = fma_(n_e * cos_t, n_e * cos_t, ns * ns);
    if (denom_sq <= F(1e-8f)) return n_o;
    return (n_o * n_e) / sqrt_(denom_sq);
}
// walk_off_from_sin_cos (birefringence/uniaxial.rs:56).
static F walk_off_from_sin_cos(F n_o, F n_e, F sin_t, F cos_t) {
    if (abs_(n_o - n_e) < F(1e-5f)) return 0.0f;
    F n_o2 = n_o * n_o;
    F n_e2 = n_e * n_e;
    F tan_rho = (((n_o2 - n_e2) * sin_t) * cos_t) /
                max_(fma_(n_e2 * cos_t, cos_t, (n_o2 * sin_t) * sin_t), 1e-6f);
    return atan_(tan_rho);
}
// extraordinary_poynting_dir (birefringence/uniaxial.rs:72).
static V3 extraordinary_poynting_dir(V3 w, V3 c, F n_o, F n_e) {
    F cos_theta = clamp_(dot(w, c), -1.0f, 1.0f);
    F abs_cos = abs_(cos_theta);
    F sin_t = sqrt_(max_((F(1.0f) - abs_cos) * (F(1.0f) + abs_cos), 0.0f));
    F delta = walk_off_from_sin_cos(n_o, n_e, sin_t, abs_cos);
    if (abs_(delta) < F(1e-5f)) return w;
    V3 c_proj = normalize_or_zero(c - cos_theta * w);
    if (length_squared(c_proj) < F(1e-6f)) return w;
    F sign = (cos_theta >= F(0.0f)) ? F(1.0f) : F(-1.0f);
    return normalize(w * cos_(delta) - (sign * c_proj) * sin_(delta));
}
// ordinary_eigen_polarization / extraordinary_eigen_polarization (uniaxial.rs:95-110).
static V3 ordinary_eigen_polarization(V3 w, V3 c) {
    V3 cr = cross(w, c);
    if (length_squared(cr) > F(1e-8f)) return normalize(cr);
    V3 t;
    stable_orthonormal_basis(normalize_or_zero(w), &t, nullptr);
    return t;
}
static V3 extraordinary_eigen_polarization(V3 w, V3 c) {
    return normalize_or_zero(cross(w, ordinary_eigen_polarization(w, c)));
}
// assigned_mode_e_field_uniaxial (birefringence/absorption_tensor.rs:144).
static V3 assigned_mode_e_field_uniaxial(V3 k, V3 c, bool is_e, F n_o_hero, F n_e_hero) {
    if (!is_e) return ordinary_eigen_polarization(k, c);
    V3 kc = cross(k, c);
    if (length_squared(kc) < F(1e-8f)) return extraordinary_eigen_polarization(k, c);
    V3 s = extraordinary_poynting_dir(k, c, n_o_hero, n_e_hero);
    return normalize(cross(kc, s));
}
// AbsorptionTensor3::uniaxial(..).quadratic_form (absorption_tensor.rs:39, :80): the
// tensor's local frame (a1, a2, c_hat) projected onto a unit field direction.
struct TensorFrame {
    V3 a1, a2, c;
};
static TensorFrame tensor_frame(V3 c_axis) {
    TensorFrame f;
    f.c = normalize_or_zero(c_axis);
    stable_orthonormal_basis(f.c, &f.a1, &f.a2);
    return f;
}
static F quadratic_form(const TensorFrame& f, F ao, F ae, V3 e) {
    F l0 = dot(f.a1, e), l1 = dot(f.a2, e), l2 = dot(f.c, e);
    return (ao * (l0 * l0) + ao * (l1 * l1)) + ae * (l2 * l2);
}
// AbsorptionTensor3::biaxial(alpha, beta, gamma, gamma_axis).quadratic_form
// (absorption_tensor.rs:28, :39): the same frame, beta along a2.
static F quadratic_form3(const TensorFrame& f, F ao, F ab, F ae, V3 e) {
    F l0 = dot(f.a1, e), l1 = dot(f.a2, e), l2 = dot(f.c, e);
    return (ao * (l0 * l0) + ab * (l1 * l1)) + ae * (l2 * l2);
}

// ------------------------------------------------------------------------------------
// Biaxial indicatrix (birefringence/biaxial.rs, helpers.rs).  The principal frame is the
// tensor frame of the gamma axis (from_gamma_axis, biaxial.rs:58): columns a1, a2, g.
// ------------------------------------------------------------------------------------
struct Indicatrix {
    F na, nb, ng;     // n_alpha <= n_beta <= n_gamma
    TensorFrame ax;   // a1 (alpha), a2 (beta), c (gamma)
};
// GemMaterial::biaxial_indicatrix (materials/optics.rs:16) at an already evaluated n_beta.
static Indicatrix make_indicatrix(const ix_material& m, F n_beta, const TensorFrame& ax) {
    Indicatrix I;
    I.nb = n_beta;
    I.na = n_beta - F(m.biaxial_delta_beta_alpha);
    I.ng = I.na + F(m.birefringence_delta);
    I.ax = ax;
    return I;
}
// axes.transpose() * v and axes * v (glam Mat3, column order).
static inline V3 to_local(const TensorFrame& f, V3 v) { return v3(dot(f.a1, v), dot(f.a2, v), dot(f.c, v)); }
static inline V3 to_world(const TensorFrame& f, V3 l) { return (f.a1 * l.x + f.a2 * l.y) + f.c * l.z; }
// cross_fma / dot_fma (helpers.rs:42, :52).
static inline V3 cross_fma(V3 a, V3 b) {
    return v3(fma_(a.y, b.z, -(a.z * b.y)), fma_(a.z, b.x, -(a.x * b.z)), fma_(a.x, b.y, -(a.y * b.x)));
}
static inline F dot_fma(V3 a, V3 b) { return fma_(a.x, b.x, fma_(a.y, b.y, a.z * b.z)); }
// canonicalize_eigenvector_sign (helpers.rs:27).
static inline V3 canonical_sign(V3 v) {
    F ax = abs_(v.x), ay = abs_(v.y), az = abs_(v.z);
    F largest = (ax >= ay && ax >= az) ? v.x : (ay >= az ? v.y : v.z);
    return largest < F(0.0f) ? -v : v;
}
// indices_are_degenerate (biaxial.rs:176): |a - b| <= sqrt(f32::EPSILON) max(|a|, |b|, 1).
static inline bool indices_degenerate(F a, F b) {
    F scale = max_(max_(abs_(a), abs_(b)), 1.0f);
    return abs_(a - b) <= F(std::sqrt(FLT_EPSILON)) * scale;
}
// uniaxial_wave_indices (biaxial.rs:160).
static void uniaxial_wave_indices(V3 k, V3 c, F n_o, F n_e, F* n_slow, F* n_fast) {
    F theta = acos_(abs_(clamp_(dot(k, c), -1.0f, 1.0f)));
    F n_eff = effective_extraordinary_index(n_o, n_e, theta);
    *n_slow = max_(n_o, n_eff);
    *n_fast = min_(n_o, n_eff);
}
// BiaxialIndicatrix::wave_indices (biaxial.rs:105): Fresnel's equation of the wave
// normals as a quadratic in x = 1/n^2, with the degenerate closed forms first.
static void wave_indices(const Indicatrix& I, V3 wave_normal, F* n_slow, F* n_fast) {
    V3 k = normalize_or_zero(wave_normal);
    bool ab = indices_degenerate(I.na, I.nb), bg = indices_degenerate(I.nb, I.ng);
    if (ab && bg) {
        F n = ((I.na + I.nb) + I.ng) / F(3.0f);
        *n_slow = n;
        *n_fast = n;
        return;
    }
    if (ab) return uniaxial_wave_indices(k, I.ax.c, midpoint_(I.na, I.nb), I.ng, n_slow, n_fast);
    if (bg) return uniaxial_wave_indices(k, I.ax.a1, midpoint_(I.nb, I.ng), I.na, n_slow, n_fast);
    V3 l = to_local(I.ax, k);
    F a2 = l.x * l.x, b2 = l.y * l.y, g2 = l.z * l.z;
    F b1 = F(1.0f) / (I.na * I.na), b2c = F(1.0f) / (I.nb * I.nb), b3 = F(1.0f) / (I.ng * I.ng);
    F big_b = fma_(a2, b2c + b3, fma_(b2, b1 + b3, g2 * (b1 + b2c)));
    F big_c = fma_(a2, b2c * b3, fma_(b2, b1 * b3, (g2 * b1) * b2c));
    F disc = sqrt_(max_(fma_(big_b, big_b, F(-4.0f) * big_c), 0.0f));
    F x_lo = F(0.5f) * (big_b - disc);
    F x_hi = midpoint_(big_b, disc);
    *n_slow = F(1.0f) / sqrt_(max_(x_lo, 1e-12f));
    *n_fast = F(1.0f) / sqrt_(max_(x_hi, 1e-12f));
}
// precise_root_near (biaxial.rs:288): the root of the same quadratic nearest x, from the
// cancellation-free form of the discriminant.
static F precise_root_near(V3 l, const F b[3], F x) {
    F a = l.x * l.x, bb = l.y * l.y, cc = l.z * l.z;
    F big_b = fma_(a, b[1] + b[2], fma_(bb, b[0] + b[2], cc * (b[0] + b[1])));
    F xd = b[0] - b[1], yd = b[2] - b[0];
    F a_plus_c = a + cc, a_plus_bb = a + bb;
    F two_a_minus_bc = F(2.0f) * fma_(bb, -cc, a);
    F disc_sq = fma_(a_plus_c * a_plus_c, xd * xd, fma_(a_plus_bb * a_plus_bb, yd * yd, (two_a_minus_bc * xd) * yd));
    F disc = sqrt_(max_(disc_sq, 0.0f));
    F x_lo = F(0.5f) * (big_b - disc);
    F x_hi = midpoint_(big_b, disc);
    return abs_(x - x_lo) <= abs_(x - x_hi) ? x_lo : x_hi;
}
// eigenvector_world (biaxial.rs:243): the null direction of Gamma - x I as the
// sign-aligned sum of its three row-pair cross products.
static V3 eigenvector_world(const Indicatrix& I, V3 l, const F b[3], F x_in, V3 k_hat) {
    F x = precise_root_near(l, b, x_in);
    F s = fma_(b[0], l.x * l.x, fma_(b[1], l.y * l.y, (b[2] * l.z) * l.z));
    F m00 = fma_(l.x * l.x, fma_(F(2.0f), -b[0], s), b[0] - x);
    F m11 = fma_(l.y * l.y, fma_(F(2.0f), -b[1], s), b[1] - x);
    F m22 = fma_(l.z * l.z, fma_(F(2.0f), -b[2], s), b[2] - x);
    F m01 = (l.x * l.y) * ((s - b[0]) - b[1]);
    F m02 = (l.x * l.z) * ((s - b[0]) - b[2]);
    F m12 = (l.y * l.z) * ((s - b[1]) - b[2]);
    V3 r0 = v3(m00, m01, m02), r1 = v3(m01, m11, m12), r2 = v3(m02, m12, m22);
    V3 c01 = cross_fma(r0, r1), c02 = cross_fma(r0, r2), c12 = cross_fma(r1, r2);
    F s02 = dot_fma(c01, c02) < F(0.0f) ? F(-1.0f) : F(1.0f);
    F s12 = dot_fma(c01, c12) < F(0.0f) ? F(-1.0f) : F(1.0f);
    V3 vl = (c01 + c02 * s02) + c12 * s12;
    V3 vw = to_world(I.ax, vl);
    if (length_squared(vw) > F(1e-12f)) return normalize(canonical_sign(vw));
    V3 t;
    stable_orthonormal_basis(k_hat, &t, nullptr);
    return t;
}
// eigen_polarizations (biaxial.rs:197): the D direction of the slow (want_slow) or fast mode.
static V3 eigen_polarization(const Indicatrix& I, V3 wave_normal, bool want_slow) {
    V3 k = normalize_or_zero(wave_normal);
    V3 l = to_local(I.ax, k);
    F b[3] = {F(1.0f) / (I.na * I.na), F(1.0f) / (I.nb * I.nb), F(1.0f) / (I.ng * I.ng)};
    F ns, nf;
    wave_indices(I, wave_normal, &ns, &nf);
    F n = want_slow ? ns : nf;
    return eigenvector_world(I, l, b, F(1.0f) / (n * n), k);
}
// d_to_e_direction (biaxial.rs:322).
static V3 d_to_e_direction(const Indicatrix& I, V3 d) {
    V3 dl = to_local(I.ax, d);
    V3 el = v3(dl.x / (I.na * I.na), dl.y / (I.nb * I.nb), dl.z / (I.ng * I.ng));
    return normalize_or_zero(to_world(I.ax, el));
}
// poynting_direction (biaxial.rs:468).
static V3 poynting_direction(V3 wave_normal, V3 e_field) {
    V3 k = normalize_or_zero(wave_normal);
    V3 e = normalize_or_zero(e_field);
    V3 perp = k - e * dot(e, k);
    F len2 = length_squared(perp);
    if (len2 > F(1e-10f)) {
        F len = sqrt_(len2);
        return v3(perp.x / len, perp.y / len, perp.z / len);
    }
    return k;
}
// mode_poynting_dir (biaxial.rs:420) and assigned_mode_e_field (biaxial.rs:438): mode B
// (is_extraordinary) is the slow D eigenvector, mode A the fast one.
static V3 mode_poynting_dir(const Indicatrix& I, V3 wave_normal, bool want_slow) {
    V3 e = d_to_e_direction(I, eigen_polarization(I, wave_normal, want_slow));
    return poynting_direction(wave_normal, e);
}
static V3 assigned_mode_e_field_biaxial(const Indicatrix& I, V3 wave_normal, bool is_e) {
    return d_to_e_direction(I, eigen_polarization(I, wave_normal, is_e));
}
// resolve_entry_mode (biaxial.rs:370): two fixed-point steps of Snell's law against the
// mode's own direction-dependent index, seeded with n_seed.
static F resolve_entry_mode(const Indicatrix& I, V3 incident, V3 normal, F cos_i, F n_seed, bool want_slow,
                            V3* wave_dir_out) {
    F n_guess = n_seed;
    V3 wave_dir = incident;
    for (int it = 0; it < 2; ++it) {
        F eta = F(1.0f) / n_guess;
        F s2 = eta * eta * fma_(cos_i, -cos_i, 1.0f);
        if (s2 > F(1.0f)) break;
        F ct = sqrt_(max_(F(1.0f) - s2, 0.0f));
        wave_dir = normalize(eta * incident + fma_(eta, cos_i, -ct) * normal);
        F ns, nf;
        wave_indices(I, wave_dir, &ns, &nf);
        n_guess = want_slow ? ns : nf;
    }
    *wave_dir_out = wave_dir;
    return n_guess;
}

// ------------------------------------------------------------------------------------
// Closed-form uniaxial interface solves (raytracer/uniaxial_fresnel/*.rs, after Lekner,
// J. Phys.: Condens. Matter 3 (1991) 6121).
// ------------------------------------------------------------------------------------
struct Cx {
    F re, im;
};
static inline Cx cx(F re, F im) { return Cx{re, im}; }
static inline Cx cadd(Cx a, Cx b) { return cx(a.re + b.re, a.im + b.im); }
static inline Cx csub(Cx a, Cx b) { return cx(a.re - b.re, a.im - b.im); }
static inline Cx cmul(Cx a, Cx b) { return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline Cx cscale(Cx a, F s) { return cx(a.re * s, a.im * s); }
static inline Cx cconj(Cx a) { return cx(a.re, -a.im); }
static inline Cx cneg(Cx a) { return csub(cx(0.0f, 0.0f), a); }  // Cplx::ZERO.sub(a)
static inline F cnorm2(Cx a) { return fma_(a.im, a.im, a.re * a.re); }
// Cplx::div (complex.rs:79).
static inline Cx cdiv(Cx a, Cx o) {
    F denom = max_(fma_(o.im, o.im, o.re * o.re), 1e-20f);
    return cx(fma_(a.im, o.im, a.re * o.re) / denom, fma_(a.re, -o.im, a.im * o.re) / denom);
}
// Cplx::sqrt_forward_branch (complex.rs:109).
static Cx csqrt_fwd(Cx a) {
    if (raw(a.im) == 0.0f && a.re < F(0.0f)) return cx(0.0f, sqrt_(-a.re));
    F r = sqrt_(sqrt_(cnorm2(a)));
    F theta = atan2_(a.im, a.re) * F(0.5f);
    Cx out = cx(r * cos_(theta), r * sin_(theta));
    if (out.re < F(0.0f)) out = cx(-out.re, -out.im);
    if (abs_(out.re) < F(1e-9f) && out.im < F(0.0f)) out = cx(-out.re, -out.im);
    return out;
}
struct CV3 {
    V3 re, im;
};
static inline CV3 cv_real(V3 v) { return CV3{v, v3(0.0f, 0.0f, 0.0f)}; }
static inline CV3 cv_wavevector(V3 that, V3 zhat, F tangential, Cx q) {
    return CV3{that * tangential + zhat * q.re, zhat * q.im};
}
static inline CV3 cv_add(CV3 a, CV3 b) { return CV3{a.re + b.re, a.im + b.im}; }
static inline CV3 cv_scale_real(CV3 a, F s) { return CV3{a.re * s, a.im * s}; }
static inline CV3 cv_scale(CV3 a, Cx s) {
    return CV3{a.re * s.re - a.im * s.im, a.re * s.im + a.im * s.re};
}
static inline CV3 cv_cross_real(CV3 a, V3 r) { return CV3{cross(a.re, r), cross(a.im, r)}; }
static inline CV3 cv_cross(CV3 a, CV3 b) {
    return CV3{cross(a.re, b.re) - cross(a.im, b.im), cross(a.re, b.im) + cross(a.im, b.re)};
}
static inline Cx cv_dot_real(CV3 a, V3 r) { return cx(dot(a.re, r), dot(a.im, r)); }
static inline CV3 cv_conj(CV3 a) { return CV3{a.re, -a.im}; }

// UniaxialFrame::build (uniaxial_fresnel/frame.rs:55).
struct UFrame {
    V3 that, zhat, s_axis;
    F cos_i, sin_i, alpha, beta, gamma;
};
static UFrame uframe_build(V3 k, V3 normal, V3 c, F cos_i, F sin_i) {
    UFrame f;
    f.zhat = -normal;
    if (sin_i > F(1e-5f)) {
        V3 t = k + normal * cos_i;
        f.that = normalize_or_zero(v3(t.x / sin_i, t.y / sin_i, t.z / sin_i));
    } else {
        V3 fb = (abs_(f.zhat.x) < F(0.9f)) ? v3(1.0f, 0.0f, 0.0f) : v3(0.0f, 1.0f, 0.0f);
        f.that = normalize_or_zero(fb - f.zhat * dot(f.zhat, fb));
    }
    V3 s = normalize_or_zero(cross(k, normal));
    f.s_axis = (length_squared(s) > F(1e-8f)) ? s : normalize_or_zero(cross(f.zhat, f.that));
    f.cos_i = cos_i;
    f.sin_i = sin_i;
    f.alpha = dot(c, f.that);
    f.beta = dot(c, f.s_axis);
    f.gamma = dot(c, f.zhat);
    return f;
}
// uniaxial_q_roots (frame.rs:111).
struct QRoots {
    Cx qo_plus, qo_minus, qe_plus, qe_minus;
};
static QRoots uniaxial_q_roots(F n_o, F n_e, const UFrame& f, F tangential) {
    QRoots r;
    F n_o2 = n_o * n_o;
    F k2 = tangential * tangential;
    r.qo_plus = csqrt_fwd(cx(n_o2 - k2, 0.0f));
    r.qo_minus = cneg(r.qo_plus);
    if (raw(n_o) == raw(n_e)) {
        r.qe_plus = r.qo_plus;
        r.qe_minus = r.qo_minus;
        return r;
    }
    F n_e2 = n_e * n_e;
    F deleps = n_e2 - n_o2;
    F denom = fma_(f.gamma * f.gamma, deleps, n_o2);
    F d_val = n_o2 * fma_(fma_(f.beta * f.beta, -deleps, n_e2), -k2,
                          n_e2 * fma_(f.gamma * f.gamma, deleps, n_o2));
    Cx sqrt_d = csqrt_fwd(cx(d_val, 0.0f));
    Cx shift = cx(((f.alpha * f.gamma) * tangential) * deleps, 0.0f);
    Cx denom_c = cx(max_(denom, 1e-12f), 0.0f);
    r.qe_plus = cdiv(csub(sqrt_d, shift), denom_c);
    r.qe_minus = cdiv(csub(cneg(sqrt_d), shift), denom_c);
    return r;
}
// ModeFields (frame.rs:176-232): E and H of one eigenmode at amplitude 1.
struct Mode {
    CV3 e, h;
};
static Mode ordinary_mode(F n_o, V3 c, const UFrame& f, F tangential, Cx q) {
    CV3 k = cv_wavevector(f.that, f.zhat, tangential, q);
    CV3 d_o = cv_cross_real(k, c);
    Mode m;
    m.e = cv_scale_real(d_o, F(1.0f) / (n_o * n_o));
    m.h = cv_cross(k, m.e);
    return m;
}
static Mode extraordinary_mode(F n_o, F n_e, V3 c, const UFrame& f, F tangential, Cx q) {
    F n_o2 = n_o * n_o;
    F n_e2 = n_e * n_e;
    F deleps = n_e2 - n_o2;
    CV3 k = cv_wavevector(f.that, f.zhat, tangential, q);
    CV3 d_o = cv_cross_real(k, c);
    CV3 d_e = cv_cross(k, d_o);
    Cx c_dot_de = cv_dot_real(d_e, c);
    Mode m;
    m.e = cv_add(cv_scale_real(d_e, F(1.0f) / n_o2),
                 cv_scale(cv_real(c), cscale(c_dot_de, -(deleps / (n_o2 * n_e2)))));
    m.h = cv_cross(k, m.e);
    return m;
}
static Mode iso_mode(CV3 k, CV3 e) { return Mode{e, cv_cross(k, e)}; }
// poynting_z (frame.rs:237) at amplitude 1.
static F poynting_z(const Mode& m, V3 zhat) {
    Cx one = cx(1.0f, 0.0f);
    CV3 e = cv_scale(m.e, one);
    CV3 h = cv_scale(m.h, one);
    CV3 s = cv_cross(e, cv_conj(h));
    return F(0.5f) * cv_dot_real(s, zhat).re;
}
// tangential_components (linalg.rs:264).
static void tangential(const Mode& m, const UFrame& f, Cx out[4]) {
    out[0] = cv_dot_real(m.e, f.that);
    out[1] = cv_dot_real(m.e, f.s_axis);
    out[2] = cv_dot_real(m.h, f.that);
    out[3] = cv_dot_real(m.h, f.s_axis);
}
// solve4 / solve4_two_rhs (linalg.rs:172, :217): Gauss-Jordan with partial pivoting
// (strictly larger |.|^2 wins), applied to nrhs right-hand sides in lockstep.
static void solve4(Cx a[4][4], Cx* b[], int nrhs) {
    for (int col = 0; col < 4; ++col) {
        int piv = col;
        F piv_mag = cnorm2(a[col][col]);
        for (int row = col + 1; row < 4; ++row) {
            F mag = cnorm2(a[row][col]);
            if (mag > piv_mag) {
                piv = row;
                piv_mag = mag;
            }
        }
        for (int j = 0; j < 4; ++j) std::swap(a[col][j], a[piv][j]);
        for (int r = 0; r < nrhs; ++r) std::swap(b[r][col], b[r][piv]);
        Cx pivot = a[col][col];
        for (int j = col; j < 4; ++j) a[col][j] = cdiv(a[col][j], pivot);
        for (int r = 0; r < nrhs; ++r) b[r][col] = cdiv(b[r][col], pivot);
        for (int row = 0; row < 4; ++row) {
            if (row == col) continue;
            Cx factor = a[row][col];
            if (raw(cnorm2(factor)) == 0.0f) continue;
            for (int j = col; j < 4; ++j) a[row][j] = csub(a[row][j], cmul(factor, a[col][j]));
            for (int r = 0; r < nrhs; ++r) b[r][row] = csub(b[r][row], cmul(factor, b[r][col]));
        }
    }
}
// EntryIncidenceFrame / entry_incidence_frame (entry.rs:95-147).
struct EntryInc {
    Cx inc_s[4], inc_p[4], refl_s[4], refl_p[4];
};
static EntryInc entry_incidence_frame(F n1, const UFrame& f) {
    F k_tan = n1 * f.sin_i;
    CV3 k_fwd = cv_wavevector(f.that, f.zhat, k_tan, cx(n1 * f.cos_i, 0.0f));
    CV3 k_bwd = cv_wavevector(f.that, f.zhat, k_tan, cx(-n1 * f.cos_i, 0.0f));
    CV3 s_c = cv_real(f.s_axis);
    CV3 ep_bwd = cv_scale_real(cv_cross(k_bwd, s_c), F(-1.0f) / (n1 * n1));
    CV3 ep_fwd = cv_scale_real(cv_cross(k_fwd, s_c), F(-1.0f) / (n1 * n1));
    EntryInc e;
    tangential(iso_mode(k_fwd, s_c), f, e.inc_s);
    tangential(iso_mode(k_fwd, ep_fwd), f, e.inc_p);
    tangential(iso_mode(k_bwd, s_c), f, e.refl_s);
    tangential(iso_mode(k_bwd, ep_bwd), f, e.refl_p);
    return e;
}
// EntryPolarizationSolution (entry.rs:23) for s and p incidence.
struct EntrySol {
    Cx r_s[2], r_p[2], t_o[2], t_e[2];  // [0] = s incidence, [1] = p incidence
    F flux_o, flux_e;
    V3 o_hat, e_hat;
};
// entry_solve_pair_with_incidence (entry.rs:173).
static EntrySol entry_solve(const EntryInc& inc, F n1, F n_o, F n_e, V3 c, const UFrame& f) {
    F k_tan = n1 * f.sin_i;
    QRoots q = uniaxial_q_roots(n_o, n_e, f, k_tan);
    Mode fo = ordinary_mode(n_o, c, f, k_tan, q.qo_plus);
    Mode fe = extraordinary_mode(n_o, n_e, c, f, k_tan, q.qe_plus);
    Cx oc[4], ec[4];
    tangential(fo, f, oc);
    tangential(fe, f, ec);
    Cx a[4][4], bs[4], bp[4];
    for (int i = 0; i < 4; ++i) {
        a[i][0] = inc.refl_s[i];
        a[i][1] = inc.refl_p[i];
        a[i][2] = cneg(oc[i]);
        a[i][3] = cneg(ec[i]);
        bs[i] = cneg(inc.inc_s[i]);
        bp[i] = cneg(inc.inc_p[i]);
    }
    Cx* rhs[2] = {bs, bp};
    solve4(a, rhs, 2);
    EntrySol s;
    for (int p = 0; p < 2; ++p) {
        s.r_s[p] = rhs[p][0];
        s.r_p[p] = rhs[p][1];
        s.t_o[p] = rhs[p][2];
        s.t_e[p] = rhs[p][3];
    }
    s.flux_o = abs_(poynting_z(fo, f.zhat));
    s.flux_e = abs_(poynting_z(fe, f.zhat));
    s.o_hat = normalize_or_zero(fo.e.re);
    s.e_hat = normalize_or_zero(fe.e.re);
    return s;
}
// InternalPolarizationSolution / internal_solve (internal.rs:265, :334).
struct IntSol {
    Cx r_o, r_e, t_s, t_p;
    F flux_ro, flux_re, flux_ts, flux_tp, flux_inc;
};
static IntSol internal_solve(F n_mode_inc, F n_o, F n_e, V3 c, const UFrame& f, bool inc_ordinary) {
    F k_tan = n_mode_inc * f.sin_i;
    QRoots q = uniaxial_q_roots(n_o, n_e, f, k_tan);
    Mode f_inc = inc_ordinary ? ordinary_mode(n_o, c, f, k_tan, q.qo_plus)
                              : extraordinary_mode(n_o, n_e, c, f, k_tan, q.qe_plus);
    Mode f_o_bwd = ordinary_mode(n_o, c, f, k_tan, q.qo_minus);
    Mode f_e_bwd = extraordinary_mode(n_o, n_e, c, f, k_tan, q.qe_minus);
    const F n2 = 1.0f;
    F zeta = k_tan / n2;
    Cx cos_t = (abs_(zeta) <= F(1.0f)) ? cx(sqrt_(max_(fma_(zeta, -zeta, 1.0f), 0.0f)), 0.0f)
                                       : cx(0.0f, sqrt_(fma_(zeta, zeta, -1.0f)));
    CV3 k_iso = cv_wavevector(f.that, f.zhat, k_tan, cscale(cos_t, n2));
    CV3 s_c = cv_real(f.s_axis);
    CV3 ep_t = cv_scale_real(cv_cross(k_iso, s_c), F(-1.0f) / (n2 * n2));
    Mode f_s_t = iso_mode(k_iso, s_c);
    Mode f_p_t = iso_mode(k_iso, ep_t);
    Cx inc_c[4], eo_c[4], ee_c[4], es_c[4], ep_c[4];
    tangential(f_inc, f, inc_c);
    tangential(f_o_bwd, f, eo_c);
    tangential(f_e_bwd, f, ee_c);
    tangential(f_s_t, f, es_c);
    tangential(f_p_t, f, ep_c);
    Cx a[4][4], b[4];
    for (int i = 0; i < 4; ++i) {
        a[i][0] = eo_c[i];
        a[i][1] = ee_c[i];
        a[i][2] = cneg(es_c[i]);
        a[i][3] = cneg(ep_c[i]);
        b[i] = cneg(inc_c[i]);
    }
    Cx* rhs[1] = {b};
    solve4(a, rhs, 1);
    IntSol s;
    s.r_o = b[0];
    s.r_e = b[1];
    s.t_s = b[2];
    s.t_p = b[3];
    s.flux_ro = abs_(poynting_z(f_o_bwd, f.zhat));
    s.flux_re = abs_(poynting_z(f_e_bwd, f.zhat));
    s.flux_ts = abs_(poynting_z(f_s_t, f.zhat));
    s.flux_tp = abs_(poynting_z(f_p_t, f.zhat));
    s.flux_inc = abs_(poynting_z(f_inc, f.zhat));
    return s;
}
// azimuth2_in_frame (mueller.rs:455).
static void azimuth2_in_frame(V3 dir, V3 s_axis, V3 p_axis, F* cos2, F* sin2) {
    F s = dot(dir, s_axis);
    F p = dot(dir, p_axis);
    F norm = max_(fma_(p, p, s * s), 1e-12f);
    *cos2 = fma_(p, -p, s * s) / norm;
    *sin2 = ((F(2.0f) * s) * p) / norm;
}
// jones_to_mueller (mueller.rs:478), column-major like glam's Mat4.
static M4 jones_to_mueller(Cx j_ss, Cx j_sp, Cx j_ps, Cx j_pp) {
    F m_ss = cnorm2(j_ss), m_sp = cnorm2(j_sp), m_ps = cnorm2(j_ps), m_pp = cnorm2(j_pp);
    Cx a_ssp = cmul(j_ss, cconj(j_sp));
    Cx a_pep = cmul(j_ps, cconj(j_pp));
    Cx a_plus = cadd(a_ssp, a_pep);
    Cx a_minus = csub(a_ssp, a_pep);
    Cx b_sp = cmul(j_ss, cconj(j_ps));
    Cx b_pp = cmul(j_sp, cconj(j_pp));
    Cx c_sspp = cmul(j_ss, cconj(j_pp));
    Cx c_spps = cmul(j_sp, cconj(j_ps));
    F i_i = F(0.5f) * (((m_ss + m_ps) + m_sp) + m_pp);
    F i_q = F(0.5f) * (((m_ss + m_ps) - m_sp) - m_pp);
    F i_u = a_plus.re, i_v = a_plus.im;
    F q_i = F(0.5f) * (((m_ss - m_ps) + m_sp) - m_pp);
    F q_q = midpoint_((m_ss - m_ps) - m_sp, m_pp);
    F q_u = a_minus.re, q_v = a_minus.im;
    F u_i = b_sp.re + b_pp.re;
    F u_q = b_sp.re - b_pp.re;
    F u_u = c_sspp.re + c_spps.re;
    F u_v = c_sspp.im - c_spps.im;
    F v_i = -(b_sp.im + b_pp.im);
    F v_q = -(b_sp.im) + b_pp.im;
    F v_u = -(c_sspp.im + c_spps.im);
    F v_v = c_sspp.re - c_spps.re;
    return M4{{i_i, q_i, u_i, v_i, i_q, q_q, u_q, v_q, i_u, q_u, u_u, v_u, i_v, q_v, u_v, v_v}};
}
// mode_power (mueller.rs:541).
static F mode_power(Cx t_s, Cx t_p, F mode_flux, F inc_flux, const Stokes& st) {
    F m_s = cnorm2(t_s);
    F m_p = cnorm2(t_p);
    Cx cr = cmul(t_s, cconj(t_p));
    F rawv = fma_(cr.im, st.v, fma_(cr.re, st.u, F(0.5f) * fma_(m_s, st.i + st.q, m_p * (st.i - st.q))));
    return (mode_flux / max_(inc_flux, 1e-12f)) * rawv;
}
// entry_eigenmode_selection (refraction/uniaxial_entry.rs:50): returns false for None.
static bool entry_eigenmode_selection(V3 c, V3 cpn, V3 k, const Stokes& hs, F* p_o, F* cos2,
                                      F* sin2) {
    if (hs.i <= F(1e-7f) || length_squared(cpn) <= F(1e-6f)) return false;
    if (fma_(hs.q, hs.q, hs.u * hs.u) <= F(1e-12f)) return false;
    V3 o_hat = ordinary_eigen_polarization(k, c);
    V3 p_hat = cross(k, cpn);
    F s_comp = dot(o_hat, cpn);
    F p_comp = dot(o_hat, p_hat);
    *cos2 = fma_(s_comp, s_comp, -(p_comp * p_comp));
    *sin2 = (F(2.0f) * s_comp) * p_comp;
    *p_o = clamp_(F(0.5f) + (F(0.5f) * fma_(hs.q, *cos2, hs.u * *sin2)) / hs.i, 0.0f, 1.0f);
    return true;
}

// ------------------------------------------------------------------------------------
// One traced path (transport/inner/bounce_body.rs:216-764).
// ------------------------------------------------------------------------------------
struct Path {
    const ix_scene* sc;
    uint32_t seed;
    F lambdas[8];
    F n_ch[8];     // ordinary (or isotropic) index per channel
    F n_e_at[8];   // extraordinary_index_at per channel (uniaxial only)
    F alpha_ch_o[8];
    F alpha_ch_e[8];
    F alpha_ch_b[8];  // beta-ray absorption (biaxial only; the alpha-ray value without abs_beta)
    bool absorbing;
    bool aniso;
    bool biaxial;     // biaxial indicatrix (cache.hero_indicatrix.is_some())
    bool has_carry;   // pending_light_mis: the BSDF pdf of the last light-sampled bounce's
    F carry_pdf;      // continuation, consumed by the next escape (bounce_body.rs:372)
    TensorFrame ax;   // principal / absorption frame of the optic (gamma) axis
    bool is_e;  // the eigenmode assigned at the last entry (or by internal coupling)
    V3 c_axis;  // the material's optic axis as stored (RayMaterialContext::c_axis)
    Stokes stokes[8];
    F radiance[8];
    F path_pdf[8];
    F split[8];
    uint8_t compat[8];
    Ray ray;
    V3 k;
    bool inside;
    bool has_prev;
    V3 prev_pn;
    bool escaped;
    V3 observer;
    uint32_t splits;
};

// try_split_exit_channel (refraction/exit_split.rs:128).
static void try_split_exit_channel(Path& P, V3 hit_point, int k, V3 dir_k, F transmitted_i) {
    Ray probe{hit_point + dir_k * F(1e-4f), dir_k};
    Hit h;
    bool carved, entering;
    if (intersect_scene(P.sc, probe, &h, &carved, &entering)) return;
    F env = environment_channel(P.sc->environment, dir_k, P.lambdas[k], P.observer);
    P.split[k] = fma_(max_(transmitted_i, 0.0f) * F(1.0f), env, P.split[k]);
    P.splits++;
}

// narrow_compat (refraction/context.rs:219) with the hero at channel 0.
static void narrow_compat(Path& P, const V3 dirs[8], const bool have_dir[8], const bool hero_match[8]) {
    for (int a = 0; a < 8; ++a)
        for (int b = a + 1; b < 8; ++b) {
            bool m;
            if (a == 0)
                m = hero_match[b];
            else if (have_dir[a] && have_dir[b])
                m = dot(dirs[a], dirs[b]) >= DIRECTION_MATCH_COS_TOL;
            else
                m = true;
            if (!m) {
                P.compat[a] &= (uint8_t)~(1u << b);
                P.compat[b] &= (uint8_t)~(1u << a);
            }
        }
}

// Snell-refracted wave normal at index ratio eta (reflect_refract.rs:192-197).
static inline V3 snell_dir(F eta, F cos_i, V3 k, V3 normal) {
    F sin2_t = min_(eta * eta * fma_(cos_i, -cos_i, 1.0f), 1.0f);
    F cos_t = sqrt_(max_(F(1.0f) - sin2_t, 0.0f));
    return normalize(eta * k + fma_(eta, cos_i, -cos_t) * normal);
}

// BounceRefractionGeometry (refraction/geometry.rs:24, :306) for an isotropic or a
// uniaxial material.
struct Geo {
    F cos_i, sin_i;
    F n_o_hero, n_e_hero;  // n_e_hero: the constant-offset form, used for walk-off only
    F n1, n2, sin2_t;
    F n1_ch[8], n2_ch[8], sin2_t_ch[8];
    bool has_frame;
    UFrame frame;
    // Biaxial material: mode A (fast root at the mode-A wave normal) and mode B (slow root
    // at the mode-B wave normal) indices per channel (geometry.rs:255).
    bool is_biaxial;
    F n_biax_a_ch[8], n_biax_b_ch[8];
};
// The hero channel's (channel 0's) and channel c's indicatrix.
static Indicatrix channel_indicatrix(const Path& P, int c) {
    return make_indicatrix(P.sc->material, P.n_ch[c], P.ax);
}

// theta_c_for_bounce (refraction/geometry.rs:75), uniaxial only.
static F theta_c_for_bounce(const Path& P, V3 normal, V3 k, F cos_i) {
    if (!P.inside) {
        F n_o_seed = P.n_ch[0];
        F n_e_seed = P.n_e_at[0];
        F n_guess = n_o_seed;
        F theta = 0.0f;
        for (int it = 0; it < 2; ++it) {
            F eta = F(1.0f) / n_guess;
            F s2 = eta * eta * fma_(cos_i, -cos_i, 1.0f);
            if (s2 > F(1.0f)) break;
            F ct = sqrt_(max_(F(1.0f) - s2, 0.0f));
            V3 w = normalize(eta * k + fma_(eta, cos_i, -ct) * normal);
            theta = acos_(abs_(clamp_(dot(w, P.c_axis), -1.0f, 1.0f)));
            n_guess = effective_extraordinary_index(n_o_seed, n_e_seed, theta);
        }
        return theta;
    }
    return acos_(abs_(clamp_(dot(k, P.c_axis), -1.0f, 1.0f)));
}

static Geo compute_geo(const Path& P, V3 normal) {
    Geo g;
    V3 k = P.k;
    g.cos_i = clamp_(dot(-k, normal), 0.0f, 1.0f);
    g.sin_i = sqrt_(max_(fma_(g.cos_i, -g.cos_i, 1.0f), 0.0f));
    F n_eff[8];
    if (P.aniso) {
        F theta = theta_c_for_bounce(P, normal, k, g.cos_i);
        for (int c = 0; c < 8; ++c) n_eff[c] = effective_extraordinary_index(P.n_ch[c], P.n_e_at[c], theta);
    } else {
        for (int c = 0; c < 8; ++c) n_eff[c] = P.n_ch[c];
    }
    g.n_o_hero = P.n_ch[0];
    g.n_e_hero = g.n_o_hero + F(P.sc->material.birefringence_delta);
    g.is_biaxial = P.biaxial;
    if (P.biaxial) {
        // hero_biaxial_wave_dirs + per_channel_biaxial_indices (geometry.rs:220-285): the
        // hero's indicatrix resolves each mode's wave normal on entry (the tracked wave
        // normal inside); every channel evaluates its own indicatrix there.
        const Indicatrix hero = channel_indicatrix(P, 0);
        V3 dir_a = k, dir_b = k;
        if (!P.inside) {
            resolve_entry_mode(hero, k, normal, g.cos_i, P.n_ch[0], false, &dir_a);
            resolve_entry_mode(hero, k, normal, g.cos_i, P.n_ch[0], true, &dir_b);
        }
        for (int c = 0; c < 8; ++c) {
            const Indicatrix ic = channel_indicatrix(P, c);
            F ns, nf;
            wave_indices(ic, dir_a, &ns, &nf);
            g.n_biax_a_ch[c] = nf;
            wave_indices(ic, dir_b, &ns, &nf);
            g.n_biax_b_ch[c] = ns;
        }
    }
    // n_medium_ch: mode A (the ordinary indices for a uniaxial material) while inside in
    // that mode, else mode B (n_eff).
    const bool ordinary_medium = P.aniso && P.inside && !P.is_e;
    F n_med[8];
    for (int c = 0; c < 8; ++c) {
        const F mode_a = P.biaxial ? g.n_biax_a_ch[c] : P.n_ch[c];
        const F mode_b = P.biaxial ? g.n_biax_b_ch[c] : n_eff[c];
        n_med[c] = ordinary_medium ? mode_a : mode_b;
    }
    g.n1 = P.inside ? n_med[0] : F(1.0f);
    g.n2 = P.inside ? F(1.0f) : n_med[0];
    F eta = g.n1 / g.n2;
    g.sin2_t = eta * eta * fma_(g.cos_i, -g.cos_i, 1.0f);
    for (int c = 0; c < 8; ++c) {
        g.n1_ch[c] = P.inside ? n_med[c] : F(1.0f);
        g.n2_ch[c] = P.inside ? F(1.0f) : n_med[c];
        F etak = g.n1_ch[c] / g.n2_ch[c];
        g.sin2_t_ch[c] = etak * etak * fma_(g.cos_i, -g.cos_i, 1.0f);
    }
    g.has_frame = P.aniso && !P.biaxial;
    if (g.has_frame) g.frame = uframe_build(k, normal, P.c_axis, g.cos_i, g.sin_i);
    return g;
}

// poynting_dir_for_mode (refraction/geometry.rs:440): both biaxial modes walk off.
static V3 poynting_dir_for_mode(const Path& P, const Geo& g, V3 k, bool inside, bool is_e) {
    if (!inside || !P.aniso) return k;
    if (g.is_biaxial) return mode_poynting_dir(channel_indicatrix(P, 0), k, is_e);
    if (!is_e) return k;
    return extraordinary_poynting_dir(k, P.c_axis, g.n_o_hero, g.n_e_hero);
}

// What one bounce dispatch decides (transport/bounce.rs:108-160).
struct Outcome {
    V3 new_k, new_s;
    bool new_inside;
    int update;  // -1: is_extraordinary unchanged, else its new value
    bool has_p_o;
    F p_o;  // the closed-form R_o / (R_o + R_e) for internal mode coupling
};

// apply_tir_bounce (refraction/tir.rs:41-116).
static void apply_tir_bounce(Path& P, const Geo& g, V3 k, V3 normal, Outcome* o) {
    if (g.has_frame && length_squared(cross(k, P.c_axis)) > F(1e-6f)) {
        for (int c = 0; c < 8; ++c) {
            IntSol sol = internal_solve(g.n1_ch[c], P.n_ch[c], P.n_e_at[c], P.c_axis, g.frame, !P.is_e);
            F flux_inc = max_(sol.flux_inc, 1e-12f);
            F ro_pow = cnorm2(sol.r_o) * sol.flux_ro;
            F re_pow = cnorm2(sol.r_e) * sol.flux_re;
            F r_total = min_((ro_pow + re_pow) / flux_inc, 1.0f);
            P.stokes[c] = scale(P.stokes[c], r_total);
            if (g.sin2_t_ch[c] <= F(1.0f))
                P.path_pdf[c] = P.path_pdf[c] * clamp_(r_total, R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
            if (c == 0) {
                o->has_p_o = true;
                o->p_o = ro_pow / max_(ro_pow + re_pow, 1e-12f);
            }
        }
    } else {
        for (int c = 0; c < 8; ++c) {
            F n1k = g.n1_ch[c], n2k = g.n2_ch[c];
            if (g.sin2_t_ch[c] > F(1.0f)) {
                P.stokes[c] = apply(tir_retardation(tir_phase_delta(n1k, g.cos_i, g.sin_i)), P.stokes[c]);
            } else {
                F cos_t_k = sqrt_(max_(F(1.0f) - g.sin2_t_ch[c], 0.0f));
                F r_s, r_p;
                fresnel_rs_rp(n1k, n2k, g.cos_i, cos_t_k, &r_s, &r_p);
                P.stokes[c] = apply(fresnel_reflection(r_s, r_p), P.stokes[c]);
                P.path_pdf[c] =
                    P.path_pdf[c] * clamp_(r_unpol_of(r_s, r_p), R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
            }
        }
    }
    o->new_k = reflect(k, normal);
    o->new_s = poynting_dir_for_mode(P, g, o->new_k, P.inside, P.is_e);
    o->new_inside = P.inside;
}

// apply_partial_reflect_bounce (refraction/reflect_refract.rs:33).
static void apply_partial_reflect(Path& P, const Geo& g, F r_unpol) {
    for (int c = 0; c < 8; ++c) {
        F n1k = g.n1_ch[c], n2k = g.n2_ch[c];
        M4 mm;
        if (g.sin2_t_ch[c] > F(1.0f)) {
            mm = tir_retardation(tir_phase_delta(n1k, g.cos_i, g.sin_i));
        } else {
            F cos_t_k = sqrt_(max_(F(1.0f) - g.sin2_t_ch[c], 0.0f));
            F rs, rp;
            fresnel_rs_rp(n1k, n2k, g.cos_i, cos_t_k, &rs, &rp);
            P.path_pdf[c] = P.path_pdf[c] * clamp_(r_unpol_of(rs, rp), R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
            mm = fresnel_reflection(rs, rp);
        }
        P.stokes[c] = scale(apply(mm, P.stokes[c]), F(1.0f) / r_unpol);
    }
}

// apply_refract_bounce + apply_refract_channel + compute_channel_transmission
// (refraction/reflect_refract.rs:121-591, exit_split.rs:51): the scalar-Fresnel refract
// branch of an isotropic material or of the degenerate uniaxial case.
static void apply_refract_bounce(Path& P, const Geo& g, F r_unpol, V3 k, V3 normal, V3 hit_point,
                                 bool use_e, bool has_az, F az_c, F az_s, Outcome* o) {
    const bool entering = !P.inside && P.aniso;
    const bool biaxial_entry = entering && g.is_biaxial;
    const F cos_i = g.cos_i;
    V3 refr, final_refr;
    if (biaxial_entry) {
        // The selected mode's own index and walk-off (reflect_refract.rs:160-180).
        F n2_hero_dir = use_e ? g.n_biax_b_ch[0] : g.n_biax_a_ch[0];
        refr = snell_dir(g.n1 / n2_hero_dir, cos_i, k, normal);
        final_refr = mode_poynting_dir(channel_indicatrix(P, 0), refr, use_e);
    } else {
        F n2_hero_dir = (entering && !use_e) ? g.n_o_hero : g.n2;
        refr = snell_dir(g.n1 / n2_hero_dir, cos_i, k, normal);
        final_refr = (entering && use_e) ? extraordinary_poynting_dir(refr, P.c_axis, g.n_o_hero, g.n_e_hero)
                                         : refr;
    }
    V3 dirs[8];
    bool have_dir[8];
    bool hero_match[8];
    for (int c = 0; c < 8; ++c) {
        Stokes original = P.stokes[c];
        F n1k = g.n1_ch[c];
        F n2k = (entering && !use_e) ? (g.is_biaxial ? g.n_biax_a_ch[c] : P.n_ch[c]) : g.n2_ch[c];
        F ratio = n1k / n2k;
        F sin2_t_k = (ratio * ratio) * fma_(cos_i, -cos_i, 1.0f);
        if (sin2_t_k > F(1.0f)) {
            P.stokes[c] = scale(P.stokes[c], 0.0f);
            P.path_pdf[c] = 0.0f;
            have_dir[c] = false;
            hero_match[c] = false;
            continue;
        }
        F cos_t_k = sqrt_(max_(F(1.0f) - sin2_t_k, 0.0f));
        F eta_k = n1k / n2k;
        V3 refr_k = normalize(eta_k * k + fma_(eta_k, cos_i, -cos_t_k) * normal);
        V3 final_k = biaxial_entry ? mode_poynting_dir(channel_indicatrix(P, c), refr_k, use_e)
                     : (entering && use_e)
                         ? extraordinary_poynting_dir(refr_k, P.c_axis, P.n_ch[c],
                                                      P.n_ch[c] + F(P.sc->material.birefringence_delta))
                         : refr_k;
        bool matches = dot(final_k, final_refr) >= DIRECTION_MATCH_COS_TOL;
        // Transmission at this channel's own index, projected onto the selected
        // eigenmode at an anisotropic entry (reflect_refract.rs:362, exit_split.rs:69).
        F two_n1_cos = F(2.0f) * n1k * cos_i;
        F t_s = two_n1_cos / fma_(n2k, cos_t_k, n1k * cos_i);
        F t_p = two_n1_cos / fma_(n1k, cos_t_k, n2k * cos_i);
        M4 tm = fresnel_transmission(n1k, n2k, cos_i, cos_t_k, t_s, t_p);
        Stokes incident = original;
        if (entering && has_az) incident = Stokes{original.i, original.i * az_c, original.i * az_s, 0.0f};
        Stokes transmitted = scale(apply(tm, incident), F(1.0f) / (F(1.0f) - r_unpol));
        F r_s, r_p;
        fresnel_rs_rp(n1k, n2k, cos_i, cos_t_k, &r_s, &r_p);
        F r_unpol_k = clamp_(r_unpol_of(r_s, r_p), R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
        if (matches) {
            P.stokes[c] = transmitted;
            P.path_pdf[c] = P.path_pdf[c] * (F(1.0f) - r_unpol_k);
        } else {
            // apply_channel_chromatic_termination (reflect_refract.rs:444).
            F prefix = P.path_pdf[c];
            P.stokes[c] = scale(P.stokes[c], 0.0f);
            P.path_pdf[c] = prefix * (F(1.0f) - r_unpol_k);
            bool is_exit = P.inside && !entering;
            if (is_exit && intensity(original) > F(0.0f))
                try_split_exit_channel(P, hit_point, c, refr_k, intensity(transmitted));
        }
        dirs[c] = final_k;
        have_dir[c] = true;
        hero_match[c] = matches;
    }
    if (!P.inside) narrow_compat(P, dirs, have_dir, hero_match);
    o->new_k = refr;
    o->new_s = final_refr;
    o->new_inside = !P.inside;
    o->update = entering ? (use_e ? 1 : 0) : -1;
}

// apply_partial_fresnel_bounce's scalar-Fresnel path (refraction/dispatch.rs:162-380):
// mode selection at an anisotropic entry, the reflect/transmit draw, then the branch.
static void apply_scalar_fresnel(Path& P, const Geo& g, V3 k, V3 normal, V3 cpn, V3 hit_point,
                                 uint32_t bounce, Outcome* o) {
    const bool entering = !P.inside && P.aniso;
    // resolve_entry_mode_selection (dispatch.rs:162).
    F p_o = 0.5f, cos2 = 0.0f, sin2 = 0.0f;
    // A biaxial material has no ordinary eigenmode to weigh: 50 / 50 (dispatch.rs:176).
    bool has_sel = entering && !g.is_biaxial &&
                   entry_eigenmode_selection(P.c_axis, cpn, k, P.stokes[0], &p_o, &cos2, &sin2);
    if (!has_sel) p_o = 0.5f;
    F msr = unit_draw(P.seed, bounce, BIREFRINGENT_SPLIT_STREAM);
    bool use_e = entering ? (msr < F(1.0f) - p_o) : P.is_e;
    F az_c = use_e ? -cos2 : cos2;
    F az_s = use_e ? -sin2 : sin2;
    // compute_entry_reflect_probability (dispatch.rs:230).
    bool ord_sel = entering && !g.is_biaxial && !use_e;
    F n2 = ord_sel ? g.n_o_hero : g.n2;
    F sin2_t = g.sin2_t;
    if (ord_sel) {
        F eta = g.n1 / n2;
        sin2_t = eta * eta * fma_(g.cos_i, -g.cos_i, 1.0f);
    }
    F cos_t = sqrt_(max_(F(1.0f) - sin2_t, 0.0f));
    F r_s, r_p;
    fresnel_rs_rp(g.n1, n2, g.cos_i, cos_t, &r_s, &r_p);
    F r_unpol = clamp_(r_unpol_of(r_s, r_p), R_UNPOL_SELECT_MIN, R_UNPOL_SELECT_MAX);
    F rng = unit_draw(P.seed, bounce, FRESNEL_BRANCH_STREAM);
    if (rng < r_unpol) {
        apply_partial_reflect(P, g, r_unpol);
        o->new_k = reflect(k, normal);
        o->new_s = poynting_dir_for_mode(P, g, o->new_k, P.inside, P.is_e);
        o->new_inside = P.inside;
    } else {
        apply_refract_bounce(P, g, r_unpol, k, normal, hit_point, use_e, has_sel, az_c, az_s, o);
    }
}

// apply_uniaxial_entry_bounce (refraction/uniaxial_entry.rs:108-412).
static void apply_uniaxial_entry(Path& P, const Geo& g, V3 k, V3 normal, uint32_t bounce, Outcome* o) {
    const UFrame& f = g.frame;
    const V3 c_axis = P.c_axis;
    const F delta_n = F(P.sc->material.birefringence_delta);
    EntryInc inc = entry_incidence_frame(1.0f, f);
    EntrySol sh = entry_solve(inc, 1.0f, P.n_ch[0], P.n_e_at[0], c_axis, f);
    M4 mh = jones_to_mueller(sh.r_s[0], sh.r_s[1], sh.r_p[0], sh.r_p[1]);
    F r_branch = clamp_(mh.c[0], R_UNPOL_SELECT_MIN, R_UNPOL_SELECT_MAX);
    F inc_flux = F(0.5f) * f.cos_i;
    F p_o_raw = mode_power(sh.t_o[0], sh.t_o[1], sh.flux_o, inc_flux, P.stokes[0]);
    F p_e_raw = mode_power(sh.t_e[0], sh.t_e[1], sh.flux_e, inc_flux, P.stokes[0]);
    F p_o_hero = clamp_(p_o_raw / max_(p_o_raw + p_e_raw, 1e-12f), R_UNPOL_SELECT_MIN, R_UNPOL_SELECT_MAX);
    F msr = unit_draw(P.seed, bounce, BIREFRINGENT_SPLIT_STREAM);
    bool use_e = msr < F(1.0f) - p_o_hero;
    F p_frac = use_e ? F(1.0f) - p_o_hero : p_o_hero;
    F n2_hero_dir = use_e ? g.n2 : g.n_o_hero;
    V3 refr = snell_dir(g.n1 / n2_hero_dir, g.cos_i, k, normal);
    V3 final_refr = use_e ? extraordinary_poynting_dir(refr, c_axis, g.n_o_hero, g.n_e_hero) : refr;
    V3 p_axis_t = cross(refr, f.s_axis);
    F rng = unit_draw(P.seed, bounce, FRESNEL_BRANCH_STREAM);
    if (rng < r_branch) {
        for (int c = 0; c < 8; ++c) {
            EntrySol s = entry_solve(inc, 1.0f, P.n_ch[c], P.n_e_at[c], c_axis, f);
            M4 mk = jones_to_mueller(s.r_s[0], s.r_s[1], s.r_p[0], s.r_p[1]);
            F r_unpol_k = clamp_(mk.c[0], R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
            P.stokes[c] = scale(apply(mk, P.stokes[c]), F(1.0f) / r_branch);
            P.path_pdf[c] = P.path_pdf[c] * r_unpol_k;
        }
        o->new_k = o->new_s = reflect(k, normal);
        o->new_inside = false;
        return;
    }
    V3 dirs[8];
    bool have_dir[8];
    bool hero_match[8];
    for (int c = 0; c < 8; ++c) {
        F n_o_k = P.n_ch[c];
        F n2k_dir = use_e ? g.n2_ch[c] : n_o_k;
        F ratio = g.n1 / n2k_dir;
        F sin2_t_k = (ratio * ratio) * fma_(g.cos_i, -g.cos_i, 1.0f);
        if (sin2_t_k > F(1.0f)) {
            P.stokes[c] = scale(P.stokes[c], 0.0f);
            P.path_pdf[c] = 0.0f;
            have_dir[c] = false;
            hero_match[c] = false;
            continue;
        }
        F cos_t_k = sqrt_(max_(F(1.0f) - sin2_t_k, 0.0f));
        F eta_k = g.n1 / n2k_dir;
        V3 refr_k = normalize(eta_k * k + fma_(eta_k, g.cos_i, -cos_t_k) * normal);
        V3 final_k = use_e ? extraordinary_poynting_dir(refr_k, c_axis, n_o_k, n_o_k + delta_n) : refr_k;
        dirs[c] = final_k;
        have_dir[c] = true;
        bool matches = dot(final_k, final_refr) >= DIRECTION_MATCH_COS_TOL;
        hero_match[c] = matches;
        EntrySol s = entry_solve(inc, 1.0f, n_o_k, P.n_e_at[c], c_axis, f);
        M4 mk = jones_to_mueller(s.r_s[0], s.r_s[1], s.r_p[0], s.r_p[1]);
        F t_unpol_k = clamp_(F(1.0f) - mk.c[0], R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
        if (!matches) {
            P.stokes[c] = scale(P.stokes[c], 0.0f);
            P.path_pdf[c] = P.path_pdf[c] * t_unpol_k;
            continue;
        }
        Cx t_s_row = use_e ? s.t_e[0] : s.t_o[0];
        Cx t_p_row = use_e ? s.t_e[1] : s.t_o[1];
        F flux_k = use_e ? s.flux_e : s.flux_o;
        V3 mode_dir = use_e ? s.e_hat : s.o_hat;
        F deposit = mode_power(t_s_row, t_p_row, flux_k, inc_flux, P.stokes[c]) / p_frac;
        F c2, s2;
        azimuth2_in_frame(mode_dir, f.s_axis, p_axis_t, &c2, &s2);
        P.stokes[c] = scale(Stokes{deposit, deposit * c2, deposit * s2, 0.0f}, F(1.0f) / (F(1.0f) - r_branch));
        P.path_pdf[c] = P.path_pdf[c] * t_unpol_k;
    }
    narrow_compat(P, dirs, have_dir, hero_match);
    o->new_k = refr;
    o->new_s = final_refr;
    o->new_inside = true;
    o->update = use_e ? 1 : 0;
}

// compute_uniaxial_exit_transmission (refraction/uniaxial_internal.rs:212).
static Stokes uniaxial_exit_transmission(const IntSol& sol, F r_branch, F incident_i, F* i_unit_out) {
    F flux_inc = max_(sol.flux_inc, 1e-12f);
    Cx ts_n = cscale(sol.t_s, sqrt_(sol.flux_ts / flux_inc));
    Cx tp_n = cscale(sol.t_p, sqrt_(sol.flux_tp / flux_inc));
    F i_unit = cnorm2(ts_n) + cnorm2(tp_n);
    F q_unit = cnorm2(ts_n) - cnorm2(tp_n);
    Cx cr = cmul(ts_n, cconj(tp_n));
    F u_unit = F(2.0f) * cr.re;
    F v_unit = F(-2.0f) * cr.im;
    *i_unit_out = i_unit;
    return scale(Stokes{incident_i * i_unit, incident_i * q_unit, incident_i * u_unit, incident_i * v_unit},
                 F(1.0f) / (F(1.0f) - r_branch));
}

// apply_uniaxial_internal_bounce (refraction/uniaxial_internal.rs:68-353).
static void apply_uniaxial_internal(Path& P, const Geo& g, V3 k, V3 normal, V3 hit_point, uint32_t bounce,
                                    Outcome* o) {
    const UFrame& f = g.frame;
    const bool inc_o = !P.is_e;
    IntSol sh = internal_solve(g.n1_ch[0], P.n_ch[0], P.n_e_at[0], P.c_axis, f, inc_o);
    F flux_inc_hero = max_(sh.flux_inc, 1e-12f);
    F ro_pow = cnorm2(sh.r_o) * sh.flux_ro;
    F re_pow = cnorm2(sh.r_e) * sh.flux_re;
    F r_branch = clamp_((ro_pow + re_pow) / flux_inc_hero, R_UNPOL_SELECT_MIN, R_UNPOL_SELECT_MAX);
    F p_o_exact = ro_pow / max_(ro_pow + re_pow, 1e-12f);
    F rng = unit_draw(P.seed, bounce, FRESNEL_BRANCH_STREAM);
    if (rng < r_branch) {
        for (int c = 0; c < 8; ++c) {
            IntSol sol = (c == 0) ? sh : internal_solve(g.n1_ch[c], P.n_ch[c], P.n_e_at[c], P.c_axis, f, inc_o);
            F flux_inc = max_(sol.flux_inc, 1e-12f);
            F r_total_k = min_(fma_(cnorm2(sol.r_e), sol.flux_re, cnorm2(sol.r_o) * sol.flux_ro) / flux_inc, 1.0f);
            P.stokes[c] = scale(P.stokes[c], r_total_k / r_branch);
            P.path_pdf[c] = P.path_pdf[c] * clamp_(r_total_k, R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
        }
        o->new_k = o->new_s = reflect(k, normal);
        o->new_inside = true;
        o->has_p_o = true;
        o->p_o = p_o_exact;
        return;
    }
    V3 hero_refr = snell_dir(g.n1 / g.n2, g.cos_i, k, normal);
    for (int c = 0; c < 8; ++c) {
        F original_i = P.stokes[c].i;
        F n_inc_k = g.n1_ch[c];
        F n2k = g.n2_ch[c];
        F ratio = n_inc_k / n2k;
        F sin2_t_k = (ratio * ratio) * fma_(g.cos_i, -g.cos_i, 1.0f);
        if (sin2_t_k > F(1.0f)) {
            P.stokes[c] = scale(P.stokes[c], 0.0f);
            P.path_pdf[c] = 0.0f;
            continue;
        }
        F cos_t_k = sqrt_(max_(F(1.0f) - sin2_t_k, 0.0f));
        F eta_k = n_inc_k / n2k;
        V3 refr_k = normalize(eta_k * k + fma_(eta_k, g.cos_i, -cos_t_k) * normal);
        bool matches = dot(refr_k, hero_refr) >= DIRECTION_MATCH_COS_TOL;
        IntSol sol = (c == 0) ? sh : internal_solve(n_inc_k, P.n_ch[c], P.n_e_at[c], P.c_axis, f, inc_o);
        F i_unit;
        Stokes transmitted = uniaxial_exit_transmission(sol, r_branch, original_i, &i_unit);
        F t_unpol_k = clamp_(i_unit, R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
        if (!matches) {
            F prefix = P.path_pdf[c];
            P.stokes[c] = scale(P.stokes[c], 0.0f);
            P.path_pdf[c] = prefix * t_unpol_k;
            if (original_i > F(0.0f))
                try_split_exit_channel(P, hit_point, c, refr_k, intensity(transmitted));
            continue;
        }
        P.stokes[c] = transmitted;
        P.path_pdf[c] = P.path_pdf[c] * t_unpol_k;
    }
    o->new_k = o->new_s = hero_refr;
    o->new_inside = false;
}

// apply_absorption (raytracer/absorption.rs:99-197): the mean over the two eigenmodes
// for an isotropic material, the assigned eigenmode's field for a uniaxial one.
// Frosted facets (optics/raytracer/scattering/frosted.rs, scattering/mod.rs:110), with
// next-event estimation toward the sun under DaylightSun, the one modelled environment
// that enables it (environment_supports_nee, environment/nee.rs:60; HDR maps are not
// modelled).
static const uint32_t FROSTED_DIR_U_STREAM = 0x27D4EB2Fu;  // sampling.rs:24
static const uint32_t FROSTED_DIR_V_STREAM = 0x165667B1u;  // sampling.rs:25

// frosted_orthonormal_basis (scattering/mod.rs:110).
static void frosted_orthonormal_basis(V3 n, V3* t, V3* b) {
    const V3 a = abs_(n.x) > F(0.9f) ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    *t = normalize_or_zero(a - n * dot(n, a));
    *b = cross(n, *t);
}
// shading_normal_for_hit (transport/inner.rs:54): a carved stone rounds a plane facet's
// edges only away from the tools (four probes a rounding radius out along the facet's
// frosted basis); a tool facet keeps its own normal.
static V3 shading_normal_for_hit(const ix_scene* sc, V3 hit_point, int facet, V3 hit_normal, F radius) {
    const bool carved = sc->n_tools > 0 && sc->tools;
    if (!carved || radius <= F(0.0f))
        return shading_normal_near_edge(sc->planes, sc->n_planes, hit_point, facet, hit_normal, radius);
    if ((uint32_t)facet >= sc->n_planes) return hit_normal;
    V3 u, v;
    frosted_orthonormal_basis(hit_normal, &u, &v);
    const V3 dirs[4] = {u, -u, v, -v};
    for (const V3& dir : dirs) {
        const V3 probe = hit_point + dir * radius;
        for (uint32_t k = 0; k < sc->n_tools; ++k)
            if (tool_contains(sc->tools[k], probe)) return hit_normal;
    }
    return shading_normal_near_edge(sc->planes, sc->n_planes, hit_point, facet, hit_normal, radius);
}
// cosine_weighted_hemisphere (frosted.rs:34): (2 pi) u2 as the angle, glam's left-to-right
// sum of the three scaled basis vectors.
static V3 cosine_weighted_hemisphere(F u1, F u2, V3 n) {
    const F r = sqrt_(u1);
    const F theta = F(2.0f * 3.14159265358979323846f) * u2;
    const F sin_t = sin_(theta), cos_t = cos_(theta);
    V3 t, b;
    frosted_orthonormal_basis(n, &t, &b);
    return normalize_or_zero((t * (r * cos_t) + b * (r * sin_t)) + n * sqrt_(max_(F(1.0f) - u1, 0.0f)));
}
// apply_frosted_bounce (frosted.rs:289) with NEE off: a cosine-weighted diffuse
// reflection or transmission chosen by the hero's unpolarised Fresnel reflectance
// (always reflection past the hero's critical angle); every channel is depolarised and
// its path pdf takes the chosen branch's probability.  An anisotropic entry draws its
// eigenmode with probability one half.
// sun_cone_direction (environment/sun.rs:70): a direction uniform in the sun's cone.
static V3 sun_cone_direction(V3 key, F u0, F u1) {
    const F one_minus_cos = u0 * F(SUN_ONE_MINUS_COS);
    const F cos_t = F(1.0f) - one_minus_cos;
    const F sin_t = sqrt_(max_(one_minus_cos * (F(2.0f) - one_minus_cos), 0.0f));
    const F phi = F(2.0f * 3.14159265358979323846f) * u1;
    const F sin_p = sin_(phi), cos_p = cos_(phi);
    const V3 a = abs_(key.x) > F(0.9f) ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    const V3 t = normalize_or_zero(a - key * dot(key, a));
    const V3 b = cross(key, t);
    return normalize_or_zero((t * (sin_t * cos_p) + b * (sin_t * sin_p)) + key * cos_t);
}
// balance_heuristic (scattering/mod.rs:102).
static F balance_heuristic(F a, F b) {
    const F denom = a + b;
    return denom > F(1e-12f) ? a / denom : F(0.0f);
}
// environment_nee_pdf (environment/nee.rs:144) for DaylightSun: uniform over the disc.
static F sun_nee_pdf(const ix_environment& env, V3 dir) {
    return dot(dir, load3(env.key_dir)) >= F(SUN_DISC_COS) ? F(1.0f) / F(SUN_SOLID_ANGLE) : F(0.0f);
}
// nee_contribution_frosted_exterior (scattering/frosted.rs:98) for the DaylightSun sky:
// one sun-cone light sample, a shadow probe on a carved stone, the balance heuristic
// against the Lambertian cos / pi density, deposited into every channel's radiance.
static void frosted_sun_nee(Path& P, V3 origin, V3 ext_normal, uint32_t bounce) {
    const ix_environment& env = P.sc->environment;
    const F u0 = unit_draw(P.seed, bounce, FROSTED_NEE_ENV_DIR_U_STREAM);
    const F u1 = unit_draw(P.seed, bounce, FROSTED_NEE_ENV_DIR_V_STREAM);
    const V3 dir = sun_cone_direction(load3(env.key_dir), u0, u1);
    const F pdf = F(1.0f) / F(SUN_SOLID_ANGLE);
    const F cos_light = dot(dir, ext_normal);
    if (cos_light <= F(0.0f)) return;
    if (P.sc->n_tools && P.sc->tools) {
        Hit h;
        bool carved, entering;
        if (intersect_scene(P.sc, Ray{origin + dir * F(1e-4f), dir}, &h, &carved, &entering)) return;
    }
    const F brdf_pdf = cos_light / F(3.14159265358979323846f);
    const F mis = balance_heuristic(pdf, brdf_pdf);
    if (mis <= F(0.0f)) return;
    const F common = (brdf_pdf * mis) / pdf;
    for (int c = 0; c < 8; ++c) {
        // EnvNeeSample::radiance (environment/nee.rs:47): geometry x (spd x exposure).
        const F env_k = F(env.sun_factor) * (spectral_power(env, P.lambdas[c]) * F(env.exposure));
        P.radiance[c] = ((intensity(P.stokes[c]) * common) * env_k) + P.radiance[c];
    }
}
static void apply_frosted_bounce(Path& P, const Geo& g, V3 normal, V3 hit_point, uint32_t bounce, Outcome* o) {
    // NEE is on under DaylightSun (environment_supports_nee, nee.rs:60); the reflect of an
    // outside hit and the transmit of an inside one are the exterior-side events.
    const bool nee = P.sc->environment.model == IX_ENV_DAYLIGHT_SUN;
    const F u1 = unit_draw(P.seed, bounce, FROSTED_DIR_U_STREAM);
    const F u2 = unit_draw(P.seed, bounce, FROSTED_DIR_V_STREAM);
    o->update = -1;
    o->has_p_o = false;
    o->p_o = 0.0f;
    if (g.sin2_t > F(1.0f)) {
        const V3 d = cosine_weighted_hemisphere(u1, u2, normal);
        for (int c = 0; c < 8; ++c) P.stokes[c] = unpolarized(intensity(P.stokes[c]));
        o->new_k = o->new_s = d;
        o->new_inside = P.inside;
        return;
    }
    const F cos_t = sqrt_(max_(F(1.0f) - g.sin2_t, 0.0f));
    const F r_s = fma_(g.n2, -cos_t, g.n1 * g.cos_i) / fma_(g.n2, cos_t, g.n1 * g.cos_i);
    const F r_p = fma_(g.n1, -cos_t, g.n2 * g.cos_i) / fma_(g.n1, cos_t, g.n2 * g.cos_i);
    const F r_unpol = clamp_(F(0.5f) * fma_(r_p, r_p, r_s * r_s), 1e-4f, 1.0f - 1e-4f);
    const F rng_bounce = unit_draw(P.seed, bounce, FRESNEL_BRANCH_STREAM);
    if (rng_bounce < r_unpol) {
        const V3 d = cosine_weighted_hemisphere(u1, u2, normal);
        for (int c = 0; c < 8; ++c) {
            P.stokes[c] = unpolarized(intensity(P.stokes[c]));
            P.path_pdf[c] = P.path_pdf[c] * r_unpol;
        }
        if (nee && !P.inside) {
            frosted_sun_nee(P, hit_point, normal, bounce);
            P.has_carry = true;
            P.carry_pdf = dot(d, normal) / F(3.14159265358979323846f);
        }
        o->new_k = o->new_s = d;
        o->new_inside = P.inside;
        return;
    }
    const V3 d = cosine_weighted_hemisphere(u1, u2, -normal);
    const bool entering_anisotropic = !P.inside && P.aniso;
    if (entering_anisotropic) o->update = unit_draw(P.seed, bounce, BIREFRINGENT_SPLIT_STREAM) < F(0.5f) ? 1 : 0;
    const F t_unpol = F(1.0f) - r_unpol;
    for (int c = 0; c < 8; ++c) {
        P.stokes[c] = unpolarized(intensity(P.stokes[c]));
        P.path_pdf[c] = P.path_pdf[c] * t_unpol;
    }
    if (nee && P.inside) {
        frosted_sun_nee(P, hit_point, -normal, bounce);
        P.has_carry = true;
        P.carry_pdf = dot(d, -normal) / F(3.14159265358979323846f);
    }
    o->new_k = o->new_s = d;
    o->new_inside = !P.inside;
}

// channel_absorption_alphas_assigned (raytracer/absorption.rs): each channel's alpha
// along the current wave normal, for the assigned mode of a uniaxial material.
static void channel_alphas(const Path& P, F alpha[8]) {
    TensorFrame tf = tensor_frame(P.c_axis);
    if (P.biaxial) {
        // The hero indicatrix's assigned-mode field against each channel's biaxial
        // tensor (absorption.rs:227-242, wavelength_cache.rs:44-52).
        V3 e_mode = assigned_mode_e_field_biaxial(channel_indicatrix(P, 0), P.k, P.is_e);
        for (int c = 0; c < 8; ++c)
            alpha[c] = quadratic_form3(tf, P.alpha_ch_o[c], P.alpha_ch_b[c], P.alpha_ch_e[c], e_mode);
        return;
    }
    if (!P.aniso) {
        V3 ea = ordinary_eigen_polarization(P.k, P.c_axis);
        V3 eb = normalize_or_zero(cross(P.k, ea));
        for (int c = 0; c < 8; ++c)
            alpha[c] = midpoint_(quadratic_form(tf, P.alpha_ch_o[c], P.alpha_ch_e[c], ea),
                                 quadratic_form(tf, P.alpha_ch_o[c], P.alpha_ch_e[c], eb));
    } else {
        V3 e_mode = assigned_mode_e_field_uniaxial(P.k, P.c_axis, P.is_e, P.n_ch[0], P.n_e_at[0]);
        for (int c = 0; c < 8; ++c) alpha[c] = quadratic_form(tf, P.alpha_ch_o[c], P.alpha_ch_e[c], e_mode);
    }
}
#if defined(IX_ORACLE_AVX2) && !defined(IX_COUNT_FLOPS)
// exp_f32x8 (simd/exp_poly.rs:122), the AVX2 level: exp_lane's steps on 8 lanes at once
// (the clamp with _mm256_min/max_ps's second-operand rule, floor of x log2e + 1/2, the
// two-constant reduction and the polynomial with fused multiply-adds, 2^n from the
// exponent bits) -- bit-identical to exp_lane per lane.
static void exp8(const float in[8], float out[8]) {
    uint32_t c1bits = 0x3F318000u;
    float c1f;
    std::memcpy(&c1f, &c1bits, 4);
    __m256 x = _mm256_loadu_ps(in);
    x = _mm256_min_ps(x, _mm256_set1_ps(88.02875f));
    x = _mm256_max_ps(x, _mm256_set1_ps(-87.33654f));
    const __m256 n = _mm256_floor_ps(_mm256_fmadd_ps(x, _mm256_set1_ps(1.44269504088896340736f), _mm256_set1_ps(0.5f)));
    x = _mm256_fmadd_ps(n, _mm256_set1_ps(-c1f), x);
    x = _mm256_fmadd_ps(n, _mm256_set1_ps(2.1219444e-4f), x);
    const __m256 z = _mm256_mul_ps(x, x);
    __m256 p = _mm256_set1_ps(1.9875691e-4f);
    p = _mm256_fmadd_ps(p, x, _mm256_set1_ps(1.3981999e-3f));
    p = _mm256_fmadd_ps(p, x, _mm256_set1_ps(8.333452e-3f));
    p = _mm256_fmadd_ps(p, x, _mm256_set1_ps(4.1665796e-2f));
    p = _mm256_fmadd_ps(p, x, _mm256_set1_ps(1.6666665e-1f));
    p = _mm256_fmadd_ps(p, x, _mm256_set1_ps(5.0000003e-1f));
    p = _mm256_add_ps(_mm256_fmadd_ps(p, z, x), _mm256_set1_ps(1.0f));
    const __m256i e = _mm256_slli_epi32(_mm256_add_epi32(_mm256_cvttps_epi32(n), _mm256_set1_epi32(127)), 23);
    _mm256_storeu_ps(out, _mm256_mul_ps(p, _mm256_castsi256_ps(e)));
}
#endif
static void apply_absorption(Path& P, F path_len) {
    const ix_material& m = P.sc->material;
    F alpha[8];
    channel_alphas(P, alpha);
    F scaled_len = path_len * F(m.absorption_path_scale);
#if defined(IX_ORACLE_AVX2) && !defined(IX_COUNT_FLOPS)
    float arg[8], e[8];
    for (int c = 0; c < 8; ++c) arg[c] = -alpha[c] * scaled_len;
    exp8(arg, e);
    for (int c = 0; c < 8; ++c) P.stokes[c] = scale(P.stokes[c], e[c]);
#else
    for (int c = 0; c < 8; ++c) P.stokes[c] = scale(P.stokes[c], exp_lane(-alpha[c] * scaled_len));
#endif
}

enum { TERM_ESCAPED = 0, TERM_RR = 1, TERM_CAP = 2, TERM_SCATTER_ABSORBED = 3 };

// apply_russian_roulette (transport/bounce.rs:355): false when the path is killed.
static bool russian_roulette(Path& P, uint32_t bounce) {
    F max_i = 0.0f;
    for (int c = 0; c < 8; ++c) max_i = max_(max_i, intensity(P.stokes[c]));
    F q = clamp_(max_i, 0.05f, 1.0f);
    F rr = unit_draw(P.seed, bounce, RUSSIAN_ROULETTE_STREAM);
    if (rr > q) return false;
    for (int c = 0; c < 8; ++c) P.stokes[c] = scale(P.stokes[c], F(1.0f) / q);
    for (int c = 0; c < 8; ++c) P.split[c] = P.split[c] / q;
    return true;
}

// Henyey-Greenstein interior scattering (optics/raytracer/scattering/hg.rs).
static const uint32_t DISTANCE_SAMPLE_STREAM = 0xA24BAED4u;  // sampling.rs:28
static const uint32_t PHASE_DIR_U_STREAM = 0x9FB21C65u;      // sampling.rs:31
static const uint32_t PHASE_DIR_V_STREAM = 0x1CE4E5B9u;      // sampling.rs:32
// sample_henyey_greenstein_direction (hg.rs:390).
static V3 sample_hg_direction(F u1, F u2, F g, V3 forward) {
    F cos_theta;
    if (abs_(g) < F(1e-3f)) {
        cos_theta = fma_(2.0f, -u1, 1.0f);
    } else {
        F one_minus_g2 = fma_(g, -g, 1.0f);
        F denom = fma_(F(2.0f) * g, u1, F(1.0f) - g);
        F sq = one_minus_g2 / denom;
        cos_theta = fma_(sq, -sq, fma_(g, g, 1.0f)) / (F(2.0f) * g);
    }
    cos_theta = clamp_(cos_theta, -1.0f, 1.0f);
    F sin_theta = sqrt_(max_(fma_(cos_theta, -cos_theta, 1.0f), 0.0f));
    F phi = F(2.0f * 3.14159265358979323846f) * u2;
    F sin_p = sin_(phi), cos_p = cos_(phi);
    V3 t, b;
    frosted_orthonormal_basis(forward, &t, &b);
    return normalize_or_zero((t * (sin_theta * cos_p) + b * (sin_theta * sin_p)) + forward * cos_theta);
}
enum { SCATTER_NONE = 0, SCATTER_SURVIVED = 1, SCATTER_KILLED = 2 };
// try_scatter_step (hg.rs:256-340) with maybe_scatter_or_extinguish (hg.rs:21-84), without
// next-event estimation (no light-sampling technique in the modelled environments) and
// without zoning: a free flight drawn with the hero's extinction either scatters inside
// the segment -- each channel reweighted by its transmittance, depolarised, the HG lobe
// about the old direction, roulette after bounce 4 -- or reaches the facet with every
// channel's survival relative to the hero's.
static int scatter_step(Path& P, F hit_t, uint32_t bounce) {
    const ix_material& m = P.sc->material;
    F alpha[8];
    if (P.absorbing) {
        channel_alphas(P, alpha);
    } else {
        for (int c = 0; c < 8; ++c) alpha[c] = 0.0f;
    }
    const F path_scale = m.absorption_path_scale;
    const F sigma_s = F(m.scattering_sigma_s) / path_scale;
    const F sigma_t_hero = alpha[0] + sigma_s;
    const F dist_rand = unit_draw(P.seed, bounce, DISTANCE_SAMPLE_STREAM);
    const F one_minus_u = max_(F(1.0f) - dist_rand, 1e-7f);
    const F t_free = -ln_(one_minus_u) / sigma_t_hero;
    const F hit_scaled = hit_t * path_scale;
    if (t_free < hit_scaled) {
        const F pdf_hero = sigma_t_hero * one_minus_u;
        for (int c = 0; c < 8; ++c) {
            const F sigma_t = alpha[c] + sigma_s;
            const F tr = exp_lane(-(alpha[c] + sigma_s) * t_free);
            const F weight = tr * sigma_s / pdf_hero;
            P.stokes[c] = unpolarized(intensity(P.stokes[c]) * weight);
            P.path_pdf[c] = P.path_pdf[c] * (sigma_t * tr);
        }
        const F u1 = unit_draw(P.seed, bounce, PHASE_DIR_U_STREAM);
        const F u2 = unit_draw(P.seed, bounce, PHASE_DIR_V_STREAM);
        const V3 old_dir = P.ray.dir;
        const V3 new_dir = sample_hg_direction(u1, u2, F(m.scattering_g), old_dir);
        const F t_model = t_free / path_scale;
        P.ray = Ray{P.ray.origin + t_model * old_dir, new_dir};
        P.k = new_dir;
        P.has_prev = false;  // depolarised: no plane of incidence to rotate from
        if (bounce > 4 && !russian_roulette(P, bounce)) return SCATTER_KILLED;
        return SCATTER_SURVIVED;
    }
    F survive[8];
    for (int c = 0; c < 8; ++c) survive[c] = exp_lane(-(alpha[c] + sigma_s) * hit_scaled);
    const F survive_hero = survive[0];
    for (int c = 0; c < 8; ++c) {
        P.stokes[c] = scale(P.stokes[c], survive[c] / max_(survive_hero, 1e-30f));
        P.path_pdf[c] = P.path_pdf[c] * survive[c];
    }
    return SCATTER_NONE;
}

// PathEvents::facet (transport/path_events.rs:55-79): the first facet event, the first
// inside-to-outside transition, internal events before it and a re-entry after it.
static void record_facet(ixo_path_events* ev, uint32_t bounce, const Hit& hit, bool inside_before,
                         bool inside_after, V3 dir_after) {
    if (ev->first_facet < 0) {
        ev->first_facet = hit.facet;
        ev->first_entered = inside_after ? 1u : 0u;
    }
    const bool exited = ev->exit_facet >= 0;
    if (inside_before && !inside_after && !exited) {
        ev->exit_facet = hit.facet;
        store3(ev->exit_normal, hit.normal);
        store3(ev->exit_dir, dir_after);
        ev->exit_bounce = bounce;
    } else if (inside_before && inside_after && !exited) {
        ev->bounces_before_exit += 1;
    } else if (!inside_before && inside_after && exited) {
        ev->reentered = 1;
    }
}

static V3 trace_path(const ix_scene* sc, Ray initial, uint32_t seed, F hero_rand,
                     ixo_path_info* info, ixo_path_events* ev = nullptr) {
    if (ev) {
        std::memset(ev, 0, sizeof(*ev));
        ev->first_facet = -1;
        ev->exit_facet = -1;
    }
    Path P;
    P.sc = sc;
    P.seed = seed;
    P.splits = 0;
    hero_wavelengths(hero_rand, P.lambdas);
    const ix_material& m = sc->material;
    P.absorbing = absorption_present(m.abs_o) || absorption_present(m.abs_e);
    P.aniso = m.anisotropic != 0;
    P.biaxial = m.biaxial != 0;
    if (P.biaxial && m.has_abs_beta) P.absorbing = P.absorbing || absorption_present(m.abs_beta);
    P.is_e = false;
    P.c_axis = load3(m.c_axis);
    P.ax = tensor_frame(P.c_axis);
    for (int c = 0; c < 8; ++c) {
        P.n_ch[c] = dispersion_eval(m.dispersion, P.lambdas[c]);
        P.n_e_at[c] = P.aniso ? extraordinary_index_at(m, P.lambdas[c], P.n_ch[c]) : P.n_ch[c];
        P.alpha_ch_o[c] = P.absorbing ? spectral_absorption(m.abs_o, P.lambdas[c]) : F(0.0f);
        P.alpha_ch_e[c] = P.absorbing ? spectral_absorption(m.abs_e, P.lambdas[c]) : F(0.0f);
        P.alpha_ch_b[c] = (P.absorbing && P.biaxial && m.has_abs_beta) ? spectral_absorption(m.abs_beta, P.lambdas[c])
                                                                       : P.alpha_ch_o[c];
        P.stokes[c] = unpolarized(1.0f);
        P.radiance[c] = 0.0f;
        P.path_pdf[c] = 1.0f;
        P.split[c] = 0.0f;
        P.compat[c] = 0xFF;
    }
    P.ray = initial;
    P.k = initial.dir;
    P.has_carry = false;
    P.carry_pdf = 0.0f;
    P.inside = false;
    P.has_prev = false;
    P.escaped = false;
    P.observer = -initial.dir;
    F glare = clamp_(sc->environment.surface_glare, 0.0f, 1.0f);
    uint32_t term = TERM_CAP;
    uint32_t bounce = 0;
    uint32_t iterations = 0;
    for (bounce = 0; bounce < sc->max_bounces; ++bounce) {
        iterations = bounce + 1;
        Hit hit;
        bool carved = false, entering = false;
        // pending_light_mis.take() (bounce_body.rs:372): only this iteration's escape reads it.
        const bool had_carry = P.has_carry;
        const F carry_pdf = P.carry_pdf;
        P.has_carry = false;
        if (!intersect_scene(sc, P.ray, &hit, &carved, &entering)) {
            // handle_miss (bounce_body/miss.rs:33) + accumulate_miss_radiance (bounce.rs:40).
            const F mis = had_carry ? balance_heuristic(carry_pdf, sun_nee_pdf(sc->environment, P.ray.dir)) : F(1.0f);
            F env[8];
            environment_channels(sc->environment, P.ray.dir, P.lambdas, P.observer, env);
            for (int c = 0; c < 8; ++c)
                P.radiance[c] = fma_(intensity(P.stokes[c]) * mis, env[c], P.radiance[c]);
            P.escaped = true;
            term = TERM_ESCAPED;
            if (ev) {  // PathEvents::miss (path_events.rs:88)
                ev->has_escaped_dir = 1;
                store3(ev->escaped_dir, P.ray.dir);
            }
            break;
        }
        // A carved stone's hit tells which medium the ray is in (bounce_body.rs:391-397):
        // the restart may have stepped over a second boundary within 1e-4.
        if (carved) P.inside = !entering;
        // The interior segment may end in a scattering event first (bounce_body.rs:408-417).
        if (P.inside && m.scattering_sigma_s > 0.0f) {
            const int sc_out = scatter_step(P, hit.t, bounce);
            if (ev && sc_out != SCATTER_NONE) ev->scattered = 1;  // PathEvents::scatter (path_events.rs:96)
            if (sc_out == SCATTER_KILLED) {
                term = TERM_SCATTER_ABSORBED;  // bounce_body.rs:527
                break;
            }
            if (sc_out == SCATTER_SURVIVED) continue;
        }
        // facet_event (bounce_body.rs:611).
        V3 hit_point = P.ray.origin + hit.t * P.ray.dir;
        V3 normal = shading_normal_for_hit(sc, hit_point, hit.facet, hit.normal, m.edge_rounding_radius);
        // rotate_stokes_to_plane_of_incidence (raytracer/absorption.rs:69).
        V3 cpn = normalize_or_zero(cross(P.k, normal));
        if (P.has_prev && length_squared(cpn) > F(1e-6f) && length_squared(P.prev_pn) > F(1e-6f)) {
            F cos_psi = clamp_(dot(P.prev_pn, cpn), -1.0f, 1.0f);
            F sin_psi = dot(cross(P.prev_pn, cpn), normalize_or_zero(P.k));
            F psi = atan2_(sin_psi, cos_psi);
            M4 rot = frame_rotation(psi);
            for (int c = 0; c < 8; ++c) P.stokes[c] = apply(rot, P.stokes[c]);
        }
        P.has_prev = true;
        P.prev_pn = cpn;
        // apply_interior_segment (transport/inner.rs:170).
        if (P.inside) {
            normal = -normal;
            if (P.absorbing && m.scattering_sigma_s <= 0.0f) apply_absorption(P, hit.t);
        }
        Geo g = compute_geo(P, normal);
        // dispatch_bounce (transport/bounce.rs:108) + try_dispatch_uniaxial_bounce
        // (refraction/dispatch.rs:67).
        Outcome o;
        o.update = -1;
        o.has_p_o = false;
        o.p_o = 0.0f;
        // facet_finish_for (bounce_body.rs:656): Polished past the end of the list.
        const bool frosted =
            sc->facet_finishes && (uint32_t)hit.facet < sc->n_finishes && sc->facet_finishes[hit.facet] != 0;
        if (frosted) {
            apply_frosted_bounce(P, g, normal, hit_point, bounce, &o);
        } else if (g.sin2_t > F(1.0f)) {
            apply_tir_bounce(P, g, P.k, normal, &o);
        } else {
            const bool nondegenerate = g.has_frame && length_squared(cross(P.k, P.c_axis)) > F(1e-6f);
            if (!P.inside && P.aniso && nondegenerate)
                apply_uniaxial_entry(P, g, P.k, normal, bounce, &o);
            else if (P.inside && nondegenerate)
                apply_uniaxial_internal(P, g, P.k, normal, hit_point, bounce, &o);
            else
                apply_scalar_fresnel(P, g, P.k, normal, cpn, hit_point, bounce, &o);
        }
        const bool was_internal_reflection = P.inside && o.update < 0 && o.new_inside == P.inside;
        const bool inside_before = P.inside;
        P.ray.dir = o.new_s;
        P.ray.origin = hit_point + o.new_s * F(1e-4f);
        P.k = o.new_k;
        P.inside = o.new_inside;
        // record_facet (bounce_body.rs:680), after the dispatch and before glare / roulette.
        if (ev) record_facet(ev, bounce, hit, inside_before, P.inside, P.ray.dir);
        if (o.update >= 0) P.is_e = o.update != 0;
        // maybe_apply_internal_mode_coupling (transport/bounce.rs:470).
        if (P.aniso && was_internal_reflection) {
            F p_o = 0.5f;
            if (o.has_p_o) {
                p_o = o.p_o;
            } else if (!P.biaxial) {
                F po, c2, s2;
                if (entry_eigenmode_selection(P.c_axis, cpn, P.k, P.stokes[0], &po, &c2, &s2)) p_o = po;
            }
            P.is_e = unit_draw(P.seed, bounce, MODE_COUPLING_STREAM) >= p_o;
        }
        // Surface glare (bounce_body.rs:691-697).
        if (bounce == 0 && !P.inside && glare < F(1.0f) && !frosted) {
            for (int c = 0; c < 8; ++c) P.stokes[c] = scale(P.stokes[c], glare);
        }
        // apply_russian_roulette (transport/bounce.rs:355).
        if (bounce > 4 && !russian_roulette(P, bounce)) {
            term = TERM_RR;
            break;
        }
    }
    // finish (bounce_body.rs:724).
    if (P.escaped)
        for (int c = 0; c < 8; ++c) P.radiance[c] = P.radiance[c] + P.split[c];
    const F norm_factor = F(50.0f) / F(106.856f);
    V3 xyz = v3(0.0f, 0.0f, 0.0f);
    for (int c = 0; c < 8; ++c) {
        F family = 0.0f;
        bool first = true;
        for (int j = 0; j < 8; ++j)
            if (P.compat[c] & (1u << j)) {
                family = first ? P.path_pdf[j] : family + P.path_pdf[j];
                first = false;
            }
        F w = (family <= F(1e-12f)) ? F(1.0f) : (F(8.0f) * P.path_pdf[0]) / family;
        F weighted = P.radiance[c] * w;
        xyz = xyz + cmf(P.lambdas[c]) * (weighted * norm_factor);
    }
    xyz = xyz + v3(0.0f, 0.0f, 0.0f);  // + nee_xyz (always zero without NEE)
    if (sc->environment.model != IX_ENV_UNIFORM) {
        // apply_von_kries_white_balance (color.rs:252), run for every Studio environment.
        V3 lms = mat3_fma(BRADFORD_XYZ_TO_LMS, xyz);
        V3 wb = sc->environment.white_balance ? load3(sc->environment.wb_lms) : v3(1.0f, 1.0f, 1.0f);
        xyz = mat3_fma(BRADFORD_LMS_TO_XYZ, mulv(lms, wb));
    }
    xyz = vmax0(xyz);
    if (ev) ev->termination = term;  // attributed.rs:61
    if (info) {
        info->bounces = iterations;
        info->termination = term;
        info->escaped = P.escaped ? 1u : 0u;
        info->exit_splits = P.splits;
    }
    return xyz;
}

static bool scene_supported(const ix_scene* sc) {
    if (!sc) return false;
    if (sc->n_planes > 0 && !sc->planes) return false;
    return true;
}

// cpu_sample_xyz (renderer/cpu_frame.rs:45).
static V3 sample_xyz(const ix_scene* sc, uint32_t pixel, const Rot& rot, uint32_t sample,
                     ixo_path_info* info, ixo_path_events* ev = nullptr, V3* camera_dir = nullptr) {
    uint32_t width = sc->width;
    uint32_t x = pixel % width, y = pixel / width;
    Draws d = sample_draws(pixel, sample, rot);
    Ray ray = generate_ray(sc->camera, F((float)x), F((float)y), F((float)width),
                           F((float)sc->height), d.jx, d.jy);
    if (camera_dir) *camera_dir = ray.dir;
    return trace_path(sc, ray, d.seed, d.hero, info, ev);
}

static inline bool xyz_finite(V3 v) { return is_finite_(v.x) && is_finite_(v.y) && is_finite_(v.z); }

// ------------------------------------------------------------------------------------
// Analytic optical metrics: evaluate_gem_optical_metrics (color/metrics/evaluate.rs:158)
// and what it calls -- the fan geometry (fan.rs), exit lighting (lighting.rs,
// visibility.rs), the single-index interior trace (ray_trace.rs), aperture-sample
// classification and fire (classify.rs), temporal scintillation (scintillation.rs) and
// the finish (accumulate.rs).  Frosted facets and concave tools are not modelled.
// ------------------------------------------------------------------------------------
// f32::to_degrees: a multiply by the f32 rounding of 180/pi.
static inline F to_degrees(F rad) { return rad * F(57.2957795130823208767981548141051703f); }

// measure_model_width (render_setup/stone_width.rs:27): the narrower of the x and z
// extents of the solid's vertices, in f64 (planes n.x + d <= 0 as n.x <= -d).
static double model_width(const float* planes, uint32_t n) {
    struct P {
        double x, y, z, m;
    };
    std::vector<P> ps;
    for (uint32_t i = 0; i < n; ++i) {
        P p{planes[4 * i], planes[4 * i + 1], planes[4 * i + 2], -(double)planes[4 * i + 3]};
        bool dup = false;
        for (const P& q : ps) {
            double c = p.x * q.x + p.y * q.y + p.z * q.z;
            if (c > 1.0 - 1e-12 && std::fabs(p.m - q.m) < 1e-9) dup = true;
        }
        if (!dup) ps.push_back(p);
    }
    double x_min = INFINITY, x_max = -INFINITY, z_min = INFINITY, z_max = -INFINITY;
    size_t count = 0;
    const size_t m = ps.size();
    for (size_t a = 0; a < m; ++a)
        for (size_t b = a + 1; b < m; ++b)
            for (size_t c = b + 1; c < m; ++c) {
                const P &A = ps[a], &B = ps[b], &Cc = ps[c];
                // Cramer: v = (m_a (B x C) + m_b (C x A) + m_c (A x B)) / det.
                double bcx = B.y * Cc.z - B.z * Cc.y, bcy = B.z * Cc.x - B.x * Cc.z, bcz = B.x * Cc.y - B.y * Cc.x;
                double det = A.x * bcx + A.y * bcy + A.z * bcz;
                if (std::fabs(det) < 1e-12) continue;
                double cax = Cc.y * A.z - Cc.z * A.y, cay = Cc.z * A.x - Cc.x * A.z, caz = Cc.x * A.y - Cc.y * A.x;
                double abx = A.y * B.z - A.z * B.y, aby = A.z * B.x - A.x * B.z, abz = A.x * B.y - A.y * B.x;
                double vx = (A.m * bcx + B.m * cax + Cc.m * abx) / det;
                double vy = (A.m * bcy + B.m * cay + Cc.m * aby) / det;
                double vz = (A.m * bcz + B.m * caz + Cc.m * abz) / det;
                bool ok = std::isfinite(vx) && std::isfinite(vy) && std::isfinite(vz);
                for (size_t k = 0; ok && k < m; ++k)
                    if (ps[k].x * vx + ps[k].y * vy + ps[k].z * vz - ps[k].m > 1e-9) ok = false;
                if (!ok) continue;
                ++count;
                x_min = std::min(x_min, vx);
                x_max = std::max(x_max, vx);
                z_min = std::min(z_min, vz);
                z_max = std::max(z_max, vz);
            }
    if (count < 4) return NAN;
    double dx = x_max - x_min, dz = z_max - z_min;
    return dx <= dz ? dx : dz;
}

// The exit lighting of the metrics (lighting.rs:137-209, visibility.rs:30-58).
struct MetricLighting {
    ix_environment env;  // exposure 1, no tray, the default head-shadow cosines
    F spec;              // spectral power at 550 nm
    F threshold;
    F head_shadow_cos;
};
static F metric_radiance(const MetricLighting& L, V3 dir) {
    return lighting_radiance(direction_lighting(L.env, dir, v3(0.0f, 0.0f, 0.0f)), L.env, L.spec);
}
// hemisphere_direction (lighting.rs:74).
static V3 hemisphere_direction(int index) {
    F y = (F((float)index) + F(0.5f)) / F(96.0f);
    F ring = sqrt_(max_(fma_(y, -y, 1.0f), 0.0f));
    F a = F((float)index) * F(2.3999632f);
    return v3(ring * cos_(a), y, ring * sin_(a));
}
static bool metric_lighting(int32_t preset, float light_yaw, float light_pitch, float head_shadow_deg,
                            MetricLighting* out) {
    // scoring_preset (lighting.rs:125): the ASET view scores as the iso-hemisphere.
    if (ixo_environment_preset(preset == 12 ? 1 : preset, 1.0f, light_yaw, light_pitch, 0.0f, 1.0f, 16.0f,
                               &out->env) != 0)
        return false;
    const bool studio = out->env.model == IX_ENV_STUDIO;
    out->spec = spectral_power(out->env, 550.0f);
    // head_shadow_cone_cos (visibility.rs:16).
    if (studio || std::isnan(head_shadow_deg) || head_shadow_deg == 16.0f) {
        out->head_shadow_cos = 0.96f;
    } else if (head_shadow_deg <= 0.0f) {
        out->head_shadow_cos = 2.0f;
    } else {
        F offset = acos_(0.96f) - to_radians(16.0f);
        out->head_shadow_cos = cos_(to_radians(clamp_(head_shadow_deg, 1.0f, 89.0f)) + offset);
    }
    // ambient_level: the median of 96 hemisphere radiances (lighting.rs:101).
    float samples[96];
    for (int i = 0; i < 96; ++i) samples[i] = raw(metric_radiance(*out, hemisphere_direction(i)));
    std::sort(samples, samples + 96);
    F factor = studio ? F(4.0f) : F(0.5f);
    out->threshold = max_(F(samples[48]) * factor, 1.17549435e-38f);
    return true;
}

// The metrics' interior trace at one index (ray_trace.rs:166-352), unfrosted.
enum { FATE_ENTRY_BLOCKED = 0, FATE_LEAKED = 1, FATE_EXITED_UP = 2, FATE_ABSORBED = 3 };
struct ExitPath {
    V3 dir;
    F transmittance, exit_cos;
    int facet;
    uint32_t bounces;
    F path_len;
};
// fresnel_transmittance (ray_trace.rs:35).
static F fresnel_transmittance(F n1, F n2, F cos_i, F cos_t) {
    F denom_s = fma_(n2, cos_t, n1 * cos_i);
    F denom_p = fma_(n2, cos_i, n1 * cos_t);
    if (abs_(denom_s) < F(1e-6f) || abs_(denom_p) < F(1e-6f)) return 0.0f;
    F rs = fma_(n2, -cos_t, n1 * cos_i) / denom_s;
    F rp = fma_(n2, -cos_i, n1 * cos_t) / denom_p;
    F r = midpoint_(rs * rs, rp * rp);
    return clamp_(F(1.0f) - r, 0.0f, 1.0f);
}
static int trace_entry(const float* planes, uint32_t n, V3 entry_point, V3 incoming, V3 n_entry, F cos_i,
                       F index, ExitPath* exit) {
    F inv = F(1.0f) / index;
    F sin2_t = (F(1.0f) / (index * index)) * fma_(cos_i, -cos_i, 1.0f);
    if (sin2_t > F(1.0f)) return FATE_ENTRY_BLOCKED;
    F cos_t = sqrt_(F(1.0f) - sin2_t);
    V3 dir = normalize(inv * incoming + fma_(inv, cos_i, -cos_t) * n_entry);
    F entry_t = fresnel_transmittance(1.0f, index, cos_i, cos_t);
    V3 point = entry_point + dir * F(1e-4f);
    F sin_crit = F(1.0f) / index;
    bool leaked = false, up = false;
    F path_len = 0.0f;
    for (uint32_t bounce = 0; bounce < 10; ++bounce) {
        Hit h;
        if (!intersect(planes, n, Ray{point, dir}, &h)) break;
        path_len = path_len + h.t;
        V3 next = point + h.t * dir;
        V3 n_out = h.normal;
        F cos_theta = clamp_(dot(dir, n_out), 0.0f, 1.0f);
        F sin_theta = sqrt_(max_(fma_(cos_theta, -cos_theta, 1.0f), 0.0f));
        if (sin_theta < sin_crit) {
            F sin2_out = (index * index) * fma_(cos_theta, -cos_theta, 1.0f);
            if (sin2_out <= F(1.0f)) {
                F cos_out = sqrt_(F(1.0f) - sin2_out);
                V3 out_dir = normalize(index * dir + fma_(index, -cos_theta, cos_out) * n_out);
                // Escape::record (ray_trace.rs:110).
                if (n_out.y < F(-0.05f)) {
                    leaked = true;
                } else if (out_dir.y > F(0.05f)) {
                    up = true;
                    exit->dir = out_dir;
                    exit->transmittance = fresnel_transmittance(index, 1.0f, cos_theta, cos_out);
                    exit->exit_cos = cos_out;
                    exit->facet = h.facet;
                    exit->bounces = bounce;
                }
                break;
            }
        }
        dir = normalize(dir - (F(2.0f) * cos_theta) * n_out);
        point = next + dir * F(1e-4f);
    }
    if (leaked) return FATE_LEAKED;
    if (up) {
        exit->transmittance = entry_t * exit->transmittance;
        exit->path_len = path_len;
        return FATE_EXITED_UP;
    }
    return FATE_ABSORBED;
}

// The whole-pose evaluation (evaluate.rs:229-392).
struct MetricStone {
    const float* planes;
    uint32_t n;
    F lateral, standoff;
    F nd, n_f, n_c;
};
static V3 fan_origin(const MetricStone& s, V3 f, V3 r, V3 u, F gu, F gv) {
    return (-f * s.standoff + (gu * s.lateral) * r) + (gv * s.lateral) * u;
}
enum { CLS_NONE = -1, CLS_BLOCKED = 0, CLS_WINDOWED = 1, CLS_EXTINCT = 2, CLS_RETURNED = 3 };
// classify_aperture_sample + classify_ray + fire_sample (classify.rs:47-190).
static int classify_aperture(const MetricStone& s, const MetricLighting& L, V3 f, V3 r, V3 u, F gu, F gv,
                             F sub_r, F sub_u, bool* has_fire, F* fire_angle, F* fire_weight) {
    *has_fire = false;
    V3 dir = normalize((f + sub_r * r) + sub_u * u);
    Ray ray{fan_origin(s, f, r, u, gu, gv), dir};
    Hit h;
    if (!intersect(s.planes, s.n, ray, &h)) return CLS_NONE;
    V3 p = ray.origin + h.t * ray.dir;
    F cos_i = clamp_(dot(-ray.dir, h.normal), 0.0f, 1.0f);
    ExitPath ex;
    int fate = trace_entry(s.planes, s.n, p, ray.dir, h.normal, cos_i, s.nd, &ex);
    if (fate == FATE_ENTRY_BLOCKED) return CLS_BLOCKED;
    if (fate == FATE_LEAKED) return CLS_WINDOWED;
    if (fate == FATE_ABSORBED) return CLS_EXTINCT;
    // returned_or_reason (visibility.rs:42) with the observer at -forward.
    if (dot(ex.dir, -f) > L.head_shadow_cos) return CLS_EXTINCT;
    if (!(metric_radiance(L, ex.dir) > L.threshold)) return CLS_EXTINCT;
    ExitPath ef, ec;
    int ff = trace_entry(s.planes, s.n, p, ray.dir, h.normal, cos_i, s.n_f, &ef);
    int fc = trace_entry(s.planes, s.n, p, ray.dir, h.normal, cos_i, s.n_c, &ec);
    if (ff == FATE_EXITED_UP && fc == FATE_EXITED_UP && ef.facet == ec.facet && ef.bounces == ec.bounces) {
        F cos_sep = clamp_(dot(ef.dir, ec.dir), -1.0f, 1.0f);
        *fire_angle = to_degrees(acos_(cos_sep));
        F energy = (ex.transmittance * ef.transmittance) * ec.transmittance;
        F radiance = max_(ef.exit_cos, 0.0f) * max_(ec.exit_cos, 0.0f);
        *fire_weight = energy * radiance;
        *has_fire = true;
    }
    return CLS_RETURNED;
}
// cell_returned_at_yaw_offset (scintillation.rs:85).
static bool temporal_returned(const MetricStone& s, const MetricLighting& L, const ix_camera& cam, F gu, F gv) {
    V3 f = load3(cam.forward), r = load3(cam.right), u = load3(cam.up);
    Ray ray{fan_origin(s, f, r, u, gu, gv), f};
    Hit h;
    if (!intersect(s.planes, s.n, ray, &h)) return false;
    V3 p = ray.origin + h.t * ray.dir;
    F cos_i = clamp_(dot(-ray.dir, h.normal), 0.0f, 1.0f);
    ExitPath ex;
    if (trace_entry(s.planes, s.n, p, ray.dir, h.normal, cos_i, s.nd, &ex) != FATE_EXITED_UP) return false;
    if (dot(ex.dir, -f) > L.head_shadow_cos) return false;
    return metric_radiance(L, ex.dir) > L.threshold;
}

static void evaluate_metrics(const float* planes, uint32_t n, const ix_material& m, F cam_yaw, F cam_pitch,
                             const MetricLighting& L, float out[5]) {
    MetricStone s;
    s.planes = planes;
    s.n = n;
    double w = model_width(planes, n);
    F half_width = (std::isfinite(w) && w > 0.0) ? F((float)(w * 0.5)) : F(1.0f);
    s.standoff = F(2.5f) * half_width;
    s.lateral = (F(0.95f) * half_width) / sqrt_(0.70f);
    s.nd = max_(dispersion_eval(m.dispersion, 589.3f), 1.1f);
    s.n_f = max_(dispersion_eval(m.dispersion, 486.1f), 1.001f);
    s.n_c = max_(dispersion_eval(m.dispersion, 656.3f), 1.001f);
    ix_camera cam;
    camera_new(cam_yaw, cam_pitch, 1.0f, 42.0f, &cam);
    const F offsets[5] = {-3.0f, -1.5f, 0.0f, 1.5f, 3.0f};
    ix_camera tcam[5];
    for (int k = 0; k < 5; ++k) camera_new(cam_yaw + to_radians(offsets[k]), cam_pitch, 1.0f, 42.0f, &tcam[k]);
    const F subs[5][2] = {{0.0f, 0.0f}, {0.08f, 0.0f}, {-0.08f, 0.0f}, {0.0f, 0.08f}, {0.0f, -0.08f}};
    V3 f = load3(cam.forward), r = load3(cam.right), u = load3(cam.up);
    uint32_t total = 0, windowed = 0, extinct = 0, returned = 0, cells = 0;
    F fire_sum = 0.0f, frac_sum = 0.0f, frac_sq = 0.0f, tvar_sum = 0.0f;
    for (int ix = 0; ix < 18; ++ix)
        for (int iz = 0; iz < 18; ++iz) {
            F gu = fma_((F((float)ix) + F(0.5f)) / F(18.0f), 2.0f, -1.0f);
            F gv = fma_((F((float)iz) + F(0.5f)) / F(18.0f), 2.0f, -1.0f);
            if (fma_(gv, gv, gu * gu) > F(0.70f)) continue;
            uint32_t cell_total = 0, cell_returned = 0;
            for (int k = 0; k < 5; ++k) {
                bool has_fire;
                F angle, weight;
                int cls = classify_aperture(s, L, f, r, u, gu, gv, subs[k][0], subs[k][1], &has_fire, &angle, &weight);
                if (cls == CLS_NONE) continue;
                ++total;
                ++cell_total;
                if (cls == CLS_WINDOWED) ++windowed;
                else if (cls == CLS_EXTINCT) ++extinct;
                else if (cls == CLS_RETURNED) {
                    ++returned;
                    ++cell_returned;
                    if (has_fire) fire_sum = fma_(angle, weight, fire_sum);
                }
            }
            if (cell_total > 0) {
                F frac = F((float)cell_returned) / F((float)cell_total);
                frac_sum = frac_sum + frac;
                frac_sq = fma_(frac, frac, frac_sq);
                ++cells;
                uint32_t t_ret = 0;
                for (int k = 0; k < 5; ++k) t_ret += temporal_returned(s, L, tcam[k], gu, gv) ? 1u : 0u;
                F tp = F((float)t_ret) / F(5.0f);
                tvar_sum = tvar_sum + fma_(tp, -tp, tp);
            }
        }
    // finish_metrics (accumulate.rs:99).
    F n_total = F((float)std::max(total, 1u));
    out[0] = raw(clamp_(F((float)returned) / n_total * F(100.0f), 0.0f, 100.0f));
    out[1] = raw(max_(fire_sum / n_total * F(275.0f), 0.1f));
    // spatial / temporal / combined scintillation (scintillation.rs:119-160).
    F spatial = 0.0f;
    if (cells > 0) {
        F mean = frac_sum / F((float)cells);
        if (mean > F(1e-4f)) {
            F var = max_(fma_(mean, -mean, frac_sq / F((float)cells)), 0.0f);
            F cv = sqrt_(var) / mean;
            spatial = clamp_(cv / (F(1.0f) + cv) * F(100.0f), 0.0f, 100.0f);
        }
    }
    F temporal = cells > 0 ? clamp_(tvar_sum / F((float)cells) / F(0.24f) * F(100.0f), 0.0f, 100.0f) : F(0.0f);
    out[2] = raw(clamp_(fma_(0.4f, temporal, F(0.6f) * spatial), 0.0f, 100.0f));
    out[3] = raw(clamp_(F((float)windowed) / n_total * F(100.0f), 0.0f, 100.0f));
    out[4] = raw(clamp_(F((float)extinct) / n_total * F(100.0f), 0.0f, 100.0f));
}

// ------------------------------------------------------------------------------------
// Spectral attribution: classify_path (color/metrics/attribution.rs:75-98) through
// class_index (renderer/attribution_map.rs:39-58), and AttributionPixel::add
// (attribution_map.rs:105-120).
// ------------------------------------------------------------------------------------
static uint32_t classify_events(const ixo_path_events& ev, V3 observer, const MetricLighting& L) {
    if (ev.first_facet < 0) return IX_CLASS_MISS;
    if (!ev.first_entered) return IX_CLASS_GLARE;
    if (ev.exit_facet < 0) {
        // unexited_reason (attribution.rs:57): roulette, the bounce cap, or an escape
        // without an exit event (the analytical map's "no intersection").
        if (ev.termination == TERM_RR || ev.termination == TERM_SCATTER_ABSORBED) return IX_CLASS_KILLED;
        if (ev.termination == TERM_CAP) return IX_CLASS_BUDGET;
        return IX_CLASS_NO_INTERSECTION;
    }
    if (F(ev.exit_normal[1]) < F(-0.05f)) return IX_CLASS_WINDOWED;  // WINDOW_NORMAL_Y
    const V3 dir = load3(ev.exit_dir);
    if (dir.y > F(0.05f)) {  // UPWARD_DIR_Y
        // returned_or_reason (visibility.rs:55) and is_illuminated (lighting.rs:207).
        if (dot(dir, observer) > L.head_shadow_cos) return IX_CLASS_SHADOW;
        return metric_radiance(L, dir) > L.threshold ? IX_CLASS_RETURNED : IX_CLASS_UNLIT;
    }
    return IX_CLASS_SIDE_EXIT;
}

static void attribution_add(ix_attribution_pixel* p, uint32_t cls, uint32_t scattered, uint32_t fluoresced,
                            float y) {
    auto sat = [](uint32_t a) { return a == UINT32_MAX ? a : a + 1u; };
    p->samples = sat(p->samples);
    if (cls >= IX_ATTRIBUTION_CLASSES) return;
    p->hits = sat(p->hits);
    p->counts[cls] = sat(p->counts[cls]);
    if (std::isfinite(y)) {
        p->y_sum[cls] = raw(F(p->y_sum[cls]) + F(y));
        p->y_sq_sum[cls] = raw(F(p->y_sq_sum[cls]) + F(y) * F(y));
    }
    p->scattered += scattered ? 1u : 0u;
    p->fluoresced += fluoresced ? 1u : 0u;
}


// ------------------------------------------------------------------------------------
// The display pipeline after the path (renderer/guide_pass.rs, renderer/denoise/,
// renderer/tonemap.rs, color/space.rs, color/gamut.rs).  Plain f32 arithmetic in the
// reference's operation order; `mul_add` is std::fma; expf / powf are the libm calls
// Rust's f32::exp / f32::powf make on Linux.
// ------------------------------------------------------------------------------------
static inline F pow_(F a, F b) { return F(powf(raw(a), raw(b))); }

// Guide pass: path_signature (guide_pass.rs:560-625).
static const uint32_t SIG_EXIT_BIT = 0x8000u, SIG_ESCAPE = 0xFFFFu;
static inline uint32_t fnv_mix(uint32_t hash, uint32_t word) {
    for (int shift = 0; shift < 32; shift += 8) {
        hash ^= (word >> shift) & 0xFFu;
        hash *= 0x01000193u;
    }
    return hash;
}
// guide_pass.rs `unit`: v / |v| with an unfused dot (glam's Vec3 / f32 divides each lane).
static inline V3 unit_div(V3 v) {
    F len = sqrt_(dot(v, v));
    if (len > F(0.0f)) return v3(v.x / len, v.y / len, v.z / len);
    return v;
}
static uint32_t path_signature(const Ray& ray, const Hit& first, const float* planes, uint32_t n, F n_d) {
    if (std::isnan(raw(n_d)) || n_d <= F(1.0f)) return 0;
    uint32_t hash = fnv_mix(0x811c9dc5u, (uint32_t)first.facet);
    V3 incident = unit_div(ray.dir);
    F cos_i = max_(-dot(incident, first.normal), 0.0f);
    F eta = F(1.0f) / n_d;
    F k = F(1.0f) - eta * eta * (F(1.0f) - cos_i * cos_i);
    if (k <= F(0.0f)) return std::max(fnv_mix(hash, SIG_ESCAPE), 1u);
    V3 dir = unit_div(incident * eta + first.normal * (eta * cos_i - sqrt_(k)));
    V3 origin = ray.origin + ray.dir * first.t;
    for (int b = 0; b < 3; ++b) {  // SIGNATURE_BOUNCES
        Ray probe{origin + dir * F(1.0e-4f), dir};
        Hit hit;
        if (!intersect(planes, n, probe, &hit)) {
            hash = fnv_mix(hash, SIG_ESCAPE);
            break;
        }
        origin = probe.origin + dir * hit.t;
        const uint32_t facet = (uint32_t)hit.facet & 0x7FFFu;
        F cos_t = dot(dir, hit.normal);
        F sin_sq = n_d * n_d * (F(1.0f) - cos_t * cos_t);
        if (sin_sq > F(1.0f)) {
            hash = fnv_mix(hash, facet);
            dir = unit_div(dir - hit.normal * (F(2.0f) * cos_t));
        } else {
            hash = fnv_mix(hash, facet | SIG_EXIT_BIT);
            break;
        }
    }
    return std::max(hash, 1u);
}
// fill_rows (guide_pass.rs:640-690) for one pixel.
static void guide_pixel(const ix_camera& cam, uint32_t x, uint32_t y, uint32_t w, uint32_t h,
                        const float* planes, uint32_t n, F n_d, float* depth, float* normal,
                        int32_t* facet, uint32_t* sig) {
    Ray ray = generate_ray(cam, F((float)x), F((float)y), F((float)w), F((float)h), 0.0f, 0.0f);
    Hit hit;
    if (intersect(planes, n, ray, &hit)) {
        *depth = raw(hit.t);
        store3(normal, hit.normal);
        *facet = hit.facet;
        if (sig) *sig = path_signature(ray, hit, planes, n, n_d);
    } else {
        *depth = 1.0e6f;
        normal[0] = normal[1] = normal[2] = 0.0f;
        *facet = -1;
        if (sig) *sig = 0;
    }
}

// A-Trous (denoise/pass.rs).
static const float B3_SPLINE[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
static const float SIGMA_EPS = 1.0e-8f;
static inline F sanitize(F v) { return is_finite_(v) ? v : F(0.0f); }
static inline bool finite3(V3 v) { return is_finite_(v.x) && is_finite_(v.y) && is_finite_(v.z); }
// unit_normal_or_zero (pass.rs:67).
static inline V3 unit_normal_or_zero(V3 n) {
    n = v3(sanitize(n.x), sanitize(n.y), sanitize(n.z));
    F len = sqrt_(dot(n, n));
    if (len <= F(SIGMA_EPS)) return v3(0.0f, 0.0f, 0.0f);
    return v3(n.x / len, n.y / len, n.z / len);
}
// cos_pow (pass.rs:87): repeated squaring for a power-of-two integer exponent, else powf.
static inline F cos_pow(F base, F power) {
    const float p = raw(power);
    if (p >= 0.0f && p == std::floor(p) && p <= 4294967295.0f) {
        const uint32_t ip = (uint32_t)p;
        if (ip != 0 && (ip & (ip - 1)) == 0) {
            F v = base;
            for (uint32_t s = ip; s > 1; s >>= 1) v = v * v;
            return v;
        }
    }
    return pow_(base, power);
}
static inline bool is_zero3(V3 v) { return v.x == F(0.0f) && v.y == F(0.0f) && v.z == F(0.0f); }
struct TapConst {
    F neg_inv_sigma_depth, neg_inv_two_sigma_color_sq, normal_power;
};
// atrous_pixel (pass.rs:330-378) with tap_contribution (pass.rs:283-316).
static V3 atrous_pixel(const float* src, const float* depth, const float* nrm_n, const int32_t* facet_id,
                       const uint32_t* sig, uint32_t width, uint32_t height, uint32_t x, uint32_t y,
                       int64_t stride, const TapConst& tc) {
    const size_t ci = (size_t)y * width + x;
    V3 raw_c = load3(src + 3 * ci);
    V3 color = finite3(raw_c) ? raw_c : v3(0.0f, 0.0f, 0.0f);
    const int32_t facet = facet_id[ci];
    if (facet < 0) return color;
    const uint32_t csig = sig ? sig[ci] : 0u;
    const F cdepth = depth[ci];
    const V3 cnormal = load3(nrm_n + 3 * ci);
    V3 sum = v3(0.0f, 0.0f, 0.0f);
    F wsum = 0.0f;
    for (int ky = 0; ky < 5; ++ky) {
        const int64_t sy = (int64_t)y + (int64_t)(ky - 2) * stride;
        if (sy < 0 || sy >= (int64_t)height) continue;
        for (int kx = 0; kx < 5; ++kx) {
            const int64_t sx = (int64_t)x + (int64_t)(kx - 2) * stride;
            if (sx < 0 || sx >= (int64_t)width) continue;
            const size_t idx = (size_t)sy * width + (size_t)sx;
            const F kernel_w = F(B3_SPLINE[ky]) * F(B3_SPLINE[kx]);
            if (facet_id[idx] != facet) continue;
            if (sig && sig[idx] != csig) continue;
            const V3 texel = load3(src + 3 * idx);
            if (!finite3(texel)) continue;
            F wn;
            const V3 qn = load3(nrm_n + 3 * idx);
            if (is_zero3(cnormal) || is_zero3(qn)) {
                wn = 1.0f;
            } else {
                F c = max_(clamp_(dot(cnormal, qn), -1.0f, 1.0f), 0.0f);
                wn = cos_pow(c, max_(tc.normal_power, 0.0f));
            }
            if (wn == F(0.0f)) continue;
            const F gap = abs_(sanitize(cdepth) - sanitize(F(depth[idx])));
            const F wd = gap == F(0.0f) ? F(1.0f) : exp_(gap * tc.neg_inv_sigma_depth);
            const V3 d = color - texel;
            const F dist_sq = dot(d, d);
            const F wc = dist_sq == F(0.0f) ? F(1.0f) : exp_(dist_sq * tc.neg_inv_two_sigma_color_sq);
            const F w = kernel_w * F(1.0f) * wn * wd * wc;
            sum = sum + texel * w;
            wsum = wsum + w;
        }
    }
    if (wsum > F(SIGMA_EPS)) return v3(sum.x / wsum, sum.y / wsum, sum.z / wsum);
    return color;
}
template <typename Fn>
static void parallel_rows(uint32_t rows, int threads, Fn fn) {
    if (threads <= 1 || rows < 2) {
        for (uint32_t y = 0; y < rows; ++y) fn(y);
        return;
    }
    std::vector<std::thread> pool;
    std::atomic<uint32_t> next{0};
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&] {
            for (uint32_t y; (y = next.fetch_add(1)) < rows;) fn(y);
        });
    for (auto& th : pool) th.join();
}
static int display_threads(int threads) {
    if (threads > 0) return threads;
    const unsigned hc = std::thread::hardware_concurrency();
    return hc ? (int)hc : 8;
}
// AtrousDenoiser::denoise_into_with_threads (denoise/mod.rs:280-345).
static void atrous_denoise(const float* color, const float* depth, const float* normal, const int32_t* facet_id,
                           const uint32_t* sig, uint32_t width, uint32_t height, uint32_t spp,
                           const ix_atrous_params& p, float* out, int threads) {
    const size_t len = (size_t)width * height;
    if (len == 0) return;
    const F n0 = max_(p.taper_reference_spp, SIGMA_EPS);
    const F taper = F(1.0f) / sqrt_(F(1.0f) + F((float)spp) / n0);
    const uint32_t passes = std::min(std::max(p.num_passes, 1u), 8u);
    if (taper < F(p.taper_identity_epsilon)) {
        std::memcpy(out, color, len * 3 * sizeof(float));
        return;
    }
    const F sce = max_(F(p.sigma_color) * taper, 0.0f);
    std::vector<float> buf[2] = {std::vector<float>(color, color + 3 * len), std::vector<float>(3 * len)};
    std::vector<float> nrm_n(3 * len);
    for (size_t i = 0; i < len; ++i) store3(nrm_n.data() + 3 * i, unit_normal_or_zero(load3(normal + 3 * i)));
    const F sd = max_(p.sigma_depth, SIGMA_EPS);
    const F scs = max_(sce * sce, SIGMA_EPS);
    TapConst tc{F(-1.0f) / sd, F(-1.0f) / (F(2.0f) * scs), F(p.normal_power)};
    const int nt = display_threads(threads);
    for (uint32_t pass = 0; pass < passes; ++pass) {
        const float* src = buf[pass & 1].data();
        float* dst = buf[(pass & 1) ^ 1].data();
        parallel_rows(height, nt, [&](uint32_t y) {
            for (uint32_t x = 0; x < width; ++x)
                store3(dst + 3 * ((size_t)y * width + x),
                       atrous_pixel(src, depth, nrm_n.data(), facet_id, sig, width, height, x, y,
                                    (int64_t)1 << pass, tc));
        });
    }
    std::memcpy(out, buf[passes & 1].data(), len * 3 * sizeof(float));
}

// ColorSpace tables (color/space.rs:159-196).
static const float XYZ_TO_RGB[4][3][3] = {
    {{3.2404542f, -1.5371385f, -0.4985314f}, {-0.969266f, 1.8760108f, 0.041556f}, {0.0556434f, -0.2040259f, 1.0572252f}},
    {{2.493497f, -0.9313836f, -0.40271078f}, {-0.829489f, 1.762664f, 0.023624686f}, {0.03584583f, -0.07617239f, 0.9568845f}},
    {{1.7166512f, -0.35567078f, -0.2533663f}, {-0.6666843f, 1.6164812f, 0.015768546f}, {0.017639857f, -0.042770613f, 0.9421031f}},
    {{1.6410234f, -0.3248033f, -0.2364247f}, {-0.66366286f, 1.6153316f, 0.016756348f}, {0.011721894f, -0.008284442f, 0.98839486f}},
};
static const float WHITE_XY[4][2] = {{0.3127f, 0.3290f}, {0.3127f, 0.3290f}, {0.3127f, 0.3290f}, {0.32168f, 0.33767f}};
// ColorSpace::xyz_to_linear (space.rs:210).
static inline V3 xyz_to_linear(uint32_t sp, V3 c) {
    const float (*m)[3] = XYZ_TO_RGB[sp];
    return v3(fma_(m[0][0], c.x, fma_(m[0][1], c.y, F(m[0][2]) * c.z)),
              fma_(m[1][0], c.x, fma_(m[1][1], c.y, F(m[1][2]) * c.z)),
              fma_(m[2][0], c.x, fma_(m[2][1], c.y, F(m[2][2]) * c.z)));
}
// project_to_gamut_bounded (gamut.rs:43-101).
static V3 project_to_gamut_bounded(V3 c, uint32_t sp, F mx) {
    const F sum = c.x + c.y + c.z;
    if (!is_finite_(sum) || sum <= F(1e-6f)) return v3(0.0f, 0.0f, 0.0f);
    const F x = c.x / sum, y = c.y / sum;
    const F lum = max_(c.y, 0.0f);
    auto in_range = [&](V3 v) {
        return v.x >= F(0.0f) && v.y >= F(0.0f) && v.z >= F(0.0f) && v.x <= mx && v.y <= mx && v.z <= mx;
    };
    const V3 lin = xyz_to_linear(sp, c);
    if (in_range(lin)) return lin;
    const F wx = WHITE_XY[sp][0], wy = WHITE_XY[sp][1];
    auto mapped = [&](F t) {
        const F xp = fma_(wx - x, t, x);
        const F yp = fma_(wy - y, t, y);
        if (yp > F(1e-6f)) return v3((xp / yp) * lum, lum, ((F(1.0f) - xp - yp) / yp) * lum);
        return v3((wx / wy) * lum, lum, ((F(1.0f) - wx - wy) / wy) * lum);
    };
    V3 resolved = vmax0(xyz_to_linear(sp, mapped(1.0f)));
    for (uint32_t i = 0; i <= 32; ++i) {
        const F t = F((float)i) / F(32.0f);
        const V3 cand = xyz_to_linear(sp, mapped(t));
        if (in_range(cand)) {
            resolved = cand;
            break;
        }
    }
    return resolved;
}
// TransferFunction::encode (space.rs:54-75).
static inline F transfer_encode(uint32_t sp, F lin) {
    if (sp == IX_COLOR_SPACE_SRGB || sp == IX_COLOR_SPACE_DISPLAY_P3) {
        if (lin <= F(0.0031308f)) return lin * F(12.92f);
        return fma_(1.055f, pow_(lin, F(1.0f) / F(2.4f)), -0.055f);
    }
    if (sp == IX_COLOR_SPACE_REC2020) {
        const F alpha = 1.0992968f, beta = 0.01805397f;
        if (lin < beta) return lin * F(4.5f);
        return fma_(alpha, pow_(lin, 0.45f), -(alpha - F(1.0f)));
    }
    return lin;
}
// aces_tonemap (optics/raytracer/color.rs:372).
static inline F aces_tonemap(F y) {
    return (y * fma_(2.51f, y, 0.03f)) / fma_(y, fma_(2.43f, y, 0.59f), 0.14f);
}
// ColorSpace::encode with ToneMap::AcesFilmic { exposure: 1.0 } (space.rs:234-278).
static void color_encode(V3 c, uint32_t sp, uint8_t out[4]) {
    out[3] = 255;
    const F sum = c.x + c.y + c.z;
    if (!is_finite_(sum) || sum <= F(1e-6f)) {
        out[0] = out[1] = out[2] = 0;
        return;
    }
    const F exposure = 1.0f;
    const F lum = max_(c.y, 0.0f);
    const F exposed = max_(lum * exposure, 0.0f);
    const F y_tm = aces_tonemap(exposed);
    const F scale = (y_tm / max_(exposed, 1e-5f)) * exposure;
    const V3 rgb = project_to_gamut_bounded(c * scale, sp, 1.0f);
    const F ch[3] = {rgb.x, rgb.y, rgb.z};
    for (int k = 0; k < 3; ++k) {
        const F lin = is_finite_(ch[k]) ? clamp_(ch[k], 0.0f, 1.0f) : F(0.0f);
        const F enc = clamp_(transfer_encode(sp, lin), 0.0f, 1.0f);
        out[k] = (uint8_t)raw(fma_(enc, 255.0f, 0.5f));
    }
}
}  // namespace ixo

using namespace ixo;

extern "C" {

uint32_t ixo_hash_u32(uint32_t x) { return hash_u32(x); }
float ixo_low_discrepancy_base2(uint32_t n) { return raw(low_discrepancy_base2(n)); }
float ixo_radical_inverse_base(uint32_t n, uint32_t base) {
    return raw(radical_inverse_base(n, base));
}
void ixo_pixel_rotations(uint32_t pixel, float out[3]) {
    Rot r = pixel_rotations(pixel);
    out[0] = raw(r.jx);
    out[1] = raw(r.jy);
    out[2] = raw(r.hero);
}
void ixo_sample_draws(uint32_t pixel, uint32_t sample, const float rot[3], uint32_t* seed,
                      float out[3]) {
    Rot r = rot ? Rot{rot[0], rot[1], rot[2]} : pixel_rotations(pixel);
    Draws d = sample_draws(pixel, sample, r);
    *seed = d.seed;
    out[0] = raw(d.jx);
    out[1] = raw(d.jy);
    out[2] = raw(d.hero);
}
void ixo_camera_new(float yaw, float pitch, float distance, float fov_deg, ix_camera* out) {
    camera_new(yaw, pitch, distance, fov_deg, out);
}
void ixo_generate_ray(const ix_camera* cam, float sx, float sy, float w, float h, float jx,
                      float jy, float origin[3], float dir[3]) {
    Ray r = generate_ray(*cam, sx, sy, w, h, jx, jy);
    store3(origin, r.origin);
    store3(dir, r.dir);
}
void ixo_hero_wavelengths(float hero_rand, float out[8]) {
    F l[8];
    hero_wavelengths(hero_rand, l);
    for (int k = 0; k < 8; ++k) out[k] = raw(l[k]);
}
float ixo_dispersion_eval(const ix_dispersion* d, float lambda_nm) {
    return raw(dispersion_eval(*d, lambda_nm));
}
void ixo_cmf(float lambda_nm, float out[3]) { store3(out, cmf(lambda_nm)); }
float ixo_d65(float lambda_nm) { return raw(d65(lambda_nm)); }
float ixo_exp_lane(float x) { return raw(exp_lane(x)); }
float ixo_tir_phase_delta(float n1, float cos_i, float sin_i) {
    return raw(tir_phase_delta(n1, cos_i, sin_i));
}
void ixo_fresnel_reflect_apply(float r_s, float r_p, const float s_in[4], float s_out[4]) {
    Stokes s{s_in[0], s_in[1], s_in[2], s_in[3]};
    Stokes o = apply(fresnel_reflection(r_s, r_p), s);
    s_out[0] = raw(o.i);
    s_out[1] = raw(o.q);
    s_out[2] = raw(o.u);
    s_out[3] = raw(o.v);
}
float ixo_spectral_absorption(const ix_absorption* a, float lambda_nm) { return raw(spectral_absorption(*a, lambda_nm)); }

void ixo_rotate_stokes(const float k[3], const float normal[3], const float prev_pn[3], uint32_t has_prev,
                       const float s_in[4], float s_out[4], float cpn_out[3]) {
    // rotate_stokes_to_plane_of_incidence (raytracer/absorption.rs:69) as facet_event calls it.
    const V3 kk = load3(k), nn = load3(normal), prev = load3(prev_pn);
    Stokes st{s_in[0], s_in[1], s_in[2], s_in[3]};
    const V3 cpn = normalize_or_zero(cross(kk, nn));
    if (has_prev && length_squared(cpn) > F(1e-6f) && length_squared(prev) > F(1e-6f)) {
        F cos_psi = clamp_(dot(prev, cpn), -1.0f, 1.0f);
        F sin_psi = dot(cross(prev, cpn), normalize_or_zero(kk));
        st = apply(frame_rotation(atan2_(sin_psi, cos_psi)), st);
    }
    s_out[0] = raw(st.i), s_out[1] = raw(st.q), s_out[2] = raw(st.u), s_out[3] = raw(st.v);
    store3(cpn_out, cpn);
}

void ixo_fresnel_channel(float n1, float n2, float cos_i, const float s_in[4], float out[13]) {
    // One channel of apply_partial_reflect_bounce / apply_tir_bounce (reflected Stokes,
    // before the 1 / r_unpol selection weight) and of apply_refract_channel (transmitted
    // Stokes, before 1 / (1 - r_unpol)), with the same geometry the bounce computes.
    const Stokes st{s_in[0], s_in[1], s_in[2], s_in[3]};
    const F one_m_c2 = fma_(F(cos_i), -F(cos_i), 1.0f);
    const F sin_i = sqrt_(max_(one_m_c2, 0.0f));
    const F eta = F(n1) / F(n2);
    const F s2 = eta * eta * one_m_c2;
    for (int i = 0; i < 13; ++i) out[i] = 0.0f;
    if (s2 > F(1.0f)) {
        const Stokes r = apply(tir_retardation(tir_phase_delta(n1, cos_i, sin_i)), st);
        out[0] = raw(r.i), out[1] = raw(r.q), out[2] = raw(r.u), out[3] = raw(r.v);
        out[12] = 1.0f;
        return;
    }
    const F cos_t = sqrt_(max_(F(1.0f) - s2, 0.0f));
    F r_s, r_p;
    fresnel_rs_rp(n1, n2, cos_i, cos_t, &r_s, &r_p);
    const Stokes r = apply(fresnel_reflection(r_s, r_p), st);
    const F two = F(2.0f) * F(n1) * F(cos_i);
    const F t_s = two / fma_(F(n2), cos_t, F(n1) * F(cos_i));
    const F t_p = two / fma_(F(n1), cos_t, F(n2) * F(cos_i));
    const Stokes t = apply(fresnel_transmission(n1, n2, cos_i, cos_t, t_s, t_p), st);
    out[0] = raw(r.i), out[1] = raw(r.q), out[2] = raw(r.u), out[3] = raw(r.v);
    out[4] = raw(t.i), out[5] = raw(t.q), out[6] = raw(t.u), out[7] = raw(t.v);
    out[8] = raw(r_s), out[9] = raw(r_p), out[10] = raw(t_s), out[11] = raw(t_p);
}

// The biaxial indicatrix of `m` at n_beta (its absorption at lambda) evaluated at wave normal k:
// out[0..1] wave_indices (slow, fast); out[2..7] eigen_polarizations (slow xyz, fast xyz);
// out[8..13] mode_poynting_dir (slow, fast); out[14..21] resolve_entry_mode against
// `normal` at cos_i seeded with n_beta (slow n, dir xyz, fast n, dir xyz); out[22..23]
// the assigned-mode alpha of the biaxial tensor (mode B, mode A).
void ixo_biaxial_bundle(const ix_material* m, const float k[3], const float normal[3], float cos_i,
                        float lambda_nm, float n_beta_in, float out[24]) {
    const V3 kk = load3(k), nn = load3(normal);
    const F n_beta = n_beta_in;
    const TensorFrame ax = tensor_frame(load3(m->c_axis));
    const Indicatrix I = make_indicatrix(*m, n_beta, ax);
    F ns, nf;
    wave_indices(I, kk, &ns, &nf);
    out[0] = raw(ns);
    out[1] = raw(nf);
    store3(out + 2, eigen_polarization(I, kk, true));
    store3(out + 5, eigen_polarization(I, kk, false));
    store3(out + 8, mode_poynting_dir(I, kk, true));
    store3(out + 11, mode_poynting_dir(I, kk, false));
    V3 d;
    out[14] = raw(resolve_entry_mode(I, kk, nn, cos_i, n_beta, true, &d));
    store3(out + 15, d);
    out[18] = raw(resolve_entry_mode(I, kk, nn, cos_i, n_beta, false, &d));
    store3(out + 19, d);
    const F ao = spectral_absorption(m->abs_o, lambda_nm), ae = spectral_absorption(m->abs_e, lambda_nm);
    const F ab = m->has_abs_beta ? spectral_absorption(m->abs_beta, lambda_nm) : ao;
    out[22] = raw(quadratic_form3(ax, ao, ab, ae, assigned_mode_e_field_biaxial(I, kk, true)));
    out[23] = raw(quadratic_form3(ax, ao, ab, ae, assigned_mode_e_field_biaxial(I, kk, false)));
}
// A tool's ray interval (ToolPrimitive::ray_interval): 1 and out = (t_lo, t_hi), or 0.
int ixo_tool_ray_interval(const ix_tool* t, const float origin[3], const float dir[3], float out[2]) {
    F lo, hi;
    if (!tool_ray_interval(*t, Ray{load3(origin), load3(dir)}, &lo, &hi)) return 0;
    out[0] = raw(lo);
    out[1] = raw(hi);
    return 1;
}
int ixo_tool_contains(const ix_tool* t, const float p[3]) { return tool_contains(*t, load3(p)) ? 1 : 0; }
// The distance to the nearest piece surface (boundary_gap, tool.rs:550).
float ixo_tool_boundary_gap(const ix_tool* t, const float p[3]) {
    Piece ps[6];
    const int n = tool_pieces(*t, ps);
    F best = INFINITY;
    for (int i = 0; i < n; ++i) {
        V3 nn;
        best = min_(best, abs_(piece_sd_normal(ps[i], load3(p), &nn)));
    }
    return n ? raw(best) : 0.0f;
}
void ixo_tool_outward_normal(const ix_tool* t, const float p[3], float out[3]) {
    store3(out, tool_outward_normal(*t, load3(p)));
}
// intersect_stone_soa_side: returns 1 on a hit (t, normal, facet, and for a carved
// stone entering 0 / 1, else -1 in *entering), 0 on a miss.
int ixo_intersect_stone(const float* planes, uint32_t n_planes, const ix_tool* tools, uint32_t n_tools,
                        const float origin[3], const float dir[3], float* t, float normal[3], int32_t* facet,
                        int32_t* entering) {
    ix_scene sc{};
    sc.planes = planes;
    sc.n_planes = n_planes;
    sc.tools = tools;
    sc.n_tools = n_tools;
    Hit h;
    bool carved = false, ent = false;
    if (!intersect_scene(&sc, Ray{load3(origin), load3(dir)}, &h, &carved, &ent)) return 0;
    *t = raw(h.t);
    store3(normal, h.normal);
    *facet = h.facet;
    *entering = carved ? (ent ? 1 : 0) : -1;
    return 1;
}
// sample_environment_for_nee under DaylightSun (environment/nee.rs:81): the disc draw
// for (u0, u1) into dir, returning its pdf.
float ixo_sun_nee_sample(const ix_environment* env, float u0, float u1, float dir[3]) {
    store3(dir, sun_cone_direction(load3(env->key_dir), u0, u1));
    return raw(F(1.0f) / F(SUN_SOLID_ANGLE));
}
// environment_nee_pdf under DaylightSun (environment/nee.rs:144).
float ixo_sun_nee_pdf(const ix_environment* env, const float dir[3]) { return raw(sun_nee_pdf(*env, load3(dir))); }
float ixo_balance_heuristic(float a, float b) { return raw(balance_heuristic(a, b)); }
// nee_contribution_frosted_exterior (scattering/frosted.rs:98) under the scene's
// DaylightSun: the deposit of one event at `origin` into radiance[8], the channels at
// lambdas[8] with unpolarised intensities[8].
void ixo_frosted_sun_nee(const ix_scene* sc, const float origin[3], const float ext_normal[3], uint32_t seed,
                         uint32_t bounce, const float lambdas[8], const float intensities[8], float radiance[8]) {
    Path P{};
    P.sc = sc;
    P.seed = seed;
    for (int c = 0; c < 8; ++c) {
        P.lambdas[c] = lambdas[c];
        P.stokes[c] = Stokes{F(intensities[c]), F(0.0f), F(0.0f), F(0.0f)};
        P.radiance[c] = radiance[c];
    }
    frosted_sun_nee(P, load3(origin), load3(ext_normal), bounce);
    for (int c = 0; c < 8; ++c) radiance[c] = raw(P.radiance[c]);
}
float ixo_channel_alpha(const ix_material* m, const float k[3], float lambda_nm) {
    // The non-birefringent branch of channel_absorption_alphas_assigned
    // (raytracer/absorption.rs:197): the midpoint of the tensor's quadratic form over the
    // two eigen-polarisations of the wave normal.
    const V3 c_axis = load3(m->c_axis), kk = load3(k);
    const F ao = spectral_absorption(m->abs_o, lambda_nm), ae = spectral_absorption(m->abs_e, lambda_nm);
    const TensorFrame tf = tensor_frame(c_axis);
    const V3 ea = ordinary_eigen_polarization(kk, c_axis);
    const V3 eb = normalize_or_zero(cross(kk, ea));
    return raw(midpoint_(quadratic_form(tf, ao, ae, ea), quadratic_form(tf, ao, ae, eb)));
}

int ixo_intersect(const float* planes, uint32_t n_planes, const float origin[3],
                  const float dir[3], float* t, int32_t* facet) {
    Ray r{load3(origin), load3(dir)};
    Hit h;
    if (!intersect(planes, n_planes, r, &h)) return 0;
    *t = raw(h.t);
    *facet = h.facet;
    return 1;
}

// Lighting presets by the reference's LightingPreset::index (environment/mod.rs:475-493):
// 1 IsoHemisphere, 7 Daylight, 8 Incandescent, 9 IlluminantA, 10 RingLights,
// 11 DarkSpotlight.  Parameters from LightingPreset::params (environment/mod.rs:318-411).
int ixo_environment_preset(int32_t preset, float exposure, float light_yaw, float light_pitch,
                           float backdrop, float surface_glare, float head_shadow_deg,
                           ix_environment* out) {
    std::memset(out, 0, sizeof(*out));
    // LightingPreset::params / model / uses_d65 / uv_line (environment/mod.rs:318-560).
    float temp_k = 6500.0f, spot = 1.0f;
    float tent[5] = {1.0f, 1.0f, 1.0f, 0.02f, 0.0f};  // walls, cards, spark, ground, flat
    bool d65_spec = true, uv = false;
    float uv_centre = 0.0f, uv_fwhm = 0.0f;
    uint32_t model;
    switch (preset) {
        case 0: model = IX_ENV_LIGHT_TENT; temp_k = 5000.0f; d65_spec = false; break;
        case 1: model = IX_ENV_ISO_HEMISPHERE; break;
        case 2: model = IX_ENV_LIGHT_TENT; spot = 0.0f; tent[0] = 5.0f; tent[1] = 0.0f; tent[2] = 0.0f;
                tent[3] = 0.8f; tent[4] = 1.0f; break;
        case 3: model = IX_ENV_LIGHT_TENT; tent[0] = 3.0f; tent[1] = 0.0f; tent[3] = 0.05f; break;
        case 4: model = IX_ENV_LIGHT_TENT; tent[0] = 0.4f; tent[1] = 0.0f; tent[2] = 0.0f; tent[3] = 0.03f; break;
        case 5: model = IX_ENV_DAYLIGHT_DOME; break;
        case 6: model = IX_ENV_DAYLIGHT_SUN; break;
        case 7: model = IX_ENV_STUDIO; break;
        case 8: model = IX_ENV_STUDIO; temp_k = 3200.0f; spot = 1.2f; d65_spec = false; break;
        case 9: model = IX_ENV_STUDIO; temp_k = 2856.0f; spot = 1.2f; d65_spec = false; break;
        case 10: model = IX_ENV_STUDIO; temp_k = 5000.0f; spot = 1.6f; d65_spec = false; break;
        case 11: model = IX_ENV_STUDIO; temp_k = 6000.0f; spot = 2.4f; d65_spec = false; break;
        case 12: model = IX_ENV_ASET; break;
        case 13: model = IX_ENV_STUDIO; d65_spec = false; uv = true; uv_centre = 365.0f; uv_fwhm = 10.0f; break;
        case 14: model = IX_ENV_STUDIO; d65_spec = false; uv = true; uv_centre = 395.0f; uv_fwhm = 12.0f; break;
        default: return -1;
    }
    out->model = model;
    out->spectrum = model == IX_ENV_ASET ? IX_SPEC_WAVELENGTH
                    : uv                 ? IX_SPEC_GAUSSIAN
                    : d65_spec           ? IX_SPEC_D65
                                         : IX_SPEC_BLACKBODY;
    if (uv) {
        out->line_centre_nm = uv_centre;
        // fwhm / (2 sqrt(2 ln 2)) in f32 (mod.rs:560).
        out->line_sigma_nm = uv_fwhm / (2.0f * std::sqrt(2.0f * 0.6931472f));
    }
    out->tent_walls = tent[0];
    out->tent_cards = tent[1];
    out->tent_spark = tent[2];
    out->tent_ground = tent[3];
    out->tent_flat = tent[4];
    out->exposure = exposure;
    out->spot_mult = spot;
    out->ambient_fill = uv ? 0 : 1;
    out->backdrop = backdrop;
    // clamp_surface_glare (environment/source.rs:170).
    out->surface_glare = (surface_glare >= 1.0f || std::isnan(surface_glare)) ? 1.0f
                         : (surface_glare > 0.0f ? surface_glare : 0.0f);
    // head_shadow_cosines (environment/mod.rs:128) after clamp_head_shadow_deg (:146).
    float deg = head_shadow_deg;
    if (std::isnan(deg)) deg = 16.0f;
    else if (deg <= 0.0f) deg = 0.0f;
    else if (deg < 3.0f) deg = 3.0f;
    else if (deg > 88.0f) deg = 88.0f;
    if (deg == 16.0f) {
        out->shadow_cos[0] = 0.9510565f;
        out->shadow_cos[1] = 0.9702957f;
    } else if (deg <= 0.0f) {
        out->shadow_cos[0] = 2.0f;
        out->shadow_cos[1] = 3.0f;
    } else {
        float dd = deg < 3.0f ? 3.0f : (deg > 88.0f ? 88.0f : deg);
        out->shadow_cos[0] = raw(cos_(to_radians(F(dd) + F(2.0f))));
        out->shadow_cos[1] = raw(cos_(to_radians(F(dd) - F(2.0f))));
    }
    F t_k, den;
    blackbody_norm(temp_k, &t_k, &den);
    out->bb_t_k = raw(t_k);
    out->bb_denom_560 = raw(den);
    // StudioRig::new (optics/studio_rig.rs:33).
    F cos_pitch = cos_(light_pitch), sin_pitch = sin_(light_pitch);
    F cos_yaw = cos_(light_yaw), sin_yaw = sin_(light_yaw);
    store3(out->key_dir, normalize(v3(cos_pitch * sin_yaw, sin_pitch, cos_pitch * cos_yaw)));
    const F PI = 3.14159265358979323846f;
    F fill_yaw = fma_(PI, 0.78f, light_yaw);
    F fill_pitch = clamp_(F(light_pitch) * F(0.65f), 0.15f, 1.2f);
    store3(out->fill_dir, normalize(v3(cos_(fill_pitch) * sin_(fill_yaw), sin_(fill_pitch),
                                       cos_(fill_pitch) * cos_(fill_yaw))));
    F step = PI * F(2.0f) / F(16.0f);
    for (int i = 0; i < IX_RING_LIGHTS; ++i) {
        F angle = fma_(F((float)i), step, light_yaw);
        store3(out->ring_dirs[i],
               normalize(v3(sin_(angle) * F(0.75f), sin_pitch * F(0.8f), cos_(angle) * F(0.75f))));
    }
    // sun_radiance_factor (sun.rs:25): the disc's radiance, faded below the horizon.
    out->sun_factor = raw(F(SUN_RADIANCE) * smoothstep(-0.05f, 0.05f, F(out->key_dir[1])));
    // illuminant_white_balance (color.rs:328): identity unless the preset uses one
    // (uses_white_balance, mod.rs:553: neither D65 nor a UV lamp nor the ASET view).
    if (!d65_spec && !uv && model != IX_ENV_ASET) {
        out->white_balance = 1;
        store3(out->wb_lms, illuminant_white_balance(temp_k));
    } else {
        out->white_balance = 0;
        out->wb_lms[0] = out->wb_lms[1] = out->wb_lms[2] = 1.0f;
    }
    out->uniform_radiance = 0.0f;
    return 0;
}

int ixo_metrics(const float* planes, uint32_t n_planes, const ix_material* material, float cam_yaw,
                float cam_pitch, int32_t preset, float light_yaw, float light_pitch,
                float head_shadow_deg, float out[5]) {
    if (!planes || n_planes == 0 || !material) return -1;
    MetricLighting L;
    if (!metric_lighting(preset, light_yaw, light_pitch, head_shadow_deg, &L)) return -1;
    evaluate_metrics(planes, n_planes, *material, cam_yaw, cam_pitch, L, out);
    return 0;
}

float ixo_metrics_half_width(const float* planes, uint32_t n_planes) {
    double w = model_width(planes, n_planes);
    return (std::isfinite(w) && w > 0.0) ? (float)(w * 0.5) : 1.0f;
}

int ixo_metrics_lighting(int32_t preset, float light_yaw, float light_pitch, float head_shadow_deg,
                         float out[3]) {
    MetricLighting L;
    if (!metric_lighting(preset, light_yaw, light_pitch, head_shadow_deg, &L)) return -1;
    out[0] = raw(L.threshold);
    out[1] = raw(L.head_shadow_cos);
    out[2] = raw(L.spec);
    return 0;
}

int ixo_trace_ray_events(const ix_scene* scene, const float origin[3], const float dir[3],
                         uint32_t seed, float hero_rand, float xyz[3], ixo_path_events* events) {
    if (!scene_supported(scene) || !events) return -1;
    Ray r{load3(origin), load3(dir)};
    store3(xyz, trace_path(scene, r, seed, hero_rand, nullptr, events));
    return 0;
}

void ixo_path_events_reset(ixo_path_events* events) {
    std::memset(events, 0, sizeof(*events));
    events->first_facet = -1;
    events->exit_facet = -1;
}

void ixo_path_events_facet(ixo_path_events* events, uint32_t bounce, int32_t facet, const float normal[3],
                           uint32_t inside_before, uint32_t inside_after, const float dir_after[3]) {
    Hit h;
    h.t = 1.0f;
    h.normal = load3(normal);
    h.facet = facet;
    record_facet(events, bounce, h, inside_before != 0, inside_after != 0, load3(dir_after));
}

int ixo_classify_path(const ixo_path_events* events, const float observer[3], int32_t preset,
                      float light_yaw, float light_pitch, float head_shadow_deg) {
    MetricLighting L;
    if (!events || !metric_lighting(preset, light_yaw, light_pitch, head_shadow_deg, &L)) return -1;
    return (int)classify_events(*events, load3(observer), L);
}

void ixo_attribution_add(ix_attribution_pixel* pixel, uint32_t class_code, uint32_t scattered,
                         uint32_t fluoresced, float y) {
    attribution_add(pixel, class_code, scattered, fluoresced, y);
}

int64_t ixo_attribute_pixels(const ix_scene* scene, int32_t preset, float light_yaw,
                             float light_pitch, float head_shadow_deg, uint32_t pixel_begin,
                             uint32_t pixel_end, uint32_t sample_offset, uint32_t spp,
                             uint32_t threads, ix_attribution_pixel* map, double* sums_f64) {
    if (!scene_supported(scene) || !map) return -1;
    MetricLighting L;
    if (!metric_lighting(preset, light_yaw, light_pitch, head_shadow_deg, &L)) return -1;
    if (threads == 0) threads = 1;
    std::vector<int64_t> dropped(threads, 0);
    auto worker = [&](uint32_t t) {
        for (uint32_t pixel = pixel_begin + t; pixel < pixel_end; pixel += threads) {
            Rot rot = pixel_rotations(pixel);
            ix_attribution_pixel& ap = map[pixel - pixel_begin];
            double sd[3] = {0.0, 0.0, 0.0};
            for (uint32_t s = 0; s < spp; ++s) {
                ixo_path_events ev;
                V3 cam_dir;
                V3 xyz = sample_xyz(scene, pixel, rot, sample_offset + s, nullptr, &ev, &cam_dir);
                // The observer is the reverse of the camera ray (attribution_tests.rs:129).
                const uint32_t cls = classify_events(ev, -cam_dir, L);
                attribution_add(&ap, cls, ev.scattered, 0, raw(xyz.y));
                if (xyz_finite(xyz)) {
                    sd[0] += (double)raw(xyz.x);
                    sd[1] += (double)raw(xyz.y);
                    sd[2] += (double)raw(xyz.z);
                } else {
                    dropped[t]++;
                }
            }
            if (sums_f64) {
                size_t o = 3 * (size_t)(pixel - pixel_begin);
                sums_f64[o] += sd[0];
                sums_f64[o + 1] += sd[1];
                sums_f64[o + 2] += sd[2];
            }
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto& th : pool) th.join();
    int64_t total = 0;
    for (auto d : dropped) total += d;
    return total;
}

void ixo_environment_uniform(float radiance, ix_environment* out) {
    std::memset(out, 0, sizeof(*out));
    out->model = IX_ENV_UNIFORM;
    out->spectrum = IX_SPEC_FLAT;
    out->exposure = 1.0f;
    out->surface_glare = 1.0f;
    out->wb_lms[0] = out->wb_lms[1] = out->wb_lms[2] = 1.0f;
    out->uniform_radiance = radiance;
}

float ixo_environment_channel(const ix_environment* env, const float dir[3], float lambda_nm,
                              const float observer[3]) {
    return raw(environment_channel(*env, load3(dir), lambda_nm,
                                   observer ? load3(observer) : v3(0.0f, 0.0f, 0.0f)));
}

int ixo_trace_ray(const ix_scene* scene, const float origin[3], const float dir[3],
                  uint32_t seed, float hero_rand, float xyz[3], ixo_path_info* info) {
    if (!scene_supported(scene)) return -1;
    Ray r{load3(origin), load3(dir)};
    store3(xyz, trace_path(scene, r, seed, hero_rand, info));
    return 0;
}

int ixo_trace_sample(const ix_scene* scene, uint32_t pixel, uint32_t sample, float xyz[3],
                     ixo_path_info* info) {
    if (!scene_supported(scene)) return -1;
    store3(xyz, sample_xyz(scene, pixel, pixel_rotations(pixel), sample, info));
    return 0;
}

int64_t ixo_trace_frame(const ix_scene* scene, uint32_t sample_offset, uint32_t spp,
                        uint32_t threads, float* sums_f32, double* sums_f64) {
    if (!scene_supported(scene)) return -1;
    uint32_t num_pixels = scene->width * scene->height;
    if (threads == 0) threads = 1;
    std::vector<int64_t> dropped(threads, 0);
    auto worker = [&](uint32_t first) {
        // trace_pixels_interleaved (cpu_frame.rs:104): pixel = first, first + stride, ...
        for (uint32_t pixel = first; pixel < num_pixels; pixel += threads) {
            Rot rot = pixel_rotations(pixel);
            V3 sum = v3(0.0f, 0.0f, 0.0f);
            double sd[3] = {0.0, 0.0, 0.0};
            for (uint32_t s = 0; s < spp; ++s) {
                V3 xyz = sample_xyz(scene, pixel, rot, sample_offset + s, nullptr);
                // add_finite_sample (sampling.rs:237).
                if (xyz_finite(xyz)) {
                    sum = sum + xyz;
                    sd[0] += (double)raw(xyz.x);
                    sd[1] += (double)raw(xyz.y);
                    sd[2] += (double)raw(xyz.z);
                } else {
                    dropped[first]++;
                }
            }
            if (sums_f32) store3(sums_f32 + 3 * (size_t)pixel, sum);
            if (sums_f64) {
                sums_f64[3 * (size_t)pixel] = sd[0];
                sums_f64[3 * (size_t)pixel + 1] = sd[1];
                sums_f64[3 * (size_t)pixel + 2] = sd[2];
            }
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto& th : pool) th.join();
    int64_t total = 0;
    for (auto d : dropped) total += d;
    return total;
}

int64_t ixo_trace_pixels(const ix_scene* scene, uint32_t pixel_begin, uint32_t pixel_end,
                         uint32_t sample_offset, uint32_t spp, uint32_t threads,
                         double* sums_f64) {
    if (!scene_supported(scene)) return -1;
    if (threads == 0) threads = 1;
    std::vector<int64_t> dropped(threads, 0);
    auto worker = [&](uint32_t t) {
        for (uint32_t pixel = pixel_begin + t; pixel < pixel_end; pixel += threads) {
            Rot rot = pixel_rotations(pixel);
            double sd[3] = {0.0, 0.0, 0.0};
            for (uint32_t s = 0; s < spp; ++s) {
                V3 xyz = sample_xyz(scene, pixel, rot, sample_offset + s, nullptr);
                if (xyz_finite(xyz)) {
                    sd[0] += (double)raw(xyz.x);
                    sd[1] += (double)raw(xyz.y);
                    sd[2] += (double)raw(xyz.z);
                } else {
                    dropped[t]++;
                }
            }
            size_t o = 3 * (size_t)(pixel - pixel_begin);
            sums_f64[o] = sd[0];
            sums_f64[o + 1] = sd[1];
            sums_f64[o + 2] = sd[2];
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto& th : pool) th.join();
    int64_t total = 0;
    for (auto d : dropped) total += d;
    return total;
}

int64_t ixo_trace_pixel_set(const ix_scene* scenes, uint32_t n_scenes, const uint32_t* scene_of,
                            const uint32_t* pixel, const uint32_t* spp, uint32_t n, uint32_t sample_offset,
                            uint32_t threads, double* sums_f64) {
    for (uint32_t i = 0; i < n_scenes; ++i)
        if (!scene_supported(&scenes[i])) return -1;
    for (uint32_t k = 0; k < n; ++k)
        if (scene_of[k] >= n_scenes || pixel[k] >= scenes[scene_of[k]].width * scenes[scene_of[k]].height) return -1;
    if (threads == 0) threads = 1;
    std::atomic<uint32_t> next{0};
    std::vector<int64_t> dropped(threads, 0);
    auto worker = [&](uint32_t t) {
        for (;;) {
            const uint32_t k = next.fetch_add(1, std::memory_order_relaxed);
            if (k >= n) break;
            const ix_scene* sc = &scenes[scene_of[k]];
            Rot rot = pixel_rotations(pixel[k]);
            double sd[3] = {0.0, 0.0, 0.0};
            for (uint32_t s = 0; s < spp[k]; ++s) {
                V3 xyz = sample_xyz(sc, pixel[k], rot, sample_offset + s, nullptr);
                if (xyz_finite(xyz)) {
                    sd[0] += (double)raw(xyz.x);
                    sd[1] += (double)raw(xyz.y);
                    sd[2] += (double)raw(xyz.z);
                } else {
                    dropped[t]++;
                }
            }
            if (sums_f64) {
                sums_f64[3 * (size_t)k] = sd[0];
                sums_f64[3 * (size_t)k + 1] = sd[1];
                sums_f64[3 * (size_t)k + 2] = sd[2];
            }
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto& th : pool) th.join();
    int64_t total = 0;
    for (auto d : dropped) total += d;
    return total;
}

int ixo_simd_build(void) {
#if defined(IX_ORACLE_AVX2) && !defined(IX_COUNT_FLOPS)
    return 1;
#else
    return 0;
#endif
}

int ixo_trace_samples(const ix_scene* scene, uint32_t pixel_begin, uint32_t pixel_end,
                      uint32_t sample_offset, uint32_t spp, uint32_t threads, float* xyz,
                      uint32_t* bounces) {
    if (!scene_supported(scene)) return -1;
    if (threads == 0) threads = 1;
    auto worker = [&](uint32_t t) {
        for (uint32_t pixel = pixel_begin + t; pixel < pixel_end; pixel += threads) {
            Rot rot = pixel_rotations(pixel);
            for (uint32_t s = 0; s < spp; ++s) {
                ixo_path_info info;
                V3 v = sample_xyz(scene, pixel, rot, sample_offset + s, &info);
                size_t o = (size_t)(pixel - pixel_begin) * spp + s;
                store3(xyz + 3 * o, v);
                if (bounces) bounces[o] = info.bounces;
            }
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto& th : pool) th.join();
    return 0;
}

uint32_t ixo_standard_round_brilliant(float* out) {
    const F PI = 3.14159265358979323846f;
    const F gear = 96.0f;
    uint32_t n = 0;
    auto push = [&](V3 nrm, F d) {
        V3 u = normalize(nrm);  // GpuFacetPlane::new (geometry/plane.rs:44)
        out[4 * n] = raw(u.x);
        out[4 * n + 1] = raw(u.y);
        out[4 * n + 2] = raw(u.z);
        out[4 * n + 3] = raw(d);
        ++n;
    };
    auto azimuth = [&](F g) { return F(2.0f) * PI * (g + F(0.0f)) / gear; };
    auto tier = [&](const float* idx, int count, F angle_deg, bool crown, F d) {
        F a = to_radians(angle_deg);
        for (int i = 0; i < count; ++i) {
            F phi = azimuth(idx[i]);
            V3 nrm = v3(sin_(a) * cos_(phi), crown ? cos_(a) : -cos_(a), sin_(a) * sin_(phi));
            push(nrm, d);
        }
    };
    static const float stars[8] = {6, 18, 30, 42, 54, 66, 78, 90};
    static const float mains[8] = {0, 12, 24, 36, 48, 60, 72, 84};
    static const float halves[16] = {95, 1, 11, 13, 23, 25, 35, 37, 47, 49, 59, 61, 71, 73, 83, 85};
    push(v3(0.0f, 1.0f, 0.0f), -0.32f);
    tier(stars, 8, 15.0f, true, -0.45f);
    tier(mains, 8, 34.5f, true, -0.59f);
    tier(halves, 16, 41.0f, true, -0.67f);
    for (int i = 0; i < 16; ++i) {
        F phi = F(2.0f) * PI * F((float)i) / F(16.0f);
        push(v3(cos_(phi), 0.0f, sin_(phi)), -1.0f);
    }
    tier(mains, 8, 41.0f, false, -0.67f);
    tier(halves, 16, 42.5f, false, -0.68f);
    push(v3(0.0f, -1.0f, 0.0f), -0.88f);
    return n;
}

int ixo_counting_build(void) {
#ifdef IX_COUNT_FLOPS
    return 1;
#else
    return 0;
#endif
}

int ixo_count_flops(const ix_scene* scene, uint32_t pixel_begin, uint32_t pixel_end,
                    uint32_t pixel_step, uint32_t sample_offset, uint32_t spp,
                    ixo_flop_counts* out) {
#ifdef IX_COUNT_FLOPS
    if (!scene_supported(scene)) return -1;
    g_cnt = Counters();
    uint64_t paths = 0;
    if (pixel_step == 0) pixel_step = 1;
    for (uint32_t pixel = pixel_begin; pixel < pixel_end; pixel += pixel_step) {
        Rot rot = pixel_rotations(pixel);
        for (uint32_t s = 0; s < spp; ++s) {
            (void)sample_xyz(scene, pixel, rot, sample_offset + s, nullptr);
            ++paths;
        }
    }
    out->add = g_cnt.add;
    out->mul = g_cnt.mul;
    out->fma = g_cnt.fma;
    out->div = g_cnt.div;
    out->sqrt = g_cnt.sqrt;
    out->transcendental = g_cnt.transc;
    out->paths = paths;
    return 0;
#else
    (void)scene; (void)pixel_begin; (void)pixel_end; (void)pixel_step; (void)sample_offset;
    (void)spp; (void)out;
    return -1;
#endif
}


// ---- display pipeline --------------------------------------------------------------
void ixo_atrous_params_default(ix_atrous_params* p) {
    // AtrousParams::default (denoise/mod.rs:194).
    *p = ix_atrous_params{5u, 0.35f, 0.1f, 64.0f, 4.0f, 0.02f};
}
void ixo_generate_guide_buffers(uint32_t width, uint32_t height, const ix_camera* cam, const float* planes,
                                uint32_t n_planes, float n_d, float* depth, float* normal, int32_t* facet_id,
                                uint32_t* path_sig, int threads) {
    parallel_rows(height, display_threads(threads), [&](uint32_t y) {
        for (uint32_t x = 0; x < width; ++x) {
            const size_t i = (size_t)y * width + x;
            guide_pixel(*cam, x, y, width, height, planes, n_planes, F(n_d), depth + i, normal + 3 * i,
                        facet_id + i, path_sig ? path_sig + i : nullptr);
        }
    });
}
float ixo_n_d(const ix_dispersion* d) {
    // DispersionModel::n_d (optics/dispersion.rs:264): the index at 589.3 nm.
    return raw(dispersion_eval(*d, F(589.3f)));
}
void ixo_atrous_denoise(const float* color, const float* depth, const float* normal, const int32_t* facet_id,
                        const uint32_t* path_sig, uint32_t width, uint32_t height, uint32_t spp,
                        const ix_atrous_params* params, float* out, int threads) {
    atrous_denoise(color, depth, normal, facet_id, path_sig, width, height, spp, *params, out, threads);
}
void ixo_color_encode(const float xyz[3], uint32_t color_space, uint8_t out[4]) {
    color_encode(load3(xyz), color_space, out);
}
void ixo_tonemap_to_rgba(const float* xyz, uint64_t pixels, float scale, uint32_t color_space, uint8_t* rgba,
                         int threads) {
    // tonemap_chunk / tonemap_chunk_in (tonemap.rs:85, 165): encode(xyz * scale).
    const uint64_t rows = (pixels + 4095) / 4096;
    parallel_rows((uint32_t)rows, display_threads(threads), [&](uint32_t r) {
        const uint64_t end = std::min<uint64_t>(pixels, (uint64_t)(r + 1) * 4096);
        for (uint64_t i = (uint64_t)r * 4096; i < end; ++i)
            color_encode(load3(xyz + 3 * i) * F(scale), color_space, rgba + 4 * i);
    });
}
void ixo_denoise_and_tonemap_frame(uint32_t width, uint32_t height, uint32_t spp, const float* accum,
                                   const float* depth, const float* normal, const int32_t* facet_id,
                                   const uint32_t* path_sig, const ix_atrous_params* params, uint8_t* rgba,
                                   int threads) {
    // denoise_and_tonemap_frame_with_params_into (frame_denoise.rs:40-80).
    const size_t len = (size_t)width * height;
    std::vector<float> avg(3 * len, 0.0f), filtered(3 * len, 0.0f);
    if (spp == 0) {
        ixo_tonemap_to_rgba(filtered.data(), len, 1.0f, IX_COLOR_SPACE_SRGB, rgba, threads);
        return;
    }
    const F inv = F(1.0f) / F((float)spp);
    for (size_t i = 0; i < 3 * len; ++i) avg[i] = raw(F(accum[i]) * inv);
    atrous_denoise(avg.data(), depth, normal, facet_id, path_sig, width, height, spp, *params, filtered.data(),
                   threads);
    ixo_tonemap_to_rgba(filtered.data(), len, 1.0f, IX_COLOR_SPACE_SRGB, rgba, threads);
}

/* Counting build only: the floating-point operations of one A-Trous denoise of the given
 * frame (all passes), tallied like ixo_count_flops; `paths` holds pixel-passes. */
int ixo_count_denoise_flops(const float* color, const float* depth, const float* normal, const int32_t* facet_id,
                            const uint32_t* path_sig, uint32_t width, uint32_t height, uint32_t spp,
                            const ix_atrous_params* params, ixo_flop_counts* out) {
#ifdef IX_COUNT_FLOPS
    const size_t len = (size_t)width * height;
    std::vector<float> tmp(3 * len);
    g_cnt = Counters{};
    atrous_denoise(color, depth, normal, facet_id, path_sig, width, height, spp, *params, tmp.data(), 1);
    out->add = g_cnt.add;
    out->mul = g_cnt.mul;
    out->fma = g_cnt.fma;
    out->div = g_cnt.div;
    out->sqrt = g_cnt.sqrt;
    out->transcendental = g_cnt.transc;
    out->paths = (uint64_t)len * std::min(std::max(params->num_passes, 1u), 8u);
    return 0;
#else
    (void)color; (void)depth; (void)normal; (void)facet_id; (void)path_sig; (void)width; (void)height;
    (void)spp; (void)params; (void)out;
    return -1;
#endif
}

void ixo_shading_normal_near_edge(const float* planes, uint32_t n_planes, const float hit_point[3], int32_t facet,
                                  const float hit_normal[3], float radius, float out[3]) {
    store3(out, shading_normal_near_edge(planes, n_planes, load3(hit_point), facet, load3(hit_normal), F(radius)));
}

}  // extern "C"
