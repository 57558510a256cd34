// ix_display.cu -- the display pipeline after the path on sm_100a: guide-buffer prepass,
// edge-avoiding A-Trous denoise and tone-map to RGBA8.
//
// Reference (crates/indicatrix/src/): renderer/guide_pass.rs (fill_rows :640-690,
// path_signature :560-625), renderer/denoise/pass.rs (atrous_pixel :330-378,
// tap_contribution :283-316, unit_normal_or_zero :67, cos_pow :87), renderer/denoise/
// mod.rs (denoise_into_with_threads :280-345), renderer/tonemap.rs, color/space.rs
// (ColorSpace::encode :234-278, TransferFunction::encode :54-75, matrices :159-196),
// color/gamut.rs (project_to_gamut_bounded :43-101), optics/raytracer/color.rs
// (aces_tonemap :372).
//
// Layout: one thread per pixel everywhere.  The A-Trous passes read the colour with the
// pixel's sanitised depth as one float4 (one 16-byte load per tap), the facet id and path
// signature as int2 and, unless the normals are the facets' own, the unit normal as
// float4; a 32 x 8 block makes every tap of a warp one contiguous 32-pixel row segment,
// so the dilated taps stay coalesced at every stride.  The last pass writes RGBA8 directly (the tone-map is fused into it), so the
// filtered colour never goes back to HBM.
//
// Built twice like the transport: IX_EXACT=1 (-fmad=false; exp and pow rounded from
// double, which is the correctly rounded value for all but a few inputs in 10^8) and
// the fast build (contraction, single-precision expf / powf).  The guide pass and the
// packing are geometry and bookkeeping: they are built once, exact, and shared.
#include "ix_device.cuh"
#include "ix_display_launch.h"

#if IX_EXACT
#define IX_DISP_FN(name) name##_exact
#else
#define IX_DISP_FN(name) name##_fast
#endif

namespace ix {
namespace disp {
namespace {

// XYZ -> linear RGB of each ColorSpace, row-major (color/space.rs:159-183), and the
// spaces' white points (space.rs:187-195).  Numeric tables of the colour science,
// identical by necessity.
__constant__ float c_xyz_to_rgb[4][9] = {
    {3.2404542f, -1.5371385f, -0.4985314f, -0.969266f, 1.8760108f, 0.041556f, 0.0556434f, -0.2040259f,
     1.0572252f},
    {2.493497f, -0.9313836f, -0.40271078f, -0.829489f, 1.762664f, 0.023624686f, 0.03584583f, -0.07617239f,
     0.9568845f},
    {1.7166512f, -0.35567078f, -0.2533663f, -0.6666843f, 1.6164812f, 0.015768546f, 0.017639857f,
     -0.042770613f, 0.9421031f},
    {1.6410234f, -0.3248033f, -0.2364247f, -0.66366286f, 1.6153316f, 0.016756348f, 0.011721894f,
     -0.008284442f, 0.98839486f},
};
__constant__ float c_white_xy[4][2] = {{0.3127f, 0.3290f}, {0.3127f, 0.3290f}, {0.3127f, 0.3290f},
                                       {0.32168f, 0.33767f}};
// B3-spline taps for offsets -2..2 (pass.rs:38).
__constant__ float c_b3[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};

IX_DEV float exp_disp(float x) {
#if IX_EXACT
    return (float)exp((double)x);
#else
    return expf(x);
#endif
}
IX_DEV float pow_disp(float x, float y) {
#if IX_EXACT
    return (float)pow((double)x, (double)y);
#else
    return powf(x, y);
#endif
}
IX_DEV bool finite3(float4 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }
IX_DEV float sanitize(float v) { return isfinite(v) ? v : 0.0f; }

// ColorSpace::xyz_to_linear (space.rs:210): mul_add chain per row.
IX_DEV V3 xyz_to_linear(uint32_t sp, V3 c) {
    const float* m = c_xyz_to_rgb[sp];
    return v3(fmaf(m[0], c.x, fmaf(m[1], c.y, m[2] * c.z)), fmaf(m[3], c.x, fmaf(m[4], c.y, m[5] * c.z)),
              fmaf(m[6], c.x, fmaf(m[7], c.y, m[8] * c.z)));
}
IX_DEV bool in_range(V3 v, float mx) {
    return v.x >= 0.0f && v.y >= 0.0f && v.z >= 0.0f && v.x <= mx && v.y <= mx && v.z <= mx;
}
// project_to_gamut_bounded (gamut.rs:43-101): walk the chromaticity toward the white
// point at constant luminance in 32 steps; the first step whose RGB is in [0, mx] wins.
//
// The walk is the reference's, step for step, but only over the steps that can pass.  In
// exact arithmetic, with yp(t) > 0 on the whole walk, step t's RGB is (lum / yp(t)) M c(t)
// with c(t) = (xp, yp, 1 - xp - yp) linear in t, so each of the six range conditions is a
// linear inequality alpha + beta t >= 0 and the steps that can pass form one interval.
// The bounds are computed with a margin of 1e-5 relative to the magnitudes involved
// (the float evaluation of a step, and of the bounds' own coefficients, errs by a few
// 1e-7 of them) and widened by a step on each side; every step outside is out of range in float arithmetic too, and the
// steps inside are evaluated exactly as the reference does, in order.  Inputs outside
// the analysed domain (lum <= 0, chromaticity y <= 1e-3, |x|, |y| > 8) walk all 33 steps.
IX_DEV V3 gamut_step(uint32_t sp, float x, float y, float lum, float wx, float wy, float t) {
    const float xp = fmaf(wx - x, t, x);
    const float yp = fmaf(wy - y, t, y);
    if (yp > 1e-6f) return xyz_to_linear(sp, v3((xp / yp) * lum, lum, (((1.0f - xp) - yp) / yp) * lum));
    return xyz_to_linear(sp, v3((wx / wy) * lum, lum, (((1.0f - wx) - wy) / wy) * lum));
}
IX_DEV void walk_bounds(uint32_t sp, float x, float y, float lum, float wx, float wy, float mx, int* i_begin,
                        int* i_end) {
    *i_begin = 0;
    *i_end = 32;
    if (!(lum > 0.0f) || !(y > 1e-3f) || !(fabsf(x) <= 8.0f) || !(fabsf(y) <= 8.0f) || !isfinite(mx)) return;
    const float dx = wx - x, dy = wy - y;
    const float cbound = 2.0f + 2.0f * fmaxf(1.0f, fmaxf(fabsf(x), fabsf(y)));
    float lo = 0.0f, hi = 1.0f;
    const float* r = c_xyz_to_rgb[sp];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float m0 = r[3 * k], m1 = r[3 * k + 1], m2 = r[3 * k + 2];
        // The coefficients' own float error is below 1e-6 of these magnitudes, the margin
        // 1e-5 of them, so the half-lines below contain every step that can pass.
        const float a = m0 * x + m1 * y + m2 * (1.0f - x - y);
        const float bcoef = m0 * dx + m1 * dy - m2 * (dx + dy);
        const float s = (fabsf(m0) + fabsf(m1) + fabsf(m2)) * cbound * 1e-5f;
        // lower: a + b t >= -s ; upper: mx (y + dy t) - lum (a + b t) >= -s_up, whose
        // margin also covers the rounding of the mx y and mx dy terms.
        const float s_up = lum * s + (fabsf(mx * y) + fabsf(mx * dy)) * 1e-5f;
        const float alpha[2] = {a + s, mx * y - lum * a + s_up};
        const float beta[2] = {bcoef, mx * dy - lum * bcoef};
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (beta[c] > 0.0f) {
                lo = fmaxf(lo, -alpha[c] / beta[c]);
            } else if (beta[c] < 0.0f) {
                hi = fminf(hi, -alpha[c] / beta[c]);
            } else if (alpha[c] < 0.0f) {
                lo = 2.0f;  // this condition fails at every step
            }
        }
    }
    if (!(lo <= hi)) {
        *i_begin = 1;
        *i_end = 0;
        return;
    }
    // The bounds are within 1e-6 of the half-lines' ends; one step of slack either side.
    *i_begin = max(0, (int)ceilf(32.0f * lo) - 1);
    *i_end = min(32, (int)floorf(32.0f * hi) + 1);
}
IX_DEV V3 project_to_gamut_bounded(V3 c, uint32_t sp, float mx) {
    const float sum = (c.x + c.y) + c.z;
    if (!isfinite(sum) || sum <= 1e-6f) return v3(0.0f, 0.0f, 0.0f);
    const float x = c.x / sum, y = c.y / sum;
    const float lum = fmaxf(c.y, 0.0f);
    const V3 lin = xyz_to_linear(sp, c);
    if (in_range(lin, mx)) return lin;
    const float wx = c_white_xy[sp][0], wy = c_white_xy[sp][1];
    int i0, i1;
    walk_bounds(sp, x, y, lum, wx, wy, mx, &i0, &i1);
    for (int i = i0; i <= i1; ++i) {
        const V3 cand = gamut_step(sp, x, y, lum, wx, wy, (float)i / 32.0f);
        if (in_range(cand, mx)) return cand;
    }
    const V3 w = gamut_step(sp, x, y, lum, wx, wy, 1.0f);
    return v3(fmaxf(w.x, 0.0f), fmaxf(w.y, 0.0f), fmaxf(w.z, 0.0f));
}
// TransferFunction::encode (space.rs:54-75).
IX_DEV float transfer_encode(uint32_t sp, float lin) {
    if (sp <= IX_COLOR_SPACE_DISPLAY_P3) {
        if (lin <= 0.0031308f) return lin * 12.92f;
        return fmaf(1.055f, pow_disp(lin, 1.0f / 2.4f), -0.055f);
    }
    if (sp == IX_COLOR_SPACE_REC2020) {
        const float alpha = 1.0992968f, beta = 0.01805397f;
        if (lin < beta) return lin * 4.5f;
        return fmaf(alpha, pow_disp(lin, 0.45f), -(alpha - 1.0f));
    }
    return lin;
}
IX_DEV unsigned int encode_channel(uint32_t sp, float c) {
    const float lin = isfinite(c) ? clampf_(c, 0.0f, 1.0f) : 0.0f;
    const float enc = clampf_(transfer_encode(sp, lin), 0.0f, 1.0f);
    return __float2uint_rz(fmaf(enc, 255.0f, 0.5f));
}
// ColorSpace::encode with ToneMap::AcesFilmic { exposure: 1.0 } (space.rs:234-278) and
// aces_tonemap (optics/raytracer/color.rs:372) on the luminance.
IX_DEV uchar4 color_encode(V3 c, uint32_t sp) {
    const float sum = (c.x + c.y) + c.z;
    if (!isfinite(sum) || sum <= 1e-6f) return make_uchar4(0, 0, 0, 255);
    const float exposure = 1.0f;
    const float lum = fmaxf(c.y, 0.0f);
    const float exposed = fmaxf(lum * exposure, 0.0f);
    const float y_tm = (exposed * fmaf(2.51f, exposed, 0.03f)) / fmaf(exposed, fmaf(2.43f, exposed, 0.59f), 0.14f);
    const float scale = (y_tm / fmaxf(exposed, 1e-5f)) * exposure;
    const V3 rgb = project_to_gamut_bounded(c * scale, sp, 1.0f);
    return make_uchar4((unsigned char)encode_channel(sp, rgb.x), (unsigned char)encode_channel(sp, rgb.y),
                       (unsigned char)encode_channel(sp, rgb.z), 255);
}

// cos_pow (pass.rs:87) for the exponent the host resolved: 2^squarings by repeated
// squaring, or pow.
IX_DEV float cos_pow(float base, float power, int squarings) {
    if (squarings >= 0) {
        float v = base;
        for (int s = 0; s < squarings; ++s) v = v * v;
        return v;
    }
    return pow_disp(base, power);
}

// One output pixel of an A-Trous pass (atrous_pixel, pass.rs:330-378): the weights of
// tap_contribution (:283-316) in the reference's factor order, the taps row by row.
//
// Colour and depth travel together (float4 {x, y, z, sanitised depth}); the 5 taps of a
// row are loaded before any is used (coordinates clamped into the image, the mask says
// which count), so a thread keeps up to 15 loads in flight instead of one.  With
// FACET_NORMALS the guides' normal is a function of the facet id (the guide pass writes
// the plane normal), so a tap that passes the facet test has the centre's normal bit for
// bit and its normal weight is the centre's own, computed once: the tap needs no normal.
template <bool TONEMAP, bool FACET_NORMALS>
__global__ void __launch_bounds__(256) atrous_pass_kernel(PassLaunch L) {
    const int x = (int)(blockIdx.x * 32u + threadIdx.x);
    const int y = (int)(blockIdx.y * 8u + threadIdx.y);
    const int w = (int)L.width, h = (int)L.height;
    if (x >= w || y >= h) return;
    const size_t ci = (size_t)y * (size_t)w + (size_t)x;
    const float4 raw = L.src[ci];
    const V3 color = finite3(raw) ? v3(raw.x, raw.y, raw.z) : v3(0.0f, 0.0f, 0.0f);
    const float cdepth = raw.w;
    const int2 cf = L.fs[ci];
    V3 out = color;
    if (cf.x >= 0) {
        const float4 cn = L.nrm[ci];
        const bool c_zero = cn.x == 0.0f && cn.y == 0.0f && cn.z == 0.0f;
        float wn_self = 1.0f;
        if (FACET_NORMALS && !c_zero) {
            const float c = fmaxf(clampf_((cn.x * cn.x + cn.y * cn.y) + cn.z * cn.z, -1.0f, 1.0f), 0.0f);
            wn_self = cos_pow(c, L.normal_power, L.squarings);
        }
        V3 sum = v3(0.0f, 0.0f, 0.0f);
        float wsum = 0.0f;
#pragma unroll
        for (int ky = 0; ky < 5; ++ky) {
            const int sy = y + (ky - 2) * L.stride;
            if (sy < 0 || sy >= h) continue;
            const float hy = c_b3[ky];
            const size_t row = (size_t)sy * (size_t)w;
            int2 q[5];
            float4 t[5], qn[5];
            bool ok[5];
#pragma unroll
            for (int kx = 0; kx < 5; ++kx) {
                const int sx = x + (kx - 2) * L.stride;
                ok[kx] = sx >= 0 && sx < w;
                const size_t idx = row + (size_t)min(max(sx, 0), w - 1);
                q[kx] = L.fs[idx];
                t[kx] = L.src[idx];
                if (!FACET_NORMALS) qn[kx] = L.nrm[idx];
            }
#pragma unroll
            for (int kx = 0; kx < 5; ++kx) {
                // Facet identity, then the interior path signature (0 everywhere when
                // the frame has none): hard rejections.
                if (!ok[kx] || q[kx].x != cf.x || q[kx].y != cf.y) continue;
                if (!finite3(t[kx])) continue;
                float wn = 1.0f;
                if (FACET_NORMALS) {
                    wn = wn_self;
                } else if (!c_zero && !(qn[kx].x == 0.0f && qn[kx].y == 0.0f && qn[kx].z == 0.0f)) {
                    const float c = fmaxf(
                        clampf_((cn.x * qn[kx].x + cn.y * qn[kx].y) + cn.z * qn[kx].z, -1.0f, 1.0f), 0.0f);
                    wn = cos_pow(c, L.normal_power, L.squarings);
                }
                if (wn == 0.0f) continue;
                const float gap = fabsf(cdepth - t[kx].w);
                const float wd = gap == 0.0f ? 1.0f : exp_disp(gap * L.neg_inv_sigma_depth);
                const float dx = color.x - t[kx].x, dy = color.y - t[kx].y, dz = color.z - t[kx].z;
                const float dist_sq = (dx * dx + dy * dy) + dz * dz;
                const float wc = dist_sq == 0.0f ? 1.0f : exp_disp(dist_sq * L.neg_inv_two_sigma_color_sq);
                // kernel_w * wf * wn * wd * wc with the facet weight wf = 1.
                const float wgt = (((hy * c_b3[kx]) * wn) * wd) * wc;
                sum = v3(sum.x + t[kx].x * wgt, sum.y + t[kx].y * wgt, sum.z + t[kx].z * wgt);
                wsum = wsum + wgt;
            }
        }
        if (wsum > 1.0e-8f) out = v3(sum.x / wsum, sum.y / wsum, sum.z / wsum);
    }
    if (TONEMAP)
        L.rgba[ci] = color_encode(out * 1.0f, IX_COLOR_SPACE_SRGB);
    else
        L.dst[ci] = make_float4(out.x, out.y, out.z, cdepth);
}

__global__ void __launch_bounds__(256) tonemap_kernel(TonemapLaunch L) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < L.pixels;
         i += (uint64_t)gridDim.x * blockDim.x) {
        V3 c;
        if (L.xyz3) {
            c = v3(L.xyz3[3 * i], L.xyz3[3 * i + 1], L.xyz3[3 * i + 2]);
        } else {
            const float4 v = L.xyz4[i];
            c = v3(v.x, v.y, v.z);
        }
        L.rgba[i] = color_encode(c * L.scale, L.space);
    }
}

__global__ void __launch_bounds__(256) unpack_kernel(UnpackLaunch L) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < L.pixels;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float4 v = L.src[i];
        L.dst[3 * i] = v.x;
        L.dst[3 * i + 1] = v.y;
        L.dst[3 * i + 2] = v.z;
    }
}

#if IX_EXACT
// unit_normal_or_zero (pass.rs:67): sanitise, then n / |n|, or zero when |n| <= 1e-8.
IX_DEV V3 unit_normal_or_zero(V3 n) {
    n = v3(sanitize(n.x), sanitize(n.y), sanitize(n.z));
    const float len = __fsqrt_rn(dot(n, n));
    if (len <= 1.0e-8f) return v3(0.0f, 0.0f, 0.0f);
    return v3(__fdiv_rn(n.x, len), __fdiv_rn(n.y, len), __fdiv_rn(n.z, len));
}
// guide_pass.rs `unit`: v / |v| with an unfused dot.
IX_DEV V3 unit_div(V3 v) {
    const float len = __fsqrt_rn(dot(v, v));
    if (len > 0.0f) return v3(__fdiv_rn(v.x, len), __fdiv_rn(v.y, len), __fdiv_rn(v.z, len));
    return v;
}
IX_DEV uint32_t fnv_mix(uint32_t hash, uint32_t word) {
#pragma unroll
    for (int shift = 0; shift < 32; shift += 8) {
        hash ^= (word >> shift) & 0xFFu;
        hash *= 0x01000193u;
    }
    return hash;
}
// path_signature (guide_pass.rs:560-625): the un-jittered centre ray's entry refraction
// at n_d, then up to SIGNATURE_BOUNCES = 3 interior hits, TIR continuing the walk, the
// first exit ending it; FNV-1a over the facets met, 0 reserved for "no signature".
IX_DEV uint32_t path_signature(const float4* planes, int n, V3 origin0, V3 dir0, float t0, int facet0, V3 normal0,
                               float n_d) {
    const uint32_t SIG_EXIT_BIT = 0x8000u, SIG_ESCAPE = 0xFFFFu;
    if (isnan(n_d) || n_d <= 1.0f) return 0u;
    uint32_t hash = fnv_mix(0x811c9dc5u, (uint32_t)facet0);
    const V3 incident = unit_div(dir0);
    const float cos_i = fmaxf(-dot(incident, normal0), 0.0f);
    const float eta = __fdiv_rn(1.0f, n_d);
    const float k = 1.0f - eta * eta * (1.0f - cos_i * cos_i);
    if (k <= 0.0f) return max(fnv_mix(hash, SIG_ESCAPE), 1u);
    V3 dir = unit_div(incident * eta + normal0 * (eta * cos_i - __fsqrt_rn(k)));
    V3 origin = origin0 + dir0 * t0;
    for (int b = 0; b < 3; ++b) {
        const V3 po = origin + dir * 1.0e-4f;
        const Hit hit = intersect_planes(planes, n, po, dir);
        if (hit.facet < 0) {
            hash = fnv_mix(hash, SIG_ESCAPE);
            break;
        }
        origin = po + dir * hit.t;
        const float4 p = planes[hit.facet];
        const V3 hn = v3(p.x, p.y, p.z);
        const uint32_t facet = (uint32_t)hit.facet & 0x7FFFu;
        const float cos_t = dot(dir, hn);
        const float sin_sq = n_d * n_d * (1.0f - cos_t * cos_t);
        if (sin_sq > 1.0f) {
            hash = fnv_mix(hash, facet);
            dir = unit_div(dir - hn * (2.0f * cos_t));
        } else {
            hash = fnv_mix(hash, facet | SIG_EXIT_BIT);
            break;
        }
    }
    return max(hash, 1u);
}

// fill_rows (guide_pass.rs:640-690): one un-jittered camera ray per pixel, its first hit,
// and the signature; the planes staged in shared memory once per block.
__global__ void __launch_bounds__(128) guide_kernel(GuideLaunch L) {
    __shared__ float4 s_planes[IX_MAX_PLANES];
    const int n = (int)L.n_planes;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_planes[i] = L.planes[i];
    __syncthreads();
    const uint64_t pixels = (uint64_t)L.width * L.height;
    for (uint64_t pix = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; pix < pixels;
         pix += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = (uint32_t)(pix % L.width), y = (uint32_t)(pix / L.width);
        const Ray ray = generate_ray(L.camera, (float)x, (float)y, (float)L.width, (float)L.height, 0.0f, 0.0f);
        const Hit hit = intersect_planes(s_planes, n, ray.origin, ray.dir);
        float depth = 1.0e6f;
        V3 normal = v3(0.0f, 0.0f, 0.0f);
        int facet = -1;
        uint32_t sig = 0u;
        if (hit.facet >= 0) {
            const float4 p = s_planes[hit.facet];
            depth = hit.t;
            normal = v3(p.x, p.y, p.z);
            facet = hit.facet;
            sig = path_signature(s_planes, n, ray.origin, ray.dir, hit.t, facet, normal, L.n_d);
        }
        if (L.depth) L.depth[pix] = depth;
        if (L.normal) {
            L.normal[3 * pix] = normal.x;
            L.normal[3 * pix + 1] = normal.y;
            L.normal[3 * pix + 2] = normal.z;
        }
        if (L.facet) L.facet[pix] = facet;
        if (L.sig) L.sig[pix] = sig;
        if (L.nrm) {
            const V3 u = unit_normal_or_zero(normal);
            L.nrm[pix] = make_float4(u.x, u.y, u.z, sanitize(depth));
        }
        if (L.fs) L.fs[pix] = make_int2(facet, (int)sig);
    }
}

__global__ void __launch_bounds__(256) pack_kernel(PackLaunch L) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < L.pixels;
         i += (uint64_t)gridDim.x * blockDim.x) {
        float depth;
        if (L.depth) {
            // Guides in the reference layout -> unit normal (w: sanitised depth), (facet, sig).
            const V3 u = unit_normal_or_zero(v3(L.normal[3 * i], L.normal[3 * i + 1], L.normal[3 * i + 2]));
            depth = sanitize(L.depth[i]);
            L.nrm[i] = make_float4(u.x, u.y, u.z, depth);
            L.fs[i] = make_int2(L.facet[i], L.sig ? (int)L.sig[i] : 0);
        } else {
            depth = L.nrm[i].w;  // packed by the guide pass
        }
        if (L.color_out)
            L.color_out[i] = make_float4(L.color[3 * i] * L.scale, L.color[3 * i + 1] * L.scale,
                                         L.color[3 * i + 2] * L.scale, depth);
    }
}
#endif

unsigned int linear_blocks(uint64_t n) {
    const uint64_t b = (n + 255) / 256;
    return (unsigned int)(b < 1 ? 1 : (b > 65535ull * 8 ? 65535ull * 8 : b));
}

}  // namespace

cudaError_t IX_DISP_FN(launch_atrous_pass)(const PassLaunch& L, cudaStream_t s) {
    if (L.width == 0 || L.height == 0) return cudaSuccess;
    const dim3 block(32, 8), grid((L.width + 31) / 32, (L.height + 7) / 8);
    if (L.rgba) {
        if (L.facet_normals)
            atrous_pass_kernel<true, true><<<grid, block, 0, s>>>(L);
        else
            atrous_pass_kernel<true, false><<<grid, block, 0, s>>>(L);
    } else {
        if (L.facet_normals)
            atrous_pass_kernel<false, true><<<grid, block, 0, s>>>(L);
        else
            atrous_pass_kernel<false, false><<<grid, block, 0, s>>>(L);
    }
    return cudaGetLastError();
}
cudaError_t IX_DISP_FN(launch_tonemap)(const TonemapLaunch& L, cudaStream_t s) {
    if (L.pixels == 0) return cudaSuccess;
    tonemap_kernel<<<linear_blocks(L.pixels), 256, 0, s>>>(L);
    return cudaGetLastError();
}
cudaError_t IX_DISP_FN(launch_unpack)(const UnpackLaunch& L, cudaStream_t s) {
    if (L.pixels == 0) return cudaSuccess;
    unpack_kernel<<<linear_blocks(L.pixels), 256, 0, s>>>(L);
    return cudaGetLastError();
}
#if IX_EXACT
cudaError_t launch_guides_exact(const GuideLaunch& L, cudaStream_t s) {
    const uint64_t pixels = (uint64_t)L.width * L.height;
    if (pixels == 0) return cudaSuccess;
    if (L.n_planes > IX_MAX_PLANES) return cudaErrorInvalidValue;
    const uint64_t b = (pixels + 127) / 128;
    guide_kernel<<<(unsigned int)(b > 65535ull * 8 ? 65535ull * 8 : b), 128, 0, s>>>(L);
    return cudaGetLastError();
}
cudaError_t launch_pack_exact(const PackLaunch& L, cudaStream_t s) {
    if (L.pixels == 0) return cudaSuccess;
    pack_kernel<<<linear_blocks(L.pixels), 256, 0, s>>>(L);
    return cudaGetLastError();
}
#endif

}  // namespace disp
}  // namespace ix
