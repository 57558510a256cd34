// ix_transport.cuh -- one spectral path traced by an 8-lane group (sm_100a).
//
// GPU-first layout of the reference's per-sample estimator
// (optics/raytracer/transport/inner/bounce_body.rs:216-764): a path carries 8
// hero-wavelength channels, so a path is traced by 8 lanes of a warp, lane c holding
// channel c (its wavelength, index, absorption, Stokes vector, path pdf, exit-split
// radiance and MIS family mask).  What the reference computes once per path (the ray,
// the hero's decisions, the lighting direction) every lane of the group computes from
// identical inputs; what it loops over channels for, each lane does for its own channel.
// The slab intersection is split across the group (lane c scans planes c, c+8, ...) and
// reduced with shuffles to the first plane attaining the extremum, which is exactly the
// plane the reference's sequential scan keeps.  A warp holds 4 independent paths.
//
// Every group-level branch condition is computed from bit-identical inputs in the 8
// lanes, so a group never diverges internally and all shuffles use the group's mask.
#pragma once

#include "ix_device.cuh"
#include "ix_launch.h"
#include "ix_uniaxial.cuh"
#include "ix_biaxial.cuh"
#include "ix_tools.cuh"

namespace ix {

constexpr float DIRECTION_MATCH_COS_TOL = 1.0f - 1e-6f;  // refraction/mod.rs:137
constexpr float R_UNPOL_PDF_MIN = 1e-4f;                 // refraction/mod.rs:143
constexpr float R_UNPOL_PDF_MAX = 1.0f - 1e-4f;          // refraction/mod.rs:146
constexpr float R_UNPOL_SELECT_MIN = 0.02f;              // refraction/mod.rs:153
constexpr float R_UNPOL_SELECT_MAX = 0.98f;              // refraction/mod.rs:156

// Scene as the kernels see it: the host POD (in kernel parameter space) with `planes`
// pointing at device memory, plus per-scene flags resolved on the host.
struct DevScene {
    const ix_scene& s;
    uint32_t absorbing;   // the material has any absorption term
    uint32_t aniso;       // uniaxial birefringence
    uint32_t scattering;  // Henyey-Greenstein interior scattering (uniaxial instantiation)
    uint32_t rounded;     // rounded facet edges (uniaxial instantiation)
    uint32_t biaxial;     // biaxial indicatrix (extended instantiation)
    uint32_t concave;     // concave tools carve the stone (extended instantiation)
};
IX_DEV DevScene make_scene(const ix_scene& s, uint32_t flags) {
    return DevScene{s, (flags & SCENE_ABSORBING) ? 1u : 0u, (flags & SCENE_UNIAXIAL) ? 1u : 0u,
                    (flags & SCENE_SCATTERING) ? 1u : 0u, (flags & SCENE_ROUNDED) ? 1u : 0u,
                    (flags & SCENE_BIAXIAL) ? 1u : 0u, (flags & SCENE_CONCAVE) ? 1u : 0u};
}

// The 8 lanes of one path: `mask` selects them in the warp, `c` is this lane's channel.
struct Group {
    unsigned mask;
    int c;
};
IX_DEV Group make_group() {
    const int lane = (int)(threadIdx.x & 31u);
    return Group{0xFFu << (lane & ~7), lane & 7};
}
IX_DEV float gshfl(const Group& g, float v, int src) { return __shfl_sync(g.mask, v, src, 8); }
IX_DEV int gshfl(const Group& g, int v, int src) { return __shfl_sync(g.mask, v, src, 8); }
IX_DEV float gxor(const Group& g, float v, int m) { return __shfl_xor_sync(g.mask, v, m, 8); }
IX_DEV int gxor(const Group& g, int v, int m) { return __shfl_xor_sync(g.mask, v, m, 8); }

// Per-lane path state.  The first block is identical in the group's 8 lanes.
struct LanePath {
    uint32_t seed;
    uint32_t bounce;
    V3 o, d;
    V3 prev_pn;
    V3 observer;
    float n_hero;
    bool inside;
    bool has_prev;
    int facet;  // facet of the last facet event
    // channel c of the path
    float lambda;
    float n;
    float alpha;
    Stokes st;
    float pdf;
    float split;
    uint32_t compat;  // MIS family of this channel (refraction/context.rs:219)
    // Uniaxial transport only (the isotropic kernels never touch these).
    V3 k;              // wave normal; the ray direction `d` is the Poynting direction
    bool is_e;         // eigenmode assigned at the last entry or internal coupling
    float n_e;         // extraordinary_index_at for channel c; for a biaxial material the
                       // channel's beta-ray absorption (biaxial paths use no e index)
    float n_e_hero;    // channel 0's
    float alpha_e;     // e-ray (gamma-ray) absorption of channel c
    // Extended transport under the DaylightSun model only: the radiance next-event
    // estimation deposited so far, and the BSDF pdf of the last frosted light-sampled
    // bounce's continuation (pending_light_mis, bounce_body.rs:202), read by the next escape.
    float nee_rad;
    float carry_pdf;
    bool has_carry;
};

// ------------------------------------------------------------------------------------
// Cooperative slab intersection (simd/slab.rs:120-160; intersect.rs:101-127), with the
// division-free candidate filter of intersect_planes (ix_device.cuh).
//
// Two kinds of plane are passed over without a division; neither can change the hit the
// full scan returns:
//  * an entering plane (denom < 0) the origin is not outside of (side <= 0): its t <= 0.
//    If every entering plane is of this kind the scan's t_near stays <= 0, below both
//    the 1e-4 an entry needs and t_far (>= 0 unless the scan misses anyway); otherwise
//    the first plane with side > 0 takes t_near past every such t, and after it they
//    fail the filter.  So t_near, and near_idx whenever it is used, come out the same.
//  * an exiting plane (denom > 0) the origin is outside of (side > 0): the ray leaves
//    that half-space for good, the scan's t_far ends at most at this plane's negative t,
//    and it reports a miss -- returned at once, as for a parallel plane outside.
// ------------------------------------------------------------------------------------
// The scan itself: the entering planes' largest t and the first plane attaining it, the
// exiting planes' smallest t and its plane; false when the ray misses at once (a parallel
// plane or a receding plane the origin is outside of).
struct Slab {
    float t_near, t_far;
    int near_idx, far_idx;
};
IX_DEV bool group_slab(const Group& g, const float4* __restrict__ planes, int n, V3 o, V3 d, Slab& out) {
    float t_near = -1e30f, t_far = 1e30f;
    int near_idx = -1, far_idx = -1;
    int outside = 0;
    for (int i = g.c; i < n; i += 8) {
        float4 p = planes[i];
        float denom = (p.x * d.x + p.y * d.y) + p.z * d.z;
        float side = p.w + ((p.x * o.x + p.y * o.y) + p.z * o.z);
        if (fabsf(denom) > 1e-7f) {
            const bool entering = denom < 0.0f;
            if (!entering && side > 0.0f) {
                outside = 1;
                break;
            }
            // One division site for both kinds keeps the lanes of a group together.
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
            outside = 1;
            break;
        }
    }
    // Reduce to the first plane attaining the max t_near / min t_far (sequential-scan
    // semantics: a later plane replaces the running extremum only when strictly better).
#pragma unroll
    for (int m = 4; m > 0; m >>= 1) {
        float tn = gxor(g, t_near, m);
        int ni = gxor(g, near_idx, m);
        float tf = gxor(g, t_far, m);
        int fi = gxor(g, far_idx, m);
        outside |= gxor(g, outside, m);
        if (tn > t_near || (tn == t_near && ni >= 0 && (near_idx < 0 || ni < near_idx))) {
            t_near = tn;
            near_idx = ni;
        }
        if (tf < t_far || (tf == t_far && fi >= 0 && (far_idx < 0 || fi < far_idx))) {
            t_far = tf;
            far_idx = fi;
        }
    }
    out.t_near = t_near;
    out.t_far = t_far;
    out.near_idx = near_idx;
    out.far_idx = far_idx;
    return !outside;
}
IX_DEV Hit group_intersect(const Group& g, const float4* __restrict__ planes, int n, V3 o, V3 d) {
    Hit h;
    h.facet = -1;
    h.t = 0.0f;
    Slab s;
    if (!group_slab(g, planes, n, o, d, s) || s.t_near > s.t_far) return h;
    if (s.t_near > 1e-4f) {
        h.t = s.t_near;
        h.facet = s.near_idx >= 0 ? s.near_idx : 0;
    } else if (s.t_far > 1e-4f) {
        h.t = s.t_far;
        h.facet = s.far_idx >= 0 ? s.far_idx : 0;
    }
    return h;
}

// ------------------------------------------------------------------------------------
// A stone carved by concave tools (intersect_stone.rs:62-170, carve): the slab and every
// tool's interval are boundary events; walked in (t, event) order -- f32::total_cmp, then
// slab entry, slab exit, tool k's entry, tool k's exit -- the ray is in the material while
// it is inside the slab and inside no tool, and the hit is the first change of that state
// past the 1e-4 restart epsilon.  Lane c takes tools c, c + 8, ...; each step of the walk
// is the group's smallest event past the previous one.  Out of line and by value: only
// the extended instantiation calls it, and only for a carved stone.
// ------------------------------------------------------------------------------------
struct CarvedHit {
    float t;
    int facet;  // -1: a miss; tool k is facet n_planes + k
    V3 normal;  // the boundary's outward normal (a tool's points into the cavity)
    int entering;
};
// The event's 64-bit sort key: total_cmp's order of t (its bits, negatives' magnitude
// bits flipped, as an unsigned offset) above the event id.
IX_DEV unsigned long long event_key(float t, uint32_t id) {
    const int32_t b = __float_as_int(t);
    const uint32_t ord = (uint32_t)(b ^ (int32_t)(((uint32_t)(b >> 31)) >> 1)) ^ 0x80000000u;
    return ((unsigned long long)ord << 32) | id;
}
IX_DEV float event_t(unsigned long long key) {
    const int32_t ord = (int32_t)((uint32_t)(key >> 32) ^ 0x80000000u);
    return __int_as_float(ord ^ (int32_t)(((uint32_t)(ord >> 31)) >> 1));
}
static __device__ __noinline__ CarvedHit group_carved_hit(Group g, const float4* __restrict__ planes, int n_planes,
                                                          const ix_tool* __restrict__ tools, int n_tools, V3 o,
                                                          V3 d) {
    constexpr int PER_LANE = IX_MAX_TOOLS / 8;
    CarvedHit out{0.0f, -1, v3(0.0f, 0.0f, 0.0f), 0};
    Slab s;
    if (!group_slab(g, planes, n_planes, o, d, s) || s.t_near > s.t_far) return out;
    float lo[PER_LANE], hi[PER_LANE];
    uint32_t valid = 0;
#pragma unroll 1
    for (int i = 0; i < PER_LANE; ++i) {
        const int k = g.c + 8 * i;
        if (k < n_tools && tool_ray_interval(tools[k], o, d, lo[i], hi[i])) valid |= 1u << i;
    }
    unsigned long long prev = 0ull;
    bool first = true;
    int plane_depth = 0, tool_depth = 0;
    bool inside = false;
#pragma unroll 1
    for (int step = 0; step < 2 + 2 * IX_MAX_TOOLS; ++step) {
        unsigned long long best = ~0ull;
        auto consider = [&](float t, uint32_t id) {
            const unsigned long long e = event_key(t, id);
            if ((first || e > prev) && e < best) best = e;
        };
        if (g.c == 0) {
            consider(s.t_near, 0u);
            consider(s.t_far, 1u);
        }
#pragma unroll 1
        for (int i = 0; i < PER_LANE; ++i)
            if ((valid >> i) & 1u) {
                const uint32_t k = (uint32_t)(g.c + 8 * i);
                consider(lo[i], 2u + 2u * k);
                consider(hi[i], 3u + 2u * k);
            }
#pragma unroll
        for (int m = 4; m > 0; m >>= 1) {
            const unsigned long long other = __shfl_xor_sync(g.mask, best, m, 8);
            best = other < best ? other : best;
        }
        if (best == ~0ull) break;
        prev = best;
        first = false;
        const uint32_t id = (uint32_t)(best & 0xFFFFFFFFull);
        const float t = event_t(best);
        if (id == 0u)
            ++plane_depth;
        else if (id == 1u)
            --plane_depth;
        else if ((id & 1u) == 0u)
            ++tool_depth;
        else
            --tool_depth;
        const bool now_inside = plane_depth > 0 && tool_depth <= 0;
        if (now_inside == inside) continue;
        inside = now_inside;
        if (t <= 1e-4f) continue;
        out.t = t;
        out.entering = now_inside ? 1 : 0;
        if (id <= 1u) {
            const int idx = id == 0u ? s.near_idx : s.far_idx;
            out.facet = idx >= 0 ? idx : 0;
            out.normal = idx >= 0 ? v3(planes[idx].x, planes[idx].y, planes[idx].z) : v3(0.0f, 0.0f, 0.0f);
        } else {
            const int ti = (int)((id - 2u) >> 1);
            out.facet = n_planes + ti;
            out.normal = vneg_(tool_outward_normal(tools[ti], vadd_(o, vmul_(d, t))));
        }
        return out;
    }
    return out;
}
// shading_normal_for_hit's carved arm (transport/inner.rs:54): a tool facet keeps its
// normal, and a plane facet rounds its edges only where no tool lies within the rounding
// radius along the facet's frosted basis.
static __device__ __noinline__ int carved_near_tool(V3 hit_point, V3 normal, float radius,
                                                    const ix_tool* __restrict__ tools, int n_tools) {
    const V3 u = stable_basis_t_(normal), v = cross_(normal, u);
    const V3 dirs[4] = {u, vneg_(u), v, vneg_(v)};
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
        const V3 probe = vadd_(hit_point, vmul_(dirs[j], radius));
#pragma unroll 1
        for (int k = 0; k < n_tools; ++k)
            if (tool_contains(tools[k], probe)) return 1;
    }
    return 0;
}

// The exit-split probes' copy of the scan, out of line (probes are rare next to bounces).
static __device__ __noinline__ Hit probe_intersect(Group g, const float4* __restrict__ planes, int n, V3 o,
                                                   V3 d) {
    return group_intersect(g, planes, n, o, d);
}

// A ray that starts strictly outside the half-space of facet `f` and moves away from it
// meets no facet of the stone (an intersection of half-spaces): every point of the ray
// stays outside f.  The slab scan reports the same miss -- f's update leaves its t_far at
// most f's negative distance, below the 1e-4 every hit needs -- so a caller may skip the
// scan.  The 1e-6 margins keep the test inside the region where the scan's own rounding
// also sees |denom| > 1e-7 and side > 0.
IX_DEV bool leaves_stone_through(const float4* __restrict__ planes, int f, V3 o, V3 d) {
    const float4 p = planes[f];
    const float denom = (p.x * d.x + p.y * d.y) + p.z * d.z;
    const float side = p.w + ((p.x * o.x + p.y * o.y) + p.z * o.z);
    return denom > 1e-6f && side > 1e-6f;
}

// The bounce's intersection: after an exit (or an outside reflection) through facet
// P.facet the ray has left the stone and the scan is skipped.
IX_DEV Hit group_next_hit(const Group& g, const LanePath& P, const float4* __restrict__ planes, int n) {
    if (!P.inside && P.has_prev && leaves_stone_through(planes, P.facet, P.o, P.d)) {
        Hit h;
        h.facet = -1;
        h.t = 0.0f;
        return h;
    }
    return group_intersect(g, planes, n, P.o, P.d);
}

// rotate_stokes_to_plane_of_incidence (raytracer/absorption.rs:69): the new plane of
// incidence's normal normalize_or_zero(k x n); with a previous one, the channel's Stokes
// vector is rotated by the signed angle between the two planes about k.
IX_DEV V3 rotate_to_plane_of_incidence(Stokes& st, bool has_prev, V3 prev_pn, V3 k_hat, V3 normal) {
    // Uncontracted: at normal incidence k x n is exactly zero and the plane stays undefined
    // (no rotation), as on the CPU.
    const V3 cpn = normalize_or_zero(cross_rn(k_hat, normal));
    if (has_prev && length_squared(cpn) > 1e-6f && length_squared(prev_pn) > 1e-6f) {
        float cos_psi = clampf_(dot(prev_pn, cpn), -1.0f, 1.0f);
        float sin_psi = dot(cross(prev_pn, cpn), normalize_or_zero(k_hat));
        float s2, c2;
        rotation_2psi(sin_psi, cos_psi, c2, s2);
        st = rotate(st, c2, s2);
    }
    return cpn;
}

// ------------------------------------------------------------------------------------
// Path setup: PathState::new (bounce_body.rs:260-356).
// ------------------------------------------------------------------------------------
template <int UNI>
IX_DEV void group_init_ray(const Group& g, LanePath& P, const DevScene& S, Ray r, uint32_t seed,
                           float hero_rand) {
    const ix_scene& sc = S.s;
    P.seed = seed;
    P.bounce = 0;
    // wrapped_hero_wavelengths (transport/mod.rs:58): channel c of the comb.
    float lambda_hero = fmaf(hero_rand, 400.0f, 380.0f);
    float offset = fmaf((float)g.c, 50.0f, lambda_hero - 380.0f);
    P.lambda = 380.0f + rem_euclid_400(offset);
    P.n = dispersion_eval(sc.material.dispersion, P.lambda);
    P.n_hero = gshfl(g, P.n, 0);
    P.alpha = S.absorbing ? spectral_absorption(sc.material.abs_o, P.lambda) : 0.0f;
    P.st = Stokes{1.0f, 0.0f, 0.0f, 0.0f};
    P.pdf = 1.0f;
    P.split = 0.0f;
    P.compat = 0xFFu;
    P.o = r.origin;
    P.d = r.dir;
    P.observer = -r.dir;
    P.inside = false;
    P.has_prev = false;
    P.prev_pn = v3(0.0f, 0.0f, 0.0f);
    if constexpr (UNI) {
        P.k = r.dir;
        P.is_e = false;
        P.n_e = S.aniso ? extraordinary_index_at(sc.material, P.lambda, P.n) : P.n;
        P.n_e_hero = gshfl(g, P.n_e, 0);
        P.alpha_e = S.absorbing ? spectral_absorption(sc.material.abs_e, P.lambda) : 0.0f;
        if constexpr (UNI == TRANSPORT_EXTENDED) {
            P.nee_rad = 0.0f;
            P.carry_pdf = 0.0f;
            P.has_carry = false;
            if (S.biaxial)  // the beta-ray alpha; the alpha ray's without beta bands (wavelength_cache.rs:37-52)
                P.n_e = (S.absorbing && sc.material.has_abs_beta) ? spectral_absorption(sc.material.abs_beta, P.lambda)
                                                                  : P.alpha;
        }
    }
}

// One (pixel, absolute sample) as renderer/cpu_frame.rs:45-70 traces it.
template <int UNI>
IX_DEV void group_init(const Group& g, LanePath& P, const DevScene& S, uint32_t pixel,
                       uint32_t sample) {
    const ix_scene& sc = S.s;
    Draws dr = sample_draws(pixel, sample);
    uint32_t x = pixel % sc.width, y = pixel / sc.width;
    Ray r = generate_ray(sc.camera, (float)x, (float)y, (float)sc.width, (float)sc.height,
                         dr.jx, dr.jy);
    group_init_ray<UNI>(g, P, S, r, dr.seed, dr.hero);
}

// ------------------------------------------------------------------------------------
// Per-channel physics.
// ------------------------------------------------------------------------------------
// tir_phase_delta (refraction/tir.rs:33).
// IEEE square root and division in both builds: near the critical angle the radicand
// n^2 sin^2 - 1 cancels, and an approximate square root or quotient there moves the
// retarder by far more than its budget.
IX_DEV float tir_tan_half(float n1k, float cos_i, float sin_i) {
    return __fdiv_rn(cos_i * __fsqrt_rn(fmaxf(fmaf(n1k * n1k * sin_i, sin_i, -1.0f), 0.0f)),
                     fmaxf(n1k * sin_i * sin_i, 1e-6f));
}
IX_DEV float tir_phase_delta(float n1k, float cos_i, float sin_i) {
    // atan rounded to f32 from double, as a correctly rounding libm's atanf.
    return 2.0f * (float)atan((double)tir_tan_half(n1k, cos_i, sin_i));
}
// The channel's TIR retarder (tir.rs:98-116, polarization.rs:184).  The fast build forms
// cos(delta) and sin(delta) of delta = 2 atan(t) without a transcendental:
// cos = (1 - t^2) / (1 + t^2), sin = 2t / (1 + t^2).
IX_DEV Stokes tir_retard(const Stokes& s, float n1k, float cos_i, float sin_i) {
#if IX_EXACT
    return tir_retard_apply(s, tir_phase_delta(n1k, cos_i, sin_i));
#else
    const float t = tir_tan_half(n1k, cos_i, sin_i);
    const float inv = 1.0f / fmaf(t, t, 1.0f);
    const float cd = fmaf(-t, t, 1.0f) * inv;
    const float sd = (2.0f * t) * inv;
    return Stokes{s.i, s.q, cd * s.u + sd * s.v, (-sd) * s.u + cd * s.v};
#endif
}
IX_DEV void fresnel_rs_rp(float n1, float n2, float cos_i, float cos_t, float& r_s, float& r_p) {
    r_s = fmaf(n2, -cos_t, n1 * cos_i) / fmaf(n2, cos_t, n1 * cos_i);
    r_p = fmaf(n1, -cos_t, n2 * cos_i) / fmaf(n1, cos_t, n2 * cos_i);
}
IX_DEV float r_unpol_of(float r_s, float r_p) { return 0.5f * fmaf(r_p, r_p, r_s * r_s); }

// Beer-Lambert for an isotropic material (raytracer/absorption.rs:99, :197): the channel
// alpha is the midpoint of the absorption tensor's quadratic form over the two
// eigen-polarisations of the wave normal.
// The channel alpha of a non-birefringent material along wave normal k_hat (ao: its
// spectral alpha).
IX_DEV float iso_channel_alpha(const ix_material& m, float ao, V3 k_hat) {
    V3 raw_c = load3(m.c_axis);
    V3 c_axis = normalize_or_zero(raw_c);
    V3 ax = (fabsf(c_axis.x) > 0.9f) ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    V3 a1 = normalize_or_zero(ax - c_axis * dot(c_axis, ax));
    V3 a2 = cross(c_axis, a1);
    V3 cr = cross(k_hat, raw_c);
    V3 ea;
    if (length_squared(cr) > 1e-8f) {
        ea = normalize(cr);
    } else {
        V3 nk = normalize_or_zero(k_hat);
        V3 ax2 = (fabsf(nk.x) > 0.9f) ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
        ea = normalize_or_zero(ax2 - nk * dot(nk, ax2));
    }
    V3 eb = normalize_or_zero(cross(k_hat, ea));
    float la0 = dot(a1, ea), la1 = dot(a2, ea), la2 = dot(c_axis, ea);
    float lb0 = dot(a1, eb), lb1 = dot(a2, eb), lb2 = dot(c_axis, eb);
    float qa = (ao * (la0 * la0) + ao * (la1 * la1)) + ao * (la2 * la2);
    float qb = (ao * (lb0 * lb0) + ao * (lb1 * lb1)) + ao * (lb2 * lb2);
    return midpointf_(qa, qb);
}
IX_DEV void lane_absorption(LanePath& P, const DevScene& S, V3 k_hat, float len) {
    const ix_material& m = S.s.material;
    const float alpha = iso_channel_alpha(m, P.alpha, k_hat);
    P.st = scale(P.st, exp_lane(-alpha * (len * m.absorption_path_scale)));
}

// Escape radiance of channel c along `dir` (environment/rig.rs:18-49, :728).
// Out of line: it runs once per path (the escape) and per exit-split probe, so one copy
// of the lighting models keeps the bounce loop's instruction footprint small.
static __device__ __noinline__ float lane_environment(const ix_environment& env, V3 dir, V3 observer,
                                                     float lambda) {
    Lighting L = direction_lighting(env, dir, observer);
    return lighting_radiance(L, env, spectral_power(env, lambda));
}
// Every lighting model's escape radiance (environment_radiance_ext), out of line, for
// the extended instantiation only.
static __device__ __noinline__ float lane_environment_ext(const ix_environment& env, V3 dir, V3 observer,
                                                         float lambda) {
    return environment_radiance_ext(env, dir, observer, lambda);
}
template <int UNI>
IX_DEV float lane_env(const ix_environment& env, V3 dir, V3 observer, float lambda) {
    if constexpr (UNI == TRANSPORT_EXTENDED)
        return lane_environment_ext(env, dir, observer, lambda);
    else
        return lane_environment(env, dir, observer, lambda);
}

enum BounceResult { BOUNCE_CONTINUE = 0, BOUNCE_ESCAPED = 1, BOUNCE_KILLED = 2 };

// try_split_exit_channel (refraction/exit_split.rs:128): at an exit, each diverging live
// channel probes its own refracted direction `dir_k`; the group scans each probe
// together and the probing lane adds its transmitted intensity times the radiance found.
template <int UNI = TRANSPORT_ISOTROPIC>
IX_DEV void group_exit_probes(const Group& g, LanePath& P, const DevScene& S, const float4* __restrict__ planes,
                              V3 hit_point, bool want_probe, V3 dir_k, float t_intensity) {
    // A probe leaving through the exit facet itself cannot meet the stone: its channel
    // goes straight to the environment, every such lane at once.
    const bool clear = want_probe && leaves_stone_through(planes, P.facet, hit_point + dir_k * 1e-4f, dir_k);
    if (clear) {
        const float e = lane_env<UNI>(S.s.environment, dir_k, P.observer, P.lambda);
        P.split = fmaf(fmaxf(t_intensity, 0.0f), e, P.split);
    }
    unsigned probes = (__ballot_sync(g.mask, want_probe && !clear) >> (threadIdx.x & 24u)) & 0xFFu;
    while (probes) {
        const int j = __ffs(probes) - 1;
        probes &= probes - 1;
        const V3 dj = v3(gshfl(g, dir_k.x, j), gshfl(g, dir_k.y, j), gshfl(g, dir_k.z, j));
        const Hit ph = probe_intersect(g, planes, (int)S.s.n_planes, hit_point + dj * 1e-4f, dj);
        if (ph.facet < 0 && g.c == j) {
            const float e = lane_env<UNI>(S.s.environment, dj, P.observer, P.lambda);
            P.split = fmaf(fmaxf(t_intensity, 0.0f), e, P.split);
        }
    }
}

// The exit probes of a carved stone: no shortcut (a probe may meet the stone again across
// a cavity), each probe through the carved intersection (exit_split.rs:140).
IX_DEV void group_exit_probes_carved(const Group& g, LanePath& P, const DevScene& S, const float4* __restrict__ planes,
                                     V3 hit_point, bool want_probe, V3 dir_k, float t_intensity) {
    unsigned probes = (__ballot_sync(g.mask, want_probe) >> (threadIdx.x & 24u)) & 0xFFu;
    while (probes) {
        const int j = __ffs(probes) - 1;
        probes &= probes - 1;
        const V3 dj = v3(gshfl(g, dir_k.x, j), gshfl(g, dir_k.y, j), gshfl(g, dir_k.z, j));
        const CarvedHit ph = group_carved_hit(g, planes, (int)S.s.n_planes, S.s.tools, (int)S.s.n_tools,
                                              hit_point + dj * 1e-4f, dj);
        if (ph.facet < 0 && g.c == j) {
            const float e = lane_env<TRANSPORT_EXTENDED>(S.s.environment, dj, P.observer, P.lambda);
            P.split = fmaf(fmaxf(t_intensity, 0.0f), e, P.split);
        }
    }
}

// narrow_compat (refraction/context.rs:219) with the hero at channel 0: channel pairs
// whose directions differ leave each other's MIS family.  `status` is 0 for a channel
// with no transmitted direction, 1 when its direction matches the hero's, 2 otherwise.
// This 8-channel shuffle loop stays rolled (unrolling it measured 4 % slower: the loop
// body grows and instruction fetch is a leading stall); group_finish's two loops are
// unrolled (measured 8 % faster on the batch workload: their shuffles issue ahead of the
// dependent adds).
IX_DEV void group_narrow_compat(const Group& g, LanePath& P, int status, V3 dir_k) {
#pragma unroll 1
    for (int j = 0; j < 8; ++j) {
        const float dx = gshfl(g, dir_k.x, j), dy = gshfl(g, dir_k.y, j), dz = gshfl(g, dir_k.z, j);
        const int sj = gshfl(g, status, j);
        if (j == g.c) continue;
        bool m;
        if (g.c == 0)
            m = sj == 1;
        else if (j == 0)
            m = status == 1;
        else if (status != 0 && sj != 0)
            m = dot(dir_k, v3(dx, dy, dz)) >= DIRECTION_MATCH_COS_TOL;
        else
            m = true;
        if (!m) P.compat &= ~(1u << j);
    }
}

// The channel's scalar-Fresnel reflection (apply_tir_bounce's isotropic arm,
// refraction/tir.rs:98-116, and apply_partial_reflect_bounce, reflect_refract.rs:33):
// the TIR retarder past the channel's own critical angle, else the Fresnel reflection
// with its reflectance folded into the channel pdf.
IX_DEV Stokes lane_scalar_reflect(LanePath& P, float n1k, float n2k, float s2k, float cos_i, float sin_i) {
    if (s2k > 1.0f) return tir_retard(P.st, n1k, cos_i, sin_i);
    const float cos_t_k = __fsqrt_rn(fmaxf(1.0f - s2k, 0.0f));
    float rs, rp;
    fresnel_rs_rp(n1k, n2k, cos_i, cos_t_k, rs, rp);
    P.pdf = P.pdf * clampf_(r_unpol_of(rs, rp), R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
    return fresnel_reflect_apply(P.st, rs, rp);
}

// ------------------------------------------------------------------------------------
// Frosted (bruted) facets: apply_frosted_bounce (optics/raytracer/scattering/frosted.rs:289).
// Next-event estimation, which the reference enables for an HDR map or the DaylightSun
// model (environment_supports_nee, environment/nee.rs:60), runs under DaylightSun in the
// extended transport instantiation (frosted_sun_nee below); HDR maps are not carried.
// ------------------------------------------------------------------------------------
constexpr uint32_t FROSTED_DIR_U_STREAM = 0x27D4EB2Fu;  // sampling.rs:24
constexpr uint32_t FROSTED_DIR_V_STREAM = 0x165667B1u;  // sampling.rs:25

// facet_finish_for (bounce_body.rs:656): Polished past the end of the finish list.
IX_DEV bool facet_frosted(const DevScene& S, int f) {
    return S.s.facet_finishes && (uint32_t)f < S.s.n_finishes && S.s.facet_finishes[f] != 0;
}
// cosine_weighted_hemisphere (frosted.rs:34) on frosted_orthonormal_basis
// (scattering/mod.rs:110): the angle is (2 pi) u2, the three scaled basis vectors are
// summed left to right.
IX_DEV V3 cosine_weighted_hemisphere(float u1, float u2, V3 n) {
    const float r = sqrtf(u1);
    const float theta = (2.0f * 3.14159265358979323846f) * u2;
    float sin_t, cos_t;
    sincosf(theta, &sin_t, &cos_t);
    const V3 a = fabsf(n.x) > 0.9f ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    const V3 t = normalize_or_zero(a - n * dot(n, a));
    const V3 b = cross(n, t);
    return normalize_or_zero((t * (r * cos_t) + b * (r * sin_t)) + n * sqrtf(fmaxf(1.0f - u1, 0.0f)));
}
// The frosted bounce of one channel: a cosine-weighted diffuse reflection or
// transmission, chosen by the hero's unpolarised Fresnel reflectance (n1, n2, cos_i,
// sin2_t are the hero's geometry, identical in the 8 lanes), always reflection past the
// hero's critical angle.  Returns the new direction (the same in every lane), the factor
// the channel's path pdf takes (the chosen branch's probability) and whether the ray
// crossed the facet; the caller depolarises the channel.  Out of line and by value, so
// the polished bounce around the call compiles exactly as it does without it (the fast
// build's multiply-add contraction, and with it every sum, stays the same in every
// kernel that inlines the bounce).
struct FrostedScatter {
    V3 dir;
    float pdf_factor;
    int transmit;
};
static __device__ __noinline__ FrostedScatter frosted_scatter(uint32_t seed, uint32_t bounce, V3 normal, float n1,
                                                       float n2, float cos_i, float sin2_t) {
    const float u1 = unit_draw(seed, bounce, FROSTED_DIR_U_STREAM);
    const float u2 = unit_draw(seed, bounce, FROSTED_DIR_V_STREAM);
    FrostedScatter out{v3(0.0f, 0.0f, 0.0f), 1.0f, 0};
    if (!(sin2_t > 1.0f)) {
        const float cos_t = sqrtf(fmaxf(1.0f - sin2_t, 0.0f));
        float r_s, r_p;
        fresnel_rs_rp(n1, n2, cos_i, cos_t, r_s, r_p);
        const float r_unpol = clampf_(r_unpol_of(r_s, r_p), R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
        out.transmit = unit_draw(seed, bounce, FRESNEL_BRANCH_STREAM) < r_unpol ? 0 : 1;
        out.pdf_factor = out.transmit ? 1.0f - r_unpol : r_unpol;
    }
    out.dir = cosine_weighted_hemisphere(u1, u2, out.transmit ? -normal : normal);
    return out;
}
// Applies a frosted scatter's pdf factor and depolarisation to this channel.
IX_DEV void lane_frosted_apply(LanePath& P, const FrostedScatter& f) {
    P.pdf = P.pdf * f.pdf_factor;
    P.st = Stokes{intensity(P.st), 0.0f, 0.0f, 0.0f};
}

// nee_contribution_frosted_exterior (scattering/frosted.rs:98) under DaylightSun: one
// direction drawn uniformly over the sun's disc (sun_cone_direction, environment/sun.rs:70,
// with 1 - cos kept exact), rejected behind the facet and, on a carved stone, when a shadow
// probe from 1e-4 along it meets the stone; weighted by the balance heuristic against the
// Lambertian cos / pi density the diffuse draw has there.  Returns the channel's deposit,
// (I * common) * (sun factor * (spd * exposure)), or 0.  The 8 lanes share the direction
// and every decision (the hit point, normal and draws are the path's), so the group enters
// the shadow probe together.  Out of line: the extended instantiation's frosted arms only.
constexpr uint32_t FROSTED_NEE_ENV_DIR_U_STREAM = 0x6A09E667u;  // sampling.rs:52
constexpr uint32_t FROSTED_NEE_ENV_DIR_V_STREAM = 0xBB67AE85u;  // sampling.rs:53
constexpr float SUN_ONE_MINUS_COS = 1.1086464e-5f;              // 186 x 2^-24, sun.rs:55
constexpr float SUN_SOLID_ANGLE = 6.965831e-5f;                 // 2 pi x SUN_ONE_MINUS_COS, sun.rs:57
IX_DEV V3 sun_cone_direction(V3 key, float u0, float u1) {
    const float one_minus_cos = u0 * SUN_ONE_MINUS_COS;
    const float cos_t = 1.0f - one_minus_cos;
    const float sin_t = sqrtf(fmaxf(one_minus_cos * (2.0f - one_minus_cos), 0.0f));
    float sin_p, cos_p;
    sincosf((2.0f * 3.14159265358979323846f) * u1, &sin_p, &cos_p);
    const V3 a = fabsf(key.x) > 0.9f ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    const V3 t = normalize_or_zero(a - key * dot(key, a));
    const V3 b = cross(key, t);
    return normalize_or_zero((t * (sin_t * cos_p) + b * (sin_t * sin_p)) + key * cos_t);
}
// balance_heuristic (scattering/mod.rs:102).
IX_DEV float balance_heuristic(float a, float b) {
    const float denom = a + b;
    return denom > 1e-12f ? a / denom : 0.0f;
}
// environment_nee_pdf (environment/nee.rs:144) for the sun: uniform over its disc.
IX_DEV float sun_nee_pdf(const ix_environment& env, V3 dir) {
    return dot(dir, load3(env.key_dir)) >= SUN_DISC_COS ? 1.0f / SUN_SOLID_ANGLE : 0.0f;
}
static __device__ __noinline__ float frosted_sun_nee(Group g, DevScene S, const float4* __restrict__ planes,
                                                     uint32_t seed, uint32_t bounce, V3 origin, V3 ext_normal,
                                                     float lambda, float intensity_now) {
    const ix_environment& env = S.s.environment;
    const float u0 = unit_draw(seed, bounce, FROSTED_NEE_ENV_DIR_U_STREAM);
    const float u1 = unit_draw(seed, bounce, FROSTED_NEE_ENV_DIR_V_STREAM);
    const V3 dir = sun_cone_direction(load3(env.key_dir), u0, u1);
    const float pdf = 1.0f / SUN_SOLID_ANGLE;
    const float cos_light = dot(dir, ext_normal);
    if (cos_light <= 0.0f) return 0.0f;
    if (S.concave) {
        const CarvedHit h = group_carved_hit(g, planes, (int)S.s.n_planes, S.s.tools, (int)S.s.n_tools,
                                             origin + dir * 1e-4f, dir);
        if (h.facet >= 0) return 0.0f;
    }
    const float brdf_pdf = cos_light / 3.14159265358979323846f;
    const float mis = balance_heuristic(pdf, brdf_pdf);
    if (mis <= 0.0f) return 0.0f;
    const float common = (brdf_pdf * mis) / pdf;
    const float env_k = env.sun_factor * (spectral_power_ext(env, lambda) * env.exposure);
    return (intensity_now * common) * env_k;
}
// The exterior-side frosted events (the reflect of an outside hit, the transmit of an
// inside one; apply_frosted_bounce's NEE eligibility) under DaylightSun: the deposit and
// the carry the next escape weighs itself with.  `normal` faces the incident side.
IX_DEV void frosted_exterior_event(const Group& g, LanePath& P, const DevScene& S, const float4* __restrict__ planes,
                                   const FrostedScatter& f, bool inside0, V3 normal, V3 hit_point, uint32_t bounce) {
    if (S.s.environment.model != IX_ENV_DAYLIGHT_SUN || (f.transmit ? !inside0 : inside0)) return;
    const V3 ext_normal = f.transmit ? -normal : normal;
    P.nee_rad = frosted_sun_nee(g, S, planes, P.seed, bounce, hit_point, ext_normal, P.lambda, intensity(P.st)) +
                P.nee_rad;
    P.has_carry = true;
    P.carry_pdf = dot(f.dir, ext_normal) / 3.14159265358979323846f;
}
// The escape of the extended instantiation: the carried balance weight against the sun's
// light samples (handle_miss, bounce_body/miss.rs:40), folded onto the deposits so far.
IX_DEV float escape_with_carry(const LanePath& P, const ix_environment& env, float radiance) {
    const float mis = P.has_carry ? balance_heuristic(P.carry_pdf, sun_nee_pdf(env, P.d)) : 1.0f;
    return fmaf(intensity(P.st) * mis, radiance, P.nee_rad);
}

// ------------------------------------------------------------------------------------
// shading_normal_near_edge (optics/raytracer/intersect.rs:196): within
// `edge_rounding_radius` of another facet's plane the shading normal blends, by a
// smoothstep of the distance, toward the bisector with the nearest plane.  The 8 lanes of
// the group scan the planes together; the nearest is the first of the minimal distance,
// as the reference's strict `<` keeps.  Out of line: rounded stones only.
// ------------------------------------------------------------------------------------
static __device__ __noinline__ V3 group_shading_normal(Group g, const float4* __restrict__ planes, int n, V3 x,
                                                       int facet, V3 hit_normal, float radius) {
    float best = INFINITY;
    int best_i = 0x7FFFFFFF;
    for (int i = g.c; i < n; i += 8) {
        if (i == facet) continue;
        const float4 p = planes[i];
        const float dist = -(p.w + ((p.x * x.x + p.y * x.y) + p.z * x.z));
        if (dist < best) {
            best = dist;
            best_i = i;
        }
    }
#pragma unroll
    for (int m = 4; m > 0; m >>= 1) {
        const float ob = gxor(g, best, m);
        const int oi = gxor(g, best_i, m);
        if (ob < best || (ob == best && oi < best_i)) {
            best = ob;
            best_i = oi;
        }
    }
    if (!(best < radius) || best_i == 0x7FFFFFFF) return hit_normal;
    const float4 q = planes[best_i];
    const V3 nearest = v3(q.x, q.y, q.z);
    const float t = clampf_(1.0f - best / radius, 0.0f, 1.0f);
    const float smooth_t = t * t * fmaf(2.0f, -t, 3.0f);
    const V3 bis = normalize_or_zero(hit_normal + nearest);
    return normalize_or_zero(hit_normal * (1.0f - smooth_t) + bis * smooth_t);
}

// ------------------------------------------------------------------------------------
// Henyey-Greenstein interior scattering: try_scatter_step (scattering/hg.rs:256-340) with
// maybe_scatter_or_extinguish (:21-84) and sample_henyey_greenstein_direction (:390),
// without next-event estimation (no light-sampling technique in the modelled
// environments) or zoning.  Runs in the uniaxial instantiation of the transport (which
// also traces isotropic materials), so the isotropic one carries none of it.
// ------------------------------------------------------------------------------------
constexpr uint32_t DISTANCE_SAMPLE_STREAM = 0xA24BAED4u;  // sampling.rs:28
constexpr uint32_t PHASE_DIR_U_STREAM = 0x9FB21C65u;      // sampling.rs:31
constexpr uint32_t PHASE_DIR_V_STREAM = 0x1CE4E5B9u;      // sampling.rs:32
IX_DEV float log_scatter(float x) {
#if IX_EXACT
    return (float)log((double)x);
#else
    return logf(x);
#endif
}
struct ScatterResult {
    float st_factor;  // scattered: the channel's new (unpolarised) intensity; else survival ratio
    float pdf_factor;
    V3 dir;           // scattered: the HG direction about the old one
    float t_model;    // scattered: distance to the event in model units
    int scattered;
};
// One channel of the segment's free-flight draw (the hero's extinction decides, through
// lane 0 of the group; every lane takes the same branch).  Out of line and by value, like
// frosted_scatter, so the bounce around the call compiles as it does without it; one copy
// per transport instantiation (UNI), so the extended one's callers leave the uniaxial
// kernels' copy, and its register allocation, alone.
template <int UNI>
static __device__ __noinline__ ScatterResult scatter_or_survive(Group g, uint32_t seed, uint32_t bounce, float alpha,
                                                                float sigma_s_model, float path_scale, float g_hg,
                                                                float hit_t, float intensity_now, V3 forward) {
    ScatterResult r;
    const float sigma_s = sigma_s_model / path_scale;
    const float sigma_t = alpha + sigma_s;
    const float sigma_t_hero = gshfl(g, sigma_t, 0);
    const float dist_rand = unit_draw(seed, bounce, DISTANCE_SAMPLE_STREAM);
    const float one_minus_u = fmaxf(1.0f - dist_rand, 1e-7f);
    const float t_free = -log_scatter(one_minus_u) / sigma_t_hero;
    const float hit_scaled = hit_t * path_scale;
    if (t_free < hit_scaled) {
        const float pdf_hero = sigma_t_hero * one_minus_u;
        const float tr = exp_lane(-sigma_t * t_free);
        r.st_factor = intensity_now * (tr * sigma_s / pdf_hero);
        r.pdf_factor = sigma_t * tr;
        // sample_henyey_greenstein_direction: cos theta from u1, the azimuth (2 pi) u2
        // about the old direction in frosted_orthonormal_basis.
        const float u1 = unit_draw(seed, bounce, PHASE_DIR_U_STREAM);
        const float u2 = unit_draw(seed, bounce, PHASE_DIR_V_STREAM);
        float cos_theta;
        if (fabsf(g_hg) < 1e-3f) {
            cos_theta = fmaf(2.0f, -u1, 1.0f);
        } else {
            const float one_minus_g2 = fmaf(g_hg, -g_hg, 1.0f);
            const float denom = fmaf(2.0f * g_hg, u1, 1.0f - g_hg);
            const float sq = one_minus_g2 / denom;
            cos_theta = fmaf(sq, -sq, fmaf(g_hg, g_hg, 1.0f)) / (2.0f * g_hg);
        }
        cos_theta = clampf_(cos_theta, -1.0f, 1.0f);
        const float sin_theta = sqrtf(fmaxf(fmaf(cos_theta, -cos_theta, 1.0f), 0.0f));
        float sin_p, cos_p;
        sincosf((2.0f * 3.14159265358979323846f) * u2, &sin_p, &cos_p);
        const V3 a = fabsf(forward.x) > 0.9f ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
        const V3 t = normalize_or_zero(a - forward * dot(forward, a));
        const V3 b = cross(forward, t);
        r.dir = normalize_or_zero((t * (sin_theta * cos_p) + b * (sin_theta * sin_p)) + forward * cos_theta);
        r.t_model = t_free / path_scale;
        r.scattered = 1;
        return r;
    }
    const float survive = exp_lane(-sigma_t * hit_scaled);
    const float survive_hero = gshfl(g, survive, 0);
    r.st_factor = survive / fmaxf(survive_hero, 1e-30f);
    r.pdf_factor = survive;
    r.dir = forward;
    r.t_model = 0.0f;
    r.scattered = 0;
    return r;
}

// One iteration of the bounce loop (bounce_body.rs:361-423 and facet_event :611-707).
// On BOUNCE_ESCAPED `esc` is this channel's escape radiance already weighted by its
// Stokes intensity (accumulate_miss_radiance, transport/bounce.rs:40).
// The isotropic bounce in three phases, which the megakernel runs back to back and the
// wavefront pipeline (ix_wavefront.cu) runs in separate kernels with the path state in
// HBM between them:
//   bounce_hit       the intersection; at a facet, the Stokes frame rotation and the
//                    interior segment's absorption (the path state's only changes);
//   bounce_geometry  the facet's refraction geometry and the dispatch decision (frosted,
//                    reflect, refract) -- a pure function of the path state and t, so the
//                    wavefront recomputes it after the state's round trip through HBM;
//   bounce_arm       the chosen arm, the new ray, surface glare and roulette.
struct BounceGeom {
    V3 normal, hit_point, k_hat;
    float cos_i, one_m_c2, sin_i, n1, n2, eta, sin2_t, n1k, n2k, r_unpol;
    bool tir, reflect, frosted;
    // the channel's own Snell geometry and Fresnel amplitudes at its index
    float ratio, s2k, cos_t_k, rs, rp, r_k;
    bool lane_tir;
};

// Returns BOUNCE_ESCAPED (esc set) or BOUNCE_CONTINUE with P.facet the hit facet and `t`
// its distance.
IX_DEV int bounce_hit(const Group& g, LanePath& P, const DevScene& S, const float4* __restrict__ planes, float& esc,
                      float& t) {
    const ix_scene& sc = S.s;
    Hit hit = group_next_hit(g, P, planes, (int)sc.n_planes);
    if (hit.facet < 0) {
        esc = fmaf(intensity(P.st), lane_environment(sc.environment, P.d, P.observer, P.lambda), 0.0f);
        return BOUNCE_ESCAPED;
    }
    P.facet = hit.facet;
    t = hit.t;
    const float4 pl = planes[hit.facet];
    const V3 normal = v3(pl.x, pl.y, pl.z);
    const V3 k_hat = P.d;  // isotropic: wave normal == ray direction
    const V3 cpn = rotate_to_plane_of_incidence(P.st, P.has_prev, P.prev_pn, k_hat, normal);
    P.has_prev = true;
    P.prev_pn = cpn;
    // apply_interior_segment (transport/inner.rs:170).
    if (P.inside && S.absorbing) lane_absorption(P, S, k_hat, hit.t);
    return BOUNCE_CONTINUE;
}

IX_DEV void bounce_geometry(const LanePath& P, const DevScene& S, const float4* __restrict__ planes, float t,
                            BounceGeom& G) {
    const float4 pl = planes[P.facet];
    G.k_hat = P.d;
    G.hit_point = P.o + t * P.d;
    G.normal = P.inside ? -v3(pl.x, pl.y, pl.z) : v3(pl.x, pl.y, pl.z);
    // compute_bounce_refraction_geometry (refraction/geometry.rs:306), isotropic.
    G.cos_i = clampf_(dot(-G.k_hat, G.normal), 0.0f, 1.0f);
    G.one_m_c2 = fmaf(G.cos_i, -G.cos_i, 1.0f);
    G.sin_i = __fsqrt_rn(fmaxf(G.one_m_c2, 0.0f));  // IEEE: the TIR retarder is ill-conditioned in it
    G.n1 = P.inside ? P.n_hero : 1.0f;
    G.n2 = P.inside ? 1.0f : P.n_hero;
    G.eta = __fdiv_rn(G.n1, G.n2);  // IEEE: it decides TIR and the hero's direction
    G.sin2_t = G.eta * G.eta * G.one_m_c2;
    G.n1k = P.inside ? P.n : 1.0f;
    G.n2k = P.inside ? 1.0f : P.n;
    // dispatch_bounce (transport/bounce.rs:108): a frosted facet scatters diffusely;
    // otherwise the hero decides TIR (sin2_t > 1), else apply_partial_fresnel_bounce
    // (refraction/dispatch.rs:307) draws reflect vs refract.
    G.tir = G.sin2_t > 1.0f;
    G.r_unpol = 1.0f;
    G.reflect = G.tir;
    if (!G.tir) {
        float cos_t = sqrtf(fmaxf(1.0f - G.sin2_t, 0.0f));
        float r_s, r_p;
        fresnel_rs_rp(G.n1, G.n2, G.cos_i, cos_t, r_s, r_p);
        G.r_unpol = clampf_(r_unpol_of(r_s, r_p), R_UNPOL_SELECT_MIN, R_UNPOL_SELECT_MAX);
        G.reflect = unit_draw(P.seed, P.bounce, FRESNEL_BRANCH_STREAM) < G.r_unpol;
    }
    G.frosted = facet_frosted(S, P.facet);
    // The channel's own Snell geometry and Fresnel amplitudes at its index, which the
    // reflect and refract arms both use: formed once here, before the arms split the
    // warp's groups, instead of once in each arm.
    G.ratio = __fdiv_rn(G.n1k, G.n2k);
    G.s2k = (G.ratio * G.ratio) * G.one_m_c2;
    G.lane_tir = G.s2k > 1.0f;
    G.cos_t_k = G.lane_tir ? 0.0f : __fsqrt_rn(fmaxf(1.0f - G.s2k, 0.0f));
    G.rs = 1.0f;
    G.rp = 1.0f;
    if (!G.lane_tir) fresnel_rs_rp(G.n1k, G.n2k, G.cos_i, G.cos_t_k, G.rs, G.rp);
    G.r_k = clampf_(r_unpol_of(G.rs, G.rp), R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
}

// Returns BOUNCE_CONTINUE or BOUNCE_KILLED (roulette).
IX_DEV int bounce_arm(const Group& g, LanePath& P, const DevScene& S, const float4* __restrict__ planes,
                      const BounceGeom& G) {
    const uint32_t bounce = P.bounce;
    V3 new_dir;
    bool new_inside = P.inside;
    if (G.frosted) {
        const FrostedScatter f = frosted_scatter(P.seed, bounce, G.normal, G.n1, G.n2, G.cos_i, G.sin2_t);
        lane_frosted_apply(P, f);
        new_dir = f.dir;
        if (f.transmit) new_inside = !P.inside;
    } else if (G.reflect) {
        // apply_tir_bounce (tir.rs:98-116) / apply_partial_reflect_bounce
        // (reflect_refract.rs:33): the channel's TIR retarder or Fresnel reflection; a
        // partial reflection divides by the selection probability (TIR scales by 1).
        Stokes s;
        if (G.lane_tir) {
            s = tir_retard(P.st, G.n1k, G.cos_i, G.sin_i);
        } else {
            s = fresnel_reflect_apply(P.st, G.rs, G.rp);
            P.pdf = P.pdf * G.r_k;
        }
        P.st = scale(s, G.tir ? 1.0f : 1.0f / G.r_unpol);
        new_dir = G.k_hat - 2.0f * dot(G.k_hat, G.normal) * G.normal;
    } else {
        // apply_refract_bounce (reflect_refract.rs:121): the hero's direction, then each
        // channel's own Snell direction, transmission and direction match
        // (apply_refract_channel :517, compute_channel_refraction_geometry :255).
        const float sin2_t_dir = fminf(G.eta * G.eta * G.one_m_c2, 1.0f);
        // The directions entering the match test take IEEE divide / sqrt (normalize_dir).
        const float cos_t_dir = __fsqrt_rn(fmaxf(1.0f - sin2_t_dir, 0.0f));
        const V3 final_refr = normalize_dir(G.eta * G.k_hat + fmaf(G.eta, G.cos_i, -cos_t_dir) * G.normal);
        int status = 0;  // 0 channel TIR, 1 direction matches the hero, 2 diverges
        V3 dir_k = v3(0.0f, 0.0f, 0.0f);
        float t_intensity = 0.0f;
        const Stokes original = P.st;
        if (G.lane_tir) {
            P.st = scale(P.st, 0.0f);
            P.pdf = 0.0f;
        } else {
            dir_k = normalize_dir(G.ratio * G.k_hat + fmaf(G.ratio, G.cos_i, -G.cos_t_k) * G.normal);
            status = dot(dir_k, final_refr) >= DIRECTION_MATCH_COS_TOL ? 1 : 2;
            const float two = 2.0f * G.n1k * G.cos_i;
            const float t_s = two / fmaf(G.n2k, G.cos_t_k, G.n1k * G.cos_i);
            const float t_p = two / fmaf(G.n1k, G.cos_t_k, G.n2k * G.cos_i);
            const Stokes transmitted =
                scale(fresnel_transmit_apply(original, G.n1k, G.n2k, G.cos_i, G.cos_t_k, t_s, t_p),
                      1.0f / (1.0f - G.r_unpol));
            P.pdf = P.pdf * (1.0f - G.r_k);
            // apply_channel_chromatic_termination (reflect_refract.rs:444): a diverging
            // channel's radiance is zeroed (its pdf keeps accumulating).
            P.st = status == 1 ? transmitted : scale(original, 0.0f);
            t_intensity = intensity(transmitted);
        }
        group_exit_probes(g, P, S, planes, G.hit_point, status == 2 && P.inside && intensity(original) > 0.0f,
                          dir_k, t_intensity);
        if (!P.inside) group_narrow_compat(g, P, status, dir_k);
        new_dir = final_refr;
        new_inside = !P.inside;
    }
    P.d = new_dir;
    P.o = G.hit_point + new_dir * 1e-4f;
    P.inside = new_inside;

    // Surface glare (bounce_body.rs:691-697): the outside reflection of a polished facet.
    const float glare = clampf_(S.s.environment.surface_glare, 0.0f, 1.0f);
    if (bounce == 0 && !P.inside && glare < 1.0f && !G.frosted) P.st = scale(P.st, glare);
    // apply_russian_roulette (transport/bounce.rs:355): q from the brightest channel.
    if (bounce > 4) {
        float max_i = intensity(P.st);
#pragma unroll
        for (int m = 4; m > 0; m >>= 1) max_i = fmaxf(max_i, gxor(g, max_i, m));
        const float q = clampf_(fmaxf(0.0f, max_i), 0.05f, 1.0f);
        if (unit_draw(P.seed, bounce, RUSSIAN_ROULETTE_STREAM) > q) return BOUNCE_KILLED;
        P.st = scale(P.st, 1.0f / q);
        P.split = P.split / q;
    }
    P.bounce = bounce + 1;
    return BOUNCE_CONTINUE;
}

IX_DEV int group_bounce(const Group& g, LanePath& P, const DevScene& S,
                        const float4* __restrict__ planes, float& esc) {
    float t = 0.0f;
    if (bounce_hit(g, P, S, planes, esc, t) == BOUNCE_ESCAPED) return BOUNCE_ESCAPED;
    BounceGeom G;
    bounce_geometry(P, S, planes, t, G);
    return bounce_arm(g, P, S, planes, G);
}

// ------------------------------------------------------------------------------------
// The bounce of the uniaxial transport instantiation: an isotropic material, a
// pleochroic one, or a uniaxial crystal (transport/bounce.rs:108-160,
// refraction/dispatch.rs:67-380, uniaxial_entry.rs, uniaxial_internal.rs, tir.rs:41).
// Group-level decisions come from the hero (lane 0): its closed-form solve sets the
// reflect probability and the eigenmode draw; every lane solves its own channel.
// The path carries the wave normal `k` beside the (walked-off) ray direction `d`.
// ------------------------------------------------------------------------------------
// A carved stone's hit (extended instantiation): the intersection's own normal, and the
// medium the ray is in taken from the intersection (bounce_body.rs:391-397: the 1e-4
// restart may have stepped over a second boundary, a tool's rim on a facet).
struct BounceHit {
    Hit hit;
    V3 normal;  // carved only
    int carved;
};
template <int UNI>
IX_DEV BounceHit bounce_next_hit(const Group& g, LanePath& P, const DevScene& S, const float4* __restrict__ planes) {
    BounceHit b;
    b.carved = 0;
    if constexpr (UNI == TRANSPORT_EXTENDED) {
        if (S.concave) {
            const CarvedHit ch = group_carved_hit(g, planes, (int)S.s.n_planes, S.s.tools, (int)S.s.n_tools, P.o, P.d);
            b.hit.t = ch.t;
            b.hit.facet = ch.facet;
            b.normal = ch.normal;
            b.carved = 1;
            if (ch.facet >= 0) P.inside = ch.entering == 0;
            return b;
        }
    }
    b.hit = group_next_hit(g, P, planes, (int)S.s.n_planes);
    return b;
}
// The geometric normal at the hit: the carved intersection's, else the facet plane's.
IX_DEV V3 bounce_hit_normal(const BounceHit& bh, const float4* __restrict__ planes) {
    if (bh.carved) return bh.normal;
    const float4 pl = planes[bh.hit.facet];
    return v3(pl.x, pl.y, pl.z);
}
// The shading normal at a hit: rounded edges (shading_normal_near_edge), on a carved
// stone only away from its tools.
template <int UNI>
IX_DEV V3 bounce_shading_normal(const Group& g, const DevScene& S, const float4* __restrict__ planes,
                                const BounceHit& bh, V3 hit_point, V3 normal) {
    if (!S.rounded) return normal;
    const float radius = S.s.material.edge_rounding_radius;
    if constexpr (UNI == TRANSPORT_EXTENDED) {
        if (bh.carved && ((uint32_t)bh.hit.facet >= S.s.n_planes ||
                          carved_near_tool(hit_point, normal, radius, S.s.tools, (int)S.s.n_tools)))
            return normal;
    }
    return group_shading_normal(g, planes, (int)S.s.n_planes, hit_point, bh.hit.facet, normal, radius);
}
template <int UNI>
IX_DEV void bounce_exit_probes(const Group& g, LanePath& P, const DevScene& S, const float4* __restrict__ planes,
                               const BounceHit& bh, V3 hit_point, bool want_probe, V3 dir_k, float t_int) {
    if constexpr (UNI == TRANSPORT_EXTENDED) {
        if (bh.carved) {
            group_exit_probes_carved(g, P, S, planes, hit_point, want_probe, dir_k, t_int);
            return;
        }
    }
    group_exit_probes<UNI>(g, P, S, planes, hit_point, want_probe, dir_k, t_int);
}

template <int UNI>
IX_DEV int group_bounce_uniaxial(const Group& g, LanePath& P, const DevScene& S,
                                 const float4* __restrict__ planes, float& esc) {
    const ix_scene& sc = S.s;
    const ix_material& mat = sc.material;
    const uint32_t bounce = P.bounce;
    const BounceHit bh = bounce_next_hit<UNI>(g, P, S, planes);
    const Hit hit = bh.hit;
    if (hit.facet < 0) {
        if constexpr (UNI == TRANSPORT_EXTENDED)
            esc = escape_with_carry(P, sc.environment, lane_env<UNI>(sc.environment, P.d, P.observer, P.lambda));
        else
            esc = fmaf(intensity(P.st), lane_env<UNI>(sc.environment, P.d, P.observer, P.lambda), 0.0f);
        return BOUNCE_ESCAPED;
    }
    // pending_light_mis.take() (bounce_body.rs:372): only this iteration's escape reads it.
    if constexpr (UNI == TRANSPORT_EXTENDED) P.has_carry = false;
    const V3 c_axis = load3(mat.c_axis);
    const bool aniso = S.aniso != 0;
    // The channel's alpha along the wave normal: the assigned eigenmode's field for a
    // crystal, the mean over both eigen-polarisations otherwise (absorption.rs:99-197).
    auto channel_alpha = [&](V3 k) {
        if (aniso) {
            const V3 e = assigned_mode_e_field(k, c_axis, P.is_e, P.n_hero, P.n_e_hero);
            return absorption_quadratic_form(c_axis, P.alpha, P.alpha_e, e);
        }
        const V3 ea = ordinary_eigen_polarization(k, c_axis);
        const V3 eb = normalize_or_zero(cross(k, ea));
        return midpointf_(absorption_quadratic_form(c_axis, P.alpha, P.alpha_e, ea),
                          absorption_quadratic_form(c_axis, P.alpha, P.alpha_e, eb));
    };
    if (S.scattering && P.inside) {
        // The interior segment may end in a scattering event first (bounce_body.rs:408-417).
        const ScatterResult r = scatter_or_survive<UNI>(g, P.seed, bounce, S.absorbing ? channel_alpha(P.k) : 0.0f,
                                                   mat.scattering_sigma_s, mat.absorption_path_scale,
                                                   mat.scattering_g, hit.t, intensity(P.st), P.d);
        P.pdf = P.pdf * r.pdf_factor;
        if (r.scattered) {
            P.st = Stokes{r.st_factor, 0.0f, 0.0f, 0.0f};
            P.o = P.o + r.t_model * P.d;
            P.d = r.dir;
            P.k = r.dir;
            P.has_prev = false;  // depolarised: no plane of incidence to rotate from
            if (bounce > 4) {
                float max_i = intensity(P.st);
#pragma unroll
                for (int mm = 4; mm > 0; mm >>= 1) max_i = fmaxf(max_i, gxor(g, max_i, mm));
                const float q = clampf_(fmaxf(0.0f, max_i), 0.05f, 1.0f);
                if (unit_draw(P.seed, bounce, RUSSIAN_ROULETTE_STREAM) > q) return BOUNCE_KILLED;
                P.st = scale(P.st, 1.0f / q);
                P.split = P.split / q;
            }
            P.bounce = bounce + 1;
            return BOUNCE_CONTINUE;
        }
        P.st = scale(P.st, r.st_factor);
    }
    P.facet = hit.facet;
    const V3 hit_point = P.o + hit.t * P.d;
    V3 normal = bounce_shading_normal<UNI>(g, S, planes, bh, hit_point, bounce_hit_normal(bh, planes));
    const V3 k_hat = P.k;

    // rotate_stokes_to_plane_of_incidence, about the wave normal k.
    const V3 cpn = rotate_to_plane_of_incidence(P.st, P.has_prev, P.prev_pn, k_hat, normal);
    P.has_prev = true;
    P.prev_pn = cpn;

    // apply_interior_segment + apply_absorption (transport/inner.rs:170,
    // raytracer/absorption.rs:99-197): the assigned eigenmode's field for a crystal, the
    // mean over both eigen-polarisations otherwise.
    if (P.inside) {
        normal = -normal;
        if (S.absorbing && !S.scattering) {
            const float alpha = channel_alpha(k_hat);
            P.st = scale(P.st, exp_lane(-alpha * (hit.t * mat.absorption_path_scale)));
        }
    }

    // compute_bounce_refraction_geometry (refraction/geometry.rs:306).
    const float cos_i = clampf_(dot(-k_hat, normal), 0.0f, 1.0f);
    const float one_m_c2 = fmaf(cos_i, -cos_i, 1.0f);
    const float sin_i = __fsqrt_rn(fmaxf(one_m_c2, 0.0f));  // IEEE: the TIR retarder is ill-conditioned in it
    float n_eff = P.n, n_eff_hero = P.n_hero;
    if (aniso) {
        // theta_c_for_bounce (geometry.rs:75): two fixed-point steps on entry.
        ThetaC theta;
        if (!P.inside) {
            float n_guess = P.n_hero;
            theta = ThetaC{0.0f, 1.0f};
#pragma unroll
            for (int it = 0; it < 2; ++it) {
                const float e = 1.0f / n_guess;
                const float s2 = e * e * one_m_c2;
                if (s2 > 1.0f) break;
                const float ct = sqrtf(fmaxf(1.0f - s2, 0.0f));
                const V3 w = normalize(e * k_hat + fmaf(e, cos_i, -ct) * normal);
                theta = theta_from_cos(fabsf(clampf_(dot(w, c_axis), -1.0f, 1.0f)));
                n_guess = effective_extraordinary_index(P.n_hero, P.n_e_hero, theta);
            }
        } else {
            theta = theta_from_cos(fabsf(clampf_(dot(k_hat, c_axis), -1.0f, 1.0f)));
        }
        n_eff = effective_extraordinary_index(P.n, P.n_e, theta);
        n_eff_hero = gshfl(g, n_eff, 0);
    }
    const bool inside0 = P.inside;
    const bool ord_medium = aniso && inside0 && !P.is_e;
    const float n_med = ord_medium ? P.n : n_eff;
    const float n_med_hero = ord_medium ? P.n_hero : n_eff_hero;
    const float n1 = inside0 ? n_med_hero : 1.0f;
    const float n2 = inside0 ? 1.0f : n_med_hero;
    const float eta = __fdiv_rn(n1, n2);  // IEEE: it decides TIR and the hero's direction
    const float sin2_t = eta * eta * one_m_c2;
    const float n1k = inside0 ? n_med : 1.0f;
    const float n2k = inside0 ? 1.0f : n_med;
    const float etak = __fdiv_rn(n1k, n2k);
    const float s2k = etak * etak * one_m_c2;
    const float n_o_hero = P.n_hero;
    const float n_e_hero_c = n_o_hero + mat.birefringence_delta;  // walk-off directions only
    const float delta_n = mat.birefringence_delta;
    const bool nondeg = aniso && length_squared(cross(k_hat, c_axis)) > 1e-6f;

    V3 new_k, new_s;
    bool new_inside = inside0;
    int update = -1;
    bool has_p_o = false;
    float p_o_exact = 0.0f;
    int status = 0;
    bool narrow = false, want_probe = false;
    V3 dir_k = v3(0.0f, 0.0f, 0.0f);
    float t_int = 0.0f;

    const bool frosted = facet_frosted(S, hit.facet);
    if (frosted) {
        // apply_frosted_bounce (frosted.rs:289): the diffuse lobe is both the wave normal
        // and the ray; an anisotropic entry draws its eigenmode with probability 1/2.
        const FrostedScatter f = frosted_scatter(P.seed, bounce, normal, n1, n2, cos_i, sin2_t);
        lane_frosted_apply(P, f);
        new_k = f.dir;
        new_s = new_k;
        if (f.transmit) {
            new_inside = !inside0;
            if (!inside0 && aniso) update = unit_draw(P.seed, bounce, BIREFRINGENT_SPLIT_STREAM) < 0.5f ? 1 : 0;
        }
        if constexpr (UNI == TRANSPORT_EXTENDED)
            frosted_exterior_event(g, P, S, planes, f, inside0, normal, hit_point, bounce);
    } else if (sin2_t > 1.0f) {
        // apply_tir_bounce (tir.rs:41): forced reflection.
        if (nondeg) {
            const UFrame f = uframe_build(k_hat, normal, c_axis, cos_i, sin_i);
            const IntSol sol = internal_solve(n1k, P.n, P.n_e, c_axis, f, !P.is_e);
            const float ro = cnorm2(sol.r_o) * sol.flux_ro;
            const float re = cnorm2(sol.r_e) * sol.flux_re;
            const float r_total = fminf((ro + re) / fmaxf(sol.flux_inc, 1e-12f), 1.0f);
            P.st = scale(P.st, r_total);
            if (s2k <= 1.0f) P.pdf = P.pdf * clampf_(r_total, R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
            p_o_exact = gshfl(g, ro / fmaxf(ro + re, 1e-12f), 0);
            has_p_o = true;
        } else {
            P.st = lane_scalar_reflect(P, n1k, n2k, s2k, cos_i, sin_i);
        }
        new_k = k_hat - 2.0f * dot(k_hat, normal) * normal;
        new_s = (aniso && inside0 && P.is_e) ? extraordinary_poynting_dir(new_k, c_axis, n_o_hero, n_e_hero_c) : new_k;
    } else if (nondeg && !inside0) {
        // apply_uniaxial_entry_bounce (uniaxial_entry.rs:108).
        const UFrame f = uframe_build(k_hat, normal, c_axis, cos_i, sin_i);
        const EntryInc inc = entry_incidence_frame(1.0f, f);
        const EntrySol s = entry_solve(inc, 1.0f, P.n, P.n_e, c_axis, f);
        const float r_unpol_k = jones_r_unpol(s.r_s[0], s.r_s[1], s.r_p[0], s.r_p[1]);
        const float r_branch = clampf_(gshfl(g, r_unpol_k, 0), R_UNPOL_SELECT_MIN, R_UNPOL_SELECT_MAX);
        const float inc_flux = 0.5f * f.cos_i;
        const float p_o_raw = mode_power(s.t_o[0], s.t_o[1], s.flux_o, inc_flux, P.st);
        const float p_e_raw = mode_power(s.t_e[0], s.t_e[1], s.flux_e, inc_flux, P.st);
        const float p_o_hero = gshfl(
            g, clampf_(p_o_raw / fmaxf(p_o_raw + p_e_raw, 1e-12f), R_UNPOL_SELECT_MIN, R_UNPOL_SELECT_MAX), 0);
        const bool use_e = unit_draw(P.seed, bounce, BIREFRINGENT_SPLIT_STREAM) < 1.0f - p_o_hero;
        const float p_frac = use_e ? 1.0f - p_o_hero : p_o_hero;
        const float e_dir = __fdiv_rn(n1, use_e ? n2 : n_o_hero);
        const float c_dir = __fsqrt_rn(fmaxf(1.0f - fminf(e_dir * e_dir * one_m_c2, 1.0f), 0.0f));
        const V3 refr = normalize_dir(e_dir * k_hat + fmaf(e_dir, cos_i, -c_dir) * normal);
        const V3 final_refr = use_e ? extraordinary_poynting_dir(refr, c_axis, n_o_hero, n_e_hero_c) : refr;
        if (unit_draw(P.seed, bounce, FRESNEL_BRANCH_STREAM) < r_branch) {
            const M4 mk = jones_to_mueller(s.r_s[0], s.r_s[1], s.r_p[0], s.r_p[1]);
            P.st = scale(apply_m4(mk, P.st), 1.0f / r_branch);
            P.pdf = P.pdf * clampf_(mk.c[0], R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
            new_k = new_s = k_hat - 2.0f * dot(k_hat, normal) * normal;
            new_inside = false;
        } else {
            const float n2k_dir = use_e ? n2k : P.n;
            const float ratio = __fdiv_rn(n1, n2k_dir);
            const float s2 = (ratio * ratio) * one_m_c2;
            if (s2 > 1.0f) {
                P.st = scale(P.st, 0.0f);
                P.pdf = 0.0f;
            } else {
                const float cos_t_k = __fsqrt_rn(fmaxf(1.0f - s2, 0.0f));
                const V3 refr_k = normalize_dir(ratio * k_hat + fmaf(ratio, cos_i, -cos_t_k) * normal);
                dir_k = use_e ? extraordinary_poynting_dir(refr_k, c_axis, P.n, P.n + delta_n) : refr_k;
                status = dot(dir_k, final_refr) >= DIRECTION_MATCH_COS_TOL ? 1 : 2;
                const float t_unpol = clampf_(1.0f - r_unpol_k, R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
                if (status == 1) {
                    const float deposit =
                        mode_power(use_e ? s.t_e[0] : s.t_o[0], use_e ? s.t_e[1] : s.t_o[1],
                                   use_e ? s.flux_e : s.flux_o, inc_flux, P.st) / p_frac;
                    float c2, s2a;
                    azimuth2_in_frame(use_e ? s.e_hat : s.o_hat, f.s_axis, cross(refr, f.s_axis), c2, s2a);
                    P.st = scale(Stokes{deposit, deposit * c2, deposit * s2a, 0.0f}, 1.0f / (1.0f - r_branch));
                } else {
                    P.st = scale(P.st, 0.0f);
                }
                P.pdf = P.pdf * t_unpol;
            }
            narrow = true;
            new_k = refr;
            new_s = final_refr;
            new_inside = true;
            update = use_e ? 1 : 0;
        }
    } else if (nondeg) {
        // apply_uniaxial_internal_bounce (uniaxial_internal.rs:68).
        const UFrame f = uframe_build(k_hat, normal, c_axis, cos_i, sin_i);
        const IntSol sol = internal_solve(n1k, P.n, P.n_e, c_axis, f, !P.is_e);
        const float flux_inc = fmaxf(sol.flux_inc, 1e-12f);
        const float ro = cnorm2(sol.r_o) * sol.flux_ro;
        const float re = cnorm2(sol.r_e) * sol.flux_re;
        const float r_branch =
            gshfl(g, clampf_((ro + re) / flux_inc, R_UNPOL_SELECT_MIN, R_UNPOL_SELECT_MAX), 0);
        const float p_o_h = gshfl(g, ro / fmaxf(ro + re, 1e-12f), 0);
        if (unit_draw(P.seed, bounce, FRESNEL_BRANCH_STREAM) < r_branch) {
            const float r_total_k =
                fminf(fmaf(cnorm2(sol.r_e), sol.flux_re, cnorm2(sol.r_o) * sol.flux_ro) / flux_inc, 1.0f);
            P.st = scale(P.st, r_total_k / r_branch);
            P.pdf = P.pdf * clampf_(r_total_k, R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
            new_k = new_s = k_hat - 2.0f * dot(k_hat, normal) * normal;
            has_p_o = true;
            p_o_exact = p_o_h;
        } else {
            const float c_dir = __fsqrt_rn(fmaxf(1.0f - fminf(eta * eta * one_m_c2, 1.0f), 0.0f));
            const V3 hero_refr = normalize_dir(eta * k_hat + fmaf(eta, cos_i, -c_dir) * normal);
            const float original_i = P.st.i;
            if (s2k > 1.0f) {
                P.st = scale(P.st, 0.0f);
                P.pdf = 0.0f;
            } else {
                const float cos_t_k = __fsqrt_rn(fmaxf(1.0f - s2k, 0.0f));
                dir_k = normalize_dir(etak * k_hat + fmaf(etak, cos_i, -cos_t_k) * normal);
                status = dot(dir_k, hero_refr) >= DIRECTION_MATCH_COS_TOL ? 1 : 2;
                float i_unit;
                const Stokes tr = uniaxial_exit_transmission(sol, r_branch, original_i, i_unit);
                P.pdf = P.pdf * clampf_(i_unit, R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
                P.st = status == 1 ? tr : scale(P.st, 0.0f);
                want_probe = status == 2 && original_i > 0.0f;
                t_int = intensity(tr);
            }
            new_k = new_s = hero_refr;
            new_inside = false;
        }
    } else {
        // apply_partial_fresnel_bounce's scalar path (dispatch.rs:162-380): an isotropic
        // material, or a uniaxial one with k along the optic axis.
        const bool entering = aniso && !inside0;
        bool has_sel = false;
        float p_o = 0.5f, c2 = 0.0f, s2 = 0.0f;
        if (entering) {
            // resolve_entry_mode_selection (dispatch.rs:162): the hero's Stokes state.
            float po_l = 0.5f, c2_l = 0.0f, s2_l = 0.0f;
            const bool sel_l = entry_eigenmode_selection(c_axis, cpn, k_hat, P.st, po_l, c2_l, s2_l);
            has_sel = gshfl(g, sel_l ? 1 : 0, 0) != 0;
            p_o = has_sel ? gshfl(g, po_l, 0) : 0.5f;
            c2 = gshfl(g, c2_l, 0);
            s2 = gshfl(g, s2_l, 0);
        }
        const bool use_e = entering ? unit_draw(P.seed, bounce, BIREFRINGENT_SPLIT_STREAM) < 1.0f - p_o : P.is_e;
        const bool ord_sel = entering && !use_e;
        // compute_entry_reflect_probability (dispatch.rs:230).
        const float n2s = ord_sel ? n_o_hero : n2;
        float sin2_ts = sin2_t;
        if (ord_sel) {
            const float e2 = n1 / n2s;
            sin2_ts = e2 * e2 * one_m_c2;
        }
        float r_s, r_p;
        fresnel_rs_rp(n1, n2s, cos_i, sqrtf(fmaxf(1.0f - sin2_ts, 0.0f)), r_s, r_p);
        const float r_unpol = clampf_(r_unpol_of(r_s, r_p), R_UNPOL_SELECT_MIN, R_UNPOL_SELECT_MAX);
        if (unit_draw(P.seed, bounce, FRESNEL_BRANCH_STREAM) < r_unpol) {
            P.st = scale(lane_scalar_reflect(P, n1k, n2k, s2k, cos_i, sin_i), 1.0f / r_unpol);
            new_k = k_hat - 2.0f * dot(k_hat, normal) * normal;
            new_s = (aniso && inside0 && P.is_e) ? extraordinary_poynting_dir(new_k, c_axis, n_o_hero, n_e_hero_c)
                                                 : new_k;
        } else {
            // apply_refract_bounce / apply_refract_channel (reflect_refract.rs:121-591).
            const float e_dir = __fdiv_rn(n1, n2s);
            const float c_dir = __fsqrt_rn(fmaxf(1.0f - fminf(e_dir * e_dir * one_m_c2, 1.0f), 0.0f));
            const V3 refr = normalize_dir(e_dir * k_hat + fmaf(e_dir, cos_i, -c_dir) * normal);
            const bool walk = entering && use_e;
            const V3 final_refr = walk ? extraordinary_poynting_dir(refr, c_axis, n_o_hero, n_e_hero_c) : refr;
            const float n2k_r = ord_sel ? P.n : n2k;
            const float ratio = __fdiv_rn(n1k, n2k_r);
            const float s2r = (ratio * ratio) * one_m_c2;
            const Stokes original = P.st;
            if (s2r > 1.0f) {
                P.st = scale(P.st, 0.0f);
                P.pdf = 0.0f;
            } else {
                const float cos_t_k = __fsqrt_rn(fmaxf(1.0f - s2r, 0.0f));
                const V3 refr_k = normalize_dir(ratio * k_hat + fmaf(ratio, cos_i, -cos_t_k) * normal);
                dir_k = walk ? extraordinary_poynting_dir(refr_k, c_axis, P.n, P.n + delta_n) : refr_k;
                status = dot(dir_k, final_refr) >= DIRECTION_MATCH_COS_TOL ? 1 : 2;
                const float two = 2.0f * n1k * cos_i;
                const float t_s = two / fmaf(n2k_r, cos_t_k, n1k * cos_i);
                const float t_p = two / fmaf(n1k, cos_t_k, n2k_r * cos_i);
                // The selected eigenmode's projection at an anisotropic entry.
                const float az_c = use_e ? -c2 : c2, az_s = use_e ? -s2 : s2;
                const Stokes incident = (entering && has_sel)
                                            ? Stokes{original.i, original.i * az_c, original.i * az_s, 0.0f}
                                            : original;
                const Stokes transmitted =
                    scale(fresnel_transmit_apply(incident, n1k, n2k_r, cos_i, cos_t_k, t_s, t_p),
                          1.0f / (1.0f - r_unpol));
                float rs, rp;
                fresnel_rs_rp(n1k, n2k_r, cos_i, cos_t_k, rs, rp);
                P.pdf = P.pdf * (1.0f - clampf_(r_unpol_of(rs, rp), R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX));
                P.st = status == 1 ? transmitted : scale(original, 0.0f);
                t_int = intensity(transmitted);
                want_probe = status == 2 && inside0 && intensity(original) > 0.0f;
            }
            narrow = !inside0;
            new_k = refr;
            new_s = final_refr;
            new_inside = !inside0;
            update = entering ? (use_e ? 1 : 0) : -1;
        }
    }
    bounce_exit_probes<UNI>(g, P, S, planes, bh, hit_point, want_probe, dir_k, t_int);
    if (narrow) group_narrow_compat(g, P, status, dir_k);

    const bool was_internal_reflection = inside0 && update < 0 && new_inside == inside0;
    P.d = new_s;
    P.o = hit_point + new_s * 1e-4f;
    P.k = new_k;
    P.inside = new_inside;
    if (update >= 0) P.is_e = update != 0;
    // maybe_apply_internal_mode_coupling (transport/bounce.rs:470): an internal
    // reflection relabels the eigenmode with the closed-form R_o / (R_o + R_e), else the
    // hero's polarisation weight.
    if (aniso && was_internal_reflection) {
        float p_o = p_o_exact;
        if (!has_p_o) {
            float po_l = 0.5f, a, b;
            if (!entry_eigenmode_selection(c_axis, cpn, P.k, P.st, po_l, a, b)) po_l = 0.5f;
            p_o = gshfl(g, po_l, 0);
        }
        P.is_e = unit_draw(P.seed, bounce, MODE_COUPLING_STREAM) >= p_o;
    }

    // Surface glare (bounce_body.rs:691-697), polished facets only, and Russian roulette
    // (transport/bounce.rs:355).
    const float glare = clampf_(sc.environment.surface_glare, 0.0f, 1.0f);
    if (bounce == 0 && !P.inside && glare < 1.0f && !frosted) P.st = scale(P.st, glare);
    if (bounce > 4) {
        float max_i = intensity(P.st);
#pragma unroll
        for (int m = 4; m > 0; m >>= 1) max_i = fmaxf(max_i, gxor(g, max_i, m));
        const float q = clampf_(fmaxf(0.0f, max_i), 0.05f, 1.0f);
        if (unit_draw(P.seed, bounce, RUSSIAN_ROULETTE_STREAM) > q) return BOUNCE_KILLED;
        P.st = scale(P.st, 1.0f / q);
        P.split = P.split / q;
    }
    P.bounce = bounce + 1;
    return BOUNCE_CONTINUE;
}

// ------------------------------------------------------------------------------------
// One bounce of a path in a biaxial crystal (transport/bounce.rs:108-160 with the
// biaxial arms of refraction/geometry.rs:220-400, dispatch.rs:162-300,
// reflect_refract.rs:121-330 and absorption.rs:227): no closed-form uniaxial solve, so
// every interface takes the scalar-Fresnel path; the two eigenmodes ("mode A", the fast
// root, and "mode B", the slow root, in the is_e slot) take their indices from each
// channel's own indicatrix at the hero's wave normal (resolved per mode by a two-step
// fixed point on entry), the entry split is 50 / 50, both modes walk off, and the
// trichroic tensor absorbs along the assigned mode's field.  Out of line and by value:
// the uniaxial bounce, and every kernel that inlines it, compiles as it does without it.
// ------------------------------------------------------------------------------------
struct BiaxialStep {
    LanePath P;
    float esc;
    int result;
};
static __device__ __noinline__ BiaxialStep group_bounce_biaxial(Group g, LanePath P, DevScene S,
                                                                 const float4* __restrict__ planes) {
    BiaxialStep out{P, 0.0f, BOUNCE_CONTINUE};
    const ix_scene& sc = S.s;
    const ix_material& mat = sc.material;
    const uint32_t bounce = P.bounce;
    const BounceHit bh = bounce_next_hit<TRANSPORT_EXTENDED>(g, P, S, planes);
    const Hit hit = bh.hit;
    if (hit.facet < 0) {
        out.esc = escape_with_carry(P, sc.environment,
                                    lane_env<TRANSPORT_EXTENDED>(sc.environment, P.d, P.observer, P.lambda));
        out.P = P;
        out.result = BOUNCE_ESCAPED;
        return out;
    }
    P.has_carry = false;  // pending_light_mis.take() (bounce_body.rs:372)
    const BiaxFrame F = biax_frame(load3(mat.c_axis));
    const Indicatrix hero = make_indicatrix(mat, P.n_hero), own = make_indicatrix(mat, P.n);
    // channel_absorption_alphas_assigned (absorption.rs:227): the hero indicatrix's
    // assigned-mode field against this channel's (alpha, beta, gamma) tensor; n_e holds
    // the beta-ray alpha.
    auto channel_alpha = [&](V3 k) {
        const V3 e = assigned_mode_e_field_biaxial(hero, F, k, P.is_e);
        return biaxial_quadratic_form(F, P.alpha, P.n_e, P.alpha_e, e);
    };
    if (S.scattering && P.inside) {
        const ScatterResult r =
            scatter_or_survive<TRANSPORT_EXTENDED>(g, P.seed, bounce, S.absorbing ? channel_alpha(P.k) : 0.0f,
                                                   mat.scattering_sigma_s, mat.absorption_path_scale,
                                                   mat.scattering_g, hit.t, intensity(P.st), P.d);
        P.pdf = P.pdf * r.pdf_factor;
        if (r.scattered) {
            P.st = Stokes{r.st_factor, 0.0f, 0.0f, 0.0f};
            P.o = P.o + r.t_model * P.d;
            P.d = r.dir;
            P.k = r.dir;
            P.has_prev = false;
            if (bounce > 4) {
                float max_i = intensity(P.st);
#pragma unroll
                for (int mm = 4; mm > 0; mm >>= 1) max_i = fmaxf(max_i, gxor(g, max_i, mm));
                const float q = clampf_(fmaxf(0.0f, max_i), 0.05f, 1.0f);
                if (unit_draw(P.seed, bounce, RUSSIAN_ROULETTE_STREAM) > q) {
                    out.P = P;
                    out.result = BOUNCE_KILLED;
                    return out;
                }
                P.st = scale(P.st, 1.0f / q);
                P.split = P.split / q;
            }
            P.bounce = bounce + 1;
            out.P = P;
            return out;
        }
        P.st = scale(P.st, r.st_factor);
    }
    P.facet = hit.facet;
    const V3 hit_point = P.o + hit.t * P.d;
    V3 normal = bounce_shading_normal<TRANSPORT_EXTENDED>(g, S, planes, bh, hit_point, bounce_hit_normal(bh, planes));
    const V3 k_hat = P.k;
    const V3 cpn = rotate_to_plane_of_incidence(P.st, P.has_prev, P.prev_pn, k_hat, normal);
    P.has_prev = true;
    P.prev_pn = cpn;
    if (P.inside) {
        normal = -normal;
        if (S.absorbing && !S.scattering)
            P.st = scale(P.st, exp_lane(-channel_alpha(k_hat) * (hit.t * mat.absorption_path_scale)));
    }

    // compute_bounce_refraction_geometry's biaxial arm (geometry.rs:306-400).
    const float cos_i = clampf_(dot(-k_hat, normal), 0.0f, 1.0f);
    const float one_m_c2 = fmaf(cos_i, -cos_i, 1.0f);
    const float sin_i = __fsqrt_rn(fmaxf(one_m_c2, 0.0f));
    const bool inside0 = P.inside;
    V3 dir_a = k_hat, dir_b = k_hat;
    if (!inside0) {
        resolve_entry_mode(hero, F, k_hat, normal, cos_i, P.n_hero, false, dir_a);
        resolve_entry_mode(hero, F, k_hat, normal, cos_i, P.n_hero, true, dir_b);
    }
    float ns, nf;
    wave_indices(own, F, dir_a, ns, nf);
    const float n_a = nf;
    wave_indices(own, F, dir_b, ns, nf);
    const float n_b = ns;
    const float n_a_hero = gshfl(g, n_a, 0), n_b_hero = gshfl(g, n_b, 0);
    const bool mode_a_medium = inside0 && !P.is_e;
    const float n_med = mode_a_medium ? n_a : n_b;
    const float n_med_hero = mode_a_medium ? n_a_hero : n_b_hero;
    const float n1 = inside0 ? n_med_hero : 1.0f;
    const float n2 = inside0 ? 1.0f : n_med_hero;
    const float eta = __fdiv_rn(n1, n2);
    const float sin2_t = eta * eta * one_m_c2;
    const float n1k = inside0 ? n_med : 1.0f;
    const float n2k = inside0 ? 1.0f : n_med;
    const float etak = __fdiv_rn(n1k, n2k);
    const float s2k = etak * etak * one_m_c2;

    V3 new_k, new_s;
    bool new_inside = inside0;
    int update = -1;
    int status = 0;
    bool narrow = false, want_probe = false;
    V3 dir_k = v3(0.0f, 0.0f, 0.0f);
    float t_int = 0.0f;
    const bool frosted = facet_frosted(S, hit.facet);
    if (frosted) {
        const FrostedScatter f = frosted_scatter(P.seed, bounce, normal, n1, n2, cos_i, sin2_t);
        lane_frosted_apply(P, f);
        new_k = new_s = f.dir;
        if (f.transmit) {
            new_inside = !inside0;
            if (!inside0) update = unit_draw(P.seed, bounce, BIREFRINGENT_SPLIT_STREAM) < 0.5f ? 1 : 0;
        }
        frosted_exterior_event(g, P, S, planes, f, inside0, normal, hit_point, bounce);
    } else if (sin2_t > 1.0f) {
        // apply_tir_bounce's scalar arm (tir.rs:98-116); the reflected wave normal's mode
        // walks off (poynting_dir_for_mode, geometry.rs:440).
        P.st = lane_scalar_reflect(P, n1k, n2k, s2k, cos_i, sin_i);
        new_k = k_hat - 2.0f * dot(k_hat, normal) * normal;
        new_s = mode_poynting_dir(hero, F, new_k, P.is_e);
    } else {
        // apply_partial_fresnel_bounce (dispatch.rs:162-300): 50 / 50 at an entry.
        const bool entering = !inside0;
        const bool use_e = entering ? unit_draw(P.seed, bounce, BIREFRINGENT_SPLIT_STREAM) < 0.5f : P.is_e;
        float r_s, r_p;
        fresnel_rs_rp(n1, n2, cos_i, sqrtf(fmaxf(1.0f - sin2_t, 0.0f)), r_s, r_p);
        const float r_unpol = clampf_(r_unpol_of(r_s, r_p), R_UNPOL_SELECT_MIN, R_UNPOL_SELECT_MAX);
        if (unit_draw(P.seed, bounce, FRESNEL_BRANCH_STREAM) < r_unpol) {
            P.st = scale(lane_scalar_reflect(P, n1k, n2k, s2k, cos_i, sin_i), 1.0f / r_unpol);
            new_k = k_hat - 2.0f * dot(k_hat, normal) * normal;
            new_s = inside0 ? mode_poynting_dir(hero, F, new_k, P.is_e) : new_k;
        } else {
            // apply_refract_bounce (reflect_refract.rs:121-200): on entry the selected
            // mode's own index and walk-off, per channel its own indicatrix.
            // The hero's direction and each channel's own are formed by one correctly
            // rounded routine, so the hero lane's channel direction is the hero direction
            // bit for bit: the eigen-direction amplifies any difference near an optic
            // axis, and the hero must never fail its own match test (geometry.rs:366).
            auto refract_rn = [&](float eta, float& cos_t) {
                const float s2 = fminf(mul_(mul_(eta, eta), one_m_c2), 1.0f);
                cos_t = __fsqrt_rn(fmaxf(sub_(1.0f, s2), 0.0f));
                return normalize_(vadd_(vmul_(k_hat, eta), vmul_(normal, fmaf(eta, cos_i, -cos_t))));
            };
            const float n2_dir = entering ? (use_e ? n_b_hero : n_a_hero) : n2;
            float c_dir;
            const V3 refr = refract_rn(div_(n1, n2_dir), c_dir);
            const V3 final_refr = entering ? mode_poynting_dir(hero, F, refr, use_e) : refr;
            const float n2k_r = (entering && !use_e) ? n_a : n2k;
            const float ratio = div_(n1k, n2k_r);
            const float s2r = mul_(mul_(ratio, ratio), one_m_c2);
            const Stokes original = P.st;
            if (s2r > 1.0f) {
                P.st = scale(P.st, 0.0f);
                P.pdf = 0.0f;
            } else {
                float cos_t_k;
                const V3 refr_k = refract_rn(ratio, cos_t_k);
                dir_k = entering ? mode_poynting_dir(own, F, refr_k, use_e) : refr_k;
                status = dot(dir_k, final_refr) >= DIRECTION_MATCH_COS_TOL ? 1 : 2;
                const float two = 2.0f * n1k * cos_i;
                const float t_s = two / fmaf(n2k_r, cos_t_k, n1k * cos_i);
                const float t_p = two / fmaf(n1k, cos_t_k, n2k_r * cos_i);
                const Stokes transmitted =
                    scale(fresnel_transmit_apply(original, n1k, n2k_r, cos_i, cos_t_k, t_s, t_p),
                          1.0f / (1.0f - r_unpol));
                float rs, rp;
                fresnel_rs_rp(n1k, n2k_r, cos_i, cos_t_k, rs, rp);
                P.pdf = P.pdf * (1.0f - clampf_(r_unpol_of(rs, rp), R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX));
                P.st = status == 1 ? transmitted : scale(original, 0.0f);
                t_int = intensity(transmitted);
                want_probe = status == 2 && inside0 && intensity(original) > 0.0f;
            }
            narrow = entering;
            new_k = refr;
            new_s = final_refr;
            new_inside = !inside0;
            update = entering ? (use_e ? 1 : 0) : -1;
        }
    }
    bounce_exit_probes<TRANSPORT_EXTENDED>(g, P, S, planes, bh, hit_point, want_probe, dir_k, t_int);
    if (narrow) group_narrow_compat(g, P, status, dir_k);

    const bool was_internal_reflection = inside0 && update < 0 && new_inside == inside0;
    P.d = new_s;
    P.o = hit_point + new_s * 1e-4f;
    P.k = new_k;
    P.inside = new_inside;
    if (update >= 0) P.is_e = update != 0;
    // maybe_apply_internal_mode_coupling (transport/bounce.rs:441-470): a blanket 50 / 50.
    if (was_internal_reflection) P.is_e = unit_draw(P.seed, bounce, MODE_COUPLING_STREAM) >= 0.5f;

    const float glare = clampf_(sc.environment.surface_glare, 0.0f, 1.0f);
    if (bounce == 0 && !P.inside && glare < 1.0f && !frosted) P.st = scale(P.st, glare);
    if (bounce > 4) {
        float max_i = intensity(P.st);
#pragma unroll
        for (int m = 4; m > 0; m >>= 1) max_i = fmaxf(max_i, gxor(g, max_i, m));
        const float q = clampf_(fmaxf(0.0f, max_i), 0.05f, 1.0f);
        if (unit_draw(P.seed, bounce, RUSSIAN_ROULETTE_STREAM) > q) {
            out.P = P;
            out.result = BOUNCE_KILLED;
            return out;
        }
        P.st = scale(P.st, 1.0f / q);
        P.split = P.split / q;
    }
    P.bounce = bounce + 1;
    out.P = P;
    return out;
}

// The extended instantiation's uniaxial bounce, out of line and by value like the biaxial
// one: every kernel (task loop, pool, per-path check) then runs the same compiled bounce, so
// the fast build's multiply-add contraction, and with it each path's result, is the same
// whichever kernel traces the path.
static __device__ __noinline__ BiaxialStep group_bounce_extended(Group g, LanePath P, DevScene S,
                                                                  const float4* __restrict__ planes) {
    BiaxialStep out{P, 0.0f, BOUNCE_CONTINUE};
    out.result = group_bounce_uniaxial<TRANSPORT_EXTENDED>(g, P, S, planes, out.esc);
    out.P = P;
    return out;
}

// UNI is the transport instantiation (transport_class): TRANSPORT_ISOTROPIC the isotropic
// megakernel, TRANSPORT_UNIAXIAL the uniaxial bounce, TRANSPORT_EXTENDED the out-of-line
// uniaxial and biaxial bounces (kept out of the uniaxial kernels, whose register allocation
// the call sites would change).
template <int UNI>
IX_DEV int group_step(const Group& g, LanePath& P, const DevScene& S, const float4* __restrict__ planes, float& esc) {
    if constexpr (UNI == TRANSPORT_EXTENDED) {
        const BiaxialStep r =
            S.biaxial ? group_bounce_biaxial(g, P, S, planes) : group_bounce_extended(g, P, S, planes);
        P = r.P;
        esc = r.esc;
        return r.result;
    } else if constexpr (UNI == TRANSPORT_UNIAXIAL) {
        return group_bounce_uniaxial<UNI>(g, P, S, planes, esc);
    } else {
        return group_bounce(g, P, S, planes, esc);
    }
}

// finish (bounce_body.rs:724-764): commit the exit splits of an escaped path, integrate
// each channel over its MIS family (optics/raytracer/color.rs:145), apply the Bradford
// round trip for studio environments (color.rs:252) and floor at zero.  Every lane of
// the group returns the path's XYZ.
// `esc` is the escape radiance (with the extended instantiation's next-event deposits
// folded in); a path that did not escape keeps only those deposits.
template <int UNI = TRANSPORT_ISOTROPIC>
IX_DEV V3 group_finish(const Group& g, const LanePath& P, const DevScene& S, bool escaped, float esc) {
    // family pdf: the sum, in ascending channel order, over this channel's family.
    float family = 0.0f;
    bool first = true;
    const float pdf0 = gshfl(g, P.pdf, 0);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float pj = gshfl(g, P.pdf, j);
        if (P.compat & (1u << j)) {
            family = first ? pj : family + pj;
            first = false;
        }
    }
    const float w = (family <= 1e-12f) ? 1.0f : (8.0f * pdf0) / family;
    float rad;
    if constexpr (UNI == TRANSPORT_EXTENDED)
        rad = escaped ? esc + P.split : P.nee_rad;
    else
        rad = escaped ? esc + P.split : 0.0f;
    const float s = (rad * w) * (50.0f / 106.856f);
    const V3 c = cmf(P.lambda);
    const float cx = c.x * s, cy = c.y * s, cz = c.z * s;
    // xyz += cmf_k * (...), folded in channel order as the reference folds it.
    float x = 0.0f, y = 0.0f, z = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        x = x + gshfl(g, cx, j);
        y = y + gshfl(g, cy, j);
        z = z + gshfl(g, cz, j);
    }
    x = x + 0.0f;
    y = y + 0.0f;
    z = z + 0.0f;
    const ix_environment& env = S.s.environment;
    if (env.model != IX_ENV_UNIFORM) {
        float l = fmaf(0.8951f, x, fmaf(0.2664f, y, -0.1614f * z));
        float m = fmaf(-0.7502f, x, fmaf(1.7135f, y, 0.0367f * z));
        float q = fmaf(0.0389f, x, fmaf(-0.0685f, y, 1.0296f * z));
        l = l * env.wb_lms[0];
        m = m * env.wb_lms[1];
        q = q * env.wb_lms[2];
        x = fmaf(0.986993f, l, fmaf(-0.147054f, m, 0.159963f * q));
        y = fmaf(0.432305f, l, fmaf(0.518360f, m, 0.049291f * q));
        z = fmaf(-0.008529f, l, fmaf(0.040043f, m, 0.968487f * q));
    }
    return v3(fmaxf(x, 0.0f), fmaxf(y, 0.0f), fmaxf(z, 0.0f));
}

// A whole path by one group (the check kernels' per-path entry).
template <int UNI>
IX_DEV V3 group_trace(const Group& g, LanePath& P, const DevScene& S, const float4* planes,
                      uint32_t* iterations) {
    float esc = 0.0f;
    int r = BOUNCE_CONTINUE;
    uint32_t it = 0;
    while (P.bounce < S.s.max_bounces) {
        r = group_step<UNI>(g, P, S, planes, esc);
        ++it;
        if (r != BOUNCE_CONTINUE) break;
    }
    if (iterations) *iterations = it;
    return group_finish<UNI>(g, P, S, r == BOUNCE_ESCAPED, esc);
}

}  // namespace ix
