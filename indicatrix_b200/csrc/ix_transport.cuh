// ix_transport.cuh -- one spectral path on the GPU: setup, one bounce, finish.
//
// The path is split into three device functions so the megakernel can regenerate a
// finished lane with its next sample while the warp's other lanes keep bouncing (the
// bounce body, where nearly all the work is, then runs converged across lanes that are
// on different paths).  Together they compute what the reference's
// trace_spectral_ray_core computes for one (pixel, absolute sample)
// (optics/raytracer/transport/inner/bounce_body.rs:216-764) for a convex, polished,
// non-scattering, non-fluorescent stone with an isotropic material -- the scenes
// `ix_scene_routes_to_gpu` admits.
#pragma once

#include "ix_device.cuh"

namespace ix {

constexpr float DIRECTION_MATCH_COS_TOL = 1.0f - 1e-6f;  // refraction/mod.rs:137
constexpr float R_UNPOL_PDF_MIN = 1e-4f;                 // refraction/mod.rs:143
constexpr float R_UNPOL_PDF_MAX = 1.0f - 1e-4f;          // refraction/mod.rs:146
constexpr float R_UNPOL_SELECT_MIN = 0.02f;              // refraction/mod.rs:153
constexpr float R_UNPOL_SELECT_MAX = 0.98f;              // refraction/mod.rs:156

// Scene as the kernels see it: the host POD with `planes` pointing at device memory and
// a few per-scene flags resolved on the host.
struct DevScene {
    const ix_scene& s;   // lives in kernel parameter space (__grid_constant__)
    uint32_t absorbing;  // the material has any absorption term
};

struct PathState {
    uint32_t seed;
    uint32_t bounce;
    float lambdas[8];
    float n_ch[8];
    float alpha[8];
    Stokes st[8];
    float pdf[8];
    float split[8];
    uint32_t compat_lo, compat_hi;  // compat[k] as bytes: k<4 in lo, k>=4 in hi
    V3 o, d;
    V3 prev_pn;
    V3 observer;
    bool inside;
    bool has_prev;
};

IX_DEV uint32_t compat_get(const PathState& P, int k) {
    uint32_t w = (k < 4) ? P.compat_lo : P.compat_hi;
    return (w >> (8 * (k & 3))) & 0xFFu;
}
IX_DEV void compat_clear_bit(PathState& P, int k, int bit) {
    uint32_t m = ~(1u << (8 * (k & 3) + bit));
    if (k < 4)
        P.compat_lo &= m;
    else
        P.compat_hi &= m;
}

// PathState::new (bounce_body.rs:260-356) for an explicit ray, seed and hero draw
// (trace_spectral_ray, transport/mod.rs:118).
IX_DEV void path_init_ray(PathState& P, const DevScene& S, Ray r, uint32_t seed, float hero) {
    const ix_scene& sc = S.s;
    P.seed = seed;
    P.bounce = 0;
    hero_wavelengths(hero, P.lambdas);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        P.n_ch[k] = dispersion_eval(sc.material.dispersion, P.lambdas[k]);
        P.alpha[k] = S.absorbing ? spectral_absorption(sc.material.abs_o, P.lambdas[k]) : 0.0f;
        P.st[k] = Stokes{1.0f, 0.0f, 0.0f, 0.0f};
        P.pdf[k] = 1.0f;
        P.split[k] = 0.0f;
    }
    P.compat_lo = P.compat_hi = 0xFFFFFFFFu;
    P.o = r.origin;
    P.d = r.dir;
    P.observer = -r.dir;
    P.inside = false;
    P.has_prev = false;
    P.prev_pn = v3(0.0f, 0.0f, 0.0f);
}

// One (pixel, absolute sample) as renderer/cpu_frame.rs:45-70 traces it.
IX_DEV void path_init(PathState& P, const DevScene& S, uint32_t pixel, uint32_t sample) {
    const ix_scene& sc = S.s;
    Draws dr = sample_draws(pixel, sample);
    uint32_t x = pixel % sc.width, y = pixel / sc.width;
    Ray r = generate_ray(sc.camera, (float)x, (float)y, (float)sc.width, (float)sc.height,
                         dr.jx, dr.jy);
    path_init_ray(P, S, r, dr.seed, dr.hero);
}

// try_split_exit_channel (refraction/exit_split.rs:128): one extra intersection, then an
// environment lookup at the channel's own wavelength if the probe escapes.
IX_DEV void split_exit_channel(PathState& P, const DevScene& S, const float4* planes, V3 hit,
                               int k, V3 dir_k, float transmitted_i) {
    V3 o = hit + dir_k * 1e-4f;
    Hit h = intersect_planes(planes, (int)S.s.n_planes, o, dir_k);
    if (h.facet >= 0) return;
    const ix_environment& env = S.s.environment;
    Lighting L = direction_lighting(env, dir_k, P.observer);
    float e = lighting_radiance(L, env, spectral_power(env, P.lambdas[k]));
    P.split[k] = fmaf(fmaxf(transmitted_i, 0.0f), e, P.split[k]);
}

// Beer-Lambert for an isotropic material (raytracer/absorption.rs:99, :197): the channel
// alpha is the midpoint of the absorption tensor's quadratic form over the two
// eigen-polarisations of the wave normal.
IX_DEV void isotropic_absorption(PathState& P, const DevScene& S, V3 k_hat, float len) {
    const ix_material& m = S.s.material;
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
    float qa0 = la0 * la0, qa1 = la1 * la1, qa2 = la2 * la2;
    float qb0 = lb0 * lb0, qb1 = lb1 * lb1, qb2 = lb2 * lb2;
    float scaled = len * m.absorption_path_scale;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float ao = P.alpha[k];
        float qa = (ao * qa0 + ao * qa1) + ao * qa2;
        float qb = (ao * qb0 + ao * qb1) + ao * qb2;
        float alpha = midpointf_(qa, qb);
        P.st[k] = scale(P.st[k], exp_lane(-alpha * scaled));
    }
}

// tir_phase_delta (refraction/tir.rs:33).
IX_DEV float tir_phase_delta(float n1k, float cos_i, float sin_i) {
    float tan_half = (cos_i * sqrtf(fmaxf(fmaf(n1k * n1k * sin_i, sin_i, -1.0f), 0.0f))) /
                     fmaxf(n1k * sin_i * sin_i, 1e-6f);
    return 2.0f * atanf(tan_half);
}
IX_DEV void fresnel_rs_rp(float n1, float n2, float cos_i, float cos_t, float& r_s, float& r_p) {
    r_s = fmaf(n2, -cos_t, n1 * cos_i) / fmaf(n2, cos_t, n1 * cos_i);
    r_p = fmaf(n1, -cos_t, n2 * cos_i) / fmaf(n1, cos_t, n2 * cos_i);
}
IX_DEV float r_unpol_of(float r_s, float r_p) { return 0.5f * fmaf(r_p, r_p, r_s * r_s); }

enum BounceResult { BOUNCE_CONTINUE = 0, BOUNCE_ESCAPED = 1, BOUNCE_KILLED = 2 };

// One iteration of the bounce loop (bounce_body.rs:361-423 and facet_event :611-707).
// On BOUNCE_ESCAPED, `env_out` holds the escape radiance per channel already weighted by
// the channel's Stokes intensity (accumulate_miss_radiance, transport/bounce.rs:40).
IX_DEV int path_bounce(PathState& P, const DevScene& S, const float4* __restrict__ planes,
                       float env_out[8]) {
    const ix_scene& sc = S.s;
    const uint32_t bounce = P.bounce;
    Hit hit = intersect_planes(planes, (int)sc.n_planes, P.o, P.d);
    if (hit.facet < 0) {
        const ix_environment& env = sc.environment;
        Lighting L = direction_lighting(env, P.d, P.observer);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float e = lighting_radiance(L, env, spectral_power(env, P.lambdas[k]));
            env_out[k] = fmaf(intensity(P.st[k]), e, 0.0f);
        }
        return BOUNCE_ESCAPED;
    }
    float4 pl = planes[hit.facet];
    V3 normal = v3(pl.x, pl.y, pl.z);
    V3 hit_point = P.o + hit.t * P.d;
    const V3 k_hat = P.d;  // isotropic: wave normal == ray direction

    // rotate_stokes_to_plane_of_incidence (raytracer/absorption.rs:69).
    V3 cpn = normalize_or_zero(cross(k_hat, normal));
    if (P.has_prev && length_squared(cpn) > 1e-6f && length_squared(P.prev_pn) > 1e-6f) {
        float cos_psi = clampf_(dot(P.prev_pn, cpn), -1.0f, 1.0f);
        float sin_psi = dot(cross(P.prev_pn, cpn), normalize_or_zero(k_hat));
        float psi = atan2f(sin_psi, cos_psi);
        float s2, c2;
        sincosf(2.0f * psi, &s2, &c2);
#pragma unroll
        for (int k = 0; k < 8; ++k) P.st[k] = rotate(P.st[k], c2, s2);
    }
    P.has_prev = true;
    P.prev_pn = cpn;

    // apply_interior_segment (transport/inner.rs:170).
    if (P.inside) {
        normal = -normal;
        if (S.absorbing) isotropic_absorption(P, S, k_hat, hit.t);
    }

    // compute_bounce_refraction_geometry (refraction/geometry.rs:306), isotropic.
    const float cos_i = clampf_(dot(-k_hat, normal), 0.0f, 1.0f);
    const float one_m_c2 = fmaf(cos_i, -cos_i, 1.0f);
    const float sin_i = sqrtf(fmaxf(one_m_c2, 0.0f));
    const float n1 = P.inside ? P.n_ch[0] : 1.0f;
    const float n2 = P.inside ? 1.0f : P.n_ch[0];
    const float eta = n1 / n2;
    const float sin2_t = eta * eta * one_m_c2;

    V3 new_dir;
    bool new_inside = P.inside;
    if (sin2_t > 1.0f) {
        // apply_tir_bounce, isotropic arm (refraction/tir.rs:98-116).
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float n1k = P.inside ? P.n_ch[k] : 1.0f;
            float n2k = P.inside ? 1.0f : P.n_ch[k];
            float etak = n1k / n2k;
            float s2k = etak * etak * one_m_c2;
            if (s2k > 1.0f) {
                P.st[k] = tir_retard_apply(P.st[k], tir_phase_delta(n1k, cos_i, sin_i));
            } else {
                float cos_t_k = sqrtf(fmaxf(1.0f - s2k, 0.0f));
                float r_s, r_p;
                fresnel_rs_rp(n1k, n2k, cos_i, cos_t_k, r_s, r_p);
                P.st[k] = fresnel_reflect_apply(P.st[k], r_s, r_p);
                P.pdf[k] = P.pdf[k] * clampf_(r_unpol_of(r_s, r_p), R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
            }
        }
        new_dir = k_hat - 2.0f * dot(k_hat, normal) * normal;
    } else {
        // apply_partial_fresnel_bounce (refraction/dispatch.rs:307).
        float cos_t = sqrtf(fmaxf(1.0f - sin2_t, 0.0f));
        float r_s, r_p;
        fresnel_rs_rp(n1, n2, cos_i, cos_t, r_s, r_p);
        const float r_unpol = clampf_(r_unpol_of(r_s, r_p), R_UNPOL_SELECT_MIN, R_UNPOL_SELECT_MAX);
        const float rng = unit_draw(P.seed, bounce, FRESNEL_BRANCH_STREAM);
        if (rng < r_unpol) {
            // apply_partial_reflect_bounce (reflect_refract.rs:33).
            const float inv = 1.0f / r_unpol;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                float n1k = P.inside ? P.n_ch[k] : 1.0f;
                float n2k = P.inside ? 1.0f : P.n_ch[k];
                float etak = n1k / n2k;
                float s2k = etak * etak * one_m_c2;
                Stokes s;
                if (s2k > 1.0f) {
                    s = tir_retard_apply(P.st[k], tir_phase_delta(n1k, cos_i, sin_i));
                } else {
                    float cos_t_k = sqrtf(fmaxf(1.0f - s2k, 0.0f));
                    float rs, rp;
                    fresnel_rs_rp(n1k, n2k, cos_i, cos_t_k, rs, rp);
                    P.pdf[k] = P.pdf[k] * clampf_(r_unpol_of(rs, rp), R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
                    s = fresnel_reflect_apply(P.st[k], rs, rp);
                }
                P.st[k] = scale(s, inv);
            }
            new_dir = k_hat - 2.0f * dot(k_hat, normal) * normal;
        } else {
            // apply_refract_bounce + apply_refract_channel (reflect_refract.rs:121-591).
            float sin2_t_dir = fminf(eta * eta * one_m_c2, 1.0f);
            float cos_t_dir = sqrtf(fmaxf(1.0f - sin2_t_dir, 0.0f));
            V3 final_refr = normalize(eta * k_hat + fmaf(eta, cos_i, -cos_t_dir) * normal);
            const float inv_t = 1.0f / (1.0f - r_unpol);
            V3 dirs[8];
            uint32_t have_dir = 0, hero_match = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                float n1k = P.inside ? P.n_ch[k] : 1.0f;
                float n2k = P.inside ? 1.0f : P.n_ch[k];
                float ratio = n1k / n2k;
                float s2k = (ratio * ratio) * one_m_c2;
                dirs[k] = v3(0.0f, 0.0f, 0.0f);
                if (s2k > 1.0f) {
                    P.st[k] = scale(P.st[k], 0.0f);
                    P.pdf[k] = 0.0f;
                    continue;
                }
                float cos_t_k = sqrtf(fmaxf(1.0f - s2k, 0.0f));
                V3 refr_k = normalize(ratio * k_hat + fmaf(ratio, cos_i, -cos_t_k) * normal);
                bool match = dot(refr_k, final_refr) >= DIRECTION_MATCH_COS_TOL;
                float two = 2.0f * n1k * cos_i;
                float t_s = two / fmaf(n2k, cos_t_k, n1k * cos_i);
                float t_p = two / fmaf(n1k, cos_t_k, n2k * cos_i);
                Stokes original = P.st[k];
                Stokes transmitted =
                    scale(fresnel_transmit_apply(original, n1k, n2k, cos_i, cos_t_k, t_s, t_p), inv_t);
                float rs, rp;
                fresnel_rs_rp(n1k, n2k, cos_i, cos_t_k, rs, rp);
                float r_unpol_k = clampf_(r_unpol_of(rs, rp), R_UNPOL_PDF_MIN, R_UNPOL_PDF_MAX);
                P.pdf[k] = P.pdf[k] * (1.0f - r_unpol_k);
                if (match) {
                    P.st[k] = transmitted;
                } else {
                    // apply_channel_chromatic_termination (reflect_refract.rs:444).
                    P.st[k] = scale(P.st[k], 0.0f);
                    if (P.inside && intensity(original) > 0.0f)
                        split_exit_channel(P, S, planes, hit_point, k, refr_k, intensity(transmitted));
                }
                dirs[k] = refr_k;
                have_dir |= 1u << k;
                hero_match |= (match ? 1u : 0u) << k;
            }
            if (!P.inside) {
                // narrow_compat (refraction/context.rs:219), hero channel 0.
#pragma unroll
                for (int a = 0; a < 8; ++a)
#pragma unroll
                    for (int b = a + 1; b < 8; ++b) {
                        bool m;
                        if (a == 0)
                            m = (hero_match >> b) & 1u;
                        else if (((have_dir >> a) & 1u) && ((have_dir >> b) & 1u))
                            m = dot(dirs[a], dirs[b]) >= DIRECTION_MATCH_COS_TOL;
                        else
                            m = true;
                        if (!m) {
                            compat_clear_bit(P, a, b);
                            compat_clear_bit(P, b, a);
                        }
                    }
            }
            new_dir = final_refr;
            new_inside = !P.inside;
        }
    }
    P.d = new_dir;
    P.o = hit_point + new_dir * 1e-4f;
    P.inside = new_inside;

    // Surface glare (bounce_body.rs:691-697).
    const float glare = clampf_(sc.environment.surface_glare, 0.0f, 1.0f);
    if (bounce == 0 && !P.inside && glare < 1.0f) {
#pragma unroll
        for (int k = 0; k < 8; ++k) P.st[k] = scale(P.st[k], glare);
    }
    // apply_russian_roulette (transport/bounce.rs:355).
    if (bounce > 4) {
        float max_i = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) max_i = fmaxf(max_i, intensity(P.st[k]));
        float q = clampf_(max_i, 0.05f, 1.0f);
        float rr = unit_draw(P.seed, bounce, RUSSIAN_ROULETTE_STREAM);
        if (rr > q) return BOUNCE_KILLED;
        float inv_q = 1.0f / q;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            P.st[k] = scale(P.st[k], inv_q);
            P.split[k] = P.split[k] / q;
        }
    }
    P.bounce = bounce + 1;
    return BOUNCE_CONTINUE;
}

// finish (bounce_body.rs:724-764): commit the exit splits of an escaped path, integrate
// each channel over its MIS family (optics/raytracer/color.rs:145), apply the Bradford
// round trip for studio environments (color.rs:252) and floor at zero.
IX_DEV V3 path_finish(const PathState& P, const DevScene& S, bool escaped, const float env_i[8]) {
    const float norm_factor = 50.0f / 106.856f;
    float x = 0.0f, y = 0.0f, z = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        uint32_t ck = compat_get(P, k);
        float family = 0.0f;
        bool first = true;
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (ck & (1u << j)) {
                family = first ? P.pdf[j] : family + P.pdf[j];
                first = false;
            }
        float w = (family <= 1e-12f) ? 1.0f : (8.0f * P.pdf[0]) / family;
        float rad = escaped ? env_i[k] + P.split[k] : 0.0f;
        float weighted = rad * w;
        V3 c = cmf(P.lambdas[k]);
        float s = weighted * norm_factor;
        x = x + c.x * s;
        y = y + c.y * s;
        z = z + c.z * s;
    }
    x = x + 0.0f;
    y = y + 0.0f;
    z = z + 0.0f;
    const ix_environment& env = S.s.environment;
    if (env.model != IX_ENV_UNIFORM) {
        float l = fmaf(0.8951f, x, fmaf(0.2664f, y, -0.1614f * z));
        float m = fmaf(-0.7502f, x, fmaf(1.7135f, y, 0.0367f * z));
        float s = fmaf(0.0389f, x, fmaf(-0.0685f, y, 1.0296f * z));
        if (env.white_balance) {
            l = l * env.wb_lms[0];
            m = m * env.wb_lms[1];
            s = s * env.wb_lms[2];
        } else {
            l = l * 1.0f;
            m = m * 1.0f;
            s = s * 1.0f;
        }
        x = fmaf(0.986993f, l, fmaf(-0.147054f, m, 0.159963f * s));
        y = fmaf(0.432305f, l, fmaf(0.518360f, m, 0.049291f * s));
        z = fmaf(-0.008529f, l, fmaf(0.040043f, m, 0.968487f * s));
    }
    return v3(fmaxf(x, 0.0f), fmaxf(y, 0.0f), fmaxf(z, 0.0f));
}

}  // namespace ix
