// ix_biaxial.cuh -- the biaxial optical indicatrix on the device
// (crates/indicatrix/src/optics/birefringence/biaxial.rs, helpers.rs,
// absorption_tensor.rs).  One lane evaluates one channel's indicatrix: n_beta is the
// channel's dispersion index, n_alpha = n_beta - biaxial_delta_beta_alpha and
// n_gamma = n_alpha + birefringence_delta (GemMaterial::biaxial_indicatrix,
// materials/optics.rs:16), all in the principal frame of the gamma axis (the material's
// c_axis completed by stable_orthonormal_basis, from_gamma_axis, biaxial.rs:58), which is
// also the frame of the trichroic absorption tensor.  Operation order follows the
// reference step for step (Fresnel's equation of the wave normals as a quadratic in
// 1/n^2, the cancellation-free discriminant for the eigenvector root, the sign-aligned
// sum of row-pair cross products for the null direction, the fused cross and dot of
// helpers.rs), so the exact build reproduces the CPU bits.
#pragma once

#include "ix_device.cuh"
#include "ix_uniaxial.cuh"

namespace ix {

// The indicatrix is ill-conditioned where two mode indices nearly meet (the eigenvector
// follows the root to 1 / gap, and the quadratic's discriminant is a small difference of
// large terms), so every operation here is rounded individually in both builds: correctly
// rounded products, sums, quotients and square roots (no multiply-add contraction, no
// approximate divide), the reference's own fused multiply-adds as fmaf.  The fast build
// then computes the biaxial functions bit for bit as the exact build does.
IX_DEV float mul_(float a, float b) { return __fmul_rn(a, b); }
IX_DEV float add_(float a, float b) { return __fadd_rn(a, b); }
IX_DEV float sub_(float a, float b) { return __fsub_rn(a, b); }
IX_DEV float div_(float a, float b) { return __fdiv_rn(a, b); }
// f32::midpoint: the sum halved (exactly), rounded once.
IX_DEV float mid_(float a, float b) { return mul_(add_(a, b), 0.5f); }
IX_DEV V3 vadd_(V3 a, V3 b) { return v3(add_(a.x, b.x), add_(a.y, b.y), add_(a.z, b.z)); }
IX_DEV V3 vsub_(V3 a, V3 b) { return v3(sub_(a.x, b.x), sub_(a.y, b.y), sub_(a.z, b.z)); }
IX_DEV V3 vmul_(V3 a, float s) { return v3(mul_(a.x, s), mul_(a.y, s), mul_(a.z, s)); }
IX_DEV float dot_(V3 a, V3 b) { return add_(add_(mul_(a.x, b.x), mul_(a.y, b.y)), mul_(a.z, b.z)); }
IX_DEV V3 cross_(V3 a, V3 b) {
    return v3(sub_(mul_(a.y, b.z), mul_(b.y, a.z)), sub_(mul_(a.z, b.x), mul_(b.z, a.x)),
              sub_(mul_(a.x, b.y), mul_(b.x, a.y)));
}
IX_DEV V3 normalize_(V3 a) { return vmul_(a, div_(1.0f, __fsqrt_rn(dot_(a, a)))); }
IX_DEV V3 normalize_or_zero_(V3 a) {
    const float rcp = div_(1.0f, __fsqrt_rn(dot_(a, a)));
    if (isfinite(rcp) && rcp > 0.0f) return vmul_(a, rcp);
    return v3(0.0f, 0.0f, 0.0f);
}
// stable_orthonormal_basis (helpers.rs:13), first vector.
IX_DEV V3 stable_basis_t_(V3 n) {
    const V3 a = (fabsf(n.x) > 0.9f) ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    return normalize_or_zero_(vsub_(a, vmul_(n, dot_(n, a))));
}

// Principal frame: columns a1 (alpha), a2 (beta), g (gamma).
struct BiaxFrame {
    V3 a1, a2, g;
};
IX_DEV BiaxFrame biax_frame(V3 c_axis) {
    BiaxFrame f;
    f.g = normalize_or_zero_(c_axis);
    f.a1 = stable_basis_t_(f.g);
    f.a2 = cross_(f.g, f.a1);
    return f;
}
struct Indicatrix {
    float na, nb, ng;
};
IX_DEV Indicatrix make_indicatrix(const ix_material& m, float n_beta) {
    Indicatrix I;
    I.nb = n_beta;
    I.na = sub_(n_beta, m.biaxial_delta_beta_alpha);
    I.ng = add_(I.na, m.birefringence_delta);
    return I;
}
// axes.transpose() * v and axes * v (glam Mat3, column order).
IX_DEV V3 biax_local(const BiaxFrame& f, V3 v) { return v3(dot_(f.a1, v), dot_(f.a2, v), dot_(f.g, v)); }
IX_DEV V3 biax_world(const BiaxFrame& f, V3 l) { return vadd_(vadd_(vmul_(f.a1, l.x), vmul_(f.a2, l.y)), vmul_(f.g, l.z)); }
// cross_fma / dot_fma (helpers.rs:42, :52).
IX_DEV V3 cross_fma(V3 a, V3 b) {
    return v3(fmaf(a.y, b.z, -mul_(a.z, b.y)), fmaf(a.z, b.x, -mul_(a.x, b.z)), fmaf(a.x, b.y, -mul_(a.y, b.x)));
}
IX_DEV float dot_fma(V3 a, V3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, mul_(a.z, b.z))); }
// canonicalize_eigenvector_sign (helpers.rs:27): the largest component positive.
IX_DEV V3 canonical_sign(V3 v) {
    const float ax = fabsf(v.x), ay = fabsf(v.y), az = fabsf(v.z);
    const float largest = (ax >= ay && ax >= az) ? v.x : (ay >= az ? v.y : v.z);
    return largest < 0.0f ? -v : v;
}
// indices_are_degenerate (biaxial.rs:176): |a - b| <= sqrt(f32::EPSILON) max(|a|, |b|, 1);
// sqrt(2^-23) correctly rounded to f32 is 0x39B504F3.
IX_DEV bool indices_degenerate(float a, float b) {
    const float scale = fmaxf(fmaxf(fabsf(a), fabsf(b)), 1.0f);
    return fabsf(sub_(a, b)) <= mul_(__uint_as_float(0x39B504F3u), scale);
}
// 1 / n^2 of each principal index (b_coeffs, biaxial.rs:92).
IX_DEV float inv_sq(float n) { return div_(1.0f, mul_(n, n)); }
// BiaxialIndicatrix::wave_indices (biaxial.rs:105): (n_slow, n_fast) at wave normal w.
IX_DEV void wave_indices(const Indicatrix& I, const BiaxFrame& F, V3 w, float& n_slow, float& n_fast) {
    const V3 k = normalize_or_zero_(w);
    const bool ab = indices_degenerate(I.na, I.nb), bg = indices_degenerate(I.nb, I.ng);
    if (ab && bg) {
        n_slow = n_fast = div_(add_(add_(I.na, I.nb), I.ng), 3.0f);
        return;
    }
    if (ab || bg) {
        // uniaxial_wave_indices (biaxial.rs:160): optic axis gamma (n_o = mid(alpha, beta))
        // or alpha (n_o = mid(beta, gamma)).
        const V3 c = ab ? F.g : F.a1;
        const float n_o = ab ? mid_(I.na, I.nb) : mid_(I.nb, I.ng);
        const float n_e = ab ? I.ng : I.na;
        const float n_eff =
            effective_extraordinary_index(n_o, n_e, theta_from_cos(fabsf(clampf_(dot_(k, c), -1.0f, 1.0f))));
        n_slow = fmaxf(n_o, n_eff);
        n_fast = fminf(n_o, n_eff);
        return;
    }
    const V3 l = biax_local(F, k);
    const float a2 = mul_(l.x, l.x), b2 = mul_(l.y, l.y), g2 = mul_(l.z, l.z);
    const float b1 = inv_sq(I.na), b2c = inv_sq(I.nb), b3 = inv_sq(I.ng);
    const float big_b = fmaf(a2, add_(b2c, b3), fmaf(b2, add_(b1, b3), mul_(g2, add_(b1, b2c))));
    const float big_c = fmaf(a2, mul_(b2c, b3), fmaf(b2, mul_(b1, b3), mul_(mul_(g2, b1), b2c)));
    const float disc = __fsqrt_rn(fmaxf(fmaf(big_b, big_b, mul_(-4.0f, big_c)), 0.0f));
    const float x_lo = mul_(0.5f, sub_(big_b, disc));
    const float x_hi = mid_(big_b, disc);
    n_slow = div_(1.0f, __fsqrt_rn(fmaxf(x_lo, 1e-12f)));
    n_fast = div_(1.0f, __fsqrt_rn(fmaxf(x_hi, 1e-12f)));
}
// precise_root_near (biaxial.rs:288).
IX_DEV float precise_root_near(V3 l, float b0, float b1, float b2, float x) {
    const float a = mul_(l.x, l.x), bb = mul_(l.y, l.y), cc = mul_(l.z, l.z);
    const float big_b = fmaf(a, add_(b1, b2), fmaf(bb, add_(b0, b2), mul_(cc, add_(b0, b1))));
    const float xd = sub_(b0, b1), yd = sub_(b2, b0);
    const float a_plus_c = add_(a, cc), a_plus_bb = add_(a, bb);
    const float two_a_minus_bc = mul_(2.0f, fmaf(bb, -cc, a));
    const float disc_sq = fmaf(mul_(a_plus_c, a_plus_c), mul_(xd, xd),
                               fmaf(mul_(a_plus_bb, a_plus_bb), mul_(yd, yd), mul_(mul_(two_a_minus_bc, xd), yd)));
    const float disc = __fsqrt_rn(fmaxf(disc_sq, 0.0f));
    const float x_lo = mul_(0.5f, sub_(big_b, disc));
    const float x_hi = mid_(big_b, disc);
    return fabsf(sub_(x, x_lo)) <= fabsf(sub_(x, x_hi)) ? x_lo : x_hi;
}
// eigen_polarizations (biaxial.rs:197) for one mode, through eigenvector_world
// (biaxial.rs:243): the D direction of the slow (want_slow) or the fast mode.
IX_DEV V3 eigen_polarization(const Indicatrix& I, const BiaxFrame& F, V3 w, bool want_slow) {
    const V3 k = normalize_or_zero_(w);
    const V3 l = biax_local(F, k);
    const float b0 = inv_sq(I.na), b1 = inv_sq(I.nb), b2 = inv_sq(I.ng);
    float ns, nf;
    wave_indices(I, F, w, ns, nf);
    const float n = want_slow ? ns : nf;
    const float x = precise_root_near(l, b0, b1, b2, inv_sq(n));
    const float xx = mul_(l.x, l.x), yy = mul_(l.y, l.y), zz = mul_(l.z, l.z);
    const float s = fmaf(b0, xx, fmaf(b1, yy, mul_(mul_(b2, l.z), l.z)));
    const float m00 = fmaf(xx, fmaf(2.0f, -b0, s), sub_(b0, x));
    const float m11 = fmaf(yy, fmaf(2.0f, -b1, s), sub_(b1, x));
    const float m22 = fmaf(zz, fmaf(2.0f, -b2, s), sub_(b2, x));
    const float m01 = mul_(mul_(l.x, l.y), sub_(sub_(s, b0), b1));
    const float m02 = mul_(mul_(l.x, l.z), sub_(sub_(s, b0), b2));
    const float m12 = mul_(mul_(l.y, l.z), sub_(sub_(s, b1), b2));
    const V3 r0 = v3(m00, m01, m02), r1 = v3(m01, m11, m12), r2 = v3(m02, m12, m22);
    const V3 c01 = cross_fma(r0, r1), c02 = cross_fma(r0, r2), c12 = cross_fma(r1, r2);
    const float s02 = dot_fma(c01, c02) < 0.0f ? -1.0f : 1.0f;
    const float s12 = dot_fma(c01, c12) < 0.0f ? -1.0f : 1.0f;
    const V3 vw = biax_world(F, vadd_(vadd_(c01, vmul_(c02, s02)), vmul_(c12, s12)));
    if (dot_(vw, vw) > 1e-12f) return normalize_(canonical_sign(vw));
    return stable_basis_t_(k);
}
// d_to_e_direction (biaxial.rs:322): E = eps^-1 D in the principal frame.
IX_DEV V3 d_to_e_direction(const Indicatrix& I, const BiaxFrame& F, V3 d) {
    const V3 dl = biax_local(F, d);
    const V3 el = v3(div_(dl.x, mul_(I.na, I.na)), div_(dl.y, mul_(I.nb, I.nb)), div_(dl.z, mul_(I.ng, I.ng)));
    return normalize_or_zero_(biax_world(F, el));
}
// poynting_direction (biaxial.rs:468): k tilted to be perpendicular to E.
IX_DEV V3 poynting_direction(V3 w, V3 e_field) {
    const V3 k = normalize_or_zero_(w);
    const V3 e = normalize_or_zero_(e_field);
    const V3 perp = vsub_(k, vmul_(e, dot_(e, k)));
    const float len2 = dot_(perp, perp);
    if (len2 > 1e-10f) {
        const float len = __fsqrt_rn(len2);
        return v3(div_(perp.x, len), div_(perp.y, len), div_(perp.z, len));
    }
    return k;
}
// mode_poynting_dir (biaxial.rs:420): mode B (is_extraordinary) is the slow mode.
IX_DEV V3 mode_poynting_dir(const Indicatrix& I, const BiaxFrame& F, V3 w, bool want_slow) {
    return poynting_direction(w, d_to_e_direction(I, F, eigen_polarization(I, F, w, want_slow)));
}
// assigned_mode_e_field (biaxial.rs:438).
IX_DEV V3 assigned_mode_e_field_biaxial(const Indicatrix& I, const BiaxFrame& F, V3 w, bool is_e) {
    return d_to_e_direction(I, F, eigen_polarization(I, F, w, is_e));
}
// resolve_entry_mode (biaxial.rs:370): two fixed-point steps of Snell's law against the
// mode's direction-dependent index, seeded with n_seed.  Returns the index; the wave
// normal it was evaluated at goes to `dir`.
IX_DEV float resolve_entry_mode(const Indicatrix& I, const BiaxFrame& F, V3 incident, V3 normal, float cos_i,
                                float n_seed, bool want_slow, V3& dir) {
    float n_guess = n_seed;
    dir = incident;
#pragma unroll 1
    for (int it = 0; it < 2; ++it) {
        const float eta = div_(1.0f, n_guess);
        const float s2 = mul_(mul_(eta, eta), fmaf(cos_i, -cos_i, 1.0f));
        if (s2 > 1.0f) break;
        const float ct = __fsqrt_rn(fmaxf(sub_(1.0f, s2), 0.0f));
        dir = normalize_(vadd_(vmul_(incident, eta), vmul_(normal, fmaf(eta, cos_i, -ct))));
        float ns, nf;
        wave_indices(I, F, dir, ns, nf);
        n_guess = want_slow ? ns : nf;
    }
    return n_guess;
}
// AbsorptionTensor3::biaxial(alpha, beta, gamma, gamma_axis).quadratic_form
// (absorption_tensor.rs:28, :39).
IX_DEV float biaxial_quadratic_form(const BiaxFrame& F, float ao, float ab, float ae, V3 e) {
    const float l0 = dot_(F.a1, e), l1 = dot_(F.a2, e), l2 = dot_(F.g, e);
    return add_(add_(mul_(ao, mul_(l0, l0)), mul_(ab, mul_(l1, l1))), mul_(ae, mul_(l2, l2)));
}

}  // namespace ix
