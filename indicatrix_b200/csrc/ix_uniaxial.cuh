// ix_uniaxial.cuh -- uniaxial birefringence on the device (sm_100a).
//
// The closed-form isotropic/uniaxial interface solution the reference ships
// (optics/raytracer/uniaxial_fresnel/*.rs, after Lekner, J. Phys.: Condens. Matter 3
// (1991) 6121): the ordinary/extraordinary wavevector roots, the mode fields, the 4x4
// complex boundary-matching system and its Gauss-Jordan solve, the Jones-to-Mueller
// conversion, plus the walk-off and eigen-polarisation helpers of
// optics/birefringence/uniaxial.rs.  In the group transport each lane solves its own
// channel's interface; the hero's solve is lane 0's.
//
// The 4x4 systems live in registers: every loop is unrolled, and the partial-pivoting
// row swap is a select over the (compile-time) candidate rows, so no array is ever
// indexed by a run-time value.
#pragma once

#include "ix_device.cuh"

namespace ix {

constexpr uint32_t BIREFRINGENT_SPLIT_STREAM = 0x2545F491u;  // sampling.rs:17
constexpr uint32_t MODE_COUPLING_STREAM = 0xCC9E2D51u;       // sampling.rs:21

// ------------------------------------------------------------------------------------
// Birefringence helpers (birefringence/uniaxial.rs, helpers.rs, absorption_tensor.rs).
// ------------------------------------------------------------------------------------
// extraordinary_index_at (materials/optics.rs:42).
IX_DEV float extraordinary_index_at(const ix_material& m, float lambda_nm, float n_o) {
    if (m.has_e_dispersion) return dispersion_eval(m.e_dispersion, lambda_nm);
    return n_o + m.birefringence_delta;
}
// stable_orthonormal_basis (birefringence/helpers.rs:13), first vector.
IX_DEV V3 stable_basis_t(V3 n) {
    V3 a = (fabsf(n.x) > 0.9f) ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    return normalize_or_zero(a - n * dot(n, a));
}
// The angle theta_c between the wave normal and the optic axis, carried as the |cos| it
// is taken from (geometry.rs:108, :118).  The exact build forms theta = acos(|cos|) and
// later its sincos as the reference does; the fast build keeps cos and forms
// sin = sqrt(1 - cos^2) from it (no transcendental).
struct ThetaC {
    float theta, cos_abs;
};
IX_DEV ThetaC theta_from_cos(float cos_abs) {
#if IX_EXACT
    return ThetaC{acosf(cos_abs), cos_abs};
#else
    return ThetaC{0.0f, cos_abs};
#endif
}
// effective_extraordinary_index (uniaxial.rs:33).
IX_DEV float effective_extraordinary_index(float n_o, float n_e, ThetaC th) {
    if (fabsf(n_o - n_e) < 1e-5f) return n_o;
    float sin_t, cos_t;
#if IX_EXACT
    sincosf(th.theta, &sin_t, &cos_t);
#else
    cos_t = th.cos_abs;
    sin_t = sqrtf(fmaxf(fmaf(-cos_t, cos_t, 1.0f), 0.0f));
#endif
    float ns = n_o * sin_t;
    float denom_sq = fmaf(n_e * cos_t, n_e * cos_t, ns * ns);
    if (denom_sq <= 1e-8f) return n_o;
    return (n_o * n_e) / sqrtf(denom_sq);
}
// walk_off_from_sin_cos (uniaxial.rs:56).
IX_DEV float walk_off_from_sin_cos(float n_o, float n_e, float sin_t, float cos_t) {
    if (fabsf(n_o - n_e) < 1e-5f) return 0.0f;
    float n_o2 = n_o * n_o;
    float n_e2 = n_e * n_e;
    float tan_rho = (((n_o2 - n_e2) * sin_t) * cos_t) / fmaxf(fmaf(n_e2 * cos_t, cos_t, (n_o2 * sin_t) * sin_t), 1e-6f);
    return atanf(tan_rho);
}
// extraordinary_poynting_dir (uniaxial.rs:72): the walked-off energy direction.
IX_DEV V3 extraordinary_poynting_dir(V3 w, V3 c, float n_o, float n_e) {
    float cos_theta = clampf_(dot(w, c), -1.0f, 1.0f);
    float abs_cos = fabsf(cos_theta);
    float sin_t = sqrtf(fmaxf((1.0f - abs_cos) * (1.0f + abs_cos), 0.0f));
    float delta = walk_off_from_sin_cos(n_o, n_e, sin_t, abs_cos);
    if (fabsf(delta) < 1e-5f) return w;
    V3 c_proj = normalize_or_zero(c - cos_theta * w);
    if (length_squared(c_proj) < 1e-6f) return w;
    float sign = (cos_theta >= 0.0f) ? 1.0f : -1.0f;
    float sd, cd;
    sincosf(delta, &sd, &cd);
    return normalize_dir(w * cd - (sign * c_proj) * sd);  // compared in the match test
}
// ordinary_eigen_polarization (uniaxial.rs:95).
IX_DEV V3 ordinary_eigen_polarization(V3 w, V3 c) {
    V3 cr = cross(w, c);
    if (length_squared(cr) > 1e-8f) return normalize(cr);
    return stable_basis_t(normalize_or_zero(w));
}
// assigned_mode_e_field_uniaxial (absorption_tensor.rs:144).
IX_DEV V3 assigned_mode_e_field(V3 k, V3 c, bool is_e, float n_o_hero, float n_e_hero) {
    if (!is_e) return ordinary_eigen_polarization(k, c);
    V3 kc = cross(k, c);
    if (length_squared(kc) < 1e-8f) return normalize_or_zero(cross(k, ordinary_eigen_polarization(k, c)));
    return normalize(cross(kc, extraordinary_poynting_dir(k, c, n_o_hero, n_e_hero)));
}
// AbsorptionTensor3::uniaxial(ao, ae, c).quadratic_form(e) (absorption_tensor.rs:39, :80).
IX_DEV float absorption_quadratic_form(V3 c_axis, float ao, float ae, V3 e) {
    V3 c = normalize_or_zero(c_axis);
    V3 a1 = stable_basis_t(c);
    V3 a2 = cross(c, a1);
    float l0 = dot(a1, e), l1 = dot(a2, e), l2 = dot(c, e);
    return (ao * (l0 * l0) + ao * (l1 * l1)) + ae * (l2 * l2);
}

// ------------------------------------------------------------------------------------
// Complex scalars and 3-vectors (uniaxial_fresnel/complex.rs).
// ------------------------------------------------------------------------------------
struct Cx {
    float re, im;
};
IX_DEV Cx cx(float re, float im) { return Cx{re, im}; }
IX_DEV Cx cadd(Cx a, Cx b) { return cx(a.re + b.re, a.im + b.im); }
IX_DEV Cx csub(Cx a, Cx b) { return cx(a.re - b.re, a.im - b.im); }
IX_DEV Cx cmul(Cx a, Cx b) { return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
IX_DEV Cx cscale(Cx a, float s) { return cx(a.re * s, a.im * s); }
IX_DEV Cx cconj(Cx a) { return cx(a.re, -a.im); }
IX_DEV Cx cneg(Cx a) { return csub(cx(0.0f, 0.0f), a); }
IX_DEV float cnorm2(Cx a) { return fmaf(a.im, a.im, a.re * a.re); }
// Cplx::div (complex.rs:79).  The fast build takes one reciprocal of the divisor's
// squared norm for both components.
IX_DEV Cx cdiv(Cx a, Cx o) {
    float denom = fmaxf(fmaf(o.im, o.im, o.re * o.re), 1e-20f);
#if IX_EXACT
    return cx(fmaf(a.im, o.im, a.re * o.re) / denom, fmaf(a.re, -o.im, a.im * o.re) / denom);
#else
    const float inv = 1.0f / denom;
    return cx(fmaf(a.im, o.im, a.re * o.re) * inv, fmaf(a.re, -o.im, a.im * o.re) * inv);
#endif
}
// Cplx::sqrt_forward_branch (complex.rs:109): the root with re > 0, or im > 0 when
// evanescent; a pure negative real takes sqrt(-re) directly.  The exact build forms the
// polar root as the reference does (|z|^(1/2) at half the atan2 angle); the fast build
// uses the algebraic principal root, re = sqrt((|z| + x) / 2), im = y / (2 re) (for
// x < 0 the mirrored form, free of cancellation), which is the same branch: re >= 0 and
// im with the sign of y.
IX_DEV Cx csqrt_fwd(Cx a) {
    if (a.im == 0.0f && a.re < 0.0f) return cx(0.0f, sqrtf(-a.re));
#if IX_EXACT
    float r = sqrtf(sqrtf(cnorm2(a)));
    float theta = atan2f(a.im, a.re) * 0.5f;
    float st, ct;
    sincosf(theta, &st, &ct);
    Cx out = cx(r * ct, r * st);
#else
    const float m = sqrtf(cnorm2(a));
    Cx out;
    if (a.re >= 0.0f) {
        const float re = sqrtf(0.5f * (m + a.re));
        out = cx(re, re > 0.0f ? a.im / (2.0f * re) : 0.0f);
    } else {
        const float im = sqrtf(0.5f * (m - a.re));
        out = cx(fabsf(a.im) / (2.0f * im), copysignf(im, a.im));
    }
#endif
    if (out.re < 0.0f) out = cx(-out.re, -out.im);
    if (fabsf(out.re) < 1e-9f && out.im < 0.0f) out = cx(-out.re, -out.im);
    return out;
}
struct CV3 {
    V3 re, im;
};
IX_DEV CV3 cv_real(V3 v) { return CV3{v, v3(0.0f, 0.0f, 0.0f)}; }
IX_DEV CV3 cv_wavevector(V3 that, V3 zhat, float tangential, Cx q) {
    return CV3{that * tangential + zhat * q.re, zhat * q.im};
}
IX_DEV CV3 cv_add(CV3 a, CV3 b) { return CV3{a.re + b.re, a.im + b.im}; }
IX_DEV CV3 cv_scale_real(CV3 a, float s) { return CV3{a.re * s, a.im * s}; }
IX_DEV CV3 cv_scale(CV3 a, Cx s) { return CV3{a.re * s.re - a.im * s.im, a.re * s.im + a.im * s.re}; }
IX_DEV CV3 cv_cross_real(CV3 a, V3 r) { return CV3{cross(a.re, r), cross(a.im, r)}; }
IX_DEV CV3 cv_cross(CV3 a, CV3 b) {
    return CV3{cross(a.re, b.re) - cross(a.im, b.im), cross(a.re, b.im) + cross(a.im, b.re)};
}
IX_DEV Cx cv_dot_real(CV3 a, V3 r) { return cx(dot(a.re, r), dot(a.im, r)); }
IX_DEV CV3 cv_conj(CV3 a) { return CV3{a.re, -a.im}; }

// ------------------------------------------------------------------------------------
// Incidence frame, q-roots and mode fields (uniaxial_fresnel/frame.rs).
// ------------------------------------------------------------------------------------
struct UFrame {
    V3 that, zhat, s_axis;
    float cos_i, sin_i, alpha, beta, gamma;
};
// UniaxialFrame::build (frame.rs:55).
IX_DEV UFrame uframe_build(V3 k, V3 normal, V3 c, float cos_i, float sin_i) {
    UFrame f;
    f.zhat = -normal;
    if (sin_i > 1e-5f) {
        V3 t = k + normal * cos_i;
        f.that = normalize_or_zero(v3(t.x / sin_i, t.y / sin_i, t.z / sin_i));
    } else {
        V3 fb = (fabsf(f.zhat.x) < 0.9f) ? v3(1.0f, 0.0f, 0.0f) : v3(0.0f, 1.0f, 0.0f);
        f.that = normalize_or_zero(fb - f.zhat * dot(f.zhat, fb));
    }
    V3 s = normalize_or_zero(cross_rn(k, normal));  // uncontracted: exactly zero at normal incidence
    f.s_axis = (length_squared(s) > 1e-8f) ? s : normalize_or_zero(cross(f.zhat, f.that));
    f.cos_i = cos_i;
    f.sin_i = sin_i;
    f.alpha = dot(c, f.that);
    f.beta = dot(c, f.s_axis);
    f.gamma = dot(c, f.zhat);
    return f;
}
struct QRoots {
    Cx qo_plus, qo_minus, qe_plus, qe_minus;
};
// uniaxial_q_roots (frame.rs:111).
IX_DEV QRoots uniaxial_q_roots(float n_o, float n_e, const UFrame& f, float tangential) {
    QRoots r;
    float n_o2 = n_o * n_o;
    float k2 = tangential * tangential;
    r.qo_plus = csqrt_fwd(cx(n_o2 - k2, 0.0f));
    r.qo_minus = cneg(r.qo_plus);
    if (n_o == n_e) {
        r.qe_plus = r.qo_plus;
        r.qe_minus = r.qo_minus;
        return r;
    }
    float n_e2 = n_e * n_e;
    float deleps = n_e2 - n_o2;
    float denom = fmaf(f.gamma * f.gamma, deleps, n_o2);
    float d_val = n_o2 * fmaf(fmaf(f.beta * f.beta, -deleps, n_e2), -k2, n_e2 * fmaf(f.gamma * f.gamma, deleps, n_o2));
    Cx sqrt_d = csqrt_fwd(cx(d_val, 0.0f));
    Cx shift = cx(((f.alpha * f.gamma) * tangential) * deleps, 0.0f);
    Cx denom_c = cx(fmaxf(denom, 1e-12f), 0.0f);
    r.qe_plus = cdiv(csub(sqrt_d, shift), denom_c);
    r.qe_minus = cdiv(csub(cneg(sqrt_d), shift), denom_c);
    return r;
}
// ModeFields (frame.rs:176-232): E and H at amplitude 1.
struct Mode {
    CV3 e, h;
};
IX_DEV Mode ordinary_mode(float n_o, V3 c, const UFrame& f, float tangential, Cx q) {
    CV3 k = cv_wavevector(f.that, f.zhat, tangential, q);
    Mode m;
    m.e = cv_scale_real(cv_cross_real(k, c), 1.0f / (n_o * n_o));
    m.h = cv_cross(k, m.e);
    return m;
}
IX_DEV Mode extraordinary_mode(float n_o, float n_e, V3 c, const UFrame& f, float tangential, Cx q) {
    float n_o2 = n_o * n_o;
    float n_e2 = n_e * n_e;
    float deleps = n_e2 - n_o2;
    CV3 k = cv_wavevector(f.that, f.zhat, tangential, q);
    CV3 d_e = cv_cross(k, cv_cross_real(k, c));
    Cx c_dot_de = cv_dot_real(d_e, c);
    Mode m;
    m.e = cv_add(cv_scale_real(d_e, 1.0f / n_o2), cv_scale(cv_real(c), cscale(c_dot_de, -(deleps / (n_o2 * n_e2)))));
    m.h = cv_cross(k, m.e);
    return m;
}
IX_DEV Mode iso_mode(CV3 k, CV3 e) { return Mode{e, cv_cross(k, e)}; }
// poynting_z (frame.rs:237) at amplitude 1: 0.5 Re(E x H*) . zhat.
IX_DEV float poynting_z(const Mode& m, V3 zhat) {
    const Cx one = cx(1.0f, 0.0f);
    CV3 s = cv_cross(cv_scale(m.e, one), cv_conj(cv_scale(m.h, one)));
    return 0.5f * cv_dot_real(s, zhat).re;
}
// tangential_components (linalg.rs:264).
IX_DEV void tangential(const Mode& m, const UFrame& f, Cx out[4]) {
    out[0] = cv_dot_real(m.e, f.that);
    out[1] = cv_dot_real(m.e, f.s_axis);
    out[2] = cv_dot_real(m.h, f.that);
    out[3] = cv_dot_real(m.h, f.s_axis);
}

// solve4 / solve4_two_rhs (linalg.rs:172, :217): Gauss-Jordan elimination with partial
// pivoting (a later row wins only with a strictly larger |.|^2).  Columns left of the
// pivot are never read again, so the swap only moves columns >= col.
template <int NRHS>
IX_DEV void solve4(Cx a[4][4], Cx b[NRHS][4]) {
#pragma unroll
    for (int col = 0; col < 4; ++col) {
        int piv = col;
        float piv_mag = cnorm2(a[col][col]);
#pragma unroll
        for (int row = col + 1; row < 4; ++row) {
            float mag = cnorm2(a[row][col]);
            if (mag > piv_mag) {
                piv = row;
                piv_mag = mag;
            }
        }
#pragma unroll
        for (int row = col + 1; row < 4; ++row) {
            const bool sw = piv == row;
#pragma unroll
            for (int j = col; j < 4; ++j) {
                Cx x = a[col][j], y = a[row][j];
                a[col][j] = sw ? y : x;
                a[row][j] = sw ? x : y;
            }
#pragma unroll
            for (int r = 0; r < NRHS; ++r) {
                Cx x = b[r][col], y = b[r][row];
                b[r][col] = sw ? y : x;
                b[r][row] = sw ? x : y;
            }
        }
        const Cx pivot = a[col][col];
#if IX_EXACT
#pragma unroll
        for (int j = col; j < 4; ++j) a[col][j] = cdiv(a[col][j], pivot);
#pragma unroll
        for (int r = 0; r < NRHS; ++r) b[r][col] = cdiv(b[r][col], pivot);
#else
        // One complex reciprocal of the pivot scales the whole row.
        const float inv = 1.0f / fmaxf(cnorm2(pivot), 1e-20f);
        const Cx rp = cx(pivot.re * inv, -pivot.im * inv);
#pragma unroll
        for (int j = col; j < 4; ++j) a[col][j] = cmul(a[col][j], rp);
#pragma unroll
        for (int r = 0; r < NRHS; ++r) b[r][col] = cmul(b[r][col], rp);
#endif
#pragma unroll
        for (int row = 0; row < 4; ++row) {
            if (row == col) continue;
            const Cx factor = a[row][col];
            if (cnorm2(factor) == 0.0f) continue;
#pragma unroll
            for (int j = col; j < 4; ++j) a[row][j] = csub(a[row][j], cmul(factor, a[col][j]));
#pragma unroll
            for (int r = 0; r < NRHS; ++r) b[r][row] = csub(b[r][row], cmul(factor, b[r][col]));
        }
    }
}

// ------------------------------------------------------------------------------------
// The two interfaces (uniaxial_fresnel/entry.rs, internal.rs).
// ------------------------------------------------------------------------------------
// EntryIncidenceFrame (entry.rs:95-147): the air-side s/p modes' tangential components,
// independent of the channel.
struct EntryInc {
    Cx inc_s[4], inc_p[4], refl_s[4], refl_p[4];
};
IX_DEV EntryInc entry_incidence_frame(float n1, const UFrame& f) {
    const float k_tan = n1 * f.sin_i;
    CV3 k_fwd = cv_wavevector(f.that, f.zhat, k_tan, cx(n1 * f.cos_i, 0.0f));
    CV3 k_bwd = cv_wavevector(f.that, f.zhat, k_tan, cx(-n1 * f.cos_i, 0.0f));
    CV3 s_c = cv_real(f.s_axis);
    CV3 ep_bwd = cv_scale_real(cv_cross(k_bwd, s_c), -1.0f / (n1 * n1));
    CV3 ep_fwd = cv_scale_real(cv_cross(k_fwd, s_c), -1.0f / (n1 * n1));
    EntryInc e;
    tangential(iso_mode(k_fwd, s_c), f, e.inc_s);
    tangential(iso_mode(k_fwd, ep_fwd), f, e.inc_p);
    tangential(iso_mode(k_bwd, s_c), f, e.refl_s);
    tangential(iso_mode(k_bwd, ep_bwd), f, e.refl_p);
    return e;
}
// EntryPolarizationSolution for s ([0]) and p ([1]) incidence (entry.rs:23).
struct EntrySol {
    Cx r_s[2], r_p[2], t_o[2], t_e[2];
    float flux_o, flux_e;
    V3 o_hat, e_hat;
};
// entry_solve_pair_with_incidence (entry.rs:173).
IX_DEV EntrySol entry_solve(const EntryInc& inc, float n1, float n_o, float n_e, V3 c, const UFrame& f) {
    const float k_tan = n1 * f.sin_i;
    QRoots q = uniaxial_q_roots(n_o, n_e, f, k_tan);
    Mode fo = ordinary_mode(n_o, c, f, k_tan, q.qo_plus);
    Mode fe = extraordinary_mode(n_o, n_e, c, f, k_tan, q.qe_plus);
    Cx oc[4], ec[4];
    tangential(fo, f, oc);
    tangential(fe, f, ec);
    Cx a[4][4], b[2][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        a[i][0] = inc.refl_s[i];
        a[i][1] = inc.refl_p[i];
        a[i][2] = cneg(oc[i]);
        a[i][3] = cneg(ec[i]);
        b[0][i] = cneg(inc.inc_s[i]);
        b[1][i] = cneg(inc.inc_p[i]);
    }
    solve4<2>(a, b);
    EntrySol s;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        s.r_s[p] = b[p][0];
        s.r_p[p] = b[p][1];
        s.t_o[p] = b[p][2];
        s.t_e[p] = b[p][3];
    }
    s.flux_o = fabsf(poynting_z(fo, f.zhat));
    s.flux_e = fabsf(poynting_z(fe, f.zhat));
    s.o_hat = normalize_or_zero(fo.e.re);
    s.e_hat = normalize_or_zero(fe.e.re);
    return s;
}
// InternalPolarizationSolution (internal.rs:265).
struct IntSol {
    Cx r_o, r_e, t_s, t_p;
    float flux_ro, flux_re, flux_ts, flux_tp, flux_inc;
};
// internal_solve (internal.rs:334): crystal (incident mode o or e) to air (n2 = 1).
IX_DEV IntSol internal_solve(float n_mode_inc, float n_o, float n_e, V3 c, const UFrame& f, bool inc_ordinary) {
    const float k_tan = n_mode_inc * f.sin_i;
    QRoots q = uniaxial_q_roots(n_o, n_e, f, k_tan);
    Mode f_inc = inc_ordinary ? ordinary_mode(n_o, c, f, k_tan, q.qo_plus)
                              : extraordinary_mode(n_o, n_e, c, f, k_tan, q.qe_plus);
    Mode f_o_bwd = ordinary_mode(n_o, c, f, k_tan, q.qo_minus);
    Mode f_e_bwd = extraordinary_mode(n_o, n_e, c, f, k_tan, q.qe_minus);
    const float n2 = 1.0f;
    const float zeta = k_tan / n2;
    const Cx cos_t = (fabsf(zeta) <= 1.0f) ? cx(sqrtf(fmaxf(fmaf(zeta, -zeta, 1.0f), 0.0f)), 0.0f)
                                           : cx(0.0f, sqrtf(fmaf(zeta, zeta, -1.0f)));
    CV3 k_iso = cv_wavevector(f.that, f.zhat, k_tan, cscale(cos_t, n2));
    CV3 s_c = cv_real(f.s_axis);
    CV3 ep_t = cv_scale_real(cv_cross(k_iso, s_c), -1.0f / (n2 * n2));
    Mode f_s_t = iso_mode(k_iso, s_c);
    Mode f_p_t = iso_mode(k_iso, ep_t);
    Cx inc_c[4], eo_c[4], ee_c[4], es_c[4], ep_c[4];
    tangential(f_inc, f, inc_c);
    tangential(f_o_bwd, f, eo_c);
    tangential(f_e_bwd, f, ee_c);
    tangential(f_s_t, f, es_c);
    tangential(f_p_t, f, ep_c);
    Cx a[4][4], b[1][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        a[i][0] = eo_c[i];
        a[i][1] = ee_c[i];
        a[i][2] = cneg(es_c[i]);
        a[i][3] = cneg(ep_c[i]);
        b[0][i] = cneg(inc_c[i]);
    }
    solve4<1>(a, b);
    IntSol s;
    s.r_o = b[0][0];
    s.r_e = b[0][1];
    s.t_s = b[0][2];
    s.t_p = b[0][3];
    s.flux_ro = fabsf(poynting_z(f_o_bwd, f.zhat));
    s.flux_re = fabsf(poynting_z(f_e_bwd, f.zhat));
    s.flux_ts = fabsf(poynting_z(f_s_t, f.zhat));
    s.flux_tp = fabsf(poynting_z(f_p_t, f.zhat));
    s.flux_inc = fabsf(poynting_z(f_inc, f.zhat));
    return s;
}

// ------------------------------------------------------------------------------------
// Stokes/Mueller integration (uniaxial_fresnel/mueller.rs).
// ------------------------------------------------------------------------------------
// jones_to_mueller (mueller.rs:478) as 16 column-major entries.
struct M4 {
    float c[16];
};
IX_DEV M4 jones_to_mueller(Cx j_ss, Cx j_sp, Cx j_ps, Cx j_pp) {
    float m_ss = cnorm2(j_ss), m_sp = cnorm2(j_sp), m_ps = cnorm2(j_ps), m_pp = cnorm2(j_pp);
    Cx a_ssp = cmul(j_ss, cconj(j_sp));
    Cx a_pep = cmul(j_ps, cconj(j_pp));
    Cx a_plus = cadd(a_ssp, a_pep);
    Cx a_minus = csub(a_ssp, a_pep);
    Cx b_sp = cmul(j_ss, cconj(j_ps));
    Cx b_pp = cmul(j_sp, cconj(j_pp));
    Cx c_sspp = cmul(j_ss, cconj(j_pp));
    Cx c_spps = cmul(j_sp, cconj(j_ps));
    M4 m;
    m.c[0] = 0.5f * (((m_ss + m_ps) + m_sp) + m_pp);
    m.c[1] = 0.5f * (((m_ss - m_ps) + m_sp) - m_pp);
    m.c[2] = b_sp.re + b_pp.re;
    m.c[3] = -(b_sp.im + b_pp.im);
    m.c[4] = 0.5f * (((m_ss + m_ps) - m_sp) - m_pp);
    m.c[5] = midpointf_((m_ss - m_ps) - m_sp, m_pp);
    m.c[6] = b_sp.re - b_pp.re;
    m.c[7] = -(b_sp.im) + b_pp.im;
    m.c[8] = a_plus.re;
    m.c[9] = a_minus.re;
    m.c[10] = c_sspp.re + c_spps.re;
    m.c[11] = -(c_sspp.im + c_spps.im);
    m.c[12] = a_plus.im;
    m.c[13] = a_minus.im;
    m.c[14] = c_sspp.im - c_spps.im;
    m.c[15] = c_sspp.re - c_spps.re;
    return m;
}
// glam Mat4 * Vec4: ((col0 i + col1 q) + col2 u) + col3 v.
IX_DEV Stokes apply_m4(const M4& m, const Stokes& s) {
    return Stokes{((m.c[0] * s.i + m.c[4] * s.q) + m.c[8] * s.u) + m.c[12] * s.v,
                  ((m.c[1] * s.i + m.c[5] * s.q) + m.c[9] * s.u) + m.c[13] * s.v,
                  ((m.c[2] * s.i + m.c[6] * s.q) + m.c[10] * s.u) + m.c[14] * s.v,
                  ((m.c[3] * s.i + m.c[7] * s.q) + m.c[11] * s.u) + m.c[15] * s.v};
}
// The unpolarised reflectance, jones_to_mueller(..).col(0)[0] alone.
IX_DEV float jones_r_unpol(Cx j_ss, Cx j_sp, Cx j_ps, Cx j_pp) {
    return 0.5f * (((cnorm2(j_ss) + cnorm2(j_ps)) + cnorm2(j_sp)) + cnorm2(j_pp));
}
// mode_power (mueller.rs:541).
IX_DEV float mode_power(Cx t_s, Cx t_p, float mode_flux, float inc_flux, const Stokes& st) {
    float m_s = cnorm2(t_s);
    float m_p = cnorm2(t_p);
    Cx cr = cmul(t_s, cconj(t_p));
    float raw = fmaf(cr.im, st.v, fmaf(cr.re, st.u, 0.5f * fmaf(m_s, st.i + st.q, m_p * (st.i - st.q))));
    return (mode_flux / fmaxf(inc_flux, 1e-12f)) * raw;
}
// azimuth2_in_frame (mueller.rs:455).
IX_DEV void azimuth2_in_frame(V3 dir, V3 s_axis, V3 p_axis, float& cos2, float& sin2) {
    float s = dot(dir, s_axis);
    float p = dot(dir, p_axis);
    float norm = fmaxf(fmaf(p, p, s * s), 1e-12f);
    cos2 = fmaf(p, -p, s * s) / norm;
    sin2 = ((2.0f * s) * p) / norm;
}
// compute_uniaxial_exit_transmission (refraction/uniaxial_internal.rs:212).
IX_DEV Stokes uniaxial_exit_transmission(const IntSol& sol, float r_branch, float incident_i, float& i_unit) {
    const float flux_inc = fmaxf(sol.flux_inc, 1e-12f);
    Cx ts_n = cscale(sol.t_s, sqrtf(sol.flux_ts / flux_inc));
    Cx tp_n = cscale(sol.t_p, sqrtf(sol.flux_tp / flux_inc));
    i_unit = cnorm2(ts_n) + cnorm2(tp_n);
    float q_unit = cnorm2(ts_n) - cnorm2(tp_n);
    Cx cr = cmul(ts_n, cconj(tp_n));
    return scale(Stokes{incident_i * i_unit, incident_i * q_unit, incident_i * (2.0f * cr.re),
                        incident_i * (-2.0f * cr.im)},
                 1.0f / (1.0f - r_branch));
}
// entry_eigenmode_selection (refraction/uniaxial_entry.rs:50); false for None.
IX_DEV bool entry_eigenmode_selection(V3 c, V3 cpn, V3 k, const Stokes& hs, float& p_o, float& cos2, float& sin2) {
    if (hs.i <= 1e-7f || length_squared(cpn) <= 1e-6f) return false;
    if (fmaf(hs.q, hs.q, hs.u * hs.u) <= 1e-12f) return false;
    V3 o_hat = ordinary_eigen_polarization(k, c);
    V3 p_hat = cross(k, cpn);
    float s_comp = dot(o_hat, cpn);
    float p_comp = dot(o_hat, p_hat);
    cos2 = fmaf(s_comp, s_comp, -(p_comp * p_comp));
    sin2 = (2.0f * s_comp) * p_comp;
    p_o = clampf_(0.5f + (0.5f * fmaf(hs.q, cos2, hs.u * sin2)) / hs.i, 0.0f, 1.0f);
    return true;
}

}  // namespace ix
