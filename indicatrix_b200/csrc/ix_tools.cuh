// ix_tools.cuh -- concave tools on the device (crates/indicatrix/src/geometry/tool.rs,
// geometry/tool/interval.rs): the pieces a tool decomposes into (balls, cone frusta, the
// six-plane wedges of an across-axis sweep), each piece's ray interval and signed
// distance, a tool's interval as the hull of its pieces' and its outward normal as the
// nearest piece's.  Every operation is rounded individually in both builds (the
// correctly rounded helpers of ix_biaxial.cuh, the reference's fused multiply-adds as
// fmaf), so a carved stone's boundaries are the CPU's bit for bit and the first boundary
// the carve picks never moves between builds.
#pragma once

#include "ix_biaxial.cuh"
#include "ix_device.cuh"

namespace ix {

enum : uint32_t { TOOL_BALL = 0, TOOL_CYLINDER = 1, TOOL_FRUSTUM = 2, TOOL_BICONE = 3 };
enum : uint32_t { SWEEP_NONE = 0, SWEEP_ALONG = 1, SWEEP_ACROSS = 2 };
enum : int { PIECE_BALL = 0, PIECE_FRUSTUM = 1, PIECE_WEDGE = 2 };
constexpr int MAX_PIECES = 6;

struct Piece {
    int kind;
    V3 c, a, d;
    float r, hl, s, r0, r1;
};
IX_DEV V3 vneg_(V3 a) { return v3(-a.x, -a.y, -a.z); }
IX_DEV Piece ball_piece(V3 c, float r) {
    Piece p{};
    p.kind = PIECE_BALL;
    p.c = c;
    p.r = r;
    return p;
}
IX_DEV Piece frustum_piece(V3 c, V3 a, float hl, float r0, float r1) {
    Piece p{};
    p.kind = PIECE_FRUSTUM;
    p.c = c;
    p.a = a;
    p.hl = hl;
    p.r0 = r0;
    p.r1 = r1;
    return p;
}
// ToolPrimitive::pieces (tool.rs:470).
IX_DEV int tool_pieces(const ix_tool& t, Piece out[MAX_PIECES]) {
    if (t.kind > TOOL_BICONE || t.sweep_kind > SWEEP_ACROSS) return 0;
    const V3 c = v3(t.origin[0], t.origin[1], t.origin[2]), a = v3(t.axis[0], t.axis[1], t.axis[2]);
    const float stroke = t.profile[2];
    const bool swept = t.sweep_kind != SWEEP_NONE && stroke > 0.0f;
    int n = 0;
    if (t.kind == TOOL_BALL) {
        const float r = t.origin[3];
        if (swept) {
            const V3 dir = t.sweep_kind == SWEEP_ALONG ? a : v3(t.sweep_dir[0], t.sweep_dir[1], t.sweep_dir[2]);
            out[n++] = ball_piece(vsub_(c, vmul_(dir, stroke)), r);
            out[n++] = ball_piece(vadd_(c, vmul_(dir, stroke)), r);
            out[n++] = frustum_piece(c, dir, stroke, r, r);
        } else {
            out[n++] = ball_piece(c, r);
        }
        return n;
    }
    // segments (tool.rs:430): (z_lo, z_hi, r_lo, r_hi) along the axis, and the peak.
    const float hl = t.axis[3], rim = t.origin[3], rn = t.profile[0], rp = t.profile[1];
    float seg[2][4];
    int ns = 1;
    float peak_z, peak_r;
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
    const V3 sweep_dir = v3(t.sweep_dir[0], t.sweep_dir[1], t.sweep_dir[2]);
#pragma unroll 1
    for (int i = 0; i < ns; ++i) {
        const float z_mid = mul_(0.5f, add_(seg[i][0], seg[i][1]));
        const float half = mul_(0.5f, sub_(seg[i][1], seg[i][0]));
        const V3 centre = vadd_(c, vmul_(a, z_mid));
        if (!swept) {
            out[n++] = frustum_piece(vadd_(centre, v3(0.0f, 0.0f, 0.0f)), a, half, seg[i][2], seg[i][3]);
        } else if (t.sweep_kind == SWEEP_ALONG) {
            const V3 shift = seg[i][3] >= seg[i][2] ? vmul_(vneg_(a), stroke) : vmul_(a, stroke);
            out[n++] = frustum_piece(vadd_(centre, shift), a, half, seg[i][2], seg[i][3]);
        } else {
            out[n++] = frustum_piece(vadd_(centre, vmul_(vneg_(sweep_dir), stroke)), a, half, seg[i][2], seg[i][3]);
            out[n++] = frustum_piece(vadd_(centre, vmul_(sweep_dir, stroke)), a, half, seg[i][2], seg[i][3]);
            Piece w{};
            w.kind = PIECE_WEDGE;
            w.c = centre;
            w.a = a;
            w.d = sweep_dir;
            w.hl = half;
            w.s = stroke;
            w.r0 = seg[i][2];
            w.r1 = seg[i][3];
            out[n++] = w;
        }
    }
    if (swept && t.sweep_kind == SWEEP_ALONG) out[n++] = frustum_piece(vadd_(c, vmul_(a, peak_z)), a, stroke, peak_r, peak_r);
    return n;
}
// quadratic_roots (interval.rs:8): a t^2 + 2 b t + c = 0 in the stable form.
IX_DEV bool quadratic_roots(float a, float b, float c, float& lo, float& hi) {
    const float disc = fmaf(b, b, -mul_(a, c));
    if (disc <= mul_(1e-7f, fmaf(b, b, fabsf(mul_(a, c))))) return false;
    const float sq = __fsqrt_rn(disc);
    const float q = -add_(b, copysignf(sq, b));
    const float r1 = div_(q, a), r2 = div_(c, q);
    lo = r1 <= r2 ? r1 : r2;
    hi = r1 <= r2 ? r2 : r1;
    return true;
}
IX_DEV bool cap_range(float z0, float dz, float hl, float& s0, float& s1) {
    if (fabsf(dz) > 1e-7f) {
        const float t1 = div_(sub_(-hl, z0), dz), t2 = div_(sub_(hl, z0), dz);
        s0 = t1 <= t2 ? t1 : t2;
        s1 = t1 <= t2 ? t2 : t1;
        return true;
    }
    if (fabsf(z0) <= hl) {
        s0 = -1e30f;
        s1 = 1e30f;
        return true;
    }
    return false;
}
IX_DEV bool clip_range(float lo, float hi, float s0, float s1, float& l, float& h) {
    l = fmaxf(lo, s0);
    h = fminf(hi, s1);
    return l <= h;
}
// The three interval kinds (interval.rs:22, :52, :112).
IX_DEV bool piece_interval(const Piece& pc, V3 ro, V3 rd, float& lo_out, float& hi_out) {
    const V3 o = vsub_(ro, pc.c);
    if (pc.kind == PIECE_BALL)
        return quadratic_roots(dot_(rd, rd), dot_(o, rd), fmaf(pc.r, -pc.r, dot_(o, o)), lo_out, hi_out);
    if (pc.kind == PIECE_FRUSTUM) {
        const float z0 = dot_(o, pc.a), dz = dot_(rd, pc.a);
        float s0, s1;
        if (!cap_range(z0, dz, pc.hl, s0, s1)) return false;
        const float rm = mul_(0.5f, add_(pc.r0, pc.r1));
        const float k = div_(sub_(pc.r1, pc.r0), mul_(2.0f, pc.hl));
        const V3 p = vsub_(o, vmul_(pc.a, z0)), q = vsub_(rd, vmul_(pc.a, dz));
        const float rz0 = fmaf(k, z0, rm);
        const float rate = mul_(k, dz);
        const float qa = fmaf(rate, -rate, dot_(q, q));
        const float qb = fmaf(-rate, rz0, dot_(p, q));
        const float qc = fmaf(rz0, -rz0, dot_(p, p));
        if (fabsf(qa) <= 1e-7f) {
            if (fabsf(qb) <= 1e-7f) {
                if (!(qc <= 0.0f)) return false;
                lo_out = s0;
                hi_out = s1;
                return true;
            }
            const float t = div_(-qc, mul_(2.0f, qb));
            return qb > 0.0f ? clip_range(-1e30f, t, s0, s1, lo_out, hi_out) : clip_range(t, 1e30f, s0, s1, lo_out, hi_out);
        }
        float lo, hi;
        if (!quadratic_roots(qa, qb, qc, lo, hi)) return false;
        if (qa > 0.0f) return clip_range(lo, hi, s0, s1, lo_out, hi_out);
        float xl, xh, yl, yh;
        const bool x = clip_range(-1e30f, lo, s0, s1, xl, xh);
        const bool y = clip_range(hi, 1e30f, s0, s1, yl, yh);
        if (x && y) {
            lo_out = fminf(xl, yl);
            hi_out = fmaxf(xh, yh);
            return true;
        }
        if (x || y) {
            lo_out = x ? xl : yl;
            hi_out = x ? xh : yh;
            return true;
        }
        return false;
    }
    // wedge_interval: six planes about the wedge's frame.
    const V3 w = cross_(pc.a, pc.d);
    const float k = div_(sub_(pc.r1, pc.r0), mul_(2.0f, pc.hl));
    const float rm = mul_(0.5f, add_(pc.r0, pc.r1));
    const V3 ak = vmul_(pc.a, k);
    const V3 fn[6] = {pc.a, vneg_(pc.a), pc.d, vneg_(pc.d), vsub_(w, ak), vsub_(vneg_(w), ak)};
    const float fe[6] = {-pc.hl, -pc.hl, -pc.s, -pc.s, -rm, -rm};
    float t_near = -1e30f, t_far = 1e30f;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const float denom = dot_(fn[i], rd);
        const float side = add_(dot_(fn[i], o), fe[i]);
        if (fabsf(denom) > 1e-7f) {
            const float t = div_(-side, denom);
            if (denom < 0.0f)
                t_near = fmaxf(t_near, t);
            else
                t_far = fminf(t_far, t);
        } else if (side > 0.0f) {
            return false;
        }
    }
    if (!(t_near <= t_far)) return false;
    lo_out = t_near;
    hi_out = t_far;
    return true;
}
// ToolPrimitive::ray_interval (tool.rs:580): the hull of the pieces' intervals.
IX_DEV bool tool_ray_interval(const ix_tool& t, V3 o, V3 d, float& lo, float& hi) {
    Piece ps[MAX_PIECES];
    const int n = tool_pieces(t, ps);
    bool any = false;
#pragma unroll 1
    for (int i = 0; i < n; ++i) {
        float c, e;
        if (!piece_interval(ps[i], o, d, c, e)) continue;
        lo = any ? fminf(lo, c) : c;
        hi = any ? fmaxf(hi, e) : e;
        any = true;
    }
    return any;
}
// Vec3::any_orthonormal_vector (glam; Duff et al., JCGT 2017).
IX_DEV V3 any_orthonormal_vector(V3 n) {
    const float sign = signbit(n.z) ? -1.0f : 1.0f;
    const float a = div_(-1.0f, add_(sign, n.z));
    const float b = mul_(mul_(n.x, n.y), a);
    return v3(b, add_(sign, mul_(mul_(n.y, n.y), a)), -n.y);
}
// Piece::sd_normal (tool.rs:228).
IX_DEV float piece_sd_normal(const Piece& pc, V3 p, V3& n_out) {
    const V3 q = vsub_(p, pc.c);
    if (pc.kind == PIECE_BALL) {
        const float len = __fsqrt_rn(dot_(q, q));
        n_out = len > 1e-12f ? v3(div_(q.x, len), div_(q.y, len), div_(q.z, len)) : v3(0.0f, 0.0f, 1.0f);
        return sub_(len, pc.r);
    }
    if (pc.kind == PIECE_FRUSTUM) {
        const float z = dot_(q, pc.a);
        const V3 perp = vsub_(q, vmul_(pc.a, z));
        const float rho = __fsqrt_rn(dot_(perp, perp));
        const V3 rho_hat = rho > 1e-12f ? v3(div_(perp.x, rho), div_(perp.y, rho), div_(perp.z, rho))
                                        : any_orthonormal_vector(pc.a);
        const float cap_sd = z >= 0.0f ? sub_(z, pc.hl) : sub_(-z, pc.hl);
        const V3 cap_n = z >= 0.0f ? pc.a : vneg_(pc.a);
        const float dr = sub_(pc.r1, pc.r0);
        const float len = __fsqrt_rn(fmaf(mul_(4.0f, pc.hl), pc.hl, mul_(dr, dr)));
        const float rm = mul_(0.5f, add_(pc.r0, pc.r1));
        const float side_sd = div_(fmaf(z, -dr, mul_(mul_(sub_(rho, rm), 2.0f), pc.hl)), len);
        const V3 side_n = vsub_(vmul_(rho_hat, div_(mul_(2.0f, pc.hl), len)), vmul_(pc.a, div_(dr, len)));
        if (side_sd > cap_sd) {
            n_out = side_n;
            return side_sd;
        }
        n_out = cap_n;
        return cap_sd;
    }
    const V3 w = cross_(pc.a, pc.d);
    const float z = dot_(q, pc.a), x = dot_(q, pc.d), y = dot_(q, w);
    const float k = div_(sub_(pc.r1, pc.r0), mul_(2.0f, pc.hl));
    const float rm = mul_(0.5f, add_(pc.r0, pc.r1));
    const float kappa = div_(1.0f, __fsqrt_rn(fmaf(k, k, 1.0f)));
    float best = z >= 0.0f ? sub_(z, pc.hl) : sub_(-z, pc.hl);
    V3 best_n = z >= 0.0f ? pc.a : vneg_(pc.a);
    const float along = x >= 0.0f ? sub_(x, pc.s) : sub_(-x, pc.s);
    if (along > best) {
        best = along;
        best_n = x >= 0.0f ? pc.d : vneg_(pc.d);
    }
    const float sp = mul_(sub_(sub_(y, rm), mul_(k, z)), kappa);
    if (sp > best) {
        best = sp;
        best_n = vmul_(vsub_(w, vmul_(pc.a, k)), kappa);
    }
    const float sn = mul_(sub_(sub_(-y, rm), mul_(k, z)), kappa);
    if (sn > best) {
        best = sn;
        best_n = vmul_(vsub_(vneg_(w), vmul_(pc.a, k)), kappa);
    }
    n_out = best_n;
    return best;
}
// outward_normal (tool.rs:560) and contains (tool.rs:545).
IX_DEV V3 tool_outward_normal(const ix_tool& t, V3 p) {
    Piece ps[MAX_PIECES];
    const int n = tool_pieces(t, ps);
    float best = INFINITY;
    V3 best_n = v3(0.0f, 0.0f, 1.0f);
#pragma unroll 1
    for (int i = 0; i < n; ++i) {
        V3 nn;
        const float sd = fabsf(piece_sd_normal(ps[i], p, nn));
        if (sd < best) {
            best = sd;
            best_n = nn;
        }
    }
    return best_n;
}
IX_DEV bool tool_contains(const ix_tool& t, V3 p) {
    Piece ps[MAX_PIECES];
    const int n = tool_pieces(t, ps);
#pragma unroll 1
    for (int i = 0; i < n; ++i) {
        V3 nn;
        if (piece_sd_normal(ps[i], p, nn) <= 0.0f) return true;
    }
    return false;
}

}  // namespace ix
