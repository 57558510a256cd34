// ix_design.cpp -- a parametric round brilliant's facet half-spaces and material, built
// on the host in double precision and rounded to the f32 rows the transport reads
// (include/ix_design.h).  The half-space layout is the one of
// indicatrix_b200/geometry.py:round_brilliant (this library's own parametric builder;
// the reference's fixed builder, geometry/cuts/round_brilliant.rs:71-155, takes no
// parameters), so the Python builder and this one give the same planes.
#include <cmath>
#include <cstring>
#include <initializer_list>

#include "../../include/ix_design.h"

namespace {

constexpr double kPi = 3.14159265358979323846;
// Fraunhofer F, C and the sodium D line, micrometres.
constexpr double kLambdaF = 0.4861, kLambdaC = 0.6563, kLambdaD = 0.5893;
// A 1.0-diameter stone has a 6.5 mm girdle: 0.65 cm per model unit.
constexpr float kCmPerModelUnit = 0.65f;

struct Plane {
    double n[3];
    double d;
};

double rad(double deg) { return deg * kPi / 180.0; }

// The unit normal of a facet `angle_deg` from the girdle plane at azimuth `phi`, pointing
// up (crown) or down (pavilion), and the plane through `point`.
Plane facet(double angle_deg, double phi, bool crown, double px, double py, double pz) {
    const double a = rad(angle_deg);
    double n[3] = {std::sin(a) * std::cos(phi), crown ? std::cos(a) : -std::cos(a), std::sin(a) * std::sin(phi)};
    const double len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    Plane p;
    for (int i = 0; i < 3; ++i) p.n[i] = n[i] / len;
    p.d = -(p.n[0] * px + p.n[1] * py + p.n[2] * pz);
    return p;
}

bool finite_all(const ix_design* d) {
    const float* f = &d->crown_deg;
    for (int i = 0; i < IX_DESIGN_PARAMS; ++i)
        if (!std::isfinite(f[i])) return false;
    return true;
}

bool angle_ok(double deg) { return deg > 0.0 && deg < 89.0; }

bool geometry_ok(const ix_design* d) {
    return finite_all(d) && angle_ok(d->crown_deg) && angle_ok(d->pavilion_deg) &&
           angle_ok((double)d->crown_deg + d->star_offset_deg) &&
           angle_ok((double)d->crown_deg + d->upper_half_offset_deg) &&
           angle_ok((double)d->pavilion_deg + d->lower_half_offset_deg) && d->table_pct > 0.0f &&
           d->table_pct < 100.0f && d->girdle_pct >= 0.0f && d->girdle_pct < 50.0f;
}

}  // namespace

extern "C" {

uint32_t ix_design_planes(const ix_design* d, uint32_t girdle_segments, float* planes, uint32_t cap) {
    if (!d || !geometry_ok(d)) return 0;
    if (girdle_segments == 0) girdle_segments = 64;
    if (girdle_segments > 4096) return 0;
    const uint32_t n_sym = 8;
    const uint32_t count = 1 + n_sym + n_sym + 2 * n_sym + girdle_segments + n_sym + 2 * n_sym;
    if (!planes) return count;
    const double R = 0.5, h = 0.5 * d->girdle_pct / 100.0, r_t = 0.5 * d->table_pct / 100.0;
    const double step = 2.0 * kPi / n_sym, half = step / 8.0;
    const double y_table = h + (R - r_t) * std::tan(rad(d->crown_deg));
    uint32_t k = 0;
    auto put = [&](const Plane& p) {
        if (k < cap) {
            // Renormalise in double, then round (the Python builder's to_f32).
            const double len = std::sqrt(p.n[0] * p.n[0] + p.n[1] * p.n[1] + p.n[2] * p.n[2]);
            planes[4 * k + 0] = (float)(p.n[0] / len);
            planes[4 * k + 1] = (float)(p.n[1] / len);
            planes[4 * k + 2] = (float)(p.n[2] / len);
            planes[4 * k + 3] = (float)(p.d / len);
        }
        ++k;
    };
    put(Plane{{0.0, 1.0, 0.0}, -y_table});
    // Stars: their top edges are the table's edges between adjacent main tips.
    const double star = (double)d->crown_deg + d->star_offset_deg;
    const double edge_r = r_t * std::cos(step / 2.0);
    for (uint32_t m = 0; m < n_sym; ++m) {
        const double phi = (m + 0.5) * step;
        put(facet(star, phi, true, edge_r * std::cos(phi), y_table, edge_r * std::sin(phi)));
    }
    for (uint32_t m = 0; m < n_sym; ++m) {
        const double phi = m * step;
        put(facet(d->crown_deg, phi, true, R * std::cos(phi), h, R * std::sin(phi)));
    }
    const double uh = (double)d->crown_deg + d->upper_half_offset_deg;
    for (uint32_t m = 0; m < n_sym; ++m)
        for (int s = -1; s <= 1; s += 2) {
            const double phi = m * step + s * half;
            put(facet(uh, phi, true, R * std::cos(phi), h, R * std::sin(phi)));
        }
    for (uint32_t i = 0; i < girdle_segments; ++i) {
        const double phi = 2.0 * kPi * i / girdle_segments;
        put(Plane{{std::cos(phi), 0.0, std::sin(phi)}, -R});
    }
    for (uint32_t m = 0; m < n_sym; ++m) {
        const double phi = m * step;
        put(facet(d->pavilion_deg, phi, false, R * std::cos(phi), -h, R * std::sin(phi)));
    }
    const double lh = (double)d->pavilion_deg + d->lower_half_offset_deg;
    for (uint32_t m = 0; m < n_sym; ++m)
        for (int s = -1; s <= 1; s += 2) {
            const double phi = m * step + s * half;
            put(facet(lh, phi, false, R * std::cos(phi), -h, R * std::sin(phi)));
        }
    return count;
}

int ix_design_material(const ix_design* d, ix_material* out) {
    if (!d || !out || !finite_all(d)) return -1;
    if (!(d->n_d > 1.0f && d->n_d < 4.0f) || !(d->dispersion >= 0.0f && d->dispersion < 1.0f)) return -1;
    if (!(d->absorb_peak >= 0.0f)) return -1;
    if (d->absorb_peak > 0.0f && !(d->absorb_width_nm > 0.0f && d->absorb_center_nm > 0.0f)) return -1;
    std::memset(out, 0, sizeof(*out));
    // Cauchy n = A + B / l^2: n_F - n_C = B (1 / l_F^2 - 1 / l_C^2), A from n_D.
    const double B = d->dispersion / (1.0 / (kLambdaF * kLambdaF) - 1.0 / (kLambdaC * kLambdaC));
    const double A = d->n_d - B / (kLambdaD * kLambdaD);
    out->dispersion.kind = IX_DISP_CAUCHY;
    out->dispersion.b[0] = (float)A;
    out->dispersion.b[1] = (float)B;
    out->dispersion.b[2] = 0.0f;
    out->anisotropic = 0;
    out->c_axis[1] = 1.0f;
    if (d->absorb_peak > 0.0f) {
        for (ix_absorption* ab : {&out->abs_o, &out->abs_e}) {
            ab->n_bands = 1;
            ab->bands[0].center_nm = d->absorb_center_nm;
            ab->bands[0].width_nm = d->absorb_width_nm;
            ab->bands[0].peak = d->absorb_peak;
            ab->bands[0].shape = IX_BAND_GAUSS_WAVELENGTH;
        }
    }
    out->absorption_path_scale = kCmPerModelUnit;
    return 0;
}

}  // extern "C"
