// ix_metrics.cu -- the analytic optical metrics on the device (sm_100a).
//
// evaluate_gem_optical_metrics (color/metrics/evaluate.rs:158-392) for a batch of camera
// poses: one CTA per pose.  The CTA stages its stone's planes in shared memory, derives
// the exit-lighting threshold (the median of 96 hemisphere radiances, lighting.rs:101),
// then each thread takes grid cells of the 18 x 18 fan (fan.rs) and classifies the cell's
// 5 aperture rays (classify.rs) -- a single-index interior trace of at most 10 bounces
// (ray_trace.rs:264-352), with n_F / n_C companion traces for fire -- and its 5
// yaw-jittered rays for temporal scintillation (scintillation.rs:85).  Per-cell results
// go to shared memory and one thread folds them in the reference's (ix, iz, sample)
// order, so every f32 sum is formed exactly as the CPU forms it.
//
// Compiled twice like ix_kernels.cu (IX_EXACT=1 with -fmad=false, IX_EXACT=0).
#include "ix_device.cuh"
#include "ix_launch.h"

#if IX_EXACT
#define IX_SFX(name) name##_exact
#else
#define IX_SFX(name) name##_fast
#endif

namespace ix {

namespace {

constexpr int GRID = 18;
constexpr int CELLS = GRID * GRID;
constexpr int METRICS_THREADS = 128;

enum { FATE_ENTRY_BLOCKED = 0, FATE_LEAKED = 1, FATE_EXITED_UP = 2, FATE_ABSORBED = 3 };

struct ExitPath {
    V3 dir;
    float transmittance, exit_cos, path_len;
    int facet;
    uint32_t bounces;
};

// fresnel_transmittance (ray_trace.rs:35).
IX_DEV float fresnel_transmittance(float n1, float n2, float cos_i, float cos_t) {
    const float denom_s = fmaf(n2, cos_t, n1 * cos_i);
    const float denom_p = fmaf(n2, cos_i, n1 * cos_t);
    if (fabsf(denom_s) < 1e-6f || fabsf(denom_p) < 1e-6f) return 0.0f;
    const float rs = fmaf(n2, -cos_t, n1 * cos_i) / denom_s;
    const float rp = fmaf(n2, -cos_i, n1 * cos_t) / denom_p;
    return clampf_(1.0f - midpointf_(rs * rs, rp * rp), 0.0f, 1.0f);
}

IX_DEV V3 plane_normal(const float4* planes, int i) {
    const float4 p = planes[i];
    return v3(p.x, p.y, p.z);
}

// trace_wavelength_detail + trace_interior (ray_trace.rs:240-352), unfrosted.
IX_DEV int trace_entry(const float4* __restrict__ planes, int n, V3 entry_point, V3 incoming, V3 n_entry,
                       float cos_i, float index, ExitPath& ex) {
    const float inv = 1.0f / index;
    const float sin2_t = (1.0f / (index * index)) * fmaf(cos_i, -cos_i, 1.0f);
    if (sin2_t > 1.0f) return FATE_ENTRY_BLOCKED;
    const float cos_t = sqrtf(1.0f - sin2_t);
    V3 dir = normalize(inv * incoming + fmaf(inv, cos_i, -cos_t) * n_entry);
    const float entry_t = fresnel_transmittance(1.0f, index, cos_i, cos_t);
    V3 point = entry_point + dir * 1e-4f;
    const float sin_crit = 1.0f / index;
    bool leaked = false, up = false;
    float path_len = 0.0f;
    for (uint32_t bounce = 0; bounce < 10; ++bounce) {
        const Hit h = intersect_planes(planes, n, point, dir);
        if (h.facet < 0) break;
        path_len = path_len + h.t;
        const V3 next = point + h.t * dir;
        const V3 n_out = plane_normal(planes, h.facet);
        const float cos_theta = clampf_(dot(dir, n_out), 0.0f, 1.0f);
        const float sin_theta = sqrtf(fmaxf(fmaf(cos_theta, -cos_theta, 1.0f), 0.0f));
        if (sin_theta < sin_crit) {
            const float sin2_out = (index * index) * fmaf(cos_theta, -cos_theta, 1.0f);
            if (sin2_out <= 1.0f) {
                const float cos_out = sqrtf(1.0f - sin2_out);
                const V3 out_dir = normalize(index * dir + fmaf(index, -cos_theta, cos_out) * n_out);
                // Escape::record (ray_trace.rs:110).
                if (n_out.y < -0.05f) {
                    leaked = true;
                } else if (out_dir.y > 0.05f) {
                    up = true;
                    ex.dir = out_dir;
                    ex.transmittance = fresnel_transmittance(index, 1.0f, cos_theta, cos_out);
                    ex.exit_cos = cos_out;
                    ex.facet = h.facet;
                    ex.bounces = bounce;
                }
                break;
            }
        }
        dir = normalize(dir - (2.0f * cos_theta) * n_out);
        point = next + dir * 1e-4f;
    }
    if (leaked) return FATE_LEAKED;
    if (up) {
        ex.transmittance = entry_t * ex.transmittance;
        ex.path_len = path_len;
        return FATE_EXITED_UP;
    }
    return FATE_ABSORBED;
}

struct Fan {
    float standoff, lateral;
    // FanGeometry::origin (fan.rs:89).
    IX_DEV V3 origin(V3 f, V3 r, V3 u, float gu, float gv) const {
        return (-f * standoff + (gu * lateral) * r) + (gv * lateral) * u;
    }
};

enum { CLS_NONE = -1, CLS_BLOCKED = 0, CLS_WINDOWED = 1, CLS_EXTINCT = 2, CLS_RETURNED = 3 };

struct CellOut {
    uint8_t total, returned, windowed, extinct, temporal_returned, fire_mask;
    float angle[5];
    float weight[5];
};

IX_DEV V3 basis_vec(const MetricsPoseDev& p, int k, int which) {
    const float* b = p.basis[k] + 3 * which;
    return v3(b[0], b[1], b[2]);
}

}  // namespace

// SCORE: SCORE_RIG for the studio rigs and the iso-hemisphere, SCORE_EXT for every other
// lighting model (the launch picks by the scoring environment's model).
template <int SCORE>
__global__ void __launch_bounds__(METRICS_THREADS) IX_SFX(metrics_kernel)(const __grid_constant__ MetricsLaunch L) {
    __shared__ float4 s_planes[IX_MAX_PLANES];
    __shared__ float s_rad[96];
    __shared__ float s_threshold;
    __shared__ CellOut s_cells[CELLS];
    const MetricsPoseDev& pose = L.poses[blockIdx.x];
    const MetricsStoneDev stone = L.stones[pose.stone];
    const int n = (int)stone.n_planes;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_planes[i] = L.planes[stone.plane_offset + i];
    // The exit-lighting threshold; its barriers also publish the plane cache.
    const float threshold = exit_lighting_threshold<SCORE>(L.env, L.spec, L.factor, L.dirs, s_rad, &s_threshold);
    const ExitScorerT<SCORE> sc{L.env, L.spec, threshold, L.head_shadow_cos};
    const float nd = fmaxf(dispersion_eval(stone.dispersion, 589.3f), 1.1f);
    const float n_f = fmaxf(dispersion_eval(stone.dispersion, 486.1f), 1.001f);
    const float n_c = fmaxf(dispersion_eval(stone.dispersion, 656.3f), 1.001f);
    const Fan fan{2.5f * stone.half_width, (0.95f * stone.half_width) / sqrtf(0.70f)};
    const V3 f = basis_vec(pose, 0, 0), r = basis_vec(pose, 0, 1), u = basis_vec(pose, 0, 2);
    const float subs[5][2] = {{0.0f, 0.0f}, {0.08f, 0.0f}, {-0.08f, 0.0f}, {0.0f, 0.08f}, {0.0f, -0.08f}};

    for (int cell = threadIdx.x; cell < CELLS; cell += blockDim.x) {
        const int ix = cell / GRID, iz = cell % GRID;
        CellOut co;
        co.total = co.returned = co.windowed = co.extinct = co.temporal_returned = co.fire_mask = 0;
        const float gu = fmaf(((float)ix + 0.5f) / (float)GRID, 2.0f, -1.0f);
        const float gv = fmaf(((float)iz + 0.5f) / (float)GRID, 2.0f, -1.0f);
        if (fmaf(gv, gv, gu * gu) <= 0.70f) {
            // classify_aperture_sample (classify.rs:47) for the 5 aperture offsets.
            for (int k = 0; k < 5; ++k) {
                co.angle[k] = 0.0f;
                co.weight[k] = 0.0f;
                const V3 dir = normalize((f + subs[k][0] * r) + subs[k][1] * u);
                const V3 o = fan.origin(f, r, u, gu, gv);
                const Hit h = intersect_planes(s_planes, n, o, dir);
                if (h.facet < 0) continue;
                ++co.total;
                const V3 p = o + h.t * dir;
                const V3 nrm = plane_normal(s_planes, h.facet);
                const float cos_i = clampf_(dot(-dir, nrm), 0.0f, 1.0f);
                ExitPath ex;
                const int fate = trace_entry(s_planes, n, p, dir, nrm, cos_i, nd, ex);
                if (fate == FATE_LEAKED) {
                    ++co.windowed;
                } else if (fate == FATE_ABSORBED) {
                    ++co.extinct;
                } else if (fate == FATE_EXITED_UP) {
                    if (!sc.returned(ex.dir, f)) {
                        ++co.extinct;
                        continue;
                    }
                    ++co.returned;
                    if (!L.want_fire) continue;
                    // fire_sample (classify.rs:162).
                    ExitPath ef, ec;
                    const int ff = trace_entry(s_planes, n, p, dir, nrm, cos_i, n_f, ef);
                    const int fc = trace_entry(s_planes, n, p, dir, nrm, cos_i, n_c, ec);
                    if (ff == FATE_EXITED_UP && fc == FATE_EXITED_UP && ef.facet == ec.facet &&
                        ef.bounces == ec.bounces) {
                        const float cos_sep = clampf_(dot(ef.dir, ec.dir), -1.0f, 1.0f);
                        co.angle[k] = acosf(cos_sep) * 57.2957795130823208767981548141051703f;
                        co.weight[k] = ((ex.transmittance * ef.transmittance) * ec.transmittance) *
                                       (fmaxf(ef.exit_cos, 0.0f) * fmaxf(ec.exit_cos, 0.0f));
                        co.fire_mask |= (uint8_t)(1u << k);
                    }
                }
            }
            // cell_temporal_variance (scintillation.rs:85-117): the count of returned
            // rays over the 5 yaw-jittered poses.
            if (co.total > 0 && L.want_fire) {
                for (int k = 0; k < 5; ++k) {
                    const V3 tf = basis_vec(pose, k + 1, 0), tr = basis_vec(pose, k + 1, 1),
                             tu = basis_vec(pose, k + 1, 2);
                    const V3 o = fan.origin(tf, tr, tu, gu, gv);
                    const Hit h = intersect_planes(s_planes, n, o, tf);
                    if (h.facet < 0) continue;
                    const V3 p = o + h.t * tf;
                    const V3 nrm = plane_normal(s_planes, h.facet);
                    const float cos_i = clampf_(dot(-tf, nrm), 0.0f, 1.0f);
                    ExitPath ex;
                    if (trace_entry(s_planes, n, p, tf, nrm, cos_i, nd, ex) != FATE_EXITED_UP) continue;
                    if (sc.returned(ex.dir, tf)) ++co.temporal_returned;
                }
            }
        }
        s_cells[cell] = co;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    // run_grid / sample_cell / finish_metrics (evaluate.rs:302-392, accumulate.rs:99-160).
    uint32_t total = 0, windowed = 0, extinct = 0, returned = 0, cells = 0;
    float fire_sum = 0.0f, frac_sum = 0.0f, frac_sq = 0.0f, tvar_sum = 0.0f;
    for (int cell = 0; cell < CELLS; ++cell) {
        const CellOut& co = s_cells[cell];
        total += co.total;
        windowed += co.windowed;
        extinct += co.extinct;
        returned += co.returned;
        for (int k = 0; k < 5; ++k)
            if (co.fire_mask & (1u << k)) fire_sum = fmaf(co.angle[k], co.weight[k], fire_sum);
        if (co.total > 0) {
            const float frac = (float)co.returned / (float)co.total;
            frac_sum = frac_sum + frac;
            frac_sq = fmaf(frac, frac, frac_sq);
            ++cells;
            const float tp = (float)co.temporal_returned / 5.0f;
            tvar_sum = tvar_sum + fmaf(tp, -tp, tp);
        }
    }
    const float n_total = (float)(total > 0 ? total : 1u);
    float* out = L.out + (size_t)blockIdx.x * 5;
    out[0] = clampf_((float)returned / n_total * 100.0f, 0.0f, 100.0f);
    out[3] = clampf_((float)windowed / n_total * 100.0f, 0.0f, 100.0f);
    out[4] = clampf_((float)extinct / n_total * 100.0f, 0.0f, 100.0f);
    if (!L.want_fire) {
        out[1] = 25.0f;  // placeholder_metrics (evaluate.rs:210)
        out[2] = 75.0f;
        return;
    }
    out[1] = fmaxf(fire_sum / n_total * 275.0f, 0.1f);
    float spatial = 0.0f;
    if (cells > 0) {
        const float mean = frac_sum / (float)cells;
        if (mean > 1e-4f) {
            const float var = fmaxf(fmaf(mean, -mean, frac_sq / (float)cells), 0.0f);
            const float cv = sqrtf(var) / mean;
            spatial = clampf_(cv / (1.0f + cv) * 100.0f, 0.0f, 100.0f);
        }
    }
    const float temporal = cells > 0 ? clampf_(tvar_sum / (float)cells / 0.24f * 100.0f, 0.0f, 100.0f) : 0.0f;
    out[2] = clampf_(fmaf(0.4f, temporal, 0.6f * spatial), 0.0f, 100.0f);
}

cudaError_t IX_SFX(launch_metrics)(const MetricsLaunch& l, cudaStream_t stream) {
    if (l.n_poses == 0) return cudaSuccess;
    if (rig_scored(l.env))
        IX_SFX(metrics_kernel)<SCORE_RIG><<<l.n_poses, METRICS_THREADS, 0, stream>>>(l);
    else
        IX_SFX(metrics_kernel)<SCORE_EXT><<<l.n_poses, METRICS_THREADS, 0, stream>>>(l);
    return cudaGetLastError();
}

}  // namespace ix
