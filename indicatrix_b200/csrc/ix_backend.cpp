// ix_backend.cpp -- host side of the C ABI declared in include/ix_cuda.h.
//
// The reference's GpuBackend (crates/indicatrix/src/renderer/gpu_backend/backend.rs)
// re-designed for one CUDA device: a backend owns a stream, pooled device buffers and
// pinned host staging; requests take a FIFO ticket (gpu_backend/turnstile.rs:24-115) so
// concurrent callers are served in arrival order; a device error marks the backend lost
// and turns the request into a decline (gpu_backend/mod.rs:151-164, recovery.rs:13-79).
//
// Host scene construction (camera, environment presets) follows the reference's own
// host formulas; this file is compiled with -ffp-contract=off so those round exactly as
// the reference does.

#include "../../include/ix_cuda.h"
#include "../../include/ix_cie_tables.h"
#include "../../include/ix_design.h"
#include "ix_backend_state.h"
#include "ix_launch.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

using namespace ixh;

namespace {

uint32_t pixels_per_task(uint32_t spp) {
    // About 64 paths per warp task (16 per 8-lane group), whole pixels, at most 8: small
    // tasks keep every warp busy to the end of a launch (a single frame at 256^2 x 64 spp
    // measured 2x faster than with 256-path tasks).
    uint32_t ppt = spp ? 64u / spp : 1u;
    return std::max(1u, std::min(8u, ppt));
}

// The chunking of enqueue_frame: launches of `chunk_paths` (default 64M paths), whole
// pixels each.  The reference's first launch of at most 1M paths (gpu/frame/mod.rs:
// 355-361) keeps a display GPU's watchdog away; a compute B200 has none, and a 1M-path
// launch cannot fill its 148 SMs (the results do not depend on the chunking).
// Kernel variant of single-scene calls when the options name none: the path-pool loop,
// 128 threads, the 32-warps-per-SM register budget.
constexpr uint32_t kDefaultVariant = 2 + 3 * ix::SHAPE_POOL_128;
// Scenes that need the uniaxial transport default to the static task loop with the
// 16-warp budget: measured fastest for it (the pool loop's larger body costs the bigger
// uniaxial kernel more instruction fetch than it saves).
constexpr uint32_t kDefaultUniaxialVariant = 2 + 3 * ix::SHAPE_TASKS;

uint64_t chunk_budget(const ix_backend* b, int launch_index) {
    (void)launch_index;
    return b->chunk_paths ? b->chunk_paths : (64ull << 20);
}

// Enqueue the trace launches for pixels [0, n_pixels) of `sc` (device planes) into
// d_out; chunked so no single launch exceeds the path budget.  A launch covers whole
// pixels, so the sums do not depend on the chunking.  The path-pool shapes add into
// fixed-point sums of the launch's pixels (b->d_acc) and round them into d_out after each
// launch; a pixel's samples beyond FIXED_MAX_SAMPLES go to later launches of the same
// pixels.  With `attr`, every launch is the attributed trace kernel (static task loop),
// followed by the fold of its records into d_map (the frame's attribution map on the
// device).  Returns the launch count or -1 on a CUDA error (b->last_error set).
// The single-scene kernel variant for a scene with transport flags `flags`: the one the
// options pinned, else the backend's default for its transport.
uint32_t frame_variant(const ix_backend* b, uint32_t flags) {
    if (b->variant_pinned) return b->variant;
    return ix::needs_uniaxial_kernel(flags) ? kDefaultUniaxialVariant : b->variant;
}

int enqueue_frame(ix_backend* b, const ix_scene& sc, uint32_t sample_offset, uint32_t spp,
                  double* d_out, int accumulate, cudaStream_t stream,
                  const volatile uint8_t* cancel, bool* cancelled,
                  const ix::AttrLaunch* attr = nullptr, ix_attribution_pixel* d_map = nullptr) {
    const uint64_t n_pixels64 = (uint64_t)sc.width * sc.height;
    if (n_pixels64 > 0xFFFFFFFFull) {
        b->last_error = "frame has more than 2^32 - 1 pixels";
        return -1;
    }
    const uint32_t n_pixels = (uint32_t)n_pixels64;
    const bool exact = b->precision == IX_PRECISION_EXACT;
    ix::TraceLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.scene = sc;
    L.flags = ix::scene_flags(sc);
    L.pixels_per_task = pixels_per_task(spp);
    L.task_counter = b->d_counter;
    L.dropped = b->d_dropped;
    L.variant = attr ? 0 : (int)frame_variant(b, L.flags);
    const int shape = ix::variant_shape(L.variant);
    const bool pool = ix::shape_is_pool(shape);
    L.threads = ix::shape_threads(shape);
    const int uni = ix::transport_class(L.flags);
    L.blocks = b->sm_count * (exact ? b->bps_exact[uni][L.variant] : b->bps_fast[uni][L.variant]);
    if (attr) L.blocks = b->sm_count * (exact ? b->bps_attr_exact[uni] : b->bps_attr_fast[uni]);
    if (L.blocks <= 0) {
        b->last_error = "kernel variant not available in this build";
        return -1;
    }
    // Sample blocks: one for the static task loop, FIXED_MAX_SAMPLES at most for the pool.
    const uint32_t block = pool ? std::min<uint32_t>(spp, ix::FIXED_MAX_SAMPLES) : spp;
    int launches = 0;
    for (uint32_t s0 = 0; s0 < spp; s0 += block) {
        const uint32_t sb = std::min(block, spp - s0);
        L.sample_offset = sample_offset + s0;
        L.spp = sb;
        L.accumulate = s0 == 0 ? accumulate : 1;
        uint32_t begin = 0;
        while (begin < n_pixels) {
            if (cancel && *cancel) {
                *cancelled = true;
                return launches;
            }
            uint64_t px = std::max<uint64_t>(1, chunk_budget(b, launches) / std::max<uint32_t>(sb, 1));
            uint32_t n = (uint32_t)std::min<uint64_t>(px, n_pixels - begin);
            L.pixel_begin = begin;
            L.n_pixels = n;
            L.out = d_out + (size_t)begin * 3;
            if (pool) {
                if (fail(b, grow_device(&b->d_acc, &b->acc_cap, (size_t)n * ix::FIXED_WORDS), "sums alloc")) return -1;
                L.acc = b->d_acc;
            }
            if (attr) {
                cudaError_t e = exact ? ix::launch_trace_attributed_exact(L, *attr, stream)
                                      : ix::launch_trace_attributed_fast(L, *attr, stream);
                if (fail(b, e, "attributed trace launch")) return -1;
                const ix::AttrFoldLaunch F{attr->cls, attr->y, d_map + begin, n, sb};
                e = exact ? ix::launch_attribution_fold_exact(F, stream) : ix::launch_attribution_fold_fast(F, stream);
                if (fail(b, e, "attribution fold")) return -1;
            } else {
                cudaError_t e = exact ? ix::launch_trace_exact(L, stream) : ix::launch_trace_fast(L, stream);
                if (fail(b, e, "trace launch")) return -1;
            }
            ++launches;
            begin += n;
        }
    }
    return launches;
}

// Kernels one trace launch of a scene's single-scene variant takes: the trace kernel, and
// for the path-pool shapes the rounding of its fixed-point sums.
uint32_t kernels_per_launch(const ix_backend* b, const ix_scene& sc) {
    return ix::shape_is_pool(ix::variant_shape((int)frame_variant(b, ix::scene_flags(sc)))) ? 2u : 1u;
}

// Points a device copy of host scene `sc` at the backend's copy of its facet finishes
// (none: all polished).  Caller holds the turn.  False on a CUDA error.
bool upload_finishes(ix_backend* b, ix_scene& sc, cudaStream_t st) {
    if (!sc.facet_finishes || sc.n_finishes == 0) {
        sc.facet_finishes = nullptr;
        sc.n_finishes = 0;
        return true;
    }
    if (fail(b, grow_device(&b->d_finishes, &b->finishes_cap, (size_t)sc.n_finishes), "finishes alloc") ||
        fail(b, cudaMemcpyAsync(b->d_finishes, sc.facet_finishes, sc.n_finishes, cudaMemcpyHostToDevice, st),
             "finishes upload"))
        return false;
    sc.facet_finishes = b->d_finishes;
    return true;
}
// ... and at the backend's copy of its concave tools (none: a convex stone).
bool upload_tools(ix_backend* b, ix_scene& sc, cudaStream_t st) {
    if (!sc.tools || sc.n_tools == 0) {
        sc.tools = nullptr;
        sc.n_tools = 0;
        return true;
    }
    if (fail(b, grow_device(&b->d_tools, &b->tools_cap, (size_t)sc.n_tools), "tools alloc") ||
        fail(b, cudaMemcpyAsync(b->d_tools, sc.tools, sc.n_tools * sizeof(ix_tool), cudaMemcpyHostToDevice, st),
             "tools upload"))
        return false;
    sc.tools = b->d_tools;
    return true;
}

template <typename AccT>
int accumulate_impl(ix_backend* b, const ix_scene* scene, uint32_t sample_offset, uint32_t spp,
                    AccT* accum, const volatile uint8_t* cancel) {
    if (!b || !scene || !accum) return IX_DECLINED;
    if (b->lost) return IX_DECLINED;
    if (!ix_scene_routes_to_gpu(scene)) return IX_DECLINED;
    const uint64_t n_pixels = (uint64_t)scene->width * scene->height;
    if (b->limits.max_pixels && n_pixels > b->limits.max_pixels) return IX_DECLINED;
    if (b->limits.max_spp && spp > b->limits.max_spp) return IX_DECLINED;
    if (b->limits.max_paths_per_call && n_pixels * spp > b->limits.max_paths_per_call) return IX_DECLINED;
    if (cancel && *cancel) return IX_CANCELLED;
    if (n_pixels == 0 || spp == 0) return IX_DONE;
    Turn turn(b);
    if (fail(b, cudaSetDevice(b->device), "set device")) return IX_DECLINED;
    if (fail(b, grow_device(&b->d_planes, &b->planes_cap, (size_t)scene->n_planes * 4), "planes alloc"))
        return IX_DECLINED;
    if (fail(b, grow_device(&b->d_sums, &b->sums_cap, (size_t)n_pixels * 3), "sums alloc"))
        return IX_DECLINED;
    if (fail(b, grow_pinned(&b->h_sums, &b->hsums_cap, (size_t)n_pixels * 3), "host alloc"))
        return IX_DECLINED;
    if (scene->n_planes &&
        fail(b, cudaMemcpyAsync(b->d_planes, scene->planes, (size_t)scene->n_planes * 16,
                                cudaMemcpyHostToDevice, b->stream), "planes upload"))
        return IX_DECLINED;
    if (fail(b, cudaMemsetAsync(b->d_dropped, 0, sizeof(unsigned long long), b->stream), "reset"))
        return IX_DECLINED;
    ix_scene sc = *scene;
    sc.planes = b->d_planes;
    if (!upload_finishes(b, sc, b->stream) || !upload_tools(b, sc, b->stream)) return IX_DECLINED;
    bool cancelled = false;
    if (fail(b, cudaEventRecord(b->ev0, b->stream), "event")) return IX_DECLINED;
    int launches = enqueue_frame(b, sc, sample_offset, spp, b->d_sums, 0, b->stream, cancel, &cancelled);
    if (launches < 0) return IX_DECLINED;
    if (fail(b, cudaEventRecord(b->ev1, b->stream), "event")) return IX_DECLINED;
    if (cancelled) {
        cudaStreamSynchronize(b->stream);
        return IX_CANCELLED;
    }
    auto t0 = std::chrono::steady_clock::now();
    if (fail(b, cudaMemcpyAsync(b->h_sums, b->d_sums, (size_t)n_pixels * 3 * sizeof(double),
                                cudaMemcpyDeviceToHost, b->stream), "sums download"))
        return IX_DECLINED;
    unsigned long long dropped = 0;
    if (fail(b, cudaMemcpyAsync(&dropped, b->d_dropped, sizeof(dropped), cudaMemcpyDeviceToHost,
                                b->stream), "dropped download"))
        return IX_DECLINED;
    if (fail(b, cudaStreamSynchronize(b->stream), "trace")) return IX_DECLINED;
    if (cancel && *cancel) return IX_CANCELLED;
    for (size_t i = 0; i < (size_t)n_pixels * 3; ++i) accum[i] += (AccT)b->h_sums[i];
    auto t1 = std::chrono::steady_clock::now();
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->timing.kernel_ms = ms;
    b->timing.reduce_ms = std::chrono::duration<float, std::milli>(t1 - t0).count();
    b->timing.paths = n_pixels * spp;
    b->timing.launches = (uint32_t)launches * kernels_per_launch(b, sc);
    b->dropped = dropped;
    return IX_DONE;
}

// ------------------------------------------------------------------------------------
// Host scene construction: the reference's host formulas, rounded as it rounds them.
// ------------------------------------------------------------------------------------
struct H3 {
    float x, y, z;
};
inline H3 h3(float x, float y, float z) { return H3{x, y, z}; }
inline float hdot(H3 a, H3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline H3 hcross(H3 a, H3 b) {
    return h3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
inline H3 hnormalize(H3 a) {
    float r = 1.0f / std::sqrt(hdot(a, a));
    return h3(a.x * r, a.y * r, a.z * r);
}
inline void hstore(float* p, H3 v) {
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
}
inline float to_radians(float deg) { return deg * (3.14159265358979323846f / 180.0f); }

const float kCmf[81][3] = IX_CIE1931_CMF_INIT;

H3 cmf_host(float lambda) {
    if (!(lambda >= 380.0f && lambda <= 780.0f)) return h3(0.0f, 0.0f, 0.0f);
    float position = (lambda - 380.0f) / 5.0f;
    int i0 = std::min((int)std::floor(position), 79);
    float t = position - (float)i0;
    const float* lo = kCmf[i0];
    const float* hi = kCmf[i0 + 1];
    return h3(lo[0] + (hi[0] - lo[0]) * t, lo[1] + (hi[1] - lo[1]) * t, lo[2] + (hi[2] - lo[2]) * t);
}
inline float powi5(float x) {
    float x2 = x * x;
    return x * (x2 * x2);
}
void blackbody_norm(float temp_k, float* t_k, float* den) {
    *t_k = std::fmax(temp_k, 1000.0f);
    float e = std::exp(std::fmin(14388000.0f / (560.0f * *t_k), 80.0f));
    *den = std::fmax(e - 1.0f, 1e-6f);
}
float blackbody(float t_k, float den, float lambda) {
    float e = std::exp(std::fmin(14388000.0f / (lambda * t_k), 80.0f));
    float d = std::fmax(e - 1.0f, 1e-6f);
    float v = powi5(560.0f / lambda) * (den / d);
    return v < 0.01f ? 0.01f : (v > 20.0f ? 20.0f : v);
}
H3 bradford_xyz_to_lms(H3 v) {
    return h3(std::fma(0.8951f, v.x, std::fma(0.2664f, v.y, -0.1614f * v.z)),
              std::fma(-0.7502f, v.x, std::fma(1.7135f, v.y, 0.0367f * v.z)),
              std::fma(0.0389f, v.x, std::fma(-0.0685f, v.y, 1.0296f * v.z)));
}
// compute_illuminant_white_balance (optics/raytracer/color.rs:277).
H3 white_balance(float temp_k) {
    float t_k, den;
    blackbody_norm(temp_k, &t_k, &den);
    H3 w = h3(0.0f, 0.0f, 0.0f);
    for (int step = 0; step <= 400; ++step) {
        float lambda = 380.0f + (float)step;
        H3 c = cmf_host(lambda);
        float p = blackbody(t_k, den, lambda);
        w = h3(w.x + c.x * p, w.y + c.y * p, w.z + c.z * p);
    }
    float ty = std::fmax(w.y, 1e-6f);
    const float wx = 0.3127f, wy = 0.3290f;
    H3 target = h3((wx / wy) * ty, ty, ((1.0f - wx - wy) / wy) * ty);
    H3 s = bradford_xyz_to_lms(w), t = bradford_xyz_to_lms(target);
    return h3(s.x > 1e-6f ? t.x / s.x : 1.0f, s.y > 1e-6f ? t.y / s.y : 1.0f,
              s.z > 1e-6f ? t.z / s.z : 1.0f);
}

// ------------------------------------------------------------------------------------
// Host setup of the analytic metrics (color/metrics/prepared.rs, fan.rs, lighting.rs,
// visibility.rs, camera.rs): per stone and per lighting, computed once per call.
// ------------------------------------------------------------------------------------
const float kD65[41] = IX_CIE_D65_SPD_INIT;

// d65_relative_spectral_power (environment/spectral.rs:49) on [380, 780] nm.
float d65_host(float lambda) {
    float c = lambda < 380.0f ? 380.0f : (lambda > 780.0f ? 780.0f : lambda);
    float position = (c - 380.0f) / 10.0f;
    int i0 = std::min((int)std::floor(position), 39);
    float frac = position - (float)i0;
    return std::fma(frac, kD65[i0 + 1] - kD65[i0], kD65[i0]) / 100.0f;
}

// measure_model_width (render_setup/stone_width.rs:27, geometry/stone_metrics/measure.rs):
// the narrower horizontal extent (x or z) of the solid's vertices, in f64.  A vertex is
// any point where three planes meet and no plane is violated by more than 1e-9.
double solid_width(const float* planes, uint32_t n) {
    std::vector<std::array<double, 4>> pl;  // n.x <= m with m = -d
    for (uint32_t i = 0; i < n; ++i) {
        std::array<double, 4> p{planes[4 * i], planes[4 * i + 1], planes[4 * i + 2], -(double)planes[4 * i + 3]};
        bool same = false;
        for (const auto& q : pl)
            if (p[0] * q[0] + p[1] * q[1] + p[2] * q[2] > 1.0 - 1e-12 && std::fabs(p[3] - q[3]) < 1e-9) same = true;
        if (!same) pl.push_back(p);
    }
    const size_t m = pl.size();
    double lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
    size_t found = 0;
    auto cr = [](const std::array<double, 4>& a, const std::array<double, 4>& b, double o[3]) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    for (size_t i = 0; i < m; ++i)
        for (size_t j = i + 1; j < m; ++j)
            for (size_t k = j + 1; k < m; ++k) {
                double jk[3], ki[3], ij[3];
                cr(pl[j], pl[k], jk);
                double det = pl[i][0] * jk[0] + pl[i][1] * jk[1] + pl[i][2] * jk[2];
                if (std::fabs(det) < 1e-12) continue;
                cr(pl[k], pl[i], ki);
                cr(pl[i], pl[j], ij);
                double v[3];
                for (int a = 0; a < 3; ++a) v[a] = (pl[i][3] * jk[a] + pl[j][3] * ki[a] + pl[k][3] * ij[a]) / det;
                if (!std::isfinite(v[0]) || !std::isfinite(v[1]) || !std::isfinite(v[2])) continue;
                bool inside = true;
                for (size_t q = 0; inside && q < m; ++q)
                    inside = pl[q][0] * v[0] + pl[q][1] * v[1] + pl[q][2] * v[2] - pl[q][3] <= 1e-9;
                if (!inside) continue;
                ++found;
                lo[0] = std::min(lo[0], v[0]);
                hi[0] = std::max(hi[0], v[0]);
                lo[1] = std::min(lo[1], v[2]);
                hi[1] = std::max(hi[1], v[2]);
            }
    if (found < 4) return NAN;
    const double dx = hi[0] - lo[0], dz = hi[1] - lo[1];
    return dx <= dz ? dx : dz;
}

// head_shadow_cone_cos (visibility.rs:16).
float metrics_head_shadow_cos(bool studio, float deg) {
    if (studio || std::isnan(deg) || deg == 16.0f) return 0.96f;
    if (deg <= 0.0f) return 2.0f;
    const float offset = std::acos(0.96f) - to_radians(16.0f);
    const float c = deg < 1.0f ? 1.0f : (deg > 89.0f ? 89.0f : deg);
    return std::cos(to_radians(c) + offset);
}

// ExitLighting::new (lighting.rs:137) for a lighting preset: the preset at exposure 1, no
// tray and the default head-shadow edges, its spectral power at 550 nm, the threshold
// factor over the median hemisphere radiance, the observer cone and the 96 hemisphere
// probe directions (hemisphere_direction, lighting.rs:74).  Every preset scores: the ASET
// view as the iso-hemisphere (scoring_preset, lighting.rs:125); a UV lamp's line spectrum
// at 550 nm.  False for an unknown preset.
bool exit_lighting_setup(const ix_metrics_lighting& lighting, ix_environment* env, float* spec, float* factor,
                         float* head_shadow_cos, float dirs[96][3]) {
    const int32_t scoring = lighting.preset == 12 ? 1 : lighting.preset;
    if (ix_environment_preset(scoring, 1.0f, lighting.light_yaw, lighting.light_pitch, 0.0f, 1.0f, 16.0f, env) != 0)
        return false;
    const bool studio = env->model == IX_ENV_STUDIO;
    if (env->spectrum == IX_SPEC_GAUSSIAN) {
        const float z = (550.0f - env->line_centre_nm) / env->line_sigma_nm;
        *spec = std::exp((-0.5f * z) * z);
    } else {
        *spec = env->spectrum == IX_SPEC_D65 ? d65_host(550.0f) : blackbody(env->bb_t_k, env->bb_denom_560, 550.0f);
    }
    *factor = studio ? 4.0f : 0.5f;
    *head_shadow_cos = metrics_head_shadow_cos(studio, lighting.head_shadow_deg);
    for (int i = 0; i < 96; ++i) {
        const float y = ((float)i + 0.5f) / 96.0f;
        const float ring = std::sqrt(std::fmax(std::fma(y, -y, 1.0f), 0.0f));
        const float a = (float)i * 2.3999632f;
        dirs[i][0] = ring * std::cos(a);
        dirs[i][1] = y;
        dirs[i][2] = ring * std::sin(a);
    }
    return true;
}

}  // namespace

extern "C" {

ix_backend* ix_backend_create(const ix_backend_options* opts) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        (void)cudaGetLastError();
        return nullptr;
    }
    // threads_per_block: 0 (any CTA size) or one of the sizes the path-pool shapes come in.
    if (opts && opts->threads_per_block != 0 && opts->threads_per_block != 64 && opts->threads_per_block != 128 &&
        opts->threads_per_block != 256)
        return nullptr;
    if (opts && opts->kernel_variant > (uint32_t)ix_backend::kVariants) return nullptr;
    ix_backend* b = new ix_backend();
    if (opts) {
        b->device = opts->device;
        b->pipeline = opts->pipeline;
        b->precision = opts->precision;
        b->batch_threads = opts->threads_per_block;
        b->chunk_paths = opts->chunk_paths;
    }
    if (b->device < 0 || b->device >= n) {
        delete b;
        return nullptr;
    }
    cudaDeviceProp prop;
    if (cudaSetDevice(b->device) != cudaSuccess ||
        cudaGetDeviceProperties(&prop, b->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
        cudaMalloc((void**)&b->d_counter, sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc((void**)&b->d_dropped, sizeof(unsigned long long)) != cudaSuccess) {
        (void)cudaGetLastError();
        ix_backend_destroy(b);
        return nullptr;
    }
    b->sm_count = prop.multiProcessorCount;
    b->label = prop.name;
    static_assert(ix_backend::kVariants == ix::N_VARIANTS, "variant table size");
    static_assert(ix_backend::kClasses == ix::N_TRANSPORT_CLASSES, "transport table size");
    for (int u = 0; u < ix::N_TRANSPORT_CLASSES; ++u)
        for (int v = 0; v < ix::N_VARIANTS; ++v) {
            const int threads = ix::shape_threads(ix::variant_shape(v));
            b->bps_exact[u][v] = ix::trace_blocks_per_sm_exact(threads, v, u, nullptr);
            b->bps_fast[u][v] = ix::trace_blocks_per_sm_fast(threads, v, u, nullptr);
        }
    for (int u = 0; u < ix::N_TRANSPORT_CLASSES; ++u) {
        b->bps_attr_exact[u] = std::max(1, ix::trace_attributed_blocks_per_sm_exact((int)b->threads, u));
        b->bps_attr_fast[u] = std::max(1, ix::trace_attributed_blocks_per_sm_fast((int)b->threads, u));
    }
    // Option 0 = the measured default; k >= 1 = variant k - 1 (budget + 3 * shape).
    b->variant = kDefaultVariant;
    if (opts && opts->kernel_variant >= 1) {
        b->variant = opts->kernel_variant - 1;
        b->variant_pinned = true;
    }
    if (b->bps_exact[0][b->variant] <= 0 || b->bps_fast[0][b->variant] <= 0) {
        // Single-scene calls run only the variants both builds carry.
        ix_backend_destroy(b);
        return nullptr;
    }
    b->batch_variant = b->variant;
    if (b->batch_threads && (uint32_t)ix::shape_threads(ix::variant_shape(b->batch_variant)) != b->batch_threads)
        b->batch_variant = b->batch_threads == 64 ? 2 + 3 * ix::SHAPE_POOL_64
                                                  : (b->batch_threads == 256 ? 2 + 3 * ix::SHAPE_POOL_256
                                                                             : 2 + 3 * ix::SHAPE_POOL_128);
    return b;
}

void ix_backend_destroy(ix_backend* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    cudaFree(b->d_planes);
    cudaFree(b->d_sums);
    cudaFree(b->d_counter);
    cudaFree(b->d_dropped);
    cudaFree(b->d_check);
    cudaFree(b->d_attr_cls);
    cudaFree(b->d_attr_y);
    cudaFree(b->d_attr_map);
    cudaFree(b->d_batch_out);
    cudaFree(b->d_finishes);
    cudaFree(b->d_tools);
    cudaFree(b->d_acc);
    display_state_free(b->display);
    radiance_state_free(b->radiance);
    if (b->h_attr_map) cudaFreeHost(b->h_attr_map);
    if (b->h_sums) cudaFreeHost(b->h_sums);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    (void)cudaGetLastError();
    delete b;
}

int ix_backend_label(const ix_backend* b, char* buf, size_t len) {
    if (!b || !buf || len == 0) return -1;
    std::snprintf(buf, len, "%s", b->label.c_str());
    return 0;
}

void ix_set_pipeline_kind(ix_backend* b, uint32_t kind) {
    if (b) b->pipeline = kind;
}

void ix_set_work_limits(ix_backend* b, const ix_work_limits* limits) {
    if (b && limits) b->limits = *limits;
}

void ix_set_precision(ix_backend* b, uint32_t precision) {
    if (b) b->precision = precision ? IX_PRECISION_EXACT : IX_PRECISION_FAST;
}

int ix_scene_routes_to_gpu(const ix_scene* s) {
    if (!s) return 0;
    if (s->n_planes > IX_MAX_PLANES || (s->n_planes && !s->planes)) return 0;
    if (s->width == 0 || s->height == 0) return 0;
    if ((uint64_t)s->width * s->height > 0xFFFFFFFFull) return 0;  // pixel indices are 32-bit
    const ix_material& m = s->material;
    if (m.has_e_dispersion && m.e_dispersion.kind > IX_DISP_CAUCHY) return 0;
    const ix_environment& e = s->environment;
    if (e.model > IX_ENV_DAYLIGHT_SUN && e.model != IX_ENV_UNIFORM) return 0;
    // The UV lamps are fluorescence sources; their scenes never reach the GPU
    // (gpu_backend/mod.rs:288-298).
    if (e.spectrum == IX_SPEC_GAUSSIAN) return 0;
    // DaylightSun enables next-event estimation (environment_supports_nee,
    // environment/nee.rs:60): the frosted facets' light samples are traced; a
    // Henyey-Greenstein event takes none under an analytic sun and carries no weight
    // (nee_contribution_hg_scatter and phase_pdf_for_mis are HDR-map only,
    // scattering/hg_nee.rs:165, hg.rs:573), so a scattering stone traces as it does
    // under any other model.
    if (m.dispersion.kind > IX_DISP_CAUCHY) return 0;
    // A biaxial indicatrix is traced as the anisotropic transport's biaxial arm; an
    // isotropic material carrying one (the reference's eigen-polarisation mean of the
    // isotropic absorption branch over a biaxial indicatrix) is not built.
    if (m.biaxial && !m.anisotropic) return 0;
    // Concave tools (tool_routing.rs:81): at most IX_MAX_TOOLS, each one valid.
    if (s->n_tools > IX_MAX_TOOLS || (s->n_tools && !s->tools)) return 0;
    for (uint32_t k = 0; k < s->n_tools; ++k)
        if (ix_tool_validate(&s->tools[k]) != IX_TOOL_OK) return 0;
    return 1;
}

int ix_tool_validate(const ix_tool* t) {
    // ToolPrimitive::validate (geometry/tool.rs:360), its checks in its order.
    if (!t) return IX_TOOL_NON_FINITE;
    for (int i = 0; i < 4; ++i)
        if (!std::isfinite(t->origin[i]) || !std::isfinite(t->axis[i]) || !std::isfinite(t->profile[i]) ||
            !std::isfinite(t->sweep_dir[i]))
            return IX_TOOL_NON_FINITE;
    if (t->kind > 3u) return IX_TOOL_UNKNOWN_KIND;
    if (t->sweep_kind > 2u) return IX_TOOL_UNKNOWN_SWEEP;
    if (t->pad[0] || t->pad[1] || t->profile[3] != 0.0f || t->sweep_dir[3] != 0.0f) return IX_TOOL_PADDING_NOT_ZERO;
    const float radii[3] = {t->origin[3], t->profile[0], t->profile[1]};
    const float hl = t->axis[3], stroke = t->profile[2];
    bool neg = false, all_nonpos = true;
    for (float r : radii) {
        neg = neg || r < 0.0f;
        all_nonpos = all_nonpos && r <= 0.0f;
    }
    const bool ball = t->kind == 0u;
    if (neg || all_nonpos || hl < 0.0f || (!ball && hl <= 0.0f) || (ball && hl != 0.0f) || stroke < 0.0f)
        return IX_TOOL_NON_POSITIVE_RADIUS;
    // Vec3::length: the square root of the left-to-right dot product, in f32.
    auto length = [](const float* v) {
        const float d = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
        return std::sqrt(d);
    };
    if (std::fabs(length(t->axis) - 1.0f) > 1e-4f) return IX_TOOL_AXIS_NOT_UNIT;
    if (t->sweep_kind == 2u) {
        const float dd = (t->sweep_dir[0] * t->axis[0] + t->sweep_dir[1] * t->axis[1]) + t->sweep_dir[2] * t->axis[2];
        if (std::fabs(length(t->sweep_dir) - 1.0f) > 1e-4f || std::fabs(dd) > 1e-4f) return IX_TOOL_AXIS_NOT_UNIT;
    }
    return IX_TOOL_OK;
}

// The scene with the call's tools when it passes any (ntools > 0), else the scene's own.
static ix_scene with_tools(const ix_scene* scene, const ix_tool* tools, uint32_t ntools) {
    ix_scene s = *scene;
    if (ntools) {
        s.tools = tools;
        s.n_tools = ntools;
    }
    return s;
}

int ix_scene_routes_to_gpu_with_tools(const ix_scene* scene, const ix_tool* tools, uint32_t ntools) {
    if (!scene) return 0;
    const ix_scene s = with_tools(scene, tools, ntools);
    return ix_scene_routes_to_gpu(&s);
}

int ix_accumulate(ix_backend* b, const ix_scene* scene, const ix_tool* tools, uint32_t ntools,
                  uint32_t sample_offset, uint32_t spp, float* accum_xyz, const volatile uint8_t* cancel) {
    if (!ix_scene_routes_to_gpu_with_tools(scene, tools, ntools)) return IX_DECLINED;
    const ix_scene s = with_tools(scene, tools, ntools);
    return accumulate_impl<float>(b, &s, sample_offset, spp, accum_xyz, cancel);
}

int ix_accumulate_f64(ix_backend* b, const ix_scene* scene, const ix_tool* tools, uint32_t ntools,
                      uint32_t sample_offset, uint32_t spp, double* accum_xyz, const volatile uint8_t* cancel) {
    if (!ix_scene_routes_to_gpu_with_tools(scene, tools, ntools)) return IX_DECLINED;
    const ix_scene s = with_tools(scene, tools, ntools);
    return accumulate_impl<double>(b, &s, sample_offset, spp, accum_xyz, cancel);
}

int ix_accumulate_attributed(ix_backend* b, const ix_scene* scene, const ix_metrics_lighting* lighting,
                             uint32_t sample_offset, uint32_t spp, double* accum_xyz,
                             ix_attribution_pixel* attribution, const volatile uint8_t* cancel) {
    if (!b || !scene || !accum_xyz || !lighting) return IX_DECLINED;
    const uint64_t n_pixels = (uint64_t)scene->width * scene->height;
    // AttributionMap::checked (attribution_map.rs:201): a map of more than
    // MAX_DIAGNOSTIC_PIXELS pixels accepts no sample; the frame is still traced.
    if (!attribution || n_pixels > IX_ATTRIBUTION_MAX_PIXELS)
        return accumulate_impl<double>(b, scene, sample_offset, spp, accum_xyz, cancel);
    // The recorder does not follow interior scattering events (PathEvents::scatter).
    if (b->lost) return IX_DECLINED;
    if (!ix_scene_routes_to_gpu(scene)) return IX_DECLINED;
    if (b->limits.max_pixels && n_pixels > b->limits.max_pixels) return IX_DECLINED;
    if (b->limits.max_spp && spp > b->limits.max_spp) return IX_DECLINED;
    if (b->limits.max_paths_per_call && n_pixels * spp > b->limits.max_paths_per_call) return IX_DECLINED;
    ix::AttrLaunch A;
    std::memset(&A, 0, sizeof(A));
    if (!exit_lighting_setup(*lighting, &A.env, &A.spec, &A.factor, &A.head_shadow_cos, A.dirs)) return IX_DECLINED;
    if (cancel && *cancel) return IX_CANCELLED;
    if (n_pixels == 0 || spp == 0) return IX_DONE;
    // The records of the largest launch: whole pixels of at most max(budget, spp) paths.
    const uint64_t max_budget = std::max(chunk_budget(b, 0), chunk_budget(b, 1));
    const size_t records = (size_t)std::min<uint64_t>(n_pixels * spp, std::max<uint64_t>(max_budget, spp));
    Turn turn(b);
    if (fail(b, cudaSetDevice(b->device), "set device")) return IX_DECLINED;
    if (fail(b, grow_device(&b->d_planes, &b->planes_cap, (size_t)scene->n_planes * 4), "planes alloc") ||
        fail(b, grow_device(&b->d_sums, &b->sums_cap, (size_t)n_pixels * 3), "sums alloc") ||
        fail(b, grow_pinned(&b->h_sums, &b->hsums_cap, (size_t)n_pixels * 3), "host alloc") ||
        fail(b, grow_device(&b->d_attr_cls, &b->attr_cls_cap, records), "attribution alloc") ||
        fail(b, grow_device(&b->d_attr_y, &b->attr_y_cap, records), "attribution alloc") ||
        fail(b, grow_device(&b->d_attr_map, &b->attr_map_cap, (size_t)n_pixels), "attribution alloc") ||
        fail(b, grow_pinned(&b->h_attr_map, &b->hattr_map_cap, (size_t)n_pixels), "attribution host alloc"))
        return IX_DECLINED;
    const size_t map_bytes = (size_t)n_pixels * sizeof(ix_attribution_pixel);
    std::memcpy(b->h_attr_map, attribution, map_bytes);
    if (scene->n_planes &&
        fail(b, cudaMemcpyAsync(b->d_planes, scene->planes, (size_t)scene->n_planes * 16,
                                cudaMemcpyHostToDevice, b->stream), "planes upload"))
        return IX_DECLINED;
    if (fail(b, cudaMemcpyAsync(b->d_attr_map, b->h_attr_map, map_bytes, cudaMemcpyHostToDevice, b->stream),
             "attribution upload") ||
        fail(b, cudaMemsetAsync(b->d_dropped, 0, sizeof(unsigned long long), b->stream), "reset"))
        return IX_DECLINED;
    ix_scene sc = *scene;
    sc.planes = b->d_planes;
    if (!upload_finishes(b, sc, b->stream) || !upload_tools(b, sc, b->stream)) return IX_DECLINED;
    A.cls = b->d_attr_cls;
    A.y = b->d_attr_y;
    bool cancelled = false;
    if (fail(b, cudaEventRecord(b->ev0, b->stream), "event")) return IX_DECLINED;
    const int launches =
        enqueue_frame(b, sc, sample_offset, spp, b->d_sums, 0, b->stream, cancel, &cancelled, &A, b->d_attr_map);
    if (launches < 0) return IX_DECLINED;
    if (fail(b, cudaEventRecord(b->ev1, b->stream), "event")) return IX_DECLINED;
    if (cancelled) {
        cudaStreamSynchronize(b->stream);
        return IX_CANCELLED;
    }
    auto t0 = std::chrono::steady_clock::now();
    unsigned long long dropped = 0;
    if (fail(b, cudaMemcpyAsync(b->h_sums, b->d_sums, (size_t)n_pixels * 3 * sizeof(double),
                                cudaMemcpyDeviceToHost, b->stream), "sums download") ||
        fail(b, cudaMemcpyAsync(b->h_attr_map, b->d_attr_map, map_bytes, cudaMemcpyDeviceToHost, b->stream),
             "attribution download") ||
        fail(b, cudaMemcpyAsync(&dropped, b->d_dropped, sizeof(dropped), cudaMemcpyDeviceToHost, b->stream),
             "dropped download"))
        return IX_DECLINED;
    if (fail(b, cudaStreamSynchronize(b->stream), "attributed trace")) return IX_DECLINED;
    if (cancel && *cancel) return IX_CANCELLED;
    for (size_t i = 0; i < (size_t)n_pixels * 3; ++i) accum_xyz[i] += b->h_sums[i];
    std::memcpy(attribution, b->h_attr_map, map_bytes);
    auto t1 = std::chrono::steady_clock::now();
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->timing.kernel_ms = ms;
    b->timing.reduce_ms = std::chrono::duration<float, std::milli>(t1 - t0).count();
    b->timing.paths = n_pixels * spp;
    b->timing.launches = (uint32_t)launches * 2;  // the attributed trace and its record fold
    b->dropped = dropped;
    return IX_DONE;
}

}  // extern "C"

// ------------------------------------------------------------------------------------
// Batched plans: many scenes (stones x tilts) traced by one persistent launch.
// ------------------------------------------------------------------------------------
struct ix_batch_plan {
    ix_backend* b = nullptr;
    uint32_t n_scenes = 0, n_jobs = 0, total_tasks = 0, total_chunks = 0;
    uint64_t out_doubles = 0, paths = 0;
    bool pool_ok = true;  // every job fits the path-pool loop (spp <= FIXED_MAX_SAMPLES)
    unsigned long long* d_acc = nullptr;  // fixed-point sums, FIXED_WORDS per pixel of every job
    ix_scene* d_scenes = nullptr;
    uint32_t* d_flags = nullptr;
    uint32_t uniaxial = 0;  // transport instantiation (ix::TransportClass): the largest of the scenes'
    ix::BatchJob* d_jobs = nullptr;
    float* d_planes = nullptr;
    double* d_out = nullptr;
    uint32_t* d_counter = nullptr;
    unsigned long long* d_dropped = nullptr;
    std::vector<ix::BatchJob> jobs;
    std::vector<uint64_t> job_out;  // first double of each job's sums
    std::vector<uint32_t> h_max_bounces;  // per scene
    // CUDA graph of [counter reset, batch kernel], rebuilt when the stream or the variant
    // changes.
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t graph_stream = nullptr;
    int graph_variant = -1;
    uint32_t variant = 0;
    bool tuned = false;
    bool out_pooled = false;  // d_out is the backend's pooled buffer
    // The wavefront pipeline's buffers (allocated on its first run) and its two-iteration
    // CUDA graph.
    uint32_t* wf_pw = nullptr;
    uint32_t* wf_queues = nullptr;
    uint32_t* wf_counts = nullptr;
    unsigned long long* wf_claim = nullptr;
    uint32_t wf_capacity = 0;
    unsigned long long* h_wf = nullptr;  // pinned: the claim counter, the next active count
    cudaGraph_t wf_graph = nullptr;
    cudaGraphExec_t wf_exec = nullptr;
    cudaStream_t wf_stream = nullptr;
    uint32_t wf_iterations = 0;  // of the last wavefront run
    uint8_t* d_finishes = nullptr;  // every scene's facet finishes, back to back
    ix_tool* d_tools = nullptr;     // every scene's concave tools, back to back
};

namespace {

void plan_free_graph(ix_batch_plan* p) {
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    p->exec = nullptr;
    p->graph = nullptr;
    p->graph_variant = -1;
}

// Resident CTAs per SM of batch variant `v` for plan `p` in the backend's rounding build
// (0: the build does not carry it, or the plan cannot run it).
int plan_blocks_per_sm(const ix_batch_plan* p, uint32_t v) {
    if (v == (uint32_t)ix::VARIANT_WAVEFRONT) {
        // Isotropic plans only; the same padded path space as the pool loop.
        if (p->uniaxial || !p->pool_ok) return 0;
        return p->b->precision == IX_PRECISION_EXACT ? ix::wavefront_blocks_per_sm_exact()
                                                     : ix::wavefront_blocks_per_sm_fast();
    }
    if (v >= (uint32_t)ix::N_VARIANTS) return 0;
    const int shape = ix::variant_shape((int)v);
    if (ix::shape_is_pool(shape) && !p->pool_ok) return 0;
    const int threads = ix::shape_threads(shape);
    return p->b->precision == IX_PRECISION_EXACT ? ix::batch_blocks_per_sm_exact(threads, (int)v, (int)p->uniaxial)
                                                 : ix::batch_blocks_per_sm_fast(threads, (int)v, (int)p->uniaxial);
}

// Enqueues one launch of variant `variant` over every `stride`-th task / chunk of the plan
// (stride 1: the whole plan) and, for the path-pool shapes, the rounding of its sums.
// The wavefront pipeline over the whole plan on `st`: start, then iterations from a
// two-iteration CUDA graph until every path has been claimed and no slot is active (the
// host reads the claim counter and the next active count every 16 iterations), then the
// fixed-point sums rounded to f64.  Synchronises `st`.
cudaError_t plan_run_wavefront(ix_batch_plan* p, cudaStream_t st) {
    ix_backend* b = p->b;
    const bool exact = b->precision == IX_PRECISION_EXACT;
    const int bps = plan_blocks_per_sm(p, ix::VARIANT_WAVEFRONT);
    if (bps <= 0) return cudaErrorInvalidValue;
    const uint64_t total_slots = (uint64_t)p->total_chunks * 32ull;
    const uint64_t pixels = p->out_doubles / 3;
    cudaError_t e = cudaSuccess;
    if (!p->wf_pw) {
        const uint32_t cap = (uint32_t)std::min<uint64_t>(1ull << 20, std::max<uint64_t>(total_slots, 1024));
        // One 512-byte state record per slot (path words, then lane words).
        e = cudaMalloc((void**)&p->wf_pw, (size_t)128 * cap * sizeof(uint32_t));
        if (e == cudaSuccess) e = cudaMalloc((void**)&p->wf_queues, (size_t)ix::WF_QUEUES * cap * sizeof(uint32_t));
        if (e == cudaSuccess) e = cudaMalloc((void**)&p->wf_counts, ix::WF_QUEUES * sizeof(uint32_t));
        if (e == cudaSuccess) e = cudaMalloc((void**)&p->wf_claim, sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMallocHost((void**)&p->h_wf, 2 * sizeof(unsigned long long));
        if (e != cudaSuccess) return e;
        p->wf_capacity = cap;
    }
    ix::WaveLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.scenes = p->d_scenes;
    L.flags = p->d_flags;
    L.jobs = p->d_jobs;
    L.n_jobs = p->n_jobs;
    L.total_slots = total_slots;
    L.acc = p->d_acc;
    L.dropped = p->d_dropped;
    L.claim = p->wf_claim;
    L.capacity = p->wf_capacity;
    L.pw = p->wf_pw;
    L.queues = p->wf_queues;
    L.counts = p->wf_counts;
    L.blocks = b->sm_count * bps;
    if (!p->wf_exec || p->wf_stream != st) {
        if (p->wf_exec) cudaGraphExecDestroy(p->wf_exec);
        if (p->wf_graph) cudaGraphDestroy(p->wf_graph);
        p->wf_exec = nullptr;
        p->wf_graph = nullptr;
        e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        cudaError_t e1 = exact ? ix::launch_wavefront_iteration_exact(L, 0, st) : ix::launch_wavefront_iteration_fast(L, 0, st);
        cudaError_t e2 = exact ? ix::launch_wavefront_iteration_exact(L, 1, st) : ix::launch_wavefront_iteration_fast(L, 1, st);
        cudaError_t e3 = cudaStreamEndCapture(st, &p->wf_graph);
        if (e1 != cudaSuccess) return e1;
        if (e2 != cudaSuccess) return e2;
        if (e3 != cudaSuccess) return e3;
        e = cudaGraphInstantiate(&p->wf_exec, p->wf_graph, 0);
        if (e != cudaSuccess) return e;
        p->wf_stream = st;
    }
    e = cudaMemsetAsync(p->d_acc, 0, pixels * ix::FIXED_WORDS * sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->wf_counts, 0, ix::WF_QUEUES * sizeof(uint32_t), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->wf_claim, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = exact ? ix::launch_wavefront_start_exact(L, st) : ix::launch_wavefront_start_fast(L, st);
    if (e != cudaSuccess) return e;
    // Every path advances one bounce per iteration and ends within max_bounces + 1 of them,
    // so the iterations are bounded: a run past the bound is an error, not a wait.  (A slot
    // whose claim lands in a job's padding retires early, so the slots left carry a few
    // more paths each; the bound allows twice the even share.)
    uint32_t max_bounces = 0;
    for (uint32_t j = 0; j < p->n_scenes; ++j) max_bounces = std::max(max_bounces, p->h_max_bounces[j]);
    const uint64_t bound = 2 * (total_slots / p->wf_capacity + 2) * (uint64_t)(max_bounces + 2) + 64;
    uint64_t iterations = 0;
    for (;;) {
        for (int k = 0; k < 8 && e == cudaSuccess; ++k) e = cudaGraphLaunch(p->wf_exec, st);
        iterations += 16;
        if (e == cudaSuccess) e = cudaMemcpyAsync(p->h_wf, p->wf_claim, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(p->h_wf + 1, p->wf_counts + ix::WF_ACTIVE0, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
        const uint32_t active = (uint32_t)(p->h_wf[1] & 0xFFFFFFFFull);
        if (active == 0 && p->h_wf[0] >= total_slots) break;
        if (iterations > bound) return cudaErrorLaunchTimeout;
    }
    p->wf_iterations = (uint32_t)std::min<uint64_t>(iterations, 0xFFFFFFFFull);
    return ix::launch_fixed_to_f64(p->d_acc, p->d_out, pixels, 0, st);
}

cudaError_t plan_enqueue(ix_batch_plan* p, cudaStream_t st, uint32_t variant, uint32_t stride = 1) {
    if (variant == (uint32_t)ix::VARIANT_WAVEFRONT) return plan_run_wavefront(p, st);
    ix_backend* b = p->b;
    const bool exact = b->precision == IX_PRECISION_EXACT;
    const int bps = plan_blocks_per_sm(p, variant);
    if (bps <= 0) return cudaErrorInvalidValue;
    const int shape = ix::variant_shape((int)variant);
    ix::BatchLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.scenes = p->d_scenes;
    L.flags = p->d_flags;
    L.uniaxial = p->uniaxial;
    L.jobs = p->d_jobs;
    L.n_jobs = p->n_jobs;
    L.total_tasks = p->total_tasks;
    L.total_chunks = p->total_chunks;
    L.out = p->d_out;
    L.accumulate = 0;
    L.task_counter = p->d_counter;
    L.dropped = p->d_dropped;
    L.stride = std::max<uint32_t>(1, stride);
    L.threads = ix::shape_threads(shape);
    L.variant = (int)variant;
    L.blocks = b->sm_count * bps;
    const uint64_t pixels = p->out_doubles / 3;
    if (ix::shape_is_pool(shape)) {
        L.acc = p->d_acc;
        cudaError_t e = cudaMemsetAsync(p->d_acc, 0, pixels * ix::FIXED_WORDS * sizeof(unsigned long long), st);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = exact ? ix::launch_batch_exact(L, st) : ix::launch_batch_fast(L, st);
    if (e != cudaSuccess || !ix::shape_is_pool(shape)) return e;
    return ix::launch_fixed_to_f64(p->d_acc, p->d_out, pixels, 0, st);
}

// ix_batch_plan_run / ix_batch_plan_download for a caller that already holds the
// backend's turn.
int plan_run_locked(ix_batch_plan* p, cudaStream_t st) {
    ix_backend* b = p->b;
    if (fail(b, cudaSetDevice(b->device), "set device")) return IX_DECLINED;
    if (p->variant == (uint32_t)ix::VARIANT_WAVEFRONT) {
        // Host-driven: its iteration count depends on the paths, so it is not one graph.
        if (fail(b, cudaEventRecord(b->ev0, st), "event")) return IX_DECLINED;
        if (fail(b, plan_run_wavefront(p, st), "wavefront")) return IX_DECLINED;
        if (fail(b, cudaEventRecord(b->ev1, st), "event")) return IX_DECLINED;
        b->timing.paths = p->paths;
        b->timing.launches = 3 * p->wf_iterations + 2;
        return IX_DONE;
    }
    if (!p->exec || p->graph_stream != st || p->graph_variant != (int)p->variant) {
        plan_free_graph(p);
        if (fail(b, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "graph capture")) return IX_DECLINED;
        cudaError_t e = plan_enqueue(p, st, p->variant);
        cudaError_t e2 = cudaStreamEndCapture(st, &p->graph);
        if (fail(b, e, "batch launch") || fail(b, e2, "graph capture")) return IX_DECLINED;
        if (fail(b, cudaGraphInstantiate(&p->exec, p->graph, 0), "graph instantiate")) return IX_DECLINED;
        p->graph_stream = st;
        p->graph_variant = (int)p->variant;
    }
    if (fail(b, cudaEventRecord(b->ev0, st), "event")) return IX_DECLINED;
    if (fail(b, cudaGraphLaunch(p->exec, st), "graph launch")) return IX_DECLINED;
    if (fail(b, cudaEventRecord(b->ev1, st), "event")) return IX_DECLINED;
    b->timing.paths = p->paths;
    b->timing.launches = ix::shape_is_pool(ix::variant_shape((int)p->variant)) ? 2 : 1;
    return IX_DONE;
}
int plan_download_locked(ix_batch_plan* p, double* host_out) {
    ix_backend* b = p->b;
    if (fail(b, cudaMemcpyAsync(host_out, p->d_out, p->out_doubles * sizeof(double), cudaMemcpyDeviceToHost,
                                b->stream), "batch download"))
        return -1;
    if (fail(b, cudaStreamSynchronize(b->stream), "batch download")) return -1;
    return 0;
}

}  // namespace

extern "C" {

// ix_batch_plan_create for a caller that holds the backend's turn.  With `pooled_out` the
// plan's sums live in the backend's pooled device buffer (the one-shot batch entry, which
// destroys its plan within the same turn).
static ix_batch_plan* plan_create_locked(ix_backend* b, const ix_scene* scenes, uint32_t n_scenes,
                                         const ix_batch_job* jobs, uint32_t n_jobs, bool pooled_out) {
    if (fail(b, cudaSetDevice(b->device), "set device")) return nullptr;
    ix_batch_plan* p = new ix_batch_plan();
    p->b = b;
    p->n_scenes = n_scenes;
    p->n_jobs = n_jobs;
    // Job table: tasks of ~64 paths (static task loop) and chunks of 32 paths (path-pool
    // loop), jobs laid out back to back.
    uint64_t task = 0, out = 0, chunk = 0;
    p->jobs.resize(n_jobs);
    p->job_out.resize(n_jobs);
    for (uint32_t j = 0; j < n_jobs; ++j) {
        const ix_batch_job& in = jobs[j];
        if (in.scene >= n_scenes || in.spp == 0) {
            delete p;
            return nullptr;
        }
        const ix_scene& sc = scenes[in.scene];
        ix::BatchJob& bj = p->jobs[j];
        bj.scene = in.scene;
        bj.n_pixels = sc.width * sc.height;
        bj.spp = in.spp;
        bj.ppt = pixels_per_task(in.spp);
        bj.task_begin = (uint32_t)task;
        bj.sample_offset = in.sample_offset;
        bj.out_offset = out;
        const uint64_t job_paths = (uint64_t)bj.n_pixels * in.spp;
        if ((uint64_t)sc.width * sc.height > 0xFFFFFFFFull || job_paths > 0xFFFFFFFFull - 32) {
            delete p;
            return nullptr;
        }
        bj.paths = (uint32_t)job_paths;
        bj.chunk_begin = (uint32_t)std::min<uint64_t>(chunk, 0xFFFFFFFFull);
        bj.acc_offset = out / 3 * ix::FIXED_WORDS;
        if (in.spp > ix::FIXED_MAX_SAMPLES) p->pool_ok = false;
        p->job_out[j] = out;
        task += (bj.n_pixels + bj.ppt - 1) / bj.ppt;
        chunk += (job_paths + 31) / 32;
        out += (uint64_t)bj.n_pixels * 3;
        p->paths += job_paths;
    }
    if (task >= 0xFFFFFFFFull) {
        delete p;
        return nullptr;
    }
    if (chunk >= 0xFFFFFFFFull) p->pool_ok = false;
    p->total_tasks = (uint32_t)task;
    p->total_chunks = p->pool_ok ? (uint32_t)chunk : 0;
    p->out_doubles = out;
    uint64_t plane_floats = 0;
    for (uint32_t i = 0; i < n_scenes; ++i) plane_floats += (uint64_t)scenes[i].n_planes * 4;
    std::vector<ix_scene> dev_scenes(scenes, scenes + n_scenes);
    std::vector<uint32_t> flags(n_scenes);
    std::vector<float> planes(std::max<uint64_t>(plane_floats, 4));
    std::vector<uint8_t> finishes;
    std::vector<size_t> finish_off(n_scenes, 0);
    for (uint32_t i = 0; i < n_scenes; ++i)
        if (scenes[i].facet_finishes && scenes[i].n_finishes) {
            finish_off[i] = finishes.size();
            finishes.insert(finishes.end(), scenes[i].facet_finishes,
                            scenes[i].facet_finishes + scenes[i].n_finishes);
        }
    std::vector<ix_tool> tools;
    std::vector<size_t> tool_off(n_scenes, 0);
    for (uint32_t i = 0; i < n_scenes; ++i)
        if (scenes[i].tools && scenes[i].n_tools) {
            tool_off[i] = tools.size();
            tools.insert(tools.end(), scenes[i].tools, scenes[i].tools + scenes[i].n_tools);
        }
    uint64_t off = 0;
    bool ok = cudaMalloc((void**)&p->d_planes, planes.size() * sizeof(float)) == cudaSuccess;
    ok = ok && (finishes.empty() || (cudaMalloc((void**)&p->d_finishes, finishes.size()) == cudaSuccess &&
                                     cudaMemcpy(p->d_finishes, finishes.data(), finishes.size(),
                                                cudaMemcpyHostToDevice) == cudaSuccess));
    ok = ok && (tools.empty() || (cudaMalloc((void**)&p->d_tools, tools.size() * sizeof(ix_tool)) == cudaSuccess &&
                                  cudaMemcpy(p->d_tools, tools.data(), tools.size() * sizeof(ix_tool),
                                             cudaMemcpyHostToDevice) == cudaSuccess));
    for (uint32_t i = 0; ok && i < n_scenes; ++i) {
        std::memcpy(planes.data() + off, scenes[i].planes, (size_t)scenes[i].n_planes * 16);
        dev_scenes[i].planes = p->d_planes + off;
        const bool has_finishes = scenes[i].facet_finishes && scenes[i].n_finishes;
        dev_scenes[i].facet_finishes = has_finishes ? p->d_finishes + finish_off[i] : nullptr;
        dev_scenes[i].n_finishes = has_finishes ? scenes[i].n_finishes : 0;
        const bool has_tools = scenes[i].tools && scenes[i].n_tools;
        dev_scenes[i].tools = has_tools ? p->d_tools + tool_off[i] : nullptr;
        dev_scenes[i].n_tools = has_tools ? scenes[i].n_tools : 0;
        flags[i] = ix::scene_flags(dev_scenes[i]);
        p->h_max_bounces.push_back(scenes[i].max_bounces);
        p->uniaxial = std::max(p->uniaxial, (uint32_t)ix::transport_class(flags[i]));
        off += (uint64_t)scenes[i].n_planes * 4;
    }
    ok = ok && cudaMalloc((void**)&p->d_scenes, n_scenes * sizeof(ix_scene)) == cudaSuccess &&
         cudaMalloc((void**)&p->d_flags, n_scenes * sizeof(uint32_t)) == cudaSuccess &&
         cudaMalloc((void**)&p->d_jobs, n_jobs * sizeof(ix::BatchJob)) == cudaSuccess &&
         (pooled_out ? grow_device(&b->d_batch_out, &b->batch_out_cap, std::max<uint64_t>(out, 1))
                     : cudaMalloc((void**)&p->d_out, std::max<uint64_t>(out, 1) * sizeof(double))) == cudaSuccess &&
         cudaMalloc((void**)&p->d_counter, sizeof(uint32_t)) == cudaSuccess &&
         cudaMalloc((void**)&p->d_dropped, sizeof(unsigned long long)) == cudaSuccess &&
         (!p->pool_ok || cudaMalloc((void**)&p->d_acc, std::max<uint64_t>(out / 3, 1) * ix::FIXED_WORDS *
                                                          sizeof(unsigned long long)) == cudaSuccess);
    if (ok && pooled_out) {
        p->d_out = b->d_batch_out;
        p->out_pooled = true;
    }
    ok = ok && cudaMemcpy(p->d_planes, planes.data(), planes.size() * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(p->d_scenes, dev_scenes.data(), n_scenes * sizeof(ix_scene), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(p->d_flags, flags.data(), n_scenes * sizeof(uint32_t), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(p->d_jobs, p->jobs.data(), n_jobs * sizeof(ix::BatchJob), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(p->d_dropped, 0, sizeof(unsigned long long)) == cudaSuccess;
    p->variant = b->batch_variant;
    if (b->pipeline == IX_PIPELINE_WAVEFRONT && ok && plan_blocks_per_sm(p, ix::VARIANT_WAVEFRONT) > 0)
        p->variant = ix::VARIANT_WAVEFRONT;
    if (ok && plan_blocks_per_sm(p, p->variant) <= 0) p->variant = ix::variant_budget((int)p->variant % ix::N_VARIANTS);
    if (!ok) {
        fail(b, cudaGetLastError(), "batch plan");
        ix_batch_plan_destroy(p);
        return nullptr;
    }
    return p;
}

ix_batch_plan* ix_batch_plan_create(ix_backend* b, const ix_scene* scenes, uint32_t n_scenes,
                                    const ix_batch_job* jobs, uint32_t n_jobs) {
    if (!b || !scenes || !jobs || n_scenes == 0 || n_jobs == 0 || b->lost) return nullptr;
    for (uint32_t i = 0; i < n_scenes; ++i)
        if (!ix_scene_routes_to_gpu(&scenes[i])) return nullptr;
    Turn turn(b);
    return plan_create_locked(b, scenes, n_scenes, jobs, n_jobs, false);
}

int ix_batch_plan_run(ix_batch_plan* p, void* stream) {
    if (!p || p->b->lost) return IX_DECLINED;
    Turn turn(p->b);
    return plan_run_locked(p, stream ? (cudaStream_t)stream : p->b->stream);
}

int ix_batch_plan_autotune(ix_batch_plan* p, int reps, uint32_t* chosen) {
    if (!p || p->b->lost) return -1;
    ix_backend* b = p->b;
    Turn turn(b);
    if (fail(b, cudaSetDevice(b->device), "set device")) return -1;
    // Each candidate is timed on every stride-th task / chunk of the plan: about 1/16 of
    // its work, spread over all its jobs, and never fewer claims than the grid has warps.
    // The sample ranks the candidates; the best kFinalists then run the whole plan once
    // each and the fastest of those is kept (a strided sample changes the job mix each warp
    // sees, which can reorder candidates a few percent apart).
    const uint64_t units = std::max<uint64_t>(1, std::min(p->total_tasks, p->pool_ok ? p->total_chunks : p->total_tasks));
    const uint64_t min_claims = (uint64_t)b->sm_count * 64 * 4;
    const uint32_t stride = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(16, units / min_claims));
    auto time_variant = [&](uint32_t v, uint32_t st, float* ms) -> bool {
        if (fail(b, cudaEventRecord(b->ev0, b->stream), "event")) return false;
        if (fail(b, plan_enqueue(p, b->stream, v, st), "autotune launch")) return false;
        if (fail(b, cudaEventRecord(b->ev1, b->stream), "event")) return false;
        if (fail(b, cudaStreamSynchronize(b->stream), "autotune")) return false;
        *ms = 0.0f;
        cudaEventElapsedTime(ms, b->ev0, b->ev1);
        return true;
    };
    std::vector<std::pair<float, uint32_t>> ranked;
    for (uint32_t v = 0; v < (uint32_t)ix::N_VARIANTS; ++v) {
        if (plan_blocks_per_sm(p, v) <= 0) continue;
        if (b->batch_threads && (uint32_t)ix::shape_threads(ix::variant_shape((int)v)) != b->batch_threads) continue;
        float total = 0.0f;
        for (int r = 0; r < std::max(1, reps) + 1; ++r) {
            float ms = 0.0f;
            if (!time_variant(v, stride, &ms)) return -1;
            if (r > 0) total += ms;  // the first run of a candidate warms it up
        }
        ranked.emplace_back(total, v);
    }
    uint32_t best_v = p->variant;
    if (!ranked.empty()) {
        std::sort(ranked.begin(), ranked.end());
        best_v = ranked[0].second;
        if (stride > 1 && ranked.size() > 1) {
            // Finalists: the two best of the sample, and the best of each loop (static
            // tasks, path pool) -- the sample favours neither loop reliably.
            std::vector<uint32_t> finalists;
            auto add = [&](uint32_t v) {
                if (std::find(finalists.begin(), finalists.end(), v) == finalists.end()) finalists.push_back(v);
            };
            add(ranked[0].second);
            add(ranked[1].second);
            for (bool pool : {false, true})
                for (const auto& r : ranked)
                    if (ix::shape_is_pool(ix::variant_shape((int)r.second)) == pool) {
                        add(r.second);
                        break;
                    }
            // The wavefront pipeline (isotropic plans) runs the whole plan only.
            if (plan_blocks_per_sm(p, ix::VARIANT_WAVEFRONT) > 0) add((uint32_t)ix::VARIANT_WAVEFRONT);
            float best = 1e30f;
            for (uint32_t v : finalists) {
                float ms = 0.0f;
                if (!time_variant(v, 1, &ms)) return -1;
                if (ms < best) {
                    best = ms;
                    best_v = v;
                }
            }
        }
    }
    p->variant = best_v;
    p->tuned = true;
    b->batch_variant = best_v;  // later plans of this backend start from the pick
    if (chosen) *chosen = best_v;
    return 0;
}

int ix_batch_plan_set_variant(ix_batch_plan* p, uint32_t variant) {
    if (!p || p->b->lost) return -1;
    Turn turn(p->b);
    if (plan_blocks_per_sm(p, variant) <= 0) return -1;
    p->variant = variant;
    return 0;
}

int ix_batch_plan_download(ix_batch_plan* p, double* host_out) {
    if (!p || !host_out || p->b->lost) return -1;
    Turn turn(p->b);
    return plan_download_locked(p, host_out);
}

uint64_t ix_batch_plan_output_size(const ix_batch_plan* p) { return p ? p->out_doubles : 0; }
const double* ix_batch_plan_device_output(const ix_batch_plan* p) { return p ? p->d_out : nullptr; }
uint64_t ix_batch_plan_paths(const ix_batch_plan* p) { return p ? p->paths : 0; }
uint32_t ix_batch_plan_variant(const ix_batch_plan* p) { return p ? p->variant : 0; }

uint64_t ix_batch_plan_job_offset(const ix_batch_plan* p, uint32_t job) {
    return (p && job < p->n_jobs) ? p->job_out[job] : 0;
}

void ix_batch_plan_destroy(ix_batch_plan* p) {
    if (!p) return;
    cudaSetDevice(p->b->device);
    cudaStreamSynchronize(p->b->stream);
    plan_free_graph(p);
    cudaFree(p->d_scenes);
    cudaFree(p->d_flags);
    cudaFree(p->d_jobs);
    cudaFree(p->d_planes);
    cudaFree(p->d_finishes);
    cudaFree(p->d_tools);
    if (!p->out_pooled) cudaFree(p->d_out);
    cudaFree(p->d_acc);
    cudaFree(p->d_counter);
    cudaFree(p->d_dropped);
    if (p->wf_exec) cudaGraphExecDestroy(p->wf_exec);
    if (p->wf_graph) cudaGraphDestroy(p->wf_graph);
    cudaFree(p->wf_pw);
    cudaFree(p->wf_queues);
    cudaFree(p->wf_counts);
    cudaFree(p->wf_claim);
    if (p->h_wf) cudaFreeHost(p->h_wf);
    (void)cudaGetLastError();
    delete p;
}

int ix_accumulate_batch(ix_backend* b, ix_batch_item* items, uint32_t n_items, const volatile uint8_t* cancel,
                        ix_batch_done_fn on_done, void* user) {
    if (!b || (!items && n_items)) return IX_DECLINED;
    if (n_items == 0) return IX_DONE;
    // on_done (backend.rs:451): once per item, in index order, after its outcome is final.
    auto report = [&](uint32_t i) {
        if (on_done) on_done(user, i, items[i].status);
    };
    if (cancel && *cancel) {
        for (uint32_t j = 0; j < n_items; ++j) {
            items[j].status = IX_CANCELLED;
            report(j);
        }
        return IX_CANCELLED;
    }
    // Items the CUDA path cannot trace are declined individually; the rest run in one
    // persistent launch.
    std::vector<ix_scene> scenes;
    std::vector<ix_batch_job> jobs;
    std::vector<uint32_t> which;
    for (uint32_t i = 0; i < n_items; ++i) {
        items[i].status = IX_DECLINED;
        if (!items[i].scene || !items[i].accum_xyz || !ix_scene_routes_to_gpu(items[i].scene)) continue;
        if (items[i].spp == 0 || items[i].scene->width * items[i].scene->height == 0) {
            items[i].status = IX_DONE;
            continue;
        }
        jobs.push_back(ix_batch_job{(uint32_t)scenes.size(), items[i].sample_offset, items[i].spp});
        scenes.push_back(*items[i].scene);
        which.push_back(i);
    }
    {
        // Items that will not be traced (declined, or nothing to trace) are final now.
        size_t k = 0;
        for (uint32_t i = 0; i < n_items; ++i) {
            if (k < which.size() && which[k] == i) {
                ++k;
                continue;
            }
            report(i);
        }
    }
    if (!jobs.empty()) {
        if (b->lost) {
            for (uint32_t k : which) report(k);
            return IX_DECLINED;
        }
        // One turn for the whole call: the plan's sums sit in the backend's pooled device
        // buffer and come back through its pinned staging buffer, which no other call may
        // touch meanwhile.
        Turn turn(b);
        ix_batch_plan* p = plan_create_locked(b, scenes.data(), (uint32_t)scenes.size(), jobs.data(),
                                              (uint32_t)jobs.size(), true);
        if (!p) {
            for (uint32_t k : which) report(k);
            return IX_DECLINED;
        }
        bool ok = !fail(b, grow_pinned(&b->h_sums, &b->hsums_cap, (size_t)p->out_doubles), "host alloc") &&
                  plan_run_locked(p, b->stream) == IX_DONE && plan_download_locked(p, b->h_sums) == 0;
        if (ok && !(cancel && *cancel)) {
            // Add into the callers' accumulators, items split over a few host threads.
            const unsigned nt = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
            auto add = [&](unsigned t) {
                for (size_t k = t; k < which.size(); k += nt) {
                    ix_batch_item& it = items[which[k]];
                    const double* src = b->h_sums + p->job_out[k];
                    const size_t n = (size_t)it.scene->width * it.scene->height * 3;
                    for (size_t e = 0; e < n; ++e) it.accum_xyz[e] += src[e];
                }
            };
            std::vector<std::thread> pool;
            for (unsigned t = 1; t < nt && t < which.size(); ++t) pool.emplace_back(add, t);
            add(0);
            for (auto& th : pool) th.join();
            for (uint32_t k : which) items[k].status = IX_DONE;
        } else if (ok) {
            for (uint32_t k : which) items[k].status = IX_CANCELLED;
        }
        ix_batch_plan_destroy(p);
    }
    for (uint32_t k : which) report(k);
    int overall = IX_DONE;
    for (uint32_t i = 0; i < n_items; ++i)
        if (items[i].status != IX_DONE) {
            overall = items[i].status;
            break;
        }
    return overall;
}

// Whether the device can read `p` (device or managed memory); a null array is fine.
static bool device_readable(const void* p) {
    if (!p) return true;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int ix_accumulate_device(ix_backend* b, const ix_scene* scene, uint32_t sample_offset,
                         uint32_t spp, double* d_accum_xyz, int accumulate, void* stream) {
    if (!b || !scene || !d_accum_xyz) return IX_DECLINED;
    if (b->lost || !ix::routes_device_scene(scene)) return IX_DECLINED;
    // A host array here would fault the kernel: decline it instead.
    if (!device_readable(scene->planes) || !device_readable(scene->facet_finishes) ||
        !device_readable(scene->tools) || !device_readable(d_accum_xyz))
        return IX_DECLINED;
    if ((uint64_t)scene->width * scene->height == 0 || spp == 0) return IX_DONE;
    Turn turn(b);
    cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    if (fail(b, cudaSetDevice(b->device), "set device")) return IX_DECLINED;
    bool cancelled = false;
    if (fail(b, cudaEventRecord(b->ev0, st), "event")) return IX_DECLINED;
    int launches = enqueue_frame(b, *scene, sample_offset, spp, d_accum_xyz, accumulate, st, nullptr, &cancelled);
    if (launches < 0) return IX_DECLINED;
    if (fail(b, cudaEventRecord(b->ev1, st), "event")) return IX_DECLINED;
    b->timing.paths = (uint64_t)scene->width * scene->height * spp;
    b->timing.launches = (uint32_t)launches * kernels_per_launch(b, *scene);
    return IX_DONE;
}

int ix_is_lost(const ix_backend* b) { return b ? (b->lost ? 1 : 0) : 1; }

int ix_try_recover(ix_backend* b) {
    if (!b) return 0;
    if (!b->lost) return 1;
    // A sticky device error needs a fresh context; probe with a synchronize.
    cudaSetDevice(b->device);
    cudaError_t e = cudaStreamSynchronize(b->stream);
    (void)cudaGetLastError();
    if (e == cudaSuccess) {
        b->lost = false;
        b->last_error.clear();
        return 1;
    }
    return 0;
}

int ix_last_error(const ix_backend* b, char* buf, size_t len) {
    if (!b || !buf || len == 0) return -1;
    std::snprintf(buf, len, "%s", b->last_error.c_str());
    return (int)b->last_error.size();
}

int ix_last_timing(const ix_backend* b, ix_timing* out) {
    if (!b || !out) return -1;
    ix_timing t = b->timing;
    if (t.launches && b->ev1) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess) t.kernel_ms = ms;
        (void)cudaGetLastError();
    }
    *out = t;
    return 0;
}

uint64_t ix_last_dropped(const ix_backend* b) { return b ? b->dropped : 0; }

int ix_probe_fp32_peak(ix_backend* b, double* flops) {
    if (!b || !flops) return -1;
    Turn turn(b);
    if (fail(b, cudaSetDevice(b->device), "set device")) return -1;
    if (fail(b, ix::fp32_probe(b->sm_count, 5, b->stream, flops), "fp32 probe")) return -1;
    return 0;
}

void ix_camera_new(float yaw, float pitch, float distance, float fov_deg, ix_camera* out) {
    float cos_p = std::cos(pitch), sin_p = std::sin(pitch), cos_y = std::cos(yaw), sin_y = std::sin(yaw);
    H3 origin = h3(distance * cos_p * sin_y, distance * sin_p, distance * cos_p * cos_y);
    H3 forward = hnormalize(h3(-origin.x, -origin.y, -origin.z));
    H3 world_up = std::fabs(cos_p) < 1e-4f ? h3(0.0f, 0.0f, -1.0f)
                  : (cos_p < 0.0f ? h3(0.0f, -1.0f, 0.0f) : h3(0.0f, 1.0f, 0.0f));
    H3 right = hnormalize(hcross(forward, world_up));
    H3 up = hnormalize(hcross(right, forward));
    hstore(out->origin, origin);
    hstore(out->forward, forward);
    hstore(out->right, right);
    hstore(out->up, up);
    out->fov_tan = std::tan(to_radians(fov_deg) * 0.5f);
}

int ix_environment_preset(int32_t preset, float exposure, float light_yaw, float light_pitch,
                          float backdrop, float surface_glare, float head_shadow_deg,
                          ix_environment* out) {
    if (!out) return -1;
    std::memset(out, 0, sizeof(*out));
    // LightingPreset::params / model / uses_d65 / uv_line (environment/mod.rs:318-560).
    float temp_k = 6500.0f, spot = 1.0f;
    float tent[5] = {1.0f, 1.0f, 1.0f, 0.02f, 0.0f};  // walls, cards, spark, ground, flat
    bool d65 = true, uv = false;
    float uv_centre = 0.0f, uv_fwhm = 0.0f;
    uint32_t model;
    switch (preset) {
        case 0: model = IX_ENV_LIGHT_TENT; temp_k = 5000.0f; d65 = false; break;        // LightTent
        case 1: model = IX_ENV_ISO_HEMISPHERE; break;                                    // IsoHemisphere
        case 2: model = IX_ENV_LIGHT_TENT; spot = 0.0f; tent[0] = 5.0f; tent[1] = 0.0f;  // WhiteTray
                tent[2] = 0.0f; tent[3] = 0.8f; tent[4] = 1.0f; break;
        case 3: model = IX_ENV_LIGHT_TENT; tent[0] = 3.0f; tent[1] = 0.0f; tent[3] = 0.05f; break;  // ShopLights
        case 4: model = IX_ENV_LIGHT_TENT; tent[0] = 0.4f; tent[1] = 0.0f; tent[2] = 0.0f;          // WindowDaylight
                tent[3] = 0.03f; break;
        case 5: model = IX_ENV_DAYLIGHT_DOME; break;                                     // DaylightDome
        case 6: model = IX_ENV_DAYLIGHT_SUN; break;                                      // DaylightSun
        case 7: model = IX_ENV_STUDIO; break;                                            // Daylight
        case 8: model = IX_ENV_STUDIO; temp_k = 3200.0f; spot = 1.2f; d65 = false; break;  // Incandescent
        case 9: model = IX_ENV_STUDIO; temp_k = 2856.0f; spot = 1.2f; d65 = false; break;  // IlluminantA
        case 10: model = IX_ENV_STUDIO; temp_k = 5000.0f; spot = 1.6f; d65 = false; break;  // RingLights
        case 11: model = IX_ENV_STUDIO; temp_k = 6000.0f; spot = 2.4f; d65 = false; break;  // DarkSpotlight
        case 12: model = IX_ENV_ASET; break;                                             // Aset
        case 13: model = IX_ENV_STUDIO; d65 = false; uv = true; uv_centre = 365.0f; uv_fwhm = 10.0f; break;
        case 14: model = IX_ENV_STUDIO; d65 = false; uv = true; uv_centre = 395.0f; uv_fwhm = 12.0f; break;
        default: return -1;
    }
    out->model = model;
    out->spectrum = model == IX_ENV_ASET ? IX_SPEC_WAVELENGTH : uv ? IX_SPEC_GAUSSIAN : d65 ? IX_SPEC_D65
                                                                                              : IX_SPEC_BLACKBODY;
    if (uv) {
        out->line_centre_nm = uv_centre;
        out->line_sigma_nm = uv_fwhm / (2.0f * std::sqrt(2.0f * 0.6931472f));  // fwhm / (2 sqrt(2 ln 2))
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
    out->surface_glare = (surface_glare >= 1.0f || std::isnan(surface_glare)) ? 1.0f
                         : (surface_glare > 0.0f ? surface_glare : 0.0f);
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
        out->shadow_cos[0] = std::cos(to_radians(deg + 2.0f));
        out->shadow_cos[1] = std::cos(to_radians(deg - 2.0f));
    }
    float t_k, den;
    blackbody_norm(temp_k, &t_k, &den);
    out->bb_t_k = t_k;
    out->bb_denom_560 = den;
    float cp = std::cos(light_pitch), sp = std::sin(light_pitch);
    float cy = std::cos(light_yaw), sy = std::sin(light_yaw);
    hstore(out->key_dir, hnormalize(h3(cp * sy, sp, cp * cy)));
    const float PI = 3.14159265358979323846f;
    float fill_yaw = std::fma(PI, 0.78f, light_yaw);
    float fp = light_pitch * 0.65f;
    fp = fp < 0.15f ? 0.15f : (fp > 1.2f ? 1.2f : fp);
    hstore(out->fill_dir, hnormalize(h3(std::cos(fp) * std::sin(fill_yaw), std::sin(fp),
                                        std::cos(fp) * std::cos(fill_yaw))));
    float step = PI * 2.0f / 16.0f;
    for (int i = 0; i < IX_RING_LIGHTS; ++i) {
        float a = std::fma((float)i, step, light_yaw);
        hstore(out->ring_dirs[i], hnormalize(h3(std::sin(a) * 0.75f, sp * 0.8f, std::cos(a) * 0.75f)));
    }
    // sun_radiance_factor (sun.rs:25): SUN_RADIANCE x horizon_blend(key_dir).
    {
        const float y = out->key_dir[1];
        float t = (y - -0.05f) / (0.05f - -0.05f);
        t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
        out->sun_factor = 40000.0f * (t * t * std::fma(-2.0f, t, 3.0f));
    }
    // uses_white_balance (mod.rs:553): neither D65 nor a UV lamp nor the ASET view.
    if (!d65 && !uv && model != IX_ENV_ASET) {
        out->white_balance = 1;
        hstore(out->wb_lms, white_balance(temp_k));
    } else {
        out->white_balance = 0;
        out->wb_lms[0] = out->wb_lms[1] = out->wb_lms[2] = 1.0f;
    }
    return 0;
}

int ix_evaluate_gem_optical_metrics_batch(ix_backend* b, const ix_metrics_stone* stones, uint32_t n_stones,
                                          const ix_metrics_lighting* lighting, const ix_metrics_pose* poses,
                                          uint32_t n_poses, uint32_t want_fire_and_scintillation,
                                          ix_gem_metrics* out) {
    if (!b || b->lost || !stones || !lighting || (!poses && n_poses) || (!out && n_poses) || n_stones == 0)
        return IX_DECLINED;
    if (n_poses == 0) return IX_DONE;
    for (uint32_t s = 0; s < n_stones; ++s)
        if (!stones[s].planes || stones[s].n_planes == 0 || stones[s].n_planes > IX_MAX_PLANES ||
            stones[s].dispersion.kind > IX_DISP_CAUCHY)
            return IX_DECLINED;
    for (uint32_t p = 0; p < n_poses; ++p)
        if (poses[p].stone >= n_stones) return IX_DECLINED;
    ix::MetricsLaunch L;
    std::memset(&L, 0, sizeof(L));
    if (!exit_lighting_setup(*lighting, &L.env, &L.spec, &L.factor, &L.head_shadow_cos, L.dirs)) return IX_DECLINED;
    L.want_fire = want_fire_and_scintillation ? 1u : 0u;
    L.n_poses = n_poses;
    std::vector<float> planes;
    std::vector<ix::MetricsStoneDev> dstones(n_stones);
    for (uint32_t s = 0; s < n_stones; ++s) {
        dstones[s].plane_offset = (uint32_t)(planes.size() / 4);
        dstones[s].n_planes = stones[s].n_planes;
        const double w = solid_width(stones[s].planes, stones[s].n_planes);
        dstones[s].half_width = (std::isfinite(w) && w > 0.0) ? (float)(w * 0.5) : 1.0f;
        dstones[s].dispersion = stones[s].dispersion;
        planes.insert(planes.end(), stones[s].planes, stones[s].planes + 4 * (size_t)stones[s].n_planes);
    }
    // camera_view_basis for the pose and its SCINT_TEMPORAL_YAW_OFFSETS_DEG jitters
    // (camera.rs:15, scintillation.rs:13-40).
    static const float kOffsets[5] = {-3.0f, -1.5f, 0.0f, 1.5f, 3.0f};
    std::vector<ix::MetricsPoseDev> dposes(n_poses);
    for (uint32_t p = 0; p < n_poses; ++p) {
        dposes[p].stone = poses[p].stone;
        for (int k = 0; k < 6; ++k) {
            ix_camera cam;
            const float yaw = k == 0 ? poses[p].cam_yaw : poses[p].cam_yaw + to_radians(kOffsets[k - 1]);
            ix_camera_new(yaw, poses[p].cam_pitch, 1.0f, 42.0f, &cam);
            std::memcpy(dposes[p].basis[k] + 0, cam.forward, 12);
            std::memcpy(dposes[p].basis[k] + 3, cam.right, 12);
            std::memcpy(dposes[p].basis[k] + 6, cam.up, 12);
        }
    }
    Turn turn(b);
    if (fail(b, cudaSetDevice(b->device), "set device")) return IX_DECLINED;
    float *d_planes = nullptr, *d_out = nullptr;
    ix::MetricsStoneDev* d_stones = nullptr;
    ix::MetricsPoseDev* d_poses = nullptr;
    bool ok = cudaMalloc((void**)&d_planes, planes.size() * sizeof(float)) == cudaSuccess &&
              cudaMalloc((void**)&d_stones, n_stones * sizeof(ix::MetricsStoneDev)) == cudaSuccess &&
              cudaMalloc((void**)&d_poses, n_poses * sizeof(ix::MetricsPoseDev)) == cudaSuccess &&
              cudaMalloc((void**)&d_out, (size_t)n_poses * 5 * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(d_planes, planes.data(), planes.size() * sizeof(float), cudaMemcpyHostToDevice,
                               b->stream) == cudaSuccess &&
         cudaMemcpyAsync(d_stones, dstones.data(), n_stones * sizeof(ix::MetricsStoneDev), cudaMemcpyHostToDevice,
                         b->stream) == cudaSuccess &&
         cudaMemcpyAsync(d_poses, dposes.data(), n_poses * sizeof(ix::MetricsPoseDev), cudaMemcpyHostToDevice,
                         b->stream) == cudaSuccess;
    if (ok) {
        L.planes = reinterpret_cast<const float4*>(d_planes);
        L.stones = d_stones;
        L.poses = d_poses;
        L.out = d_out;
        cudaError_t e = b->precision == IX_PRECISION_EXACT ? ix::launch_metrics_exact(L, b->stream)
                                                           : ix::launch_metrics_fast(L, b->stream);
        ok = !fail(b, e, "metrics launch");
        std::vector<float> host((size_t)n_poses * 5);
        ok = ok && !fail(b, cudaMemcpyAsync(host.data(), d_out, host.size() * sizeof(float), cudaMemcpyDeviceToHost,
                                            b->stream), "metrics download");
        ok = ok && !fail(b, cudaStreamSynchronize(b->stream), "metrics sync");
        if (ok)
            for (uint32_t p = 0; p < n_poses; ++p)
                out[p] = ix_gem_metrics{host[5 * p], host[5 * p + 1], host[5 * p + 2], host[5 * p + 3],
                                        host[5 * p + 4]};
    } else {
        fail(b, cudaGetLastError(), "metrics buffers");
    }
    cudaFree(d_planes);
    cudaFree(d_stones);
    cudaFree(d_poses);
    cudaFree(d_out);
    return ok ? IX_DONE : IX_DECLINED;
}

int ix_evaluate_gem_optical_metrics(ix_backend* b, const float* planes, uint32_t n_planes,
                                    const ix_material* material, float cam_yaw, float cam_pitch,
                                    const ix_metrics_lighting* lighting, ix_gem_metrics* out) {
    if (!material) return IX_DECLINED;
    ix_metrics_stone stone{planes, n_planes, material->dispersion};
    ix_metrics_pose pose{0, cam_yaw, cam_pitch};
    return ix_evaluate_gem_optical_metrics_batch(b, &stone, 1, lighting, &pose, 1, 1, out);
}

int ix_evaluate_angular_profile_at_azimuth(ix_backend* b, const float* planes, uint32_t n_planes,
                                           const ix_material* material, float cam_yaw,
                                           const ix_metrics_lighting* lighting, float* out) {
    if (!material || !out) return IX_DECLINED;
    // sample_elevation_sweep (profile.rs:72) over PROFILE_ANGLES_DEG (types.rs:27):
    // elevations 0, 5, ..., 90 degrees, fire-less passes.
    ix_metrics_stone stone{planes, n_planes, material->dispersion};
    ix_metrics_pose poses[IX_PROFILE_ANGLES];
    for (int i = 0; i < IX_PROFILE_ANGLES; ++i) poses[i] = ix_metrics_pose{0, cam_yaw, to_radians(5.0f * (float)i)};
    ix_gem_metrics m[IX_PROFILE_ANGLES];
    const int rc = ix_evaluate_gem_optical_metrics_batch(b, &stone, 1, lighting, poses, IX_PROFILE_ANGLES, 0, m);
    if (rc != IX_DONE) return rc;
    for (int i = 0; i < IX_PROFILE_ANGLES; ++i) {
        out[i] = m[i].brilliance_pct;
        out[IX_PROFILE_ANGLES + i] = m[i].extinction_pct;
        out[2 * IX_PROFILE_ANGLES + i] = m[i].windowing_pct;
    }
    return IX_DONE;
}

int ix_evaluate_axis_profiles(ix_backend* b, const float* planes, uint32_t n_planes, const ix_material* material,
                              const float* azimuths_deg, uint32_t n_axes, const ix_metrics_lighting* lighting,
                              float* out) {
    if (!material || !out || (!azimuths_deg && n_axes)) return IX_DECLINED;
    if (n_axes == 0) return IX_DONE;
    // axis_poses (pose_batch.rs:104): table-up first, then pitches 0..89 degrees at the
    // positive azimuth and at the opposite one, all fire-less; tilt_slot (:117) places
    // pose `job` at curve index 90, 180 - (job - 1), or job - 91.
    constexpr int HALF = 90;
    std::vector<ix_metrics_pose> poses;
    poses.reserve((size_t)n_axes * IX_AXIS_TILTS);
    for (uint32_t a = 0; a < n_axes; ++a) {
        const float positive = to_radians(azimuths_deg[a]);
        const float negative = to_radians(azimuths_deg[a] + 180.0f);
        poses.push_back(ix_metrics_pose{0, positive, to_radians(90.0f)});
        for (int i = 0; i < HALF; ++i) poses.push_back(ix_metrics_pose{0, positive, to_radians((float)i)});
        for (int i = 0; i < HALF; ++i) poses.push_back(ix_metrics_pose{0, negative, to_radians((float)i)});
    }
    ix_metrics_stone stone{planes, n_planes, material->dispersion};
    std::vector<ix_gem_metrics> m(poses.size());
    const int rc = ix_evaluate_gem_optical_metrics_batch(b, &stone, 1, lighting, poses.data(),
                                                         (uint32_t)poses.size(), 0, m.data());
    if (rc != IX_DONE) return rc;
    for (uint32_t a = 0; a < n_axes; ++a) {
        float* curves = out + (size_t)a * 3 * IX_AXIS_TILTS;
        for (int job = 0; job < IX_AXIS_TILTS; ++job) {
            const int slot = job == 0 ? HALF : (job <= HALF ? 2 * HALF - (job - 1) : job - 1 - HALF);
            const ix_gem_metrics& g = m[(size_t)a * IX_AXIS_TILTS + job];
            curves[slot] = g.brilliance_pct;
            curves[IX_AXIS_TILTS + slot] = g.extinction_pct;
            curves[2 * IX_AXIS_TILTS + slot] = g.windowing_pct;
        }
    }
    return IX_DONE;
}

void ix_environment_uniform(float radiance, ix_environment* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->model = IX_ENV_UNIFORM;
    out->spectrum = IX_SPEC_FLAT;
    out->exposure = 1.0f;
    out->surface_glare = 1.0f;
    out->wb_lms[0] = out->wb_lms[1] = out->wb_lms[2] = 1.0f;
    out->uniform_radiance = radiance;
}

int ix_debug_check(ix_backend* b, const ix_scene* scene, int32_t fn, uint32_t n,
                   const uint32_t* in, uint32_t in_stride, uint32_t* out, uint32_t out_stride) {
    if (!b || !scene || (n && (!in || !out))) return -1;
    if (scene->n_planes > IX_MAX_PLANES) return -1;
    // 32-bit words each check function reads from / writes to a row (ix::CheckFn order):
    // rows narrower than that are refused before anything reaches the device.
    static const uint8_t kIn[] = {2, 1, 1, 1, 1, 1, 3, 7, 7, 6, 2, 2, 1, 8, 14, 7, 4, 9};
    static const uint8_t kOut[] = {4, 8, 1, 3, 1, 1, 1, 6, 1, 2, 4, 6, 1, 4, 7, 13, 1, 24};
    static_assert(sizeof(kIn) == ix::CHECK_BIAXIAL + 1 && sizeof(kOut) == sizeof(kIn), "check table");
    if (fn < 0 || fn >= (int32_t)sizeof(kIn) || in_stride < kIn[fn] || out_stride < kOut[fn]) return -1;
    Turn turn(b);
    if (fail(b, cudaSetDevice(b->device), "set device")) return -1;
    size_t in_words = (size_t)n * in_stride, out_words = (size_t)n * out_stride;
    if (fail(b, grow_device(&b->d_check, &b->check_cap, in_words + out_words + 1), "check alloc")) return -1;
    if (fail(b, grow_device(&b->d_planes, &b->planes_cap, (size_t)scene->n_planes * 4 + 4), "planes alloc"))
        return -1;
    if (scene->n_planes &&
        fail(b, cudaMemcpyAsync(b->d_planes, scene->planes, (size_t)scene->n_planes * 16,
                                cudaMemcpyHostToDevice, b->stream), "planes upload"))
        return -1;
    if (in_words && fail(b, cudaMemcpyAsync(b->d_check, in, in_words * 4, cudaMemcpyHostToDevice, b->stream),
                         "check upload"))
        return -1;
    ix::CheckLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.scene = *scene;
    L.scene.planes = b->d_planes;
    if (!upload_finishes(b, L.scene, b->stream) || !upload_tools(b, L.scene, b->stream)) return -1;
    L.flags = ix::scene_flags(*scene);
    L.fn = fn;
    L.n = n;
    L.in_stride = in_stride;
    L.out_stride = out_stride;
    L.in = b->d_check;
    L.out = b->d_check + in_words;
    cudaError_t e = b->precision == IX_PRECISION_EXACT ? ix::launch_check_exact(L, b->stream)
                                                        : ix::launch_check_fast(L, b->stream);
    if (fail(b, e, "check launch")) return -1;
    if (out_words && fail(b, cudaMemcpyAsync(out, L.out, out_words * 4, cudaMemcpyDeviceToHost, b->stream),
                          "check download"))
        return -1;
    if (fail(b, cudaStreamSynchronize(b->stream), "check")) return -1;
    return 0;
}

}  // extern "C"

// ---- design batches (include/ix_design.h) --------------------------------------------
extern "C" int ix_evaluate_designs(ix_backend* b, const ix_design* designs, uint32_t n, const ix_design_view* view,
                                   float* out) {
    if (!b || !designs || !view || !view->cameras || !out || n == 0 || view->n_views == 0 || view->spp < 2 ||
        view->width == 0 || view->height == 0 || b->lost)
        return IX_DECLINED;
    // One scene per design and view; two jobs per scene, over the two halves of the
    // sample range, for the split-half metrics.
    const uint64_t n_scenes = (uint64_t)n * view->n_views, n_jobs = 2 * n_scenes;
    const uint32_t spp_a = view->spp / 2, spp_b = view->spp - spp_a;
    if (n_jobs > (1u << 24) || (uint64_t)view->sample_offset + view->spp > 0xFFFFFFFFull) {
        b->last_error = "too many designs x views in one call";
        return IX_DECLINED;
    }
    const uint32_t girdle = view->girdle_segments ? view->girdle_segments : 64;
    const uint32_t count = ix_design_planes(&designs[0], girdle, nullptr, 0);
    if (count == 0) {
        b->last_error = "design out of its domain";
        return IX_DECLINED;
    }
    std::vector<float> planes((size_t)n * count * 4);
    std::vector<ix_scene> scenes(n_scenes);
    std::vector<ix_batch_job> jobs(n_jobs);
    for (uint32_t i = 0; i < n; ++i) {
        ix_material mat;
        float* pl = planes.data() + (size_t)i * count * 4;
        if (ix_design_planes(&designs[i], girdle, pl, count) != count || ix_design_material(&designs[i], &mat) != 0) {
            b->last_error = "design out of its domain";
            return IX_DECLINED;
        }
        for (uint32_t v = 0; v < view->n_views; ++v) {
            const uint64_t j = (uint64_t)i * view->n_views + v;
            ix_scene& sc = scenes[j];
            std::memset(&sc, 0, sizeof(sc));
            sc.camera = view->cameras[v];
            sc.width = view->width;
            sc.height = view->height;
            sc.planes = pl;
            sc.n_planes = count;
            sc.material = mat;
            sc.max_bounces = view->max_bounces;
            sc.environment = view->environment;
            jobs[2 * j] = ix_batch_job{(uint32_t)j, view->sample_offset, spp_a};
            jobs[2 * j + 1] = ix_batch_job{(uint32_t)j, view->sample_offset + spp_a, spp_b};
        }
    }
    for (uint64_t j = 0; j < n_scenes; ++j)
        if (!ix_scene_routes_to_gpu(&scenes[j])) {
            b->last_error = "design scene does not route to the GPU";
            return IX_DECLINED;
        }
    Turn turn(b);
    ix_batch_plan* p =
        plan_create_locked(b, scenes.data(), (uint32_t)n_scenes, jobs.data(), (uint32_t)n_jobs, true);
    if (!p) return IX_DECLINED;
    int rc = IX_DONE;
    float* d_metrics = nullptr;
    if (fail(b, cudaMalloc((void**)&d_metrics, n_scenes * 3 * sizeof(float)), "metrics buffer") ||
        fail(b, cudaEventRecord(b->ev0, b->stream), "event") ||
        fail(b, plan_enqueue(p, b->stream, p->variant), "design batch launch") ||
        fail(b, ix::launch_image_metrics(p->d_scenes, p->d_jobs, (uint32_t)n_scenes, p->d_out, d_metrics, b->stream),
             "image metrics") ||
        fail(b, cudaEventRecord(b->ev1, b->stream), "event") ||
        fail(b, cudaMemcpyAsync(out, d_metrics, n_scenes * 3 * sizeof(float), cudaMemcpyDeviceToHost, b->stream),
             "metrics download") ||
        fail(b, cudaStreamSynchronize(b->stream), "design batch"))
        rc = IX_DECLINED;
    if (rc == IX_DONE) {
        b->timing.paths = p->paths;
        b->timing.launches = (ix::shape_is_pool(ix::variant_shape((int)p->variant)) ? 2u : 1u) + 1u;
    }
    cudaFree(d_metrics);
    ix_batch_plan_destroy(p);
    return rc;
}
