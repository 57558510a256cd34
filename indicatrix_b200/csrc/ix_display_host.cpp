// ix_display_host.cpp -- host side of include/ix_display.h: the display pipeline after the
// path (guide pass, A-Trous denoise, tone-map) on the backend's stream and FIFO turn.
//
// The host part of AtrousDenoiser::denoise_into_with_threads (renderer/denoise/mod.rs:
// 280-345) -- taper, identity short-circuit, pass count, the per-call constants -- is
// resolved here in f32 with -ffp-contract=off, as the reference computes it; the passes
// run on the device, the last one with the sRGB tone-map fused in.  Device buffers are
// pooled in DisplayState and grow on demand; the guides of ix_display_frame are cached
// on the device per camera, planes, image size and signature index.

#include "../../include/ix_display.h"
#include "ix_backend_state.h"
#include "ix_display_launch.h"

#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

using namespace ixh;

// A few host threads that copy between pageable caller memory and the pinned staging
// ring; `run(fn)` calls fn(t) for t = 0..size()-1 (t = 0 on the calling thread) and
// returns when all have finished.
class CopyPool {
public:
    CopyPool() {
        const unsigned hc = std::thread::hardware_concurrency();
        n_ = std::max(1u, std::min(8u, hc ? hc : 1u));
        for (unsigned t = 1; t < n_; ++t) workers_.emplace_back([this, t] { loop(t); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& w : workers_) w.join();
    }
    unsigned size() const { return n_; }
    void run(const std::function<void(unsigned)>& fn) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            fn_ = &fn;
            pending_ = n_ - 1;
            ++generation_;
        }
        cv_.notify_all();
        fn(0);
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return pending_ == 0; });
        fn_ = nullptr;
    }

private:
    void loop(unsigned t) {
        uint64_t seen = 0;
        for (;;) {
            const std::function<void(unsigned)>* fn;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || generation_ != seen; });
                if (stop_) return;
                seen = generation_;
                fn = fn_;
            }
            (*fn)(t);
            std::lock_guard<std::mutex> lk(mu_);
            if (--pending_ == 0) done_cv_.notify_all();
        }
    }
    unsigned n_ = 1;
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(unsigned)>* fn_ = nullptr;
    unsigned pending_ = 0;
    uint64_t generation_ = 0;
    bool stop_ = false;
};

constexpr size_t STAGE_CHUNK = 4u << 20;  // bytes per pinned slot

struct DisplayState {
    // Pinned two-slot ring for host <-> device copies of caller buffers, and the threads
    // that fill and drain it.
    uint8_t* h_stage = nullptr;
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    CopyPool pool;
    float* d_planes = nullptr;
    size_t planes_cap = 0;
    // Guides in the reference layout (uploaded or computed).
    float* d_depth = nullptr;
    size_t depth_cap = 0;
    float* d_normal = nullptr;
    size_t normal_cap = 0;
    int32_t* d_facet = nullptr;
    size_t facet_cap = 0;
    uint32_t* d_sig = nullptr;
    size_t sig_cap = 0;
    // Packed guides and the colour ping-pong of the passes.
    float4* d_nrm = nullptr;
    size_t nrm_cap = 0;
    int2* d_fs = nullptr;
    size_t fs_cap = 0;
    float4* d_col[2] = {nullptr, nullptr};
    size_t col_cap[2] = {0, 0};
    // Host-layout colour in / out (3 floats per pixel) and RGBA8 out.
    float* d_xyz = nullptr;
    size_t xyz_cap = 0;
    uchar4* d_rgba = nullptr;
    size_t rgba_cap = 0;
    // Guide cache of ix_display_frame.
    bool cached = false;
    std::vector<uint8_t> cache_key;
    // Stage timing of the last call.
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    ix_display_timing timing{0.0f, 0.0f, 0.0f, 0, 0};
    bool pending = false;  // an asynchronous call's events are still to be read
};

void display_state_free(DisplayState* d) {
    if (!d) return;
    if (d->h_stage) cudaFreeHost(d->h_stage);
    for (cudaEvent_t e : d->stage_ev)
        if (e) cudaEventDestroy(e);
    cudaFree(d->d_planes);
    cudaFree(d->d_depth);
    cudaFree(d->d_normal);
    cudaFree(d->d_facet);
    cudaFree(d->d_sig);
    cudaFree(d->d_nrm);
    cudaFree(d->d_fs);
    cudaFree(d->d_col[0]);
    cudaFree(d->d_col[1]);
    cudaFree(d->d_xyz);
    cudaFree(d->d_rgba);
    for (cudaEvent_t e : d->ev)
        if (e) cudaEventDestroy(e);
    delete d;
}

namespace {

using namespace ix::disp;

constexpr float SIGMA_EPS = 1.0e-8f;

DisplayState* state(ix_backend* b) {
    if (!b->display) {
        b->display = new DisplayState();
        for (cudaEvent_t& e : b->display->ev)
            if (cudaEventCreate(&e) != cudaSuccess) e = nullptr;
        for (cudaEvent_t& e : b->display->stage_ev)
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) e = nullptr;
        if (cudaMallocHost((void**)&b->display->h_stage, 2 * STAGE_CHUNK) != cudaSuccess)
            b->display->h_stage = nullptr;
    }
    return b->display;
}

bool exact(const ix_backend* b) { return b->precision == IX_PRECISION_EXACT; }

cudaError_t pass_launch(const ix_backend* b, const PassLaunch& L, cudaStream_t st) {
    return exact(b) ? launch_atrous_pass_exact(L, st) : launch_atrous_pass_fast(L, st);
}
cudaError_t tonemap_launch(const ix_backend* b, const TonemapLaunch& L, cudaStream_t st) {
    return exact(b) ? launch_tonemap_exact(L, st) : launch_tonemap_fast(L, st);
}
cudaError_t unpack_launch(const ix_backend* b, const UnpackLaunch& L, cudaStream_t st) {
    return exact(b) ? launch_unpack_exact(L, st) : launch_unpack_fast(L, st);
}

// The per-call constants of denoise_into_with_threads (denoise/mod.rs:318-345).
struct Resolved {
    bool identity;       // taper below the cut-off: exact copy of the colour
    uint32_t passes;
    PassLaunch pass;     // constants only
};
Resolved resolve(const ix_atrous_params& p, uint32_t spp) {
    Resolved r{};
    const float n0 = std::fmax(p.taper_reference_spp, SIGMA_EPS);
    const float taper = 1.0f / std::sqrt(1.0f + (float)spp / n0);
    r.passes = std::min(std::max(p.num_passes, 1u), 8u);
    r.identity = taper < p.taper_identity_epsilon;
    const float sce = std::fmax(p.sigma_color * taper, 0.0f);
    const float sd = std::fmax(p.sigma_depth, SIGMA_EPS);
    const float scs = std::fmax(sce * sce, SIGMA_EPS);
    r.pass.neg_inv_sigma_depth = -1.0f / sd;
    r.pass.neg_inv_two_sigma_color_sq = -1.0f / (2.0f * scs);
    // normal_weight_unit's cos_pow(cos, power.max(0)) (pass.rs:118): a power-of-two whole
    // exponent is squared that many times, anything else goes through pow.
    const float power = std::fmax(p.normal_power, 0.0f);
    r.pass.normal_power = power;
    r.pass.squarings = -1;
    if (power >= 0.0f && power == std::floor(power) && power <= 4294967295.0f) {
        const double ip = (double)power;
        const uint64_t u = (uint64_t)ip;
        if (u != 0 && (u & (u - 1)) == 0) {
            int s = 0;
            while ((1ull << s) < u) ++s;
            r.pass.squarings = s;
        }
    }
    return r;
}

bool alloc_frame(ix_backend* b, DisplayState* d, uint64_t n, bool guides_raw, bool xyz, bool rgba) {
    cudaError_t e = grow_device(&d->d_nrm, &d->nrm_cap, n);
    if (e == cudaSuccess) e = grow_device(&d->d_fs, &d->fs_cap, n);
    if (e == cudaSuccess) e = grow_device(&d->d_col[0], &d->col_cap[0], n);
    if (e == cudaSuccess) e = grow_device(&d->d_col[1], &d->col_cap[1], n);
    if (e == cudaSuccess && guides_raw) {
        e = grow_device(&d->d_depth, &d->depth_cap, n);
        if (e == cudaSuccess) e = grow_device(&d->d_normal, &d->normal_cap, 3 * n);
        if (e == cudaSuccess) e = grow_device(&d->d_facet, &d->facet_cap, n);
        if (e == cudaSuccess) e = grow_device(&d->d_sig, &d->sig_cap, n);
    }
    if (e == cudaSuccess && xyz) e = grow_device(&d->d_xyz, &d->xyz_cap, 3 * n);
    if (e == cudaSuccess && rgba) e = grow_device(&d->d_rgba, &d->rgba_cap, n);
    return !fail(b, e, "display buffers");
}

cudaError_t h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
}
cudaError_t d2h(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s) : cudaSuccess;
}

// Caller memory is pageable: it goes through the pinned ring in 4 MB chunks, the host
// threads copying chunk k + 1 while the DMA engine moves chunk k.  Without a ring (pinned
// allocation failed) the plain pageable copy is used.
void parallel_copy(DisplayState* d, void* dst, const void* src, size_t bytes) {
    const unsigned nt = d->pool.size();
    const size_t part = (bytes + nt - 1) / nt;
    d->pool.run([&](unsigned t) {
        const size_t off = (size_t)t * part;
        if (off < bytes) std::memcpy((uint8_t*)dst + off, (const uint8_t*)src + off, std::min(part, bytes - off));
    });
}
cudaError_t h2d_staged(DisplayState* d, void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (!d->h_stage || !d->stage_ev[0] || !d->stage_ev[1] || bytes < (256u << 10)) return h2d(dst, src, bytes, st);
    for (size_t off = 0, k = 0; off < bytes; off += STAGE_CHUNK, ++k) {
        const int slot = (int)(k & 1);
        const size_t len = std::min(STAGE_CHUNK, bytes - off);
        cudaError_t e = cudaEventSynchronize(d->stage_ev[slot]);  // the slot's previous DMA
        if (e != cudaSuccess) return e;
        uint8_t* h = d->h_stage + slot * STAGE_CHUNK;
        parallel_copy(d, h, (const uint8_t*)src + off, len);
        e = cudaMemcpyAsync((uint8_t*)dst + off, h, len, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaEventRecord(d->stage_ev[slot], st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
// Device -> caller memory; returns when `dst` holds the data (it waits for the stream).
cudaError_t d2h_staged(DisplayState* d, void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (!d->h_stage || !d->stage_ev[0] || !d->stage_ev[1] || bytes < (256u << 10)) {
        cudaError_t e = d2h(dst, src, bytes, st);
        return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
    }
    const size_t chunks = (bytes + STAGE_CHUNK - 1) / STAGE_CHUNK;
    auto issue = [&](size_t k) {
        const int slot = (int)(k & 1);
        const size_t off = k * STAGE_CHUNK, len = std::min(STAGE_CHUNK, bytes - off);
        cudaError_t e = cudaEventSynchronize(d->stage_ev[slot]);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d->h_stage + slot * STAGE_CHUNK, (const uint8_t*)src + off, len,
                                cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaEventRecord(d->stage_ev[slot], st);
        return e;
    };
    cudaError_t e = issue(0);
    for (size_t k = 0; k < chunks && e == cudaSuccess; ++k) {
        const int slot = (int)(k & 1);
        const size_t off = k * STAGE_CHUNK, len = std::min(STAGE_CHUNK, bytes - off);
        e = cudaEventSynchronize(d->stage_ev[slot]);
        if (e != cudaSuccess) break;
        // Chunk k has landed; start chunk k + 1 into the other slot before copying out.
        if (k + 1 < chunks) e = issue(k + 1);
        parallel_copy(d, (uint8_t*)dst + off, d->h_stage + slot * STAGE_CHUNK, len);
    }
    return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
}

void record(DisplayState* d, int i, cudaStream_t st) {
    if (d->ev[i]) cudaEventRecord(d->ev[i], st);
}
float elapsed(DisplayState* d, int a, int c) {
    float ms = 0.0f;
    if (d->ev[a] && d->ev[c] && cudaEventElapsedTime(&ms, d->ev[a], d->ev[c]) == cudaSuccess) return ms;
    return 0.0f;
}

// The passes over the packed guides in d_nrm / d_fs and the colour in d_col[0]; the last
// pass writes RGBA8 into `rgba` when it is given, else colour.  Returns the index of the
// colour buffer holding the result (rgba == null) and counts the launches.
int run_passes(ix_backend* b, DisplayState* d, const Resolved& r, uint32_t w, uint32_t h, uchar4* rgba,
               bool facet_normals, uint32_t* launches, cudaError_t* err, cudaStream_t st) {
    int cur = 0;
    *err = cudaSuccess;
    for (uint32_t pass = 0; pass < r.passes && *err == cudaSuccess; ++pass) {
        PassLaunch L = r.pass;
        L.width = w;
        L.height = h;
        L.stride = 1 << pass;
        L.src = d->d_col[cur];
        L.nrm = d->d_nrm;
        L.fs = d->d_fs;
        L.facet_normals = facet_normals ? 1 : 0;
        const bool last = pass + 1 == r.passes;
        L.dst = (last && rgba) ? nullptr : d->d_col[cur ^ 1];
        L.rgba = (last && rgba) ? rgba : nullptr;
        *err = pass_launch(b, L, st);
        ++*launches;
        cur ^= 1;
    }
    return cur;
}

// The frame after packing: identity -> tone-map the average; else the passes with the
// tone-map fused into the last.  d_col[0] holds the average.
cudaError_t frame_after_pack(ix_backend* b, DisplayState* d, const Resolved& r, uint32_t w, uint32_t h,
                             bool facet_normals, uint32_t* launches, cudaStream_t st) {
    const uint64_t n = (uint64_t)w * h;
    if (r.identity) {
        TonemapLaunch T{n, nullptr, d->d_col[0], 1.0f, IX_COLOR_SPACE_SRGB, d->d_rgba};
        ++*launches;
        return tonemap_launch(b, T, st);
    }
    cudaError_t e;
    run_passes(b, d, r, w, h, d->d_rgba, facet_normals, launches, &e, st);
    return e;
}

bool guide_key(const ix_scene& sc, uint32_t with_sig, float n_d, std::vector<uint8_t>* key) {
    key->clear();
    auto put = [&](const void* p, size_t n) {
        const uint8_t* c = (const uint8_t*)p;
        key->insert(key->end(), c, c + n);
    };
    put(&sc.camera, sizeof(sc.camera));
    put(&sc.width, sizeof(sc.width));
    put(&sc.height, sizeof(sc.height));
    put(&sc.n_planes, sizeof(sc.n_planes));
    put(sc.planes, 4 * sizeof(float) * sc.n_planes);
    put(&with_sig, sizeof(with_sig));
    put(&n_d, sizeof(n_d));
    return true;
}

// DispersionModel::n_d (optics/dispersion.rs:264): evaluate_unclamped (:179-209) at
// 589.3 nm, in f32 as the reference rounds it (no clamp: 589.3 nm is in the visible).
float n_d_of(const ix_dispersion& m) {
    const float um = 589.3f * 1e-3f;
    const float l2 = um * um;
    if (m.kind == IX_DISP_SELLMEIER1) return std::sqrt(std::fmax(1.0f + (m.b[0] * l2) / (l2 - m.c[0]), 1.0f));
    if (m.kind == IX_DISP_SELLMEIER3) {
        float n2 = 1.0f;
        n2 += (m.b[0] * l2) / (l2 - m.c[0]);
        n2 += (m.b[1] * l2) / (l2 - m.c[1]);
        n2 += (m.b[2] * l2) / (l2 - m.c[2]);
        return std::sqrt(std::fmax(n2, 1.0f));
    }
    const float l4 = l2 * l2;
    return std::fmax((m.b[0] + m.b[1] / l2) + m.b[2] / l4, 1.0f);
}

}  // namespace

extern "C" {

void ix_atrous_params_default(ix_atrous_params* out) {
    // AtrousParams::default (denoise/mod.rs:194).
    if (out) *out = ix_atrous_params{5u, 0.35f, 0.1f, 64.0f, 4.0f, 0.02f};
}

int ix_display_last_timing(const ix_backend* b, ix_display_timing* out) {
    if (!b || !out || !b->display) return IX_DECLINED;
    DisplayState* d = b->display;
    if (d->pending) {
        // The device form returned before its kernels ran: wait for its last event.
        if (!d->ev[3] || cudaEventSynchronize(d->ev[3]) != cudaSuccess) return IX_DECLINED;
        d->timing.guide_ms = elapsed(d, 0, 1);
        d->timing.pack_ms = 0.0f;
        d->timing.atrous_ms = elapsed(d, 2, 3);
        d->pending = false;
    }
    *out = d->timing;
    return IX_DONE;
}

int ix_generate_guide_buffers(ix_backend* b, uint32_t width, uint32_t height, const ix_camera* camera,
                              const float* planes, uint32_t n_planes, float n_d, float* depth, float* normal,
                              int32_t* facet_id, uint32_t* path_sig) {
    if (!b || b->lost || !camera || (!planes && n_planes) || n_planes > IX_MAX_PLANES) return IX_DECLINED;
    const uint64_t n = (uint64_t)width * height;
    if (n && (!depth || !normal || !facet_id)) return IX_DECLINED;
    if (n == 0) return IX_DONE;
    Turn turn(b);
    if (fail(b, cudaSetDevice(b->device), "set device")) return IX_DECLINED;
    DisplayState* d = state(b);
    cudaError_t e = grow_device(&d->d_planes, &d->planes_cap, 4 * (size_t)std::max(n_planes, 1u));
    if (e == cudaSuccess) e = grow_device(&d->d_depth, &d->depth_cap, n);
    if (e == cudaSuccess) e = grow_device(&d->d_normal, &d->normal_cap, 3 * n);
    if (e == cudaSuccess) e = grow_device(&d->d_facet, &d->facet_cap, n);
    if (e == cudaSuccess) e = grow_device(&d->d_sig, &d->sig_cap, n);
    if (fail(b, e, "guide buffers")) return IX_DECLINED;
    d->cached = false;  // the raw guide buffers are shared with the frame cache
    const auto t0 = std::chrono::steady_clock::now();
    e = h2d(d->d_planes, planes, 16 * (size_t)n_planes, b->stream);
    record(d, 0, b->stream);
    GuideLaunch G{*camera, width, height, reinterpret_cast<const float4*>(d->d_planes), n_planes, n_d,
                  d->d_depth, d->d_normal, d->d_facet, path_sig ? d->d_sig : nullptr, nullptr, nullptr};
    if (e == cudaSuccess) e = launch_guides_exact(G, b->stream);
    record(d, 1, b->stream);
    if (e == cudaSuccess) e = d2h_staged(d, depth, d->d_depth, 4 * n, b->stream);
    if (e == cudaSuccess) e = d2h_staged(d, normal, d->d_normal, 12 * n, b->stream);
    if (e == cudaSuccess) e = d2h_staged(d, facet_id, d->d_facet, 4 * n, b->stream);
    if (e == cudaSuccess && path_sig) e = d2h_staged(d, path_sig, d->d_sig, 4 * n, b->stream);
    if (fail(b, e, "guide pass")) return IX_DECLINED;
    d->pending = false;
    d->timing = ix_display_timing{elapsed(d, 0, 1), 0.0f, 0.0f, 0, 1};
    b->timing = ix_timing{elapsed(d, 0, 1),
                          std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count(),
                          n, 1};
    return IX_DONE;
}

int ix_atrous_denoise(ix_backend* b, const float* color, const float* depth, const float* normal,
                      const int32_t* facet_id, const uint32_t* path_sig, uint32_t width, uint32_t height,
                      uint32_t spp, const ix_atrous_params* params, float* out) {
    if (!b || b->lost || !params) return IX_DECLINED;
    const uint64_t n = (uint64_t)width * height;
    if (n == 0) return IX_DONE;
    if (!color || !depth || !normal || !facet_id || !out || color == out) return IX_DECLINED;
    const Resolved r = resolve(*params, spp);
    if (r.identity) {
        std::memcpy(out, color, 12 * n);
        return IX_DONE;
    }
    Turn turn(b);
    if (fail(b, cudaSetDevice(b->device), "set device")) return IX_DECLINED;
    DisplayState* d = state(b);
    if (!alloc_frame(b, d, n, true, true, false)) return IX_DECLINED;
    d->cached = false;
    const auto t0 = std::chrono::steady_clock::now();
    cudaError_t e = h2d_staged(d, d->d_xyz, color, 12 * n, b->stream);
    if (e == cudaSuccess) e = h2d_staged(d, d->d_depth, depth, 4 * n, b->stream);
    if (e == cudaSuccess) e = h2d_staged(d, d->d_normal, normal, 12 * n, b->stream);
    if (e == cudaSuccess) e = h2d_staged(d, d->d_facet, facet_id, 4 * n, b->stream);
    if (e == cudaSuccess && path_sig) e = h2d_staged(d, d->d_sig, path_sig, 4 * n, b->stream);
    record(d, 0, b->stream);
    PackLaunch P{n, d->d_depth, d->d_normal, d->d_facet, path_sig ? d->d_sig : nullptr, d->d_nrm, d->d_fs,
                 d->d_xyz, 1.0f, d->d_col[0]};
    if (e == cudaSuccess) e = launch_pack_exact(P, b->stream);
    record(d, 1, b->stream);
    uint32_t launches = 1;
    int cur = 0;
    if (e == cudaSuccess) cur = run_passes(b, d, r, width, height, nullptr, false, &launches, &e, b->stream);
    record(d, 2, b->stream);
    UnpackLaunch U{n, d->d_col[cur], d->d_xyz};
    if (e == cudaSuccess) e = unpack_launch(b, U, b->stream);
    ++launches;
    record(d, 3, b->stream);
    if (e == cudaSuccess) e = d2h_staged(d, out, d->d_xyz, 12 * n, b->stream);
    if (fail(b, e, "denoise")) return IX_DECLINED;
    d->pending = false;
    d->timing = ix_display_timing{0.0f, elapsed(d, 0, 1), elapsed(d, 1, 2), r.passes, launches};
    b->timing = ix_timing{elapsed(d, 0, 3),
                          std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count(),
                          n, launches};
    return IX_DONE;
}

static int tonemap_impl(ix_backend* b, const float* xyz, uint64_t pixels, float scale, uint32_t space,
                        uint8_t* rgba) {
    if (!b || b->lost || space > IX_COLOR_SPACE_ACESCG) return IX_DECLINED;
    if (pixels == 0) return IX_DONE;
    if (!xyz || !rgba) return IX_DECLINED;
    Turn turn(b);
    if (fail(b, cudaSetDevice(b->device), "set device")) return IX_DECLINED;
    DisplayState* d = state(b);
    cudaError_t e = grow_device(&d->d_xyz, &d->xyz_cap, 3 * pixels);
    if (e == cudaSuccess) e = grow_device(&d->d_rgba, &d->rgba_cap, pixels);
    if (fail(b, e, "tonemap buffers")) return IX_DECLINED;
    const auto t0 = std::chrono::steady_clock::now();
    e = h2d_staged(d, d->d_xyz, xyz, 12 * pixels, b->stream);
    record(d, 0, b->stream);
    TonemapLaunch T{pixels, d->d_xyz, nullptr, scale, space, d->d_rgba};
    if (e == cudaSuccess) e = tonemap_launch(b, T, b->stream);
    record(d, 1, b->stream);
    if (e == cudaSuccess) e = d2h_staged(d, rgba, d->d_rgba, 4 * pixels, b->stream);
    if (fail(b, e, "tonemap")) return IX_DECLINED;
    d->pending = false;
    d->timing = ix_display_timing{0.0f, 0.0f, 0.0f, 0, 1};
    b->timing = ix_timing{elapsed(d, 0, 1),
                          std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count(),
                          pixels, 1};
    return IX_DONE;
}

int ix_tonemap_to_rgba(ix_backend* b, const float* xyz, uint64_t pixels, float scale, uint8_t* rgba) {
    return tonemap_impl(b, xyz, pixels, scale, IX_COLOR_SPACE_SRGB, rgba);
}

int ix_tonemap_accumulation(ix_backend* b, uint32_t width, uint32_t height, uint32_t samples_per_pixel,
                            const float* accum, uint32_t color_space, uint8_t* rgba) {
    // tonemap_accumulation (tonemap.rs:213): encode(accum * (1 / spp)).
    const float inv = 1.0f / (float)samples_per_pixel;
    return tonemap_impl(b, accum, (uint64_t)width * height, inv, color_space, rgba);
}

int ix_denoise_and_tonemap_frame(ix_backend* b, uint32_t width, uint32_t height, uint32_t spp, const float* accum,
                                 const float* depth, const float* normal, const int32_t* facet_id,
                                 const uint32_t* path_sig, const ix_atrous_params* params, uint8_t* rgba) {
    if (!b || b->lost || !params) return IX_DECLINED;
    const uint64_t n = (uint64_t)width * height;
    if (n == 0) return IX_DONE;
    if (!accum || !depth || !normal || !facet_id || !rgba) return IX_DECLINED;
    if (spp == 0) {
        // frame_denoise.rs:48: the tone-map of an all-zero frame.
        for (uint64_t i = 0; i < n; ++i) {
            rgba[4 * i] = rgba[4 * i + 1] = rgba[4 * i + 2] = 0;
            rgba[4 * i + 3] = 255;
        }
        return IX_DONE;
    }
    const Resolved r = resolve(*params, spp);
    Turn turn(b);
    if (fail(b, cudaSetDevice(b->device), "set device")) return IX_DECLINED;
    DisplayState* d = state(b);
    if (!alloc_frame(b, d, n, true, true, true)) return IX_DECLINED;
    d->cached = false;
    const auto t0 = std::chrono::steady_clock::now();
    cudaError_t e = h2d_staged(d, d->d_xyz, accum, 12 * n, b->stream);
    if (e == cudaSuccess) e = h2d_staged(d, d->d_depth, depth, 4 * n, b->stream);
    if (e == cudaSuccess) e = h2d_staged(d, d->d_normal, normal, 12 * n, b->stream);
    if (e == cudaSuccess) e = h2d_staged(d, d->d_facet, facet_id, 4 * n, b->stream);
    if (e == cudaSuccess && path_sig) e = h2d_staged(d, d->d_sig, path_sig, 4 * n, b->stream);
    record(d, 0, b->stream);
    const float inv = 1.0f / (float)spp;
    PackLaunch P{n, d->d_depth, d->d_normal, d->d_facet, path_sig ? d->d_sig : nullptr, d->d_nrm, d->d_fs,
                 d->d_xyz, inv, d->d_col[0]};
    if (e == cudaSuccess) e = launch_pack_exact(P, b->stream);
    record(d, 1, b->stream);
    uint32_t launches = 1;
    if (e == cudaSuccess) e = frame_after_pack(b, d, r, width, height, false, &launches, b->stream);
    record(d, 2, b->stream);
    if (e == cudaSuccess) e = d2h_staged(d, rgba, d->d_rgba, 4 * n, b->stream);
    if (fail(b, e, "denoise and tonemap")) return IX_DECLINED;
    d->pending = false;
    d->timing = ix_display_timing{0.0f, elapsed(d, 0, 1), elapsed(d, 1, 2), r.identity ? 0u : r.passes, launches};
    b->timing = ix_timing{elapsed(d, 0, 2),
                          std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count(),
                          n, launches};
    return IX_DONE;
}

// The shared body of ix_display_frame and ix_display_frame_device: `accum_dev` and
// `rgba_dev` are device pointers (the host entry stages through the pooled buffers).
static int display_frame_impl(ix_backend* b, const ix_scene* scene, uint32_t with_signature, uint32_t spp,
                              const float* accum_host, const float* accum_dev, const ix_atrous_params* params,
                              uint8_t* rgba_host, uint8_t* rgba_dev, cudaStream_t stream) {
    if (!b || b->lost || !scene || !params) return IX_DECLINED;
    const ix_scene& sc = *scene;
    if ((!sc.planes && sc.n_planes) || sc.n_planes > IX_MAX_PLANES) return IX_DECLINED;
    const uint64_t n = (uint64_t)sc.width * sc.height;
    if (n == 0) return IX_DONE;
    if ((!accum_host && !accum_dev) || (!rgba_host && !rgba_dev)) return IX_DECLINED;
    if (spp == 0 && rgba_host) {
        for (uint64_t i = 0; i < n; ++i) {
            rgba_host[4 * i] = rgba_host[4 * i + 1] = rgba_host[4 * i + 2] = 0;
            rgba_host[4 * i + 3] = 255;
        }
        return IX_DONE;
    }
    const Resolved r = resolve(*params, spp);
    const float n_d = with_signature ? n_d_of(sc.material.dispersion) : 0.0f;
    Turn turn(b);
    if (fail(b, cudaSetDevice(b->device), "set device")) return IX_DECLINED;
    const cudaStream_t st = stream ? stream : b->stream;
    DisplayState* d = state(b);
    if (!alloc_frame(b, d, n, false, accum_dev == nullptr, rgba_dev == nullptr)) return IX_DECLINED;
    if (fail(b, grow_device(&d->d_planes, &d->planes_cap, 4 * (size_t)std::max(sc.n_planes, 1u)), "planes"))
        return IX_DECLINED;
    const auto t0 = std::chrono::steady_clock::now();
    cudaError_t e = cudaSuccess;
    uint32_t launches = 0;
    std::vector<uint8_t> key;
    guide_key(sc, with_signature, n_d, &key);
    record(d, 0, st);
    if (!d->cached || key != d->cache_key) {
        // The guides depend only on the camera pose and the facet geometry (guide_pass.rs
        // module docs): computed once per pose, reused for every frame of it.
        e = h2d(d->d_planes, sc.planes, 16 * (size_t)sc.n_planes, st);
        GuideLaunch G{sc.camera, sc.width, sc.height, reinterpret_cast<const float4*>(d->d_planes), sc.n_planes, n_d,
                      nullptr, nullptr, nullptr, nullptr, d->d_nrm, d->d_fs};
        if (e == cudaSuccess) e = launch_guides_exact(G, st);
        ++launches;
        d->cached = e == cudaSuccess;
        d->cache_key = key;
    }
    record(d, 1, st);
    const float* src = accum_dev;
    if (!src) {
        if (e == cudaSuccess) e = h2d_staged(d, d->d_xyz, accum_host, 12 * n, st);
        src = d->d_xyz;
    }
    record(d, 2, st);
    if (spp == 0) {
        // rgba_dev only: the tone-map of zeros.
        if (e == cudaSuccess) e = cudaMemsetAsync(d->d_col[0], 0, 16 * n, st);
        TonemapLaunch T{n, nullptr, d->d_col[0], 1.0f, IX_COLOR_SPACE_SRGB, reinterpret_cast<uchar4*>(rgba_dev)};
        if (e == cudaSuccess) e = tonemap_launch(b, T, st);
        ++launches;
    } else {
        const float inv = 1.0f / (float)spp;
        PackLaunch P{n, nullptr, nullptr, nullptr, nullptr, d->d_nrm, nullptr, src, inv, d->d_col[0]};
        if (e == cudaSuccess) e = launch_pack_exact(P, st);
        ++launches;
        uchar4* out = rgba_dev ? reinterpret_cast<uchar4*>(rgba_dev) : d->d_rgba;
        uchar4* keep = d->d_rgba;
        d->d_rgba = out;
        if (e == cudaSuccess) e = frame_after_pack(b, d, r, sc.width, sc.height, true, &launches, st);
        d->d_rgba = keep;
    }
    record(d, 3, st);
    // The host form waits for its RGBA8; the device form stays asynchronous on `st`.
    if (rgba_host && e == cudaSuccess) e = d2h_staged(d, rgba_host, d->d_rgba, 4 * n, st);
    if (fail(b, e, "display frame")) {
        d->cached = false;
        return IX_DECLINED;
    }
    if (!rgba_host) {
        // Stage times are read from the events when ix_display_last_timing asks.
        d->pending = true;
        d->timing = ix_display_timing{0.0f, 0.0f, 0.0f, r.identity || spp == 0 ? 0u : r.passes, launches};
        b->timing.launches = launches;
        b->timing.paths = n;
        return IX_DONE;
    }
    d->pending = false;
    d->timing = ix_display_timing{elapsed(d, 0, 1), 0.0f, elapsed(d, 2, 3), r.identity ? 0u : r.passes, launches};
    b->timing = ix_timing{elapsed(d, 0, 3),
                          std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count(),
                          n, launches};
    return IX_DONE;
}

int ix_display_frame(ix_backend* b, const ix_scene* scene, uint32_t with_signature, uint32_t spp,
                     const float* accum, const ix_atrous_params* params, uint8_t* rgba) {
    return display_frame_impl(b, scene, with_signature, spp, accum, nullptr, params, rgba, nullptr, nullptr);
}

int ix_display_frame_device(ix_backend* b, const ix_scene* scene, uint32_t with_signature, uint32_t spp,
                            const float* accum_dev, const ix_atrous_params* params, uint8_t* rgba_dev,
                            void* stream) {
    if (!accum_dev || !rgba_dev) return IX_DECLINED;
    return display_frame_impl(b, scene, with_signature, spp, nullptr, accum_dev, params, nullptr, rgba_dev,
                              (cudaStream_t)stream);
}

}  // extern "C"
