// ix_backend_state.h -- the backend object behind the C ABI and the host helpers every
// entry-point file shares: the FIFO turn (gpu_backend/turnstile.rs:24-115), the
// device-error-to-lost-backend rule (gpu_backend/mod.rs:151-164) and pooled buffers.
#pragma once

#include "../../include/ix_cuda.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <mutex>
#include <string>

struct DisplayState;  // the display pipeline's pooled buffers (ix_display_host.cpp)
void display_state_free(DisplayState* d);
struct RadianceState;  // the radiance codec's device and pinned buffers (ix_radiance.cpp)
void radiance_state_free(RadianceState* r);

struct ix_backend {
    int device = 0;
    uint32_t pipeline = IX_PIPELINE_MEGAKERNEL;
    uint32_t precision = IX_PRECISION_FAST;
    uint32_t threads = 128;
    uint64_t chunk_paths = 0;
    ix_work_limits limits{0, 0, 0};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // Pooled buffers.
    float* d_planes = nullptr;
    size_t planes_cap = 0;
    double* d_sums = nullptr;
    size_t sums_cap = 0;
    double* h_sums = nullptr;
    size_t hsums_cap = 0;
    uint32_t* d_counter = nullptr;
    unsigned long long* d_dropped = nullptr;
    uint32_t* d_check = nullptr;
    size_t check_cap = 0;
    // Spectral attribution: per-sample class / luminance records of one launch and the
    // frame's attribution map.
    uint8_t* d_attr_cls = nullptr;
    size_t attr_cls_cap = 0;
    float* d_attr_y = nullptr;
    size_t attr_y_cap = 0;
    ix_attribution_pixel* d_attr_map = nullptr;
    size_t attr_map_cap = 0;
    ix_attribution_pixel* h_attr_map = nullptr;
    size_t hattr_map_cap = 0;
    // The one-shot batch entry's device sums.
    double* d_batch_out = nullptr;
    size_t batch_out_cap = 0;
    // A host scene's per-facet finishes, copied for the kernels.
    uint8_t* d_finishes = nullptr;
    size_t finishes_cap = 0;
    ix_tool* d_tools = nullptr;  // the call's concave tools
    size_t tools_cap = 0;
    // Fixed-point per-pixel sums of the path-pool kernels (FIXED_WORDS per pixel of a launch).
    unsigned long long* d_acc = nullptr;
    size_t acc_cap = 0;
    int sm_count = 0;
    // Kernel variant (budget + 3 * shape, ix_launch.h) of single-scene calls.
    uint32_t variant = 0;
    bool variant_pinned = false;  // ix_backend_options.kernel_variant chose it
    // Variant new batch plans start from: the last autotuner pick (or `variant`).
    uint32_t batch_variant = 0;
    // CTA size new batch plans are restricted to (0: any; 64, 128 or 256).
    uint32_t batch_threads = 0;
    // Resident CTAs per SM by [transport instantiation (ix::TransportClass)][variant]
    // (0: not in this build).
    static constexpr int kVariants = 12, kClasses = 3;
    int bps_exact[kClasses][kVariants] = {}, bps_fast[kClasses][kVariants] = {};
    // ... and of the attributed trace kernels by [transport instantiation].
    int bps_attr_exact[kClasses] = {1, 1, 1}, bps_attr_fast[kClasses] = {1, 1, 1};
    std::string label;
    // State.
    bool lost = false;
    std::string last_error;
    ix_timing timing{0.0f, 0.0f, 0, 0};
    uint64_t dropped = 0;
    // FIFO turnstile.
    std::mutex mu;
    std::condition_variable cv;
    uint64_t next_ticket = 0, serving = 0;
    // Guide buffers, colour ping-pong and output of the display pipeline.
    DisplayState* display = nullptr;
    // Payload bytes of the radiance codec's device forms.
    RadianceState* radiance = nullptr;
};

namespace ixh {


struct Turn {
    ix_backend* b;
    explicit Turn(ix_backend* be) : b(be) {
        std::unique_lock<std::mutex> lk(b->mu);
        uint64_t mine = b->next_ticket++;
        b->cv.wait(lk, [&] { return b->serving == mine; });
    }
    ~Turn() {
        std::lock_guard<std::mutex> lk(b->mu);
        b->serving++;
        b->cv.notify_all();
    }
};

inline bool fail(ix_backend* b, cudaError_t e, const char* where) {
    if (e == cudaSuccess) return false;
    b->lost = true;
    b->last_error = std::string(where) + ": " + cudaGetErrorString(e);
    (void)cudaGetLastError();
    return true;
}

template <typename T>
inline cudaError_t grow_device(T** p, size_t* cap, size_t need) {
    if (*cap >= need && *p) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    size_t n = std::max(need, (size_t)1);
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e == cudaSuccess) *cap = n;
    return e;
}

template <typename T>
inline cudaError_t grow_pinned(T** p, size_t* cap, size_t need) {
    if (*cap >= need && *p) return cudaSuccess;
    if (*p) cudaFreeHost(*p);
    *p = nullptr;
    *cap = 0;
    size_t n = std::max(need, (size_t)1);
    cudaError_t e = cudaMallocHost((void**)p, n * sizeof(T));
    if (e == cudaSuccess) *cap = n;
    return e;
}

}  // namespace ixh
