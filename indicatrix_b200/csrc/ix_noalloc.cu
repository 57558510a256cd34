// ix_noalloc.cu -- an accumulate entry point that allocates nothing.
//
// Who needs it: callers that cannot call cudaMalloc -- for example a host that hands
// this library device memory from its own pool or arena allocator and forbids any other
// allocation on the device (a graphics engine's resource manager, a plug-in sandbox, an
// embedded runtime with a fixed memory budget), or code running where the CUDA
// allocator is unavailable.  They own the scene's planes and the output sums; the only
// other memory the trace kernel needs -- its work-claiming counters and the dropped-
// sample counter -- lives in the file-scope device array below, which exists on every
// GPU that loads this library from module load until process exit.
//
// The array's name is only a host-side stand-in in host code, not a device address, so
// the address is fetched with cudaGetSymbolAddress once per device (with that device
// current) and passed to the kernel as a plain pointer.

#include "../../include/ix_cuda.h"
#include "ix_launch.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

namespace {

// Scratch layout (32-bit words): one work counter per launch of a call, then the 64-bit
// dropped-sample counter.
constexpr int kMaxLaunches = IX_NOALLOC_MAX_LAUNCHES;
constexpr int kScratchWords = kMaxLaunches + 2;
constexpr uint64_t kChunkPaths = 64ull << 20;  // paths per launch
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];

struct DeviceSetup {
    bool ready = false;
    uint32_t* scratch = nullptr;  // device address of g_noalloc_scratch
    int sm_count = 0;
    int blocks_per_sm[ix::N_TRANSPORT_CLASSES] = {0, 0, 0};  // by transport instantiation (TransportClass)
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mu;

// First call on a device: resolve the scratch address and the launch shape.  Allocates
// nothing (symbol lookup and attribute / occupancy queries only).
int setup_device(int dev, DeviceSetup** out) {
    if (dev < 0 || dev >= kMaxDevices) return IX_NOALLOC_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    DeviceSetup& s = g_setup[dev];
    if (!s.ready) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            (void)cudaGetLastError();
            return IX_NOALLOC_ERR_CUDA;
        }
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
            (void)cudaGetLastError();
            return IX_NOALLOC_ERR_CUDA;
        }
        s.scratch = static_cast<uint32_t*>(p);
        s.sm_count = sms;
        for (int u = 0; u < ix::N_TRANSPORT_CLASSES; ++u)
            s.blocks_per_sm[u] = std::max(1, ix::trace_blocks_per_sm_fast(128, 2, u, nullptr));
        s.ready = true;
    }
    *out = &s;
    return 0;
}

}  // namespace

extern "C" int ix_accumulate_device_noalloc(const ix_scene* scene, uint32_t sample_offset,
                                            uint32_t spp, double* d_accum_xyz, int accumulate,
                                            void* stream) {
    if (!scene || !d_accum_xyz) return IX_NOALLOC_ERR_ARGS;
    if (!ix::routes_device_scene(scene)) return IX_DECLINED;
    const uint64_t n_pixels = (uint64_t)scene->width * scene->height;
    if (n_pixels == 0 || spp == 0) return IX_DONE;
    // Every launch needs its own counter slot: reject what would need more launches than
    // the scratch array holds, before touching the device.
    const uint64_t px_per_launch = std::max<uint64_t>(1, kChunkPaths / spp);
    const uint64_t launches = (n_pixels + px_per_launch - 1) / px_per_launch;
    if (launches > (uint64_t)kMaxLaunches) return IX_NOALLOC_ERR_TOO_LARGE;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return IX_NOALLOC_ERR_CUDA;
    }
    DeviceSetup* s = nullptr;
    if (setup_device(dev, &s) != 0) return IX_NOALLOC_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The array keeps the previous call's contents: clear the counters first.
    if (cudaMemsetAsync(s->scratch, 0, sizeof(uint32_t) * kScratchWords, st) != cudaSuccess) {
        (void)cudaGetLastError();
        return IX_NOALLOC_ERR_CUDA;
    }
    ix::TraceLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.scene = *scene;  // planes and facet finishes in device memory, as ix_accumulate_device
    L.flags = ix::scene_flags(*scene);
    L.sample_offset = sample_offset;
    L.spp = spp;
    uint32_t ppt = 256u / spp;
    L.pixels_per_task = std::max(1u, std::min(8u, ppt));
    L.accumulate = accumulate ? 1 : 0;
    L.dropped = reinterpret_cast<unsigned long long*>(s->scratch + kMaxLaunches);
    L.threads = 128;
    L.variant = 2;
    L.blocks = s->sm_count * s->blocks_per_sm[ix::transport_class(L.flags)];
    uint64_t begin = 0;
    for (int k = 0; begin < n_pixels; ++k) {
        const uint32_t n = (uint32_t)std::min<uint64_t>(px_per_launch, n_pixels - begin);
        L.pixel_begin = (uint32_t)begin;
        L.n_pixels = n;
        L.out = d_accum_xyz + begin * 3;
        L.task_counter = s->scratch + k;
        if (ix::launch_trace_fast(L, st) != cudaSuccess) {
            (void)cudaGetLastError();
            return IX_NOALLOC_ERR_CUDA;
        }
        begin += n;
    }
    return IX_DONE;
}
