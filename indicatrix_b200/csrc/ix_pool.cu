// ix_pool.cu -- the path-pool trace megakernels (single scene and batched).
//
// Compiled twice by the build (IX_EXACT=1 with -fmad=false, IX_EXACT=0 with
// contraction); every symbol is suffixed accordingly.
//
// The loop (B200-first; the reference's WGSL kernel runs one thread per (pixel, sample)
// tuple and reduces per-tuple XYZ in a second pass):
//   * a path is traced by an 8-lane group, one lane per hero-wavelength channel
//     (ix_transport.cuh); a warp holds 4 paths in flight;
//   * a warp claims 32 paths at a time from a global chunk counter, and its 32 lanes
//     prepare their camera samples together (sample draws and camera ray, one path per
//     lane) into the warp's ring in shared memory;
//   * whenever a group's path finishes, the group takes the next prepared path from the
//     ring, so a warp keeps 4 paths in flight until the launch runs out of work: no warp
//     waits at the end of a task for its slowest group;
//   * a finished path's XYZ is added into its pixel's fixed-point sums with integer
//     reductions at the L2 (ix_launch.h, FIXED_WORDS): integer addition is associative,
//     so the sums are exact and the same bits whatever order the paths finish in, and
//     fixed_to_f64_kernel (ix_fixed.cu) rounds them to f64 once.
// Batched launches claim chunks across jobs (stones x tilts) in order; a warp switches its
// shared-memory plane slot to a new job only once its 4 groups are idle.
#include "ix_fixed.cuh"
#include "ix_launch.h"
#include "ix_transport.cuh"

#if IX_EXACT
#define IX_SFX(name) name##_exact
#else
#define IX_SFX(name) name##_fast
#endif

namespace ix {

namespace {

constexpr uint32_t POOL_CHUNK = 32;   // paths a warp claims at once: one camera sample per lane
constexpr uint32_t POOL_RING = 64;    // prepared camera samples a warp holds
constexpr uint32_t NO_CHUNK = 0xFFFFFFFFu;
constexpr unsigned FULL = 0xFFFFFFFFu;

// A prepared camera sample (its origin is the camera's, the same for every path).
struct PoolEntry {
    float d[3];
    uint32_t seed;
    float hero;
    uint32_t row;  // the path's accumulator row (pixel within its job)
};
// What a warp traces now: one job's scene, sample range and accumulator rows.
struct PoolJob {
    const ix_scene* scene;
    unsigned long long* acc;  // the job's first accumulator row
    uint32_t flags;
    uint32_t scene_index;
    uint32_t n_pixels;
    uint32_t pixel_begin;     // frame pixel of row 0
    uint32_t spp;
    uint32_t sample_offset;
    uint32_t chunk_begin;
    uint32_t paths;
};
struct WarpPool {
    PoolEntry e[POOL_RING];
    PoolJob job;      // the ring's job
    PoolJob pending;  // a claimed chunk's job, waiting for the warp to drain
};

// The warp fills its ring from `chunk` of job `J`: lane l prepares path
// (chunk - chunk_begin) * 32 + l, sample-major within the job.  Returns the paths added.
IX_DEV uint32_t pool_fill(WarpPool& wp, const PoolJob& J, uint32_t chunk, uint32_t tail) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t first = (chunk - J.chunk_begin) * POOL_CHUNK;
    const uint32_t n_valid = min(POOL_CHUNK, J.paths - first);
    __syncwarp();  // every lane has read the slots this fill may reuse
    if (lane < n_valid) {
        const uint32_t i = first + lane;
        const uint32_t s = i / J.n_pixels;
        const uint32_t row = i - s * J.n_pixels;
        const uint32_t pixel = J.pixel_begin + row;
        const ix_scene& sc = *J.scene;
        const Draws dr = sample_draws(pixel, J.sample_offset + s);
        const Ray r = generate_ray(sc.camera, (float)(pixel % sc.width), (float)(pixel / sc.width), (float)sc.width,
                                   (float)sc.height, dr.jx, dr.jy);
        PoolEntry& e = wp.e[(tail + lane) % POOL_RING];
        e.d[0] = r.dir.x;
        e.d[1] = r.dir.y;
        e.d[2] = r.dir.z;
        e.seed = dr.seed;
        e.hero = dr.hero;
        e.row = row;
    }
    __syncwarp();
    return n_valid;
}

// The path-pool loop of one warp.  `job_of(chunk, &job)` fills the job a global chunk
// belongs to and returns its index; `load_planes(job)` returns the job's planes (called
// with the warp converged and its groups idle).  The k-th claim on `counter` takes chunk
// k * stride while that is below total_chunks.  Returns the samples this lane dropped.
template <int UNI, class JobOf, class LoadPlanes>
IX_DEV uint32_t pool_loop(const Group& g, uint32_t* counter, uint32_t total_chunks, uint32_t stride, WarpPool& wp,
                          JobOf job_of, LoadPlanes load_planes) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t gi = lane >> 3;
    uint32_t head = 0, tail = 0;  // ring cursors (warp-uniform)
    uint32_t pending = NO_CHUNK;  // a claimed chunk not yet in the ring (warp-uniform)
    int pending_job = -1, cur_job = -1;
    bool exhausted = false;
    const float4* planes = nullptr;
    bool busy = false;  // the group has a path in flight (group-uniform)
    uint32_t row = 0;   // ... and its accumulator row
    uint32_t drops = 0;
    LanePath P;
    for (;;) {
        const unsigned idle = __ballot_sync(FULL, !busy) & 0x01010101u;
        const uint32_t n_idle = __popc(idle);
        // Claim and prepare camera samples while the ring cannot serve the idle groups.
        if (tail - head < n_idle && !exhausted) {
            if (pending == NO_CHUNK) {
                uint32_t k = 0;
                if (lane == 0) k = atomicAdd(counter, 1u);
                k = __shfl_sync(FULL, k, 0);
                const uint64_t c = (uint64_t)k * stride;  // the k-th claim's chunk
                if (c < total_chunks) {
                    pending = (uint32_t)c;
                    pending_job = job_of(pending, wp.pending);
                } else {
                    exhausted = true;
                }
            }
            if (pending != NO_CHUNK) {
                if (pending_job != cur_job && n_idle == 4 && head == tail) {
                    // Drained: switch the warp to the new job.
                    __syncwarp();
                    if (lane == 0) wp.job = wp.pending;
                    __syncwarp();
                    planes = load_planes(wp.job);
                    cur_job = pending_job;
                }
                if (pending_job == cur_job) {
                    tail += pool_fill(wp, wp.job, pending, tail);
                    pending = NO_CHUNK;
                }
            }
        }
        if (exhausted && n_idle == 4 && head == tail) break;
        // Idle groups take prepared paths in group order.
        const uint32_t avail = tail - head;
        bool fresh = false;
        uint32_t slot = 0;
        if (!busy) {
            const uint32_t rank = __popc(idle & ((1u << (gi * 8u)) - 1u));
            if (rank < avail) {
                fresh = true;
                slot = (head + rank) % POOL_RING;
            }
        }
        head += min(n_idle, avail);
        if (!busy && !fresh) continue;
        const PoolJob& J = wp.job;
        const DevScene S = make_scene(*J.scene, J.flags);
        if (fresh) {
            const PoolEntry& e = wp.e[slot];
            row = e.row;
            const Ray r{load3(S.s.camera.origin), v3(e.d[0], e.d[1], e.d[2])};
            group_init_ray<UNI>(g, P, S, r, e.seed, e.hero);
            busy = true;
        }
        float esc = 0.0f;
        const uint32_t max_bounces = S.s.max_bounces;
        const bool capped = P.bounce >= max_bounces;
        const int r = capped ? (int)BOUNCE_KILLED : group_step<UNI>(g, P, S, planes, esc);
        if (r == BOUNCE_CONTINUE && P.bounce < max_bounces) continue;
        // The path finished (escaped, roulette, or reached the bounce cap).
        const V3 xyz = group_finish<UNI>(g, P, S, r == BOUNCE_ESCAPED, esc);
        drops += add_sample_fixed(g, J.acc + (size_t)row * FIXED_WORDS, xyz);
        busy = false;
    }
    return drops;
}

// Resident-warp targets of the register budgets 1 and 2 (isotropic / uniaxial transport).
template <int UNI>
constexpr int budget_warps(int budget) {
    return budget == 0 ? 0 : (UNI ? (budget == 1 ? 12 : 16) : (budget == 1 ? 24 : 32));
}
template <int WARPS, int UNI>
constexpr int budget_minb(int budget) {
    return budget_warps<UNI>(budget) == 0 ? 1
                                          : (budget_warps<UNI>(budget) / WARPS > 0 ? budget_warps<UNI>(budget) / WARPS : 1);
}

}  // namespace

// Single scene: the launch's pixels x samples; the planes are shared by the whole CTA.
template <int WARPS, int MINB, int UNI>
__global__ void __launch_bounds__(WARPS * 32, MINB) IX_SFX(pool_trace_kernel)(const __grid_constant__ TraceLaunch L) {
    __shared__ float4 s_planes[IX_MAX_PLANES];
    __shared__ WarpPool s_pool[WARPS];
    const float4* gplanes = reinterpret_cast<const float4*>(L.scene.planes);
    for (uint32_t i = threadIdx.x; i < L.scene.n_planes; i += blockDim.x) s_planes[i] = gplanes[i];
    __syncthreads();
    const Group g = make_group();
    WarpPool& wp = s_pool[threadIdx.x >> 5];
    const uint32_t paths = L.n_pixels * L.spp;
    const uint32_t total_chunks = (paths + POOL_CHUNK - 1) / POOL_CHUNK;
    auto job_of = [&](uint32_t, PoolJob& j) {
        if ((threadIdx.x & 31u) == 0) {
            j.scene = &L.scene;
            j.acc = L.acc;
            j.flags = L.flags;
            j.scene_index = 0;
            j.n_pixels = L.n_pixels;
            j.pixel_begin = L.pixel_begin;
            j.spp = L.spp;
            j.sample_offset = L.sample_offset;
            j.chunk_begin = 0;
            j.paths = paths;
        }
        __syncwarp();
        return 0;
    };
    auto load_planes = [&](const PoolJob&) { return (const float4*)s_planes; };
    const uint32_t drops = pool_loop<UNI>(g, L.task_counter, total_chunks, 1u, wp, job_of, load_planes);
    if (drops && L.dropped) atomicAdd(L.dropped, (unsigned long long)drops);
}

// Many scenes in one persistent launch: the chunk space is the concatenation of every
// job's chunks; a warp finds a chunk's job by binary search over the jobs' first chunks
// and keeps the planes of its current job's scene in its own shared-memory slot.
template <int WARPS, int MINB, int UNI>
__global__ void __launch_bounds__(WARPS * 32, MINB) IX_SFX(pool_batch_kernel)(const __grid_constant__ BatchLaunch L) {
    __shared__ float4 s_planes[WARPS][IX_MAX_PLANES];
    __shared__ WarpPool s_pool[WARPS];
    const Group g = make_group();
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    WarpPool& wp = s_pool[warp];
    float4* slot = s_planes[warp];
    uint32_t cached_scene = 0xFFFFFFFFu;
    auto job_of = [&](uint32_t chunk, PoolJob& j) {
        uint32_t lo = 0, hi = L.n_jobs;  // last job with chunk_begin <= chunk
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (L.jobs[mid].chunk_begin <= chunk)
                lo = mid;
            else
                hi = mid;
        }
        if (lane == 0) {
            const BatchJob& b = L.jobs[lo];
            j.scene = &L.scenes[b.scene];
            j.acc = L.acc + b.acc_offset;
            j.flags = L.flags[b.scene];
            j.scene_index = b.scene;
            j.n_pixels = b.n_pixels;
            j.pixel_begin = 0;
            j.spp = b.spp;
            j.sample_offset = b.sample_offset;
            j.chunk_begin = b.chunk_begin;
            j.paths = b.paths;
        }
        __syncwarp();
        return (int)lo;
    };
    auto load_planes = [&](const PoolJob& j) {
        if (j.scene_index != cached_scene) {
            const ix_scene& sc = *j.scene;
            const float4* gp = reinterpret_cast<const float4*>(sc.planes);
            for (uint32_t i = lane; i < sc.n_planes; i += 32) slot[i] = gp[i];
            __syncwarp();
            cached_scene = j.scene_index;
        }
        return (const float4*)slot;
    };
    const uint32_t drops = pool_loop<UNI>(g, L.task_counter, L.total_chunks, L.stride, wp, job_of, load_planes);
    if (drops && L.dropped) atomicAdd(L.dropped, (unsigned long long)drops);
}

namespace {

// Kernel of (shape, budget, transport) for the single-scene and the batched loop.  The
// exact build carries the 128-thread shape only, the single-scene loop that shape only.
template <int WARPS, int UNI>
struct PoolKernels {
    static void* trace(int budget) {
        switch (budget) {
            case 1: return (void*)IX_SFX(pool_trace_kernel)<WARPS, budget_minb<WARPS, UNI>(1), UNI>;
            case 2: return (void*)IX_SFX(pool_trace_kernel)<WARPS, budget_minb<WARPS, UNI>(2), UNI>;
            default: return (void*)IX_SFX(pool_trace_kernel)<WARPS, 1, UNI>;
        }
    }
    static void* batch(int budget) {
        switch (budget) {
            case 1: return (void*)IX_SFX(pool_batch_kernel)<WARPS, budget_minb<WARPS, UNI>(1), UNI>;
            case 2: return (void*)IX_SFX(pool_batch_kernel)<WARPS, budget_minb<WARPS, UNI>(2), UNI>;
            default: return (void*)IX_SFX(pool_batch_kernel)<WARPS, 1, UNI>;
        }
    }
};

template <int UNI>
void* pick(bool batch, int variant) {
    const int shape = variant_shape(variant), budget = variant_budget(variant);
    if (shape == SHAPE_POOL_128) return batch ? PoolKernels<4, UNI>::batch(budget) : PoolKernels<4, UNI>::trace(budget);
#if !IX_EXACT
    if (shape == SHAPE_POOL_64) return batch ? PoolKernels<2, UNI>::batch(budget) : nullptr;
    if (shape == SHAPE_POOL_256) return batch ? PoolKernels<8, UNI>::batch(budget) : nullptr;
#endif
    return nullptr;
}
void* pick_kernel(bool batch, int variant, int transport) {
    if (variant < 0 || variant >= N_VARIANTS) return nullptr;
    switch (transport) {
        case TRANSPORT_EXTENDED: return pick<TRANSPORT_EXTENDED>(batch, variant);
        case TRANSPORT_UNIAXIAL: return pick<TRANSPORT_UNIAXIAL>(batch, variant);
        default: return pick<TRANSPORT_ISOTROPIC>(batch, variant);
    }
}

int blocks_per_sm(void* k, int variant) {
    if (!k) return 0;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, shape_threads(variant_shape(variant)), 0) !=
        cudaSuccess)
        return 0;
    return blocks;
}

}  // namespace

cudaError_t IX_SFX(launch_pool_trace)(const TraceLaunch& l, cudaStream_t stream) {
    void* k = pick_kernel(false, l.variant, transport_class(l.flags));
    if (!k || !l.acc || l.threads != shape_threads(variant_shape(l.variant))) return cudaErrorInvalidValue;
    if (l.scene.n_planes > IX_MAX_PLANES || l.spp > FIXED_MAX_SAMPLES) return cudaErrorInvalidValue;
    if ((uint64_t)l.n_pixels * l.spp > 0xFFFFFFFFull - POOL_CHUNK) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(l.task_counter, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(l.acc, 0, (size_t)l.n_pixels * FIXED_WORDS * sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    void* args[] = {(void*)&l};
    e = cudaLaunchKernel(k, dim3((unsigned)l.blocks), dim3((unsigned)l.threads), args, 0, stream);
    if (e != cudaSuccess) return e;
    return launch_fixed_to_f64(l.acc, l.out, l.n_pixels, l.accumulate, stream);
}

cudaError_t IX_SFX(launch_pool_batch)(const BatchLaunch& l, cudaStream_t stream) {
    void* k = pick_kernel(true, l.variant, (int)l.uniaxial);
    if (!k || !l.acc || l.n_jobs == 0 || l.stride == 0 || l.threads != shape_threads(variant_shape(l.variant)))
        return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(l.task_counter, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    void* args[] = {(void*)&l};
    return cudaLaunchKernel(k, dim3((unsigned)l.blocks), dim3((unsigned)l.threads), args, 0, stream);
}

int IX_SFX(pool_trace_blocks_per_sm)(int variant, int uniaxial) {
    return blocks_per_sm(pick_kernel(false, variant, uniaxial), variant);
}
int IX_SFX(pool_batch_blocks_per_sm)(int variant, int uniaxial) {
    return blocks_per_sm(pick_kernel(true, variant, uniaxial), variant);
}

}  // namespace ix
