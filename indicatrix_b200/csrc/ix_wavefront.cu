// ix_wavefront.cu -- the wavefront pipeline for batched isotropic scenes: the path state
// lives in HBM between kernels, and each kernel processes one event's queue, so the 4
// paths a warp carries are at the same step of the bounce (the reference's
// event_wavefront/, renderer/gpu/event_wavefront/kernels.rs:11-56, with sort-by-event
// queues).  It shares the transport with the megakernels (ix_transport.cuh: bounce_hit,
// bounce_geometry, bounce_arm, group_finish) and their fixed-point sums, so its sums are
// the megakernels' bits in the exact build.
//
// Compiled twice by the build (IX_EXACT=1 with -fmad=false, IX_EXACT=0 with
// contraction); every symbol is suffixed accordingly.
//
// One iteration (the host replays it from a CUDA graph until the work is done):
//   wf_intersect  active queue -> the hit, rotation and absorption; queues by event:
//                 reflect, refract, frosted, finish (escaped, or at the bounce cap);
//   wf_arm        the three event queues (virtually concatenated, so a warp's 4 paths
//                 share an arm) -> the arm, glare, roulette; next active queue or finish;
//   wf_finish     finish queue -> XYZ into the pixel's fixed-point sums, and the slot
//                 takes the next unclaimed path of the plan (-> next active queue).
// Queues are appended per 256-thread block: one global atomic per block and queue.
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

constexpr int WF_THREADS = 256;
constexpr int WF_GROUPS = WF_THREADS / 8;  // paths per block step

// Path words (one per path) and lane words (one per path and channel).
enum : uint32_t {
    PW_SEED = 0, PW_BOUNCE = 1, PW_O = 2, PW_D = 5, PW_PREV = 8, PW_OBS = 11, PW_NHERO = 14, PW_FLAGS = 15,
    PW_FACET = 16, PW_JOB = 17, PW_ROW = 18, PW_T = 19, PW_WORDS = 20
};
enum : uint32_t {
    LW_LAMBDA = 0, LW_N = 1, LW_ALPHA = 2, LW_ST = 3, LW_PDF = 7, LW_SPLIT = 8, LW_COMPAT = 9, LW_ESC = 10,
    LW_WORDS = 11
};
constexpr uint32_t FLAG_INSIDE = 1u, FLAG_HAS_PREV = 2u, FLAG_ESCAPED = 4u;

struct Slot {
    uint32_t job, row;
    float t, esc;
    bool escaped;
};

// A slot's state is one contiguous 512-byte record: its 20 path words (padded to 32) and
// then, per channel c, its 11 lane words (padded to 12) at 32 + 12 c.  A group moves the
// path words as broadcast 16-byte loads and each lane its own lane words as three 16-byte
// loads, so a path's state is 4 whole DRAM lines and a handful of vector instructions.
constexpr uint32_t SLOT_WORDS = 128;
constexpr uint32_t LW_BASE = 32, LW_STRIDE = 12;

IX_DEV const uint4* rec4(const WaveLaunch& L, uint32_t slot, uint32_t word) {
    return reinterpret_cast<const uint4*>(L.pw + (size_t)slot * SLOT_WORDS + word);
}
IX_DEV uint4* rec4w(const WaveLaunch& L, uint32_t slot, uint32_t word) {
    return reinterpret_cast<uint4*>(L.pw + (size_t)slot * SLOT_WORDS + word);
}

IX_DEV void wf_load(const WaveLaunch& L, uint32_t slot, const Group& g, LanePath& P, Slot& s) {
    uint32_t w[24];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const uint4 v = __ldcg(rec4(L, slot, 4 * k));
        w[4 * k] = v.x;
        w[4 * k + 1] = v.y;
        w[4 * k + 2] = v.z;
        w[4 * k + 3] = v.w;
    }
    const float* f = reinterpret_cast<const float*>(w);
    P.seed = w[PW_SEED];
    P.bounce = w[PW_BOUNCE];
    P.o = v3(f[PW_O], f[PW_O + 1], f[PW_O + 2]);
    P.d = v3(f[PW_D], f[PW_D + 1], f[PW_D + 2]);
    P.prev_pn = v3(f[PW_PREV], f[PW_PREV + 1], f[PW_PREV + 2]);
    P.observer = v3(f[PW_OBS], f[PW_OBS + 1], f[PW_OBS + 2]);
    P.n_hero = f[PW_NHERO];
    const uint32_t flags = w[PW_FLAGS];
    P.inside = (flags & FLAG_INSIDE) != 0;
    P.has_prev = (flags & FLAG_HAS_PREV) != 0;
    s.escaped = (flags & FLAG_ESCAPED) != 0;
    P.facet = (int)w[PW_FACET];
    s.job = w[PW_JOB];
    s.row = w[PW_ROW];
    s.t = f[PW_T];
    uint32_t l[12];
    const uint32_t base = LW_BASE + LW_STRIDE * (uint32_t)g.c;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const uint4 v = __ldcg(rec4(L, slot, base + 4 * k));
        l[4 * k] = v.x;
        l[4 * k + 1] = v.y;
        l[4 * k + 2] = v.z;
        l[4 * k + 3] = v.w;
    }
    const float* lf = reinterpret_cast<const float*>(l);
    P.lambda = lf[LW_LAMBDA];
    P.n = lf[LW_N];
    P.alpha = lf[LW_ALPHA];
    P.st = Stokes{lf[LW_ST], lf[LW_ST + 1], lf[LW_ST + 2], lf[LW_ST + 3]};
    P.pdf = lf[LW_PDF];
    P.split = lf[LW_SPLIT];
    P.compat = l[LW_COMPAT];
    s.esc = lf[LW_ESC];
}

IX_DEV void wf_store(const WaveLaunch& L, uint32_t slot, const Group& g, const LanePath& P, const Slot& s) {
    if (g.c == 0) {
        uint32_t w[20];
        w[PW_SEED] = P.seed;
        w[PW_BOUNCE] = P.bounce;
        w[PW_O] = __float_as_uint(P.o.x);
        w[PW_O + 1] = __float_as_uint(P.o.y);
        w[PW_O + 2] = __float_as_uint(P.o.z);
        w[PW_D] = __float_as_uint(P.d.x);
        w[PW_D + 1] = __float_as_uint(P.d.y);
        w[PW_D + 2] = __float_as_uint(P.d.z);
        w[PW_PREV] = __float_as_uint(P.prev_pn.x);
        w[PW_PREV + 1] = __float_as_uint(P.prev_pn.y);
        w[PW_PREV + 2] = __float_as_uint(P.prev_pn.z);
        w[PW_OBS] = __float_as_uint(P.observer.x);
        w[PW_OBS + 1] = __float_as_uint(P.observer.y);
        w[PW_OBS + 2] = __float_as_uint(P.observer.z);
        w[PW_NHERO] = __float_as_uint(P.n_hero);
        w[PW_FLAGS] = (P.inside ? FLAG_INSIDE : 0u) | (P.has_prev ? FLAG_HAS_PREV : 0u) | (s.escaped ? FLAG_ESCAPED : 0u);
        w[PW_FACET] = (uint32_t)P.facet;
        w[PW_JOB] = s.job;
        w[PW_ROW] = s.row;
        w[PW_T] = __float_as_uint(s.t);
#pragma unroll
        for (int k = 0; k < 5; ++k) __stcg(rec4w(L, slot, 4 * k), make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]));
    }
    uint32_t l[12];
    l[LW_LAMBDA] = __float_as_uint(P.lambda);
    l[LW_N] = __float_as_uint(P.n);
    l[LW_ALPHA] = __float_as_uint(P.alpha);
    l[LW_ST] = __float_as_uint(P.st.i);
    l[LW_ST + 1] = __float_as_uint(P.st.q);
    l[LW_ST + 2] = __float_as_uint(P.st.u);
    l[LW_ST + 3] = __float_as_uint(P.st.v);
    l[LW_PDF] = __float_as_uint(P.pdf);
    l[LW_SPLIT] = __float_as_uint(P.split);
    l[LW_COMPAT] = P.compat;
    l[LW_ESC] = __float_as_uint(s.esc);
    l[11] = 0u;
    const uint32_t base = LW_BASE + LW_STRIDE * (uint32_t)g.c;
#pragma unroll
    for (int k = 0; k < 3; ++k) __stcg(rec4w(L, slot, base + 4 * k), make_uint4(l[4 * k], l[4 * k + 1], l[4 * k + 2], l[4 * k + 3]));
}

// Block-wide append: group leaders with a destination queue (dest >= 0) append `slot`;
// one global atomic per block and queue.  Every thread of the block calls it.
IX_DEV void block_append(const WaveLaunch& L, int dest, uint32_t slot, bool leader) {
    __shared__ uint32_t s_count[WF_QUEUES], s_base[WF_QUEUES];
    const uint32_t tid = threadIdx.x;
    if (tid < WF_QUEUES) s_count[tid] = 0;
    __syncthreads();
    uint32_t rank = 0;
    if (leader && dest >= 0) rank = atomicAdd(&s_count[dest], 1u);
    __syncthreads();
    if (tid < WF_QUEUES && s_count[tid]) s_base[tid] = atomicAdd(&L.counts[tid], s_count[tid]);
    __syncthreads();
    if (leader && dest >= 0) L.queues[(size_t)dest * L.capacity + s_base[dest] + rank] = slot;
}

// The job a padded path index belongs to (the jobs' path spaces start at 32 x chunk_begin).
IX_DEV uint32_t job_of_path(const WaveLaunch& L, unsigned long long q) {
    const unsigned long long chunk = q / 32ull;
    uint32_t lo = 0, hi = L.n_jobs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((unsigned long long)L.jobs[mid].chunk_begin <= chunk)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Block-wide claim: every group with `want` takes the next padded path index; a group
// whose index is past the plan or in a job's padding gets none.  Returns the index or
// ~0ull.  Every thread of the block calls it.
IX_DEV unsigned long long block_claim(const WaveLaunch& L, bool want, bool leader) {
    __shared__ uint32_t s_need;
    __shared__ unsigned long long s_first;
    if (threadIdx.x == 0) s_need = 0;
    __syncthreads();
    uint32_t rank = 0;
    if (leader && want) rank = atomicAdd(&s_need, 1u);
    __syncthreads();
    if (threadIdx.x == 0) s_first = s_need ? atomicAdd(L.claim, (unsigned long long)s_need) : 0ull;
    __syncthreads();
    unsigned long long q = ~0ull;
    if (want && leader) q = s_first + rank;
    return q;
}

// Starts path `q` (padded index) in `slot`: camera sample, hero comb, initial state.
// Returns false (nothing stored) when q is past the plan or in a job's padding.
IX_DEV bool wf_start_path(const WaveLaunch& L, const Group& g, uint32_t slot, unsigned long long q) {
    if (q >= L.total_slots) return false;
    const uint32_t j = job_of_path(L, q);
    const BatchJob& job = L.jobs[j];
    const unsigned long long i = q - 32ull * job.chunk_begin;
    if (i >= job.paths) return false;
    const uint32_t s = (uint32_t)(i / job.n_pixels);
    const uint32_t row = (uint32_t)(i - (unsigned long long)s * job.n_pixels);
    const DevScene S = make_scene(L.scenes[job.scene], L.flags[job.scene]);
    LanePath P;
    group_init<false>(g, P, S, row, job.sample_offset + s);
    Slot st{j, row, 0.0f, 0.0f, false};
    wf_store(L, slot, g, P, st);
    return true;
}

}  // namespace

// Fills up to `capacity` slots with the plan's first paths (active queue 0).
__global__ void __launch_bounds__(WF_THREADS) IX_SFX(wf_start_kernel)(const __grid_constant__ WaveLaunch L) {
    const Group g = make_group();
    const bool leader = g.c == 0;
    const uint32_t gi = threadIdx.x >> 3;
    for (uint32_t base = blockIdx.x * WF_GROUPS; base < L.capacity; base += gridDim.x * WF_GROUPS) {
        const uint32_t slot = base + gi;
        const bool want = slot < L.capacity;
        unsigned long long q = block_claim(L, want, leader);
        q = __shfl_sync(g.mask, q, 0, 8);
        const bool started = want && wf_start_path(L, g, slot, q);
        block_append(L, started ? WF_ACTIVE0 : -1, slot, leader);
    }
}

// Active queue `parity` -> event queues.
__global__ void __launch_bounds__(WF_THREADS, 4) IX_SFX(wf_intersect_kernel)(const __grid_constant__ WaveLaunch L,
                                                                          int parity) {
    const Group g = make_group();
    const bool leader = g.c == 0;
    const uint32_t gi = threadIdx.x >> 3;
    const int q_in = WF_ACTIVE0 + parity;
    const uint32_t n = *(volatile const uint32_t*)&L.counts[q_in];
    for (uint32_t base = blockIdx.x * WF_GROUPS; base < n; base += gridDim.x * WF_GROUPS) {
        const uint32_t e = base + gi;
        int dest = -1;
        uint32_t slot = 0;
        if (e < n) {
            slot = L.queues[(size_t)q_in * L.capacity + e];
            LanePath P;
            Slot s;
            wf_load(L, slot, g, P, s);
            const BatchJob& job = L.jobs[s.job];
            const DevScene S = make_scene(L.scenes[job.scene], L.flags[job.scene]);
            const float4* planes = reinterpret_cast<const float4*>(S.s.planes);
            if (P.bounce >= S.s.max_bounces) {
                s.escaped = false;
                dest = WF_FINISH;
            } else {
                float esc = 0.0f, t = 0.0f;
                if (bounce_hit(g, P, S, planes, esc, t) == BOUNCE_ESCAPED) {
                    s.escaped = true;
                    s.esc = esc;
                    dest = WF_FINISH;
                } else {
                    s.t = t;
                    BounceGeom G;
                    bounce_geometry(P, S, planes, t, G);
                    dest = G.frosted ? WF_FROSTED : (G.reflect ? WF_REFLECT : WF_REFRACT);
                }
            }
            wf_store(L, slot, g, P, s);
        }
        block_append(L, dest, slot, leader);
    }
}

// The event queues (reflect, refract, frosted, virtually concatenated) -> next active queue
// or finish.
__global__ void __launch_bounds__(WF_THREADS, 3) IX_SFX(wf_arm_kernel)(const __grid_constant__ WaveLaunch L, int parity) {
    const Group g = make_group();
    const bool leader = g.c == 0;
    const uint32_t gi = threadIdx.x >> 3;
    const uint32_t n0 = *(volatile const uint32_t*)&L.counts[WF_REFLECT];
    const uint32_t n1 = *(volatile const uint32_t*)&L.counts[WF_REFRACT];
    const uint32_t n2 = *(volatile const uint32_t*)&L.counts[WF_FROSTED];
    const uint32_t n = n0 + n1 + n2;
    const int q_next = WF_ACTIVE0 + (1 - parity);
    for (uint32_t base = blockIdx.x * WF_GROUPS; base < n; base += gridDim.x * WF_GROUPS) {
        const uint32_t e = base + gi;
        int dest = -1;
        uint32_t slot = 0;
        if (e < n) {
            const int q = e < n0 ? WF_REFLECT : (e < n0 + n1 ? WF_REFRACT : WF_FROSTED);
            const uint32_t k = e < n0 ? e : (e < n0 + n1 ? e - n0 : e - n0 - n1);
            slot = L.queues[(size_t)q * L.capacity + k];
            LanePath P;
            Slot s;
            wf_load(L, slot, g, P, s);
            const BatchJob& job = L.jobs[s.job];
            const DevScene S = make_scene(L.scenes[job.scene], L.flags[job.scene]);
            const float4* planes = reinterpret_cast<const float4*>(S.s.planes);
            BounceGeom G;
            bounce_geometry(P, S, planes, s.t, G);
            const int r = bounce_arm(g, P, S, planes, G);
            if (r == BOUNCE_CONTINUE && P.bounce < S.s.max_bounces) {
                dest = q_next;
            } else {
                s.escaped = false;  // roulette, or the bounce cap
                dest = WF_FINISH;
            }
            wf_store(L, slot, g, P, s);
        }
        block_append(L, dest, slot, leader);
    }
}

// Finish queue -> XYZ into the sums; the slot starts the next unclaimed path.
__global__ void __launch_bounds__(WF_THREADS) IX_SFX(wf_finish_kernel)(const __grid_constant__ WaveLaunch L,
                                                                       int parity) {
    const Group g = make_group();
    const bool leader = g.c == 0;
    const uint32_t gi = threadIdx.x >> 3;
    const uint32_t n = *(volatile const uint32_t*)&L.counts[WF_FINISH];
    const int q_next = WF_ACTIVE0 + (1 - parity);
    uint32_t drops = 0;
    for (uint32_t base = blockIdx.x * WF_GROUPS; base < n; base += gridDim.x * WF_GROUPS) {
        const uint32_t e = base + gi;
        uint32_t slot = 0;
        if (e < n) {
            slot = L.queues[(size_t)WF_FINISH * L.capacity + e];
            LanePath P;
            Slot s;
            wf_load(L, slot, g, P, s);
            const BatchJob& job = L.jobs[s.job];
            const DevScene S = make_scene(L.scenes[job.scene], L.flags[job.scene]);
            const V3 xyz = group_finish(g, P, S, s.escaped, s.esc);
            drops += add_sample_fixed(g, L.acc + job.acc_offset + (size_t)s.row * FIXED_WORDS, xyz);
        }
        unsigned long long q = block_claim(L, e < n, leader);
        q = __shfl_sync(g.mask, q, 0, 8);
        const bool started = e < n && wf_start_path(L, g, slot, q);
        block_append(L, started ? q_next : -1, slot, leader);
    }
    if (drops && L.dropped) atomicAdd(L.dropped, (unsigned long long)drops);
}

namespace {

template <class K>
int resident_blocks(K k) {
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, WF_THREADS, 0) != cudaSuccess) return 0;
    return blocks;
}

}  // namespace

int IX_SFX(wavefront_blocks_per_sm)() {
    int b = resident_blocks(IX_SFX(wf_intersect_kernel));
    const int a = resident_blocks(IX_SFX(wf_arm_kernel)), f = resident_blocks(IX_SFX(wf_finish_kernel));
    if (a < b) b = a;
    if (f < b) b = f;
    return b;
}

cudaError_t IX_SFX(launch_wavefront_start)(const WaveLaunch& l, cudaStream_t stream) {
    if (!l.acc || !l.claim || !l.pw || !l.queues || !l.counts || l.capacity == 0 || l.blocks <= 0)
        return cudaErrorInvalidValue;
    IX_SFX(wf_start_kernel)<<<l.blocks, WF_THREADS, 0, stream>>>(l);
    return cudaGetLastError();
}

// One iteration: clear the queues this iteration fills, then intersect, arms, finish.
cudaError_t IX_SFX(launch_wavefront_iteration)(const WaveLaunch& l, int parity, cudaStream_t stream) {
    const int next = WF_ACTIVE0 + (1 - parity);
    cudaError_t e = cudaMemsetAsync(l.counts + next, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(l.counts + WF_REFLECT, 0, 4 * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    IX_SFX(wf_intersect_kernel)<<<l.blocks, WF_THREADS, 0, stream>>>(l, parity);
    IX_SFX(wf_arm_kernel)<<<l.blocks, WF_THREADS, 0, stream>>>(l, parity);
    IX_SFX(wf_finish_kernel)<<<l.blocks, WF_THREADS, 0, stream>>>(l, parity);
    return cudaGetLastError();
}

}  // namespace ix
