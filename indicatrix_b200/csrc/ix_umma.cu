// ix_umma.cu -- the learned surrogate's GEMMs on the 5th-generation tensor cores.
//
// One 256-thread CTA computes a 128 x NT tile of C = A B^T (A: m x k, B: n x k, both read through
// arbitrary row / column strides, so any transpose of the caller's buffers costs nothing
// extra) over a range of K: BF16 operands, FP32 accumulation in tensor memory.
//   * all 256 threads stage 64-wide K slices of A and B into shared memory in the
//     tensor cores' K-major, unswizzled canonical layout (8-row x 16-byte core matrices),
//     zero-filling past the matrix edges, STAGES slices deep: rows contiguous along K go
//     by 16-byte cp.async (in flight while earlier slices multiply), transposed views
//     element by element;
//   * one thread issues the slice's four tcgen05.mma (M 128, N NT, K 16 each) with shared
//     memory descriptors and commits them to the stage's mbarrier, which the threads wait
//     on before they refill that stage;
//   * the accumulator lives in TMEM (NT columns, allocated by warp 0); after the last
//     commit each warp reads its lane quadrant's rows (half of the columns) with tcgen05.ld,
//     transposes them through shared memory and applies the fused epilogue with coalesced
//     stores: store,
//     bias + SiLU (forward), or the SiLU derivative (backward).
// Tall-K products with few output tiles (weight gradients: K = the batch) split K over
// blockIdx.z into f32 partials that a second kernel sums in split order, so results do
// not depend on scheduling.
// Every wait has an iteration limit; a CTA that runs out records it in a status word
// (ix_mlp_status), waits once more (bounded) for its MMAs, frees its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/ix_surrogate.h"

namespace {

constexpr int TM = 128;        // rows of a tile (the MMA's M)
constexpr int BK = 64;         // K per stage: four MMAs of K 16
constexpr int THREADS = 256;      // 8 warps: staging and epilogue split over them
constexpr int STAGES = 3;      // K slices in shared memory at once
constexpr uint32_t WAIT_LIMIT = 1u << 24;  // mbarrier polls before a wait gives up
constexpr int SM_COUNT = 148;

enum Epilogue : int {
    EPI_STORE = 0,      // c = acc
    EPI_BIAS_ACT = 1,   // z = acc + bias; h = act ? silu(z) : z
    EPI_SILU_GRAD = 2,  // g = acc * silu'(zprev)
};

struct GemmParams {
    const __nv_bfloat16* a;
    const __nv_bfloat16* b;
    int64_t a_rs, a_ks;  // A(r, k) = a[r * a_rs + k * a_ks]
    int64_t b_rs, b_ks;  // B(c, k) = b[c * b_rs + k * b_ks]
    uint32_t m, n, k;
    uint32_t k_split;    // K per blockIdx.z (a multiple of BK)
    int epi;
    int act;
    const float* bias;        // EPI_BIAS_ACT: per column (may be null)
    const float* zprev;       // EPI_SILU_GRAD: m x n (ldo)
    float* out_f32;           // m x n (ldo), may be null; split partial z at + z * m * ldo
    __nv_bfloat16* out_bf16;  // m x n (ldo), may be null
    float* out_z;             // EPI_BIAS_ACT: pre-activation, may be null
    uint32_t ldo;
    unsigned int* status;     // device status word
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of a K-major, unswizzled operand: 8 x 16-byte core
// matrices, `sbo` bytes between 8-row groups, `lbo` bytes between the two 8-element K
// halves of one MMA's K 16; descriptor version 1 (sm_100), layout type 0 (no swizzle).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    return d;
}

// Instruction descriptor of kind::f16: F32 accumulator (bits 4-5 = 1), BF16 A and B (bits
// 7-9 and 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t instr_desc(int nt) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(nt >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Polls the mbarrier for the completion of the phase of parity `parity`; false when the
// iteration limit ran out first.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    for (uint32_t i = 0; i < WAIT_LIMIT; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// SiLU and its derivative: silu(z) = z s(z), silu'(z) = s(z) (1 + z (1 - s(z))) with the
// logistic s(z) = 1 / (1 + e^-z).
__device__ __forceinline__ float logistic(float z) { return 1.0f / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * logistic(z); }
__device__ __forceinline__ float silu_grad(float z) {
    const float s = logistic(z);
    return s * (1.0f + z * (1.0f - s));
}

// Stages rows [r0, r0 + R) x k [k0, k0 + BK) of an operand into `stage` in the canonical
// layout -- element (r, k) at ((k / 8) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// bytes -- with zeros at rows >= rows and k >= k_end.
template <int R>
__device__ void stage_tile(uint8_t* stage, const __nv_bfloat16* g, int64_t rs, int64_t ks, uint32_t r0, uint32_t rows,
                           uint32_t k0, uint32_t k_end, bool vec) {
    const uint32_t tid = threadIdx.x;
    if (vec) {
        // 16-byte vectors along K (ks == 1, rows 16-byte aligned); consecutive threads
        // take consecutive rows of one 8-wide K chunk.
        // cp.async with a source size: bytes past it (the matrix's edge) are zero-filled;
        // a chunk wholly outside reads nothing (size 0, from the operand's base address).
        for (uint32_t idx = tid; idx < (uint32_t)R * (BK / 8); idx += THREADS) {
            const uint32_t r = idx % R, kc = idx / R;
            const uint32_t gr = r0 + r, gk = k0 + kc * 8;
            const __nv_bfloat16* p = g;
            uint32_t bytes = 0;
            if (gr < rows && gk < k_end) {
                p = g + (int64_t)gr * rs + gk;
                bytes = 2u * min(8u, k_end - gk);
            }
            const uint32_t dst = smem_u32(stage + (kc * (R / 8) + r / 8) * 128 + (r % 8) * 16);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(p), "r"(bytes) : "memory");
        }
    } else {
        // Element by element; consecutive threads take consecutive rows (coalesced when
        // the operand's rows are adjacent in memory, i.e. a transposed view).
        for (uint32_t idx = tid; idx < (uint32_t)R * BK; idx += THREADS) {
            const uint32_t r = idx % R, kk = idx / R;
            const uint32_t gr = r0 + r, gk = k0 + kk;
            uint16_t e = 0;
            if (gr < rows && gk < k_end) e = __bfloat16_as_ushort(g[(int64_t)gr * rs + (int64_t)gk * ks]);
            *reinterpret_cast<uint16_t*>(stage + ((kk / 8) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (kk % 8) * 2) = e;
        }
    }
}

template <int NT>
__global__ void __launch_bounds__(THREADS) umma_gemm_kernel(const __grid_constant__ GemmParams P) {
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr int A_STAGE = TM * BK * 2;
    constexpr int B_STAGE = NT * BK * 2;
    __shared__ __align__(8) uint64_t s_bar[STAGES];
    __shared__ uint32_t s_taddr;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t r0 = blockIdx.x * TM, c0 = blockIdx.y * NT;
    const uint32_t k_begin = blockIdx.z * P.k_split;
    const uint32_t k_end = min(P.k, k_begin + P.k_split);
    const bool a_vec = P.a_ks == 1 && (P.a_rs % 8) == 0 && (((uintptr_t)P.a) & 15u) == 0;
    const bool b_vec = P.b_ks == 1 && (P.b_rs % 8) == 0 && (((uintptr_t)P.b) & 15u) == 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_taddr)),
                     "r"((uint32_t)NT));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int i = 0; i < STAGES; ++i) mbar_init(&s_bar[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = s_taddr;

    const uint32_t n_k = (k_end + BK - 1 - k_begin) / BK;  // k_end > k_begin (host)
    constexpr uint32_t IDESC = instr_desc(NT);
    auto a_slot = [&](uint32_t slot) { return smem + slot * A_STAGE; };
    auto b_slot = [&](uint32_t slot) { return smem + STAGES * A_STAGE + slot * B_STAGE; };
    auto load = [&](uint32_t slice) {
        const uint32_t slot = slice % STAGES, k0 = k_begin + slice * BK;
        stage_tile<TM>(a_slot(slot), P.a, P.a_rs, P.a_ks, r0, P.m, k0, k_end, a_vec);
        stage_tile<NT>(b_slot(slot), P.b, P.b_rs, P.b_ks, c0, P.n, k0, k_end, b_vec);
    };
    // Prologue: slices 0 .. STAGES - 2 in flight.  Every iteration commits one cp.async
    // group (possibly empty), so "all but the newest STAGES - 2 groups done" always means
    // "the slice about to be multiplied has landed".
#pragma unroll
    for (uint32_t i = 0; i < (uint32_t)STAGES - 1; ++i) {
        if (i < n_k) load(i);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    bool ok = true;
    for (uint32_t it = 0; it < n_k; ++it) {
        const uint32_t slot = it % STAGES;
        asm volatile("cp.async.wait_group %0;" ::"n"(STAGES - 2) : "memory");
        // Make this thread's shared-memory writes visible to the tensor cores' async proxy.
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a_base = smem_u32(a_slot(slot)), b_base = smem_u32(b_slot(slot));
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
                const uint64_t da = smem_desc(a_base + kk * 2 * (TM / 8) * 128, (TM / 8) * 128, 128);
                const uint64_t db = smem_desc(b_base + kk * 2 * (NT / 8) * 128, (NT / 8) * 128, 128);
                const uint32_t accumulate = (it > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(taddr),
                    "l"(da), "l"(db), "r"(IDESC), "r"(accumulate));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&s_bar[slot]))
                         : "memory");
        }
        // Refill the slot slice it - 1 used with slice it + STAGES - 1, once the MMAs that
        // read it are done; the CTA decides together, so every thread leaves the loop at
        // the same slice.
        const uint32_t next = it + STAGES - 1;
        if (next < n_k) {
            if (it >= 1) {
                const uint32_t prev = it - 1;
                const bool w = mbar_wait(&s_bar[prev % STAGES], (prev / STAGES) & 1u);
                if (__syncthreads_or(!w)) {
                    ok = false;
                    break;
                }
            }
            load(next);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    // The last commit tracks every MMA issued before it.
    const uint32_t last = n_k - 1;
    if (ok) ok = !__syncthreads_or(!mbar_wait(&s_bar[last % STAGES], (last / STAGES) & 1u));
    if (!ok) {
        if (tid == 0) atomicOr(P.status, 1u);
        // A last bounded chance for the tensor cores to drain before TMEM is freed.
        (void)mbar_wait(&s_bar[last % STAGES], (last / STAGES) & 1u);
    } else {
        tc_fence_after();
        // Epilogue: warp w reads TMEM lane quadrant w % 4 (tile rows 32 (w % 4) ..) and
        // column half w / 4; each tcgen05.ld gives a thread 8 consecutive columns of its
        // row.  The warp's 32 x NT/2 block goes through shared memory (the operand stages
        // are free now; rows padded by one word, so both passes are conflict-free) and
        // leaves row by row with the lanes on consecutive columns: every store and every
        // z_prev / bias load is coalesced.
        constexpr int HW = NT / 2;
        const uint32_t quad = warp & 3u, half = warp >> 2;
        float* stage = reinterpret_cast<float*>(smem) + warp * 32 * (HW + 1);
        for (int cc = 0; cc < HW; cc += 8) {
            uint32_t v[8];
            const uint32_t src = taddr + ((quad * 32u) << 16) + half * HW + (uint32_t)cc;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                : "r"(src));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int j = 0; j < 8; ++j) stage[lane * (HW + 1) + cc + j] = __uint_as_float(v[j]);
        }
        __syncwarp();
        float* out_f32 = P.out_f32 ? P.out_f32 + (size_t)blockIdx.z * P.m * P.ldo : nullptr;
        for (int r = 0; r < 32; ++r) {
            const uint32_t row = r0 + quad * 32 + r;
            if (row >= P.m) break;
            for (int c = lane; c < HW; c += 32) {
                const uint32_t col = c0 + half * HW + c;
                if (col >= P.n) break;
                float x = stage[r * (HW + 1) + c];
                const size_t o = (size_t)row * P.ldo + col;
                if (P.epi == EPI_BIAS_ACT) {
                    if (P.bias) x += P.bias[col];
                    if (P.out_z) P.out_z[o] = x;
                    if (P.act) x = silu(x);
                } else if (P.epi == EPI_SILU_GRAD) {
                    x *= silu_grad(P.zprev[o]);
                }
                if (out_f32) out_f32[o] = x;
                if (P.out_bf16) P.out_bf16[o] = __float2bfloat16_rn(x);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"((uint32_t)NT));
}

// c[i] = sum over the splits of part[z * count + i], in split order.
__global__ void __launch_bounds__(256) split_sum_kernel(const float* __restrict__ part, uint32_t splits, uint32_t m,
                                                        uint32_t n, uint32_t ldo, float* __restrict__ c, uint32_t ldc) {
    const uint64_t count = (uint64_t)m * n;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = i / n, col = i - r * n;
        float s = 0.0f;
        for (uint32_t z = 0; z < splits; ++z) s += part[(uint64_t)z * m * ldo + r * ldo + col];
        c[r * ldc + col] = s;
    }
}

template <int NT>
cudaError_t launch_nt(const GemmParams& p, uint32_t splits, cudaStream_t st) {
    // The operand stages, reused by the epilogue's 8 warps x 32 x (NT / 2 + 1) f32 staging.
    constexpr int stage_bytes = STAGES * (TM + NT) * BK * 2, epi_bytes = (THREADS / 32) * 32 * (NT / 2 + 1) * 4;
    const int smem = stage_bytes > epi_bytes ? stage_bytes : epi_bytes;
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [&] {
        attr = cudaFuncSetAttribute(umma_gemm_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    });
    if (attr != cudaSuccess) return attr;
    const dim3 grid((p.m + TM - 1) / TM, (p.n + NT - 1) / NT, splits);
    umma_gemm_kernel<NT><<<grid, THREADS, smem, st>>>(p);
    return cudaGetLastError();
}

__device__ unsigned int g_umma_status;

// Split-K workspace (device, grown on demand; the surrogate's calls are not captured).
std::mutex g_ws_mu;
float* g_ws = nullptr;
size_t g_ws_floats = 0;

float* workspace(size_t floats) {
    std::lock_guard<std::mutex> lk(g_ws_mu);
    if (floats <= g_ws_floats) return g_ws;
    if (g_ws) cudaFree(g_ws);
    g_ws = nullptr;
    g_ws_floats = 0;
    if (cudaMalloc(&g_ws, floats * sizeof(float)) != cudaSuccess) {
        (void)cudaGetLastError();
        g_ws = nullptr;
        return nullptr;
    }
    g_ws_floats = floats;
    return g_ws;
}

uint32_t tiles(uint32_t x, uint32_t t) { return (x + t - 1) / t; }

int run(GemmParams p, void* stream) {
    if (p.m == 0 || p.n == 0) return 0;
    if (p.k == 0 || !p.a || !p.b) return 1;
    if (p.m > (1u << 30) || p.n > (1u << 30) || p.k > (1u << 30)) return 1;
    void* st_ptr = nullptr;
    if (cudaGetSymbolAddress(&st_ptr, g_umma_status) != cudaSuccess) {
        (void)cudaGetLastError();
        return 1;
    }
    p.status = static_cast<unsigned int*>(st_ptr);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Tile width: the narrowest of 32 / 64 / 128 / 256 that covers n, halved (down to 32)
    // while the grid would give fewer than two CTAs per SM.
    int nt = p.n <= 32 ? 32 : p.n <= 64 ? 64 : p.n <= 128 ? 128 : 256;
    while (nt > 32 && tiles(p.m, TM) * tiles(p.n, nt) < 2u * SM_COUNT) nt >>= 1;
    // Split K when the output has few tiles and K is long (store epilogue only).
    uint32_t splits = 1;
    const uint32_t n_tiles = tiles(p.m, TM) * tiles(p.n, nt);
    if (p.epi == EPI_STORE && n_tiles < (uint32_t)SM_COUNT / 2 && p.k >= 8u * BK) {
        splits = (uint32_t)SM_COUNT / n_tiles;
        const uint32_t max_splits = p.k / (4 * BK);
        if (splits > max_splits) splits = max_splits;
        if (splits > 32) splits = 32;
        if (splits < 2) splits = 1;
    }
    p.k_split = splits == 1 ? p.k : tiles(tiles(p.k, splits), BK) * BK;
    if (splits > 1) splits = tiles(p.k, p.k_split);  // every split non-empty
    float* c = p.out_f32;
    const uint32_t ldc = p.ldo;
    if (splits > 1) {
        float* ws = workspace((size_t)splits * p.m * p.n);
        if (!ws) return 1;
        p.out_f32 = ws;
        p.ldo = p.n;
        p.out_bf16 = nullptr;
    }
    cudaError_t e;
    switch (nt) {
        case 32: e = launch_nt<32>(p, splits, s); break;
        case 64: e = launch_nt<64>(p, splits, s); break;
        case 128: e = launch_nt<128>(p, splits, s); break;
        default: e = launch_nt<256>(p, splits, s); break;
    }
    if (e == cudaSuccess && splits > 1) {
        const uint64_t count = (uint64_t)p.m * p.n;
        uint64_t blocks = (count + 255) / 256;
        if (blocks > (uint64_t)SM_COUNT * 8) blocks = (uint64_t)SM_COUNT * 8;
        split_sum_kernel<<<(unsigned)blocks, 256, 0, s>>>(p.out_f32, splits, p.m, p.n, p.ldo, c, ldc);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? 0 : 1;
}

}  // namespace

extern "C" {

int ix_mlp_gemm_bf16(int trans_a, int trans_b, uint32_t m, uint32_t n, uint32_t k, const void* a, uint32_t lda,
                     const void* b, uint32_t ldb, float* c, uint32_t ldc, void* stream) {
    // C = op(A) op(B) in the kernel's form C = A' B'^T: A'(r, kk) = op(A)(r, kk) and
    // B'(col, kk) = op(B)(kk, col).
    if (!c) return 1;
    GemmParams p{};
    p.a = static_cast<const __nv_bfloat16*>(a);
    p.b = static_cast<const __nv_bfloat16*>(b);
    p.a_rs = trans_a ? 1 : lda;
    p.a_ks = trans_a ? lda : 1;
    p.b_rs = trans_b ? ldb : 1;
    p.b_ks = trans_b ? 1 : ldb;
    p.m = m;
    p.n = n;
    p.k = k;
    p.epi = EPI_STORE;
    p.out_f32 = c;
    p.ldo = ldc;
    return run(p, stream);
}

int ix_mlp_linear(uint32_t m, uint32_t n, uint32_t k, const void* x, uint32_t ldx, const void* w, const float* bias,
                  int silu_act, float* z, float* h, void* hb, void* stream) {
    // y = x W^T: A' = x (rows of ldx), B'(col, kk) = W[col][kk].
    GemmParams p{};
    p.a = static_cast<const __nv_bfloat16*>(x);
    p.b = static_cast<const __nv_bfloat16*>(w);
    p.a_rs = ldx;
    p.a_ks = 1;
    p.b_rs = k;
    p.b_ks = 1;
    p.m = m;
    p.n = n;
    p.k = k;
    p.epi = EPI_BIAS_ACT;
    p.act = silu_act;
    p.bias = bias;
    p.out_z = z;
    p.out_f32 = h;
    p.out_bf16 = static_cast<__nv_bfloat16*>(hb);
    p.ldo = n;
    return run(p, stream);
}

int ix_mlp_backward_silu(uint32_t m, uint32_t n, uint32_t k, const void* dz_next, const void* w, const float* z_prev,
                         float* dz, void* dzb, void* stream) {
    // dz = (dz_next W) * silu'(z_prev): A' = dz_next (m x k), B'(col, kk) = W[kk][col].
    if (!z_prev) return 1;
    GemmParams p{};
    p.a = static_cast<const __nv_bfloat16*>(dz_next);
    p.b = static_cast<const __nv_bfloat16*>(w);
    p.a_rs = k;
    p.a_ks = 1;
    p.b_rs = 1;
    p.b_ks = n;
    p.m = m;
    p.n = n;
    p.k = k;
    p.epi = EPI_SILU_GRAD;
    p.zprev = z_prev;
    p.out_f32 = dz;
    p.out_bf16 = static_cast<__nv_bfloat16*>(dzb);
    p.ldo = n;
    return run(p, stream);
}

uint32_t ix_mlp_status(int reset) {
    unsigned int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_umma_status, sizeof(v)) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0xFFFFFFFFu;
    }
    if (reset) {
        const unsigned int zero = 0;
        if (cudaMemcpyToSymbol(g_umma_status, &zero, sizeof(zero)) != cudaSuccess) (void)cudaGetLastError();
    }
    return v;
}

}  // extern "C"
