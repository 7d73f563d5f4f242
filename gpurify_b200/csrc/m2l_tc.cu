// M2L on the 5th-generation tensor cores (tcgen05, kind::tf32, FP32
// accumulation in tensor memory) for order-4 Chebyshev expansions.
//
// For one offset o every target box t with a source s = t + o needs
//     L_t^T (R x 64) += E_s^T (R x 64) * K_o^T (64 x 64).
// A CTA owns two target boxes (tA, tB) and a 64-wide chunk of right-hand
// sides: D (128 x 64, FP32, in TMEM) = [E_sA^T; E_sB^T] (128 x 64, A operand)
// times K_o^T (64 x 64, B operand), accumulated over the union of the two
// boxes' offsets.  Expansions are stored E[box][r][node], so each A row (one
// right-hand side) and each B row (one target node of K_o) is a contiguous
// 256 B K-major row; rows are staged into shared memory in the 128-byte
// swizzled layout, two K-halves of 32 tf32 each, double buffered: the 128
// threads stage entry i+1 while the single issuing thread's MMAs of entry i
// run; completion is tracked by tcgen05.commit on an mbarrier per stage.
// Every mbarrier wait is bounded; on expiry the kernel records an error code,
// drains (bounded) its own MMAs, frees its TMEM and returns.
#include "farfield.cuh"

namespace gpx {

namespace {

constexpr int kThreads = 128;
constexpr uint32_t kAHalf = 128 * 128;  // 128 rows x 128 B
constexpr uint32_t kBHalf = 64 * 128;   // 64 rows x 128 B
constexpr uint32_t kAStage = 2 * kAHalf;
constexpr uint32_t kBStage = 2 * kBHalf;
constexpr uint32_t kSmemBytes = 2 * kAStage + 2 * kBStage + 64 + 1024;  // + barriers + alignment slack
constexpr uint32_t kTmemCols = 64;
constexpr int kWaitLimit = 1 << 20;

// Instruction descriptor: D F32, A/B TF32, both K-major, N = 64, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: 128 B swizzle, K-major, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;             // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024u >> 4) << 32;  // stride byte offset
    d |= (uint64_t)1 << 46;             // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;             // SWIZZLE_128B
    return d;
}

__device__ __forceinline__ uint32_t swz(uint32_t row, uint32_t chunk) {
    return (row >> 3) * 1024u + (row & 7u) * 128u + ((chunk ^ (row & 7u)) << 4);
}

__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (int i = 0; i < kWaitLimit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

__global__ void __launch_bounds__(kThreads) k_m2l_tc(TcLevel lv, const float* __restrict__ E, float* __restrict__ L,
                                                     const float* __restrict__ K32, int R, float scale,
                                                     int* __restrict__ err) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* sbase = smem_raw + (base - raw);
    uint8_t* sA = sbase;                    // 2 stages x 2 halves x 128 rows
    uint8_t* sB = sbase + 2 * kAStage;      // 2 stages x 2 halves x 64 rows
    uint64_t* bars = reinterpret_cast<uint64_t*>(sbase + 2 * kAStage + 2 * kBStage);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int item = blockIdx.x;
    const int r0 = blockIdx.y * 64;
    const int tA = lv.item_t[2 * item], tB = lv.item_t[2 * item + 1];
    const int e0 = lv.item_off[item], e1 = lv.item_off[item + 1];
    const int nent = e1 - e0;

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tslot;

    bool bad = false;
    for (int i = 0; i < nent; ++i) {
        const int st = i & 1;
        if (i >= 2) {
            const bool ok = mbar_wait(smem_u32(&bars[st]), (uint32_t)(((i - 2) >> 1) & 1));
            if (__syncthreads_or(!ok)) {
                bad = true;
                break;
            }
        }
        const int e = e0 + i;
        const int sa = lv.srcA[e], sb = lv.srcB[e];
        const float* Ko = K32 + (int64_t)lv.slot[e] * 64 * 64;
        uint8_t* a = sA + st * kAStage;
        uint8_t* b = sB + st * kBStage;
        // A: 128 rows (tA rhs 0..63, tB rhs 0..63) x 16 float4 of K
#pragma unroll 4
        for (int q = 0; q < 16; ++q) {
            const int idx = tid + kThreads * q;
            const int row = idx >> 4, c16 = idx & 15;
            const int src = row < 64 ? sa : sb;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (src >= 0) {
                v = *reinterpret_cast<const float4*>(E + ((int64_t)src * R + r0 + (row & 63)) * 64 + 4 * c16);
                v.x = to_tf32(v.x);
                v.y = to_tf32(v.y);
                v.z = to_tf32(v.z);
                v.w = to_tf32(v.w);
            }
            *reinterpret_cast<float4*>(a + (c16 >> 3) * kAHalf + swz(row, c16 & 7)) = v;
        }
        // B: 64 rows (target node m) x 16 float4 of K (source node l)
#pragma unroll 4
        for (int q = 0; q < 8; ++q) {
            const int idx = tid + kThreads * q;
            const int row = idx >> 4, c16 = idx & 15;
            const float4 v = *reinterpret_cast<const float4*>(Ko + row * 64 + 4 * c16);
            *reinterpret_cast<float4*>(b + (c16 >> 3) * kBHalf + swz(row, c16 & 7)) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t abase = smem_u32(a), bbase = smem_u32(b);
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                const uint32_t koff = (uint32_t)(s & 3) * 32u;  // 8 tf32 per MMA along K
                const uint64_t ad = desc_sw128(abase + (uint32_t)(s >> 2) * kAHalf + koff);
                const uint64_t bd = desc_sw128(bbase + (uint32_t)(s >> 2) * kBHalf + koff);
                const uint32_t acc = (i > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bars[st]))
                         : "memory");
        }
    }
    // Drain: the last commit covers every MMA issued before it.
    if (nent > 0) {
        const int last = nent - 1;
        const bool ok = mbar_wait(smem_u32(&bars[last & 1]), (uint32_t)((last >> 1) & 1));
        if (__syncthreads_or(!ok)) bad = true;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (bad) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        // Epilogue: warp w reads TMEM lanes 32w..32w+31 = rows of D.
        const int row = warp * 32 + lane;
        const int t = row < 64 ? tA : tB;
        const int r = r0 + (row & 63);
        float* dst = (t >= 0) ? L + ((int64_t)t * R + r) * 64 : nullptr;
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 16), v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (dst && nent > 0) {
#pragma unroll
                for (int k = 0; k < 16; k += 4) {
                    float4 o = make_float4(scale * __uint_as_float(v[k]), scale * __uint_as_float(v[k + 1]),
                                           scale * __uint_as_float(v[k + 2]), scale * __uint_as_float(v[k + 3]));
                    *reinterpret_cast<float4*>(dst + cb * 16 + k) = o;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

void launch_m2l_tc(Ctx& c, const TcLevel& lv, const float* E, float* L, const float* K32, int R, float scale,
                   int* err) {
    if (lv.nitems == 0) return;
    if (R % 64 != 0) throw Error(GPX_ERR_INTERNAL, "tensor-core M2L needs R a multiple of 64");
    GPX_CUDA(cudaFuncSetAttribute(k_m2l_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
    k_m2l_tc<<<dim3(lv.nitems, R / 64), kThreads, kSmemBytes, c.stream>>>(lv, E, L, K32, R, scale, err);
    GPX_LAUNCH_CHECK();
}

}  // namespace gpx
