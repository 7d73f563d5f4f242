// M2L on the 5th-generation tensor cores (tcgen05, kind::tf32, FP32
// accumulation in tensor memory) for expansions of order 4 (64 nodes) and
// order 5 (125 nodes, stored with a node stride of 128).
//
// For one offset o every target box t with a source s = t + o needs
//     L_t^T (R x NS) += E_s^T (R x NS) * K_o^T (NS x NS).
// A CTA owns kGroup target boxes of one octant class (so their interaction
// lists use the same offsets) and a 64-wide chunk of right-hand sides:
// kGroup / 2 accumulators D_h (128 x NS each, FP32, in TMEM), D_h =
// [E_s(2h)^T; E_s(2h+1)^T] (128 x NS, A operand) times K_o^T (NS x NS, B
// operand), accumulated over the union of the boxes' offsets; each operator
// tile staged in shared memory feeds every accumulator.  Expansions are
// stored E[box][r][node] and the operator table K[o][m][l] (target node m,
// source node l), both with node stride NS, so every A row (one right-hand
// side) and every B row (one target node) is a contiguous K-major row: the
// contraction over source nodes runs in chunks of 32 TF32 (one 128-byte
// swizzle atom per row), and each chunk is one pipeline stage: kGroup / 2 A
// tiles (128 rows x 128 B each) and B (NS rows x 128 B).
// Warp-specialised: four producer warps copy each stage with cp.async
// straight into the 128-byte-swizzled layout the MMA descriptors name and
// signal the stage's `full` mbarrier with cp.async.mbarrier.arrive (128
// arrivals); one thread of the fifth warp waits on `full`, issues the
// 4 kGroup / 2 K=8 MMAs of the chunk and commits them to the stage's `empty` mbarrier,
// which the producers wait on before refilling the stage.  kStages stages
// are in flight, with no block-wide barrier in the main loop.
// The tensor cores read FP32 operands as TF32 (the operator table is stored
// rounded to TF32, the expansions are truncated by the hardware).
// Every mbarrier wait is bounded; on expiry the kernel records an error code,
// drains (bounded) its own MMAs and copies, frees its TMEM and returns.
#include "farfield.cuh"

namespace gpx {

namespace {

constexpr int kProducers = 128;            // four producer warps
constexpr int kThreads = kProducers + 32;  // + the MMA warp
constexpr int kWaitLimit = 1 << 22;

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

// Byte offset of 16-byte chunk `chunk` (0..7) of row `row` in a 128B-swizzled tile.
__device__ __forceinline__ uint32_t swz(uint32_t row, uint32_t chunk) {
    return (row >> 3) * 1024u + (row & 7u) * 128u + ((chunk ^ (row & 7u)) << 4);
}

__device__ __forceinline__ void cp16(uint32_t dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0) : "memory");
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

template <int NS>
struct TcCfg {
    static constexpr int kStages = 2;
    static constexpr int kTiles = kGroup / 2;                  // A tiles (accumulators) per stage
    static constexpr uint32_t kATile = 128 * 128;              // 128 rows x 128 B
    static constexpr uint32_t kBTile = NS * 128;               // NS rows x 128 B
    static constexpr uint32_t kStage = kTiles * kATile + kBTile;  // multiple of 1024
    static constexpr uint32_t kSmem = kStages * kStage + 1024 + 256;  // + alignment slack + barriers
    static constexpr uint32_t kTmemCols = kTiles * NS;         // 128 or 256 FP32 columns
    static constexpr int kChunks = NS / 32;                    // contraction chunks per entry
    // Instruction descriptor: D F32, A/B TF32, both K-major, N = NS, M = 128.
    static constexpr uint32_t kIdesc =
        (1u << 4) | (2u << 7) | (2u << 10) | (((uint32_t)NS >> 3) << 17) | ((128u >> 4) << 24);
};

template <int NS>
__global__ void __launch_bounds__(kThreads) k_m2l_tc(TcLevel lv, const float* __restrict__ E, float* __restrict__ L,
                                                     const float* __restrict__ K32, int R, float scale,
                                                     const double* __restrict__ box_scale, int* __restrict__ err) {
    using C = TcCfg<NS>;
    constexpr int S = C::kStages;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* sbase = smem_raw + (base - raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sbase + S * C::kStage);  // full[S], empty[S]
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2 * S);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int item = blockIdx.x;
    const int r0 = blockIdx.y * 64;
    const int e0 = lv.item_off[item], e1 = lv.item_off[item + 1];
    const int total = (e1 - e0) * C::kChunks;

    uint64_t* full = bars;
    uint64_t* empty = bars + S;
    __shared__ int s_bad;
    if (tid == 0) {
        for (int k = 0; k < S; ++k) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&full[k])), "r"(kProducers));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[k])));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_bad = 0;
    }
    if (warp == 4) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(C::kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tslot;

    // Copies of chunk q (entry q / kChunks, source nodes 32 (q % kChunks) ..)
    // into stage q % S: A tile h, rows 0..63 from target 2h's source, rows
    // 64..127 from target 2h+1's (zero-filled where a target has no source at
    // this offset); B rows = the operator's target nodes.  Every producer
    // thread copies 8 pieces of 16 bytes per A tile and NS/16 of B; 8
    // consecutive threads read one 128-byte row segment.
    auto issue = [&](int q) {
        const int e = e0 + q / C::kChunks, kc = q % C::kChunks;
        const uint32_t a = base + (uint32_t)(q % S) * C::kStage;
        const uint32_t b = a + C::kTiles * C::kATile;
        int srcs[kGroup];
#pragma unroll
        for (int g = 0; g < kGroup; ++g) srcs[g] = lv.src[(int64_t)e * kGroup + g];
#pragma unroll
        for (int i = 0; i < 8 * C::kTiles; ++i) {
            const int id = tid + kProducers * i, h = id >> 10, row = (id >> 3) & 127, pc = id & 7;
            const int src = srcs[2 * h + (row >> 6)];
            const float* g = src >= 0 ? E + ((int64_t)src * R + r0 + (row & 63)) * NS + kc * 32 + pc * 4 : E;
            cp16(a + (uint32_t)h * C::kATile + swz(row, pc), g, src >= 0);
        }
        const float* Ko = K32 + (int64_t)lv.slot[e] * NS * NS + kc * 32;
#pragma unroll
        for (int i = 0; i < NS / 16; ++i) {
            const int id = tid + kProducers * i, row = id >> 3, pc = id & 7;
            cp16(b + swz(row, pc), Ko + (int64_t)row * NS + pc * 4, true);
        }
    };

    int issued = 0;  // chunks whose MMAs were committed (MMA thread)
    if (tid < kProducers) {
        for (int q = 0; q < total; ++q) {
            const int st = q % S;
            if (q >= S && !mbar_wait(smem_u32(&empty[st]), (uint32_t)(((q / S) - 1) & 1))) {
                atomicExch(&s_bad, 1);
                break;
            }
            if (*(volatile int*)&s_bad) break;
            issue(q);
            asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(&full[st]))
                         : "memory");
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else if (tid == kProducers) {
        for (int q = 0; q < total; ++q) {
            const int st = q % S;
            if (!mbar_wait(smem_u32(&full[st]), (uint32_t)((q / S) & 1))) {
                atomicExch(&s_bad, 1);
                break;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t abase = base + (uint32_t)st * C::kStage, bbase = abase + C::kTiles * C::kATile;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint64_t bd = desc_sw128(bbase + (uint32_t)k * 32u);
                const uint32_t acc = (q > 0 || k > 0) ? 1u : 0u;
#pragma unroll
                for (int h = 0; h < C::kTiles; ++h) {
                    const uint64_t ad = desc_sw128(abase + (uint32_t)h * C::kATile + (uint32_t)k * 32u);
                    asm volatile(
                        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem + (uint32_t)(h * NS)),
                        "l"(ad), "l"(bd), "r"(C::kIdesc), "r"(acc));
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&empty[st]))
                         : "memory");
            issued = q + 1;
        }
        // Drain: the last commit covers every MMA issued before it (after an
        // expired wait too, so the TMEM is idle before it is freed).
        if (issued > 0) {
            const int last = issued - 1;
            if (!mbar_wait(smem_u32(&empty[last % S]), (uint32_t)((last / S) & 1))) atomicExch(&s_bad, 1);
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (s_bad) {
        if (tid == 0) atomicExch(err, 1);
    } else if (tid < kProducers && total > 0) {
        // Epilogue: warp w (0..3) reads TMEM lanes 32w..32w+31 = rows of D_h.
        const int row = warp * 32 + lane;
#pragma unroll
        for (int h = 0; h < C::kTiles; ++h) {
            const int t = lv.item_t[(int64_t)item * kGroup + 2 * h + (row >> 6)];
            float* dst = (t >= 0) ? L + ((int64_t)t * R + r0 + (row & 63)) * NS : nullptr;
            const float sc = (t >= 0 && box_scale) ? (float)box_scale[t] : scale;
#pragma unroll
            for (int cb = 0; cb < NS / 16; ++cb) {
                uint32_t v[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(h * NS + cb * 16), v);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (dst) {
#pragma unroll
                    for (int k = 0; k < 16; k += 4) {
                        const float4 o = make_float4(sc * __uint_as_float(v[k]), sc * __uint_as_float(v[k + 1]),
                                                     sc * __uint_as_float(v[k + 2]), sc * __uint_as_float(v[k + 3]));
                        *reinterpret_cast<float4*>(dst + cb * 16 + k) = o;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 4)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::kTmemCols));
}

template <int NS>
void launch_ns(Ctx& c, const TcLevel& lv, const float* E, float* L, const float* K32, int R, float scale,
               const double* box_scale, int* err) {
    using Cf = TcCfg<NS>;
    set_smem_once(k_m2l_tc<NS>, (int)Cf::kSmem);
    k_m2l_tc<NS><<<dim3(lv.nitems, R / 64), kThreads, Cf::kSmem, c.stream>>>(lv, E, L, K32, R, scale, box_scale,
                                                                             err);
    GPX_LAUNCH_CHECK();
}

}  // namespace

void launch_m2l_tc(Ctx& c, const TcLevel& lv, int ns, const float* E, float* L, const float* K32, int R, float scale,
                   const double* box_scale, int* err) {
    if (lv.nitems == 0) return;
    if (R % 64 != 0) throw Error(GPX_ERR_INTERNAL, "tensor-core M2L needs R a multiple of 64");
    if (ns == 64)
        launch_ns<64>(c, lv, E, L, K32, R, scale, box_scale, err);
    else if (ns == 128)
        launch_ns<128>(c, lv, E, L, K32, R, scale, box_scale, err);
    else
        throw Error(GPX_ERR_INTERNAL, "tensor-core M2L runs node strides 64 and 128 (orders 4 and 5)");
}

}  // namespace gpx
