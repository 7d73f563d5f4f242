// L2P on the 5th-generation tensor cores for the mixed path (orders 4 and 5,
// node stride 64 or 128):
//     Y[j][r] += coef sum_m S[j][m] L[leaf][r][m]   for the panels j of a work item
// (S the target weights: the collocation weights of the panel centroids, or
// for the transposed operator the source weights with the area folded in).
// One CTA per (work item of <= 64 panels, 64-wide chunk of right-hand sides);
// D (M = 128 rows, of which the item's panels use the first <= 64; N = 64
// right-hand sides; FP32 in TMEM) = A B with
//   A = S (panels x nodes): K-major, one row per panel (split into TF32 hi and
//       lo parts once per solve, rows of 128 nodes);
//   B = L[leaf] (right-hand sides x nodes): K-major, one row per right-hand
//       side, split into TF32 hi and lo parts in shared memory once staged.
// D = S_hi L_hi + S_hi L_lo + S_lo L_hi is accurate to about 2^-21.  The
// contraction over the nodes runs in slices of 32 through a 2-stage ring:
// all threads copy a slice with cp.async, split its L tile, and one thread
// issues the slice's MMAs and commits them to the stage's mbarrier, which
// the copies of the slice two ahead wait on (bounded).  The epilogue adds
// coef D to the panels' FP64 rows of Y.
#include "farfield.cuh"

namespace gpx {

namespace {

constexpr int kThreads = 128;
constexpr int kWS = 128;                      // row stride of the split weight arrays
constexpr uint32_t kATile = 128 * 128;        // 128 rows x 32 FP32 (128 B)
constexpr uint32_t kBTile = 64 * 128;         // 64 rows x 32 FP32
constexpr uint32_t kStage = 2 * kATile + 2 * kBTile;  // A_hi, A_lo, B_hi, B_lo: 48 KB
constexpr uint32_t kSmemBytes = 2 * kStage + 1024 + 64 + 4096;
constexpr uint32_t kTmemCols = 64;
constexpr int kWaitLimit = 1 << 22;
// Instruction descriptor: D F32, A/B TF32, both K-major, N = 64, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major operand, 128 B swizzle: 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t desc_k_sw128(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

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

__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

template <int NS>
__global__ void __launch_bounds__(kThreads) k_l2p_tc(DevPlan p, const float* __restrict__ L,
                                                     const float* __restrict__ Shi, const float* __restrict__ Slo,
                                                     double* __restrict__ Y, int R, int Rb, double coef,
                                                     int* __restrict__ err) {
    constexpr int nsl = NS / 32;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* sbase = smem_raw + (base - raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sbase + 2 * kStage);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
    __shared__ int s_bad;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int it = blockIdx.x;
    const int t = p.item_leaf[it], r0 = p.item_row0[it];
    const int rc = blockIdx.y * 64;
    const int64_t jb = p.leaf_begin[t] + r0;
    const int cnt = (int)min((int64_t)64, p.leaf_begin[t + 1] - jb);
    const float* src = L + ((int64_t)(p.leaf_box0 + t) * Rb + rc) * NS;
    if (tid == 0) {
        for (int k = 0; k < 2; ++k) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[k])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_bad = 0;
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
    // copies of slice q into stage q % 2: A rows = the item's panels (rows
    // past cnt are not loaded: their D rows are never stored), B rows = the
    // leaf's right-hand sides (all 64 rows valid: L has Rb rows per box)
    auto issue = [&](int q) {
        const uint32_t a = base + (uint32_t)(q & 1) * kStage;
        for (int e = tid; e < 64 * 8; e += kThreads) {
            const int row = e >> 3, c = e & 7;
            if (row < cnt) {
                const int64_t off = (jb + row) * kWS + 32 * q + 4 * c;
                cp16(a + swz(row, c), Shi + off, true);
                cp16(a + kATile + swz(row, c), Slo + off, true);
            }
            cp16(a + 2 * kATile + swz(row, c), src + (int64_t)row * NS + 32 * q + 4 * c, true);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    bool bad = false;
    int committed = 0;  // slices whose MMAs thread 0 committed (uniform across the CTA)
    issue(0);
    for (int q = 0; q < nsl; ++q) {
        const int st = q & 1;
        if (q + 1 < nsl) {
            // stage (q+1)&1 last held slice q-1: its MMAs must be done
            if (q >= 1 && !mbar_wait(smem_u32(&bars[(q + 1) & 1]), (uint32_t)(((q - 1) >> 1) & 1))) bad = true;
            if (__syncthreads_or(bad)) {
                bad = true;
                break;
            }
            issue(q + 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        // split the L tile of this slice: B_hi in place, B_lo beside it
        {
            uint8_t* b = sbase + (size_t)st * kStage + 2 * kATile;
            for (int e = tid; e < 64 * 8; e += kThreads) {
                const uint32_t o = swz((uint32_t)(e >> 3), (uint32_t)(e & 7));
                float4* hp = reinterpret_cast<float4*>(b + o);
                float4* lp = reinterpret_cast<float4*>(b + kBTile + o);
                const float4 v = *hp;
                const float4 h = make_float4(to_tf32(v.x), to_tf32(v.y), to_tf32(v.z), to_tf32(v.w));
                *lp = make_float4(to_tf32(v.x - h.x), to_tf32(v.y - h.y), to_tf32(v.z - h.z), to_tf32(v.w - h.w));
                *hp = h;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t ah = base + (uint32_t)st * kStage, al = ah + kATile;
            const uint32_t bh = ah + 2 * kATile, bl = bh + kBTile;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const uint64_t adh = desc_k_sw128(ah + (uint32_t)kk * 32u), adl = desc_k_sw128(al + (uint32_t)kk * 32u);
                const uint64_t bdh = desc_k_sw128(bh + (uint32_t)kk * 32u), bdl = desc_k_sw128(bl + (uint32_t)kk * 32u);
                const uint32_t accf = (q > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(adh), "l"(bdh), "r"(kIdesc), "r"(accf));
                asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;" ::"r"(tmem), "l"(adh),
                             "l"(bdl), "r"(kIdesc));
                asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;" ::"r"(tmem), "l"(adl),
                             "l"(bdh), "r"(kIdesc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bars[st]))
                         : "memory");
        }
        committed = q + 1;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    // Drain (also after an expired wait, so the TMEM is idle before it is
    // freed): the last commit covers every MMA issued before it; the commit of
    // slice q is completion (q >> 1) of bars[q & 1].
    if (committed > 0) {
        const int last = committed - 1;
        if (!mbar_wait(smem_u32(&bars[last & 1]), (uint32_t)((last >> 1) & 1))) bad = true;
    }
    if (__syncthreads_or(bad)) {
        if (tid == 0) atomicExch(err, 1);
        bad = true;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!bad) {
        const int row = warp * 32 + lane;
        double* y = row < cnt ? Y + (jb + row) * R + rc : nullptr;
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 16), v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (y) {
#pragma unroll
                for (int k = 0; k < 16; k += 2) {
                    const int col = cb * 16 + k;
                    if (rc + col + 1 < R) {
                        double2 o = *reinterpret_cast<double2*>(y + col);
                        o.x += coef * (double)__uint_as_float(v[k]);
                        o.y += coef * (double)__uint_as_float(v[k + 1]);
                        *reinterpret_cast<double2*>(y + col) = o;
                    } else if (rc + col < R) {
                        y[col] += coef * (double)__uint_as_float(v[k]);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

void launch_l2p_tc(Ctx& c, const DevPlan& p, const float* L, const float* Shi, const float* Slo, double* Y, int R,
                   int Rb, double coef, int* err) {
    if (p.nitems == 0) return;
    if (R % 4 != 0 || Rb % 64 != 0) throw Error(GPX_ERR_INTERNAL, "tensor-core L2P needs R % 4 == 0, Rb % 64 == 0");
    const dim3 grid(p.nitems, (R + 63) / 64);
    if (p.ns == 128) {
        set_smem_once(k_l2p_tc<128>, (int)kSmemBytes);
        k_l2p_tc<128><<<grid, kThreads, kSmemBytes, c.stream>>>(p, L, Shi, Slo, Y, R, Rb, coef, err);
    } else if (p.ns == 64) {
        set_smem_once(k_l2p_tc<64>, (int)kSmemBytes);
        k_l2p_tc<64><<<grid, kThreads, kSmemBytes, c.stream>>>(p, L, Shi, Slo, Y, R, Rb, coef, err);
    } else {
        throw Error(GPX_ERR_INTERNAL, "tensor-core L2P runs node strides 64 and 128 (orders 4 and 5)");
    }
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

}  // namespace gpx
