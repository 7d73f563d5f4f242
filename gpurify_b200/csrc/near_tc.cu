// Near-field apply on the 5th-generation tensor cores (tcgen05, kind::tf32,
// FP32 accumulation in tensor memory) for the mixed path:
//     Y[rows of item][rc : rc+64] = P_t[rows][0:S] X[near sources of t][rc : rc+64]
// With 64 right-hand sides the near product does 32 flop per streamed FP32
// matrix byte, above what the FP32 CUDA cores sustain per HBM byte, so on the
// CUDA cores it is compute bound; on the tensor cores it is bound by streaming
// the near blocks from HBM.
//
// One CTA per (work item = target leaf and <= 128 of its rows, 64-wide chunk
// of right-hand sides), D = 128 x 64 FP32 in TMEM.  The contraction runs over
// the leaf's S near-source panels in slices of 32; each slice is one stage of
// a kStages ring in shared memory:
//   A (128 x 32, K-major, 128-byte swizzle) = the item's P rows, streamed from
//     HBM;
//   B_hi, B_lo (32 x 64 each, MN-major, 128-byte swizzle on a 32-byte base) = the 32 source
//     panels' rows of X_hi = tf32(x) and X_lo = tf32(x - x_hi), gathered from
//     the L2-resident split copies written by k_split_tf32.  A source row of
//     X is 64 contiguous FP32 values, which is exactly one K row of an
//     MN-major tile, so the gather is a plain copy: no transpose and no
//     per-slice register work.
// D += A B_hi + A B_lo represents X to about 2^-21, so the operator stays
// linear in X (the GMRES inner solves converge as for any fixed matrix); the
// one approximation left is P rounded once to TF32 (round to nearest, stored
// that way), a fixed perturbation the FP64 refinement removes.
// Warp-specialised: four producer warps copy each stage with cp.async
// straight into the swizzled layouts and signal the stage's `full` mbarrier
// (cp.async.mbarrier.arrive, 128 arrivals); one thread of the fifth warp
// waits on `full`, issues the eight K=8 MMAs of the slice and commits them to
// the stage's `empty` mbarrier, which the producers wait on before refilling
// the stage.  No block-wide barrier runs in the main loop.  Rows past the
// item's last row are not loaded (their D rows are never stored); source
// columns past S are zero-filled in both A and B.  Every mbarrier wait is
// bounded: on expiry the kernel records an error code, drains (bounded) its
// own MMAs and copies, frees its TMEM and returns.
#include "kernels.cuh"

namespace gpx {

namespace {

constexpr int kProducers = 128;            // four producer warps, also the epilogue
constexpr int kThreads = kProducers + 32;  // + the MMA warp
constexpr uint32_t kATile = 128 * 128;      // 128 rows x 128 B
constexpr uint32_t kBTile = 32 * 256;       // 32 K rows x 64 FP32
// Operand modes: 0 = P (TF32) and the split X_hi, X_lo gathered from global
// memory; 1 = P kept in FP32 and split into hi and lo on chip (three
// products); 2 = X gathered once as FP32 and split into hi and lo on chip
// (half the gather traffic of mode 0, the same products).
// Stage layout: A, [A_lo in mode 1], B_hi, B_lo.  Modes 0 and 2 stage 32 KB
// and three stages fit twice per SM; mode 1 stages 48 KB, two stages.
template <int MODE>
struct NearCfg {
    static constexpr bool SP = MODE == 1;
    static constexpr int kStages = SP ? 2 : 3;
    static constexpr uint32_t kALo = kATile;                          // offset of A_lo (SP)
    static constexpr uint32_t kBOff = SP ? 2 * kATile : kATile;       // offset of B_hi
    static constexpr uint32_t kStage = kBOff + 2 * kBTile;            // multiple of 1024
    // + alignment slack, barriers and TMEM slot, and 4 KB past the last
    // stage so that no MMA operand read can leave the allocation
    static constexpr uint32_t kSmemBytes = kStages * kStage + 1024 + 256 + 4096;
};
constexpr uint32_t kTmemCols = 64;
constexpr int kWaitLimit = 1 << 22;
// Instruction descriptor: D F32, A/B TF32, A K-major, B MN-major, N = 64, M = 128.
constexpr uint32_t kIdesc =
    (1u << 4) | (2u << 7) | (2u << 10) | (1u << 16) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

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

// MN-major TF32 operand: the only shared-memory layout the tensor cores take
// for 32-bit MN-major operands is SWIZZLE_128B_BASE32B (descriptor layout
// type 1): atoms of 4 K rows x 128 B (32 FP32 along MN), the 32-byte granules
// of row r stored at granule ^ r.  `lbo` = bytes between the atoms of
// consecutive 32-wide MN blocks, `sbo` = bytes between consecutive 4-row K
// groups.
__device__ __forceinline__ uint64_t desc_mn_sw128b32(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFFu) >> 4);
    d |= (uint64_t)(lbo >> 4) << 16;
    d |= (uint64_t)(sbo >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)1 << 61;
    return d;
}

// Byte offset of 16-byte chunk `chunk` of row `row` in a 128-byte-swizzled
// K-major tile.
__device__ __forceinline__ uint32_t swz(uint32_t row, uint32_t chunk) {
    return (row >> 3) * 1024u + (row & 7u) * 128u + ((chunk ^ (row & 7u)) << 4);
}

// Byte offset of 16-byte chunk q (0..15: FP32 columns 4q..4q+3) of K row k
// (0..31) in the MN-major B tile: atom (4-row K group k/4, MN block q/8) at
// (2 (k/4) + q/8) x 512 B, row k%4 of the atom, 32-byte granule (q%8)/2
// swizzled by the row.
__device__ __forceinline__ uint32_t swz_mn(uint32_t k, uint32_t q) {
    const uint32_t r = k & 3u;
    return ((k >> 2) * 2u + (q >> 3)) * 512u + r * 128u + ((((q & 7u) >> 1) ^ r) << 5) + ((q & 1u) << 4);
}

__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
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

// Mode 1 (split P): P holds full FP32 values; the producers split each
// staged A tile into TF32 hi (in place) and lo (A_lo) parts once its copies
// landed, and the MMA thread adds the third product A_lo B_hi, so the near
// apply is accurate to about 2^-21 in both P and X.  Mode 2 (split X on
// chip): Xhi is the FP32 copy of X, Xlo is unused; each producer splits the
// B chunks it copied once they landed.  In modes 1 and 2 a producer signals
// a stage after its own copies of that stage completed and were split (one
// stage of copies stays in flight per producer); in mode 0 the copies
// signal the stage themselves.
template <int MODE>
__global__ void __launch_bounds__(kThreads) k_near_apply_tc(DevPlan p, const int32_t* __restrict__ it_leaf,
                                                            const int32_t* __restrict__ it_row0,
                                                            const float* __restrict__ P,
                                                            const float* __restrict__ Xhi,
                                                            const float* __restrict__ Xlo, double* __restrict__ Y,
                                                            int R, int* __restrict__ err) {
    using Cfg = NearCfg<MODE>;
    constexpr bool SP = Cfg::SP;
    constexpr bool SB = MODE == 2;
    constexpr int kStages = Cfg::kStages;
    constexpr uint32_t kStage = Cfg::kStage;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* sbase = smem_raw + (base - raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(sbase + kStages * kStage);
    uint64_t* empty = full + kStages;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(empty + kStages);
    __shared__ int64_t s_beg[28];
    __shared__ int32_t s_pre[29];
    __shared__ int s_bad;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int t = it_leaf[blockIdx.x];
    const int r0 = it_row0[blockIdx.x];
    const int rc = blockIdx.y * 64;
    const int64_t tb = p.leaf_begin[t] + r0;
    const int m = min((int)(p.leaf_begin[t + 1] - p.leaf_begin[t]) - r0, 128);
    const int S = p.near_S[t];
    const int Sp = (S + 3) & ~3;
    const float* Pi = P + p.nval_off[t] + (int64_t)r0 * Sp;
    const int nsl = (Sp + 31) / 32;

    if (warp == 1) near_ranges_warp(p, t, lane, s_beg, s_pre);
    if (tid == 0) {
        for (int st = 0; st < kStages; ++st) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&full[st])), "r"(kProducers));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[st])));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_bad = 0;
    }
    if (warp == 4) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tslot;

    if (tid < kProducers) {
        // B: this thread copies K row kb = tid / 4 of every slice, chunks
        // 4 (tid % 4) .. 4 (tid % 4) + 3 of X_hi and X_lo.
        const int kb = tid >> 2, q0 = (tid & 3) * 4;
        int e = 0;
        // SP: split the A chunks this thread copied into stage `jj` (after
        // its copies landed), then signal the stage.
        auto split_and_signal = [&](int jj) {
            const int sst = jj % kStages;
            uint8_t* at = sbase + (size_t)sst * kStage;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int id = tid + kProducers * q, row = id >> 3, c16 = id & 7;
                if (row < m) {
                    float4* hp = reinterpret_cast<float4*>(at + swz(row, c16));
                    float4* lp = reinterpret_cast<float4*>(at + Cfg::kALo + swz(row, c16));
                    const float4 v = *hp;
                    const float4 h = make_float4(to_tf32(v.x), to_tf32(v.y), to_tf32(v.z), to_tf32(v.w));
                    *lp = make_float4(to_tf32(v.x - h.x), to_tf32(v.y - h.y), to_tf32(v.z - h.z), to_tf32(v.w - h.w));
                    *hp = h;
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&full[sst])) : "memory");
        };
        // SB: split the B chunks this thread copied into stage `jj` (K row kb,
        // chunks q0 .. q0 + 3: FP32 x into hi in place and lo beside it).
        auto split_b_and_signal = [&](int jj) {
            const int sst = jj % kStages;
            uint8_t* bt = sbase + (size_t)sst * kStage + Cfg::kBOff;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const uint32_t d = swz_mn((uint32_t)kb, (uint32_t)(q0 + i));
                float4* hp = reinterpret_cast<float4*>(bt + d);
                float4* lp = reinterpret_cast<float4*>(bt + kBTile + d);
                const float4 v = *hp;
                const float4 h = make_float4(to_tf32(v.x), to_tf32(v.y), to_tf32(v.z), to_tf32(v.w));
                *lp = make_float4(to_tf32(v.x - h.x), to_tf32(v.y - h.y), to_tf32(v.z - h.z), to_tf32(v.w - h.w));
                *hp = h;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&full[sst])) : "memory");
        };
        int signalled = 0;  // modes 1 and 2: stages split and signalled
        for (int j = 0; j < nsl; ++j) {
            const int st = j % kStages;
            if (j >= kStages && !mbar_wait(smem_u32(&empty[st]), (uint32_t)(((j / kStages) - 1) & 1))) {
                atomicExch(&s_bad, 1);
                break;
            }
            if (*(volatile int*)&s_bad) break;
            const uint32_t a = base + (uint32_t)st * kStage;
            const uint32_t bh = a + Cfg::kBOff, bl = bh + kBTile;
            const int k0 = j * 32;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int id = tid + kProducers * q, row = id >> 3, c16 = id & 7;
                if (row < m) {
                    const bool ok = k0 + 4 * c16 < Sp;
                    cp16(a + swz(row, c16), ok ? (const void*)(Pi + (int64_t)row * Sp + k0 + 4 * c16) : (const void*)P,
                         ok);
                }
            }
            const int k = k0 + kb;
            int64_t gid = -1;
            if (k < S) {
                while (s_pre[e + 1] <= k) ++e;
                gid = s_beg[e] + (k - s_pre[e]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int q = q0 + i, col = rc + 4 * q;
                const bool ok = gid >= 0 && col < R;
                const int64_t off = ok ? gid * R + col : 0;
                const uint32_t d = swz_mn((uint32_t)kb, (uint32_t)q);
                cp16(bh + d, Xhi + off, ok);
                if constexpr (!SB) cp16(bl + d, Xlo + off, ok);
            }
            if constexpr (SP || SB) {
                asm volatile("cp.async.commit_group;" ::: "memory");
                if (j >= 1) {
                    asm volatile("cp.async.wait_group 1;" ::: "memory");
                    if constexpr (SP)
                        split_and_signal(j - 1);
                    else
                        split_b_and_signal(j - 1);
                    signalled = j;
                }
            } else {
                asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(&full[st]))
                             : "memory");
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        if constexpr (SP || SB) {
            // the last issued stage (also after an expired wait: every
            // issued stage is signalled, so the MMA thread never waits on a
            // stage whose copies went out)
            const int issued_p = *(volatile int*)&s_bad ? signalled + 1 : nsl;
            for (int jj = signalled; jj < issued_p && jj < nsl; ++jj) {
                if constexpr (SP)
                    split_and_signal(jj);
                else
                    split_b_and_signal(jj);
            }
        }
    } else if (tid == kProducers) {
        int issued = 0;
        for (int j = 0; j < nsl; ++j) {
            const int st = j % kStages;
            if (!mbar_wait(smem_u32(&full[st]), (uint32_t)((j / kStages) & 1))) {
                atomicExch(&s_bad, 1);
                break;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a = base + (uint32_t)st * kStage;
            const uint32_t bh = a + Cfg::kBOff, bl = bh + kBTile;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const uint64_t ad = desc_k_sw128(a + (uint32_t)kk * 32u);
                const uint64_t bdh = desc_mn_sw128b32(bh + (uint32_t)kk * 2048u, 512u, 1024u);
                const uint64_t bdl = desc_mn_sw128b32(bl + (uint32_t)kk * 2048u, 512u, 1024u);
                const uint32_t accf = (j > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bdh), "r"(kIdesc), "r"(accf));
                asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;" ::"r"(tmem), "l"(ad), "l"(bdl),
                             "r"(kIdesc));
                if constexpr (SP) {
                    const uint64_t adl = desc_k_sw128(a + Cfg::kALo + (uint32_t)kk * 32u);
                    asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;" ::"r"(tmem), "l"(adl),
                                 "l"(bdh), "r"(kIdesc));
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&empty[st]))
                         : "memory");
            issued = j + 1;
        }
        // Drain: the last commit covers every MMA issued before it (after an
        // expired wait too, so the TMEM is idle before it is freed).
        if (issued > 0) {
            const int last = issued - 1;
            if (!mbar_wait(smem_u32(&empty[last % kStages]), (uint32_t)((last / kStages) & 1))) atomicExch(&s_bad, 1);
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (s_bad) {
        if (tid == 0) atomicExch(err, 1);
    } else if (tid < kProducers) {
        // Epilogue: warp w (0..3) reads TMEM lanes 32w..32w+31 = rows of D.
        const int row = warp * 32 + lane;
        double* dst = row < m ? Y + (tb + row) * R + rc : nullptr;
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 16), v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (dst) {
#pragma unroll
                for (int k = 0; k < 16; k += 2) {
                    const int col = cb * 16 + k;
                    if (rc + col < R)
                        *reinterpret_cast<double2*>(dst + col) =
                            make_double2((double)__uint_as_float(v[k]), (double)__uint_as_float(v[k + 1]));
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 4) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// X32 = (float) x for the FP32 far field, and the split X_hi = tf32(x),
// X_lo = tf32(x - X_hi) (round to nearest) for the tensor-core near apply.
__global__ void k_split_tf32(const double* __restrict__ X, float* __restrict__ X32, float* __restrict__ Xhi,
                             float* __restrict__ Xlo, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = X[i];
        const float hi = to_tf32((float)x);
        X32[i] = (float)x;
        Xhi[i] = hi;
        Xlo[i] = to_tf32((float)(x - (double)hi));
    }
}

__global__ void k_to_tf32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = to_tf32((float)a[i]);
}

}  // namespace

void launch_to_tf32(Ctx& c, const double* a, float* b, int64_t n) {
    if (n == 0) return;
    KTimer t(c, K_VEC, 12.0 * n, 0.0);
    k_to_tf32<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 32), 256, 0, c.stream>>>(a, b, n);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

template <int MODE>
void near_tc_launch(Ctx& c, const DevPlan& p, int nitems, const int32_t* it_leaf, const int32_t* it_row0,
                    const float* P, const float* Xa, const float* Xb, double* Y, int R, int* err) {
    const dim3 grid(nitems, (R + 63) / 64);
    set_smem_once(k_near_apply_tc<MODE>, (int)NearCfg<MODE>::kSmemBytes);
    k_near_apply_tc<MODE><<<grid, kThreads, NearCfg<MODE>::kSmemBytes, c.stream>>>(p, it_leaf, it_row0, P, Xa, Xb, Y,
                                                                                  R, err);
    GPX_LAUNCH_CHECK();
}

void launch_near_apply_tc(Ctx& c, const DevPlan& p, int64_t nnz, int nitems, const int32_t* it_leaf,
                          const int32_t* it_row0, const float* P, const float* Xhi, const float* Xlo, double* Y, int R,
                          int* err, bool split_p) {
    if (nitems == 0) return;
    if (R % 4 != 0) throw Error(GPX_ERR_INTERNAL, "tensor-core near apply needs R a multiple of 4");
    KTimer t(c, K_NEAR_APPLY, 4.0 * nnz + 16.0 * (double)p.N * R, (split_p ? 6.0 : 4.0) * (double)nnz * R);
    if (split_p)
        near_tc_launch<1>(c, p, nitems, it_leaf, it_row0, P, Xhi, Xlo, Y, R, err);
    else if (!Xlo)
        near_tc_launch<2>(c, p, nitems, it_leaf, it_row0, P, Xhi, nullptr, Y, R, err);
    else
        near_tc_launch<0>(c, p, nitems, it_leaf, it_row0, P, Xhi, Xlo, Y, R, err);
    c.launches += 1;
}

void launch_split_tf32(Ctx& c, const double* X, float* X32, float* Xhi, float* Xlo, int64_t n) {
    if (n == 0) return;
    KTimer t(c, K_VEC, 20.0 * n, 0.0);
    k_split_tf32<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16), 256, 0, c.stream>>>(X, X32, Xhi, Xlo, n);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

}  // namespace gpx
