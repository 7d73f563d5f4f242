// Near-field apply on the 5th-generation tensor cores (tcgen05, kind::tf32,
// FP32 accumulation in tensor memory) for the mixed path:
//     Y[rows of item][rc : rc+64] = P_t[rows][0:S] X[near sources of t][rc : rc+64]
// With 64 right-hand sides the near product does 32 flop per streamed FP32
// matrix byte, above what the FP32 CUDA cores sustain per HBM byte, so on the
// CUDA cores it is compute bound; on the tensor cores it is bound by streaming
// the near blocks from HBM.
//
// One CTA per (work item = target leaf and <= 128 of its rows, 64-wide chunk
// of right-hand sides), 128 threads, D = 128 x 64 FP32 in TMEM.  The
// contraction runs over the leaf's S near-source panels in slices of 32:
//   A slice (128 x 32) = P rows, K-major, streamed from HBM with cp.async into
//     a 4-stage ring of 128-byte-swizzled tiles, issued two slices ahead;
//   B slice (64 x 32) = the 32 gathered source rows of X (L2-resident),
//     loaded two slices ahead into registers and written transposed (K-major)
//     into a double buffer as two TF32 tiles, x_hi = tf32(x) and
//     x_lo = tf32(x - x_hi).
// D += A B_hi + A B_lo represents X to about 2^-21, so the operator stays
// linear in X (the GMRES inner solves converge as for any fixed matrix); the
// one approximation left is P rounded once to TF32 (round to nearest, stored
// that way), a fixed perturbation the FP64 refinement removes.
// One thread issues the eight K=8 MMAs of a slice and commits them to the
// stage's mbarrier; a stage or B buffer is refilled only after the MMAs that
// read it completed.  Every mbarrier wait is bounded: on expiry the kernel
// records an error code, drains (bounded) its own MMAs, frees its TMEM and
// returns.
#include "kernels.cuh"

namespace gpx {

namespace {

constexpr int kThreads = 128;
constexpr int kStages = 4;              // A ring; A is issued kStages - 2 slices ahead
constexpr uint32_t kATile = 128 * 128;  // 128 rows x 128 B
constexpr uint32_t kBTile = 64 * 128;   // 64 rows x 128 B
constexpr uint32_t kBBuf = 2 * kBTile;  // hi + lo
constexpr uint32_t kBOff = kStages * kATile;
constexpr uint32_t kSmemBytes = kBOff + 2 * kBBuf + 128 + 1024;  // + barriers, TMEM slot, alignment slack
constexpr uint32_t kTmemCols = 64;
constexpr int kWaitLimit = 1 << 22;
// Instruction descriptor: D F32, A/B TF32, both K-major, N = 64, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: 128 B swizzle, K-major, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Byte offset of 16-byte chunk `chunk` of row `row` in a 128-byte-swizzled tile.
__device__ __forceinline__ uint32_t swz(uint32_t row, uint32_t chunk) {
    return (row >> 3) * 1024u + (row & 7u) * 128u + ((chunk ^ (row & 7u)) << 4);
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

__global__ void __launch_bounds__(kThreads) k_near_apply_tc(DevPlan p, const int32_t* __restrict__ it_leaf,
                                                            const int32_t* __restrict__ it_row0,
                                                            const float* __restrict__ P, const float* __restrict__ X,
                                                            double* __restrict__ Y, int R, int* __restrict__ err) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* sbase = smem_raw + (base - raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sbase + kBOff + 2 * kBBuf);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + kStages);
    __shared__ int64_t s_beg[28];
    __shared__ int32_t s_pre[29];
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
        for (int st = 0; st < kStages; ++st)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[st])));
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

    // A: 1024 16-byte chunks per slice, 8 per thread.
    auto issue_a = [&](int j) {
        if (j < nsl) {
            const uint32_t a = base + (uint32_t)(j % kStages) * kATile;
            const int k0 = j * 32;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int id = tid + kThreads * q, row = id >> 3, c16 = id & 7;
                const bool ok = row < m && k0 + 4 * c16 < Sp;
                cp16(a + swz(row, c16), ok ? (const void*)(Pi + (int64_t)row * Sp + k0 + 4 * c16) : (const void*)P, ok);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // B: 32 panels x 16 quads of right-hand sides per slice; this thread's
    // panels are kk = (lane >> 1) + 16 h, its quads c4 = 2 (2 warp + g) + (lane & 1).
    int ep[2] = {0, 0};
    auto load_b = [&](int j, float4 (&v)[4]) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int k = j * 32 + (lane >> 1) + 16 * h;
            int64_t gid = -1;
            if (j < nsl && k < S) {
                while (s_pre[ep[h] + 1] <= k) ++ep[h];
                gid = s_beg[ep[h]] + (k - s_pre[ep[h]]);
            }
#pragma unroll
            for (int g = 0; g < 2; ++g) {
                const int c4 = 2 * (2 * warp + g) + (lane & 1);
                const int col = rc + 4 * c4;
                float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
                if (gid >= 0 && col < R) x = *reinterpret_cast<const float4*>(X + gid * R + col);
                v[2 * h + g] = x;
            }
        }
    };
    auto store_b = [&](int j, const float4 (&v)[4]) {
        uint8_t* b = sbase + kBOff + (size_t)(j & 1) * kBBuf;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int kk = (lane >> 1) + 16 * h;
#pragma unroll
            for (int g = 0; g < 2; ++g) {
                const int c4 = 2 * (2 * warp + g) + (lane & 1);
                const float4 x = v[2 * h + g];
                const float e[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const uint32_t off = swz(4 * c4 + i, kk >> 2) + (kk & 3) * 4;
                    const float hi = to_tf32(e[i]);
                    *reinterpret_cast<float*>(b + off) = hi;
                    *reinterpret_cast<float*>(b + kBTile + off) = to_tf32(e[i] - hi);
                }
            }
        }
    };

    bool bad = false;
    int issued = 0;  // slices whose MMAs were committed
    float4 breg[2][4];
    for (int j = 0; j < kStages - 2; ++j) issue_a(j);
    load_b(0, breg[0]);
    load_b(1, breg[1]);
    for (int j = 0; j < nsl; ++j) {
        if (j >= 2) {
            const bool ok = mbar_wait(smem_u32(&bars[(j - 2) % kStages]), (uint32_t)(((j - 2) / kStages) & 1));
            if (__syncthreads_or(!ok)) {
                bad = true;
                break;
            }
        }
        issue_a(j + kStages - 2);
        if (j & 1) {
            store_b(j, breg[1]);
            load_b(j + 2, breg[1]);
        } else {
            store_b(j, breg[0]);
            load_b(j + 2, breg[0]);
        }
        asm volatile("cp.async.wait_group %0;" ::"n"(kStages - 2) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t abase = base + (uint32_t)(j % kStages) * kATile;
            const uint32_t bbase = base + kBOff + (uint32_t)(j & 1) * kBBuf;
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                const uint64_t ad = desc_sw128(abase + (uint32_t)(s >> 1) * 32u);
                const uint64_t bd = desc_sw128(bbase + (uint32_t)(s & 1) * kBTile + (uint32_t)(s >> 1) * 32u);
                const uint32_t accf = (j > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(kIdesc), "r"(accf));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bars[j % kStages]))
                         : "memory");
        }
        issued = j + 1;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    // Drain: the last commit covers every MMA issued before it (after an
    // expired wait too, so the TMEM is idle before it is freed).
    if (issued > 0) {
        const int last = issued - 1;
        const bool ok = mbar_wait(smem_u32(&bars[last % kStages]), (uint32_t)((last / kStages) & 1));
        if (__syncthreads_or(!ok)) bad = true;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (bad) {
        if (tid == 0) atomicExch(err, 1);
    } else {
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
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
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

void launch_near_apply_tc(Ctx& c, const DevPlan& p, int64_t nnz, int nitems, const int32_t* it_leaf,
                          const int32_t* it_row0, const float* P, const float* X, double* Y, int R, int* err) {
    if (nitems == 0) return;
    if (R % 4 != 0) throw Error(GPX_ERR_INTERNAL, "tensor-core near apply needs R a multiple of 4");
    KTimer t(c, K_NEAR_APPLY, 4.0 * nnz + 12.0 * (double)p.N * R, 2.0 * (double)nnz * R);
    set_smem_once(k_near_apply_tc, (int)kSmemBytes);
    k_near_apply_tc<<<dim3(nitems, (R + 63) / 64), kThreads, kSmemBytes, c.stream>>>(p, it_leaf, it_row0, P, X, Y, R,
                                                                                     err);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

}  // namespace gpx
