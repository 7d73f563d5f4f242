// P2M on the 5th-generation tensor cores for the mixed path (orders 4 and 5,
// node stride 64 or 128):
//     E[leaf][r][m] = sum_j W[j][m] X[j][r]   over the panels j of a work item
// (W the far-field source weights with the panel area folded in).  One CTA per
// (work item of <= 64 panels, 64-wide chunk of right-hand sides); D (M = 128
// nodes, N = 64 right-hand sides, FP32 in TMEM) = A B with
//   A = W^T (nodes x panels): MN-major, one K row per panel = its weight row;
//   B = X (panels x right-hand sides): MN-major, one K row per panel = its X row.
// Both operands come split into TF32 hi and lo parts (weights once per solve,
// X by k_split_tf32 for the near apply), and D = W_hi X_hi + W_hi X_lo +
// W_lo X_hi is accurate to about 2^-21: the weights of panels whose Gauss
// points reach past their leaf carry large alternating values, which single
// TF32 products would not represent.  The whole item (at most two K slices of
// 32 panels) is staged at once; one thread issues the MMAs and commits them
// to an mbarrier (bounded wait).  The epilogue stores D column by column: for
// one right-hand side the 32 lanes of a warp write 32 consecutive nodes.
#include "farfield.cuh"

namespace gpx {

namespace {

constexpr int kThreads = 128;
constexpr int kWS = 128;                     // row stride of the split weight arrays (nodes, zero padded)
constexpr uint32_t kATile = 32 * 128 * 4;    // 32 K rows x 128 nodes
constexpr uint32_t kBTile = 32 * 64 * 4;     // 32 K rows x 64 right-hand sides
constexpr uint32_t kSlice = 2 * kATile + 2 * kBTile;  // A_hi, A_lo, B_hi, B_lo: 48 KB
constexpr uint32_t kSmemBytes = 2 * kSlice + 1024 + 64 + 4096;  // + alignment, barrier/TMEM slot, read slack
constexpr uint32_t kTmemCols = 64;
constexpr int kWaitLimit = 1 << 22;
// Instruction descriptor: D F32, A/B TF32, both MN-major, N = 64, M = 128.
constexpr uint32_t kIdesc =
    (1u << 4) | (2u << 7) | (2u << 10) | (1u << 15) | (1u << 16) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
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

// Byte offset of 16-byte chunk q of K row k in an MN-major tile with `nb`
// 32-wide MN blocks: atom (4-row K group k/4, MN block q/8) at
// (nb (k/4) + q/8) x 512 B, row k%4, 32-byte granule (q%8)/2 swizzled by the row.
__device__ __forceinline__ uint32_t swz_mn(uint32_t k, uint32_t q, uint32_t nb) {
    const uint32_t r = k & 3u;
    return ((k >> 2) * nb + (q >> 3)) * 512u + r * 128u + ((((q & 7u) >> 1) ^ r) << 5) + ((q & 1u) << 4);
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
__global__ void __launch_bounds__(kThreads) k_p2m_tc(DevPlan p, const int32_t* __restrict__ slot,
                                                     const float* __restrict__ Whi, const float* __restrict__ Wlo,
                                                     const float* __restrict__ Xhi, const float* __restrict__ Xlo,
                                                     float* __restrict__ E, int R, int Rb, int* __restrict__ err) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* sbase = smem_raw + (base - raw);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sbase + 2 * kSlice);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
    __shared__ int s_bad;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int it = blockIdx.x;
    const int t = p.item_leaf[it], r0 = p.item_row0[it];
    const int rc = blockIdx.y * 64;
    const int64_t jb = p.leaf_begin[t] + r0;
    const int cnt = (int)min((int64_t)64, p.leaf_begin[t + 1] - jb);
    const int nsl = (cnt + 31) / 32;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_bad = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // A: per slice 32 rows x 32 chunks (hi and lo); nodes past NS are zero
    for (int e = tid; e < nsl * 32 * 32; e += kThreads) {
        const int s = e >> 10, k = (e >> 5) & 31, q = e & 31;
        const int jj = 32 * s + k;
        const bool ok = jj < cnt && 4 * q < NS;
        const int64_t off = ok ? (jb + jj) * kWS + 4 * q : 0;
        const uint32_t d = base + (uint32_t)s * kSlice + swz_mn((uint32_t)k, (uint32_t)q, 4u);
        cp16(d, Whi + off, ok);
        cp16(d + kATile, Wlo + off, ok);
    }
    // B: per slice 32 rows x 16 chunks (hi and lo); right-hand sides past R are zero
    for (int e = tid; e < nsl * 32 * 16; e += kThreads) {
        const int s = e >> 9, k = (e >> 4) & 31, q = e & 15;
        const int jj = 32 * s + k, col = rc + 4 * q;
        const bool ok = jj < cnt && col < R;
        const int64_t off = ok ? (jb + jj) * R + col : 0;
        const uint32_t d = base + (uint32_t)s * kSlice + 2 * kATile + swz_mn((uint32_t)k, (uint32_t)q, 2u);
        cp16(d, Xhi + off, ok);
        cp16(d + kBTile, Xlo + off, ok);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tslot;
    if (tid == 0) {
        for (int s = 0; s < nsl; ++s) {
            const uint32_t ah = base + (uint32_t)s * kSlice, al = ah + kATile;
            const uint32_t bh = ah + 2 * kATile, bl = bh + kBTile;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const uint64_t adh = desc_mn_sw128b32(ah + (uint32_t)kk * 4096u, 512u, 2048u);
                const uint64_t adl = desc_mn_sw128b32(al + (uint32_t)kk * 4096u, 512u, 2048u);
                const uint64_t bdh = desc_mn_sw128b32(bh + (uint32_t)kk * 2048u, 512u, 1024u);
                const uint64_t bdl = desc_mn_sw128b32(bl + (uint32_t)kk * 2048u, 512u, 1024u);
                const uint32_t accf = (s > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(adh), "l"(bdh), "r"(kIdesc), "r"(accf));
                asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;" ::"r"(tmem), "l"(adh),
                             "l"(bdl), "r"(kIdesc));
                asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;" ::"r"(tmem), "l"(adl),
                             "l"(bdh), "r"(kIdesc));
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(bar))
                     : "memory");
    }
    if (!mbar_wait(smem_u32(bar), 0u)) atomicExch(&s_bad, 1);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (s_bad) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        // lane row m = node; columns = right-hand sides rc .. rc + 63
        const int m = warp * 32 + lane;
        const int64_t box = slot[it] < 0 ? (int64_t)p.leaf_box0 + t : (int64_t)p.nbox + slot[it];
        float* out = E + (box * Rb + rc) * NS + m;
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 16), v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < NS) {
#pragma unroll
                for (int k = 0; k < 16; ++k) out[(int64_t)(cb * 16 + k) * NS] = __uint_as_float(v[k]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// Whi / Wlo [N][kWS] = TF32 split of (area if mul_area) x W[N][n3], nodes past n3 zero.
__global__ void k_split_weights(const double* __restrict__ W, int n3, const double* __restrict__ area, int mul_area,
                                float* __restrict__ Whi, float* __restrict__ Wlo, int64_t N) {
    const int64_t n = N * kWS;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = i / kWS;
        const int m = (int)(i % kWS);
        double w = 0.0;
        if (m < n3) w = W[j * n3 + m] * (mul_area ? area[j] : 1.0);
        const float hi = to_tf32((float)w);
        Whi[i] = hi;
        Wlo[i] = to_tf32((float)(w - (double)hi));
    }
}

}  // namespace

void launch_split_weights(Ctx& c, const double* W, int n3, const double* area, bool mul_area, float* Whi, float* Wlo,
                          int64_t N) {
    if (n3 > kWS) throw Error(GPX_ERR_INTERNAL, "split far-field weights take at most 128 nodes");
    const int64_t n = N * kWS;
    KTimer t(c, K_VEC, 16.0 * n, 0.0);
    k_split_weights<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16), 256, 0, c.stream>>>(W, n3, area,
                                                                                                 mul_area ? 1 : 0,
                                                                                                 Whi, Wlo, N);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_p2m_tc(Ctx& c, const DevPlan& p, const int32_t* slot, const float* Whi, const float* Wlo, const float* Xhi,
                   const float* Xlo, float* E, int R, int Rb, int* err) {
    if (p.nitems == 0) return;
    if (R % 4 != 0 || Rb % 64 != 0) throw Error(GPX_ERR_INTERNAL, "tensor-core P2M needs R % 4 == 0, Rb % 64 == 0");
    const dim3 grid(p.nitems, Rb / 64);
    if (p.ns == 128) {
        set_smem_once(k_p2m_tc<128>, (int)kSmemBytes);
        k_p2m_tc<128><<<grid, kThreads, kSmemBytes, c.stream>>>(p, slot, Whi, Wlo, Xhi, Xlo, E, R, Rb, err);
    } else if (p.ns == 64) {
        set_smem_once(k_p2m_tc<64>, (int)kSmemBytes);
        k_p2m_tc<64><<<grid, kThreads, kSmemBytes, c.stream>>>(p, slot, Whi, Wlo, Xhi, Xlo, E, R, Rb, err);
    } else {
        throw Error(GPX_ERR_INTERNAL, "tensor-core P2M runs node strides 64 and 128 (orders 4 and 5)");
    }
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

}  // namespace gpx
