// Compression and decompression of expansions for the mixed path's M2L in a
// shared basis (plan.h SharedBasis): every offset's operator K_o is
// approximated by U C_o V^T with one target basis U and one source basis V
// (n3 x r, r = 64), so M2L runs on compressed expansions:
//     E^[b][r] = V^T E[b][r]          (compress, every source box)
//     L^[t][r] = sum_o C_o E^[t+o][r] (tcgen05 M2L on 64-node rows)
//     L[t][r]  = U L^[t][r]           (decompress, every target box)
// Both transforms are row GEMMs over the (box, right-hand side) rows of the
// expansion buffers,
//     Out[row][col0 + j] = sum_k In[row][k] B[col0 + j][k],
// on the 5th-generation tensor cores (kind::tf32, FP32 accumulation in TMEM).
// The inputs carry large alternating node values where panels' Gauss points
// reach past their leaf, which single TF32 products would not represent, so
// both operands are split into TF32 hi and lo parts and D = A_hi B_hi +
// A_hi B_lo + A_lo B_hi (about 2^-21): B (the basis, K-major, one row per
// output column) is split once per process; A (the expansion rows) is split
// in shared memory once a slice has landed.
// One CTA per (128 rows, 64 output columns): D = 128 x 64 FP32 in TMEM.  The
// contraction runs in slices of 32 through a 2-stage ring: all 128 threads
// copy a slice with cp.async, split their A chunks, and one thread issues the
// slice's MMAs and commits them to the stage's mbarrier, which the copies of
// the slice two ahead wait on (bounded).  The epilogue stores each row's 64
// FP32 values (rows past nrows are neither loaded nor stored).
#include "farfield.cuh"

namespace gpx {

namespace {

constexpr int kThreads = 128;
constexpr uint32_t kATile = 128 * 128;                  // 128 rows x 32 FP32 (128 B)
constexpr uint32_t kBTile = 64 * 128;                   // 64 rows x 32 FP32
constexpr uint32_t kStage = 2 * kATile + 2 * kBTile;    // A_hi, A_lo, B_hi, B_lo: 48 KB
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

// In: nrows x KD (row stride ldi); Bhi / Blo: ncols_pad x KD (row stride KD,
// K-major, zero rows past the real columns); Out: nrows x ldo, columns
// [col0, min(col0 + 64, ncols)) of each row written (ncols a multiple of 4).
template <int KD>
__global__ void __launch_bounds__(kThreads) k_rows_tc(const float* __restrict__ In, int ldi,
                                                      const float* __restrict__ Bhi, const float* __restrict__ Blo,
                                                      int ncols, float* __restrict__ Out, int ldo, int64_t nrows,
                                                      int* __restrict__ err) {
    constexpr int nsl = KD / 32;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* sbase = smem_raw + (base - raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sbase + 2 * kStage);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
    __shared__ int s_bad;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t r0 = (int64_t)blockIdx.x * 128;
    const int col0 = blockIdx.y * 64;
    const int cnt = (int)min((int64_t)128, nrows - r0);
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
    // copies of slice q into stage q % 2: A rows [r0, r0 + cnt) (rows past
    // cnt are not loaded: their D rows are never stored), B rows col0 .. +63
    auto issue = [&](int q) {
        const uint32_t a = base + (uint32_t)(q & 1) * kStage;
        for (int e = tid; e < 128 * 8; e += kThreads) {
            const int row = e >> 3, c = e & 7;
            if (row < cnt) cp16(a + swz(row, c), In + (r0 + row) * (int64_t)ldi + 32 * q + 4 * c, true);
        }
        for (int e = tid; e < 64 * 8; e += kThreads) {
            const int row = e >> 3, c = e & 7;
            const int64_t off = (int64_t)(col0 + row) * KD + 32 * q + 4 * c;
            cp16(a + 2 * kATile + swz(row, c), Bhi + off, true);
            cp16(a + 2 * kATile + kBTile + swz(row, c), Blo + off, true);
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
        // split the A tile of this slice: A_hi in place, A_lo beside it
        {
            uint8_t* at = sbase + (size_t)st * kStage;
            for (int e = tid; e < 128 * 8; e += kThreads) {
                const int row = e >> 3;
                if (row >= cnt) continue;
                const uint32_t o = swz((uint32_t)row, (uint32_t)(e & 7));
                float4* hp = reinterpret_cast<float4*>(at + o);
                float4* lp = reinterpret_cast<float4*>(at + kATile + o);
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
    // freed): the commit of slice q is completion (q >> 1) of bars[q & 1].
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
        float* o = row < cnt ? Out + (r0 + row) * (int64_t)ldo + col0 : nullptr;
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 16), v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (o) {
#pragma unroll
                for (int k = 0; k < 16; k += 4)
                    if (col0 + cb * 16 + k < ncols)
                        *reinterpret_cast<float4*>(o + cb * 16 + k) =
                        make_float4(__uint_as_float(v[k]), __uint_as_float(v[k + 1]), __uint_as_float(v[k + 2]),
                                    __uint_as_float(v[k + 3]));
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// B holds round_up(ncols, 64) rows.
template <int KD>
void launch_rows_tc(Ctx& c, const float* In, int ldi, const float* Bhi, const float* Blo, int ncols, float* Out,
                    int ldo, int64_t nrows, int* err) {
    if (nrows <= 0) return;
    if (ncols % 4 != 0 || ldi % 4 != 0 || ldo % 4 != 0 || ldo < ncols)
        throw Error(GPX_ERR_INTERNAL, "tensor-core row GEMM needs 16-byte rows");
    set_smem_once(k_rows_tc<KD>, (int)kSmemBytes);
    const dim3 grid((unsigned)((nrows + 127) / 128), (unsigned)((ncols + 63) / 64));
    k_rows_tc<KD><<<grid, kThreads, kSmemBytes, c.stream>>>(In, ldi, Bhi, Blo, ncols, Out, ldo, nrows, err);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

}  // namespace

void launch_m2l_compress(Ctx& c, const float* E, int ns, const float* Vt_hi, const float* Vt_lo, float* Eh,
                         int64_t row0, int64_t nrows, int* err) {
    const float* in = E + row0 * ns;
    float* out = Eh + row0 * kShared;
    switch (ns) {
        case 128: launch_rows_tc<128>(c, in, ns, Vt_hi, Vt_lo, kShared, out, kShared, nrows, err); break;
        case 224: launch_rows_tc<224>(c, in, ns, Vt_hi, Vt_lo, kShared, out, kShared, nrows, err); break;
        default: throw Error(GPX_ERR_INTERNAL, "shared-basis compression runs node strides 128 and 224");
    }
}

void launch_m2l_decompress(Ctx& c, const float* Lh, const float* U_hi, const float* U_lo, int ns, float* L,
                           int64_t row0, int64_t nrows, int* err) {
    // every node column of the rows written (zero past n3: U has zero rows there)
    launch_rows_tc<kShared>(c, Lh + row0 * kShared, kShared, U_hi, U_lo, ns, L + row0 * ns, ns, nrows, err);
}

}  // namespace gpx
