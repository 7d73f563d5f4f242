// Compression and decompression of expansions for the mixed path's M2L in a
// shared basis (plan.h SharedBasis): every offset's operator K_o is
// approximated by U C_o V^T with one target basis U and one source basis V
// (n3 x r, r = 64), so M2L runs on compressed expansions:
//     E^[b][r] = V^T E[b][r]          (compress, every source box)
//     L^[t][r] = sum_o C_o E^[t+o][r] (tcgen05 M2L on 64-node rows)
//     L[t][r]  = U L^[t][r]           (decompress, every target box)
// Both transforms are row GEMMs Out[rows][64-col tile] = In[rows][KD] B[KD][..]
// over the (box, right-hand side) rows of the expansion buffers, in FP32 on
// the CUDA cores (the expansions of panels whose Gauss points reach past their
// leaf carry large alternating node values, which TF32 inputs would not
// represent), so the only TF32 rounding left in the far field is the M2L's.
#include "farfield.cuh"

namespace gpx {

namespace {

constexpr int kRowsPerCta = 128;
constexpr int kColsPerCta = 64;
constexpr int kKC = 32;        // contraction chunk
constexpr int kAPad = 132;     // row stride of the transposed A chunk (16-byte aligned, bank-spread)

// Out[row][col0 + j] = sum_k In[row][k] B[k][col0 + j], rows [0, nrows),
// columns col0 + j < ncols (j < 64); In row stride ldi, Out row stride ldo, B
// is KD x ldb with ldb a multiple of 64 (columns past ncols zero).  256
// threads: thread (ty, tx) computes rows 8 ty .. 8 ty + 7, columns
// 4 tx .. 4 tx + 3 of the CTA's 128 x 64 tile.  Dynamic shared memory: the
// CTA's 64-column slice of B, then the transposed A chunk.
template <int KD>
constexpr int rows_gemm_smem() {
    return (KD * kColsPerCta + kKC * kAPad) * (int)sizeof(float);
}

template <int KD>
__global__ void __launch_bounds__(256) k_rows_gemm64(const float* __restrict__ In, int ldi,
                                                      const float* __restrict__ B, int ldb, int ncols,
                                                      float* __restrict__ Out, int ldo, int64_t nrows) {
    extern __shared__ __align__(16) float rg_smem[];
    float(*Bs)[kColsPerCta] = reinterpret_cast<float(*)[kColsPerCta]>(rg_smem);
    float(*As)[kAPad] = reinterpret_cast<float(*)[kAPad]>(rg_smem + KD * kColsPerCta);
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int64_t r0 = (int64_t)blockIdx.x * kRowsPerCta;
    const int col0 = blockIdx.y * kColsPerCta;
    for (int i = tid; i < KD * (kColsPerCta / 4); i += 256) {
        const int k = i / (kColsPerCta / 4), c4 = i % (kColsPerCta / 4);
        *reinterpret_cast<float4*>(&Bs[k][4 * c4]) =
            *reinterpret_cast<const float4*>(B + (int64_t)k * ldb + col0 + 4 * c4);
    }
    float acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    // A chunk loader: row lr = tid / 2 (0..127), 16 of the 32 chunk values
    const int lr = tid >> 1, lh = (tid & 1) * 16;
    const int64_t grow = r0 + lr;
    const bool rok = grow < nrows;
    const float* arow = In + (rok ? grow : 0) * (int64_t)ldi;
    for (int kc = 0; kc < KD; kc += kKC) {
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (rok) v = *reinterpret_cast<const float4*>(arow + kc + lh + 4 * q);
            As[lh + 4 * q + 0][lr] = v.x;
            As[lh + 4 * q + 1][lr] = v.y;
            As[lh + 4 * q + 2][lr] = v.z;
            As[lh + 4 * q + 3][lr] = v.w;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < kKC; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4*>(&As[kk][8 * ty]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[kk][8 * ty + 4]);
            const float4 b = *reinterpret_cast<const float4*>(&Bs[kc + kk][4 * tx]);
            const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bb[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], bb[j], acc[i][j]);
        }
    }
    const int col = col0 + 4 * tx;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int64_t row = r0 + 8 * ty + i;
        if (row < nrows && col < ncols)
            *reinterpret_cast<float4*>(Out + row * (int64_t)ldo + col) =
                make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
    }
}

template <int KD>
void launch_rows_gemm64(Ctx& c, const float* In, int ldi, const float* B, int ldb, int ncols, float* Out, int ldo,
                        int64_t nrows) {
    if (nrows <= 0) return;
    if (ldb % 64 != 0 || ncols % 4 != 0 || ncols > ldb || ldi % 4 != 0 || ldo % 4 != 0)
        throw Error(GPX_ERR_INTERNAL, "row GEMM needs 16-byte rows and a B stride padded to 64 columns");
    constexpr int smem = rows_gemm_smem<KD>();
    set_smem_once(k_rows_gemm64<KD>, smem);
    const dim3 grid((unsigned)((nrows + kRowsPerCta - 1) / kRowsPerCta), (unsigned)((ncols + 63) / 64));
    k_rows_gemm64<KD><<<grid, 256, smem, c.stream>>>(In, ldi, B, ldb, ncols, Out, ldo, nrows);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

}  // namespace

void launch_m2l_compress(Ctx& c, const float* E, int ns, const float* Vpad, float* Eh, int64_t row0, int64_t nrows) {
    const float* in = E + row0 * ns;
    float* out = Eh + row0 * kShared;
    switch (ns) {
        case 64: launch_rows_gemm64<64>(c, in, ns, Vpad, kShared, kShared, out, kShared, nrows); break;
        case 128: launch_rows_gemm64<128>(c, in, ns, Vpad, kShared, kShared, out, kShared, nrows); break;
        case 224: launch_rows_gemm64<224>(c, in, ns, Vpad, kShared, kShared, out, kShared, nrows); break;
        default: throw Error(GPX_ERR_INTERNAL, "shared-basis compression runs node strides 64, 128 and 224");
    }
}

void launch_m2l_decompress(Ctx& c, const float* Lh, const float* Utpad, int ns, float* L, int64_t row0,
                           int64_t nrows) {
    launch_rows_gemm64<kShared>(c, Lh + row0 * kShared, kShared, Utpad, (ns + 63) / 64 * 64, ns, L + row0 * ns, ns,
                                nrows);
}

}  // namespace gpx
