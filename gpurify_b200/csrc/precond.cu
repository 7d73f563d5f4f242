// Leaf block-Jacobi preconditioner.  Blocks are runs of up to KB (48 or 96)
// consecutive panels inside one leaf; each block's matrix is the exact
// (Wilton) self-interaction sub-block of the near field, inverted once by
// Gauss-Jordan elimination with partial pivoting in FP64 and applied as a
// small dense product per block.  The reference uses the diagonal of the same
// near-field block (cap/fmm_solver.rs:133-162); both right preconditioners
// leave the solution of P sigma = b unchanged.
#include <algorithm>
#include <vector>

#include "precond.cuh"

namespace gpx {

namespace {

// One CTA per block: invert A (b x b) read from the leaf's near block.  A and
// its inverse I live in dynamic shared memory (2 x KB x (KB+1) doubles).
template <int kB>
__global__ void __launch_bounds__(256) k_block_invert(DevPlan p, const double* __restrict__ P,
                                                      const int32_t* __restrict__ blk_leaf,
                                                      const int32_t* __restrict__ blk_row0,
                                                      const int32_t* __restrict__ blk_size,
                                                      double* __restrict__ Minv, int* __restrict__ singular) {
    const int bi = blockIdx.x;
    const int t = blk_leaf[bi], r0 = blk_row0[bi], b = blk_size[bi];
    const int Sp = (p.near_S[t] + 3) & ~3;
    const double* Pt = P + p.nval_off[t];
    extern __shared__ double bj_smem[];
    double(*A)[kB + 1] = reinterpret_cast<double(*)[kB + 1]>(bj_smem);
    double(*I)[kB + 1] = reinterpret_cast<double(*)[kB + 1]>(bj_smem + kB * (kB + 1));
    __shared__ int piv;
    __shared__ double pval;
    for (int e = threadIdx.x; e < kB * kB; e += blockDim.x) {
        const int i = e / kB, j = e % kB;
        A[i][j] = (i < b && j < b) ? Pt[(int64_t)(r0 + i) * Sp + r0 + j] : (i == j ? 1.0 : 0.0);
        I[i][j] = i == j ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int k = 0; k < b; ++k) {
        if (threadIdx.x == 0) {
            int best = k;
            double mx = fabs(A[k][k]);
            for (int i = k + 1; i < b; ++i)
                if (fabs(A[i][k]) > mx) {
                    mx = fabs(A[i][k]);
                    best = i;
                }
            piv = best;
            pval = A[best][k];
            if (mx == 0.0) atomicExch(singular, 1);
        }
        __syncthreads();
        if (piv != k)
            for (int j = threadIdx.x; j < kB; j += blockDim.x) {
                double a = A[k][j];
                A[k][j] = A[piv][j];
                A[piv][j] = a;
                double c = I[k][j];
                I[k][j] = I[piv][j];
                I[piv][j] = c;
            }
        __syncthreads();
        const double inv = pval != 0.0 ? 1.0 / pval : 0.0;
        for (int j = threadIdx.x; j < kB; j += blockDim.x) {
            A[k][j] *= inv;
            I[k][j] *= inv;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < kB * kB; e += blockDim.x) {
            const int i = e / kB, j = e % kB;
            if (i != k) {
                const double f = A[i][k];
                if (j != k) A[i][j] -= f * A[k][j];
                I[i][j] -= f * I[k][j];
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < kB; i += blockDim.x)
            if (i != k) A[i][k] = 0.0;
        __syncthreads();
    }
    double* out = Minv + (int64_t)bi * kB * kB;
    for (int e = threadIdx.x; e < kB * kB; e += blockDim.x) out[e] = I[e / kB][e % kB];
}

// One CTA per (block, 64-column chunk): Z[rows] = Minv V[rows].  256
// threads; thread (ty, tx) holds rows ty + 16 a (a < KB/16) and columns
// tx + 16 q (q < 4) in registers, so each shared-memory read feeds several
// multiply-adds.
template <int kB>
__global__ void __launch_bounds__(256) k_block_apply(const double* __restrict__ Minv,
                                                     const int64_t* __restrict__ blk_start,
                                                     const int32_t* __restrict__ blk_size, const double* __restrict__ V,
                                                     DevIndex di, double* __restrict__ Z, int R, int add) {
    constexpr int RA = kB / 16;
    V = dev_offset(V, di);
    const int bi = blockIdx.x;
    const int rc = blockIdx.y * 64;
    const int64_t s0 = blk_start[bi];
    const int b = blk_size[bi];
    extern __shared__ double bj_smem[];
    double(*Ms)[kB + 1] = reinterpret_cast<double(*)[kB + 1]>(bj_smem);
    double(*Vs)[65] = reinterpret_cast<double(*)[65]>(bj_smem + kB * (kB + 1));
    const double* M = Minv + (int64_t)bi * kB * kB;
    for (int e = threadIdx.x; e < kB * kB; e += blockDim.x) Ms[e / kB][e % kB] = M[e];
    for (int e = threadIdx.x; e < kB * 64; e += blockDim.x) {
        const int i = e >> 6, c = e & 63;
        Vs[i][c] = (i < b && rc + c < R) ? V[(s0 + i) * R + rc + c] : 0.0;
    }
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc[RA][4];
#pragma unroll
    for (int a = 0; a < RA; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[a][q] = 0.0;
    for (int k = 0; k < b; ++k) {
        double m[RA], v[4];
#pragma unroll
        for (int a = 0; a < RA; ++a) m[a] = Ms[ty + 16 * a][k];
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = Vs[k][tx + 16 * q];
#pragma unroll
        for (int a = 0; a < RA; ++a)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[a][q] += m[a] * v[q];
    }
#pragma unroll
    for (int a = 0; a < RA; ++a) {
        const int i = ty + 16 * a;
        if (i >= b) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = tx + 16 * q;
            if (rc + c >= R) continue;
            double* z = Z + (s0 + i) * R + rc + c;
            *z = add ? *z + acc[a][q] : acc[a][q];
        }
    }
}

// FP32 form for the inner solves of the mixed path (an approximate inverse
// there anyway): Minv32 rounded once from the FP64 inverses, V read as FP64
// and rounded on load, FP32 products, Z written (or added) as FP64.  One CTA
// per (block, 64-column chunk), thread (ty, tx) holds rows ty + 16 a and
// columns 4 tx .. 4 tx + 3 (so V and Z move as 32-byte rows per thread).
template <int kB>
__global__ void __launch_bounds__(256) k_block_apply32(const float* __restrict__ Minv,
                                                       const int64_t* __restrict__ blk_start,
                                                       const int32_t* __restrict__ blk_size,
                                                       const double* __restrict__ V, DevIndex di,
                                                       double* __restrict__ Z, int R, int add) {
    constexpr int RA = kB / 16;
    V = dev_offset(V, di);
    const int bi = blockIdx.x;
    const int rc = blockIdx.y * 64;
    const int64_t s0 = blk_start[bi];
    const int b = blk_size[bi];
    extern __shared__ float bj32_smem[];
    float(*Ms)[kB + 1] = reinterpret_cast<float(*)[kB + 1]>(bj32_smem);
    float4* Vs = reinterpret_cast<float4*>(bj32_smem + ((kB * (kB + 1) + 3) & ~3));  // [kB][16]
    const float* M = Minv + (int64_t)bi * kB * kB;
    for (int e = threadIdx.x; e < kB * kB; e += blockDim.x) Ms[e / kB][e % kB] = M[e];
    for (int e = threadIdx.x; e < kB * 16; e += blockDim.x) {
        const int i = e >> 4, c = 4 * (e & 15);
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (i < b) {
            const double* src = V + (s0 + i) * R + rc + c;
            if (rc + c + 3 < R) {
                const double2 a = *reinterpret_cast<const double2*>(src);
                const double2 bb = *reinterpret_cast<const double2*>(src + 2);
                v = make_float4((float)a.x, (float)a.y, (float)bb.x, (float)bb.y);
            } else {
                float t[4] = {0.f, 0.f, 0.f, 0.f};
                for (int q = 0; q < 4; ++q)
                    if (rc + c + q < R) t[q] = (float)src[q];
                v = make_float4(t[0], t[1], t[2], t[3]);
            }
        }
        Vs[e] = v;
    }
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[RA][4];
#pragma unroll
    for (int a = 0; a < RA; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[a][q] = 0.f;
    for (int k = 0; k < b; ++k) {
        const float4 v = Vs[k * 16 + tx];
#pragma unroll
        for (int a = 0; a < RA; ++a) {
            const float m = Ms[ty + 16 * a][k];
            acc[a][0] = fmaf(m, v.x, acc[a][0]);
            acc[a][1] = fmaf(m, v.y, acc[a][1]);
            acc[a][2] = fmaf(m, v.z, acc[a][2]);
            acc[a][3] = fmaf(m, v.w, acc[a][3]);
        }
    }
#pragma unroll
    for (int a = 0; a < RA; ++a) {
        const int i = ty + 16 * a;
        if (i >= b) continue;
        const int c = rc + 4 * tx;
        double* z = Z + (s0 + i) * R + c;
        if (c + 3 < R) {
            double2 z0 = make_double2(acc[a][0], acc[a][1]), z1 = make_double2(acc[a][2], acc[a][3]);
            if (add) {
                const double2 o0 = *reinterpret_cast<const double2*>(z), o1 = *reinterpret_cast<const double2*>(z + 2);
                z0.x += o0.x, z0.y += o0.y, z1.x += o1.x, z1.y += o1.y;
            }
            *reinterpret_cast<double2*>(z) = z0;
            *reinterpret_cast<double2*>(z + 2) = z1;
        } else {
            for (int q = 0; q < 4; ++q)
                if (c + q < R) z[q] = add ? z[q] + (double)acc[a][q] : (double)acc[a][q];
        }
    }
}

__global__ void k_round_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

}  // namespace

void BlockJacobi::build(Ctx& c, const Plan& pl, const DevPlan& dp, const double* P) {
    const int kB = block;
    std::vector<int32_t> leaf, row0, size;
    std::vector<int64_t> start;
    for (int64_t k = 0; k + 1 < (int64_t)pl.leaf_begin.size(); ++k) {
        const int64_t m = pl.leaf_begin[k + 1] - pl.leaf_begin[k];
        for (int64_t r = 0; r < m; r += kB) {
            leaf.push_back((int32_t)k);
            row0.push_back((int32_t)r);
            size.push_back((int32_t)std::min<int64_t>(kB, m - r));
            start.push_back(pl.leaf_begin[k] + r);
        }
    }
    nblk = (int)leaf.size();
    d_leaf.upload(leaf, c.stream);
    d_row0.upload(row0, c.stream);
    d_size.upload(size, c.stream);
    d_start.upload(start, c.stream);
    Minv.alloc((size_t)nblk * kB * kB, c.stream);
    d_sing.alloc(1, c.stream);
    d_sing.zero();
    {
        KTimer t(c, K_SMALL, 8.0 * nblk * kB * kB * 2, 2.0 * nblk * (double)kB * kB * kB);
        const int smem = (int)(sizeof(double) * 2 * kB * (kB + 1));
        if (kB == 96) {
            set_smem_once(k_block_invert<96>, smem);
            k_block_invert<96><<<nblk, 256, smem, c.stream>>>(dp, P, d_leaf.p, d_row0.p, d_size.p, Minv.p, d_sing.p);
        } else {
            set_smem_once(k_block_invert<48>, smem);
            k_block_invert<48><<<nblk, 256, smem, c.stream>>>(dp, P, d_leaf.p, d_row0.p, d_size.p, Minv.p, d_sing.p);
        }
        GPX_LAUNCH_CHECK();
        c.launches += 1;
    }
}

void BlockJacobi::make_f32(Ctx& c) {
    const int64_t n = (int64_t)nblk * block * block;
    Minv32.alloc((size_t)n, c.stream);
    KTimer t(c, K_VEC, 12.0 * n, 0.0);
    k_round_f32<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16), 256, 0, c.stream>>>(Minv.p, Minv32.p, n);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void BlockJacobi::apply32(Ctx& c, const double* V, double* Z, int64_t N, int R, bool add, const DevIndex& di) const {
    if (R % 4 != 0) throw Error(GPX_ERR_INTERNAL, "FP32 block-Jacobi apply needs R % 4 == 0");
    const int kB = block;
    KTimer t(c, K_VEC, 16.0 * N * R + 4.0 * (double)nblk * kB * kB, 2.0 * (double)N * kB * R);
    const int smem = (int)(sizeof(float) * (((kB * (kB + 1) + 3) & ~3) + kB * 64));
    const dim3 g(nblk, (R + 63) / 64);
    if (kB == 96) {
        set_smem_once(k_block_apply32<96>, smem);
        k_block_apply32<96><<<g, 256, smem, c.stream>>>(Minv32.p, d_start.p, d_size.p, V, di, Z, R, add ? 1 : 0);
    } else {
        set_smem_once(k_block_apply32<48>, smem);
        k_block_apply32<48><<<g, 256, smem, c.stream>>>(Minv32.p, d_start.p, d_size.p, V, di, Z, R, add ? 1 : 0);
    }
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void BlockJacobi::check(Ctx& c) const {
    int sing = 0;
    d_sing.download(&sing, 1);
    GPX_CUDA(cudaStreamSynchronize(c.stream));
    if (sing) throw Error(GPX_ERR_CAPACITANCE, "singular near-field block in the block-Jacobi preconditioner");
}

void BlockJacobi::apply(Ctx& c, const double* V, double* Z, int64_t N, int R, bool add, const DevIndex& di) const {
    const int kB = block;
    KTimer t(c, K_VEC, 8.0 * (2.0 * N * R + (double)nblk * kB * kB), 2.0 * (double)N * kB * R);
    const int smem = (int)(sizeof(double) * (kB * (kB + 1) + kB * 65));
    const dim3 g(nblk, (R + 63) / 64);
    if (kB == 96) {
        set_smem_once(k_block_apply<96>, smem);
        k_block_apply<96><<<g, 256, smem, c.stream>>>(Minv.p, d_start.p, d_size.p, V, di, Z, R, add ? 1 : 0);
    } else {
        set_smem_once(k_block_apply<48>, smem);
        k_block_apply<48><<<g, 256, smem, c.stream>>>(Minv.p, d_start.p, d_size.p, V, di, Z, R, add ? 1 : 0);
    }
    GPX_LAUNCH_CHECK();
    c.launches += 1;
    (void)N;
}

}  // namespace gpx
