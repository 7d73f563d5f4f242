// Multi-RHS restarted GMRES building blocks (FP64).  Vectors are N x R
// row-major (panel-major, one column per right-hand side) so a row of R values
// is one coalesced load.  All reductions are two-stage with a fixed block
// partition and a fixed summation order, so results are bit-reproducible.
#include <algorithm>

#include "gpx_common.h"
#include "krylov.cuh"

namespace gpx {

namespace {

constexpr int kRedThreads = 256;

// partial[b][i][r] = sum over rows of block b of A_i[n][r] * B[n][r].
// Eight vectors A_i per pass over the block's rows: B is read once per eight,
// and each thread keeps eight independent loads in flight per row.  Each
// partial sums the same rows in the same order as a one-vector pass.
template <class TA>
__global__ void __launch_bounds__(kRedThreads) k_multidot(const TA* __restrict__ A, int64_t strideA, int ni,
                                                          const int32_t* __restrict__ kdev,
                                                          const double* __restrict__ B, int64_t N, int R,
                                                          double* __restrict__ partial) {
    constexpr int kV = 8;
    if (kdev) ni = *kdev + 1;
    const int nsub = kRedThreads / R;
    const int r = threadIdx.x % R, sub = threadIdx.x / R;
    const int64_t per = (N + gridDim.x - 1) / gridDim.x;
    const int64_t n0 = (int64_t)blockIdx.x * per, n1 = min(N, n0 + per);
    __shared__ double red[kV][kRedThreads];
    for (int i0 = 0; i0 < ni; i0 += kV) {
        const int nv = min(kV, ni - i0);
        const TA* A0 = A + i0 * strideA;
        double acc[kV];
#pragma unroll
        for (int q = 0; q < kV; ++q) acc[q] = 0.0;
        if (sub < nsub) {
            if (nv == kV) {
#pragma unroll 2
                for (int64_t n = n0 + sub; n < n1; n += nsub) {
                    const int64_t o = n * R + r;
                    const double b = B[o];
#pragma unroll
                    for (int q = 0; q < kV; ++q) acc[q] += (double)A0[q * strideA + o] * b;
                }
            } else {
                // The last chunk of fewer than eight vectors (and the column
                // norms, one vector): fully unrolled and predicated, so the
                // accumulators stay in registers and the loads of a row issue
                // together.  Same rows, same order as the loop over nv.
#pragma unroll 2
                for (int64_t n = n0 + sub; n < n1; n += nsub) {
                    const int64_t o = n * R + r;
                    const double b = B[o];
#pragma unroll
                    for (int q = 0; q < kV; ++q)
                        if (q < nv) acc[q] += (double)A0[q * strideA + o] * b;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kV; ++q) red[q][threadIdx.x] = acc[q];
        __syncthreads();
        if (sub == 0)
            for (int q = 0; q < nv; ++q) {
                double s = red[q][r];
                for (int k = 1; k < nsub; ++k) s += red[q][k * R + r];
                partial[((int64_t)blockIdx.x * ni + i0 + q) * R + r] = s;
            }
        __syncthreads();
    }
}

// out[i][r] (+)= sum_b partial[b][i][r]; one warp per (i, r): lane l sums
// blocks l, l + 32, ... and the lanes combine in a fixed shuffle tree.
__global__ void k_reduce_blocks(const double* __restrict__ partial, int nblk, int ni, const int32_t* __restrict__ kdev,
                                int R, double* __restrict__ out, int accumulate) {
    if (kdev) ni = *kdev + 1;
    const int o = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (o >= ni * R) return;
    const int64_t stride = (int64_t)ni * R;
    double s = 0.0;
    for (int b = lane; b < nblk; b += 32) s += partial[b * stride + o];
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
    if (lane == 0) out[o] = accumulate ? out[o] + s : s;
}

// W[n][r] -= sum_{i<ni} h[i][r] * V_i[n][r]
template <class TV>
__global__ void k_multi_axpy(const TV* __restrict__ V, int64_t strideV, int ni, const int32_t* __restrict__ kdev,
                             const double* __restrict__ h, double* __restrict__ W, int64_t N, int R) {
    if (kdev) ni = *kdev + 1;
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= N * R) return;
    const int r = (int)(o % R);
    double w = W[o];
    for (int i = 0; i < ni; ++i) w -= h[i * R + r] * (double)V[i * strideV + o];
    W[o] = w;
}

// dst[n][r] = src[n][r] / s[r] when s[r] > thresh, else src (Arnoldi
// normalisation with the reference's happy-breakdown rule, krylov.rs:111-115);
// with `cur` the FP64 value also goes there (the FP32 basis keeps its newest
// vector in FP64 for the next step's preconditioner).
template <class TD>
__global__ void k_scale_cols(const double* __restrict__ src, const double* __restrict__ s, double thresh,
                             TD* __restrict__ dst, DevIndex di, double* __restrict__ cur, int64_t N, int R) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= N * R) return;
    dst = dev_offset(dst, di);
    const double d = s[o % R];
    const double v = d > thresh ? src[o] / d : src[o];
    dst[o] = (TD)v;
    if (cur) cur[o] = v;
}

__global__ void k_sqrt(double* v, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = sqrt(v[i]);
}

// Z[n][r] (+)= inv_diag[n] * V[n][r]
__global__ void k_diag_scale(const double* __restrict__ V, DevIndex di, const double* __restrict__ d,
                             double* __restrict__ Z, int64_t N, int R, int add) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= N * R) return;
    V = dev_offset(V, di);
    const double z = V[o] * d[o / R];
    Z[o] = add ? Z[o] + z : z;
}

// out[n][r] = sum_i y[i][r] V_i[n][r]
template <class TV>
__global__ void k_lincomb(const TV* __restrict__ V, int64_t strideV, int ni, const double* __restrict__ y,
                          double* __restrict__ out, int64_t N, int R) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= N * R) return;
    const int r = (int)(o % R);
    double s = 0.0;
    for (int i = 0; i < ni; ++i) s += y[i * R + r] * (double)V[i * strideV + o];
    out[o] = s;
}

// Res[n][r] = b[n][r] - AX[n][r], b the unit-conductor right-hand side
// (cap/solver.rs:55-63): 1 on the panels of conductor rhs_cond[r].
__global__ void k_residual(const int32_t* __restrict__ cond, const int32_t* __restrict__ rhs_cond,
                           const double* __restrict__ AX, double* __restrict__ Res, int64_t N, int R) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= N * R) return;
    const double b = cond[o / R] == rhs_cond[o % R] ? 1.0 : 0.0;
    Res[o] = AX ? b - AX[o] : b;
}

// Res = B - AX; X += D; zero the columns of V whose mask is set.
__global__ void k_sub(const double* __restrict__ B, const double* __restrict__ AX, double* __restrict__ Res,
                      int64_t n) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o < n) Res[o] = B[o] - AX[o];
}
__global__ void k_add(double* __restrict__ X, const double* __restrict__ D, int64_t n) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o < n) X[o] += D[o];
}
__global__ void k_zero_cols(double* __restrict__ V, const int32_t* __restrict__ mask, int64_t N, int R) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o < N * R && mask[o % R]) V[o] = 0.0;
}

// Per-column Hessenberg column k update, Givens rotation (krylov.rs:118-142,
// :195-207), residual estimate and freeze of converged columns.
__global__ void k_givens(GmresDev g, int k, const int32_t* __restrict__ kdev) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= g.R) return;
    if (kdev) k = *kdev;
    const int m = g.m, R = g.R;
    if (!g.act[r]) return;
    double* H = g.H;  // H[(i*m + k)*R + r]
    auto h = [&](int i) -> double& { return H[((int64_t)i * m + k) * R + r]; };
    // Apply the earlier rotations to the new column.  Only the running entry
    // is carried from one rotation to the next (in a register); the loads of
    // each step do not depend on the previous one, so they overlap.
    double cur = g.h1[r] + g.h2[r];
#pragma unroll 4
    for (int i = 0; i < k; ++i) {
        const double cs = g.cs[i * R + r], sn = g.sn[i * R + r];
        const double nx = g.h1[(i + 1) * R + r] + g.h2[(i + 1) * R + r];
        h(i) = cs * cur + sn * nx;
        cur = -sn * cur + cs * nx;
    }
    const double a = cur, b = g.hnorm[r];
    double c, s;
    if (b == 0.0) {
        c = 1.0;
        s = 0.0;
    } else if (fabs(b) > fabs(a)) {
        const double t = a / b;
        s = 1.0 / sqrt(1.0 + t * t);
        c = t * s;
    } else {
        const double t = b / a;
        c = 1.0 / sqrt(1.0 + t * t);
        s = t * c;
    }
    g.cs[k * R + r] = c;
    g.sn[k * R + r] = s;
    h(k) = c * a + s * b;
    h(k + 1) = 0.0;
    const double gk = g.g[k * R + r], gk1 = g.g[(k + 1) * R + r];
    g.g[k * R + r] = c * gk + s * gk1;
    g.g[(k + 1) * R + r] = -s * gk + c * gk1;
    g.kused[r] = k + 1;
    const double est = fabs(g.g[(k + 1) * R + r]) / g.bnorm[r];
    g.est[r] = est;
    if (est <= g.tol) g.act[r] = 0;
}

// Back substitution H y = g per column (krylov.rs:144-152); y[i][r].
__global__ void k_trisolve(GmresDev g) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= g.R) return;
    const int m = g.m, R = g.R, ku = g.done[r] ? 0 : g.kused[r];
    for (int i = 0; i < m; ++i) g.y[i * R + r] = 0.0;
    for (int i = ku - 1; i >= 0; --i) {
        double sum = g.g[i * R + r];
        for (int j = i + 1; j < ku; ++j) sum -= g.H[((int64_t)i * m + j) * R + r] * g.y[j * R + r];
        g.y[i * R + r] = sum / g.H[((int64_t)i * m + i) * R + r];
    }
}

// Start of a cycle: beta = ||res||, converged-at-start test, V_0 = res/beta,
// g = (beta, 0, ...), activity flags.
__global__ void k_cycle_start(GmresDev g, const double* __restrict__ beta) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= g.R) return;
    const double b = beta[r];
    const double rel = b / g.bnorm[r];
    g.resid[r] = rel;
    if (rel <= g.tol) g.done[r] = 1;
    g.act[r] = g.done[r] ? 0 : 1;
    g.kused[r] = 0;
    for (int i = 0; i <= g.m; ++i) g.g[i * g.R + r] = 0.0;
    g.g[r] = b;
    g.bcur[r] = g.done[r] ? 0.0 : b;
}

// End of a cycle: true residual check of columns whose estimate is within
// 10x of the tolerance (krylov.rs:170-181).
__global__ void k_cycle_end(GmresDev g, const double* __restrict__ rnorm) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= g.R) return;
    if (g.done[r]) return;
    const double rel = rnorm[r] / g.bnorm[r];
    g.resid[r] = rel;
    const int ku = g.kused[r];
    const double est = ku > 0 ? fabs(g.g[ku * g.R + r]) / g.bnorm[r] : rel;
    if (est <= g.tol * 10.0 && rel <= g.tol) g.done[r] = 1;
}

__global__ void k_count_active(const int32_t* act, int R, int32_t* out) {
    int c = 0;
    for (int r = threadIdx.x; r < R; r += blockDim.x) c += act[r] != 0;
    __shared__ int red[256];
    red[threadIdx.x] = c;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// Control of the device-side Arnoldi loop (one CTA of 256 threads): with
// `advance`, one more iteration has completed (*kdev += 1); the loop goes on
// while a column is still active and fewer than m iterations ran.
__global__ void k_loop_ctl(cudaGraphConditionalHandle h, const int32_t* __restrict__ act, int R,
                           int32_t* __restrict__ kdev, int m, int advance) {
    int c = 0;
    for (int r = threadIdx.x; r < R; r += blockDim.x) c += act[r] != 0;
    __shared__ int red[256];
    red[threadIdx.x] = c;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int k = *kdev + (advance ? 1 : 0);
        *kdev = k;
        cudaGraphSetConditional(h, (red[0] > 0 && k < m) ? 1u : 0u);
    }
}

__global__ void k_zero_words(float4* __restrict__ p, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

int reduce_blocks_for(int64_t N) { return (int)std::min<int64_t>(592, std::max<int64_t>(1, N / 64)); }

template <class TA>
void multidot_t(Ctx& c, const TA* A, int64_t strideA, int ni, const double* B, int64_t N, int R, double* partial,
                int nblk, double* out, int accumulate, int tag, const int32_t* kdev) {
    // with kdev the vector count is *kdev + 1 <= ni, read on the device
    {
        KTimer t(c, tag, ((double)sizeof(TA) * ni + 8.0) * (double)N * R, 2.0 * ni * (double)N * R);
        k_multidot<<<nblk, kRedThreads, 0, c.stream>>>(A, strideA, ni, kdev, B, N, R, partial);
        GPX_LAUNCH_CHECK();
    }
    {
        KTimer t(c, K_SMALL);
        k_reduce_blocks<<<blocks_for((int64_t)ni * R, 8), 256, 0, c.stream>>>(partial, nblk, ni, kdev, R, out,
                                                                              accumulate);
        GPX_LAUNCH_CHECK();
    }
    c.launches += 2;
}

void launch_multidot(Ctx& c, const double* A, int64_t strideA, int ni, const double* B, int64_t N, int R,
                     double* partial, int nblk, double* out, int accumulate, int tag, const int32_t* kdev) {
    multidot_t(c, A, strideA, ni, B, N, R, partial, nblk, out, accumulate, tag, kdev);
}

void launch_multidot(Ctx& c, const float* A, int64_t strideA, int ni, const double* B, int64_t N, int R,
                     double* partial, int nblk, double* out, int accumulate, int tag, const int32_t* kdev) {
    multidot_t(c, A, strideA, ni, B, N, R, partial, nblk, out, accumulate, tag, kdev);
}

void launch_colnorm(Ctx& c, const double* A, int64_t N, int R, double* partial, int nblk, double* out) {
    launch_multidot(c, A, 0, 1, A, N, R, partial, nblk, out, 0, K_VEC);
    KTimer t(c, K_SMALL);
    k_sqrt<<<blocks_for(R, 128), 128, 0, c.stream>>>(out, R);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

template <class TV>
void multi_axpy_t(Ctx& c, const TV* V, int64_t strideV, int ni, const double* h, double* W, int64_t N, int R,
                  const int32_t* kdev) {
    KTimer t(c, K_GS_AXPY, ((double)sizeof(TV) * ni + 16.0) * (double)N * R, 2.0 * ni * (double)N * R);
    k_multi_axpy<<<blocks_for(N * R, 256), 256, 0, c.stream>>>(V, strideV, ni, kdev, h, W, N, R);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_multi_axpy(Ctx& c, const double* V, int64_t strideV, int ni, const double* h, double* W, int64_t N, int R,
                      const int32_t* kdev) {
    multi_axpy_t(c, V, strideV, ni, h, W, N, R, kdev);
}

void launch_multi_axpy(Ctx& c, const float* V, int64_t strideV, int ni, const double* h, double* W, int64_t N, int R,
                      const int32_t* kdev) {
    multi_axpy_t(c, V, strideV, ni, h, W, N, R, kdev);
}

void launch_scale_cols(Ctx& c, const double* src, const double* sc, double thresh, double* dst, int64_t N, int R,
                       const DevIndex& di) {
    KTimer t(c, K_VEC, 16.0 * (double)N * R, (double)N * R);
    k_scale_cols<<<blocks_for(N * R, 256), 256, 0, c.stream>>>(src, sc, thresh, dst, di, (double*)nullptr, N, R);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_scale_cols(Ctx& c, const double* src, const double* sc, double thresh, float* dst, double* cur, int64_t N,
                       int R, const DevIndex& di) {
    KTimer t(c, K_VEC, 20.0 * (double)N * R, (double)N * R);
    k_scale_cols<<<blocks_for(N * R, 256), 256, 0, c.stream>>>(src, sc, thresh, dst, di, cur, N, R);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

template <class TV>
void lincomb_t(Ctx& c, const TV* V, int64_t strideV, int ni, const double* y, double* out, int64_t N, int R) {
    KTimer t(c, K_VEC, ((double)sizeof(TV) * ni + 8.0) * (double)N * R, 2.0 * ni * (double)N * R);
    k_lincomb<<<blocks_for(N * R, 256), 256, 0, c.stream>>>(V, strideV, ni, y, out, N, R);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_lincomb(Ctx& c, const double* V, int64_t strideV, int ni, const double* y, double* out, int64_t N,
                    int R) {
    lincomb_t(c, V, strideV, ni, y, out, N, R);
}

void launch_lincomb(Ctx& c, const float* V, int64_t strideV, int ni, const double* y, double* out, int64_t N, int R) {
    lincomb_t(c, V, strideV, ni, y, out, N, R);
}

void launch_diag_scale(Ctx& c, const double* V, const double* d, double* Z, int64_t N, int R, bool add,
                       const DevIndex& di) {
    KTimer t(c, K_VEC, 16.0 * (double)N * R + 8.0 * N, (double)N * R);
    k_diag_scale<<<blocks_for(N * R, 256), 256, 0, c.stream>>>(V, di, d, Z, N, R, add ? 1 : 0);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_residual(Ctx& c, const int32_t* cond, const int32_t* rhs_cond, const double* AX, double* Res, int64_t N,
                     int R) {
    KTimer t(c, K_VEC, (AX ? 16.0 : 8.0) * (double)N * R + 4.0 * N, (double)N * R);
    k_residual<<<blocks_for(N * R, 256), 256, 0, c.stream>>>(cond, rhs_cond, AX, Res, N, R);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_sub(Ctx& c, const double* B, const double* AX, double* Res, int64_t n) {
    KTimer t(c, K_VEC, 24.0 * n, (double)n);
    k_sub<<<blocks_for(n, 256), 256, 0, c.stream>>>(B, AX, Res, n);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_add(Ctx& c, double* X, const double* D, int64_t n) {
    KTimer t(c, K_VEC, 24.0 * n, (double)n);
    k_add<<<blocks_for(n, 256), 256, 0, c.stream>>>(X, D, n);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_zero_cols(Ctx& c, double* V, const int32_t* mask, int64_t N, int R) {
    KTimer t(c, K_VEC, 8.0 * N * R, 0.0);
    k_zero_cols<<<blocks_for(N * R, 256), 256, 0, c.stream>>>(V, mask, N, R);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_givens(Ctx& c, const GmresDev& g, int k, const int32_t* kdev) {
    KTimer t(c, K_SMALL);
    k_givens<<<blocks_for(g.R, 64), 64, 0, c.stream>>>(g, k, kdev);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_trisolve(Ctx& c, const GmresDev& g) {
    KTimer t(c, K_SMALL);
    k_trisolve<<<blocks_for(g.R, 64), 64, 0, c.stream>>>(g);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_cycle_start(Ctx& c, const GmresDev& g, const double* beta) {
    KTimer t(c, K_SMALL);
    k_cycle_start<<<blocks_for(g.R, 64), 64, 0, c.stream>>>(g, beta);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_cycle_end(Ctx& c, const GmresDev& g, const double* rnorm) {
    KTimer t(c, K_SMALL);
    k_cycle_end<<<blocks_for(g.R, 64), 64, 0, c.stream>>>(g, rnorm);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_loop_ctl(Ctx& c, cudaGraphConditionalHandle h, const int32_t* act, int R, int32_t* kdev, int m,
                     bool advance) {
    KTimer t(c, K_SMALL);
    k_loop_ctl<<<1, 256, 0, c.stream>>>(h, act, R, kdev, m, advance ? 1 : 0);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_zero(Ctx& c, void* p, size_t bytes) {
    if (bytes == 0) return;
    if (bytes % 16 != 0 || reinterpret_cast<uintptr_t>(p) % 16 != 0)
        throw Error(GPX_ERR_INTERNAL, "launch_zero needs 16-byte aligned, 16-byte multiple buffers");
    const int64_t n = (int64_t)(bytes / 16);
    KTimer t(c, K_VEC, (double)bytes, 0.0);
    k_zero_words<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16), 256, 0, c.stream>>>(
        reinterpret_cast<float4*>(p), n);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_count_active(Ctx& c, const int32_t* act, int R, int32_t* out) {
    KTimer t(c, K_SMALL);
    k_count_active<<<1, 256, 0, c.stream>>>(act, R, out);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

}  // namespace gpx
