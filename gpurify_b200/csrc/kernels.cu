// FP64 kernels of the potential-coefficient operator.
//
//  * near-field assembly: closed-form Wilton integral of 1/|p - r'| over each
//    source panel (integrals/panel.rs:147-208), one CTA per target leaf, one
//    warp per group of target rows, lanes over source panels staged in shared
//    memory (source geometry is prepared once per lane and reused across rows);
//  * near-field apply: dense leaf blocks times R right-hand sides, source
//    columns of X staged in shared memory, block rows broadcast by shuffle;
//  * far field: Chebyshev P2M, M2M, M2L, L2L, L2P (fmm/bbfmm.rs:209-448).
#include <algorithm>

#include "gpx_common.h"
#include "kernels.cuh"
#include "wilton.cuh"

namespace gpx {

namespace {

constexpr int kAsmThreads = 256;
constexpr int kAsmTile = 64;

// One CTA per work item (target leaf, <= 64 rows): rows of the leaf's
// P block m_t x S_t, row-major.
__global__ void __launch_bounds__(kAsmThreads, 2) k_near_assemble(DevPlan p, double* __restrict__ P, double coef) {
    const int t = p.item_leaf[blockIdx.x];
    const int r0 = p.item_row0[blockIdx.x];
    const int64_t tb = p.leaf_begin[t];
    const int m = min((int)(p.leaf_begin[t + 1] - tb), r0 + 64);
    const int S = p.near_S[t];
    const int Sp = (S + 3) & ~3;
    const int64_t off = p.nval_off[t];
    __shared__ int64_t s_beg[28];
    __shared__ int32_t s_pre[29];
    __shared__ int64_t s_gid[kAsmTile];
    if (threadIdx.x < 32) near_ranges_warp(p, t, threadIdx.x, s_beg, s_pre);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = kAsmThreads / 32;
    for (int base = 0; base < S; base += kAsmTile) {
        const int cnt = min(kAsmTile, S - base);
        if (threadIdx.x < cnt) {
            int s = base + threadIdx.x, e = 0;
            while (s_pre[e + 1] <= s) ++e;
            s_gid[threadIdx.x] = s_beg[e] + (s - s_pre[e]);
        }
        __syncthreads();
        for (int j = lane; j < cnt; j += 32) {
            SrcPanel sp;
            prep_source(p.verts + 12 * s_gid[j], sp);
            for (int row = r0 + warp; row < m; row += nw) {
                const double* c = p.cent + 3 * (tb + row);
                P[off + (int64_t)row * Sp + base + j] = coef * wilton(sp, c[0], c[1], c[2]);
            }
        }
        __syncthreads();
    }
}

__global__ void k_diag_inv(DevPlan p, const double* __restrict__ P, double* __restrict__ inv) {
    const int t = blockIdx.x;
    const int64_t tb = p.leaf_begin[t];
    const int m = (int)(p.leaf_begin[t + 1] - tb);
    const int Sp = (p.near_S[t] + 3) & ~3;
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
        double d = P[p.nval_off[t] + (int64_t)r * Sp + r];  // self leaf is the first source block
        inv[tb + r] = fabs(d) > 1e-30 ? 1.0 / d : 1.0;
    }
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Near apply as a register-tiled GEMM per work item (target leaf, <= 64 rows)
// and 64-wide chunk of right-hand sides:
//     Y[rows][0:64] = P_t[rows][0:S] X[src(0:S)][0:64],
// 64 threads, 8 x 8 outputs per thread (rows ty+8i, columns tx+8j: every
// shared-memory read is a broadcast or conflict-free), the contraction
// staged 32 source panels at a time with cp.async into a double buffer so the
// next tile's loads overlap this tile's FMAs.  T = double (plain path) or
// float (mixed path); rows of P are padded to a multiple of 4 entries and R
// is a multiple of 4, so every 16-byte copy is aligned.
template <class T>
__global__ void __launch_bounds__(64) k_near_apply(DevPlan p, const T* __restrict__ P, const T* __restrict__ X,
                                                   double* __restrict__ Y, int R) {
    constexpr int V = 16 / sizeof(T);        // elements per 16-byte copy
    constexpr int KC = 128 / sizeof(T);      // contraction chunk: 32 floats / 16 doubles
    constexpr int PP = KC + V;               // Ps row pitch (16-byte multiple, conflict-free)
    constexpr int XP = 64 + V;               // Xs row pitch
    const int t = p.item_leaf[blockIdx.x];
    const int r0 = p.item_row0[blockIdx.x];
    const int rc = blockIdx.y * 64;
    const int64_t tb = p.leaf_begin[t] + r0;
    const int m = min((int)(p.leaf_begin[t + 1] - p.leaf_begin[t]) - r0, 64);
    const int S = p.near_S[t];
    const int Sp = (S + 3) & ~3;
    const T* Pi = P + p.nval_off[t] + (int64_t)r0 * Sp;
    __shared__ int64_t s_beg[28];
    __shared__ int32_t s_pre[29];
    __shared__ int64_t s_gid[2][KC];
    __shared__ __align__(16) T Ps[2][64][PP];  // [row][k]
    __shared__ __align__(16) T Xs[2][KC][XP];  // [k][col]
    const int tid = threadIdx.x, tx = tid & 7, ty = tid >> 3;
    if (tid < 32) near_ranges_warp(p, t, tid, s_beg, s_pre);
    __syncthreads();
    const int nchunk = (Sp + KC - 1) / KC;
    auto gather_ids = [&](int c) {
        if (tid < KC) {
            const int sidx = c * KC + tid;
            int64_t g = 0;
            if (sidx < S) {
                int e = 0;
                while (s_pre[e + 1] <= sidx) ++e;
                g = s_beg[e] + (sidx - s_pre[e]);
            }
            s_gid[c & 1][tid] = g;
        }
    };
    auto issue = [&](int c) {
        const int k0 = c * KC, buf = c & 1;
#pragma unroll
        for (int q = 0; q < KC / V; ++q) {  // P tile: 64 rows x KC
            const int id = tid + 64 * q, row = id / (KC / V), kc = (id % (KC / V)) * V;
            const bool ok = row < m && k0 + kc < Sp;
            cp_async16(&Ps[buf][row][kc], ok ? (const void*)(Pi + (int64_t)row * Sp + k0 + kc) : (const void*)P, ok);
        }
#pragma unroll
        for (int q = 0; q < KC / V; ++q) {  // X tile: KC x 64 columns
            const int id = tid + 64 * q, kk = id / (64 / V), cc = (id % (64 / V)) * V;
            const bool ok = k0 + kk < S && rc + cc < R;
            cp_async16(&Xs[buf][kk][cc], ok ? (const void*)(X + s_gid[buf][kk] * R + rc + cc) : (const void*)X, ok);
        }
        cp_async_commit();
    };
    T acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = (T)0;
    gather_ids(0);
    __syncthreads();
    issue(0);
    for (int c = 0; c < nchunk; ++c) {
        if (c + 1 < nchunk) gather_ids(c + 1);
        __syncthreads();
        if (c + 1 < nchunk) {
            issue(c + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const int buf = c & 1;
#pragma unroll 4
        for (int kk = 0; kk < KC; ++kk) {
            T a[8], b[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = Ps[buf][ty + 8 * i][kk];
#pragma unroll
            for (int j = 0; j < 8; ++j) b[j] = Xs[buf][kk][tx + 8 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] += a[i] * b[j];
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int row = ty + 8 * i;
        if (row >= m) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int col = rc + tx + 8 * j;
            if (col < R) Y[(tb + row) * R + col] = (double)acc[i][j];
        }
    }
}

// 1-D Chebyshev interpolation weights S_n(x, x_m) (fmm/chebyshev.rs:41-74).
__device__ __forceinline__ void cheb_w(double x, int n, const double* roots, double* out) {
    double tx[8];
    tx[0] = 1.0;
    if (n > 1) tx[1] = x;
    for (int k = 2; k < n; ++k) tx[k] = 2.0 * x * tx[k - 1] - tx[k - 2];
    const double inv_n = 1.0 / n;
    for (int m = 0; m < n; ++m) {
        const double xm = roots[m];
        double sum = 0.5, prev = 1.0, cur = xm;
        for (int k = 1; k < n; ++k) {
            double tk;
            if (k == 1) {
                tk = xm;
            } else {
                tk = 2.0 * xm * cur - prev;
                prev = cur;
                cur = tk;
            }
            sum += tk * tx[k];
        }
        out[m] = 2.0 * inv_n * sum;
    }
}

// One thread per panel: W[j][m] for all n^3 nodes.
__global__ void k_src_weights(DevPlan p, int quad, double* __restrict__ W) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.N) return;
    const int n = p.n, n3 = p.n3;
    const double* ctr = p.leaf_ctr + 3 * p.leaf_of[j];
    const double ih = 1.0 / p.leaf_half;
    double* out = W + j * n3;
    for (int m = 0; m < n3; ++m) out[m] = 0.0;
    double w[3][8];
    if (quad == 0) {
        for (int d = 0; d < 3; ++d) cheb_w((p.cent[3 * j + d] - ctr[d]) * ih, n, p.roots, w[d]);
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b)
                for (int c = 0; c < n; ++c) out[(a * n + b) * n + c] = (w[0][a] * w[1][b]) * w[2][c];
        return;
    }
    // 2x2 Gauss rule on the bilinear map of the quad (a triangle is the quad
    // with a collapsed edge); weights normalised to sum to one.
    const double* v = p.verts + 12 * j;
    const double g = 0.57735026918962576451;
    double jw[4], pts[4][3], jsum = 0.0;
    for (int q = 0; q < 4; ++q) {
        const double u = (q & 1) ? g : -g, t = (q & 2) ? g : -g;
        const double N[4] = {0.25 * (1 - u) * (1 - t), 0.25 * (1 + u) * (1 - t), 0.25 * (1 + u) * (1 + t),
                             0.25 * (1 - u) * (1 + t)};
        const double dNu[4] = {-0.25 * (1 - t), 0.25 * (1 - t), 0.25 * (1 + t), -0.25 * (1 + t)};
        const double dNt[4] = {-0.25 * (1 - u), -0.25 * (1 + u), 0.25 * (1 + u), 0.25 * (1 - u)};
        double xu[3] = {0, 0, 0}, xt[3] = {0, 0, 0};
        for (int d = 0; d < 3; ++d) {
            pts[q][d] = 0.0;
            for (int k = 0; k < 4; ++k) {
                pts[q][d] += N[k] * v[3 * k + d];
                xu[d] += dNu[k] * v[3 * k + d];
                xt[d] += dNt[k] * v[3 * k + d];
            }
        }
        const double cx = xu[1] * xt[2] - xu[2] * xt[1], cy = xu[2] * xt[0] - xu[0] * xt[2],
                     cz = xu[0] * xt[1] - xu[1] * xt[0];
        jw[q] = sqrt(cx * cx + cy * cy + cz * cz);
        jsum += jw[q];
    }
    for (int q = 0; q < 4; ++q) {
        const double wq = jsum > 0.0 ? jw[q] / jsum : 0.25;
        for (int d = 0; d < 3; ++d) cheb_w((pts[q][d] - ctr[d]) * ih, n, p.roots, w[d]);
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b) {
                const double wab = wq * w[0][a] * w[1][b];
                for (int c = 0; c < n; ++c) out[(a * n + b) * n + c] += wab * w[2][c];
            }
    }
}

__global__ void k_potential_matrix(const double* __restrict__ sv, int64_t ns, const double* __restrict__ pts,
                                   int64_t nt, double* __restrict__ out, double coef) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t t0 = (int64_t)blockIdx.y * 64;
    if (s >= ns) return;
    SrcPanel sp;
    prep_source(sv + 12 * s, sp);
    for (int64_t t = t0; t < min(nt, t0 + 64); ++t)
        out[t * ns + s] = coef * wilton(sp, pts[3 * t], pts[3 * t + 1], pts[3 * t + 2]);
}

}  // namespace

void launch_near_assemble(Ctx& c, const DevPlan& p, int64_t nnz, double* P, double coef) {
    if (p.nleaf == 0) return;
    KTimer t(c, K_NEAR_ASSEMBLE, 8.0 * nnz, (double)nnz);
    k_near_assemble<<<p.nitems, kAsmThreads, 0, c.stream>>>(p, P, coef);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_diag_inv(Ctx& c, const DevPlan& p, const double* P, double* inv) {
    if (p.nleaf == 0) return;
    KTimer t(c, K_SMALL, 16.0 * p.N, 0.0);
    k_diag_inv<<<p.nleaf, 128, 0, c.stream>>>(p, P, inv);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_near_apply(Ctx& c, const DevPlan& p, int64_t nnz, const double* P, const double* X, double* Y, int R) {
    if (p.nleaf == 0) return;
    KTimer t(c, K_NEAR_APPLY64, 8.0 * nnz + 16.0 * (double)p.N * R, 2.0 * (double)nnz * R);
    k_near_apply<double><<<dim3(p.nitems, (R + 63) / 64), 64, 0, c.stream>>>(p, P, X, Y, R);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_near_apply32(Ctx& c, const DevPlan& p, int64_t nnz, const float* P, const float* X, double* Y, int R) {
    if (p.nleaf == 0) return;
    KTimer t(c, K_NEAR_APPLY, 4.0 * nnz + 12.0 * (double)p.N * R, 2.0 * (double)nnz * R);
    k_near_apply<float><<<dim3(p.nitems, (R + 63) / 64), 64, 0, c.stream>>>(p, P, X, Y, R);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

void launch_to_f32(Ctx& c, const double* a, float* b, int64_t n) {
    if (n == 0) return;
    KTimer t(c, K_VEC, 12.0 * n, 0.0);
    k_to_f32<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 32), 256, 0, c.stream>>>(a, b, n);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_src_weights(Ctx& c, const DevPlan& p, int quad, double* W) {
    if (p.N == 0) return;
    KTimer t(c, K_SMALL);
    k_src_weights<<<(unsigned)((p.N + 127) / 128), 128, 0, c.stream>>>(p, quad, W);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_potential_matrix(Ctx& c, const double* sv, int64_t ns, const double* pts, int64_t nt, double* out,
                             double coef) {
    if (ns == 0 || nt == 0) return;
    KTimer t(c, K_NEAR_ASSEMBLE, 8.0 * ns * nt, (double)ns * nt);
    dim3 g((unsigned)((ns + 127) / 128), (unsigned)((nt + 63) / 64));
    k_potential_matrix<<<g, 128, 0, c.stream>>>(sv, ns, pts, nt, out, coef);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

}  // namespace gpx
