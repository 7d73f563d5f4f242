// FP64 kernels of the potential-coefficient operator.
//
//  * near-field assembly: closed-form Wilton integral of 1/|p - r'| over each
//    source panel (integrals/panel.rs:147-208), one CTA per target leaf, one
//    warp per group of target rows, lanes over source panels staged in shared
//    memory (source geometry is prepared once per lane and reused across rows);
//  * near-field apply: dense leaf blocks times R right-hand sides, source
//    columns of X staged in shared memory, block rows broadcast by shuffle;
//  * far field: Chebyshev P2M, M2M, M2L, L2L, L2P (fmm/bbfmm.rs:209-448).
#include "gpx_common.h"
#include "kernels.cuh"

namespace gpx {

namespace {

struct SrcPanel {
    double v[4][3];
    double n[3];
    double lh[4][3], uh[4][3];
    double el[4];
};

// Newell normal, unit edge tangents and in-plane edge normals of one panel.
__device__ __forceinline__ void prep_source(const double* g, SrcPanel& s) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int d = 0; d < 3; ++d) s.v[i][d] = g[3 * i + d];
    double nx = 0.0, ny = 0.0, nz = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double* c = s.v[i];
        const double* d = s.v[(i + 1) & 3];
        nx += (c[1] - d[1]) * (c[2] + d[2]);
        ny += (c[2] - d[2]) * (c[0] + d[0]);
        nz += (c[0] - d[0]) * (c[1] + d[1]);
    }
    double nn = sqrt(nx * nx + ny * ny + nz * nz);
    if (nn == 0.0) {
        s.n[0] = s.n[1] = s.n[2] = 0.0;
    } else {
        s.n[0] = nx / nn;
        s.n[1] = ny / nn;
        s.n[2] = nz / nn;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double* a = s.v[i];
        const double* b = s.v[(i + 1) & 3];
        double e[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        double el = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        s.el[i] = el;
        double l[3] = {0.0, 0.0, 0.0};
        if (el != 0.0) {
            l[0] = e[0] / el;
            l[1] = e[1] / el;
            l[2] = e[2] / el;
        }
        s.lh[i][0] = l[0];
        s.lh[i][1] = l[1];
        s.lh[i][2] = l[2];
        s.uh[i][0] = l[1] * s.n[2] - l[2] * s.n[1];
        s.uh[i][1] = l[2] * s.n[0] - l[0] * s.n[2];
        s.uh[i][2] = l[0] * s.n[1] - l[1] * s.n[0];
    }
}

// Wilton integral of one prepared panel at point p (panel.rs:147-208).  A
// zero-length edge (the repeated vertex of a triangle) contributes nothing.
//
// The log term is evaluated in an algebraically identical, cancellation-free
// form: with r0^2 = pp^2 + d^2, num = r+ + s+ and den = r- + s- are formed as
// r0^2 / (r - s) when s < 0, and log(num/den) = log1p((num-den)/den) with
// num - den = el * (num + den) / (r+ + r-).  Where the reference's direct
// form rounds num or den to <= 0 it falls back to the asinh difference; the
// stable form needs no fallback, and a point on the edge line (r0 = 0)
// contributes 0 exactly as the reference's fallback does.
__device__ __forceinline__ double wilton(const SrcPanel& s, double px, double py, double pz) {
    const double d = (px - s.v[0][0]) * s.n[0] + (py - s.v[0][1]) * s.n[1] + (pz - s.v[0][2]) * s.n[2];
    const double p0[3] = {px - s.n[0] * d, py - s.n[1] * d, pz - s.n[2] * d};
    const double ad = fabs(d);
    double total = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (s.el[i] == 0.0) continue;
        const double* a = s.v[i];
        const double* b = s.v[(i + 1) & 3];
        const double am[3] = {a[0] - p0[0], a[1] - p0[1], a[2] - p0[2]};
        const double bm[3] = {b[0] - p0[0], b[1] - p0[1], b[2] - p0[2]};
        const double pp = am[0] * s.uh[i][0] + am[1] * s.uh[i][1] + am[2] * s.uh[i][2];
        const double sm = am[0] * s.lh[i][0] + am[1] * s.lh[i][1] + am[2] * s.lh[i][2];
        const double sp = bm[0] * s.lh[i][0] + bm[1] * s.lh[i][1] + bm[2] * s.lh[i][2];
        const double r0sq = pp * pp + d * d;
        const double rp = sqrt(sp * sp + r0sq);
        const double rm = sqrt(sm * sm + r0sq);
        const double num = sp >= 0.0 ? rp + sp : r0sq / (rp - sp);
        const double den = sm >= 0.0 ? rm + sm : r0sq / (rm - sm);
        double lt = 0.0;
        if (num > 0.0 && den > 0.0) lt = pp * log1p(s.el[i] * (num + den) / ((rp + rm) * den));
        double at = 0.0;
        if (ad > 0.0 && pp != 0.0) {
            const double tp = (pp * sp) / (r0sq + ad * rp);
            const double tm = (pp * sm) / (r0sq + ad * rm);
            at = ad * (atan(tp) - atan(tm));
        }
        total += lt - at;
    }
    return total;
}

constexpr int kAsmThreads = 256;
constexpr int kAsmTile = 64;

// One CTA per work item (target leaf, <= 128 rows): rows of the leaf's
// P block m_t x S_t, row-major.
__global__ void __launch_bounds__(kAsmThreads) k_near_assemble(DevPlan p, double* __restrict__ P, double coef) {
    const int t = p.item_leaf[blockIdx.x];
    const int r0 = p.item_row0[blockIdx.x];
    const int64_t tb = p.leaf_begin[t];
    const int m = min((int)(p.leaf_begin[t + 1] - tb), r0 + 128);
    const int S = p.near_S[t];
    const int64_t off = p.nval_off[t];
    __shared__ int64_t s_beg[28];
    __shared__ int32_t s_pre[29];
    __shared__ int64_t s_gid[kAsmTile];
    const int e0 = p.near_off[t], ne = p.near_off[t + 1] - e0;
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int e = 0; e < ne; ++e) {
            int src = p.near_src[e0 + e];
            s_beg[e] = p.leaf_begin[src];
            s_pre[e] = acc;
            acc += (int)(p.leaf_begin[src + 1] - p.leaf_begin[src]);
        }
        s_pre[ne] = acc;
    }
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
                P[off + (int64_t)row * S + base + j] = coef * wilton(sp, c[0], c[1], c[2]);
            }
        }
        __syncthreads();
    }
}

__global__ void k_diag_inv(DevPlan p, const double* __restrict__ P, double* __restrict__ inv) {
    const int t = blockIdx.x;
    const int64_t tb = p.leaf_begin[t];
    const int m = (int)(p.leaf_begin[t + 1] - tb);
    const int S = p.near_S[t];
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
        double d = P[p.nval_off[t] + (int64_t)r * S + r];  // self leaf is the first source block
        inv[tb + r] = fabs(d) > 1e-30 ? 1.0 / d : 1.0;
    }
}

// Near apply: CTA per target leaf, 8 warps; each lane owns columns lane and
// lane+32 of a 64-wide RHS chunk, each warp owns rows warp + 8*i.
constexpr int kNaRPW = 16;  // rows per warp per pass (128 rows per pass)
__global__ void __launch_bounds__(256) k_near_apply(DevPlan p, const double* __restrict__ P,
                                                     const double* __restrict__ X, double* __restrict__ Y, int R) {
    const int t = p.item_leaf[blockIdx.x];
    const int r0 = p.item_row0[blockIdx.x];
    const int64_t tb = p.leaf_begin[t];
    const int m = min((int)(p.leaf_begin[t + 1] - tb), r0 + 8 * kNaRPW);
    const int S = p.near_S[t];
    const int64_t off = p.nval_off[t];
    __shared__ int64_t s_beg[28];
    __shared__ int32_t s_pre[29];
    __shared__ int64_t s_gid[32];
    __shared__ double xs[32][65];
    const int e0 = p.near_off[t], ne = p.near_off[t + 1] - e0;
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int e = 0; e < ne; ++e) {
            int src = p.near_src[e0 + e];
            s_beg[e] = p.leaf_begin[src];
            s_pre[e] = acc;
            acc += (int)(p.leaf_begin[src + 1] - p.leaf_begin[src]);
        }
        s_pre[ne] = acc;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int rc = 0; rc < R; rc += 64) {
        for (int rb = r0; rb < m; rb += 8 * kNaRPW) {
            double acc0[kNaRPW], acc1[kNaRPW];
#pragma unroll
            for (int i = 0; i < kNaRPW; ++i) acc0[i] = acc1[i] = 0.0;
            for (int sb = 0; sb < S; sb += 32) {
                const int cnt = min(32, S - sb);
                __syncthreads();
                if (threadIdx.x < cnt) {
                    int s = sb + threadIdx.x, e = 0;
                    while (s_pre[e + 1] <= s) ++e;
                    s_gid[threadIdx.x] = s_beg[e] + (s - s_pre[e]);
                }
                __syncthreads();
                for (int idx = threadIdx.x; idx < 32 * 64; idx += 256) {
                    int j = idx >> 6, c = idx & 63;
                    xs[j][c] = (j < cnt && rc + c < R) ? X[s_gid[j] * R + rc + c] : 0.0;
                }
                __syncthreads();
                double pr[kNaRPW];
#pragma unroll
                for (int i = 0; i < kNaRPW; ++i) {
                    int row = rb + warp + 8 * i;
                    pr[i] = (row < m && lane < cnt) ? P[off + (int64_t)row * S + sb + lane] : 0.0;
                }
                for (int j = 0; j < cnt; ++j) {
                    const double x0 = xs[j][lane], x1 = xs[j][lane + 32];
#pragma unroll
                    for (int i = 0; i < kNaRPW; ++i) {
                        double pv = __shfl_sync(0xffffffffu, pr[i], j);
                        acc0[i] += pv * x0;
                        acc1[i] += pv * x1;
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < kNaRPW; ++i) {
                int row = rb + warp + 8 * i;
                if (row < m) {
                    if (rc + lane < R) Y[(tb + row) * R + rc + lane] = acc0[i];
                    if (rc + lane + 32 < R) Y[(tb + row) * R + rc + lane + 32] = acc1[i];
                }
            }
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

// P2M: M[leafbox][m][r] = sum_j W_j[m] * area_j * X[j][r]; one thread per (m, r).
__global__ void k_p2m(DevPlan p, const double* __restrict__ X, double* __restrict__ M, int R) {
    const int t = blockIdx.x;
    const int o = blockIdx.y * blockDim.x + threadIdx.x;
    const int n3 = p.n3;
    if (o >= n3 * R) return;
    const int mi = o / R, r = o % R;
    double acc = 0.0;
    for (int64_t j = p.leaf_begin[t]; j < p.leaf_begin[t + 1]; ++j)
        acc += p.wsrc[j * n3 + mi] * (p.area[j] * X[j * R + r]);
    M[((int64_t)(p.leaf_box0 + t) * n3 + mi) * R + r] = acc;
}

// M2M into parents of level `lvl` boxes: one thread per (parent, m', r);
// parent boxes of level lvl-1 are [pb0, pb1), children are contiguous after
// the Morton sort so each parent scans the child range given by c_first/c_count.
__global__ void k_m2m(DevPlan p, int cb0, int cb1, const int32_t* __restrict__ child_first,
                      const int32_t* __restrict__ child_count, int pb0, double* __restrict__ M, int R) {
    const int pb = pb0 + blockIdx.x;
    const int o = blockIdx.y * blockDim.x + threadIdx.x;
    const int n = p.n, n3 = p.n3;
    if (o >= n3 * R) return;
    const int mi = o / R, r = o % R;
    const int ap = mi / (n * n), bp = (mi / n) % n, cp = mi % n;
    double acc = 0.0;
    const int cf = child_first[pb], cc = child_count[pb];
    for (int ch = cf; ch < cf + cc; ++ch) {
        const int oc = p.box_octant[ch];
        const double* mx = p.m2m1d + (oc * 3 + 0) * n * n;
        const double* my = p.m2m1d + (oc * 3 + 1) * n * n;
        const double* mz = p.m2m1d + (oc * 3 + 2) * n * n;
        const double* src = M + (int64_t)ch * n3 * R + r;
        for (int a = 0; a < n; ++a) {
            double sa = 0.0;
            for (int b = 0; b < n; ++b) {
                double sb = 0.0;
                for (int c = 0; c < n; ++c) sb += mz[cp * n + c] * src[((a * n + b) * n + c) * R];
                sa += my[bp * n + b] * sb;
            }
            acc += mx[ap * n + a] * sa;
        }
    }
    M[((int64_t)pb * n3 + mi) * R + r] += acc;
    (void)cb0;
    (void)cb1;
}

// M2L at one level: CTA per target box, 64 x 64 output tile of (m, r) with a
// 4 x 4 register tile per thread; operator and source multipole tiles of 32
// along the contraction staged in shared memory.
__global__ void __launch_bounds__(256) k_m2l(DevPlan p, int b0, double* __restrict__ Lc,
                                             const double* __restrict__ M, int R, double scale) {
    const int tb = b0 + blockIdx.x;
    const int n3 = p.n3;
    __shared__ double Ks[32][65];   // [l][m]
    __shared__ double Ms[32][65];   // [l][r]
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // r-group, m-group
    const int64_t s0 = p.m2l_off[tb], s1 = p.m2l_off[tb + 1];
    if (s0 == s1) return;
    for (int mc = 0; mc < n3; mc += 64) {
        for (int rcn = 0; rcn < R; rcn += 64) {
            double acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
            for (int64_t e = s0; e < s1; ++e) {
                const int src = p.m2l_src[e];
                const double* K = p.m2l_K + (int64_t)p.m2l_slot[e] * n3 * n3;
                const double* Msrc = M + (int64_t)src * n3 * R;
                for (int lc = 0; lc < n3; lc += 32) {
                    __syncthreads();
                    for (int idx = threadIdx.x; idx < 32 * 64; idx += 256) {
                        const int a = idx >> 5, b = idx & 31;  // K row m = mc+a, col l = lc+b
                        Ks[b][a] = (mc + a < n3 && lc + b < n3) ? K[(int64_t)(mc + a) * n3 + lc + b] : 0.0;
                        const int l = idx >> 6, c = idx & 63;  // M row l = lc+l, col r = rcn+c
                        Ms[l][c] = (lc + l < n3 && rcn + c < R) ? Msrc[(int64_t)(lc + l) * R + rcn + c] : 0.0;
                    }
                    __syncthreads();
#pragma unroll 4
                    for (int l = 0; l < 32; ++l) {
                        double kv[4], mv[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) kv[i] = Ks[l][ty + 16 * i];
#pragma unroll
                        for (int j = 0; j < 4; ++j) mv[j] = Ms[l][tx + 16 * j];
#pragma unroll
                        for (int i = 0; i < 4; ++i)
#pragma unroll
                            for (int j = 0; j < 4; ++j) acc[i][j] += kv[i] * mv[j];
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    int mm = mc + ty + 16 * i, rr = rcn + tx + 16 * j;
                    if (mm < n3 && rr < R) Lc[((int64_t)tb * n3 + mm) * R + rr] += scale * acc[i][j];
                }
        }
    }
}

// L2L to children of level lvl boxes: one thread per (child, m, r).
__global__ void k_l2l(DevPlan p, int cb0, double* __restrict__ Lc, int R) {
    const int cb = cb0 + blockIdx.x;
    const int o = blockIdx.y * blockDim.x + threadIdx.x;
    const int n = p.n, n3 = p.n3;
    if (o >= n3 * R) return;
    const int mi = o / R, r = o % R;
    const int a = mi / (n * n), b = (mi / n) % n, c = mi % n;
    const int pb = p.box_parent[cb], oc = p.box_octant[cb];
    const double* mx = p.m2m1d + (oc * 3 + 0) * n * n;
    const double* my = p.m2m1d + (oc * 3 + 1) * n * n;
    const double* mz = p.m2m1d + (oc * 3 + 2) * n * n;
    const double* src = Lc + (int64_t)pb * n3 * R + r;
    double acc = 0.0;
    for (int ap = 0; ap < n; ++ap) {
        double sa = 0.0;
        for (int bp = 0; bp < n; ++bp) {
            double sb = 0.0;
            for (int cp = 0; cp < n; ++cp) sb += mz[cp * n + c] * src[((ap * n + bp) * n + cp) * R];
            sa += my[bp * n + b] * sb;
        }
        acc += mx[ap * n + a] * sa;
    }
    Lc[((int64_t)cb * n3 + mi) * R + r] += acc;
}

// L2P: Y[j][r] += coef * sum_m W_j[m] L[leafbox][m][r]; one thread per (j, r).
__global__ void k_l2p(DevPlan p, const double* __restrict__ Lc, double* __restrict__ Y, int R, double coef,
                      const int32_t* __restrict__ leaf_of) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= p.N * R) return;
    const int64_t j = o / R;
    const int r = (int)(o % R);
    const int n = p.n, n3 = p.n3;
    const double* w = p.w1d + j * 3 * n;
    const double* L = Lc + (int64_t)(p.leaf_box0 + leaf_of[j]) * n3 * R + r;
    double acc = 0.0;
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) {
            const double wab = w[a] * w[n + b];
            for (int c = 0; c < n; ++c) acc += (wab * w[2 * n + c]) * L[((a * n + b) * n + c) * R];
        }
    Y[o] += coef * acc;
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
    KTimer t(c, K_NEAR_APPLY, 8.0 * nnz + 16.0 * (double)p.N * R, 2.0 * (double)nnz * R);
    k_near_apply<<<p.nitems, 256, 0, c.stream>>>(p, P, X, Y, R);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_far_apply(Ctx& c, const DevPlan& p, const FarLaunch& f, const double* X, double* Y, int R, double* M,
                      double* Lc, double coef) {
    cudaStream_t s = c.stream;
    const int n = p.n, n3 = p.n3, L = p.L;
    const double box_bytes = 8.0 * n3 * R;
    GPX_CUDA(cudaMemsetAsync(M, 0, (size_t)p.nbox * n3 * R * sizeof(double), s));
    GPX_CUDA(cudaMemsetAsync(Lc, 0, (size_t)p.nbox * n3 * R * sizeof(double), s));
    const unsigned oc = (unsigned)((n3 * R + 255) / 256);
    {
        KTimer t(c, K_P2M, (double)p.N * (8.0 * R + 24.0 * n + 8.0) + p.nleaf * box_bytes, 2.0 * (double)p.N * n3 * R);
        k_p2m<<<dim3(p.nleaf, oc), 256, 0, s>>>(p, X, M, R);
        GPX_LAUNCH_CHECK();
        c.launches += 1;
    }
    for (int l = L; l >= 3; --l) {  // children at level l -> parents at level l-1
        const int pb0 = f.lvl_off[l - 1], npb = f.lvl_off[l] - pb0, nch = f.lvl_off[l + 1] - f.lvl_off[l];
        if (npb == 0) continue;
        KTimer t(c, K_M2M, (double)(npb + nch) * box_bytes, 2.0 * 3.0 * n * n3 * R * (double)nch);
        k_m2m<<<dim3(npb, oc), 256, 0, s>>>(p, f.lvl_off[l], f.lvl_off[l + 1], f.child_first, f.child_count, pb0, M, R);
        GPX_LAUNCH_CHECK();
        c.launches += 1;
    }
    for (int l = 2; l <= L; ++l) {
        const int b0 = f.lvl_off[l], nb = f.lvl_off[l + 1] - b0;
        if (nb == 0) continue;
        const double pairs = (double)(f.m2l_off[b0 + nb] - f.m2l_off[b0]);
        if (pairs == 0) continue;
        KTimer t(c, K_M2L, 2.0 * nb * box_bytes, 2.0 * (double)n3 * n3 * R * pairs);
        k_m2l<<<nb, 256, 0, s>>>(p, b0, Lc, M, R, 1.0 / f.lvl_half[l]);
        GPX_LAUNCH_CHECK();
        c.launches += 1;
    }
    for (int l = 2; l < L; ++l) {  // parents at level l -> children at level l+1
        const int cb0 = f.lvl_off[l + 1], ncb = f.lvl_off[l + 2] - cb0, npb = f.lvl_off[l + 1] - f.lvl_off[l];
        if (ncb == 0) continue;
        KTimer t(c, K_L2L, (double)(npb + 2 * ncb) * box_bytes, 2.0 * 3.0 * n * n3 * R * (double)ncb);
        k_l2l<<<dim3(ncb, oc), 256, 0, s>>>(p, cb0, Lc, R);
        GPX_LAUNCH_CHECK();
        c.launches += 1;
    }
    {
        KTimer t(c, K_L2P, (double)p.N * (16.0 * R + 24.0 * n) + p.nleaf * box_bytes, 2.0 * (double)p.N * n3 * R);
        k_l2p<<<(unsigned)((p.N * R + 255) / 256), 256, 0, s>>>(p, Lc, Y, R, coef, f.leaf_of);
        GPX_LAUNCH_CHECK();
        c.launches += 1;
    }
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
