// Kernels of the adjoint sensitivities dC/dp and of the transposed operator.
//
// With P sigma_j = b_j (unit potential on conductor j) and C_ij = q_i^T
// sigma_j (q_i: panel areas of conductor i, cap/solver.rs:55-71), a parameter
// p that moves the panel vertices with velocity V = dx/dp gives
//     dC_ij/dp = (dq_i/dp)^T sigma_j - lambda_i^T (dP/dp) sigma_j,
//     P^T lambda_i = q_i   (one transposed solve per conductor).
// dP/dp sigma is applied exactly: the near blocks by the Wilton closed form
// (integrals/panel.rs:147-208) evaluated on dual numbers (dual.cuh) along V,
// the far field by the same FMM with differentiated end weights
//     d(P_far) sigma = far(P2M: d(a W), L2P: S(c)) + far(P2M: a W, L2P: dS(c)),
// where W are the panels' source weights and S(c) the Chebyshev weights of the
// collocation point; the tree, expansions and translation operators are fixed.
// The transposed operator uses the transposed near blocks (gathered from the
// forward blocks: the near-leaf relation is symmetric) and the far field with
// the end weights swapped (P2M: S(c), L2P: a W); its M2L is the transpose of
// the exact Chebyshev M2L (K_o^T = K_-o).
#include "adjoint.cuh"
#include "wilton.cuh"

namespace gpx {

namespace {

template <class S>
__device__ __forceinline__ void cheb_w_t(S x, int n, const double* roots, S* out) {
    S tx[8];
    tx[0] = 1.0;
    if (n > 1) tx[1] = x;
    for (int k = 2; k < n; ++k) tx[k] = 2.0 * x * tx[k - 1] - tx[k - 2];
    const double inv_n = 1.0 / n;
    for (int m = 0; m < n; ++m) {
        const double xm = roots[m];
        S sum = 0.5;
        double prev = 1.0, cur = xm;
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

// Dual centroid and area of a panel (area-weighted fan from vertex 0,
// integrals/panel.rs:29-67) with vertex velocities v.
__device__ void panel_props_dual(const double* x, const double* v, Dual* c, Dual& a) {
    Dual q[4][3];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int d = 0; d < 3; ++d) q[i][d] = Dual(x[3 * i + d], v[3 * i + d]);
    const bool tri = x[9] == x[6] && x[10] == x[7] && x[11] == x[8];
    const int nv = tri ? 3 : 4;
    Dual asum = 0.0, acc[3] = {0.0, 0.0, 0.0};
    for (int i = 1; i < nv - 1; ++i) {
        Dual e1[3], e2[3];
        for (int d = 0; d < 3; ++d) {
            e1[d] = q[i][d] - q[0][d];
            e2[d] = q[i + 1][d] - q[0][d];
        }
        const Dual cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2],
                   cz = e1[0] * e2[1] - e1[1] * e2[0];
        const Dual t = sqrt(cx * cx + cy * cy + cz * cz) * 0.5;
        for (int d = 0; d < 3; ++d) acc[d] += (q[0][d] + q[i][d] + q[i + 1][d]) * (1.0 / 3.0) * t;
        asum += t;
    }
    for (int d = 0; d < 3; ++d) c[d] = asum == 0.0 ? q[0][d] : acc[d] / asum;
    a = asum;
}

__global__ void k_panel_dprops(DevPlan p, const double* __restrict__ V, double* __restrict__ dcent,
                               double* __restrict__ darea) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.N) return;
    Dual c[3], a;
    panel_props_dual(p.verts + 12 * j, V + 12 * j, c, a);
    for (int d = 0; d < 3; ++d) dcent[3 * j + d] = c[d].d;
    darea[j] = a.d;
}

// Derivative of the near blocks: dP[k][l] = coef * d/dp Wilton(panel l, c_k).
// Same work items and layout as the assembly (one CTA per target leaf and
// <= 64 rows); pairs where neither the source panel nor the collocation
// point moves are written as zero without evaluating the integral.
constexpr int kDThreads = 256;
constexpr int kDTile = 64;
__global__ void __launch_bounds__(kDThreads) k_near_assemble_dual(DevPlan p, const double* __restrict__ V,
                                                                  const double* __restrict__ dcent,
                                                                  double* __restrict__ dP, double coef) {
    const int t = p.item_leaf[blockIdx.x];
    const int r0 = p.item_row0[blockIdx.x];
    const int64_t tb = p.leaf_begin[t];
    const int m = min((int)(p.leaf_begin[t + 1] - tb), r0 + 64);
    const int S = p.near_S[t];
    const int Sp = (S + 3) & ~3;
    const int64_t off = p.nval_off[t];
    __shared__ int64_t s_beg[28];
    __shared__ int32_t s_pre[29];
    __shared__ int64_t s_gid[kDTile];
    if (threadIdx.x < 32) near_ranges_warp(p, t, threadIdx.x, s_beg, s_pre);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = kDThreads / 32;
    for (int base = 0; base < S; base += kDTile) {
        const int cnt = min(kDTile, S - base);
        if (threadIdx.x < cnt) {
            int s = base + threadIdx.x, e = 0;
            while (s_pre[e + 1] <= s) ++e;
            s_gid[threadIdx.x] = s_beg[e] + (s - s_pre[e]);
        }
        __syncthreads();
        for (int j = lane; j < cnt; j += 32) {
            const int64_t g = s_gid[j];
            const double* vv = V + 12 * g;
            bool src_moves = false;
            for (int k = 0; k < 12; ++k) src_moves |= vv[k] != 0.0;
            Dual gv[12];
            for (int k = 0; k < 12; ++k) gv[k] = Dual(p.verts[12 * g + k], vv[k]);
            SrcPanelT<Dual> sp;
            prep_source_t<Dual>(gv, sp);
            for (int row = r0 + warp; row < m; row += nw) {
                const double* c = p.cent + 3 * (tb + row);
                const double* dc = dcent + 3 * (tb + row);
                double val = 0.0;
                if (src_moves || dc[0] != 0.0 || dc[1] != 0.0 || dc[2] != 0.0)
                    val = coef * wilton_t<Dual>(sp, Dual(c[0], dc[0]), Dual(c[1], dc[1]), Dual(c[2], dc[2])).d;
                dP[off + (int64_t)row * Sp + base + j] = val;
            }
        }
        __syncthreads();
    }
}

// Far-field source weights of one panel as dual numbers: a * W[m] (area
// included), W from the centroid (quad 0) or the 2x2 Gauss rule (quad 1) in
// its leaf, exactly as the forward source weights are formed.
__global__ void k_dsrc_weights(DevPlan p, int quad, const double* __restrict__ V, double* __restrict__ dW) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.N) return;
    const int n = p.n, n3 = p.n3;
    const double* ctr = p.leaf_ctr + 3 * p.leaf_of[j];
    const double ih = 1.0 / p.leaf_half;
    double* out = dW + j * n3;
    Dual cen[3], area;
    panel_props_dual(p.verts + 12 * j, V + 12 * j, cen, area);
    Dual w[3][8];
    if (quad == 0) {
        for (int d = 0; d < 3; ++d) cheb_w_t<Dual>((cen[d] - ctr[d]) * ih, n, p.roots, w[d]);
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b)
                for (int c = 0; c < n; ++c) out[(a * n + b) * n + c] = (area * ((w[0][a] * w[1][b]) * w[2][c])).d;
        return;
    }
    Dual vq[4][3];
    for (int k = 0; k < 4; ++k)
        for (int d = 0; d < 3; ++d) vq[k][d] = Dual(p.verts[12 * j + 3 * k + d], V[12 * j + 3 * k + d]);
    const double g = 0.57735026918962576451;
    Dual jw[4], pts[4][3], jsum = 0.0;
    for (int q = 0; q < 4; ++q) {
        const double u = (q & 1) ? g : -g, t = (q & 2) ? g : -g;
        const double N[4] = {0.25 * (1 - u) * (1 - t), 0.25 * (1 + u) * (1 - t), 0.25 * (1 + u) * (1 + t),
                             0.25 * (1 - u) * (1 + t)};
        const double dNu[4] = {-0.25 * (1 - t), 0.25 * (1 - t), 0.25 * (1 + t), -0.25 * (1 + t)};
        const double dNt[4] = {-0.25 * (1 - u), -0.25 * (1 + u), 0.25 * (1 + u), 0.25 * (1 - u)};
        Dual xu[3] = {0.0, 0.0, 0.0}, xt[3] = {0.0, 0.0, 0.0};
        for (int d = 0; d < 3; ++d) {
            pts[q][d] = 0.0;
            for (int k = 0; k < 4; ++k) {
                pts[q][d] += N[k] * vq[k][d];
                xu[d] += dNu[k] * vq[k][d];
                xt[d] += dNt[k] * vq[k][d];
            }
        }
        const Dual cx = xu[1] * xt[2] - xu[2] * xt[1], cy = xu[2] * xt[0] - xu[0] * xt[2],
                   cz = xu[0] * xt[1] - xu[1] * xt[0];
        jw[q] = sqrt(cx * cx + cy * cy + cz * cz);
        jsum += jw[q];
    }
    for (int m = 0; m < n3; ++m) out[m] = 0.0;
    for (int q = 0; q < 4; ++q) {
        const Dual wq = jsum > 0.0 ? jw[q] / jsum : Dual(0.25);
        for (int d = 0; d < 3; ++d) cheb_w_t<Dual>((pts[q][d] - ctr[d]) * ih, n, p.roots, w[d]);
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b) {
                const Dual wab = area * wq * w[0][a] * w[1][b];
                for (int c = 0; c < n; ++c) out[(a * n + b) * n + c] += (wab * w[2][c]).d;
            }
    }
}

// Chebyshev weights of the collocation point (centroid) as an N x n3 array:
// the value (dcent == null) or its derivative along dcent.
__global__ void k_centroid_weights(DevPlan p, const double* __restrict__ dcent, double* __restrict__ out) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= p.N) return;
    const int n = p.n, n3 = p.n3;
    const double* ctr = p.leaf_ctr + 3 * p.leaf_of[j];
    const double ih = 1.0 / p.leaf_half;
    Dual w[3][8];
    for (int d = 0; d < 3; ++d)
        cheb_w_t<Dual>(Dual((p.cent[3 * j + d] - ctr[d]) * ih, dcent ? dcent[3 * j + d] * ih : 0.0), n, p.roots,
                       w[d]);
    double* o = out + j * n3;
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b)
            for (int c = 0; c < n; ++c) {
                const Dual s = (w[0][a] * w[1][b]) * w[2][c];
                o[(a * n + b) * n + c] = dcent ? s.d : s.v;
            }
}

// Transposed near blocks: PT_t[i][c] = P_u[j][pos of panel i of t in u's
// source list], u the leaf of source column c of t and j its row in u.
__global__ void __launch_bounds__(256) k_near_transpose(DevPlan p, const int32_t* __restrict__ near_rev,
                                                        const int32_t* __restrict__ near_pre,
                                                        const double* __restrict__ P, double* __restrict__ PT) {
    const int t = p.item_leaf[blockIdx.x];
    const int r0 = p.item_row0[blockIdx.x];
    const int64_t tb = p.leaf_begin[t];
    const int m = min((int)(p.leaf_begin[t + 1] - tb), r0 + 64);
    const int S = p.near_S[t];
    const int Sp = (S + 3) & ~3;
    const int64_t off = p.nval_off[t];
    const int e0 = p.near_off[t], ne = p.near_off[t + 1] - e0;
    for (int c = threadIdx.x; c < S; c += blockDim.x) {
        int e = 0;
        while (e + 1 < ne && near_pre[e0 + e + 1] <= c) ++e;
        const int u = p.near_src[e0 + e];
        const int j = c - near_pre[e0 + e];
        const int eu = p.near_off[u] + near_rev[e0 + e];
        const int Su = p.near_S[u], Spu = (Su + 3) & ~3;
        const double* src = P + p.nval_off[u] + (int64_t)j * Spu + near_pre[eu];
        for (int i = r0; i < m; ++i) PT[off + (int64_t)i * Sp + c] = src[i];
    }
}

// Partial sums over one range of panels of
//   G[i][j] = sum_k da_k [cond_k == row_i] X[k][j] - sum_k Lam[k][i] D[k][j]
// for the rows solved (row_i >= 0).  X and D are N x R, Lam is N x Ra.  Grid
// (Ra, splits); 256 threads = 64 columns x 4 panel phases; the block writes
// Gp[split][i][j] and k_sum_splits adds the splits in order (deterministic).
__global__ void k_grad_contract(const int32_t* __restrict__ cond, const int32_t* __restrict__ row_cond,
                                const double* __restrict__ darea, const double* __restrict__ X,
                                const double* __restrict__ Lam, const double* __restrict__ D, int64_t N, int R,
                                int Ra, double* __restrict__ Gp) {
    const int i = blockIdx.x, sp = blockIdx.y, nsp = gridDim.y;
    const int ci = row_cond[i];
    const int64_t k0 = N * sp / nsp, k1 = N * (sp + 1) / nsp;
    __shared__ double red[256];
    for (int j0 = 0; j0 < R; j0 += 64) {
        const int j = j0 + (threadIdx.x & 63), part = threadIdx.x >> 6;  // 4 phases over k
        double acc = 0.0;
        if (j < R && ci >= 0)
            for (int64_t k = k0 + part; k < k1; k += 4) {
                double v = -Lam[k * Ra + i] * D[k * R + j];
                if (cond[k] == ci) v += darea[k] * X[k * R + j];
                acc += v;
            }
        red[threadIdx.x] = acc;
        __syncthreads();
        if (part == 0 && j < R)
            Gp[((int64_t)sp * Ra + i) * R + j] =
                red[threadIdx.x] + red[threadIdx.x + 64] + red[threadIdx.x + 128] + red[threadIdx.x + 192];
        __syncthreads();
    }
}

__global__ void k_sum_splits(const double* __restrict__ Gp, int nsp, int64_t n, double* __restrict__ G) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    double acc = 0.0;
    for (int s = 0; s < nsp; ++s) acc += Gp[(int64_t)s * n + e];
    G[e] = acc;
}

inline unsigned blocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void launch_panel_dprops(Ctx& c, const DevPlan& p, const double* V, double* dcent, double* darea) {
    KTimer t(c, K_SMALL, 104.0 * p.N, 0.0);
    k_panel_dprops<<<blocks(p.N, 128), 128, 0, c.stream>>>(p, V, dcent, darea);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_near_assemble_dual(Ctx& c, const DevPlan& p, int64_t nnz, const double* V, const double* dcent,
                               double* dP, double coef) {
    KTimer t(c, K_NEAR_ASSEMBLE, 8.0 * nnz, 0.0);
    k_near_assemble_dual<<<p.nitems, kDThreads, 0, c.stream>>>(p, V, dcent, dP, coef);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_dsrc_weights(Ctx& c, const DevPlan& p, int quad, const double* V, double* dW) {
    KTimer t(c, K_SMALL, (8.0 * p.n3 + 96.0) * p.N, 0.0);
    k_dsrc_weights<<<blocks(p.N, 128), 128, 0, c.stream>>>(p, quad, V, dW);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_centroid_weights(Ctx& c, const DevPlan& p, const double* dcent, double* out) {
    KTimer t(c, K_SMALL, (8.0 * p.n3 + 24.0) * p.N, 0.0);
    k_centroid_weights<<<blocks(p.N, 128), 128, 0, c.stream>>>(p, dcent, out);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_near_transpose(Ctx& c, const DevPlan& p, const int32_t* near_rev, const int32_t* near_pre,
                           const double* P, double* PT, int64_t nnz) {
    KTimer t(c, K_VEC, 16.0 * nnz, 0.0);
    k_near_transpose<<<p.nitems, 256, 0, c.stream>>>(p, near_rev, near_pre, P, PT);
    GPX_LAUNCH_CHECK();
    c.launches += 1;
}

void launch_grad_contract(Ctx& c, const int32_t* cond, const int32_t* row_cond, const double* darea,
                          const double* X, const double* Lam, const double* D, int64_t N, int R, int Ra, double* Gp,
                          double* G) {
    const int nsp = grad_contract_splits(Ra);
    KTimer t(c, K_VEC, 8.0 * N * (2.0 * R + Ra) + 12.0 * N, 4.0 * (double)N * R * Ra);
    k_grad_contract<<<dim3(Ra, nsp), 256, 0, c.stream>>>(cond, row_cond, darea, X, Lam, D, N, R, Ra, Gp);
    GPX_LAUNCH_CHECK();
    const int64_t n = (int64_t)Ra * R;
    k_sum_splits<<<blocks(n, 256), 256, 0, c.stream>>>(Gp, nsp, n, G);
    GPX_LAUNCH_CHECK();
    c.launches += 2;
}

}  // namespace gpx
