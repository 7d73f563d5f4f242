// Chebyshev far field (fmm/bbfmm.rs:209-448) for R right-hand sides, in FP64
// (plain path) or FP32 (mixed path).  Expansions are stored per box as
// E[box][r][node] (node index fastest): one 64-node row per right-hand side
// is one contiguous 256 B (FP32) row, which is the K-major operand layout the
// tensor-core M2L (m2l_tc.cu) reads.
//
//  P2M  E[leaf][r][m]  = sum_j W_j[m] a_j X[j][r]          (W: source weights)
//  M2M  E[par][r][.]  += (Mx (x) My (x) Mz) E[child][r][.]  (tensor product, O(n^4))
//  M2L  L[t][r][m]    += (1/half) sum_s sum_l K_off[m][l] E[s][r][l]
//  L2L  L[child][r][.] += (Mx (x) My (x) Mz)^T L[par][r][.]
//  L2P  Y[j][r]       += coef sum_m S(c_j)[m] L[leaf][r][m]  (collocation point)
#include "farfield.cuh"

namespace gpx {

namespace {

constexpr int kRC = 8;  // right-hand sides per shared-memory chunk in M2M/L2L

// P2M: one CTA per leaf; outputs (r, m) in passes of 256 x 16 held in
// registers; the leaf's source weights and charges staged 16 panels at a time.
template <class T>
__global__ void __launch_bounds__(256) k_p2m_t(DevPlan p, const T* __restrict__ X, T* __restrict__ E, int R,
                                               int Rb) {
    const int t = blockIdx.x;
    const int n3 = p.n3;
    const int64_t j0 = p.leaf_begin[t], j1 = p.leaf_begin[t + 1];
    T* out = E + (int64_t)(p.leaf_box0 + t) * Rb * n3;
    __shared__ T Ws[16][217];
    __shared__ T Qs[16][65];
    const int nout = R * n3;
    for (int base = 0; base < nout; base += 256 * 16) {
        T acc[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) acc[q] = (T)0;
        const int rlo = base / n3, rhi = min(R, (base + 256 * 16 + n3 - 1) / n3);
        for (int r0 = (rlo / 64) * 64; r0 < rhi; r0 += 64) {
            for (int64_t jb = j0; jb < j1; jb += 16) {
                const int cnt = (int)min((int64_t)16, j1 - jb);
                __syncthreads();
                for (int e = threadIdx.x; e < 16 * n3; e += 256) {
                    const int jj = e / n3, mm = e % n3;
                    Ws[jj][mm] = jj < cnt ? (T)p.wsrc[(jb + jj) * n3 + mm] : (T)0;
                }
                for (int e = threadIdx.x; e < 16 * 64; e += 256) {
                    const int jj = e >> 6, rr = e & 63;
                    Qs[jj][rr] = (jj < cnt && r0 + rr < R) ? (T)p.area[jb + jj] * X[(jb + jj) * R + r0 + rr] : (T)0;
                }
                __syncthreads();
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int o = base + threadIdx.x + 256 * q;
                    const int r = o / n3, mm = o % n3;
                    if (o < nout && r >= r0 && r < r0 + 64) {
                        T a = acc[q];
                        for (int jj = 0; jj < cnt; ++jj) a += Ws[jj][mm] * Qs[jj][r - r0];
                        acc[q] = a;
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int o = base + threadIdx.x + 256 * q;
            if (o < nout) out[o] = acc[q];
        }
    }
}

// Three 1-D contractions of an (a,b,c) node array along z, y, x.
// transpose = false: parent from child (M2M), mat[m*n+k], k child node, m parent node.
// transpose = true : child from parent (L2L).
template <class T>
__device__ __forceinline__ void tensor3(const double* mx, const double* my, const double* mz, int n, bool transpose,
                                        T (*S0)[256], T (*S1)[256], int rc, int n3) {
    // stage z: S1[r][(a,b,c')] = sum_c Z[c'][c] S0[r][(a,b,c)]
    for (int o = threadIdx.x; o < rc * n3; o += blockDim.x) {
        const int r = o / n3, m = o % n3, a = m / (n * n), b = (m / n) % n, cp = m % n;
        T s = 0;
        for (int c = 0; c < n; ++c) s += (T)(transpose ? mz[c * n + cp] : mz[cp * n + c]) * S0[r][(a * n + b) * n + c];
        S1[r][m] = s;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < rc * n3; o += blockDim.x) {
        const int r = o / n3, m = o % n3, a = m / (n * n), bp = (m / n) % n, cp = m % n;
        T s = 0;
        for (int b = 0; b < n; ++b) s += (T)(transpose ? my[b * n + bp] : my[bp * n + b]) * S1[r][(a * n + b) * n + cp];
        S0[r][m] = s;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < rc * n3; o += blockDim.x) {
        const int r = o / n3, m = o % n3, ap = m / (n * n), bp = (m / n) % n, cp = m % n;
        T s = 0;
        for (int a = 0; a < n; ++a) s += (T)(transpose ? mx[a * n + ap] : mx[ap * n + a]) * S0[r][(a * n + bp) * n + cp];
        S1[r][m] = s;
    }
    __syncthreads();
}

// M2M: CTA per parent box; children are contiguous (Morton order).
template <class T>
__global__ void __launch_bounds__(256) k_m2m_t(DevPlan p, int pb0, const int32_t* __restrict__ child_first,
                                               const int32_t* __restrict__ child_count, T* __restrict__ E, int R,
                                               int Rb) {
    const int pb = pb0 + blockIdx.x;
    const int n = p.n, n3 = p.n3;
    __shared__ T S0[kRC][256], S1[kRC][256], A[kRC][256];
    const int cf = child_first[pb], cc = child_count[pb];
    for (int r0 = 0; r0 < R; r0 += kRC) {
        const int rc = min(kRC, R - r0);
        for (int o = threadIdx.x; o < rc * n3; o += blockDim.x) A[o / n3][o % n3] = 0;
        for (int ch = cf; ch < cf + cc; ++ch) {
            __syncthreads();
            const T* src = E + ((int64_t)ch * Rb + r0) * n3;
            for (int o = threadIdx.x; o < rc * n3; o += blockDim.x) S0[o / n3][o % n3] = src[o];
            __syncthreads();
            const int oc = p.box_octant[ch];
            tensor3<T>(p.m2m1d + (oc * 3 + 0) * n * n, p.m2m1d + (oc * 3 + 1) * n * n, p.m2m1d + (oc * 3 + 2) * n * n,
                       n, false, S0, S1, rc, n3);
            for (int o = threadIdx.x; o < rc * n3; o += blockDim.x) A[o / n3][o % n3] += S1[o / n3][o % n3];
        }
        __syncthreads();
        T* dst = E + ((int64_t)pb * Rb + r0) * n3;
        for (int o = threadIdx.x; o < rc * n3; o += blockDim.x) dst[o] += A[o / n3][o % n3];
        __syncthreads();
    }
}

// L2L: CTA per child box.
template <class T>
__global__ void __launch_bounds__(256) k_l2l_t(DevPlan p, int cb0, T* __restrict__ L, int R, int Rb) {
    const int cb = cb0 + blockIdx.x;
    const int n = p.n, n3 = p.n3;
    __shared__ T S0[kRC][256], S1[kRC][256];
    const int pb = p.box_parent[cb], oc = p.box_octant[cb];
    for (int r0 = 0; r0 < R; r0 += kRC) {
        const int rc = min(kRC, R - r0);
        __syncthreads();
        const T* src = L + ((int64_t)pb * Rb + r0) * n3;
        for (int o = threadIdx.x; o < rc * n3; o += blockDim.x) S0[o / n3][o % n3] = src[o];
        __syncthreads();
        tensor3<T>(p.m2m1d + (oc * 3 + 0) * n * n, p.m2m1d + (oc * 3 + 1) * n * n, p.m2m1d + (oc * 3 + 2) * n * n, n,
                   true, S0, S1, rc, n3);
        T* dst = L + ((int64_t)cb * Rb + r0) * n3;
        for (int o = threadIdx.x; o < rc * n3; o += blockDim.x) dst[o] += S1[o / n3][o % n3];
    }
}

// L2P: one CTA per (leaf, chunk of 16 right-hand sides): the leaf's local
// expansion rows staged in shared memory, one thread per (panel, rhs).
template <class T>
__global__ void __launch_bounds__(256) k_l2p_t(DevPlan p, const T* __restrict__ L, double* __restrict__ Y, int R,
                                               int Rb, double coef) {
    const int t = blockIdx.x;
    const int rc = blockIdx.y * 16;
    const int n = p.n, n3 = p.n3;
    const int64_t j0 = p.leaf_begin[t], j1 = p.leaf_begin[t + 1];
    __shared__ T Ls[16][217];
    const T* src = L + ((int64_t)(p.leaf_box0 + t) * Rb + rc) * n3;
    for (int e = threadIdx.x; e < 16 * n3; e += 256) {
        const int rr = e / n3, mm = e % n3;
        Ls[rr][mm] = rc + rr < R ? src[(int64_t)rr * n3 + mm] : (T)0;
    }
    __syncthreads();
    const int rr = threadIdx.x & 15;
    for (int64_t j = j0 + (threadIdx.x >> 4); j < j1; j += 16) {
        if (rc + rr >= R) continue;
        const double* w = p.w1d + j * 3 * n;
        T wz[8];
        for (int c = 0; c < n; ++c) wz[c] = (T)w[2 * n + c];
        T acc = 0;
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b) {
                const T wab = (T)(w[a] * w[n + b]);
                const T* row = &Ls[rr][(a * n + b) * n];
                T s = 0;
                for (int c = 0; c < n; ++c) s += wz[c] * row[c];
                acc += wab * s;
            }
        Y[j * R + rc + rr] += coef * (double)acc;
    }
}

// FP64 M2L: CTA per target box, 64 (m) x 64 (r) tile, 4x4 register tile per
// thread, operator and source tiles of 32 along the contraction in shared memory.
__global__ void __launch_bounds__(256) k_m2l64(DevPlan p, int b0, double* __restrict__ L, const double* __restrict__ E,
                                               int R, double scale) {
    const int tb = b0 + blockIdx.x;
    const int n3 = p.n3;
    __shared__ double Ks[32][65];  // [l][m]
    __shared__ double Ms[32][65];  // [l][r]
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
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
                const double* K = p.m2l_K + (int64_t)p.m2l_slot[e] * n3 * n3;
                const double* Es = E + (int64_t)p.m2l_src[e] * R * n3;
                for (int lc = 0; lc < n3; lc += 32) {
                    __syncthreads();
                    for (int idx = threadIdx.x; idx < 32 * 64; idx += 256) {
                        const int a = idx >> 5, b = idx & 31;  // a: m or r (64), b: l (32)
                        Ks[b][a] = (mc + a < n3 && lc + b < n3) ? K[(int64_t)(mc + a) * n3 + lc + b] : 0.0;
                        Ms[b][a] = (rcn + a < R && lc + b < n3) ? Es[(int64_t)(rcn + a) * n3 + lc + b] : 0.0;
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
                    const int mm = mc + ty + 16 * i, rr = rcn + tx + 16 * j;
                    if (mm < n3 && rr < R) L[((int64_t)tb * R + rr) * n3 + mm] += scale * acc[i][j];
                }
        }
    }
}

__device__ __forceinline__ void cp16(void* dst, const void* src, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
}

// Factored M2L for low-rank (compressed) order-4 operators K_o = U_o Vt_o, in
// two GEMM phases per level:
//   phase 1, CTA per source box s: for every column c = (pair e, k) of the
//     source's outgoing pairs, T[t_e][r][col(e,k)] = sum_l E_s[r][l] Vt_o[k][l];
//   phase 2, CTA per target box t: L_t[r][m] += scale * sum_c T_t[r][c] Ut[c][m],
//     the contraction running over the concatenated ranks of t's pairs.
// T is stored target-major (R rows x Kp_t columns per target, Kp_t = the
// summed ranks rounded up to 4) so phase 2 reads contiguous rows.
// Phase 1 as a transposed GEMM per work item (source box, up to 64 of its
// columns): C[c][r] = sum_l Vt_c[l] E_s[r][l].  The 64 gathered Vt rows (A)
// stream through a cp.async double buffer; E_s^T (B) is staged once.
template <class T>
__global__ void __launch_bounds__(64) k_m2l_fac_v(FacM2L<T> f, const int32_t* __restrict__ item_src,
                                                  const int64_t* __restrict__ item_c0,
                                                  const int32_t* __restrict__ item_cnt, const T* __restrict__ E,
                                                  int R) {
    constexpr int V = 16 / sizeof(T);
    constexpr int KC = 128 / sizeof(T);
    constexpr int PP = KC + V;
    constexpr int BP = 64 + V;
    const int it = blockIdx.x;
    const int rc = blockIdx.y * 64;
    const int s = item_src[it];
    const int64_t c0 = item_c0[it];
    const int nc = item_cnt[it];
    const int rows = min(64, R - rc);
    extern __shared__ __align__(16) unsigned char fac_smem[];
    T(*As)[64][PP] = reinterpret_cast<T(*)[64][PP]>(fac_smem);                        // [2][64][PP]: [c][l]
    T(*Bs)[BP] = reinterpret_cast<T(*)[BP]>(fac_smem + sizeof(T) * 2 * 64 * PP);      // [64][BP]:  [l][r]
    const int tid = threadIdx.x, tx = tid & 7, ty = tid >> 3;
    auto issue = [&](int ch) {
        const int k0 = ch * KC, buf = ch & 1;
#pragma unroll
        for (int q = 0; q < KC / V; ++q) {
            const int id = tid + 64 * q, row = id / (KC / V), kc = (id % (KC / V)) * V;
            const bool ok = row < nc;
            cp16(&As[buf][row][kc], ok ? (const void*)(f.Vt + f.col_vt[c0 + row] + k0 + kc) : (const void*)f.Vt, ok);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    issue(0);
    const T* Es = E + ((int64_t)s * R + rc) * 64;
    for (int e = tid; e < 64 * 64; e += 64) {
        const int r = e >> 6, l = e & 63;
        Bs[l][r] = r < rows ? Es[(int64_t)r * 64 + l] : (T)0;
    }
    T acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = (T)0;
    constexpr int nch = 64 / KC;
    for (int ch = 0; ch < nch; ++ch) {
        __syncthreads();
        if (ch + 1 < nch) {
            issue(ch + 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        const int buf = ch & 1;
#pragma unroll 4
        for (int kk = 0; kk < KC; ++kk) {
            T a[8], b[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[buf][ty + 8 * i][kk];
#pragma unroll
            for (int j = 0; j < 8; ++j) b[j] = Bs[ch * KC + kk][tx + 8 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] += a[i] * b[j];
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int c = ty + 8 * i;
        if (c >= nc) continue;
        const int tg = f.col_tgt[c0 + c];
        const int ld = (int)((f.tgt_col_off[tg + 1] - f.tgt_col_off[tg] + 3) & ~int64_t(3));
        T* dst = f.Tm + f.tgt_base[tg] * R + (int64_t)rc * ld + f.col_pos[c0 + c];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int r = tx + 8 * j;
            if (r < rows) dst[(int64_t)r * ld] = acc[i][j];
        }
    }
}

template <class T>
__global__ void __launch_bounds__(64) k_m2l_fac_u(FacM2L<T> f, int b0, T* __restrict__ L, int R, double scale) {
    constexpr int V = 16 / sizeof(T);
    constexpr int KC = 128 / sizeof(T);
    constexpr int PP = KC + V;
    constexpr int XP = 64 + V;
    const int t = b0 + blockIdx.x;
    const int rc = blockIdx.y * 64;
    const int64_t k0g = f.tgt_col_off[t], K = f.tgt_col_off[t + 1] - k0g;
    if (K == 0) return;
    const int Kp = (int)((K + 3) & ~int64_t(3));
    const T* A = f.Tm + f.tgt_base[t] * R + (int64_t)rc * Kp;
    const int m = min(64, R - rc);
    __shared__ __align__(16) T As[2][64][PP];
    __shared__ __align__(16) T Bs[2][KC][XP];
    const int tid = threadIdx.x, tx = tid & 7, ty = tid >> 3;
    const int nchunk = (Kp + KC - 1) / KC;
    auto issue = [&](int cch) {
        const int k0 = cch * KC, buf = cch & 1;
#pragma unroll
        for (int q = 0; q < KC / V; ++q) {
            const int id = tid + 64 * q, row = id / (KC / V), kc = (id % (KC / V)) * V;
            const bool ok = row < m && k0 + kc < Kp;
            cp16(&As[buf][row][kc], ok ? (const void*)(A + (int64_t)row * Kp + k0 + kc) : (const void*)f.Tm, ok);
        }
#pragma unroll
        for (int q = 0; q < KC / V; ++q) {
            const int id = tid + 64 * q, kk = id / (64 / V), cc = (id % (64 / V)) * V;
            const bool ok = k0 + kk < K;
            cp16(&Bs[buf][kk][cc], ok ? (const void*)(f.Ut + f.tgt_ut[k0g + k0 + kk] + cc) : (const void*)f.Ut, ok);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    T acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = (T)0;
    issue(0);
    for (int cch = 0; cch < nchunk; ++cch) {
        __syncthreads();
        if (cch + 1 < nchunk) {
            issue(cch + 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        const int buf = cch & 1;
#pragma unroll 4
        for (int kk = 0; kk < KC; ++kk) {
            T a[8], b[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[buf][ty + 8 * i][kk];
#pragma unroll
            for (int j = 0; j < 8; ++j) b[j] = Bs[buf][kk][tx + 8 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] += a[i] * b[j];
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int r = ty + 8 * i;
        if (r >= m) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            T* dst = L + ((int64_t)t * R + rc + r) * 64 + tx + 8 * j;
            *dst += (T)scale * acc[i][j];
        }
    }
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace

template <class T>
void launch_far_field(Ctx& c, const DevPlan& p, const FarLaunch& f, const T* X, double* Y, int R, int Rb, T* E,
                      T* L, double coef, const M2LLevelFn<T>& m2l) {
    cudaStream_t s = c.stream;
    const int n = p.n, n3 = p.n3, Lv = p.L;
    const double box_bytes = (double)sizeof(T) * n3 * R;
    GPX_CUDA(cudaMemsetAsync(E, 0, (size_t)p.nbox * n3 * Rb * sizeof(T), s));
    GPX_CUDA(cudaMemsetAsync(L, 0, (size_t)p.nbox * n3 * Rb * sizeof(T), s));
    {
        KTimer t(c, K_P2M, (double)p.N * (8.0 * R + 8.0 * n3 + 8.0) + p.nleaf * box_bytes, 2.0 * (double)p.N * n3 * R);
        k_p2m_t<T><<<p.nleaf, 256, 0, s>>>(p, X, E, R, Rb);
        GPX_LAUNCH_CHECK();
        c.launches += 1;
    }
    for (int l = Lv; l >= 3; --l) {
        const int pb0 = f.lvl_off[l - 1], npb = f.lvl_off[l] - pb0, nch = f.lvl_off[l + 1] - f.lvl_off[l];
        if (npb == 0) continue;
        KTimer t(c, K_M2M, (double)(npb + nch) * box_bytes, 2.0 * 3.0 * n * n3 * R * (double)nch);
        k_m2m_t<T><<<npb, 256, 0, s>>>(p, pb0, f.child_first, f.child_count, E, R, Rb);
        GPX_LAUNCH_CHECK();
        c.launches += 1;
    }
    for (int l = 2; l <= Lv; ++l) {
        const int b0 = f.lvl_off[l], nb = f.lvl_off[l + 1] - b0;
        if (nb == 0) continue;
        const double pairs = (double)(f.m2l_off[b0 + nb] - f.m2l_off[b0]);
        if (pairs == 0) continue;
        KTimer t(c, K_M2L, 2.0 * nb * box_bytes, 2.0 * (double)n3 * n3 * R * pairs);
        m2l(l, b0, nb, 1.0 / f.lvl_half[l]);
        c.launches += 1;
    }
    for (int l = 2; l < Lv; ++l) {
        const int cb0 = f.lvl_off[l + 1], ncb = f.lvl_off[l + 2] - cb0, npb = f.lvl_off[l + 1] - f.lvl_off[l];
        if (ncb == 0) continue;
        KTimer t(c, K_L2L, (double)(npb + 2 * ncb) * box_bytes, 2.0 * 3.0 * n * n3 * R * (double)ncb);
        k_l2l_t<T><<<ncb, 256, 0, s>>>(p, cb0, L, R, Rb);
        GPX_LAUNCH_CHECK();
        c.launches += 1;
    }
    {
        KTimer t(c, K_L2P, (double)p.N * (16.0 * R + 24.0 * n) + p.nleaf * box_bytes, 2.0 * (double)p.N * n3 * R);
        k_l2p_t<T><<<dim3(p.nleaf, cdiv(R, 16)), 256, 0, s>>>(p, L, Y, R, Rb, coef);
        GPX_LAUNCH_CHECK();
        c.launches += 1;
    }
}

template <class T>
void launch_m2l_fac(Ctx& c, const FacM2L<T>& f, const FacLevel& lv, int b0, int nb, T* L, const T* E, int R,
                    double scale) {
    constexpr int V = 16 / sizeof(T), KC = 128 / sizeof(T);
    const int smem = (int)(sizeof(T) * (2 * 64 * (KC + V) + 64 * (64 + V)));
    if (lv.nitems > 0) {
        GPX_CUDA(cudaFuncSetAttribute(k_m2l_fac_v<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        k_m2l_fac_v<T><<<dim3(lv.nitems, cdiv(R, 64)), 64, smem, c.stream>>>(f, lv.item_src, lv.item_c0, lv.item_cnt,
                                                                              E, R);
    }
    GPX_LAUNCH_CHECK();
    k_m2l_fac_u<T><<<dim3(nb, cdiv(R, 64)), 64, 0, c.stream>>>(f, b0, L, R, scale);
    GPX_LAUNCH_CHECK();
    c.launches += 1;  // the caller counts the other one
}
template void launch_m2l_fac<double>(Ctx&, const FacM2L<double>&, const FacLevel&, int, int, double*, const double*,
                                     int, double);
template void launch_m2l_fac<float>(Ctx&, const FacM2L<float>&, const FacLevel&, int, int, float*, const float*, int,
                                    double);

void launch_m2l64(Ctx& c, const DevPlan& p, int b0, int nb, double* L, const double* E, int R, double scale) {
    k_m2l64<<<nb, 256, 0, c.stream>>>(p, b0, L, E, R, scale);
    GPX_LAUNCH_CHECK();
}

template void launch_far_field<double>(Ctx&, const DevPlan&, const FarLaunch&, const double*, double*, int, int,
                                       double*, double*, double, const M2LLevelFn<double>&);
template void launch_far_field<float>(Ctx&, const DevPlan&, const FarLaunch&, const float*, double*, int, int,
                                      float*, float*, double, const M2LLevelFn<float>&);

}  // namespace gpx
