// Chebyshev far field (fmm/bbfmm.rs:209-448) for R right-hand sides, in FP64
// (plain path) or FP32 (mixed path), for expansion orders 2 to 6.
// Expansions are stored per box as E[box][r][node] with a node stride ns =
// n^3 rounded up to a multiple of 32 (node index fastest, padding nodes zero):
// one right-hand side's expansion is one contiguous, 128-byte-aligned row,
// which is also the K-major operand row of the tensor-core M2L (m2l_tc.cu).
//
//  P2M  E[leaf][r][m]  = sum_j W_j[m] a_j X[j][r]          (W: source weights)
//  M2M  E[par][r][.]   = sum_children (Mx (x) My (x) Mz) E[child][r][.]
//  M2L  L[t][r][m]    += (1/half) sum_s sum_l K_off[m][l] E[s][r][l]
//  L2L  L[child][r][.] += (Mx (x) My (x) Mz)^T L[par][r][.]
//  L2P  Y[j][r]       += coef sum_m S(c_j)[m] L[leaf][r][m]  (collocation point)
//
// P2M and L2P are register-tiled GEMMs per work item of at most 64 panels of
// one leaf (so large leaves spread over several CTAs).  M2M and L2L run one
// CTA per parent box over all eight octants at once: the 1-D operator of an axis
// depends only on the child's bit along that axis, so the eight children's
// contractions share partial sums along a binary tree (z, then y, then x for
// M2M; the reverse for L2L): 14 n^4 multiply-adds per parent and right-hand
// side instead of 24 n^4.
#include "farfield.cuh"
#include "krylov.cuh"

namespace gpx {

namespace {

__device__ __forceinline__ void cp16(void* dst, const void* src, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
}

// One 4- or 8-byte element copied global -> shared asynchronously: a CTA
// puts all its copies in flight before one wait instead of a load round trip
// per loop pass.
template <class T>
__device__ __forceinline__ void cp_elem(T* dst, const T* src) {
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "cp.async.ca copies 4, 8 or 16 bytes");
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"((int)sizeof(T)) : "memory");
}

// Panels per near-field work item (the plan's kRowsPerItem).
constexpr int kItemPanels = 64;

template <int N>
struct Ord {
    static constexpr int n3 = N * N * N;
    static constexpr int ns = (n3 + 31) & ~31;
};

// CTAs per SM the FP32 P2M and L2P are compiled for at orders <= 5: four
// (64 registers, no spills) instead of the two that 90 registers allowed, so
// more warps hide the latency of each staged slice's global loads.
template <class T, int N>
constexpr int kMinCtas() {
    return sizeof(T) == 4 && N <= 5 ? 4 : 1;
}

// P2M as a GEMM per (work item = leaf and <= 64 of its panels, 64-wide chunk
// of rows r):  E[leaf][r][m] = sum_j W[j][m] * (a_j X[j][r]).
// The work items are the near-field items (64 panels each), so a leaf of a few
// hundred panels spreads over several CTAs instead of serialising one: the
// first item of a leaf writes E[leaf], each further item writes a partial
// expansion at box index nbox + slot, and k_p2m_fix adds the partials in item
// order (deterministic).
// 256 threads; thread (tm, tr) holds nodes MI tm .. MI tm + MI - 1 and rows
// 8 tr .. 8 tr + 7.  Panels are staged KP at a time.  Every row r < Rb and node
// m < ns of the chunk is written (zeros outside r < R, m < n3).
template <class T, int N>
__global__ void __launch_bounds__(256, kMinCtas<T, N>())
    k_p2m(DevPlan p, const int32_t* __restrict__ slot, const T* __restrict__ X, const T* __restrict__ W,
          bool mul_area, T* __restrict__ E, int R, int Rb) {
    constexpr int N3 = Ord<N>::n3, NS = Ord<N>::ns, MI = NS / 32;
    constexpr int KP = sizeof(T) == 8 ? 16 : 32;  // panels per staged chunk (static shared memory <= 48 KB)
    constexpr int QW = 64 + 16 / (int)sizeof(T);  // Qs row stride: 16-byte aligned rows
    const int it = blockIdx.x;
    const int t = p.item_leaf[it], r0 = p.item_row0[it];
    const int rc = blockIdx.y * 64;
    const int64_t lb = p.leaf_begin[t];
    const int64_t j0 = lb + r0, j1 = min(lb + r0 + kItemPanels, p.leaf_begin[t + 1]);
    __shared__ T Ws[KP][NS + 1];
    __shared__ __align__(16) T Qs[KP][QW];
    const int tid = threadIdx.x, tm = tid >> 3, tr = tid & 7;
    T acc[MI][8];
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = (T)0;
    for (int64_t jb = j0; jb < j1; jb += KP) {
        const int cnt = (int)min((int64_t)KP, j1 - jb);
        __syncthreads();
        for (int e = tid; e < KP * NS; e += 256) {
            const int k = e / NS, m = e % NS;
            Ws[k][m] = (k < cnt && m < N3) ? W[(jb + k) * N3 + m] : (T)0;
        }
        for (int e = tid; e < KP * 64; e += 256) {
            const int k = e >> 6, r = e & 63;
            Qs[k][r] = (k < cnt && rc + r < R) ? (mul_area ? (T)p.area[jb + k] : (T)1) * X[(jb + k) * R + rc + r]
                                               : (T)0;
        }
        __syncthreads();
        for (int k = 0; k < cnt; ++k) {
            T a[MI], b[8];
#pragma unroll
            for (int i = 0; i < MI; ++i) a[i] = Ws[k][MI * tm + i];
            if constexpr (sizeof(T) == 4) {
                const float4 b0 = *reinterpret_cast<const float4*>(&Qs[k][8 * tr]);
                const float4 b1 = *reinterpret_cast<const float4*>(&Qs[k][8 * tr + 4]);
                b[0] = b0.x, b[1] = b0.y, b[2] = b0.z, b[3] = b0.w, b[4] = b1.x, b[5] = b1.y, b[6] = b1.z, b[7] = b1.w;
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const double2 v = *reinterpret_cast<const double2*>(&Qs[k][8 * tr + 2 * q]);
                    b[2 * q] = v.x, b[2 * q + 1] = v.y;
                }
            }
#pragma unroll
            for (int i = 0; i < MI; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] += a[i] * b[j];
        }
    }
    const int64_t box = slot[it] < 0 ? (int64_t)p.leaf_box0 + t : (int64_t)p.nbox + slot[it];
    T* out = E + (box * Rb + rc) * NS;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int r = 8 * tr + j;
        if (rc + r >= Rb) continue;
#pragma unroll
        for (int i = 0; i < MI; ++i) {
            const int m = MI * tm + i;
            out[(int64_t)r * NS + m] = (m < N3 && rc + r < R) ? acc[i][j] : (T)0;
        }
    }
}

// E[leaf] += the partial expansions of its further work items, in item order.
// One CTA per (leaf with several items, 1024-value chunk of its Rb x ns block).
template <class T>
__global__ void __launch_bounds__(256) k_p2m_fix(int nbox, int leaf_box0, const int32_t* __restrict__ fix_leaf,
                                                 const int32_t* __restrict__ fix_first,
                                                 const int32_t* __restrict__ fix_cnt, T* __restrict__ E,
                                                 int64_t block) {
    const int f = blockIdx.x;
    const int64_t e = ((int64_t)blockIdx.y * 256 + threadIdx.x) * 4;
    if (e >= block) return;
    T* dst = E + ((int64_t)leaf_box0 + fix_leaf[f]) * block + e;
    T v0 = dst[0], v1 = dst[1], v2 = dst[2], v3 = dst[3];
    const int s0 = fix_first[f], cnt = fix_cnt[f];
    for (int q = 0; q < cnt; ++q) {
        const T* src = E + ((int64_t)nbox + s0 + q) * block + e;
        v0 += src[0], v1 += src[1], v2 += src[2], v3 += src[3];
    }
    dst[0] = v0, dst[1] = v1, dst[2] = v2, dst[3] = v3;
}

// L2P as a GEMM per (work item = leaf and <= 64 of its panels, 64-wide chunk
// of r):  Y[j][r] += coef * sum_m S_j[m] L[leaf][r][m],  S_j[m] = wx[a] wy[b]
// wz[c] (the centroid's separable weights), or S_j = Wt[j] (times a_j if
// mul_area) when explicit weights are given.
// 256 threads; thread (tj, tr) holds panels 4 tj .. 4 tj + 3 and rows
// 4 tr .. 4 tr + 3; nodes are staged 32 at a time.
template <class T, int N>
__global__ void __launch_bounds__(256, kMinCtas<T, N>())
    k_l2p(DevPlan p, const T* __restrict__ L, const T* __restrict__ Wt, bool mul_area, double* __restrict__ Y, int R,
          int Rb, double coef) {
    constexpr int N3 = Ord<N>::n3, NS = Ord<N>::ns;
    constexpr int JP = kItemPanels, MK = 32, SW = 64 + 16 / (int)sizeof(T);
    const int it = blockIdx.x;
    const int t = p.item_leaf[it], r0 = p.item_row0[it];
    const int rc = blockIdx.y * 64;
    const int64_t lb = p.leaf_begin[t];
    const int64_t jb = lb + r0;
    const int cnt = (int)min((int64_t)JP, p.leaf_begin[t + 1] - jb);
    const T* src = L + ((int64_t)(p.leaf_box0 + t) * Rb + rc) * NS;
    __shared__ T wv[JP][3 * N];
    __shared__ __align__(16) T Ss[MK][SW];  // [node][panel]
    __shared__ __align__(16) T Ls[MK][SW];  // [node][row]
    const int tid = threadIdx.x, tj = tid >> 4, tr = tid & 15;
    if (!Wt)
        for (int e = tid; e < JP * 3 * N; e += 256) {
            const int jj = e / (3 * N);
            wv[jj][e % (3 * N)] = jj < cnt ? (T)p.w1d[jb * 3 * N + e] : (T)0;
        }
    T acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i][q] = (T)0;
    for (int m0 = 0; m0 < N3; m0 += MK) {
        __syncthreads();
        for (int e = tid; e < JP * MK; e += 256) {
            const int jj = e / MK, mm = e % MK, m = m0 + mm;
            T v = (T)0;
            if (m < N3 && jj < cnt) {
                v = Wt ? Wt[(jb + jj) * N3 + m] : wv[jj][m / (N * N)] * wv[jj][N + (m / N) % N] * wv[jj][2 * N + m % N];
                if (mul_area) v *= (T)p.area[jb + jj];
            }
            Ss[mm][jj] = v;
        }
        for (int e = tid; e < 64 * MK; e += 256) {
            const int mm = e % MK, r = e / MK;
            Ls[mm][r] = (m0 + mm < N3 && rc + r < R) ? src[(int64_t)r * NS + m0 + mm] : (T)0;
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < MK; ++k) {
            T a[4], b[4];
            if constexpr (sizeof(T) == 4) {
                const float4 av = *reinterpret_cast<const float4*>(&Ss[k][4 * tj]);
                const float4 bv = *reinterpret_cast<const float4*>(&Ls[k][4 * tr]);
                a[0] = av.x, a[1] = av.y, a[2] = av.z, a[3] = av.w;
                b[0] = bv.x, b[1] = bv.y, b[2] = bv.z, b[3] = bv.w;
            } else {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const double2 av = *reinterpret_cast<const double2*>(&Ss[k][4 * tj + 2 * h]);
                    const double2 bv = *reinterpret_cast<const double2*>(&Ls[k][4 * tr + 2 * h]);
                    a[2 * h] = av.x, a[2 * h + 1] = av.y, b[2 * h] = bv.x, b[2 * h + 1] = bv.y;
                }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[i][q] += a[i] * b[q];
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int jj = 4 * tj + i;
        if (jj >= cnt) continue;
        double* y = Y + (jb + jj) * R + rc + 4 * tr;
        if ((R & 1) == 0 && rc + 4 * tr + 3 < R) {  // 16-byte aligned pairs
            double2 y0 = *reinterpret_cast<double2*>(y), y1 = *reinterpret_cast<double2*>(y + 2);
            y0.x += coef * (double)acc[i][0], y0.y += coef * (double)acc[i][1];
            y1.x += coef * (double)acc[i][2], y1.y += coef * (double)acc[i][3];
            *reinterpret_cast<double2*>(y) = y0;
            *reinterpret_cast<double2*>(y + 2) = y1;
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (rc + 4 * tr + q < R) y[q] += coef * (double)acc[i][q];
        }
    }
}

// Rows of right-hand sides per M2M / L2L block.
template <class T, int N>
constexpr int tree_rc() {
    return (sizeof(T) == 8 && N >= 6) ? 4 : 8;
}
template <class T, int N>
constexpr size_t tree_smem() {
    return sizeof(T) * (size_t)(8 + 4 + 2) * tree_rc<T, N>() * Ord<N>::n3;
}
// Resident M2M / L2L blocks per SM asked of the register allocator: three
// for FP32 order 5 (56 KB of shared memory each), where the default
// allocation (80-92 registers) leaves two.
template <class T, int N>
constexpr int tree_min_blocks() {
    return (sizeof(T) == 4 && N == 5) ? 3 : 1;
}

// 1-D operators of the three axes as T: M1[axis][bit][m][k] (m parent node,
// k child node), from the plan's per-octant table mat[(o*3+axis)*n*n + m*n + k].
template <class T, int N>
__device__ __forceinline__ void load_m1(const double* m2m1d, T (*M1)[2][N * N]) {
    for (int e = threadIdx.x; e < 3 * 2 * N * N; e += blockDim.x) {
        const int axis = e / (2 * N * N), bit = (e / (N * N)) & 1, mk = e % (N * N);
        const int oct = bit << axis;  // any octant with this bit on this axis
        M1[axis][bit][mk] = (T)m2m1d[(oct * 3 + axis) * N * N + mk];
    }
}

// M2M, one CTA per (parent box, chunk of RC rows r); children are contiguous
// (Morton order).  A[oct] holds the child of octant oct (zero if absent);
// B[q] = sum_oz Z_oz A[q | oz<<2] (q = ox | oy<<1); C[ox] = sum_oy Y_oy B;
// E_par = sum_ox X_ox C[ox].  The parent row is overwritten (the parent has
// no other contribution), padding nodes written as zero.
template <class T, int N>
__global__ void __launch_bounds__(256, tree_min_blocks<T, N>()) k_m2m_tree(DevPlan p, int pb0, const int32_t* __restrict__ child_first,
                                                  const int32_t* __restrict__ child_count, T* __restrict__ E, int Rb) {
    constexpr int N3 = Ord<N>::n3, NS = Ord<N>::ns, RC = tree_rc<T, N>(), NN = N * N;
    const int pb = pb0 + blockIdx.x;
    const int r0 = blockIdx.y * RC;
    const int rc = min(RC, Rb - r0);
    extern __shared__ __align__(16) unsigned char tree_smem_raw[];
    T* A = reinterpret_cast<T*>(tree_smem_raw);  // [8][RC][N3]
    T* B = A + 8 * RC * N3;                      // [4][RC][N3]
    T* C = B + 4 * RC * N3;                      // [2][RC][N3]
    __shared__ T M1[3][2][NN];
    __shared__ int oct_s[8];
    load_m1<T, N>(p.m2m1d, M1);
    const int cf = child_first[pb], cc = child_count[pb];  // cc <= 8 (octree)
    if (threadIdx.x < cc) oct_s[threadIdx.x] = p.box_octant[cf + threadIdx.x];
    for (int e = threadIdx.x; e < 8 * RC * N3; e += blockDim.x) A[e] = (T)0;
    __syncthreads();
    // every child row of the chunk in flight at once, then one wait
    const int per = rc * N3;
    for (int e = threadIdx.x; e < cc * per; e += blockDim.x) {
        const int k = e / per, rm = e - k * per, r = rm / N3, m = rm - r * N3;
        cp_elem(A + (oct_s[k] * RC + r) * N3 + m, E + ((int64_t)(cf + k) * Rb + r0 + r) * NS + m);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    // Each stage runs one 1-D line per thread (the n values along the
    // contracted axis), so the index arithmetic is per line, not per value.
    // z: B[q][r][(a,b,c')] = sum_oz sum_c Z_oz[c'][c] A[q|oz<<2][r][(a,b,c)]
    for (int e = threadIdx.x; e < 4 * RC * NN; e += blockDim.x) {
        const int q = e / (RC * NN), r = (e / NN) % RC, ab = e % NN;
        const T* a0 = A + (q * RC + r) * N3 + ab * N;
        const T* a1 = A + ((q | 4) * RC + r) * N3 + ab * N;
        T x0[N], x1[N];
#pragma unroll
        for (int c = 0; c < N; ++c) {
            x0[c] = a0[c];
            x1[c] = a1[c];
        }
        T* out = B + (q * RC + r) * N3 + ab * N;
#pragma unroll
        for (int cp = 0; cp < N; ++cp) {
            T s = (T)0;
#pragma unroll
            for (int c = 0; c < N; ++c) s += M1[2][0][cp * N + c] * x0[c] + M1[2][1][cp * N + c] * x1[c];
            out[cp] = s;
        }
    }
    __syncthreads();
    // y: C[ox][r][(a,b',c)] = sum_oy sum_b Y_oy[b'][b] B[ox|oy<<1][r][(a,b,c)]
    for (int e = threadIdx.x; e < 2 * RC * NN; e += blockDim.x) {
        const int ox = e / (RC * NN), r = (e / NN) % RC, ac = e % NN, a = ac / N, c = ac % N;
        const T* b0 = B + (ox * RC + r) * N3 + a * NN + c;
        const T* b1 = B + ((ox | 2) * RC + r) * N3 + a * NN + c;
        T x0[N], x1[N];
#pragma unroll
        for (int b = 0; b < N; ++b) {
            x0[b] = b0[b * N];
            x1[b] = b1[b * N];
        }
        T* out = C + (ox * RC + r) * N3 + a * NN + c;
#pragma unroll
        for (int bp = 0; bp < N; ++bp) {
            T s = (T)0;
#pragma unroll
            for (int b = 0; b < N; ++b) s += M1[1][0][bp * N + b] * x0[b] + M1[1][1][bp * N + b] * x1[b];
            out[bp * N] = s;
        }
    }
    __syncthreads();
    // x: E_par[r][(a',b,c)] = sum_ox sum_a X_ox[a'][a] C[ox][r][(a,b,c)]; padding nodes zero
    T* dst = E + ((int64_t)pb * Rb + r0) * NS;
    for (int e = threadIdx.x; e < rc * NN; e += blockDim.x) {
        const int r = e / NN, bc = e % NN;
        const T* c0 = C + r * N3 + bc;
        const T* c1 = C + (RC + r) * N3 + bc;
        T x0[N], x1[N];
#pragma unroll
        for (int a = 0; a < N; ++a) {
            x0[a] = c0[a * NN];
            x1[a] = c1[a * NN];
        }
#pragma unroll
        for (int ap = 0; ap < N; ++ap) {
            T s = (T)0;
#pragma unroll
            for (int a = 0; a < N; ++a) s += M1[0][0][ap * N + a] * x0[a] + M1[0][1][ap * N + a] * x1[a];
            dst[(int64_t)r * NS + ap * NN + bc] = s;
        }
    }
    if constexpr (NS > N3)
        for (int e = threadIdx.x; e < rc * (NS - N3); e += blockDim.x) {
            const int r = e / (NS - N3), m = N3 + e % (NS - N3);
            dst[(int64_t)r * NS + m] = (T)0;
        }
}

// L2L, one CTA per (parent box, chunk of RC rows r): the transposed tree.
// C[ox] = X_ox^T L_par; B[ox|oy<<1] = Y_oy^T C[ox]; child of octant oct:
// L_child += Z_oz^T B[oct & 3].
template <class T, int N>
__global__ void __launch_bounds__(256, tree_min_blocks<T, N>()) k_l2l_tree(DevPlan p, int pb0, const int32_t* __restrict__ child_first,
                                                  const int32_t* __restrict__ child_count, T* __restrict__ L, int Rb) {
    constexpr int N3 = Ord<N>::n3, NS = Ord<N>::ns, RC = tree_rc<T, N>(), NN = N * N;
    const int pb = pb0 + blockIdx.x;
    const int r0 = blockIdx.y * RC;
    const int rc = min(RC, Rb - r0);
    extern __shared__ __align__(16) unsigned char tree_smem_raw[];
    T* Ch = reinterpret_cast<T*>(tree_smem_raw);  // [8][RC][N3]: the children's rows of the chunk
    T* B = Ch + 8 * RC * N3;                      // [4][RC][N3]
    T* C = B + 4 * RC * N3;                       // [2][RC][N3]
    T* P = B;                                     // [RC][N3]: the parent, dead once C is formed
    __shared__ T M1[3][2][NN];
    __shared__ int oct_s[8];
    load_m1<T, N>(p.m2m1d, M1);
    const int cf = child_first[pb], cc = child_count[pb];  // cc <= 8 (octree)
    if (threadIdx.x < cc) oct_s[threadIdx.x] = p.box_octant[cf + threadIdx.x];
    const T* src = L + ((int64_t)pb * Rb + r0) * NS;
    for (int e = threadIdx.x; e < RC * N3; e += blockDim.x) {
        const int r = e / N3, m = e % N3;
        if (r < rc)
            cp_elem(P + e, src + (int64_t)r * NS + m);
        else
            P[e] = (T)0;
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    // The children's current rows, needed only by the last stage: their
    // copies stay in flight through the x and y stages.
    const int per = rc * N3;
    for (int e = threadIdx.x; e < cc * per; e += blockDim.x) {
        const int k = e / per, rm = e - k * per, r = rm / N3, m = rm - r * N3;
        cp_elem(Ch + (k * RC + r) * N3 + m, L + ((int64_t)(cf + k) * Rb + r0 + r) * NS + m);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    __syncthreads();
    // x: C[ox][r][(a,b,c)] = sum_a' X_ox[a'][a] P[r][(a',b,c)]  (one line per thread)
    for (int e = threadIdx.x; e < RC * NN; e += blockDim.x) {
        const int r = e / NN, bc = e % NN;
        const T* pr = P + r * N3 + bc;
        T x[N];
#pragma unroll
        for (int ap = 0; ap < N; ++ap) x[ap] = pr[ap * NN];
#pragma unroll
        for (int ox = 0; ox < 2; ++ox) {
            T* out = C + (ox * RC + r) * N3 + bc;
#pragma unroll
            for (int a = 0; a < N; ++a) {
                T s = (T)0;
#pragma unroll
                for (int ap = 0; ap < N; ++ap) s += M1[0][ox][ap * N + a] * x[ap];
                out[a * NN] = s;
            }
        }
    }
    __syncthreads();
    // y: B[q][r][(a,b,c)] = sum_b' Y_oy[b'][b] C[ox][r][(a,b',c)],  q = ox | oy<<1
    for (int e = threadIdx.x; e < 2 * RC * NN; e += blockDim.x) {
        const int ox = e / (RC * NN), r = (e / NN) % RC, ac = e % NN, a = ac / N, c = ac % N;
        const T* cr = C + (ox * RC + r) * N3 + a * NN + c;
        T x[N];
#pragma unroll
        for (int bp = 0; bp < N; ++bp) x[bp] = cr[bp * N];
#pragma unroll
        for (int oy = 0; oy < 2; ++oy) {
            T* out = B + ((ox | (oy << 1)) * RC + r) * N3 + a * NN + c;
#pragma unroll
            for (int b = 0; b < N; ++b) {
                T s = (T)0;
#pragma unroll
                for (int bp = 0; bp < N; ++bp) s += M1[1][oy][bp * N + b] * x[bp];
                out[b * N] = s;
            }
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    // z, straight into each existing child: L_child[r][(a,b,c)] += sum_c' Z_oz[c'][c] B[oct&3][r][(a,b,c')]
    for (int e = threadIdx.x; e < cc * rc * NN; e += blockDim.x) {
        const int k = e / (rc * NN), r = (e / NN) % rc, ab = e % NN;
        const int ch = cf + k;
        const int oc = oct_s[k], q = oc & 3, oz = oc >> 2;
        const T* br = B + (q * RC + r) * N3 + ab * N;
        const T* old = Ch + (k * RC + r) * N3 + ab * N;
        T x[N];
#pragma unroll
        for (int cp = 0; cp < N; ++cp) x[cp] = br[cp];
        T* dst = L + ((int64_t)ch * Rb + r0 + r) * NS + ab * N;
#pragma unroll
        for (int c = 0; c < N; ++c) {
            T s = (T)0;
#pragma unroll
            for (int cp = 0; cp < N; ++cp) s += M1[2][oz][cp * N + c] * x[cp];
            dst[c] = old[c] + s;
        }
    }
}

// L2L as above, with the children's rows read and written in place by the
// last stage instead of prefetched: faster for FP32, whose prefetch takes
// 4-byte copies.
template <class T, int N>
__global__ void __launch_bounds__(256, tree_min_blocks<T, N>()) k_l2l_tree_inplace(DevPlan p, int pb0, const int32_t* __restrict__ child_first,
                                                  const int32_t* __restrict__ child_count, T* __restrict__ L, int Rb) {
    constexpr int N3 = Ord<N>::n3, NS = Ord<N>::ns, RC = tree_rc<T, N>(), NN = N * N;
    const int pb = pb0 + blockIdx.x;
    const int r0 = blockIdx.y * RC;
    const int rc = min(RC, Rb - r0);
    extern __shared__ __align__(16) unsigned char tree_smem_raw[];
    T* P = reinterpret_cast<T*>(tree_smem_raw);  // [RC][N3]
    T* B = P + 8 * RC * N3;                      // [4][RC][N3]
    T* C = B + 4 * RC * N3;                      // [2][RC][N3]
    __shared__ T M1[3][2][NN];
    load_m1<T, N>(p.m2m1d, M1);
    const T* src = L + ((int64_t)pb * Rb + r0) * NS;
    for (int e = threadIdx.x; e < RC * N3; e += blockDim.x) {
        const int r = e / N3, m = e % N3;
        P[e] = r < rc ? src[(int64_t)r * NS + m] : (T)0;
    }
    __syncthreads();
    // x: C[ox][r][(a,b,c)] = sum_a' X_ox[a'][a] P[r][(a',b,c)]  (one line per thread)
    for (int e = threadIdx.x; e < RC * NN; e += blockDim.x) {
        const int r = e / NN, bc = e % NN;
        const T* pr = P + r * N3 + bc;
        T x[N];
#pragma unroll
        for (int ap = 0; ap < N; ++ap) x[ap] = pr[ap * NN];
#pragma unroll
        for (int ox = 0; ox < 2; ++ox) {
            T* out = C + (ox * RC + r) * N3 + bc;
#pragma unroll
            for (int a = 0; a < N; ++a) {
                T s = (T)0;
#pragma unroll
                for (int ap = 0; ap < N; ++ap) s += M1[0][ox][ap * N + a] * x[ap];
                out[a * NN] = s;
            }
        }
    }
    __syncthreads();
    // y: B[q][r][(a,b,c)] = sum_b' Y_oy[b'][b] C[ox][r][(a,b',c)],  q = ox | oy<<1
    for (int e = threadIdx.x; e < 2 * RC * NN; e += blockDim.x) {
        const int ox = e / (RC * NN), r = (e / NN) % RC, ac = e % NN, a = ac / N, c = ac % N;
        const T* cr = C + (ox * RC + r) * N3 + a * NN + c;
        T x[N];
#pragma unroll
        for (int bp = 0; bp < N; ++bp) x[bp] = cr[bp * N];
#pragma unroll
        for (int oy = 0; oy < 2; ++oy) {
            T* out = B + ((ox | (oy << 1)) * RC + r) * N3 + a * NN + c;
#pragma unroll
            for (int b = 0; b < N; ++b) {
                T s = (T)0;
#pragma unroll
                for (int bp = 0; bp < N; ++bp) s += M1[1][oy][bp * N + b] * x[bp];
                out[b * N] = s;
            }
        }
    }
    __syncthreads();
    // z, straight into each existing child: L_child[r][(a,b,c)] += sum_c' Z_oz[c'][c] B[oct&3][r][(a,b,c')]
    const int cf = child_first[pb], cc = child_count[pb];
    for (int e = threadIdx.x; e < cc * rc * NN; e += blockDim.x) {
        const int k = e / (rc * NN), r = (e / NN) % rc, ab = e % NN;
        const int ch = cf + k;
        const int oc = p.box_octant[ch], q = oc & 3, oz = oc >> 2;
        const T* br = B + (q * RC + r) * N3 + ab * N;
        T x[N];
#pragma unroll
        for (int cp = 0; cp < N; ++cp) x[cp] = br[cp];
        T* dst = L + ((int64_t)ch * Rb + r0 + r) * NS + ab * N;
#pragma unroll
        for (int c = 0; c < N; ++c) {
            T s = (T)0;
#pragma unroll
            for (int cp = 0; cp < N; ++cp) s += M1[2][oz][cp * N + c] * x[cp];
            dst[c] += s;
        }
    }
}

// FP64 M2L with dense operators: CTA per target box, 64 (m) x 64 (r) tile,
// 4x4 register tile per thread, operator and source tiles of 32 along the
// contraction in shared memory.  K table: 343 x n3 x n3; E, L: node stride ns.
__global__ void __launch_bounds__(256) k_m2l64(DevPlan p, int b0, double* __restrict__ L, const double* __restrict__ E,
                                               int R, double scale) {
    const int tb = b0 + blockIdx.x;
    const int n3 = p.n3, ns = p.ns;
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
                const double* Es = E + (int64_t)p.m2l_src[e] * R * ns;
                for (int lc = 0; lc < n3; lc += 32) {
                    __syncthreads();
                    for (int idx = threadIdx.x; idx < 32 * 64; idx += 256) {
                        const int a = idx >> 5, b = idx & 31;  // a: m or r (64), b: l (32)
                        Ks[b][a] = (mc + a < n3 && lc + b < n3) ? K[(int64_t)(mc + a) * n3 + lc + b] : 0.0;
                        Ms[b][a] = (rcn + a < R && lc + b < n3) ? Es[(int64_t)(rcn + a) * ns + lc + b] : 0.0;
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
                    if (mm < n3 && rr < R) L[((int64_t)tb * R + rr) * ns + mm] += scale * acc[i][j];
                }
        }
    }
}

// Factored M2L for low-rank (compressed) operators K_o = U_o Vt_o, in two
// GEMM phases per level:
//   phase 1, per source box s: for every column c = (pair e, k) of the
//     source's outgoing pairs, T[t_e][r][col(e,k)] = sum_l E_s[r][l] Vt_o[k][l];
//   phase 2, per target box t: L_t[r][m] += scale * sum_c T_t[r][c] Ut[c][m],
//     the contraction running over the concatenated ranks of t's pairs.
// T is stored target-major and column-major (Kp_t columns of R values per
// target, Kp_t = the summed ranks rounded up to 4): phase 1 writes each column
// as contiguous rows of R, phase 2 reads contiguous K-chunks.
// Phase 1 as a transposed GEMM per work item (source box, up to
// kFacItemCols of its columns): C[c][r] = sum_l Vt_c[l] E_s[r][l].  E_s^T (B)
// is staged once per item; the gathered Vt rows (A) of each CT-column
// sub-block stream through a cp.async double buffer over the ns nodes.  CT
// threads, 8 x 8 outputs per thread (columns ty + (CT/8) i, rows tx + 8 j).
template <class T, int CT>
__global__ void __launch_bounds__(CT) k_m2l_fac_v(FacM2L<T> f, const int32_t* __restrict__ item_src,
                                                  const int64_t* __restrict__ item_c0,
                                                  const int32_t* __restrict__ item_cnt, const T* __restrict__ E,
                                                  int R) {
    constexpr int V = 16 / sizeof(T);
    constexpr int KC = 128 / sizeof(T);
    constexpr int PP = KC + V;
    constexpr int BP = 64 + 1;  // odd pitch: the transposed staging stores hit distinct banks
    constexpr int CS = CT / 8;  // column stride of a thread's tile
    const int ns = f.ns;
    const int it = blockIdx.x;
    const int rc = blockIdx.y * 64;
    const int s = item_src[it];
    const int64_t cbase = item_c0[it];
    const int ncols = item_cnt[it];
    const int rows = min(64, R - rc);
    extern __shared__ __align__(16) unsigned char fac_smem[];
    T(*As)[CT][PP] = reinterpret_cast<T(*)[CT][PP]>(fac_smem);                        // [2][CT][PP]: [c][l]
    T(*Bs)[BP] = reinterpret_cast<T(*)[BP]>(fac_smem + sizeof(T) * 2 * CT * PP);      // [ns][BP]:  [l][r]
    const int tid = threadIdx.x, tx = tid & 7, ty = tid >> 3;
    const int nch = ns / KC;                      // node chunks per sub-block
    const int nsub = (ncols + CT - 1) / CT;       // CT-column sub-blocks
    const int nsteps = nsub * nch;
    auto issue = [&](int step) {
        const int sub = step / nch, ch = step % nch;
        const int64_t c0 = cbase + (int64_t)CT * sub;
        const int nc = min(CT, ncols - CT * sub);
        const int k0 = ch * KC, buf = step & 1;
#pragma unroll
        for (int q = 0; q < KC / V; ++q) {
            const int id = tid + CT * q, row = id / (KC / V), kc = (id % (KC / V)) * V;
            const bool ok = row < nc;
            cp16(&As[buf][row][kc], ok ? (const void*)(f.Vt + f.col_vt[c0 + row] + k0 + kc) : (const void*)f.Vt, ok);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    issue(0);
    const T* Es = E + ((int64_t)s * R + rc) * ns;
    for (int e = tid; e < 64 * ns; e += CT) {
        const int r = e / ns, l = e % ns;
        Bs[l][r] = r < rows ? Es[(int64_t)r * ns + l] : (T)0;
    }
    T acc[8][8];
    for (int step = 0; step < nsteps; ++step) {
        const int sub = step / nch, ch = step % nch;
        if (ch == 0) {
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = (T)0;
        }
        __syncthreads();
        if (step + 1 < nsteps) {
            issue(step + 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        const int buf = step & 1;
#pragma unroll 4
        for (int kk = 0; kk < KC; ++kk) {
            T a[8], b[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[buf][ty + CS * i][kk];
#pragma unroll
            for (int j = 0; j < 8; ++j) b[j] = Bs[ch * KC + kk][tx + 8 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] += a[i] * b[j];
        }
        if (ch == nch - 1) {
            const int64_t c0 = cbase + (int64_t)CT * sub;
            const int nc = min(CT, ncols - CT * sub);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int c = ty + CS * i;
                if (c >= nc) continue;
                const int tg = f.col_tgt[c0 + c];
                T* dst = f.Tm + (f.tgt_base[tg] + f.col_pos[c0 + c]) * R + rc;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int r = tx + 8 * j;
                    if (r < rows) dst[r] = acc[i][j];
                }
            }
        }
    }
}

// Phase 2: CTA per (target box, 64 rows r, MW nodes m), MW threads, 8 x 8
// outputs per thread (rows ty + 8 i, nodes tx + (MW/8) j); the contraction
// over the target's concatenated ranks streams A = T rows and B = gathered Ut
// rows through a cp.async double buffer.
template <class T, int MW>
__global__ void __launch_bounds__(MW) k_m2l_fac_u(FacM2L<T> f, int b0, T* __restrict__ L, int R, double scale) {
    constexpr int V = 16 / sizeof(T);
    constexpr int KC = 128 / sizeof(T);
    constexpr int XP = MW + V;
    constexpr int AP = 64 + V;
    constexpr int TXN = MW / 8;
    const int ns = f.ns;
    const int t = b0 + blockIdx.x;
    const int rc = blockIdx.y * 64;
    const int m0 = blockIdx.z * MW;
    const int64_t k0g = f.tgt_col_off[t], K = f.tgt_col_off[t + 1] - k0g;
    if (K == 0) return;
    const int Kp = (int)((K + 3) & ~int64_t(3));
    const T sc = (T)(f.box_scale ? f.box_scale[t] : scale);
    const T* A = f.Tm + f.tgt_base[t] * R + rc;  // column-major: A[c][r] at c * R + r
    const int m = min(64, R - rc);
    extern __shared__ __align__(16) unsigned char facu_smem[];
    T(*As)[KC][AP] = reinterpret_cast<T(*)[KC][AP]>(facu_smem);                     // [2][KC][AP]: [c][r]
    T(*Bs)[KC][XP] = reinterpret_cast<T(*)[KC][XP]>(facu_smem + sizeof(T) * 2 * KC * AP);  // [2][KC][XP]
    const int tid = threadIdx.x, tx = tid % TXN, ty = tid / TXN;
    const int nchunk = (Kp + KC - 1) / KC;
    auto issue = [&](int cch) {
        const int k0 = cch * KC, buf = cch & 1;
        for (int id = tid; id < KC * (64 / V); id += MW) {
            const int kk = id / (64 / V), rr = (id % (64 / V)) * V;
            const bool ok = k0 + kk < Kp && rr < m;
            cp16(&As[buf][kk][rr], ok ? (const void*)(A + (int64_t)(k0 + kk) * R + rr) : (const void*)f.Tm, ok);
        }
        for (int id = tid; id < KC * (MW / V); id += MW) {
            const int kk = id / (MW / V), cc = (id % (MW / V)) * V;
            const bool ok = k0 + kk < K && m0 + cc < ns;
            cp16(&Bs[buf][kk][cc], ok ? (const void*)(f.Ut + f.tgt_ut[k0g + k0 + kk] + m0 + cc) : (const void*)f.Ut,
                 ok);
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
            for (int i = 0; i < 8; ++i) a[i] = As[buf][kk][ty + 8 * i];
#pragma unroll
            for (int j = 0; j < 8; ++j) b[j] = Bs[buf][kk][tx + TXN * j];
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
            const int mm = m0 + tx + TXN * j;
            if (mm >= ns) continue;
            T* dst = L + ((int64_t)t * R + rc + r) * ns + mm;
            *dst += sc * acc[i][j];
        }
    }
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

template <class T, int N>
void far_field_n(Ctx& c, const DevPlan& p, const FarLaunch& f, const T* X, const FarWeights<T>& w, double* Y, int R,
                 int Rb, T* E, T* L, double coef, const M2LLevelFn<T>& m2l, bool m2l_all, const P2MSplit* p2m_tc,
                 bool l_written) {
    cudaStream_t s = c.stream;
    constexpr int N3 = Ord<N>::n3, NS = Ord<N>::ns, RC = tree_rc<T, N>();
    constexpr size_t smem = tree_smem<T, N>();
    const int Lv = p.L;
    const double wb = (double)sizeof(T);
    const double box_bytes = wb * N3 * R;
    const unsigned rchunks64 = cdiv(Rb, 64), rchunks_tree = cdiv(Rb, RC);
    if (!l_written)
        launch_zero(c, L, (size_t)p.nbox * NS * Rb * sizeof(T));  // a kernel: also valid inside a device-side loop
    {
        KTimer t(c, prec_tag<T>(K_P2M), (double)p.N * (wb * R + wb * N3 + 8.0) + (p.nleaf + 2.0 * f.npart) * box_bytes,
                 2.0 * (double)p.N * N3 * R);
        if constexpr (sizeof(T) == 4 && (N == 4 || N == 5)) {
            if (p2m_tc) {
                launch_p2m_tc(c, p, f.p2m_slot, p2m_tc->whi, p2m_tc->wlo, p2m_tc->xhi, p2m_tc->xlo,
                              reinterpret_cast<float*>(E), R, Rb, p2m_tc->err);
            } else {
                k_p2m<T, N><<<dim3(p.nitems, rchunks64), 256, 0, s>>>(p, f.p2m_slot, X, w.src, w.src_area, E, R, Rb);
                GPX_LAUNCH_CHECK();
                c.launches += 1;
            }
        } else {
            k_p2m<T, N><<<dim3(p.nitems, rchunks64), 256, 0, s>>>(p, f.p2m_slot, X, w.src, w.src_area, E, R, Rb);
            GPX_LAUNCH_CHECK();
            c.launches += 1;
        }
        if (f.nfix > 0) {
            const int64_t block = (int64_t)Rb * NS;
            k_p2m_fix<T><<<dim3(f.nfix, cdiv(block, 1024)), 256, 0, s>>>(p.nbox, p.leaf_box0, f.fix_leaf, f.fix_first,
                                                                         f.fix_cnt, E, block);
            GPX_LAUNCH_CHECK();
            c.launches += 1;
        }
    }
    if (smem > 48 * 1024) {
        set_smem_once(k_m2m_tree<T, N>, (int)smem);
        set_smem_once(k_l2l_tree<T, N>, (int)smem);
        set_smem_once(k_l2l_tree_inplace<T, N>, (int)smem);
    }
    for (int l = Lv; l >= 3; --l) {
        const int pb0 = f.lvl_off[l - 1], npb = f.lvl_off[l] - pb0, nch = f.lvl_off[l + 1] - f.lvl_off[l];
        if (npb == 0) continue;
        KTimer t(c, prec_tag<T>(K_M2M), (double)(npb + nch) * box_bytes, 2.0 * 14.0 * N * N3 * R * (double)npb);
        k_m2m_tree<T, N><<<dim3(npb, rchunks_tree), 256, smem, s>>>(p, pb0, f.child_first, f.child_count, E, Rb);
        GPX_LAUNCH_CHECK();
        c.launches += 1;
    }
    if (m2l_all && Lv >= 2) {
        const int b0 = f.lvl_off[2], nb = f.lvl_off[Lv + 1] - b0;
        const double pairs = (double)(f.m2l_off[b0 + nb] - f.m2l_off[b0]);
        if (pairs > 0) {
            KTimer t(c, prec_tag<T>(K_M2L), 2.0 * nb * box_bytes, 2.0 * (double)N3 * N3 * R * pairs);
            m2l(-1, b0, nb, 0.0);
            c.launches += 1;
        }
    } else {
        for (int l = 2; l <= Lv; ++l) {
            const int b0 = f.lvl_off[l], nb = f.lvl_off[l + 1] - b0;
            if (nb == 0) continue;
            const double pairs = (double)(f.m2l_off[b0 + nb] - f.m2l_off[b0]);
            if (pairs == 0) continue;
            KTimer t(c, prec_tag<T>(K_M2L), 2.0 * nb * box_bytes, 2.0 * (double)N3 * N3 * R * pairs);
            m2l(l, b0, nb, 1.0 / f.lvl_half[l]);
            c.launches += 1;
        }
    }
    for (int l = 2; l < Lv; ++l) {
        const int pb0 = f.lvl_off[l], npb = f.lvl_off[l + 1] - pb0, ncb = f.lvl_off[l + 2] - f.lvl_off[l + 1];
        if (ncb == 0) continue;
        KTimer t(c, prec_tag<T>(K_L2L), (double)(npb + 2 * ncb) * box_bytes, 2.0 * 14.0 * N * N3 * R * (double)npb);
        if constexpr (sizeof(T) == 4)
            k_l2l_tree_inplace<T, N><<<dim3(npb, rchunks_tree), 256, smem, s>>>(p, pb0, f.child_first, f.child_count,
                                                                               L, Rb);
        else
            k_l2l_tree<T, N><<<dim3(npb, rchunks_tree), 256, smem, s>>>(p, pb0, f.child_first, f.child_count, L, Rb);
        GPX_LAUNCH_CHECK();
        c.launches += 1;
    }
    {
        KTimer t(c, prec_tag<T>(K_L2P), (double)p.N * (16.0 * R + 24.0 * N) + p.nleaf * box_bytes, 2.0 * (double)p.N * N3 * R);
        bool done = false;
        if constexpr (sizeof(T) == 4 && (N == 4 || N == 5)) {
            if (p2m_tc && p2m_tc->shi) {
                launch_l2p_tc(c, p, reinterpret_cast<const float*>(L), p2m_tc->shi, p2m_tc->slo, Y, R, Rb, coef,
                              p2m_tc->err);
                done = true;
            }
        }
        if (!done) {
            k_l2p<T, N><<<dim3(p.nitems, cdiv(R, 64)), 256, 0, s>>>(p, L, w.tgt, w.tgt_area, Y, R, Rb, coef);
            GPX_LAUNCH_CHECK();
            c.launches += 1;
        }
    }
}

}  // namespace

template <class T>
void launch_far_field(Ctx& c, const DevPlan& p, const FarLaunch& f, const T* X, const FarWeights<T>& w, double* Y,
                      int R, int Rb, T* E, T* L, double coef, const M2LLevelFn<T>& m2l, bool m2l_all,
                      const P2MSplit* p2m_tc, bool l_written) {
    switch (p.n) {
        case 2: far_field_n<T, 2>(c, p, f, X, w, Y, R, Rb, E, L, coef, m2l, m2l_all, p2m_tc, l_written); break;
        case 3: far_field_n<T, 3>(c, p, f, X, w, Y, R, Rb, E, L, coef, m2l, m2l_all, p2m_tc, l_written); break;
        case 4: far_field_n<T, 4>(c, p, f, X, w, Y, R, Rb, E, L, coef, m2l, m2l_all, p2m_tc, l_written); break;
        case 5: far_field_n<T, 5>(c, p, f, X, w, Y, R, Rb, E, L, coef, m2l, m2l_all, p2m_tc, l_written); break;
        case 6: far_field_n<T, 6>(c, p, f, X, w, Y, R, Rb, E, L, coef, m2l, m2l_all, p2m_tc, l_written); break;
        default: throw Error(GPX_ERR_INVALID_ARG, "far field runs Chebyshev orders 2 to 6");
    }
}

template <class T>
void launch_m2l_fac(Ctx& c, const FacM2L<T>& f, const FacLevel& lv, int b0, int nb, T* L, const T* E, int R,
                    double scale) {
    constexpr int V = 16 / sizeof(T), KC = 128 / sizeof(T);
    constexpr int CT = 128;
    const int smem_v = (int)(sizeof(T) * (2 * CT * (KC + V) + f.ns * (64 + 1)));
    if (lv.nitems > 0) {
        set_smem_once(k_m2l_fac_v<T, CT>, smem_v);
        k_m2l_fac_v<T, CT><<<dim3(lv.nitems, cdiv(R, 64)), CT, smem_v, c.stream>>>(f, lv.item_src, lv.item_c0,
                                                                                    lv.item_cnt, E, R);
    }
    GPX_LAUNCH_CHECK();
    if (f.ns >= 128) {
        constexpr int MW = 128;
        const int smem_u = (int)(sizeof(T) * (2 * KC * (64 + V) + 2 * KC * (MW + V)));
        set_smem_once(k_m2l_fac_u<T, MW>, smem_u);
        k_m2l_fac_u<T, MW><<<dim3(nb, cdiv(R, 64), cdiv(f.ns, MW)), MW, smem_u, c.stream>>>(f, b0, L, R, scale);
    } else {
        constexpr int MW = 64;
        const int smem_u = (int)(sizeof(T) * (2 * KC * (64 + V) + 2 * KC * (MW + V)));
        set_smem_once(k_m2l_fac_u<T, MW>, smem_u);
        k_m2l_fac_u<T, MW><<<dim3(nb, cdiv(R, 64), cdiv(f.ns, MW)), MW, smem_u, c.stream>>>(f, b0, L, R, scale);
    }
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

template void launch_far_field<double>(Ctx&, const DevPlan&, const FarLaunch&, const double*,
                                       const FarWeights<double>&, double*, int, int, double*, double*, double,
                                       const M2LLevelFn<double>&, bool, const P2MSplit*, bool);
template void launch_far_field<float>(Ctx&, const DevPlan&, const FarLaunch&, const float*, const FarWeights<float>&,
                                      double*, int, int, float*, float*, double, const M2LLevelFn<float>&, bool,
                                      const P2MSplit*, bool);

}  // namespace gpx
