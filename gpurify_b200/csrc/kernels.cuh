// Device-side view of a plan and the launch wrappers of the FP64 kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "gpx_common.h"

namespace gpx {

// Device pointers of one uploaded plan (all arrays in leaf-sorted order).
struct DevPlan {
    int n, n3, L;
    int ns;                   // node stride of one expansion row: n3 rounded up to a multiple of 32
    int64_t N;
    int32_t nleaf, nbox, leaf_box0, nitems;
    const double* verts;      // 12 per panel
    const double* cent;       // 3 per panel
    const double* area;
    const int32_t* cond;
    const double* w1d;        // 3*n per panel
    const int64_t* leaf_begin;
    const int32_t* near_off;
    const int32_t* near_src;
    const int32_t* near_S;
    const int64_t* nval_off;
    const int32_t* item_leaf;  // near-field work items (leaf, first row), <= 64 rows each
    const int32_t* item_row0;
    const int32_t* box_parent;
    const int32_t* box_octant;
    const int64_t* m2l_off;
    const int32_t* m2l_src;
    const int32_t* m2l_slot;
    const double* m2m1d;      // 24 n x n
    const double* m2l_K;      // 343 n3 x n3 (FP64 table)
    const double* leaf_ctr;   // 3 per leaf: box centre
    const int32_t* leaf_of;   // per panel: its leaf
    double leaf_half;
    double roots[8];          // Chebyshev roots of order n
    const double* wsrc;       // N x n3 far-field source weights (P2M), set by launch_src_weights
};

// Source ranges of target leaf t's near list, read by the 32 lanes of one
// warp in parallel: s_beg[e] = first panel of near leaf e, s_pre[e] = its
// offset in the concatenated source order (s_pre[ne] = S).  A near list has
// at most 27 leaves (the leaf and its 26 neighbours).
__device__ __forceinline__ void near_ranges_warp(const DevPlan& p, int t, int lane, int64_t* s_beg, int32_t* s_pre) {
    const int e0 = p.near_off[t], ne = p.near_off[t + 1] - e0;
    int64_t b = 0;
    int cnt = 0;
    if (lane < ne) {
        const int src = p.near_src[e0 + lane];
        b = p.leaf_begin[src];
        cnt = (int)(p.leaf_begin[src + 1] - b);
    }
    int inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane < ne) {
        s_beg[lane] = b;
        s_pre[lane] = inc - cnt;
    }
    if (lane == ne - 1) s_pre[ne] = inc;
}

// Wilton near-field block assembly: P (nnz doubles), one CTA per target leaf.
void launch_near_assemble(Ctx& c, const DevPlan& p, int64_t nnz, double* P, double coef);
// inv_diag[i] = 1 / P_ii (|P_ii| > 1e-30 else 1), the reference's DiagJacobi.
void launch_diag_inv(Ctx& c, const DevPlan& p, const double* P, double* inv_diag);
// Y = P_near X (overwrite), X/Y are N x R row-major.
void launch_near_apply(Ctx& c, const DevPlan& p, int64_t nnz, const double* P, const double* X, double* Y, int R);
// Node stride of an expansion row for Chebyshev order n: n^3 rounded up to a
// multiple of 32 (64, 128, 224 for orders 4, 5, 6), so every row is 128-byte
// aligned and a whole number of 32-node contraction chunks.
inline int node_stride(int n) { return (n * n * n + 31) & ~31; }

// Host-side level table plus device child ranges used to sequence the far field.
struct FarLaunch {
    const int32_t* lvl_off;      // host, L+2 entries
    const double* lvl_half;      // host, L+1 entries
    const int32_t* child_first;  // device, per box
    const int32_t* child_count;  // device, per box
    const int32_t* leaf_of;      // device, per sorted panel
    const int64_t* m2l_off;      // host, per box (pair counts per level)
    // P2M over the near-field work items: each item's expansion slot (-1:
    // the item writes its leaf's expansion; k >= 0: partial at box nbox + k),
    // and per leaf with several items the partials k_p2m_fix adds to it.
    const int32_t* p2m_slot;     // device, per near item
    const int32_t* fix_leaf;     // device, per leaf with several items
    const int32_t* fix_first;    // device: its first partial slot
    const int32_t* fix_cnt;      // device: its number of partials
    int nfix = 0, npart = 0;
};
// Y = P_near X with an FP32 copy of P, FP32 input and arithmetic (Y is FP64).
// R must be a multiple of 4 (16-byte aligned rows).
void launch_near_apply32(Ctx& c, const DevPlan& p, int64_t nnz, const float* P, const float* X, double* Y, int R);
// b = (float) a
void launch_to_f32(Ctx& c, const double* a, float* b, int64_t n);
// b = a rounded to TF32 (round to nearest), stored as FP32.
void launch_to_tf32(Ctx& c, const double* a, float* b, int64_t n);
// Y = P_near X on the tensor cores (TF32 inputs, FP32 accumulation, FP64 Y),
// work items of <= 128 rows (it_leaf, it_row0); P holds TF32-rounded values;
// X is given as its TF32 split Xhi + Xlo (launch_split_tf32), or with Xlo
// null as its FP32 copy in Xhi, split into hi and lo on chip; R a multiple
// of 4.  *err becomes nonzero if a bounded pipeline wait expired.
// split_p: P holds full FP32 values and is split into TF32 hi and lo parts on
// chip (three products instead of two; accurate to about 2^-21 in P too).
void launch_near_apply_tc(Ctx& c, const DevPlan& p, int64_t nnz, int nitems, const int32_t* it_leaf,
                          const int32_t* it_row0, const float* P, const float* Xhi, const float* Xlo, double* Y, int R,
                          int* err, bool split_p = false);
// X32 = (float) X, and its TF32 split Xhi = tf32(X), Xlo = tf32(X - Xhi)
// (n values each).
void launch_split_tf32(Ctx& c, const double* X, float* X32, float* Xhi, float* Xlo, int64_t n);
// Far-field source weights W[j][m]: the Chebyshev interpolation weights of
// panel j's charge in its leaf; quad 0: at the centroid (the reference's
// point lumping), quad 1: averaged over 2x2 Gauss points of the panel.
void launch_src_weights(Ctx& c, const DevPlan& p, int quad, double* W);
// Dense all-pairs block for arbitrary target points.
void launch_potential_matrix(Ctx& c, const double* src_verts, int64_t ns, const double* pts, int64_t nt, double* out,
                             double coef);

}  // namespace gpx
