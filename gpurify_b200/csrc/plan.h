// Host-built plan of one panel problem: leaf-sorted panels, uniform octree,
// near-field block structure and M2L interaction lists.  Everything the
// device kernels index is laid out as flat arrays here and uploaded once.
#pragma once
#include <cstdint>
#include <vector>

#include "gpx_common.h"

namespace gpx {

struct Plan {
    int n = 4;        // Chebyshev order
    int n3 = 64;      // nodes per box
    int L = 4;        // leaf level (uniform depth)
    int64_t N = 0;    // panels
    int ncond = 0;
    bool far = true;  // false: every pair is near (all-pairs path)

    // Panels in leaf-sorted order.
    std::vector<int32_t> perm;   // sorted position -> caller index
    std::vector<double> verts;   // 12 per panel
    std::vector<double> cent;    // 3 per panel (reference centroid, bit-exact)
    std::vector<double> area;    // per panel
    std::vector<int32_t> cond;   // per panel
    std::vector<double> w1d;     // 3*n per panel: 1-D Chebyshev weights in its leaf

    // Boxes, level by level; within a level sorted by Morton key of the cell.
    std::vector<int32_t> lvl_off;   // L+2 entries: boxes of level l are [lvl_off[l], lvl_off[l+1])
    std::vector<int32_t> box_cell;  // 3 per box
    std::vector<int32_t> box_parent;
    std::vector<int32_t> box_octant;
    std::vector<double> lvl_half;   // per level
    double origin[3] = {0, 0, 0};    // low corner of the root box
    std::vector<int32_t> child_first, child_count;  // per box: contiguous child range (next level)

    // Leaves (level L): leaf k is box lvl_off[L] + k; panels [leaf_begin[k], leaf_begin[k+1]).
    std::vector<int64_t> leaf_begin;
    std::vector<int32_t> leaf_of;   // per sorted panel: its leaf index
    int32_t max_leaf = 0;

    // Near field: per target leaf, the source leaves (self first, then the
    // existing neighbours in dx,dy,dz order), and the dense block offsets.
    std::vector<int32_t> near_off;    // nleaf+1
    std::vector<int32_t> near_src;    // leaf indices
    std::vector<int32_t> near_S;      // total source panels per target leaf
    std::vector<int64_t> nval_off;    // nleaf+1: value offset of each leaf's m_t x Sp_t block (Sp = S rounded up to 4)
    int32_t max_S = 0;
    // Near-field work items: (target leaf, first row), at most kRowsPerItem rows each.
    static constexpr int kRowsPerItem = 64;
    std::vector<int32_t> item_leaf, item_row0;

    // M2L: per target box (global box index), sources + operator slot.
    std::vector<int64_t> m2l_off;     // nbox+1
    std::vector<int32_t> m2l_src;
    std::vector<int32_t> m2l_slot;    // ((ox+3)*7+oy+3)*7+oz+3

    // Tensor-product M2M operators: 24 n x n matrices (octant*3+axis),
    // mat[m*n+k] = weight of child node k on parent node m (bbfmm.rs:89-112).
    std::vector<double> m2m1d;

    int64_t nleaf() const { return (int64_t)leaf_begin.size() - 1; }
    int64_t nbox() const { return (int64_t)lvl_off.back(); }
    int64_t nnz() const { return nval_off.empty() ? 0 : nval_off.back(); }  // stored entries (incl. row padding)
    int64_t near_pairs() const {
        int64_t s = 0;
        for (size_t k = 0; k + 1 < leaf_begin.size(); ++k) s += (leaf_begin[k + 1] - leaf_begin[k]) * near_S[k];
        return s;
    }
    int64_t m2l_pairs() const { return m2l_off.empty() ? 0 : m2l_off.back(); }
};

// Build the plan.  depth >= 1; depth 1 makes every pair near.
void build_plan(Plan& p, int64_t n, const double* verts, const int32_t* cond, int ncond, int order, int depth);

// Area-weighted fan centroid and area of one panel (integrals/panel.rs:29-67).
void panel_centroid_area(const double* v, double* c, double* a);

// Chebyshev roots and 1-D interpolation weights (fmm/chebyshev.rs:11-74).
std::vector<double> cheb_roots(int n);
void cheb_weights(double x, int n, const double* roots, double* out);

// M2L operator table for order n: 343 slots of n^3 x n^3 (row = target node,
// col = source node), for offsets with max|o| >= 2; dimensionless (reference
// coordinates, multiply by 1/half at use).  mode 0: QR-compressed as the
// reference (bbfmm.rs:132-174, linalg.rs:277-381), stored as the product
// U*V^T; mode 1: the exact kernel matrix.
struct M2LTable {
    int n = 0, mode = 0;
    std::vector<double> K;      // 343 * n3 * n3
    std::vector<int32_t> rank;  // per slot (n3 for exact; -1 unused)
    // Compressed mode: the factors, K = U * Vt, stored with a fixed stride of
    // n3 columns (U: n3 x n3, first rank columns used) and n3 rows (Vt: first
    // rank rows used).
    std::vector<double> U, Vt;  // 343 * n3 * n3 each
};
void build_m2l_table(M2LTable& t, int n, int mode);

// Shared-basis compression of a table's M2L operators (the mixed path's
// far field): one target basis U and one source basis V (n3 x r each,
// orthonormal columns) for every offset, K_o ~ U C_o V^T with the r x r
// core C_o = U^T K_o V.  U spans the dominant r-dimensional range of all K_o
// together (the leading eigenvectors of sum_o K_o K_o^T), V their dominant
// row space (of sum_o K_o^T K_o).  Then M2L runs on compressed expansions:
// E^ = V^T E per source box, L^ += C_o E^ per pair, L = U L^ per target box.
struct SharedBasis {
    int n = 0, mode = 0, r = 0;
    std::vector<double> U, V;  // n3 x r, row-major
    std::vector<double> C;     // 343 x r x r (zero for slots that are not M2L offsets)
    double rel_err = 0.0;      // max over slots of ||K_o - U C_o V^T||_F / ||K_o||_F
};
void build_shared_basis(const M2LTable& t, int r, SharedBasis& out);

}  // namespace gpx
