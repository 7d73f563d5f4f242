// Far-field (Chebyshev FMM) launch interface shared by the FP64 and FP32 paths.
#pragma once
#include <functional>

#include "kernels.cuh"

namespace gpx {

// Runs the M2L translations of one level: (level, first box, box count, 1/half).
template <class T>
using M2LLevelFn = std::function<void(int, int, int, double)>;

// Weights of the far field's two ends.  P2M: E[leaf][r][m] = sum_j src[j][m]
// (a_j if src_area) X[j][r]; L2P: Y[j][r] += coef sum_m tgt[j][m] (a_j if
// tgt_area) L[leaf][r][m], where tgt = null means the separable collocation
// weights S(c_j) of the panel centroid (from the plan's 1-D weights).  The
// operator P uses (W, area) at P2M and (S(c), none) at L2P; its transpose uses
// (S(c) as an array, none) at P2M and (W, area) at L2P.
template <class T>
struct FarWeights {
    const T* src = nullptr;  // N x n3
    bool src_area = true;
    const T* tgt = nullptr;  // N x n3 or null
    bool tgt_area = false;
};

// Y += coef * far-field potential of X (N x R, type T).  Expansions E and L:
// nbox x Rb x ns each (Rb >= R rows per box, node stride ns); E is written in
// full by P2M and M2M (zero padding rows and nodes), L is zeroed here.  M2L is
// supplied per level.
// m2l_all_levels: the M2L callback runs once for every level (level -1,
// first box of level 2, box count of levels 2..L) instead of once per level.
// Inputs of the tensor-core P2M (p2m_tc.cu): the source weights (area
// folded in) and the charges, each split into TF32 hi and lo parts; weight
// rows have a stride of 128 nodes.
struct P2MSplit {
    const float* whi = nullptr;
    const float* wlo = nullptr;
    const float* xhi = nullptr;
    const float* xlo = nullptr;
    int* err = nullptr;
    // L2P on the tensor cores too when given: the target weights split into
    // TF32 hi and lo parts (rows of 128 nodes)
    const float* shi = nullptr;
    const float* slo = nullptr;
};
template <class T>
void launch_far_field(Ctx& c, const DevPlan& p, const FarLaunch& f, const T* X, const FarWeights<T>& w, double* Y,
                      int R, int Rb, T* E, T* L, double coef, const M2LLevelFn<T>& m2l, bool m2l_all_levels = false,
                      const P2MSplit* p2m_tc = nullptr, bool l_written = false);
// l_written: the M2L callback overwrites every local-expansion row of levels
// 2 and deeper (the shared-basis decompression does), and L's rows of levels
// 0 and 1 are zero: L is then not cleared before the M2L.
// Whi / Wlo [N][128] = TF32 split of (area if mul_area) x W[N][n3] (n3 <= 128).
void launch_split_weights(Ctx& c, const double* W, int n3, const double* area, bool mul_area, float* Whi, float* Wlo,
                          int64_t N);
// Y += coef L2P of the far-field locals L with split target weights (orders 4 and 5).
void launch_l2p_tc(Ctx& c, const DevPlan& p, const float* L, const float* Shi, const float* Slo, double* Y, int R,
                   int Rb, double coef, int* err);
// E[leaf or partial slot] = P2M of the split weights and charges (orders 4 and 5).
void launch_p2m_tc(Ctx& c, const DevPlan& p, const int32_t* slot, const float* Whi, const float* Wlo, const float* Xhi,
                   const float* Xlo, float* E, int R, int Rb, int* err);

// FP64 M2L of one level with CUDA-core FMAs (dense operators).
void launch_m2l64(Ctx& c, const DevPlan& p, int b0, int nb, double* L, const double* E, int R, double scale);

// Factored M2L data (orders 4-6, ranks <= kFacMaxRank): low-rank factors of
// every offset, per-source column lists for phase 1 and per-target B-row lists
// for phase 2.
constexpr int kFacMaxRank = 32;
template <class T>
struct FacM2L {
    int ns = 64;                        // node stride
    const T* Vt = nullptr;              // 343 x 32 x ns, row k of slot o = Vt_o[k][:]
    const T* Ut = nullptr;              // 343 x 32 x ns, row k of slot o = U_o[:][k]
    const int64_t* src_col_off = nullptr;  // nbox + 1: phase-1 columns of each source box
    const int64_t* col_vt = nullptr;    // per column: offset of its Vt row
    const int32_t* col_tgt = nullptr;   // per column: target box
    const int32_t* col_pos = nullptr;   // per column: column in the target's T block
    const int64_t* tgt_col_off = nullptr;  // nbox + 1: phase-2 contraction range of each target
    const int64_t* tgt_ut = nullptr;    // per contraction index: offset of its Ut row
    const int64_t* tgt_base = nullptr;  // nbox: sum of padded block widths of earlier boxes
    T* Tm = nullptr;                    // target-major intermediate (Kp columns of R values per target)
    const double* box_scale = nullptr;  // per box: 1 / half-width of its level (all-levels launches)
};
// Phase-1 work items of one level: (source box, first column, column count <= kFacItemCols).
constexpr int kFacItemCols = 512;
struct FacLevel {
    int nitems = 0;
    const int32_t* item_src = nullptr;
    const int64_t* item_c0 = nullptr;
    const int32_t* item_cnt = nullptr;
};
// M2L of one level with the factored operators (two kernels).
template <class T>
void launch_m2l_fac(Ctx& c, const FacM2L<T>& f, const FacLevel& lv, int b0, int nb, T* L, const T* E, int R,
                    double scale);

// Tensor-core (tcgen05, TF32 inputs, FP32 accumulation) M2L work list of one
// level: pairs of target boxes sharing one offset loop.
// Target boxes per tensor-core M2L work item (of one octant class, so that
// their interaction lists use the same offsets): 2, one TMEM accumulator.
// Four boxes with two accumulators sharing each operator tile measured
// slower on the bench window (0.385 against 0.309 ms per launch: half the
// CTAs per SM by shared memory, and more zero-filled rows in the union of
// four boxes' offsets).
constexpr int kGroup = 2;
struct TcLevel {
    int nitems = 0;
    const int32_t* item_t = nullptr;    // kGroup per item: target boxes (trailing ones may be -1)
    const int32_t* item_off = nullptr;  // nitems + 1: entry ranges
    const int32_t* slot = nullptr;      // per entry: operator slot
    const int32_t* src = nullptr;       // kGroup per entry: each target's source box at the slot's offset, or -1
};
// L[t][r][m] = scale * sum K[m][l] E[s][r][l] for order-4 (node stride 64)
// or order-5 (node stride 128) expansions; K32: 343 x ns x ns TF32-rounded
// operators; R a multiple of 64.  err receives a nonzero code if a bounded
// wait on the tensor-core pipeline expired.  box_scale (per box, may be null):
// each target box's own scale, for launches that cover several levels.
void launch_m2l_tc(Ctx& c, const TcLevel& lv, int ns, const float* E, float* L, const float* K32, int R, float scale,
                   const double* box_scale, int* err);

// Shared-basis M2L (SharedBasis in plan.h), rank kShared: expansion rows
// (box, right-hand side) [row0, row0 + nrows) compressed, E^ = V^T E, and
// decompressed, L = U L^, on the tensor cores with both operands split into
// TF32 hi and lo parts.  Vt_hi / Vt_lo: kShared x ns (V^T, zero columns past
// n3); U_hi / U_lo: round_up(ns, 64) x kShared (U, zero rows past n3).  E / L
// rows have stride ns, E^ / L^ rows stride kShared.  *err becomes nonzero if
// a bounded pipeline wait expired.
constexpr int kShared = 64;
void launch_m2l_compress(Ctx& c, const float* E, int ns, const float* Vt_hi, const float* Vt_lo, float* Eh,
                         int64_t row0, int64_t nrows, int* err);
void launch_m2l_decompress(Ctx& c, const float* Lh, const float* U_hi, const float* U_lo, int ns, float* L,
                           int64_t row0, int64_t nrows, int* err);

}  // namespace gpx
