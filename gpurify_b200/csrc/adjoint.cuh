// Launch wrappers of the adjoint-sensitivity and transposed-operator kernels
// (adjoint.cu).  All arrays are in the plan's leaf-sorted panel order.
#pragma once
#include <algorithm>

#include "kernels.cuh"

namespace gpx {

// dcent (N x 3), darea (N): derivatives of the panel centroids and areas along
// the vertex velocity field V (N x 12).
void launch_panel_dprops(Ctx& c, const DevPlan& p, const double* V, double* dcent, double* darea);
// dP (nnz, layout of the near blocks) = coef * derivative of the Wilton near
// blocks along V (sources) and dcent (collocation points).
void launch_near_assemble_dual(Ctx& c, const DevPlan& p, int64_t nnz, const double* V, const double* dcent,
                               double* dP, double coef);
// dW (N x n3) = derivative of (area * far-field source weights) along V.
void launch_dsrc_weights(Ctx& c, const DevPlan& p, int quad, const double* V, double* dW);
// out (N x n3) = Chebyshev weights of each centroid in its leaf (dcent null)
// or their derivative along dcent.
void launch_centroid_weights(Ctx& c, const DevPlan& p, const double* dcent, double* out);
// PT = transposed near blocks of P (same block layout).
void launch_near_transpose(Ctx& c, const DevPlan& p, const int32_t* near_rev, const int32_t* near_pre,
                           const double* P, double* PT, int64_t nnz);
// Splits of the panel range per row in launch_grad_contract: about two
// blocks per SM over the Ra rows.
inline int grad_contract_splits(int Ra) { return std::max(1, std::min(64, 296 / std::max(1, Ra))); }
// G (Ra x R) = da^T [cond == row] X - Lam^T D over the N panels; Gp is scratch
// of grad_contract_splits(Ra) x Ra x R doubles.
void launch_grad_contract(Ctx& c, const int32_t* cond, const int32_t* row_cond, const double* darea,
                          const double* X, const double* Lam, const double* D, int64_t N, int R, int Ra, double* Gp,
                          double* G);

}  // namespace gpx
