// Multi-RHS GMRES building blocks (declarations).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "gpx_common.h"

namespace gpx {

// Per-column GMRES scalars on the device (one column per right-hand side).
struct GmresDev {
    int m, R;
    double tol;
    double* H;       // (m+1) x m x R : H[(i*m + k)*R + r]
    double* cs;      // m x R
    double* sn;      // m x R
    double* g;       // (m+1) x R
    double* y;       // m x R
    double* h1;      // (m+1) x R  first Gram-Schmidt pass
    double* h2;      // (m+1) x R  second pass
    double* hnorm;   // R
    double* bnorm;   // R
    double* bcur;    // R (beta of the current cycle)
    double* est;     // R
    double* resid;   // R (last true relative residual)
    int32_t* act;    // R: column still iterating in this cycle
    int32_t* done;   // R: column converged
    int32_t* kused;  // R
};

int reduce_blocks_for(int64_t N);
// Kernels of one Arnoldi step take the step index k either from the host or,
// for the device-side loop, from device memory (kdev / DevIndex; host
// arguments then give the launch sizes for the largest k).
// The basis vectors (A, V) are FP64, or FP32 for the inner solves of the
// mixed path (products and sums stay FP64).
void launch_multidot(Ctx& c, const double* A, int64_t strideA, int ni, const double* B, int64_t N, int R,
                     double* partial, int nblk, double* out, int accumulate, int tag = K_GS_DOT,
                     const int32_t* kdev = nullptr);
void launch_multidot(Ctx& c, const float* A, int64_t strideA, int ni, const double* B, int64_t N, int R,
                     double* partial, int nblk, double* out, int accumulate, int tag = K_GS_DOT,
                     const int32_t* kdev = nullptr);
void launch_colnorm(Ctx& c, const double* A, int64_t N, int R, double* partial, int nblk, double* out);
void launch_multi_axpy(Ctx& c, const double* V, int64_t strideV, int ni, const double* h, double* W, int64_t N, int R,
                       const int32_t* kdev = nullptr);
void launch_multi_axpy(Ctx& c, const float* V, int64_t strideV, int ni, const double* h, double* W, int64_t N, int R,
                       const int32_t* kdev = nullptr);
void launch_scale_cols(Ctx& c, const double* src, const double* sc, double thresh, double* dst, int64_t N, int R,
                       const DevIndex& di = DevIndex());
// FP32 basis: dst gets the rounded vector, cur (N x R, FP64) the exact one.
void launch_scale_cols(Ctx& c, const double* src, const double* sc, double thresh, float* dst, double* cur, int64_t N,
                       int R, const DevIndex& di = DevIndex());
void launch_diag_scale(Ctx& c, const double* V, const double* d, double* Z, int64_t N, int R, bool add = false,
                       const DevIndex& di = DevIndex());
void launch_lincomb(Ctx& c, const double* V, int64_t strideV, int ni, const double* y, double* out, int64_t N,
                    int R);
void launch_lincomb(Ctx& c, const float* V, int64_t strideV, int ni, const double* y, double* out, int64_t N, int R);
void launch_residual(Ctx& c, const int32_t* cond, const int32_t* rhs_cond, const double* AX, double* Res, int64_t N,
                     int R);
void launch_sub(Ctx& c, const double* B, const double* AX, double* Res, int64_t n);
void launch_add(Ctx& c, double* X, const double* D, int64_t n);
void launch_zero_cols(Ctx& c, double* V, const int32_t* mask, int64_t N, int R);
void launch_givens(Ctx& c, const GmresDev& g, int k, const int32_t* kdev = nullptr);
// Device-side loop control: counts the active columns, advances *kdev when
// `advance`, and sets the loop's condition (active columns left and *kdev < m).
void launch_loop_ctl(Ctx& c, cudaGraphConditionalHandle h, const int32_t* act, int R, int32_t* kdev, int m,
                     bool advance);
// Zero `bytes` (a multiple of 16, 16-byte aligned) with a kernel.
void launch_zero(Ctx& c, void* p, size_t bytes);
void launch_trisolve(Ctx& c, const GmresDev& g);
void launch_cycle_start(Ctx& c, const GmresDev& g, const double* beta);
void launch_cycle_end(Ctx& c, const GmresDev& g, const double* rnorm);
void launch_count_active(Ctx& c, const int32_t* act, int R, int32_t* out);

}  // namespace gpx
