// Right preconditioners of the GMRES iteration.
#pragma once
#include "kernels.cuh"
#include "plan.h"

namespace gpx {

// Leaf block-Jacobi: blocks of up to `block` (48 or 96) consecutive panels
// of one leaf, inverted from the exact near-field self block.
struct BlockJacobi {
    int block = 48;
    int nblk = 0;
    DBuf<int32_t> d_leaf, d_row0, d_size, d_sing;
    DBuf<int64_t> d_start;
    DBuf<double> Minv;
    DBuf<float> Minv32;  // FP32 copy for the mixed path's inner solves (make_f32)
    // Inverts the blocks on the device (no host wait); check() then waits for
    // the stream and fails if a block was singular.
    void build(Ctx& c, const Plan& pl, const DevPlan& dp, const double* P);
    void check(Ctx& c) const;
    // Z = M^-1 V (or Z += M^-1 V), V and Z N x R row-major.
    void apply(Ctx& c, const double* V, double* Z, int64_t N, int R, bool add,
               const DevIndex& di = DevIndex()) const;
    // FP32 inverses (after make_f32): the same product in FP32, V and Z FP64;
    // R a multiple of 4.
    void make_f32(Ctx& c);
    void apply32(Ctx& c, const double* V, double* Z, int64_t N, int R, bool add,
                 const DevIndex& di = DevIndex()) const;
};

}  // namespace gpx
