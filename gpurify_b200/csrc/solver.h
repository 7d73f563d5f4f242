// Capacitance solve orchestration (plan -> device operator -> multi-RHS GMRES).
#pragma once
#include "gpx_common.h"
#include "plan.h"

namespace gpx {

// Options after defaults are applied.
struct Opts {
    int precision = GPX_PREC_FP64;
    int order = 4, max_level = 4, m2l_mode = GPX_M2L_COMPRESSED;
    double tol = 1e-8;
    int restart = 200, max_restarts = 50;
    int dense_below = 500;
    int precond = 0;
    int skip_ground_rhs = 0;
    int inner_tol_exp = 3;
    double mesh_max_edge = 0.0;
    int64_t max_panels = 0;
    int far_quad = 0;
    int mixed_near = 0;
    int mixed_m2l = 0;
    int graphs = 1;         // capture operator applies into CUDA graphs
    int batch_streams = 0;  // batched solves: concurrent streams (0 -> default)
    int col_begin = 0, col_count = 0;  // column subset (col_count 0: every column)
    int mixed_far_tc = 0;              // mixed: P2M on the tensor cores
    int inner_basis32 = 0;             // mixed: inner GMRES basis stored in FP32
};
Opts normalize(const gpx_solve_opts* o);

// Depth the solver uses for n panels under the options (1 = all pairs);
// the automatic rule looks at the panels (may be null) to keep every leaf at
// least as large as the largest panel.
int choose_depth(const Opts& o, int64_t n, const double* verts);

// Solve the Maxwell matrix of a panel problem (farads, not k-scaled) into C
// (ncond x ncond row-major).  Columns not solved are filled by symmetry.
// With panel_eps (n values, caller panel order) each panel's charge counts
// with its own relative permittivity, C[i][j] = sum_{k on i} eps_k sigma_k a_k
// (the bridge's solve of a stack of several k, bridge.rs:409-430 ->
// cap/dielectric.rs:76-150 with conductor roles): C is then k-scaled, not
// symmetric, and columns not solved are NaN.
void cap_solve(Ctx& ctx, int64_t n, const double* verts, const int32_t* cond, int ncond, const Opts& o, double* C,
               gpx_solve_report* rep, const double* panel_eps = nullptr);

// Maxwell matrix C and its derivatives dC/dp for np vertex velocity fields V
// (np x n x 12, caller panel order): one forward and one transposed solve
// (all conductors at once), then one derivative apply per parameter.
// dCdp: np x ncond x ncond; entries of conductors not solved are NaN.
// Maxwell matrix and dC/dp along np vertex velocity fields; the rows of dC
// are the nrows listed conductors (rows null: every solved conductor), the
// other rows NaN.  Columns and rows are solved in chunks of 128.
void cap_sensitivity(Ctx& ctx, int64_t n, const double* verts, const int32_t* cond, int ncond, const Opts& o,
                     int np, const double* V, int nrows, const int32_t* rows, double* C, double* dCdp,
                     gpx_solve_report* rep);

// Autotuner: the fastest far-field configuration (order, depth, far-field
// source model, near-apply engine) whose sampled operator error against the
// all-pairs rows is at most `target`; cached by problem signature in
// cache_path (one line per signature) when given.
void autotune(Ctx& ctx, int64_t n, const double* verts, const int32_t* cond, int ncond, const Opts& base,
              double target, const char* cache_path, Opts& out, gpx_tune_report* rep);

// y = P sigma (sigma, y: n x R row-major in caller panel order).
void operator_apply(Ctx& ctx, int64_t n, const double* verts, const Opts& o, int R, const double* sigma, double* y,
                    gpx_solve_report* rep);

// Dense Wilton block.
void potential_matrix(Ctx& ctx, int64_t ns, const double* sv, int64_t nt, const double* pts, double* out);

}  // namespace gpx
