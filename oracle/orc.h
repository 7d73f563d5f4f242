/*
 * CPU oracle for the field-solver capacitance path — TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain C++17 restatement of the reference's CPU field solver
 * (crates/pex/src/bridge.rs, crates/pex/src/quasistatic/{integrals/panel.rs,
 * cap/solver.rs, cap/fmm_solver.rs, cap/mesh.rs, fmm/{tree,chebyshev,bbfmm}.rs, linalg.rs,
 * krylov.rs, simd.rs}, crates/core/src/geometry/rects.rs,
 * crates/pex/src/analytical/process_stack.rs).  Only the tests, the smoke
 * check and the CPU-baseline leg of the benchmark may load it, and only as the
 * checker.  The product library never links it.
 *
 * Parity pinning: the reference publishes no field-solver golden numbers.  The
 * oracle is pinned against the reference's own known-answer tests
 * (tests/analytic.rs, tests/cap_validation.rs, tests/fmm.rs,
 * tests/fmm_cap.rs, tests/bridge.rs) which the Python tests re-run against it.
 *
 * Panels are stored as 4 vertices x 3 doubles (12 doubles per panel).  A
 * triangle repeats its last vertex; the reference's per-edge loop skips the
 * zero-length edge and the fan triangulation adds a zero-area triangle, so
 * the result is bit-identical to the 3-vertex form.
 */
#ifndef GPX_ORACLE_H
#define GPX_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- panel geometry (integrals/panel.rs) ---- */
double orc_potential_integral(const double* verts12, const double* p3);
void orc_panel_props(const double* verts12, double* centroid3, double* area, double* normal3);

/* ---- mesh generators (cap/mesh.rs) ---- returns panel count (<= cap) */
int64_t orc_plate(double cx, double cy, double z0, double lx, double ly, int64_t nx, int64_t ny,
                  int32_t conductor, double* verts_out, int32_t* cond_out, int64_t cap);
int64_t orc_icosphere(double cx, double cy, double cz, double r, int32_t subdivisions,
                      int32_t conductor, double* verts_out, int32_t* cond_out, int64_t cap);

/* ---- rectilinear decomposition (core/geometry/rects.rs:96-176) ----
 * returns rect count (rects_out 4*i32 per rect) or a negative error:
 * -1 too few vertices, -2 non-rectilinear edge, -3 odd crossings, -4 cap exceeded */
int64_t orc_decompose_rectilinear(const int32_t* xs, const int32_t* ys, int64_t nv,
                                  int32_t* rects_out, int64_t cap);

/* ---- bridge (bridge.rs:73-147, 307-652) ----
 * Layer params table: one entry per deck PEX layer. */
typedef struct {
    uint16_t layer;
    double sheet_res_ohm_sq, area_cap_af_um2, fringe_cap_af_um, coupling_cap_af_um;
    double interlayer_cap_af_um2, via_res_ohm, thickness_nm, height_nm, dielectric_k;
} orc_layer_params;

/* Panelise the store exactly as the reference bridge would.
 * Outputs the panels (grouped by (net, layer) in BTreeMap order + ground
 * plate), their conductor index and eps, and the sorted net list.
 * mesh_max_edge_m == 0 -> reference `subdivisions` rule; > 0 -> target-edge
 * mode (every face edge at most that long; substrate plate cells at most
 * 4 x that long, no cap on their number).
 * max_panels: 0 = the reference's 20 000 limit; < 0 = unlimited.
 * Returns the panel count, or a negative error code; err_msg gets text. */
int64_t orc_bridge_panelize(const int32_t* verts_x, const int32_t* verts_y,
                            const uint32_t* poly_vert_start, const uint32_t* poly_vert_len,
                            const uint16_t* poly_layer, int64_t n_poly,
                            const uint32_t* net_of_poly, int64_t n_net_of_poly,
                            const orc_layer_params* layers, int64_t n_layers, double dbu_nm,
                            double mesh_max_edge_m, int64_t max_panels,
                            double* verts_out, int32_t* cond_out, double* eps_out, int64_t cap,
                            uint32_t* nets_out, int64_t* n_nets_out,
                            double* via_r_out /* per net in nets_out order, may be NULL */,
                            char* err_msg, int64_t err_cap);

/* ---- solvers ---- C is ncond x ncond row-major, in farads (no eps scaling). */
int orc_dense_P(int64_t n, const double* verts, double* P_out);
int orc_cap_dense(int64_t n, const double* verts, const int32_t* cond, int32_t ncond, double* C_out);
/* cap/dielectric.rs:76-150, conductor roles (bridge.rs:409-430): each panel's
 * charge weighted by its surrounding permittivity eps[k]; C comes out k-scaled. */
int orc_cap_dense_eps(int64_t n, const double* verts, const int32_t* cond, int32_t ncond, const double* eps,
                      double* C_out);
typedef struct {
    int32_t order, max_level, restart, max_restarts;
    double tol;
    int32_t threads;          /* 0 = OpenMP default */
    int32_t rhs_limit;        /* > 0: solve only rhs_limit conductors (a bounded CPU sample) */
    int32_t rhs_stride;       /* > 1: the sampled conductors are 0, stride, 2 stride, ... */
} orc_fmm_opts;
typedef struct {
    int64_t total_iterations;
    int64_t max_iterations;   /* over RHS */
    double max_residual;      /* final true relative residual, max over RHS */
    int32_t all_converged;
    int64_t nnz_near;
    int64_t n_boxes;
    double t_setup_s, t_solve_s;
} orc_fmm_report;
int orc_cap_fmm(int64_t n, const double* verts, const int32_t* cond, int32_t ncond,
                const orc_fmm_opts* opts, double* C_out, orc_fmm_report* rep);
/* The same solve in steps: build the operator and preconditioner once
 * (t_setup_s receives the seconds), then solve one conductor's column at a
 * time (0 converged, 1 not converged, -1 bad argument). */
void* orc_fmm_new(int64_t n, const double* verts, const int32_t* cond, int32_t ncond, int32_t order,
                  int32_t max_level, int32_t threads, double* t_setup_s);
int orc_fmm_solve_column(void* handle, int32_t j, double tol, int32_t restart, int32_t max_restarts,
                         double* C_col, int64_t* iterations, double* residual);
void orc_fmm_free(void* handle);
/* Dense GMRES path (cap/solver.rs:118-125, tol 1e-8 restart 100). */
int orc_cap_dense_gmres(int64_t n, const double* verts, const int32_t* cond, int32_t ncond,
                        double* C_out);

/* ---- operator pieces (for parity tests) ---- */
/* Point FMM y = K q (LaplaceFmm::matvec with P2P, or far-field only). */
int orc_fmm_point_matvec(int64_t n, const double* pts3, const double* q, int32_t order,
                         int32_t max_level, int32_t with_p2p, double* y);
/* Precorrected capacitance operator y = P sigma (FmmCapOperator::apply). */
int orc_fmm_cap_apply(int64_t n, const double* verts, int32_t order, int32_t max_level,
                      const double* sigma, double* y, int64_t* nnz_out);
/* Low-rank compressed M2L table for order n (bbfmm.rs:132-174), returned as the
 * dense product U*V^T per offset in [-3,3]^3 (343 slots of n^6 doubles, slot
 * index ((ox+3)*7+oy+3)*7+oz+3), rank per slot (-1 = not built). Offsets
 * built: all with max|o| >= 2 (the only ones an interaction list contains). */
int orc_m2l_table(int32_t order, double* k_out, int32_t* rank_out);

/* Dot product with the reference's 16-partial-sum order (simd.rs:20-45). */
double orc_dot(const double* a, const double* b, int64_t n);

#ifdef __cplusplus
}
#endif
#endif
