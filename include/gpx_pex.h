/*
 * gpx_pex.h — C ABI of the B200-native field-solver capacitance extractor.
 *
 * Drop-in boundary for the reference's `"pex_method": "field_solver"`
 * capacitance path.  Plain pointers and sizes only; caller-owned outputs; no
 * callbacks; no exceptions cross the ABI.  Every call returns a gpx_status;
 * gpx_last_error() gives the message of the last failing call on a context.
 * A context owns one CUDA stream on one device and is safe to use from one
 * thread at a time (use one context per thread for concurrency).
 *
 * Entry points and the reference interface each one replaces
 * (paths relative to the reference project root):
 *
 *   gpx_extract_quasistatic  crates/pex/src/bridge.rs:73-147 `extract_quasistatic`
 *                            (capacitance + fixed via R; the FastHenry sheet-R
 *                            solve, bridge.rs:144,180-299, stays with the caller)
 *   gpx_cap_solve_groups     crates/pex/src/bridge.rs:307-443 `solve_capacitance`
 *   gpx_cap_solve            crates/pex/src/quasistatic/cap/fmm_solver.rs:147-172
 *                            `fmm_solver::solve` and cap/solver.rs:100-134 `solve`
 *   gpx_cap_solve_eps        crates/pex/src/quasistatic/cap/dielectric.rs:76-150
 *                            `solve` with conductor roles only (FastCap list files
 *                            of C lines, cap/listfile.rs:56-77)
 *   gpx_cap_solve_batched    (no single reference function: many independent
 *                            windows; each window is one gpx_cap_solve)
 *   gpx_cap_sensitivity      (no reference counterpart: adjoint dC/dp beside the
 *                            capacitance result of cap/fmm_solver.rs:147-172)
 *   gpx_cap_sensitivity_rows (no reference counterpart: the same for a subset of
 *                            conductor rows)
 *   gpx_autotune             (no reference counterpart: replaces the fixed order 4 /
 *                            depth 4 of bridge.rs:403 by a measured choice)
 *   gpx_operator_apply       crates/pex/src/quasistatic/cap/fmm_solver.rs:109-129
 *                            `FmmCapOperator::apply`, for R right-hand sides
 *   gpx_potential_matrix     crates/pex/src/quasistatic/cap/solver.rs:81-97
 *                            `assemble_p_set` (Wilton integral, panel.rs:147-208)
 *   gpx_ctx_create/destroy   crates/backend/src/gpu.rs:270-278 (lazily created,
 *                            error-contained device context)
 */
#ifndef GPX_PEX_H
#define GPX_PEX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GPX_OK = 0,
    GPX_ERR_INVALID_ARG = 1,
    GPX_ERR_CUDA = 2,
    GPX_ERR_NO_DEVICE = 3,
    /* BridgeError variants (bridge.rs:35-56) */
    GPX_ERR_INVALID_DBU = 10,          /* InvalidDatabaseUnit */
    GPX_ERR_INVALID_PROCESS = 11,      /* InvalidProcessValue */
    GPX_ERR_UNSUPPORTED_GEOMETRY = 12, /* UnsupportedGeometry (polygon index in err_polygon) */
    GPX_ERR_GRID_CAPACITY = 13,        /* GridCapacity */
    GPX_ERR_PANEL_CAPACITY = 14,       /* PanelCapacity */
    GPX_ERR_CAPACITANCE = 15,          /* Capacitance(msg): includes GMRES non-convergence */
    GPX_ERR_NON_FINITE = 16,           /* NonFiniteResult */
    GPX_ERR_OUTPUT_CAPACITY = 20,      /* caller's output buffer too small */
    GPX_ERR_OUT_OF_MEMORY = 21,
    GPX_ERR_INTERNAL = 22
} gpx_status;

typedef struct gpx_ctx gpx_ctx;

/* Create a context on CUDA device `device` (one stream, device buffers and
 * cached M2L tables).  Fails with GPX_ERR_NO_DEVICE when no such device. */
gpx_status gpx_ctx_create(gpx_ctx** out, int device);
void gpx_ctx_destroy(gpx_ctx* ctx);
/* Message of the last failing call on `ctx` (never NULL; "" after success). */
const char* gpx_last_error(const gpx_ctx* ctx);
/* Library version string. */
const char* gpx_version(void);

typedef enum {
    GPX_PREC_FP64 = 0,  /* plain: every operator apply and all GMRES work in FP64 */
    GPX_PREC_MIXED = 1  /* FP32 far field and near apply (TF32 tensor cores for the
                           near apply and, with exact M2L, for M2L) inside an FP64
                           iterative-refinement loop */
} gpx_precision;

typedef enum {
    GPX_M2L_COMPRESSED = 0, /* QR-compressed operators, as the reference (bbfmm.rs:132-174) */
    GPX_M2L_EXACT = 1       /* uncompressed Chebyshev M2L operators */
} gpx_m2l_mode;

typedef struct {
    int32_t precision;       /* gpx_precision */
    int32_t order;           /* Chebyshev order n; 0 -> 4 (bridge.rs:403) */
    int32_t max_level;       /* uniform octree depth; 0 -> 4 (bridge.rs:403); -1 -> auto */
    int32_t m2l_mode;        /* gpx_m2l_mode */
    double tol;              /* GMRES relative residual; 0 -> 1e-8 (bridge.rs:403) */
    int32_t restart;         /* 0 -> 200 (fmm_solver.rs:164) */
    int32_t max_restarts;    /* 0 -> 50 */
    int32_t dense_below;     /* all-pairs (no far field) below this many panels;
                                0 -> 500 (bridge.rs:30), -1 -> never */
    int32_t precond;         /* 0 diagonal Jacobi (fmm_solver.rs:133-162), 1 leaf block-Jacobi (48-panel
                                blocks), 2 leaf block-Jacobi (96-panel blocks) */
    int32_t skip_ground_rhs; /* 1: do not solve the substrate column (the reference solves it);
                                the per-net result needs only the nets' columns */
    int32_t inner_tol_exp;   /* mixed: floor of the adaptive inner tolerance, 10^-x; 0 -> 3 with the
                                TF32 near apply (mixed_near 0 and 3), 5 with the FP32-accurate ones */
    double mesh_max_edge_m;  /* bridge panelisation: 0 -> reference `subdivisions` rule */
    int64_t max_panels;      /* bridge: 0 -> 20 000 (bridge.rs:29), -1 -> unlimited */
    int32_t far_quad;        /* far-field source model: 0 -> each panel's charge at its centroid
                                (the reference, fmm_solver.rs:109-115); 1 -> 2x2 Gauss points */
    int32_t mixed_near;      /* mixed: near-field apply 0 -> TF32 tensor cores (tcgen05; X split into TF32 hi
                                and lo before the apply and gathered as both), 1 -> FP32 CUDA cores, 2 ->
                                TF32 tensor cores with the near blocks kept in FP32 and split into TF32 hi
                                and lo parts on chip (three products; FP32-accurate), 3 -> as 0 with X
                                gathered once as FP32 and split on chip */
    int32_t mixed_m2l;       /* mixed: M2L 0 -> TF32 tensor cores (tcgen05) at orders 4 and 5 with centroid
                                far-field sources, else the factored low-rank form on FP32 CUDA cores;
                                1 -> always the factored form (compressed operators); 2 -> tensor cores
                                at orders 4 and 5 also with Gauss-point sources; 3 -> at orders 5 and 6
                                the operators in one shared rank-64 basis (K_o ~ U C_o V^T): expansions
                                compressed and decompressed on the tensor cores with TF32 hi and lo
                                parts, the 64 x 64 cores C_o on the tensor cores (order 4 as 2) */
    int32_t no_graphs;       /* 1: launch every operator apply directly instead of replaying it as a
                                captured CUDA graph (results are identical) */
    int32_t batch_streams;   /* gpx_cap_solve_batched: windows solved concurrently, one stream each;
                                0 -> 8 */
    int32_t col_begin;       /* gpx_cap_solve: with col_count > 0, solve only the conductor columns
                                [col_begin, col_begin + col_count) (one rank's share of a window whose
                                right-hand sides are spread over several GPUs); the other columns of
                                maxwell_out are NaN */
    int32_t col_count;       /* 0 -> every column (all but the substrate with skip_ground_rhs) */
    int32_t mixed_far_tc;    /* mixed, orders 4 and 5, tensor-core near apply: 1 -> P2M and L2P on the tensor
                                cores too (weights, charges and local expansions split into TF32 hi and lo
                                parts, FP32-accurate); 2 -> P2M only (L2P on the FP32 CUDA cores) */
    int32_t inner_basis32;   /* mixed: 1 -> inner GMRES basis stored in FP32 (products, sums and the
                                Hessenberg matrix stay FP64): twice the restart length in the same memory,
                                for inner tolerances of 1e-3 (TF32 near apply); 0 -> FP64 */
    int32_t reserved;        /* 0 */
} gpx_solve_opts;

typedef struct {
    int64_t n_panels;
    int32_t n_conductors;
    int32_t n_rhs;
    int32_t order, max_level;
    int64_t n_boxes, n_leaves, nnz_near, m2l_pairs;
    int32_t iterations;        /* max GMRES iterations over RHS (all cycles, inner solves in mixed) */
    int32_t outer_iterations;  /* mixed: refinement steps */
    int64_t operator_applies;  /* multi-RHS operator applies (FP64 + FP32) */
    double max_rel_residual;   /* final true FP64 relative residual, max over RHS */
    int32_t converged;
    int32_t dense;             /* 1 when the all-pairs path ran */
    double t_panelize_s, t_setup_s, t_solve_s, t_total_s;
    double t_near_assembly_s;  /* device time of the Wilton near-field assembly */
    int64_t kernel_launches;
    int64_t h2d_bytes, d2h_bytes;  /* host<->device copies made by the call */
    int32_t restart_used;      /* GMRES restart length after the Krylov memory budget (gpx_cap_solve) */
    int32_t reserved;
} gpx_solve_report;

/* Pre-built panels: `verts` n x 12 doubles (4 vertices x xyz, metres; a
 * triangle repeats its third vertex), `conductor` n ints in [0, n_conductors). */
typedef struct {
    int64_t n_panels;
    const double* verts;
    const int32_t* conductor;
    int32_t n_conductors;
} gpx_panel_problem;

/* Maxwell capacitance matrix (farads, no dielectric scaling) of the panel
 * problem.  maxwell_out: n_conductors x n_conductors row-major, C[i][j] =
 * charge on i per volt on j.  With opts.skip_ground_rhs the last (substrate)
 * column is filled by symmetry from its row and C[last][last] is NaN. */
gpx_status gpx_cap_solve(gpx_ctx* ctx, const gpx_panel_problem* problem, const gpx_solve_opts* opts,
                         double* maxwell_out, gpx_solve_report* report);

/* Maxwell capacitance matrix of panels that each sit in their own medium:
 * eps[k] (n_panels values, finite and > 0, caller panel order) is panel k's
 * surrounding relative permittivity, and its charge counts eps[k] times,
 * C[i][j] = sum_{k on i} eps[k] sigma_k a_k (cap/dielectric.rs:76-150 with
 * every panel a PanelRole::Conductor; the potential system is the vacuum one).
 * maxwell_out comes out k-scaled and is not symmetric: with
 * opts.skip_ground_rhs the last column is NaN.  Dielectric-interface panels
 * (PanelRole::Dielectric) are not supported. */
gpx_status gpx_cap_solve_eps(gpx_ctx* ctx, const gpx_panel_problem* problem, const double* eps,
                             const gpx_solve_opts* opts, double* maxwell_out, gpx_solve_report* report);

/* Many independent problems in one call; maxwell_out[i] per problem. */
gpx_status gpx_cap_solve_batched(gpx_ctx* ctx, const gpx_panel_problem* problems, int32_t n_problems,
                                 const gpx_solve_opts* opts, double* const* maxwell_out,
                                 gpx_solve_report* reports);

/* Adjoint sensitivities of the Maxwell matrix (north of the reference: it has
 * no gradient path; the derivative is of the same discretised operator
 * gpx_cap_solve solves).  Parameter q moves every panel vertex with velocity
 * vert_velocity[q][panel][12] (same layout as problem->verts, metres per unit
 * parameter).  maxwell_out: as gpx_cap_solve.  dmaxwell_out: n_params x
 * n_conductors x n_conductors, dC_ij/dp_q in farads per unit parameter (no
 * dielectric scaling; for a homogeneous dielectric dC_phys/dk = C).  Cost: one
 * forward and one transposed solve for all conductors, then one derivative
 * apply per parameter (Wilton near blocks differentiated exactly on dual
 * numbers, far field with differentiated end weights).  With
 * opts.skip_ground_rhs the substrate row and column of dmaxwell_out are NaN.
 * Conductors are solved in chunks of at most 128 right-hand sides (forward
 * columns and transposed rows alike); the forward charge densities of every
 * column stay resident for the derivative applies. */
gpx_status gpx_cap_sensitivity(gpx_ctx* ctx, const gpx_panel_problem* problem, const gpx_solve_opts* opts,
                               int32_t n_params, const double* vert_velocity, double* maxwell_out,
                               double* dmaxwell_out, gpx_solve_report* report);
/* As gpx_cap_sensitivity, with dC/dp for the n_rows listed conductors only
 * (rows: distinct solved conductor indices): the transposed solves run for
 * those rows alone, and the other rows of dmaxwell_out (still n_params x
 * n_conductors x n_conductors) are NaN.  The forward solve covers every
 * column, so row i of dC/dp is complete.  Used for gradients of a few nets
 * of a large block. */
gpx_status gpx_cap_sensitivity_rows(gpx_ctx* ctx, const gpx_panel_problem* problem, const gpx_solve_opts* opts,
                                    int32_t n_params, const double* vert_velocity, int32_t n_rows,
                                    const int32_t* rows, double* maxwell_out, double* dmaxwell_out,
                                    gpx_solve_report* report);

/* ---- autotuner (no reference counterpart: the reference hard-codes order 4,
 * depth 4, bridge.rs:403) ----
 * Chooses the far-field configuration for a representative panel problem: for
 * every candidate (Chebyshev order 4..6, octree depth around the automatic
 * choice, centroid or Gauss-point far-field sources, and in mixed precision
 * the near-apply engine: mixed_near 0, 3 or 1) it measures the operator's error on 512
 * sampled rows against the exact all-pairs rows (three smooth probe charge
 * densities) and times the operator apply on the device; the fastest
 * candidate whose error is at most target_rel_err / 2 wins (score: set-up +
 * 100 applies; the Maxwell matrix's error measures about 1.7x the sampled
 * operator error).
 * `tuned` receives `base` with order, max_level, far_quad, mixed_near and
 * dense_below (-1) replaced.  With cache_path (may be NULL) the choice is
 * looked up in / appended to that text file, keyed by a signature of the
 * problem (size, conductor count, aspect, mesh scale, precision, target). */
typedef struct {
    double est_rel_err;  /* sampled operator error of the chosen configuration */
    double apply_ms;     /* its operator apply, device milliseconds */
    double setup_ms;     /* its plan + near-field assembly, milliseconds */
    int32_t candidates;  /* configurations evaluated (0 when taken from the cache) */
    int32_t from_cache;
} gpx_tune_report;
gpx_status gpx_autotune(gpx_ctx* ctx, const gpx_panel_problem* problem, const gpx_solve_opts* base,
                        double target_rel_err, const char* cache_path, gpx_solve_opts* tuned,
                        gpx_tune_report* report);

/* y = P sigma for `nrhs` columns (sigma, y: n_panels x nrhs row-major, panel
 * order of `problem`), P the precorrected operator the solver uses. */
gpx_status gpx_operator_apply(gpx_ctx* ctx, const gpx_panel_problem* problem, const gpx_solve_opts* opts,
                              int32_t nrhs, const double* sigma, double* y, gpx_solve_report* report);

/* Dense block out[t][s] = (1/(4 pi eps0)) * Wilton integral of panel s at
 * point t (n_tgt x n_src row-major). */
gpx_status gpx_potential_matrix(gpx_ctx* ctx, int64_t n_src, const double* src_verts, int64_t n_tgt,
                                const double* tgt_points, double* out);

/* ---- small problems without allocation ----
 * No counterpart in the reference.
 *
 * Maxwell matrix (farads, no dielectric scaling, n_conductors x n_conductors
 * row-major, same meaning as gpx_cap_solve's maxwell_out) of a small panel
 * problem whose panels are already in device memory: d_verts (n_panels x 12
 * doubles, layout of gpx_panel_problem), d_conductor (n_panels ints) and
 * d_maxwell_out must be device (or managed) memory of the context's device.
 * The algorithm is the reference's dense path: assemble P, LU with partial
 * pivoting, one unit-potential solve per conductor, charge sums per conductor.
 *
 * Why it exists: the call allocates no memory, device or host, on its success
 * path.  It is for callers that cannot let a library allocate: a process whose
 * device memory is already carved up by its own pool allocator (an EDA tool
 * or a framework that reserves nearly all of HBM up front, where a library
 * allocation fails or fragments the pool), and tight per-window loops where
 * allocating and freeing on every call would synchronise the device.  All
 * intermediate data lives in one fixed array of 2,377,984 bytes (about
 * 2.3 MiB) of static device memory per device, present once the library is
 * loaded on that device.
 *
 * Limits: 1 <= n_panels <= 512 and 1 <= n_conductors <= 64; larger problems
 * are rejected with GPX_ERR_INVALID_ARG and a message naming the limit (use
 * gpx_cap_solve for them).  A conductor index outside [0, n_conductors) gives
 * GPX_ERR_INVALID_ARG; a zero pivot gives GPX_ERR_CAPACITANCE.
 *
 * The caller zeroes nothing: the call clears its own status word before its
 * first launch, and writes every other scratch element before reading it.
 * The call runs on the context's stream and waits for that stream before it
 * returns.  The first call on each device also does a one-time set-up: it looks
 * up the scratch array's device address, loads every kernel the entry point
 * launches (CUDA loads kernels lazily by default, and loading one takes device
 * memory) and raises one kernel's shared-memory limit.  Make that first call
 * before any stream capture on that device, and before the caller's own pool
 * reserves the device memory it means to keep; later calls take none.
 * Every call on one device uses the same scratch array, so two calls that
 * overlapped would race on it; the library therefore serialises the calls of
 * one process per device with a lock held until the call's stream work has
 * finished.  Each process has its own copy of the array. */
gpx_status gpx_cap_solve_small_static(gpx_ctx* ctx, int64_t n_panels, const double* d_verts,
                                      const int32_t* d_conductor, int32_t n_conductors, double* d_maxwell_out);

/* ---- bridge level ---- */
typedef struct {
    uint32_t net;
    double z0_m, z1_m, dielectric_k;
    int64_t rect_offset, rect_count; /* into the rects array, 4 x int32 (x0,y0,x1,y1) DBU each */
} gpx_volume_group;

/* Replaces bridge.rs:307-443 `solve_capacitance`: groups in the caller's
 * BTreeMap<(net, layer)> order.  Outputs per net (ascending net id) the net id
 * and C[i][i] in aF (scaled by k), and optionally the full (nets+1)^2 Maxwell
 * matrix in farads (k-scaled; last row/column = substrate).  Groups of several
 * k: each panel's charge is scaled by its own group's k (the substrate's by the
 * lowest group's), as bridge.rs:409-430 does through cap/dielectric.rs:76-150;
 * the reference allows that only below 500 panels, this call at any size.
 * That matrix is not symmetric, so with skip_ground_rhs its substrate column
 * is NaN instead of filled by symmetry. */
gpx_status gpx_cap_solve_groups(gpx_ctx* ctx, const gpx_volume_group* groups, int64_t n_groups,
                                const int32_t* rects, double xy_scale_m, const gpx_solve_opts* opts,
                                uint32_t* nets_out, double* cap_af_out, int64_t nets_cap, int64_t* n_nets,
                                double* maxwell_out, gpx_solve_report* report);

typedef struct {
    const int32_t* verts_x;
    const int32_t* verts_y;
    const uint32_t* poly_vert_start;
    const uint32_t* poly_vert_len;
    const uint16_t* poly_layer;
    int64_t n_poly;
} gpx_geometry_store;

typedef struct { /* io/pdk.rs:520-544 */
    uint16_t layer;
    double sheet_res_ohm_sq, area_cap_af_um2, fringe_cap_af_um, coupling_cap_af_um;
    double interlayer_cap_af_um2, via_res_ohm, thickness_nm, height_nm, dielectric_k;
} gpx_layer_params;

typedef struct {
    const gpx_layer_params* layers;
    int64_t n_layers;
    double dbu_nm;
} gpx_deck;

typedef struct { /* analytical/mod.rs:354-357 NetParasitics */
    uint32_t net;
    double r_ohm;   /* fixed via/contact resistance only */
    double cap_af;
} gpx_net_parasitics;

/* Replaces bridge.rs:73-147 `extract_quasistatic` for C (and fixed via R).
 * This call, gpx_cap_solve_groups and gpx_bridge_panelize keep their panel
 * buffers per calling thread between calls (capacity of the largest layout
 * panelised so far), so repeated calls make no fresh host allocations.
 * On GPX_ERR_UNSUPPORTED_GEOMETRY *err_polygon is the polygon index (else
 * UINT32_MAX), as lib.rs:111-123 maps it into the diagnostic. */
gpx_status gpx_extract_quasistatic(gpx_ctx* ctx, const gpx_geometry_store* store, const gpx_deck* deck,
                                   const uint32_t* net_of_poly, int64_t n_net_of_poly,
                                   const gpx_solve_opts* opts, gpx_net_parasitics* out, int64_t out_cap,
                                   int64_t* n_out, uint32_t* err_polygon, gpx_solve_report* report);

/* Panelise only (bridge.rs:445-652 + ground plate :346-379): for tests and
 * callers that keep the panels.  Returns counts in *n_panels / *n_nets. */
gpx_status gpx_bridge_panelize(gpx_ctx* ctx, const gpx_geometry_store* store, const gpx_deck* deck,
                               const uint32_t* net_of_poly, int64_t n_net_of_poly,
                               const gpx_solve_opts* opts, double* verts_out, int32_t* cond_out,
                               double* eps_out, int64_t cap, int64_t* n_panels, uint32_t* nets_out,
                               int64_t nets_cap, int64_t* n_nets, uint32_t* err_polygon);

/* ---- instrumentation ---- */
/* Kernel classes of gpx_ctx_kernel_stats.  The operator's classes are split
 * by precision: GPX_K_NEAR_APPLY .. GPX_K_L2P count the FP32 / TF32 launches
 * (the mixed path's inner operator), GPX_K_NEAR_APPLY_F64 .. GPX_K_L2P_F64 the
 * FP64 ones (the plain path, and the mixed path's refinement residuals). */
typedef enum {
    GPX_K_NEAR_ASSEMBLE = 0, GPX_K_NEAR_APPLY = 1, GPX_K_P2M = 2, GPX_K_M2M = 3, GPX_K_M2L = 4, GPX_K_L2L = 5,
    GPX_K_L2P = 6, GPX_K_GS_DOT = 7, GPX_K_GS_AXPY = 8, GPX_K_VEC = 9, GPX_K_SMALL = 10,
    GPX_K_NEAR_APPLY_F64 = 11, GPX_K_P2M_F64 = 12, GPX_K_M2M_F64 = 13, GPX_K_M2L_F64 = 14, GPX_K_L2L_F64 = 15,
    GPX_K_L2P_F64 = 16, GPX_K_COUNT = 17
} gpx_kernel_class;
/* The CUDA stream (cudaStream_t) every kernel of this context runs on. */
void* gpx_ctx_stream(gpx_ctx* ctx);
/* Per-kernel CUDA-event timing on the context stream (off by default). */
gpx_status gpx_ctx_set_profiling(gpx_ctx* ctx, int32_t on);
/* Accumulated launches, device milliseconds and algorithmic bytes / flops
 * of one kernel class since the last reset; *total_launches counts every
 * kernel this context launched. */
gpx_status gpx_ctx_kernel_stats(gpx_ctx* ctx, int32_t kernel_class, int64_t* launches, double* ms, double* bytes,
                                double* flops, int64_t* total_launches);
gpx_status gpx_ctx_reset_stats(gpx_ctx* ctx);

/* Host-only self-check of the octree plan the solver would build for these
 * panels at (order, depth): index bounds, list disjointness and exact pair
 * coverage (every ordered panel pair is near or in exactly one M2L pair).
 * stats (8 entries): leaves, boxes, near pairs, M2L box pairs, far panel
 * pairs, largest leaf, largest near row, and a 64-bit FNV-1a checksum of every
 * plan array the device kernels index (sorted panels, weights, tree, near and
 * M2L lists).  Needs no device. */
gpx_status gpx_plan_check(int64_t n_panels, const double* verts, int32_t order, int32_t depth, int64_t* stats);

#ifdef __cplusplus
}
#endif
#endif /* GPX_PEX_H */
