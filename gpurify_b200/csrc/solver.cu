// Capacitance solve on one GPU: plan upload, Wilton near-field assembly, the
// precorrected FMM operator, multi-RHS restarted GMRES with one right-hand
// side per conductor, and the Maxwell-matrix accumulation.
//
// Reference path: crates/pex/src/quasistatic/cap/fmm_solver.rs:147-172
// (FmmCapOperator + DiagJacobi + gmres per conductor) and cap/solver.rs:55-71
// (unit-conductor right-hand sides, C[i][j] += sigma_k * a_k).  Differences
// by design: all conductors are solved together (one operator apply per
// Arnoldi step serves every right-hand side) and the Arnoldi step uses
// classical Gram-Schmidt with one re-orthogonalisation pass (CGS2) instead of
// modified Gram-Schmidt, which turns k+1 dependent reductions into two.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <mutex>

#include "adjoint.cuh"
#include "farfield.cuh"
#include "kernels.cuh"
#include "krylov.cuh"
#include "precond.cuh"
#include "solver.h"

namespace gpx {

struct DevM2L {
    int n = 0, mode = 0;
    DBuf<double> K;   // FP64 operators
    DBuf<double> U, Vt;  // low-rank factors (compressed mode), stride n3
    DBuf<double> Ut64, Vt64;  // factored-M2L tables: Vt rows and transposed U rows, 343 x 32 x ns
    DBuf<float> Ut32, Vt32;
    bool factored_ok = false;
    DBuf<int32_t> d_rank;
    int max_rank = 0;
    DBuf<float> K32;  // the same, rounded to TF32 (round to nearest, ties away), 343 x ns x ns, orders 4-5
    std::vector<int32_t> rank;
    // Shared-basis compression (orders 5-6, built on first use): V^T
    // (kShared x ns) and U (round_up(ns, 64) x kShared), each split into TF32
    // hi and lo parts, and the cores C_o rounded to TF32, 343 x kShared x kShared.
    bool shared_ok = false;
    double shared_err = 0.0;
    DBuf<float> Vt_hi, Vt_lo, U_hi, U_lo, C32;
};

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Host M2L tables, built once per (order, mode) in the process and shared by
// every context (their compression is the costly part).
std::shared_ptr<const M2LTable> host_m2l(int n, int mode) {
    static std::mutex mu;
    static std::vector<std::shared_ptr<const M2LTable>> cache;
    std::lock_guard<std::mutex> lk(mu);
    for (auto& t : cache)
        if (t->n == n && t->mode == mode) return t;
    auto t = std::make_shared<M2LTable>();
    build_m2l_table(*t, n, mode);
    cache.push_back(t);
    return t;
}

// Host shared bases, built once per (order, mode) in the process.
std::shared_ptr<const SharedBasis> host_shared(int n, int mode) {
    static std::mutex mu;
    static std::vector<std::shared_ptr<const SharedBasis>> cache;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (auto& t : cache)
            if (t->n == n && t->mode == mode) return t;
    }
    auto table = host_m2l(n, mode);
    auto b = std::make_shared<SharedBasis>();
    build_shared_basis(*table, kShared, *b);
    std::lock_guard<std::mutex> lk(mu);
    for (auto& t : cache)
        if (t->n == n && t->mode == mode) return t;
    cache.push_back(b);
    return b;
}

float tf32_rna(double x) {
    float f = (float)x;
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
    std::memcpy(&f, &u, 4);
    return f;
}

// Device tables of the shared-basis M2L for a cached operator table.
void ensure_shared(Ctx& ctx, DevM2L& d) {
    if (d.shared_ok) return;
    if (d.n < 5 || d.n > 6) throw Error(GPX_ERR_INVALID_ARG, "the shared-basis M2L runs orders 5 and 6");
    auto b = host_shared(d.n, d.mode);
    const int n3 = d.n * d.n * d.n, ns = node_stride(d.n), r = kShared, ldb = (ns + 63) / 64 * 64;
    std::vector<float> vh((size_t)r * ns, 0.f), vl((size_t)r * ns, 0.f), uh((size_t)ldb * r, 0.f),
        ul((size_t)ldb * r, 0.f), c((size_t)343 * r * r, 0.f);
    for (int l = 0; l < n3; ++l)
        for (int k = 0; k < r; ++k) {
            const double v = b->V[(size_t)l * r + k], u = b->U[(size_t)l * r + k];
            vh[(size_t)k * ns + l] = tf32_rna(v);
            vl[(size_t)k * ns + l] = tf32_rna(v - (double)vh[(size_t)k * ns + l]);
            uh[(size_t)l * r + k] = tf32_rna(u);
            ul[(size_t)l * r + k] = tf32_rna(u - (double)uh[(size_t)l * r + k]);
        }
    for (size_t i = 0; i < c.size(); ++i) c[i] = tf32_rna(b->C[i]);
    d.Vt_hi.upload(vh, ctx.stream);
    d.Vt_lo.upload(vl, ctx.stream);
    d.U_hi.upload(uh, ctx.stream);
    d.U_lo.upload(ul, ctx.stream);
    d.C32.upload(c, ctx.stream);
    GPX_CUDA(cudaStreamSynchronize(ctx.stream));
    d.shared_err = b->rel_err;
    d.shared_ok = true;
}

std::shared_ptr<DevM2L> get_m2l(Ctx& ctx, int n, int mode) {
    for (auto& t : ctx.m2l_cache)
        if (t->n == n && t->mode == mode) return t;
    const M2LTable& host = *host_m2l(n, mode);
    auto d = std::make_shared<DevM2L>();
    d->n = n;
    d->mode = mode;
    d->rank = host.rank;
    d->K.upload(host.K, ctx.stream);
    if (mode == GPX_M2L_COMPRESSED) {
        d->U.upload(host.U, ctx.stream);
        d->Vt.upload(host.Vt, ctx.stream);
    }
    d->d_rank.upload(host.rank, ctx.stream);
    for (int32_t r : host.rank) d->max_rank = std::max(d->max_rank, (int)r);
    if (mode == GPX_M2L_COMPRESSED && n >= 4 && n <= 6 && d->max_rank <= kFacMaxRank) {
        // factored tables: Vt rows and transposed U rows, kFacMaxRank rows of
        // node stride ns per slot (rows beyond the rank and padding nodes zero)
        const int n3 = n * n * n, ns = node_stride(n), KR = kFacMaxRank;
        const size_t sz = (size_t)343 * KR * ns;
        std::vector<double> ut(sz, 0.0), vt(sz, 0.0);
        std::vector<float> ut32(sz, 0.f), vt32(sz, 0.f);
        for (int sl = 0; sl < 343; ++sl)
            for (int k = 0; k < std::max(0, (int)host.rank[sl]); ++k)
                for (int m = 0; m < n3; ++m) {
                    const size_t o = ((size_t)sl * KR + k) * ns + m;
                    ut[o] = host.U[((size_t)sl * n3 + m) * n3 + k];
                    vt[o] = host.Vt[((size_t)sl * n3 + k) * n3 + m];
                    ut32[o] = (float)ut[o];
                    vt32[o] = (float)vt[o];
                }
        d->Ut64.upload(ut, ctx.stream);
        d->Vt64.upload(vt, ctx.stream);
        d->Ut32.upload(ut32, ctx.stream);
        d->Vt32.upload(vt32, ctx.stream);
        d->factored_ok = true;
    }
    if (n == 4 || n == 5) {
        // TF32-rounded (nearest, ties away) operators for the tensor-core M2L,
        // node stride ns in both indices, padding zero
        const int n3 = n * n * n, ns = node_stride(n);
        std::vector<float> k32((size_t)343 * ns * ns, 0.f);
        for (int sl = 0; sl < 343; ++sl)
            for (int m = 0; m < n3; ++m)
                for (int l = 0; l < n3; ++l) {
                    float f = (float)host.K[((size_t)sl * n3 + m) * n3 + l];
                    uint32_t u;
                    std::memcpy(&u, &f, 4);
                    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
                    std::memcpy(&f, &u, 4);
                    k32[((size_t)sl * ns + m) * ns + l] = f;
                }
        d->K32.upload(k32, ctx.stream);
    }
    GPX_CUDA(cudaStreamSynchronize(ctx.stream));
    ctx.m2l_cache.push_back(d);
    return d;
}

struct DevPlanBufs {
    DBuf<double> verts, cent, area, w1d, m2m1d;
    DBuf<int32_t> cond, near_off, near_src, near_S, box_parent, box_octant, m2l_src, m2l_slot, child_first,
        child_count, leaf_of, item_leaf, item_row0, item128_leaf, item128_row0, near_rev, near_pre, p2m_slot,
        fix_leaf, fix_first, fix_cnt;
    DBuf<int64_t> leaf_begin, nval_off, m2l_off;
    DBuf<double> leaf_ctr, wsrc;
    int nitems128 = 0;
    DevPlan v{};
    FarLaunch far{};
};

void upload_plan(Ctx& ctx, const Plan& p, const DevM2L* m2l, DevPlanBufs& d) {
    cudaStream_t s = ctx.stream;
    d.verts.upload(p.verts, s);
    d.cent.upload(p.cent, s);
    d.area.upload(p.area, s);
    d.w1d.upload(p.w1d, s);
    d.m2m1d.upload(p.m2m1d, s);
    d.cond.upload(p.cond, s);
    d.near_off.upload(p.near_off, s);
    d.near_src.upload(p.near_src, s);
    d.near_S.upload(p.near_S, s);
    d.box_parent.upload(p.box_parent, s);
    d.box_octant.upload(p.box_octant, s);
    d.m2l_src.upload(p.m2l_src, s);
    d.m2l_slot.upload(p.m2l_slot, s);
    d.child_first.upload(p.child_first, s);
    d.child_count.upload(p.child_count, s);
    d.leaf_of.upload(p.leaf_of, s);
    d.leaf_begin.upload(p.leaf_begin, s);
    d.nval_off.upload(p.nval_off, s);
    d.m2l_off.upload(p.m2l_off, s);
    {
        std::vector<double> ctr((size_t)p.nleaf() * 3);
        const double hl = p.lvl_half[p.L];
        for (int64_t k = 0; k < p.nleaf(); ++k)
            for (int dd = 0; dd < 3; ++dd)
                ctr[3 * k + dd] =
                    p.origin[dd] + ((double)p.box_cell[3 * (p.lvl_off[p.L] + k) + dd] + 0.5) * 2.0 * hl;
        d.leaf_ctr.upload(ctr, s);
    }
    d.item_leaf.upload(p.item_leaf, s);
    d.item_row0.upload(p.item_row0, s);
    {
        // P2M runs over the near items: the first item of a leaf writes the
        // leaf's expansion, further items write partials that k_p2m_fix adds
        static_assert(Plan::kRowsPerItem == 64, "far-field kernels take 64-panel items");
        std::vector<int32_t> slot(p.item_leaf.size(), -1), fl, ff, fc;
        int32_t np = 0;
        for (size_t i = 0; i < p.item_leaf.size(); ++i) {
            if (p.item_row0[i] == 0) continue;
            const int32_t k = p.item_leaf[i];
            if (fl.empty() || fl.back() != k) {
                fl.push_back(k);
                ff.push_back(np);
                fc.push_back(0);
            }
            slot[i] = np++;
            fc.back() += 1;
        }
        d.p2m_slot.upload(slot, s);
        d.fix_leaf.upload(fl, s);
        d.fix_first.upload(ff, s);
        d.fix_cnt.upload(fc, s);
        d.far.p2m_slot = d.p2m_slot.p;
        d.far.fix_leaf = d.fix_leaf.p;
        d.far.fix_first = d.fix_first.p;
        d.far.fix_cnt = d.fix_cnt.p;
        d.far.nfix = (int)fl.size();
        d.far.npart = np;
    }
    {
        // per near entry (t, e): its column offset in t's concatenated source
        // list, and the index of t in the near list of leaf near_src[e]
        std::vector<int32_t> pre(p.near_src.size()), rev(p.near_src.size(), -1);
        for (int64_t t = 0; t < p.nleaf(); ++t) {
            int32_t acc = 0;
            for (int32_t e = p.near_off[t]; e < p.near_off[t + 1]; ++e) {
                pre[e] = acc;
                const int32_t u = p.near_src[e];
                acc += (int32_t)(p.leaf_begin[u + 1] - p.leaf_begin[u]);
                for (int32_t f = p.near_off[u]; f < p.near_off[u + 1]; ++f)
                    if (p.near_src[f] == (int32_t)t) rev[e] = f - p.near_off[u];
                if (rev[e] < 0) throw Error(GPX_ERR_INTERNAL, "near-leaf relation is not symmetric");
            }
        }
        d.near_pre.upload(pre, s);
        d.near_rev.upload(rev, s);
    }
    DevPlan& v = d.v;
    v.nitems = (int32_t)p.item_leaf.size();
    v.item_leaf = d.item_leaf.p;
    v.leaf_ctr = d.leaf_ctr.p;
    v.leaf_of = d.leaf_of.p;
    v.leaf_half = p.lvl_half[p.L];
    {
        std::vector<double> roots = cheb_roots(p.n);
        for (int k = 0; k < p.n && k < 8; ++k) v.roots[k] = roots[k];
    }
    v.item_row0 = d.item_row0.p;
    {
        // 128-row work items of the tensor-core near apply, largest first so
        // the last wave of CTAs holds the short items
        std::vector<std::array<int64_t, 3>> items;
        for (int64_t k = 0; k < p.nleaf(); ++k) {
            const int64_t mk = p.leaf_begin[k + 1] - p.leaf_begin[k];
            for (int64_t r = 0; r < mk; r += 128) items.push_back({std::min<int64_t>(128, mk - r) * p.near_S[k], k, r});
        }
        std::stable_sort(items.begin(), items.end(), [](const auto& a, const auto& b) { return a[0] > b[0]; });
        std::vector<int32_t> il, ir;
        for (const auto& it : items) {
            il.push_back((int32_t)it[1]);
            ir.push_back((int32_t)it[2]);
        }
        d.item128_leaf.upload(il, s);
        d.item128_row0.upload(ir, s);
        d.nitems128 = (int)il.size();
    }
    v.n = p.n;
    v.n3 = p.n3;
    v.ns = node_stride(p.n);
    v.L = p.L;
    v.N = p.N;
    v.nleaf = (int32_t)p.nleaf();
    v.nbox = (int32_t)p.nbox();
    v.leaf_box0 = p.lvl_off[p.L];
    v.verts = d.verts.p;
    v.cent = d.cent.p;
    v.area = d.area.p;
    v.cond = d.cond.p;
    v.w1d = d.w1d.p;
    v.leaf_begin = d.leaf_begin.p;
    v.near_off = d.near_off.p;
    v.near_src = d.near_src.p;
    v.near_S = d.near_S.p;
    v.nval_off = d.nval_off.p;
    v.box_parent = d.box_parent.p;
    v.box_octant = d.box_octant.p;
    v.m2l_off = d.m2l_off.p;
    v.m2l_src = d.m2l_src.p;
    v.m2l_slot = d.m2l_slot.p;
    v.m2m1d = d.m2m1d.p;
    v.m2l_K = m2l ? m2l->K.p : nullptr;
    d.far.lvl_off = p.lvl_off.data();
    d.far.lvl_half = p.lvl_half.data();
    d.far.child_first = d.child_first.p;
    d.far.child_count = d.child_count.p;
    d.far.leaf_of = d.leaf_of.p;
    d.far.m2l_off = p.m2l_off.data();
}

// Tensor-core M2L work lists of every level (groups of kGroup target boxes of
// the same octant class in Morton order sharing one offset loop).
struct TcLists {
    std::vector<TcLevel> level;  // per level (empty below 2)
    TcLevel all;                 // levels 2..L in one list
    DBuf<int32_t> item_t, item_off, slot, src;
};

void build_tc_lists(Ctx& ctx, const Plan& pl, TcLists& out) {
    std::vector<int32_t> it, ioff, sl, src;
    struct LevelRange {
        size_t it0, off0;
        int n;
    };
    std::vector<LevelRange> ranges(pl.L + 1, {0, 0, 0});
    for (int l = 2; l <= pl.L; ++l) {
        ranges[l].it0 = it.size() / kGroup;
        ranges[l].off0 = ioff.size();
        std::vector<int32_t> cls[8];
        for (int32_t b = pl.lvl_off[l]; b < pl.lvl_off[l + 1]; ++b) {
            if (pl.m2l_off[b + 1] == pl.m2l_off[b]) continue;
            const int32_t* c = &pl.box_cell[3 * b];
            cls[(c[0] & 1) | ((c[1] & 1) << 1) | ((c[2] & 1) << 2)].push_back(b);
        }
        int n = 0;
        std::vector<int32_t> per((size_t)kGroup * 343);
        for (auto& v : cls)
            for (size_t k = 0; k < v.size(); k += kGroup) {
                std::fill(per.begin(), per.end(), -1);  // per[slot * kGroup + i]
                for (int i = 0; i < kGroup; ++i) {
                    const int32_t t = k + i < v.size() ? v[k + i] : -1;
                    it.push_back(t);
                    if (t < 0) continue;
                    for (int64_t e = pl.m2l_off[t]; e < pl.m2l_off[t + 1]; ++e)
                        per[(size_t)pl.m2l_slot[e] * kGroup + i] = pl.m2l_src[e];
                }
                ioff.push_back((int32_t)sl.size());
                for (int q = 0; q < 343; ++q) {
                    bool any = false;
                    for (int i = 0; i < kGroup; ++i) any = any || per[(size_t)q * kGroup + i] >= 0;
                    if (!any) continue;
                    sl.push_back(q);
                    for (int i = 0; i < kGroup; ++i) src.push_back(per[(size_t)q * kGroup + i]);
                }
                ++n;
            }
        ranges[l].n = n;
    }
    ioff.push_back((int32_t)sl.size());
    cudaStream_t s = ctx.stream;
    out.item_t.upload(it, s);
    out.item_off.upload(ioff, s);
    out.slot.upload(sl, s);
    out.src.upload(src, s);
    out.level.assign(pl.L + 1, TcLevel());
    for (int l = 2; l <= pl.L; ++l) {
        TcLevel& v = out.level[l];
        v.nitems = ranges[l].n;
        v.item_t = out.item_t.p + (size_t)kGroup * ranges[l].it0;
        v.item_off = out.item_off.p + ranges[l].off0;
        v.slot = out.slot.p;
        v.src = out.src.p;
    }
    // every level in one launch (the per-level item lists are contiguous)
    out.all = TcLevel();
    if (pl.L >= 2) {
        out.all = out.level[2];
        int n = 0;
        for (int l = 2; l <= pl.L; ++l) n += ranges[l].n;
        out.all.nitems = n;
    }
}

// The precorrected potential operator of one plan for R right-hand sides, in
// FP64 (apply) and, for the mixed path, FP32 with tensor-core M2L (apply32).
struct Operator {
    Ctx& ctx;
    const Plan& pl;
    DevPlanBufs& d;
    int R;
    int far_quad;
    bool mixed;
    const DevM2L* m2l;
    DBuf<double> P, inv_diag, E64, L64;
    DBuf<float> P32, E32, L32, X32, W32, Sc32;
    DBuf<float> Xhi32, Xlo32;  // TF32 split of the FP32 apply's input (tensor-core near apply)
    bool p2m_tc = false;       // mixed: P2M on the tensor cores from the split weights below
    bool l2p_tc = false;       // mixed, with p2m_tc: L2P on the tensor cores too
    DBuf<float> Whi32, Wlo32;  // TF32 split of the P2M weights (area folded in), N x 128
    DBuf<float> Shi32, Slo32;  // TF32 split of the L2P weights, N x 128
    DBuf<double> Sc;  // transposed operator: collocation weights as P2M weights
    FarWeights<double> w64;
    FarWeights<float> w32;
    bool transposed = false;
    // Operator applies captured into CUDA graphs, one per (input, output,
    // kind): the first call with a pair runs directly (it also performs the
    // one-time per-kernel attribute set-up), the second captures and every
    // later call replays the graph.
    bool use_graphs = true;
    struct GraphEntry {
        const void* x;
        void* y;
        int kind;
        int seen;
        cudaGraphExec_t exec;
        int64_t nlaunch;
    };
    std::vector<GraphEntry> graphs;
    DBuf<int32_t> tc_err;
    TcLists tc;
    int precond = 0;
    int mixed_near = 0;  // 0: TF32 tensor-core near apply (X split before it), 1: FP32 CUDA cores, 2: tensor cores
                         // with P split hi/lo, 3: as 0 with X gathered as FP32 and split on chip
    BlockJacobi bj;
    bool factored = false;  // M2L through the low-rank factors (compressed operators)
    bool tc32 = false;      // mixed: FP32 M2L on the tensor cores (orders 4 and 5)
    bool shared = false;    // mixed: M2L in the shared compressed basis on the tensor cores (orders 5, 6)
    DBuf<float> Eh32, Lh32; // compressed expansions, nbox x Rb32 x kShared
    FacM2L<double> fac64;
    FacM2L<float> fac32;
    DBuf<int64_t> src_col_off, col_vt, tgt_col_off, tgt_ut, tgt_base;
    DBuf<int32_t> col_tgt, col_pos;
    DBuf<double> T64;
    DBuf<float> T32;
    std::vector<FacLevel> fac_level;
    FacLevel fac_all;
    DBuf<double> box_scale;
    DBuf<int32_t> fi_src, fi_cnt;
    DBuf<int64_t> fi_c0;
    int Rb32 = 0;
    double t_assembly_s = 0.0;
    int64_t applies = 0, applies32 = 0;

    Operator(Ctx& c, const Plan& p, DevPlanBufs& dd, int r, int fq, bool mx, const DevM2L* m)
        : ctx(c), pl(p), d(dd), R(r), far_quad(fq), mixed(mx), m2l(m) {}
    Operator(const Operator&) = delete;
    Operator& operator=(const Operator&) = delete;
    ~Operator() {
        for (auto& g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
    }

    template <class F>
    void run_captured(int kind, const void* x, void* y, F&& body) {
        if (!use_graphs || ctx.profile || ctx.capturing) {
            body();
            return;
        }
        GraphEntry* ge = nullptr;
        for (auto& g : graphs)
            if (g.x == x && g.y == y && g.kind == kind) ge = &g;
        if (!ge) {
            if (graphs.size() >= 16) {  // many distinct buffers: not worth capturing
                body();
                return;
            }
            graphs.push_back({x, y, kind, 0, nullptr, 0});
            ge = &graphs.back();
        }
        if (ge->exec) {
            GPX_CUDA(cudaGraphLaunch(ge->exec, ctx.stream));
            ctx.launches += ge->nlaunch;
            return;
        }
        if (ge->seen++ == 0) {
            body();
            return;
        }
        const int64_t l0 = ctx.launches;
        GPX_CUDA(cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal));
        cudaGraph_t g = nullptr;
        try {
            body();
        } catch (...) {
            cudaStreamEndCapture(ctx.stream, &g);
            if (g) cudaGraphDestroy(g);
            ctx.launches = l0;
            throw;
        }
        GPX_CUDA(cudaStreamEndCapture(ctx.stream, &g));
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        GPX_CUDA(e);
        ge->exec = exec;
        ge->nlaunch = ctx.launches - l0;
        GPX_CUDA(cudaGraphLaunch(exec, ctx.stream));
    }

    bool has_far() const { return pl.far && pl.m2l_pairs() > 0; }

    // Frees the near blocks (FP64 and FP32), the block-Jacobi inverses and the
    // captured applies that read them, once no solve runs with this operator
    // any more; the far field (apply_far_with) stays usable.
    void release_near() {
        for (auto& g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        graphs.clear();
        P.release();
        P32.release();
        bj.Minv.release();
        bj.Minv32.release();
    }

    // Frees everything only the mixed path's FP32 applies use (near blocks in
    // FP32, FP32 expansions, split inputs and weights, FP32 inverses), keeping
    // the FP64 near blocks and far field: after its last FP32 apply the
    // operator can still be transposed and still run apply_far_with.
    void release_mixed() {
        for (auto& g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        graphs.clear();
        P32.release();
        bj.Minv32.release();
        for (auto* b : {&E32, &L32, &X32, &W32, &Sc32, &Xhi32, &Xlo32, &Whi32, &Wlo32, &Shi32, &Slo32, &Eh32, &Lh32})
            b->release();
    }

    // Near blocks: the Wilton assembly, or (fwd given) the transpose of the
    // forward operator's blocks; then the preconditioners and the far-field
    // end weights (swapped for the transpose).
    void assemble(const Operator* fwd = nullptr) {
        cudaStream_t s = ctx.stream;
        transposed = fwd != nullptr;
        P.alloc((size_t)pl.nnz(), s);
        P.zero();  // row padding stays zero
        inv_diag.alloc((size_t)pl.N, s);
        cudaEvent_t e0, e1;
        GPX_CUDA(cudaEventCreate(&e0));
        GPX_CUDA(cudaEventCreate(&e1));
        GPX_CUDA(cudaEventRecord(e0, s));
        if (transposed)
            launch_near_transpose(ctx, d.v, d.near_rev.p, d.near_pre.p, fwd->P.p, P.p, pl.nnz());
        else
            launch_near_assemble(ctx, d.v, pl.nnz(), P.p, kCoulomb);
        GPX_CUDA(cudaEventRecord(e1, s));
        launch_diag_inv(ctx, d.v, P.p, inv_diag.p);
        if (precond >= 1) {
            bj.block = precond == 2 ? 96 : 48;
            bj.build(ctx, pl, d.v, P.p);
            if (mixed) bj.make_f32(ctx);  // every GMRES of the mixed path is an inner solve
        }
        // The host-side set-up below (far-field lists) runs while the device
        // assembles; the assembly time and the preconditioner check are read
        // at the end.
        struct Finish {
            Operator& op;
            cudaEvent_t a, b;
            bool done = false;
            void operator()() {
                GPX_CUDA(cudaEventSynchronize(b));
                float ms = 0.f;
                GPX_CUDA(cudaEventElapsedTime(&ms, a, b));
                op.t_assembly_s = ms * 1e-3;
                if (op.precond >= 1) op.bj.check(op.ctx);
                done = true;
            }
            ~Finish() {
                if (!done) cudaEventSynchronize(b);
                cudaEventDestroy(a);
                cudaEventDestroy(b);
            }
        } finish{*this, e0, e1};
        if (has_far()) {
            const int ns = node_stride(pl.n);
            if (!transposed) {
                d.wsrc.alloc((size_t)pl.N * pl.n3, s);
                launch_src_weights(ctx, d.v, far_quad, d.wsrc.p);
                d.v.wsrc = d.wsrc.p;
                w64 = FarWeights<double>{d.wsrc.p, true, nullptr, false};
            } else {
                Sc.alloc((size_t)pl.N * pl.n3, s);
                launch_centroid_weights(ctx, d.v, nullptr, Sc.p);
                w64 = FarWeights<double>{Sc.p, false, d.wsrc.p, true};
            }
            E64.alloc((size_t)(pl.nbox() + d.far.npart) * ns * R, s);  // + P2M partials
            L64.alloc((size_t)pl.nbox() * ns * R, s);
            {
                // M2L scale 1/half of each box's level, for launches covering all levels
                std::vector<double> sc(pl.nbox(), 0.0);
                for (int l = 0; l <= pl.L; ++l)
                    for (int32_t b = pl.lvl_off[l]; b < pl.lvl_off[l + 1]; ++b) sc[b] = 1.0 / pl.lvl_half[l];
                box_scale.upload(sc, s);
            }
            if (m2l && m2l->factored_ok) setup_factored();
        }
        if (mixed) {
            P32.alloc((size_t)pl.nnz(), s);
            if (mixed_near == 0 || mixed_near == 3)
                launch_to_tf32(ctx, P.p, P32.p, pl.nnz());
            else  // FP32 CUDA-core apply, or the tensor-core apply that splits P on chip
                launch_to_f32(ctx, P.p, P32.p, pl.nnz());
            X32.alloc((size_t)pl.N * R, s);
            if (mixed_near == 0 || mixed_near == 2 || p2m_tc) {  // the split X in memory
                Xhi32.alloc((size_t)pl.N * R, s);
                Xlo32.alloc((size_t)pl.N * R, s);
            }
            tc_err.alloc(1, s);
            tc_err.zero();
            if (has_far()) {
                const int ns = node_stride(pl.n);
                Rb32 = (R + 63) / 64 * 64;
                E32.alloc((size_t)(pl.nbox() + d.far.npart) * ns * Rb32, s);
                L32.alloc((size_t)pl.nbox() * ns * Rb32, s);
                W32.alloc((size_t)pl.N * pl.n3, s);
                launch_to_f32(ctx, d.wsrc.p, W32.p, pl.N * pl.n3);
                if (!transposed) {
                    w32 = FarWeights<float>{W32.p, true, nullptr, false};
                } else {
                    Sc32.alloc((size_t)pl.N * pl.n3, s);
                    launch_to_f32(ctx, Sc.p, Sc32.p, pl.N * pl.n3);
                    w32 = FarWeights<float>{Sc32.p, false, W32.p, true};
                }
                if (p2m_tc) {
                    Whi32.alloc((size_t)pl.N * 128, s);
                    Wlo32.alloc((size_t)pl.N * 128, s);
                    Shi32.alloc((size_t)pl.N * 128, s);
                    Slo32.alloc((size_t)pl.N * 128, s);
                    if (!transposed) {
                        // P2M: source weights with the area; L2P: collocation weights at the centroids
                        launch_split_weights(ctx, d.wsrc.p, pl.n3, d.area.p, true, Whi32.p, Wlo32.p, pl.N);
                        DBuf<double> S64;
                        S64.alloc((size_t)pl.N * pl.n3, s);
                        launch_centroid_weights(ctx, d.v, nullptr, S64.p);
                        launch_split_weights(ctx, S64.p, pl.n3, d.area.p, false, Shi32.p, Slo32.p, pl.N);
                    } else {
                        launch_split_weights(ctx, Sc.p, pl.n3, d.area.p, false, Whi32.p, Wlo32.p, pl.N);
                        launch_split_weights(ctx, d.wsrc.p, pl.n3, d.area.p, true, Shi32.p, Slo32.p, pl.N);
                    }
                }
                if (tc32 || shared) build_tc_lists(ctx, pl, tc);
                if (shared) {
                    ensure_shared(ctx, *const_cast<DevM2L*>(m2l));
                    Eh32.alloc((size_t)pl.nbox() * Rb32 * kShared, s);
                    Lh32.alloc((size_t)pl.nbox() * Rb32 * kShared, s);
                    Lh32.zero();
                    L32.zero();
                }
            }
        }
        finish();
    }

    // Column lists of the factored M2L: phase 1 per source box, phase 2 per
    // target box (see farfield.cu).
    void setup_factored() {
        const int64_t np = pl.m2l_pairs(), nb = pl.nbox();
        const int ns = node_stride(pl.n);
        const std::vector<int32_t>& rank = m2l->rank;  // host copy: no device round trip
        std::vector<int64_t> tcol(nb + 1, 0), base(nb, 0), pos_of_pair(np);
        std::vector<int32_t> tgt_of_pair(np);
        int64_t acc = 0;
        for (int64_t b = 0; b < nb; ++b) {
            int64_t k = 0;
            for (int64_t e = pl.m2l_off[b]; e < pl.m2l_off[b + 1]; ++e) {
                pos_of_pair[e] = k;
                tgt_of_pair[e] = (int32_t)b;
                k += rank[pl.m2l_slot[e]];
            }
            tcol[b + 1] = tcol[b] + k;
            base[b] = acc;
            acc += (k + 3) & ~int64_t(3);
        }
        std::vector<int64_t> ut(tcol[nb]);
        for (int64_t b = 0; b < nb; ++b) {
            int64_t j = tcol[b];
            for (int64_t e = pl.m2l_off[b]; e < pl.m2l_off[b + 1]; ++e)
                for (int k = 0; k < rank[pl.m2l_slot[e]]; ++k)
                    ut[j++] = ((int64_t)pl.m2l_slot[e] * kFacMaxRank + k) * ns;
        }
        // phase-1 columns grouped by source box
        std::vector<int64_t> scol(nb + 1, 0);
        for (int64_t e = 0; e < np; ++e) scol[pl.m2l_src[e] + 1] += rank[pl.m2l_slot[e]];
        for (int64_t b = 0; b < nb; ++b) scol[b + 1] += scol[b];
        std::vector<int64_t> cvt(scol[nb]), fill(scol.begin(), scol.end() - 1);
        std::vector<int32_t> ctg(scol[nb]), cps(scol[nb]);
        for (int64_t e = 0; e < np; ++e) {
            const int s = pl.m2l_src[e], slot = pl.m2l_slot[e];
            for (int k = 0; k < rank[slot]; ++k) {
                const int64_t c = fill[s]++;
                cvt[c] = ((int64_t)slot * kFacMaxRank + k) * ns;
                ctg[c] = tgt_of_pair[e];
                cps[c] = (int32_t)(pos_of_pair[e] + k);
            }
        }
        // phase-1 work items per level: each source box's columns in pieces of
        // at most kFacItemCols (one CTA stages the source expansion once per piece)
        std::vector<int32_t> isrc, icnt;
        std::vector<int64_t> ic0;
        std::vector<int> lvl_first(pl.L + 2, 0);
        for (int l = 0; l <= pl.L; ++l) {
            lvl_first[l] = (int)isrc.size();
            for (int32_t b = pl.lvl_off[l]; b < pl.lvl_off[l + 1]; ++b)
                for (int64_t c = scol[b]; c < scol[b + 1]; c += kFacItemCols) {
                    isrc.push_back(b);
                    ic0.push_back(c);
                    icnt.push_back((int32_t)std::min<int64_t>(kFacItemCols, scol[b + 1] - c));
                }
        }
        lvl_first[pl.L + 1] = (int)isrc.size();
        cudaStream_t s = ctx.stream;
        fi_src.upload(isrc, s);
        fi_cnt.upload(icnt, s);
        fi_c0.upload(ic0, s);
        fac_level.assign(pl.L + 1, FacLevel());
        for (int l = 0; l <= pl.L; ++l) {
            FacLevel& fl = fac_level[l];
            fl.nitems = lvl_first[l + 1] - lvl_first[l];
            fl.item_src = fi_src.p + lvl_first[l];
            fl.item_c0 = fi_c0.p + lvl_first[l];
            fl.item_cnt = fi_cnt.p + lvl_first[l];
        }
        // all levels in one launch: the phase-1 items of levels 2..L, and the
        // M2L scale 1/half of each box's level
        const int lf = std::min(2, pl.L + 1);
        fac_all.nitems = lvl_first[pl.L + 1] - lvl_first[lf];
        fac_all.item_src = fi_src.p + lvl_first[lf];
        fac_all.item_c0 = fi_c0.p + lvl_first[lf];
        fac_all.item_cnt = fi_cnt.p + lvl_first[lf];

        src_col_off.upload(scol, s);
        col_vt.upload(cvt, s);
        col_tgt.upload(ctg, s);
        col_pos.upload(cps, s);
        tgt_col_off.upload(tcol, s);
        tgt_ut.upload(ut, s);
        tgt_base.upload(base, s);
        auto wire = [&](auto& f) {
            f.ns = ns;
            f.box_scale = box_scale.p;
            f.src_col_off = src_col_off.p;
            f.col_vt = col_vt.p;
            f.col_tgt = col_tgt.p;
            f.col_pos = col_pos.p;
            f.tgt_col_off = tgt_col_off.p;
            f.tgt_ut = tgt_ut.p;
            f.tgt_base = tgt_base.p;
        };
        wire(fac64);
        wire(fac32);
        T64.alloc((size_t)acc * R, s);
        T64.zero();  // padding columns stay zero
        fac64.Tm = T64.p;
        fac64.Ut = m2l->Ut64.p;
        fac64.Vt = m2l->Vt64.p;
        if (mixed) {  // also with the tensor-core M2L: the stall guard may switch to this form
            Rb32 = (R + 63) / 64 * 64;
            T32.alloc((size_t)acc * Rb32, s);
            T32.zero();
            fac32.Tm = T32.p;
            fac32.Ut = m2l->Ut32.p;
            fac32.Vt = m2l->Vt32.p;
        }
        factored = true;
    }

    // Y = A X in FP64 (X, Y: N x R, leaf-sorted panel order).
    void apply(const double* X, double* Y) {
        run_captured(0, X, Y, [&] { apply_direct(X, Y); });
        applies += 1;
    }
    void apply_direct(const double* X, double* Y) {
        launch_near_apply(ctx, d.v, pl.nnz(), P.p, X, Y, R);
        if (has_far()) {
            M2LLevelFn<double> m2l_fn = [&](int level, int b0, int nb, double scale) {
                if (factored)
                    launch_m2l_fac<double>(ctx, fac64, level < 0 ? fac_all : fac_level[level], b0, nb, L64.p, E64.p,
                                           R, scale);
                else
                    launch_m2l64(ctx, d.v, b0, nb, L64.p, E64.p, R, scale);
            };
            launch_far_field<double>(ctx, d.v, d.far, X, w64, Y, R, R, E64.p, L64.p, kCoulomb, m2l_fn, factored);
        }
    }

    // Y += far field of X with the given end weights (FP64).
    void apply_far_with(const double* X, double* Y, const FarWeights<double>& w) {
        if (!has_far()) return;
        M2LLevelFn<double> m2l_fn = [&](int level, int b0, int nb, double scale) {
            if (factored)
                launch_m2l_fac<double>(ctx, fac64, level < 0 ? fac_all : fac_level[level], b0, nb, L64.p, E64.p, R,
                                       scale);
            else
                launch_m2l64(ctx, d.v, b0, nb, L64.p, E64.p, R, scale);
        };
        launch_far_field<double>(ctx, d.v, d.far, X, w, Y, R, R, E64.p, L64.p, kCoulomb, m2l_fn, factored);
    }

    // Y = A32 X: FP32 near field, FP32 far field with TF32 tensor-core M2L.
    void apply32(const double* X, double* Y) {
        run_captured(1, X, Y, [&] { apply32_direct(X, Y); });
        applies32 += 1;
    }
    void apply32_direct(const double* X, double* Y) {
        if (mixed_near == 3 && !p2m_tc) {
            // X gathered once as FP32 and split on chip
            launch_to_f32(ctx, X, X32.p, pl.N * R);
            launch_near_apply_tc(ctx, d.v, pl.nnz(), d.nitems128, d.item128_leaf.p, d.item128_row0.p, P32.p, X32.p,
                                 nullptr, Y, R, tc_err.p, false);
        } else if (mixed_near != 1) {
            launch_split_tf32(ctx, X, X32.p, Xhi32.p, Xlo32.p, pl.N * R);
            if (mixed_near == 3)
                launch_near_apply_tc(ctx, d.v, pl.nnz(), d.nitems128, d.item128_leaf.p, d.item128_row0.p, P32.p,
                                     X32.p, nullptr, Y, R, tc_err.p, false);
            else
                launch_near_apply_tc(ctx, d.v, pl.nnz(), d.nitems128, d.item128_leaf.p, d.item128_row0.p, P32.p,
                                     Xhi32.p, Xlo32.p, Y, R, tc_err.p, mixed_near == 2);
        } else {
            launch_to_f32(ctx, X, X32.p, pl.N * R);
            launch_near_apply32(ctx, d.v, pl.nnz(), P32.p, X32.p, Y, R);
        }
        if (has_far()) {
            M2LLevelFn<float> m2l_fn = [&](int level, int b0, int nb, double scale) {
                if (shared) {
                    // E^ = V^T E, L^ = sum_o C_o E^ (tensor cores), L = U L^ for the boxes [b0, b0 + nb)
                    const int ns = node_stride(pl.n);
                    const int64_t row0 = (int64_t)b0 * Rb32, nrows = (int64_t)nb * Rb32;
                    // L^ rows of boxes with M2L work are overwritten; the others stay
                    // at the zero they were allocated with
                    launch_m2l_compress(ctx, E32.p, ns, m2l->Vt_hi.p, m2l->Vt_lo.p, Eh32.p, row0, nrows, tc_err.p);
                    launch_m2l_tc(ctx, level < 0 ? tc.all : tc.level[level], kShared, Eh32.p, Lh32.p, m2l->C32.p,
                                  Rb32, (float)scale, level < 0 ? box_scale.p : nullptr, tc_err.p);
                    launch_m2l_decompress(ctx, Lh32.p, m2l->U_hi.p, m2l->U_lo.p, ns, L32.p, row0, nrows, tc_err.p);
                } else if (tc32)
                    launch_m2l_tc(ctx, level < 0 ? tc.all : tc.level[level], node_stride(pl.n), E32.p, L32.p,
                                  m2l->K32.p, Rb32, (float)scale, level < 0 ? box_scale.p : nullptr, tc_err.p);
                else
                    launch_m2l_fac<float>(ctx, fac32, level < 0 ? fac_all : fac_level[level], b0, nb, L32.p, E32.p,
                                          Rb32, scale);
            };
            const P2MSplit sp{Whi32.p, Wlo32.p, Xhi32.p, Xlo32.p, tc_err.p, l2p_tc ? Shi32.p : nullptr,
                              l2p_tc ? Slo32.p : nullptr};
            // the shared-basis decompression overwrites every local expansion of
            // levels 2 and deeper (L and L^ were cleared once, when allocated)
            launch_far_field<float>(ctx, d.v, d.far, X32.p, w32, Y, R, Rb32, E32.p, L32.p, kCoulomb, m2l_fn, true,
                                    p2m_tc ? &sp : nullptr, shared);
        }
    }

    // Z (+)= M^-1 V with the chosen right preconditioner (V offset on the
    // device by di when given).
    void precondition(const double* V, double* Z, bool add, const DevIndex& di = DevIndex()) {
        if (precond >= 1 && mixed)
            bj.apply32(ctx, V, Z, pl.N, R, add, di);
        else if (precond >= 1)
            bj.apply(ctx, V, Z, pl.N, R, add, di);
        else
            launch_diag_scale(ctx, V, inv_diag.p, Z, pl.N, R, add, di);
    }

    // Switch the FP32 M2L from the tensor cores to the factored form (kept
    // ready whenever the operators are compressed); drops captured graphs of
    // the FP32 apply.  Returns false when no factored form exists.
    bool drop_tc_m2l() {
        if ((!tc32 && !shared) || !factored) return false;
        tc32 = false;
        shared = false;
        for (auto& g : graphs)
            if (g.kind == 1) {
                if (g.exec) cudaGraphExecDestroy(g.exec);
                g.exec = nullptr;
                g.seen = 0;
                g.x = nullptr;
                g.y = nullptr;
            }
        return true;
    }

    void check_tc() {
        if (!mixed) return;
        int e = 0;
        tc_err.download(&e, 1);
        GPX_CUDA(cudaStreamSynchronize(ctx.stream));
        if (e) throw Error(GPX_ERR_CUDA, "tensor-core pipeline wait expired (near apply or M2L)");
    }
};

__global__ void k_accum_c(const int32_t* __restrict__ cond, const double* __restrict__ area,
                          const double* __restrict__ X, int64_t N, int R, double* __restrict__ C) {
    const int i = blockIdx.x;
    const int nsub = 256 / R;
    const int r = threadIdx.x % R, sub = threadIdx.x / R;
    double acc = 0.0;
    if (sub < nsub)
        for (int64_t n = sub; n < N; n += nsub)
            if (cond[n] == i) acc += X[n * R + r] * area[n];
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    if (sub == 0) {
        double s = red[r];
        for (int k = 1; k < nsub; ++k) s += red[k * R + r];
        C[(int64_t)i * R + r] = s;
    }
}

__global__ void k_clamp_min(double* v, int n, double lo) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = fmax(v[i], lo);
}

struct SolveStats {
    int iterations = 0;
    int cycles = 0;
    double max_resid = 0.0;
    bool converged = false;
    std::string hist;  // mixed path: the residual after each refinement step (for error messages)
    int m_used = 0;    // GMRES restart length after the memory budget (largest over the solves)
};

using ApplyFn = std::function<void(const double*, double*)>;
using PrecondFn = std::function<void(const double*, double*, bool, const DevIndex&)>;

// The device-side Arnoldi loop of one gmres_multi call: a CUDA graph whose
// first node evaluates the loop condition and whose conditional WHILE node
// runs one Arnoldi step per pass (operator apply, Gram-Schmidt, Givens) and
// then advances the step counter on the device.  The loop ends when every
// column has converged or the restart length is reached, so a cycle needs no
// host round trip per step.
struct ArnoldiGraph {
    cudaGraphExec_t exec = nullptr;
    ArnoldiGraph() = default;
    ArnoldiGraph(const ArnoldiGraph&) = delete;
    ArnoldiGraph& operator=(const ArnoldiGraph&) = delete;
    ~ArnoldiGraph() {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

// Restart length for a Krylov basis of (m + 1) vectors of NR values of
// elem bytes each: the requested m, cut to what fits in the larger of 16 GB
// and 60 % of the device memory free at the start of the solve (at least 20).
int restart_within_budget(int m, int64_t NR, int elem) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
    const double budget = std::max(16.0 * (1ull << 30), 0.6 * (double)free_b);
    const int64_t fit = (int64_t)(budget / ((double)elem * (double)NR)) - 1;
    return (int)std::max<int64_t>(std::min<int64_t>(20, m), std::min<int64_t>(m, fit));
}

// Restarted right-preconditioned GMRES(m) on all R columns at once
// (krylov.rs:50-191 per column); X (N x R) receives the solution.  The
// right-hand sides are B (N x R) when given, else the unit-conductor vectors
// of rhs_cond (cap/solver.rs:55-63).  With device_loop the Arnoldi steps of a
// cycle run as one graph launch (ArnoldiGraph; the first step of the call
// runs directly, which also does the kernels' one-time set-up); otherwise
// the host launches each step and reads the active-column count after it.
// TB is the storage type of the basis: double, or float for the inner
// solves of the mixed path (every product, sum and Hessenberg entry stays
// FP64; the newest vector is also kept in FP64 for the next preconditioner
// apply, so the basis is only rounded where Gram-Schmidt and the final
// combination read it).
template <class TB>
void gmres_multi_t(Ctx& ctx, const ApplyFn& A, const PrecondFn& Minv, const int32_t* d_cond,
                   const int32_t* d_rhs_cond, const double* B, int R, int64_t N, double tol, int m, int max_restarts,
                   DBuf<double>& X, SolveStats& st, bool reorth, bool device_loop) {
    constexpr bool f32 = sizeof(TB) == 4;
    cudaStream_t s = ctx.stream;
    const int64_t NR = N * R;
    // A shorter restart than asked for keeps the asked-for iteration cap
    // (max_restarts x m): more, shorter cycles.
    const int m_asked = m;
    m = restart_within_budget(m, NR, (int)sizeof(TB));
    if (m < m_asked) max_restarts = (int)std::min<int64_t>(1000, (int64_t)max_restarts * ((m_asked + m - 1) / m));
    DBuf<TB> V;
    DBuf<double> Vcur;  // FP32 basis: the newest basis vector in FP64
    DBuf<double> W, Z, Res, H, cs, sn, g, y, h1, h2, hnorm, bnorm, bcur, est, resid, beta, partial;
    DBuf<int32_t> act, done, kused, cnt, kdev;
    V.alloc((size_t)(m + 1) * NR, s);
    if (f32) Vcur.alloc(NR, s);
    W.alloc(NR, s);
    Z.alloc(NR, s);
    Res.alloc(NR, s);
    H.alloc((size_t)(m + 1) * m * R, s);
    cs.alloc((size_t)m * R, s);
    sn.alloc((size_t)m * R, s);
    g.alloc((size_t)(m + 1) * R, s);
    y.alloc((size_t)m * R, s);
    h1.alloc((size_t)(m + 1) * R, s);
    h2.alloc((size_t)(m + 1) * R, s);
    h2.zero();  // stays zero without the re-orthogonalisation pass
    for (auto* b : {&hnorm, &bnorm, &bcur, &est, &resid, &beta}) b->alloc(R, s);
    act.alloc(R, s);
    done.alloc(R, s);
    kused.alloc(R, s);
    cnt.alloc(1, s);
    kdev.alloc(1, s);
    const int nblk = reduce_blocks_for(N);
    partial.alloc((size_t)nblk * (m + 1) * R, s);
    X.alloc(NR, s);
    X.zero();
    done.zero();
    kused.zero();
    GmresDev gd{m, R, tol, H.p, cs.p, sn.p, g.p, y.p, h1.p, h2.p, hnorm.p, bnorm.p, bcur.p, est.p, resid.p,
                act.p, done.p, kused.p};
    // pinned host words: [0] active-column count, [1] loop step counter read
    // back, [2] loop step counter to start from
    int32_t* hcount = nullptr;
    GPX_CUDA(cudaMallocHost((void**)&hcount, 4 * sizeof(int32_t)));
    struct HostFree {
        int32_t* p;
        ~HostFree() { cudaFreeHost(p); }
    } hf{hcount};
    auto read_count = [&](const int32_t* flags, bool count_zero) -> int {
        launch_count_active(ctx, flags, R, cnt.p);
        GPX_CUDA(cudaMemcpyAsync(hcount, cnt.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        GPX_CUDA(cudaStreamSynchronize(s));
        return count_zero ? R - *hcount : *hcount;
    };
    // One Arnoldi step: k from the host, or (kd) from device memory.
    auto step = [&](int k, const int32_t* kd) {
        const DevIndex dk{kd, NR, 0}, dk1{kd, NR, 1};
        if constexpr (f32)
            Minv(Vcur.p, Z.p, false, DevIndex());
        else
            Minv(kd ? V.p : V.p + (int64_t)k * NR, Z.p, false, dk);
        A(Z.p, W.p);
        const int ni = kd ? m : k + 1;  // launch sizes cover the largest k
        launch_multidot(ctx, V.p, NR, ni, W.p, N, R, partial.p, nblk, h1.p, 0, K_GS_DOT, kd);
        launch_multi_axpy(ctx, V.p, NR, ni, h1.p, W.p, N, R, kd);
        if (reorth) {
            launch_multidot(ctx, V.p, NR, ni, W.p, N, R, partial.p, nblk, h2.p, 0, K_GS_DOT, kd);
            launch_multi_axpy(ctx, V.p, NR, ni, h2.p, W.p, N, R, kd);
        }
        launch_colnorm(ctx, W.p, N, R, partial.p, nblk, hnorm.p);
        if constexpr (f32)
            launch_scale_cols(ctx, W.p, hnorm.p, 1e-14, kd ? V.p : V.p + (int64_t)(k + 1) * NR, Vcur.p, N, R, dk1);
        else
            launch_scale_cols(ctx, W.p, hnorm.p, 1e-14, kd ? V.p : V.p + (int64_t)(k + 1) * NR, N, R, dk1);
        launch_givens(ctx, gd, k, kd);
    };
    ArnoldiGraph loop;
    int64_t step_launches = 0;  // kernels of one pass of the loop body
    auto build_loop = [&] {
        cudaGraph_t gr = nullptr;
        GPX_CUDA(cudaGraphCreate(&gr, 0));
        struct GraphFree {
            cudaGraph_t g;
            ~GraphFree() {
                if (g) cudaGraphDestroy(g);
            }
        } gf{gr};
        cudaGraphConditionalHandle h;
        GPX_CUDA(cudaGraphConditionalHandleCreate(&h, gr, 0, cudaGraphCondAssignDefault));
        GPX_CUDA(cudaStreamBeginCaptureToGraph(s, gr, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        try {
            launch_loop_ctl(ctx, h, act.p, R, kdev.p, m, false);
        } catch (...) {
            cudaGraph_t dummy;
            cudaStreamEndCapture(s, &dummy);
            throw;
        }
        GPX_CUDA(cudaStreamEndCapture(s, &gr));
        size_t nn = 0;
        GPX_CUDA(cudaGraphGetNodes(gr, nullptr, &nn));
        std::vector<cudaGraphNode_t> deps(nn);
        GPX_CUDA(cudaGraphGetNodes(gr, deps.data(), &nn));
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t wn;
        GPX_CUDA(cudaGraphAddNode(&wn, gr, deps.data(), nn, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        const int64_t l0 = ctx.launches;
        ctx.capturing = true;
        GPX_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        try {
            step(0, kdev.p);
            launch_loop_ctl(ctx, h, act.p, R, kdev.p, m, true);
        } catch (...) {
            ctx.capturing = false;
            cudaGraph_t dummy;
            cudaStreamEndCapture(s, &dummy);
            throw;
        }
        ctx.capturing = false;
        GPX_CUDA(cudaStreamEndCapture(s, &body));
        ctx.launches = l0;  // captured, not launched
        GPX_CUDA(cudaGraphInstantiate(&loop.exec, gr, 0));
        size_t bn = 0;
        GPX_CUDA(cudaGraphGetNodes(body, nullptr, &bn));
        step_launches = (int64_t)bn;
    };
    // ||b|| (krylov.rs:58, clamped to the smallest positive normal)
    if (B)
        GPX_CUDA(cudaMemcpyAsync(Res.p, B, (size_t)NR * sizeof(double), cudaMemcpyDeviceToDevice, s));
    else
        launch_residual(ctx, d_cond, d_rhs_cond, nullptr, Res.p, N, R);
    launch_colnorm(ctx, Res.p, N, R, partial.p, nblk, bnorm.p);
    {
        KTimer kt(ctx, K_SMALL);
        k_clamp_min<<<(R + 63) / 64, 64, 0, s>>>(bnorm.p, R, 2.2250738585072014e-308);
        GPX_LAUNCH_CHECK();
        ctx.launches += 1;
    }
    st = SolveStats();
    st.m_used = m;
    for (int cycle = 0; cycle < max_restarts; ++cycle) {
        st.cycles = cycle + 1;
        launch_colnorm(ctx, Res.p, N, R, partial.p, nblk, beta.p);
        launch_cycle_start(ctx, gd, beta.p);
        if constexpr (f32)
            launch_scale_cols(ctx, Res.p, beta.p, 0.0, V.p, Vcur.p, N, R);
        else
            launch_scale_cols(ctx, Res.p, beta.p, 0.0, V.p, N, R);
        if (read_count(act.p, false) == 0) break;
        int kmax = 0;
        if (device_loop && !loop.exec) {
            // first step of the call directly, then the loop graph
            step(0, nullptr);
            st.iterations += 1;
            kmax = 1;
            if (m > 1 && read_count(act.p, false) > 0) build_loop();
        }
        if (device_loop && loop.exec && kmax < m) {
            hcount[2] = kmax;
            GPX_CUDA(cudaMemcpyAsync(kdev.p, hcount + 2, sizeof(int32_t), cudaMemcpyHostToDevice, s));
            GPX_CUDA(cudaGraphLaunch(loop.exec, s));
            GPX_CUDA(cudaMemcpyAsync(hcount + 1, kdev.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            GPX_CUDA(cudaStreamSynchronize(s));
            const int k1 = hcount[1];
            ctx.launches += (int64_t)(k1 - kmax) * step_launches + 1;
            st.iterations += k1 - kmax;
            kmax = k1;
        } else if (!device_loop) {
            for (int k = 0; k < m; ++k) {
                step(k, nullptr);
                st.iterations += 1;
                kmax = k + 1;
                if (read_count(act.p, false) == 0) break;
            }
        }
        launch_trisolve(ctx, gd);
        launch_lincomb(ctx, V.p, NR, kmax, y.p, Z.p, N, R);
        Minv(Z.p, X.p, true, DevIndex());  // x += M^-1 (V y)  (krylov.rs:154-168)
        A(X.p, W.p);
        if (B)
            launch_sub(ctx, B, W.p, Res.p, NR);
        else
            launch_residual(ctx, d_cond, d_rhs_cond, W.p, Res.p, N, R);
        launch_colnorm(ctx, Res.p, N, R, partial.p, nblk, beta.p);
        launch_cycle_end(ctx, gd, beta.p);
        if (read_count(done.p, true) == 0) break;
    }
    std::vector<double> hres(R);
    std::vector<int32_t> hdone(R);
    resid.download(hres.data(), R);
    done.download(hdone.data(), R);
    GPX_CUDA(cudaStreamSynchronize(s));
    st.converged = true;
    for (int r = 0; r < R; ++r) {
        st.max_resid = std::max(st.max_resid, hres[r]);
        if (!hdone[r]) st.converged = false;
    }
}

void gmres_multi(Ctx& ctx, const ApplyFn& A, const PrecondFn& Minv, const int32_t* d_cond,
                 const int32_t* d_rhs_cond, const double* B, int R, int64_t N, double tol, int m, int max_restarts,
                 DBuf<double>& X, SolveStats& st, bool reorth = true, bool device_loop = false, bool basis32 = false) {
    if (basis32)
        gmres_multi_t<float>(ctx, A, Minv, d_cond, d_rhs_cond, B, R, N, tol, m, max_restarts, X, st, reorth,
                             device_loop);
    else
        gmres_multi_t<double>(ctx, A, Minv, d_cond, d_rhs_cond, B, R, N, tol, m, max_restarts, X, st, reorth,
                              device_loop);
}

}  // namespace

Opts normalize(const gpx_solve_opts* o) {
    Opts r;
    if (!o) return r;
    r.precision = o->precision;
    r.order = o->order > 0 ? o->order : 4;
    r.max_level = o->max_level != 0 ? o->max_level : 4;
    r.m2l_mode = o->m2l_mode;
    r.tol = o->tol > 0.0 ? o->tol : 1e-8;
    r.restart = o->restart > 0 ? o->restart : 200;
    r.max_restarts = o->max_restarts > 0 ? o->max_restarts : 50;
    r.dense_below = o->dense_below == 0 ? 500 : o->dense_below;
    r.precond = o->precond;
    r.skip_ground_rhs = o->skip_ground_rhs;
    // The TF32 near apply perturbs the inner operator by ~2^-11 per entry, so
    // inner solves past 1e-3 buy little; the FP32-accurate near applies
    // (CUDA cores, or tensor cores with P split) support 1e-5.
    r.inner_tol_exp = o->inner_tol_exp > 0 ? o->inner_tol_exp : ((o->mixed_near == 0 || o->mixed_near == 3) ? 3 : 5);
    r.mesh_max_edge = o->mesh_max_edge_m;
    r.max_panels = o->max_panels;
    r.far_quad = o->far_quad;
    r.mixed_near = o->mixed_near;
    r.mixed_m2l = o->mixed_m2l;
    r.graphs = o->no_graphs ? 0 : 1;
    r.batch_streams = o->batch_streams;
    r.col_begin = o->col_begin;
    r.col_count = o->col_count;
    r.mixed_far_tc = o->mixed_far_tc;
    r.inner_basis32 = o->inner_basis32;
    return r;
}

int choose_depth(const Opts& o, int64_t n, const double* verts) {
    if (o.dense_below > 0 && n < o.dense_below) return 1;
    if (o.max_level > 0) return o.max_level;
    // auto: about 32 panels per occupied leaf for surface meshes (~n^(1/2)
    // leaves per level step), but no leaf smaller than the largest panel: the
    // far field interpolates each panel's sources in its leaf's box, which
    // breaks down when panels reach far outside it
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY}, ext = 0.0;
    if (verts)
        for (int64_t i = 0; i < n; ++i) {
            const double* v = verts + 12 * i;
            double plo[3] = {INFINITY, INFINITY, INFINITY}, phi[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int k = 0; k < 4; ++k)
                for (int dd = 0; dd < 3; ++dd) {
                    plo[dd] = std::min(plo[dd], v[3 * k + dd]);
                    phi[dd] = std::max(phi[dd], v[3 * k + dd]);
                }
            for (int dd = 0; dd < 3; ++dd) {
                ext = std::max(ext, phi[dd] - plo[dd]);
                const double c = 0.5 * (plo[dd] + phi[dd]);
                lo[dd] = std::min(lo[dd], c);
                hi[dd] = std::max(hi[dd], c);
            }
        }
    const double side = verts ? std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2])) : 0.0;
    int d = 2;
    while (d < 10 && (double)n / std::pow(4.0, d) > 32.0 && (!verts || side / std::pow(2.0, d + 1) >= ext)) ++d;
    return d;
}

static void check_problem(int64_t n, const double* verts, const int32_t* cond, int ncond, const Opts& o) {
    if (n <= 0 || !verts) throw Error(GPX_ERR_CAPACITANCE, "no panels in geometry");
    if (ncond <= 0 || ncond > 4096) throw Error(GPX_ERR_INVALID_ARG, "n_conductors must be in [1, 4096]");
    if (o.order < 2 || o.order > 6) throw Error(GPX_ERR_INVALID_ARG, "Chebyshev order must be in [2, 6]");
    if (o.precision == GPX_PREC_MIXED && o.order < 4)
        throw Error(GPX_ERR_INVALID_ARG, "the mixed-precision path runs expansion orders 4 to 6");
    if (o.precision == GPX_PREC_MIXED && o.m2l_mode == GPX_M2L_EXACT && o.mixed_m2l != 3 &&
        (o.mixed_m2l == 1 || o.order > 5 || (o.far_quad != 0 && o.mixed_m2l != 2)))
        throw Error(GPX_ERR_INVALID_ARG,
                    "the mixed-precision path runs exact M2L operators on the tensor cores, at orders 4 and 5 "
                    "with centroid far-field sources (far_quad 0)");
    if (o.far_quad != 0 && o.far_quad != 1) throw Error(GPX_ERR_INVALID_ARG, "far_quad must be 0 or 1");
    if (o.precond < 0 || o.precond > 2) throw Error(GPX_ERR_INVALID_ARG, "precond must be 0, 1 or 2");
    if (o.mixed_near < 0 || o.mixed_near > 3) throw Error(GPX_ERR_INVALID_ARG, "mixed_near must be 0, 1, 2 or 3");
    if (o.mixed_m2l < 0 || o.mixed_m2l > 3) throw Error(GPX_ERR_INVALID_ARG, "mixed_m2l must be 0, 1, 2 or 3");
    if (o.mixed_far_tc < 0 || o.mixed_far_tc > 2) throw Error(GPX_ERR_INVALID_ARG, "mixed_far_tc must be 0, 1 or 2");
    if (o.inner_basis32 != 0 && o.inner_basis32 != 1) throw Error(GPX_ERR_INVALID_ARG, "inner_basis32 must be 0 or 1");
    for (int64_t i = 0; i < n; ++i) {
        if (cond && (cond[i] < 0 || cond[i] >= ncond))
            throw Error(GPX_ERR_INVALID_ARG, "panel " + std::to_string(i) + " has conductor out of range");
        for (int k = 0; k < 12; ++k)
            if (!std::isfinite(verts[12 * i + k]))
                throw Error(GPX_ERR_INVALID_ARG, "panel " + std::to_string(i) + " has a non-finite vertex");
    }
}

namespace {

// Host plans of one thread reuse the storage of the thread's previous plan:
// build_plan overwrites every field, and the pages of its vectors are
// already mapped, which saves the page faults of tens of MB per solve.  One
// plan per thread is kept between calls.
thread_local std::unique_ptr<Plan> t_spare_plan;

struct Prepared {
    std::unique_ptr<Plan> plan_owner;
    Plan& plan;
    std::shared_ptr<DevM2L> m2l;
    DevPlanBufs dp;
    std::unique_ptr<Operator> op;
    Prepared()
        : plan_owner(t_spare_plan ? std::move(t_spare_plan) : std::unique_ptr<Plan>(new Plan())), plan(*plan_owner) {}
    // the plan goes back to the thread's spare slot; op and dp, destroyed
    // after this body, still find it alive there
    ~Prepared() { t_spare_plan = std::move(plan_owner); }
    Prepared(const Prepared&) = delete;
    Prepared& operator=(const Prepared&) = delete;
};

void prepare(Ctx& ctx, int64_t n, const double* verts, const int32_t* cond, int ncond, const Opts& o, int R,
             int depth, Prepared& pr) {
    build_plan(pr.plan, n, verts, cond, ncond, o.order, depth);
    if (pr.plan.far && pr.plan.m2l_pairs() > 0) pr.m2l = get_m2l(ctx, o.order, o.m2l_mode);
    upload_plan(ctx, pr.plan, pr.m2l.get(), pr.dp);
    pr.op.reset(new Operator(ctx, pr.plan, pr.dp, R, o.far_quad, o.precision == GPX_PREC_MIXED, pr.m2l.get()));
    pr.op->precond = o.precond;
    pr.op->mixed_near = o.mixed_near;
    pr.op->use_graphs = o.graphs != 0;
    // TF32 M2L only with centroid sources: with 2x2 Gauss sources the leaf
    // expansions carry large alternating node values (sources slightly outside
    // their leaf box) and the TF32 inputs lose 1e-2 of the far field.
    pr.op->shared = o.precision == GPX_PREC_MIXED && o.mixed_m2l == 3 && (o.order == 5 || o.order == 6);
    pr.op->p2m_tc = o.precision == GPX_PREC_MIXED && o.mixed_far_tc >= 1 && o.mixed_near != 1 &&
                    (o.order == 4 || o.order == 5);
    pr.op->l2p_tc = pr.op->p2m_tc && o.mixed_far_tc == 1;
    pr.op->tc32 = !pr.op->shared && o.precision == GPX_PREC_MIXED && o.mixed_m2l != 1 &&
                  (o.order == 4 || o.order == 5) &&
                  (o.far_quad == 0 || o.m2l_mode == GPX_M2L_EXACT || o.mixed_m2l >= 2);
    pr.op->assemble();
}

// FP64 iterative refinement around inner GMRES solves with the FP32 /
// tensor-core operator: x += A32^-1 (b - A x) until the FP64 residual meets
// the tolerance (design precedent: refine.rs:45-95, f32 LU + f64 residual).
void mixed_solve(Ctx& ctx, Operator& op, const int32_t* d_cond, const int32_t* d_rhs, const double* B, int R,
                 int64_t N, const Opts& o, DBuf<double>& X, SolveStats& st, int& outer) {
    cudaStream_t s = ctx.stream;
    const int64_t NR = N * R;
    const double floor_tol = std::pow(10.0, -o.inner_tol_exp);
    DBuf<double> Res, W, D, partial, bn, rn;
    DBuf<int32_t> mask;
    Res.alloc(NR, s);
    W.alloc(NR, s);
    X.alloc(NR, s);
    X.zero();
    const int nblk = reduce_blocks_for(N);
    partial.alloc((size_t)nblk * R, s);
    bn.alloc(R, s);
    rn.alloc(R, s);
    mask.alloc(R, s);
    if (B)
        GPX_CUDA(cudaMemcpyAsync(Res.p, B, (size_t)NR * sizeof(double), cudaMemcpyDeviceToDevice, s));
    else
        launch_residual(ctx, d_cond, d_rhs, nullptr, Res.p, N, R);
    launch_colnorm(ctx, Res.p, N, R, partial.p, nblk, bn.p);
    std::vector<double> hb(R), hr(R);
    std::vector<int32_t> hm(R);
    bn.download(hb.data(), R);
    GPX_CUDA(cudaStreamSynchronize(s));
    for (double& v : hb) v = std::max(v, 2.2250738585072014e-308);
    st = SolveStats();
    outer = 0;
    const ApplyFn a32 = [&](const double* x, double* y) { op.apply32(x, y); };
    double prev_resid = INFINITY;
    for (int it = 0; it <= 12; ++it) {
        launch_colnorm(ctx, Res.p, N, R, partial.p, nblk, rn.p);
        rn.download(hr.data(), R);
        GPX_CUDA(cudaStreamSynchronize(s));
        bool all = true;
        prev_resid = it == 0 ? INFINITY : st.max_resid;
        st.max_resid = 0.0;
        for (int r = 0; r < R; ++r) {
            const double rel = hr[r] / hb[r];
            st.max_resid = std::max(st.max_resid, rel);
            hm[r] = rel <= o.tol;
            all = all && hm[r];
        }
        {
            char b[48];
            snprintf(b, sizeof b, "%s%.1e", st.hist.empty() ? "" : " ", st.max_resid);
            st.hist += b;
        }
        if (all) {
            st.converged = true;
            break;
        }
        if (it == 12) break;
        // Stall guard: a refinement step must cut the residual tenfold; if it
        // did not, the TF32 M2L (forced with Gauss-point sources) is too far
        // from the FP64 operator here, so continue with the factored FP32 M2L.
        if (st.max_resid > 0.1 * prev_resid && op.drop_tc_m2l()) st.hist += " [factored M2L from here]";
        mask.upload(hm, s);
        launch_zero_cols(ctx, Res.p, mask.p, N, R);
        // Adaptive inner tolerance: ask each inner solve for no more than the
        // outer residual still needs (x 0.3 margin), but never below the floor
        // 10^-inner_tol_exp that the FP32 operator supports.
        const double need = 0.3 * o.tol / std::max(st.max_resid, 1e-300);
        const double inner_tol = std::min(0.1, std::max(need, floor_tol));
        SolveStats in;
        // Inner solves stop at 1e-3..1e-5: one classical Gram-Schmidt pass keeps the basis
        // orthogonal far below that, so the re-orthogonalisation pass is skipped.  A basis
        // stored in FP32 (inner_basis32) holds at 1e-3; at 1e-5 it loses orthogonality and
        // the inner solves take 1.5-2.5x the iterations (measured).
        const PrecondFn pc = [&](const double* v, double* z, bool add, const DevIndex& di) {
            op.precondition(v, z, add, di);
        };
        gmres_multi(ctx, a32, pc, d_cond, d_rhs, Res.p, R, N, inner_tol, o.restart, std::min(o.max_restarts, 3), D, in,
                    false, o.graphs != 0 && !ctx.profile, o.inner_basis32 != 0);
        st.iterations += in.iterations;
        st.m_used = std::max(st.m_used, in.m_used);
        launch_add(ctx, X.p, D.p, NR);
        op.apply(X.p, W.p);
        if (B)
            launch_sub(ctx, B, W.p, Res.p, NR);
        else
            launch_residual(ctx, d_cond, d_rhs, W.p, Res.p, N, R);
        outer += 1;
    }
    op.check_tc();
}

// Solve op X = B (B null: the unit-conductor right-hand sides of d_rhs,
// cap/solver.rs:55-63) with the options' precision.  The all-pairs path
// stands in for the reference's dense LU (cap/solver.rs:114-117), so it is
// solved to a tighter tolerance that matches a direct solve.
void solve_columns(Ctx& ctx, Operator& op, const Opts& o, bool dense, const int32_t* d_cond, const int32_t* d_rhs,
                   const double* B, int R, int64_t n, DBuf<double>& X, SolveStats& st, int& outer) {
    const double tol = dense ? std::min(o.tol, 1e-12) : o.tol;
    outer = 0;
    if (o.precision == GPX_PREC_MIXED) {
        Opts oi = o;
        oi.tol = tol;
        mixed_solve(ctx, op, d_cond, d_rhs, B, R, n, oi, X, st, outer);
    } else {
        const ApplyFn a64 = [&](const double* x, double* y) { op.apply(x, y); };
        const PrecondFn pc = [&](const double* v, double* z, bool add, const DevIndex& di) {
            op.precondition(v, z, add, di);
        };
        gmres_multi(ctx, a64, pc, d_cond, d_rhs, B, R, n, tol, o.restart, o.max_restarts, X, st, true,
                    o.graphs != 0 && !ctx.profile);
    }
}

// Q[k][r] = a_k if panel k belongs to the conductor of column r, else 0.
__global__ void k_rhs_areas(const int32_t* __restrict__ cond, const double* __restrict__ area,
                            const int32_t* __restrict__ rhs, int64_t N, int R, double* __restrict__ Q) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * R) return;
    const int64_t k = i / R;
    const int r = (int)(i % R);
    Q[i] = cond[k] == rhs[r] ? area[k] : 0.0;
}

// C (ncond x ncond) from the solved columns (R x ... device X); columns not
// solved are filled by symmetry, the unsolved diagonal entry is NaN.

}  // namespace

void cap_solve(Ctx& ctx, int64_t n, const double* verts, const int32_t* cond, int ncond, const Opts& o, double* C,
               gpx_solve_report* rep, const double* panel_eps) {
    const double t0 = now_s();
    const int64_t l0 = ctx.launches;
    check_problem(n, verts, cond, ncond, o);
    const int depth = choose_depth(o, n, verts);
    const bool dense = depth == 1;
    const int Rall = (!o.skip_ground_rhs || ncond == 1) ? ncond : ncond - 1;  // conductors of a full solve
    if (o.col_count < 0 || (o.col_count > 0 && (o.col_begin < 0 || o.col_begin + o.col_count > ncond)))
        throw Error(GPX_ERR_INVALID_ARG, "column subset [col_begin, col_begin + col_count) outside the conductors");
    // conductor columns solved: [cb, cb + Rn)
    const int cb = o.col_count > 0 ? o.col_begin : 0;
    const int Rn = o.col_count > 0 ? o.col_count : Rall;
    const bool full = o.col_count == 0;
    // Conductors are solved in chunks of at most kMaxChunk columns sharing one
    // operator (its expansion and Krylov buffers are sized for one chunk).
    // Columns are padded to a multiple of 4 (16-byte rows); padding columns
    // have a zero right-hand side and converge at once.
    constexpr int kMaxChunk = 128;
    const int Rc = std::min(Rn, kMaxChunk);
    const int R = (Rc + 3) & ~3;
    if (panel_eps)
        for (int64_t k = 0; k < n; ++k)
            if (!std::isfinite(panel_eps[k]) || panel_eps[k] <= 0.0)
                throw Error(GPX_ERR_INVALID_ARG, "panel permittivities must be finite and positive (panel " +
                                                     std::to_string(k) + ")");
    Prepared pr;
    prepare(ctx, n, verts, cond, ncond, o, R, depth, pr);
    Operator& op = *pr.op;
    // charge weight of each panel in the solver's order: its area, or its
    // area times its own permittivity
    const double* d_weight = pr.dp.area.p;
    DBuf<double> eps_area;
    if (panel_eps) {
        std::vector<double> w(n);
        for (int64_t k = 0; k < n; ++k) w[k] = pr.plan.area[k] * panel_eps[pr.plan.perm[k]];
        eps_area.upload(w, ctx.stream);
        d_weight = eps_area.p;
    }
    GPX_CUDA(cudaStreamSynchronize(ctx.stream));
    const double t1 = now_s();
    SolveStats st;
    st.converged = true;
    int outer = 0;
    std::vector<double> hc((size_t)ncond * Rn);  // C[i][j] for the solved columns j
    for (int c0 = 0; c0 < Rn; c0 += Rc) {
        const int nc = std::min(Rc, Rn - c0);
        std::vector<int32_t> rhs_cond(R);
        for (int r = 0; r < R; ++r) rhs_cond[r] = r < nc ? cb + c0 + r : -1;
        DBuf<int32_t> d_rhs;
        d_rhs.upload(rhs_cond, ctx.stream);
        DBuf<double> X;
        SolveStats sc;
        int oc = 0;
        solve_columns(ctx, op, o, dense, pr.dp.cond.p, d_rhs.p, nullptr, R, n, X, sc, oc);
        st.iterations = std::max(st.iterations, sc.iterations);
        st.m_used = std::max(st.m_used, sc.m_used);
        st.max_resid = std::max(st.max_resid, sc.max_resid);
        if (!sc.converged && st.converged) st.hist = sc.hist;
        st.converged = st.converged && sc.converged;
        outer = std::max(outer, oc);
        DBuf<double> dC;
        dC.alloc((size_t)ncond * R, ctx.stream);
        {
            KTimer kt(ctx, K_VEC, (8.0 * R + 12.0) * (double)n, 2.0 * (double)n * R);
            k_accum_c<<<ncond, 256, 0, ctx.stream>>>(pr.dp.cond.p, d_weight, X.p, n, R, dC.p);
            GPX_LAUNCH_CHECK();
            ctx.launches += 1;
        }
        std::vector<double> part((size_t)ncond * R);
        dC.download(part.data(), part.size());
        GPX_CUDA(cudaStreamSynchronize(ctx.stream));
        for (int i = 0; i < ncond; ++i)
            for (int r = 0; r < nc; ++r) hc[(size_t)i * Rn + c0 + r] = part[(size_t)i * R + r];
    }
    const double t2 = now_s();
    for (int i = 0; i < ncond; ++i)
        for (int j = 0; j < ncond; ++j) {
            double v;
            if (j >= cb && j < cb + Rn)
                v = hc[(size_t)i * Rn + (j - cb)];
            else if (full && i < Rn && !panel_eps)
                v = hc[(size_t)j * Rn + i];  // substrate column by symmetry
            else
                v = std::nan("");
            C[(size_t)i * ncond + j] = v;
        }
    if (rep) {
        gpx_solve_report& r = *rep;
        r.n_panels = n;
        r.n_conductors = ncond;
        r.n_rhs = Rn;
        r.order = o.order;
        r.max_level = depth;
        r.n_boxes = pr.plan.nbox();
        r.n_leaves = pr.plan.nleaf();
        r.nnz_near = pr.plan.near_pairs();
        r.m2l_pairs = pr.plan.m2l_pairs();
        r.iterations = st.iterations;
        r.outer_iterations = outer;
        r.operator_applies = op.applies + op.applies32;
        r.max_rel_residual = st.max_resid;
        r.converged = st.converged ? 1 : 0;
        r.dense = dense ? 1 : 0;
        r.t_setup_s = t1 - t0;
        r.t_solve_s = t2 - t1;
        r.t_total_s = t2 - t0;
        r.t_near_assembly_s = op.t_assembly_s;
        r.kernel_launches = ctx.launches - l0;
        r.restart_used = st.m_used;
    }
    if (!st.converged)
        throw Error(GPX_ERR_CAPACITANCE, "GMRES did not converge: max relative residual " +
                                             std::to_string(st.max_resid) + " after " + std::to_string(st.iterations) +
                                             " iterations (restart length " + std::to_string(st.m_used) + ")" +
                                             (st.hist.empty() ? "" : "; residual after each refinement step: " + st.hist));
}

void operator_apply(Ctx& ctx, int64_t n, const double* verts, const Opts& o, int Rn, const double* sigma, double* y,
                    gpx_solve_report* rep) {
    check_problem(n, verts, nullptr, 1, o);
    if (Rn <= 0 || Rn > 256) throw Error(GPX_ERR_INVALID_ARG, "nrhs must be in [1, 256]");
    const int R = (Rn + 3) & ~3;
    const int depth = choose_depth(o, n, verts);
    Prepared pr;
    prepare(ctx, n, verts, nullptr, 1, o, R, depth, pr);
    const Plan& plan = pr.plan;
    std::vector<double> xs((size_t)n * R, 0.0), ys((size_t)n * R);
    for (int64_t s = 0; s < n; ++s)
        for (int r = 0; r < Rn; ++r) xs[(size_t)s * R + r] = sigma[(size_t)plan.perm[s] * Rn + r];
    DBuf<double> X, Y;
    X.upload(xs, ctx.stream);
    Y.alloc(xs.size(), ctx.stream);
    if (o.precision == GPX_PREC_MIXED) {
        pr.op->apply32(X.p, Y.p);
        pr.op->check_tc();
    } else {
        pr.op->apply(X.p, Y.p);
    }
    Y.download(ys.data(), ys.size());
    GPX_CUDA(cudaStreamSynchronize(ctx.stream));
    for (int64_t s = 0; s < n; ++s)
        for (int r = 0; r < Rn; ++r) y[(size_t)plan.perm[s] * Rn + r] = ys[(size_t)s * R + r];
    if (rep) {
        rep->n_panels = n;
        rep->max_level = depth;
        rep->order = o.order;
        rep->n_boxes = plan.nbox();
        rep->n_leaves = plan.nleaf();
        rep->nnz_near = plan.near_pairs();
        rep->m2l_pairs = plan.m2l_pairs();
        rep->dense = depth == 1;
        rep->t_near_assembly_s = pr.op->t_assembly_s;
    }
}

void potential_matrix(Ctx& ctx, int64_t ns, const double* sv, int64_t nt, const double* pts, double* out) {
    if (ns <= 0 || nt <= 0) return;
    DBuf<double> a, b, c;
    a.upload(sv, (size_t)ns * 12, ctx.stream);
    b.upload(pts, (size_t)nt * 3, ctx.stream);
    c.alloc((size_t)ns * nt, ctx.stream);
    launch_potential_matrix(ctx, a.p, ns, b.p, nt, c.p, kCoulomb);
    c.download(out, (size_t)ns * nt);
    GPX_CUDA(cudaStreamSynchronize(ctx.stream));
}


void cap_sensitivity(Ctx& ctx, int64_t n, const double* verts, const int32_t* cond, int ncond, const Opts& o,
                     int np, const double* V, int nrows, const int32_t* rows, double* C, double* dCdp,
                     gpx_solve_report* rep) {
    const double t0 = now_s();
    const int64_t l0 = ctx.launches;
    check_problem(n, verts, cond, ncond, o);
    if (np < 0 || np > 4096 || (np > 0 && !V)) throw Error(GPX_ERR_INVALID_ARG, "n_params must be in [0, 4096]");
    for (int64_t i = 0; i < (int64_t)np * n * 12; ++i)
        if (!std::isfinite(V[i])) throw Error(GPX_ERR_INVALID_ARG, "non-finite vertex velocity");
    const int depth = choose_depth(o, n, verts);
    const bool dense = depth == 1;
    const int Rn = (!o.skip_ground_rhs || ncond == 1) ? ncond : ncond - 1;
    // rows of dC: the listed conductors, or every solved conductor
    std::vector<int32_t> rowlist;
    if (rows) {
        if (nrows < 1 || nrows > Rn) throw Error(GPX_ERR_INVALID_ARG, "gradient rows must list 1 to n_rhs conductors");
        std::vector<char> seen(Rn, 0);
        for (int k = 0; k < nrows; ++k) {
            if (rows[k] < 0 || rows[k] >= Rn || seen[rows[k]])
                throw Error(GPX_ERR_INVALID_ARG, "gradient row " + std::to_string(rows[k]) +
                                                     " is not a solved conductor or repeats");
            seen[rows[k]] = 1;
            rowlist.push_back(rows[k]);
        }
    } else {
        for (int k = 0; k < Rn; ++k) rowlist.push_back(k);
    }
    const int nr = (int)rowlist.size();
    // Columns (forward solves) and rows (transposed solves) run in chunks of at
    // most 128 right-hand sides; the forward densities of all columns and the
    // adjoint densities of all rows stay resident (N x (Rn + nr) doubles).
    constexpr int kMaxChunk = 128;
    const int R = (std::min(Rn, kMaxChunk) + 3) & ~3;
    const int Ra = (std::min(nr, kMaxChunk) + 3) & ~3;
    cudaStream_t s = ctx.stream;
    Prepared pr;
    prepare(ctx, n, verts, cond, ncond, o, R, depth, pr);
    Operator& op = *pr.op;
    const Plan& pl = pr.plan;
    const double t_assembly = op.t_assembly_s;
    // forward: P sigma_j = b_j
    std::vector<DBuf<double>> Xs;
    std::vector<int32_t> col0;
    SolveStats st, stT;
    int outer = 0, outerT = 0, its = 0, itsT = 0;
    int64_t applies = 0;
    std::vector<double> hc((size_t)ncond * Rn);
    {
        DBuf<int32_t> d_rhs;
        DBuf<double> dC;
        dC.alloc((size_t)ncond * R, s);
        std::vector<double> part((size_t)ncond * R);
        for (int c0 = 0; c0 < Rn; c0 += R) {
            const int nc = std::min(R, Rn - c0);
            std::vector<int32_t> rc(R);
            for (int r = 0; r < R; ++r) rc[r] = r < nc ? c0 + r : -1;
            d_rhs.upload(rc, s);
            Xs.emplace_back();
            col0.push_back(c0);
            int oc = 0;
            solve_columns(ctx, op, o, dense, pr.dp.cond.p, d_rhs.p, nullptr, R, n, Xs.back(), st, oc);
            if (!st.converged)
                throw Error(GPX_ERR_CAPACITANCE, "GMRES did not converge (forward): max relative residual " +
                                                     std::to_string(st.max_resid));
            its = std::max(its, st.iterations);
            outer = std::max(outer, oc);
            {
                KTimer kt(ctx, K_VEC, (8.0 * R + 12.0) * (double)n, 2.0 * (double)n * R);
                k_accum_c<<<ncond, 256, 0, s>>>(pr.dp.cond.p, pr.dp.area.p, Xs.back().p, n, R, dC.p);
                GPX_LAUNCH_CHECK();
                ctx.launches += 1;
            }
            dC.download(part.data(), part.size());
            GPX_CUDA(cudaStreamSynchronize(s));
            for (int i = 0; i < ncond; ++i)
                for (int r = 0; r < nc; ++r) hc[(size_t)i * Rn + c0 + r] = part[(size_t)i * R + r];
        }
        op.check_tc();
    }
    for (int i = 0; i < ncond; ++i)
        for (int j = 0; j < ncond; ++j)
            C[(size_t)i * ncond + j] = j < Rn ? hc[(size_t)i * Rn + j]
                                              : (i < Rn ? hc[(size_t)j * Rn + i] : std::nan(""));
    // adjoint: P^T lambda_i = q_i for the gradient rows (its own operator of
    // width Ra; the forward near blocks are freed once transposed)
    std::vector<DBuf<double>> Lams;
    std::vector<DBuf<int32_t>> row_rhs;
    {
        std::unique_ptr<Operator> opT(new Operator(ctx, pl, pr.dp, Ra, o.far_quad, o.precision == GPX_PREC_MIXED,
                                                   pr.m2l.get()));
        opT->precond = o.precond;
        opT->mixed_near = o.mixed_near;
        opT->use_graphs = o.graphs != 0;
        opT->tc32 = op.tc32;
        opT->shared = op.shared;
        opT->p2m_tc = op.p2m_tc;
        opT->l2p_tc = op.l2p_tc;
        // the transposed operator is assembled from the forward FP64 blocks;
        // the forward operator's FP32 state goes first, its FP64 blocks right
        // after, so that at most one operator's near blocks of each kind are
        // resident beside sigma
        op.release_mixed();
        opT->assemble(&op);
        applies += op.applies + op.applies32;
        op.release_near();
        DBuf<double> Q;
        Q.alloc((size_t)n * Ra, s);
        for (int k0 = 0; k0 < nr; k0 += Ra) {
            const int nk = std::min(Ra, nr - k0);
            std::vector<int32_t> rr(Ra);
            for (int r = 0; r < Ra; ++r) rr[r] = r < nk ? rowlist[k0 + r] : -1;
            row_rhs.emplace_back();
            row_rhs.back().upload(rr, s);
            {
                KTimer kt(ctx, K_VEC, 16.0 * (double)n * Ra, 0.0);
                k_rhs_areas<<<(unsigned)((n * Ra + 255) / 256), 256, 0, s>>>(pr.dp.cond.p, pr.dp.area.p,
                                                                             row_rhs.back().p, n, Ra, Q.p);
                GPX_LAUNCH_CHECK();
                ctx.launches += 1;
            }
            Lams.emplace_back();
            int oc = 0;
            solve_columns(ctx, *opT, o, dense, pr.dp.cond.p, row_rhs.back().p, Q.p, Ra, n, Lams.back(), stT, oc);
            if (!stT.converged)
                throw Error(GPX_ERR_CAPACITANCE, "GMRES did not converge (adjoint): max relative residual " +
                                                     std::to_string(stT.max_resid));
            itsT = std::max(itsT, stT.iterations);
            outerT = std::max(outerT, oc);
        }
        opT->check_tc();
        applies += opT->applies + opT->applies32;
    }
    // per parameter: dC_ij = dq_i^T sigma_j - lambda_i^T (dP sigma_j)
    DBuf<double> dV, dcent, darea, dP, D, dW, dS, G, Gp;
    dV.alloc((size_t)n * 12, s);
    dcent.alloc((size_t)n * 3, s);
    darea.alloc((size_t)n, s);
    dP.alloc((size_t)pl.nnz(), s);
    dP.zero();
    D.alloc((size_t)n * R, s);
    G.alloc((size_t)Ra * R, s);
    Gp.alloc((size_t)grad_contract_splits(Ra) * Ra * R, s);
    if (op.has_far()) {
        dW.alloc((size_t)n * pl.n3, s);
        dS.alloc((size_t)n * pl.n3, s);
    }
    std::vector<double> vs((size_t)n * 12), hg((size_t)Ra * R);
    for (size_t e = 0; e < (size_t)np * ncond * ncond; ++e) dCdp[e] = std::nan("");
    for (int q = 0; q < np; ++q) {
        const double* Vq = V + (size_t)q * n * 12;
        for (int64_t k = 0; k < n; ++k)
            std::memcpy(&vs[(size_t)k * 12], Vq + (size_t)pl.perm[k] * 12, 12 * sizeof(double));
        dV.upload(vs, s);
        launch_panel_dprops(ctx, pr.dp.v, dV.p, dcent.p, darea.p);
        launch_near_assemble_dual(ctx, pr.dp.v, pl.nnz(), dV.p, dcent.p, dP.p, kCoulomb);
        if (op.has_far()) {
            launch_dsrc_weights(ctx, pr.dp.v, o.far_quad, dV.p, dW.p);
            launch_centroid_weights(ctx, pr.dp.v, dcent.p, dS.p);
        }
        double* out = dCdp + (size_t)q * ncond * ncond;
        for (size_t cc = 0; cc < Xs.size(); ++cc) {
            const double* X = Xs[cc].p;
            launch_near_apply(ctx, pr.dp.v, pl.nnz(), dP.p, X, D.p, R);
            if (op.has_far()) {
                op.apply_far_with(X, D.p, FarWeights<double>{dW.p, false, nullptr, false});
                op.apply_far_with(X, D.p, FarWeights<double>{pr.dp.wsrc.p, true, dS.p, false});
            }
            const int nc = std::min(R, Rn - col0[cc]);
            for (size_t rc = 0; rc < Lams.size(); ++rc) {
                launch_grad_contract(ctx, pr.dp.cond.p, row_rhs[rc].p, darea.p, X, Lams[rc].p, D.p, n, R, Ra, Gp.p,
                                     G.p);
                G.download(hg.data(), hg.size());
                GPX_CUDA(cudaStreamSynchronize(s));
                const int k0 = (int)rc * Ra, nk = std::min(Ra, nr - k0);
                for (int a = 0; a < nk; ++a)
                    for (int j = 0; j < nc; ++j)
                        out[(size_t)rowlist[k0 + a] * ncond + col0[cc] + j] = hg[(size_t)a * R + j];
            }
        }
    }
    const double t1 = now_s();
    if (rep) {
        gpx_solve_report& r = *rep;
        r.n_panels = n;
        r.n_conductors = ncond;
        r.n_rhs = Rn;
        r.order = o.order;
        r.max_level = depth;
        r.n_boxes = pl.nbox();
        r.n_leaves = pl.nleaf();
        r.nnz_near = pl.near_pairs();
        r.m2l_pairs = pl.m2l_pairs();
        r.iterations = its + itsT;
        r.outer_iterations = outer + outerT;
        r.operator_applies = applies;
        r.max_rel_residual = std::max(st.max_resid, stT.max_resid);
        r.converged = 1;
        r.dense = dense ? 1 : 0;
        r.t_solve_s = t1 - t0;
        r.t_total_s = t1 - t0;
        r.t_near_assembly_s = t_assembly;
        r.kernel_launches = ctx.launches - l0;
    }
}


namespace {

// y[s] = sum_l M[s][l] * sigma[l][r] for the sampled rows (one block per row
// and probe column).
__global__ void k_rows_apply(const double* __restrict__ M, int64_t N, const double* __restrict__ sigma, int R,
                             double* __restrict__ y) {
    const int s = blockIdx.x, r = blockIdx.y;
    double acc = 0.0;
    for (int64_t l = threadIdx.x; l < N; l += blockDim.x) acc += M[(int64_t)s * N + l] * sigma[l * R + r];
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) y[(int64_t)s * R + r] = red[0];
}

std::string tune_signature(int64_t n, const double* verts, int ncond, const Opts& o, double target) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY}, edge = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double* v = verts + 12 * i;
        for (int k = 0; k < 4; ++k)
            for (int d = 0; d < 3; ++d) {
                lo[d] = std::min(lo[d], v[3 * k + d]);
                hi[d] = std::max(hi[d], v[3 * k + d]);
            }
        double e = 0.0;
        for (int d = 0; d < 3; ++d) e += (v[3 + d] - v[d]) * (v[3 + d] - v[d]);
        edge += std::sqrt(e);
    }
    edge /= (double)n;
    const double side = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
    char buf[256];
    std::snprintf(buf, sizeof buf, "p%d_n%d_c%d_a%.1f_%.1f_%.1f_e%d_t%d", o.precision, (int)std::lround(std::log2((double)n) * 2),
                  (int)std::lround(std::log2((double)ncond + 1.0) * 2), (hi[0] - lo[0]) / side, (hi[1] - lo[1]) / side,
                  (hi[2] - lo[2]) / side, (int)std::lround(std::log2(side / std::max(edge, 1e-300)) * 2),
                  (int)std::lround(-std::log10(target) * 4));
    return buf;
}

}  // namespace

void autotune(Ctx& ctx, int64_t n, const double* verts, const int32_t* cond, int ncond, const Opts& base,
              double target, const char* cache_path, Opts& out, gpx_tune_report* rep) {
    check_problem(n, verts, cond, ncond, base);
    if (!(target > 0.0) || target >= 1.0) throw Error(GPX_ERR_INVALID_ARG, "target relative error must be in (0, 1)");
    gpx_tune_report r{};
    out = base;
    const std::string sig = tune_signature(n, verts, ncond, base, target);
    if (cache_path && *cache_path) {
        if (FILE* f = std::fopen(cache_path, "r")) {
            char key[256];
            int order, depth, fq, mn;
            double err, ams, sms;
            while (std::fscanf(f, "%255s %d %d %d %d %lf %lf %lf", key, &order, &depth, &fq, &mn, &err, &ams, &sms) == 8)
                if (sig == key) {
                    out.order = order;
                    out.max_level = depth;
                    out.far_quad = fq;
                    out.mixed_near = mn;
                    out.dense_below = -1;
                    r.est_rel_err = err;
                    r.apply_ms = ams;
                    r.setup_ms = sms;
                    r.from_cache = 1;
                }
            std::fclose(f);
            if (r.from_cache) {
                if (rep) *rep = r;
                return;
            }
        }
    }
    cudaStream_t s = ctx.stream;
    const bool mixed = base.precision == GPX_PREC_MIXED;
    // sampled target rows (evenly spaced in caller order) and their exact
    // all-pairs rows of the potential-coefficient matrix
    const int ns = (int)std::min<int64_t>(n, 512);
    std::vector<double> pts((size_t)ns * 3);
    std::vector<int64_t> rows(ns);
    for (int k = 0; k < ns; ++k) {
        rows[k] = (int64_t)((double)k * (double)n / (double)ns);
        double c[3], a;
        panel_centroid_area(verts + 12 * rows[k], c, &a);
        for (int d = 0; d < 3; ++d) pts[3 * k + d] = c[d];
    }
    // probe charge densities: constant, two smooth patterns, seeded random signs
    const int R = 4;
    std::vector<double> sig_h((size_t)n * R);
    uint64_t lcg = 0x9E3779B97F4A7C15ull;
    for (int64_t i = 0; i < n; ++i) {
        double c[3], a;
        panel_centroid_area(verts + 12 * i, c, &a);
        lcg = lcg * 6364136223846793005ull + 1442695040888963407ull;
        sig_h[(size_t)i * R + 0] = 1.0;
        sig_h[(size_t)i * R + 1] = 1.0 + 0.5 * std::sin(1e6 * c[0]) * std::cos(1e6 * c[1]);
        sig_h[(size_t)i * R + 2] = 1.0 + 0.5 * std::cos(7e5 * (c[0] + c[1]) + 3e6 * c[2]);
        sig_h[(size_t)i * R + 3] = (lcg >> 63) ? 1.0 : -1.0;
    }
    DBuf<double> dv, dpts, M, dsig, yex;
    dv.upload(verts, (size_t)n * 12, s);
    dpts.upload(pts, s);
    M.alloc((size_t)ns * n, s);
    dsig.upload(sig_h, s);
    yex.alloc((size_t)ns * R, s);
    launch_potential_matrix(ctx, dv.p, n, dpts.p, ns, M.p, kCoulomb);
    k_rows_apply<<<dim3(ns, R), 256, 0, s>>>(M.p, n, dsig.p, R, yex.p);
    GPX_LAUNCH_CHECK();
    ctx.launches += 1;
    std::vector<double> yexact((size_t)ns * R);
    yex.download(yexact.data(), yexact.size());
    GPX_CUDA(cudaStreamSynchronize(s));
    std::vector<double> ymax(R, 0.0);
    for (int k = 0; k < ns; ++k)
        for (int q = 0; q < R; ++q) ymax[q] = std::max(ymax[q], std::fabs(yexact[(size_t)k * R + q]));

    Opts probe = base;
    probe.dense_below = -1;
    Opts autodepth = base;
    autodepth.max_level = -1;
    autodepth.dense_below = -1;
    const int d0 = std::max(2, choose_depth(autodepth, n, verts));
    struct Cand {
        int order, depth, fq, mn;
    };
    std::vector<Cand> cands;
    for (int order : {4, 5, 6})
        for (int depth = std::max(2, d0 - 1); depth <= d0 + 1; ++depth)
            for (int fq : {0, 1})
                for (int mn : (mixed ? std::vector<int>{0, 3, 1} : std::vector<int>{0})) cands.push_back({order, depth, fq, mn});
    double best_score = INFINITY;
    bool found = false;
    cudaEvent_t e0, e1;
    GPX_CUDA(cudaEventCreate(&e0));
    GPX_CUDA(cudaEventCreate(&e1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } eg{e0, e1};
    for (const Cand& c : cands) {
        Opts o = probe;
        o.order = c.order;
        o.max_level = c.depth;
        o.far_quad = c.fq;
        o.mixed_near = c.mn;
        o.precond = base.precond;
        Prepared pr;
        const double t0 = now_s();
        prepare(ctx, n, verts, cond, ncond, o, R, c.depth, pr);
        GPX_CUDA(cudaStreamSynchronize(s));
        const double setup_ms = (now_s() - t0) * 1e3;
        r.candidates += 1;
        // FP64 apply for the discretisation error (the mixed path converges to
        // the FP64 operator's solution), in the plan's panel order
        std::vector<double> xs((size_t)n * R);
        for (int64_t k = 0; k < n; ++k)
            for (int q = 0; q < R; ++q) xs[(size_t)k * R + q] = sig_h[(size_t)pr.plan.perm[k] * R + q];
        DBuf<double> X, Y;
        X.upload(xs, s);
        Y.alloc(xs.size(), s);
        pr.op->apply(X.p, Y.p);
        std::vector<double> ys(xs.size());
        Y.download(ys.data(), ys.size());
        GPX_CUDA(cudaStreamSynchronize(s));
        std::vector<int64_t> inv(n);
        for (int64_t k = 0; k < n; ++k) inv[pr.plan.perm[k]] = k;
        // error of the smooth probes (the fourth, random-sign probe cancels
        // and is not scored); the Maxwell matrix's error measures about 1.7x
        // this, so the target is met with a factor of 2 to spare
        double err = 0.0;
        for (int k = 0; k < ns; ++k)
            for (int q = 0; q < 3; ++q)
                err = std::max(err, std::fabs(ys[(size_t)inv[rows[k]] * R + q] - yexact[(size_t)k * R + q]) / ymax[q]);
        if (2.0 * err > target) continue;
        // time the applies the solve iterates (two warm, three timed)
        auto one = [&] {
            if (mixed)
                pr.op->apply32(X.p, Y.p);
            else
                pr.op->apply(X.p, Y.p);
        };
        one();
        one();
        GPX_CUDA(cudaEventRecord(e0, s));
        for (int k = 0; k < 3; ++k) one();
        GPX_CUDA(cudaEventRecord(e1, s));
        GPX_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        GPX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        const double apply_ms = ms / 3.0;
        if (mixed) pr.op->check_tc();
        // a solve: setup plus about 100 applies (inner iterations of a 1e-8 solve)
        const double score = setup_ms + 100.0 * apply_ms;
        if (score < best_score) {
            best_score = score;
            found = true;
            out.order = c.order;
            out.max_level = c.depth;
            out.far_quad = c.fq;
            out.mixed_near = c.mn;
            out.dense_below = -1;
            r.est_rel_err = err;
            r.apply_ms = apply_ms;
            r.setup_ms = setup_ms;
        }
    }
    if (!found)
        throw Error(GPX_ERR_CAPACITANCE, "no far-field configuration reaches the target error " + std::to_string(target));
    if (cache_path && *cache_path) {
        if (FILE* f = std::fopen(cache_path, "a")) {
            std::fprintf(f, "%s %d %d %d %d %.6e %.6e %.6e\n", sig.c_str(), out.order, out.max_level, out.far_quad,
                         out.mixed_near, r.est_rel_err, r.apply_ms, r.setup_ms);
            std::fclose(f);
        }
    }
    if (rep) *rep = r;
}

}  // namespace gpx
