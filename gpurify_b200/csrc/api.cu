// C ABI of the gpx-pex library (include/gpx_pex.h).  Every entry point maps
// exceptions to a gpx_status and records the message on the context; nothing
// throws across the ABI.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <thread>
#include <cmath>
#include <cstring>

#include "panelize.h"
#include "solver.h"

using namespace gpx;

namespace {

thread_local std::string g_noctx_error;

gpx_status fail(gpx_ctx* ctx, gpx_status s, const std::string& msg) {
    if (ctx)
        ctx->impl.last_error = msg;
    else
        g_noctx_error = msg;
    return s;
}

// Copies host<->device byte counts of one call into its report.
struct CopyMeter {
    gpx_solve_report* r;
    int64_t h0, d0;
    explicit CopyMeter(gpx_solve_report* rep) : r(rep), h0(h2d_counter()), d0(d2h_counter()) {}
    ~CopyMeter() {
        if (r) {
            r->h2d_bytes = h2d_counter() - h0;
            r->d2h_bytes = d2h_counter() - d0;
        }
    }
};

template <class F>
gpx_status guarded(gpx_ctx* ctx, F&& f, uint32_t* err_polygon = nullptr) {
    if (err_polygon) *err_polygon = 0xFFFFFFFFu;
    try {
        if (ctx) {
            ctx->impl.last_error.clear();
            GPX_CUDA(cudaSetDevice(ctx->impl.device));
        }
        f();
        return GPX_OK;
    } catch (const Error& e) {
        if (err_polygon) *err_polygon = e.polygon;
        return fail(ctx, e.status, e.what());
    } catch (const std::bad_alloc&) {
        return fail(ctx, GPX_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(ctx, GPX_ERR_INTERNAL, e.what());
    } catch (...) {
        return fail(ctx, GPX_ERR_INTERNAL, "unknown error");
    }
}

std::vector<VolumeGroup> groups_from_abi(const gpx_volume_group* g, int64_t n, const int32_t* rects) {
    std::vector<VolumeGroup> out;
    out.reserve(n);
    for (int64_t i = 0; i < n; ++i) {
        VolumeGroup v{g[i].net, g[i].z0_m, g[i].z1_m, g[i].dielectric_k, {}};
        v.rects.reserve(g[i].rect_count);
        for (int64_t k = 0; k < g[i].rect_count; ++k) {
            const int32_t* r = rects + 4 * (g[i].rect_offset + k);
            v.rects.push_back({r[0], r[1], r[2], r[3]});
        }
        out.push_back(std::move(v));
    }
    return out;
}

// Maxwell solve of panelised groups with the bridge's k scaling and per-net
// diagonal extraction (bridge.rs:393-442).  One k everywhere: the vacuum
// solve scaled by that k.  Several k: every panel is a conductor panel in its
// own surrounding k and its charge counts k times (bridge.rs:409-430 ->
// cap/dielectric.rs:76-150 with conductor roles); the reference takes that
// path only below 500 panels (all pairs), this solver at any size.
void solve_panelized(Ctx& ctx, const PanelizeResult& pr, const Opts& o, std::vector<double>& C,
                     gpx_solve_report* rep) {
    const int ncond = (int)pr.nets.size() + 1;
    C.assign((size_t)ncond * ncond, 0.0);
    if (pr.homogeneous) {
        cap_solve(ctx, pr.panels.size(), pr.panels.verts.data(), pr.panels.cond.data(), ncond, o, C.data(), rep);
        for (double& v : C) v *= pr.first_eps;
    } else {
        cap_solve(ctx, pr.panels.size(), pr.panels.verts.data(), pr.panels.cond.data(), ncond, o, C.data(), rep,
                  pr.panels.eps.data());
    }
    for (size_t i = 0; i < pr.nets.size(); ++i) {
        const double af = C[i * ncond + i] * 1.0e18;
        if (!std::isfinite(af) || af < 0.0)
            throw Error(GPX_ERR_NON_FINITE,
                        "quasi-static solver returned a non-finite capacitance for net " + std::to_string(pr.nets[i]));
    }
}

}  // namespace

extern "C" {

const char* gpx_version(void) { return "gpx-pex 0.1.0 (sm_100a)"; }

gpx_status gpx_ctx_create(gpx_ctx** out, int device) {
    if (!out) return GPX_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0 || device < 0 || device >= count) {
        cudaGetLastError();
        g_noctx_error = "no CUDA device " + std::to_string(device);
        return GPX_ERR_NO_DEVICE;
    }
    gpx_ctx* c = new (std::nothrow) gpx_ctx();
    if (!c) return GPX_ERR_OUT_OF_MEMORY;
    gpx_status s = guarded(nullptr, [&] {
        c->impl.device = device;
        GPX_CUDA(cudaSetDevice(device));
        GPX_CUDA(cudaStreamCreateWithFlags(&c->impl.stream, cudaStreamNonBlocking));
        GPX_CUDA(cudaDeviceGetAttribute(&c->impl.sm_count, cudaDevAttrMultiProcessorCount, device));
        cudaMemPool_t pool;
        GPX_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t thresh = UINT64_MAX;  // keep freed blocks cached between solves
        GPX_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thresh));
    });
    if (s != GPX_OK) {
        if (c->impl.stream) cudaStreamDestroy(c->impl.stream);
        delete c;
        return s;
    }
    *out = c;
    return GPX_OK;
}

void gpx_ctx_destroy(gpx_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->impl.device);
    ctx->impl.m2l_cache.clear();
    if (ctx->impl.stream) {
        cudaStreamSynchronize(ctx->impl.stream);
        cudaStreamDestroy(ctx->impl.stream);
    }
    delete ctx;
}

const char* gpx_last_error(const gpx_ctx* ctx) {
    return ctx ? ctx->impl.last_error.c_str() : g_noctx_error.c_str();
}

gpx_status gpx_cap_solve(gpx_ctx* ctx, const gpx_panel_problem* pb, const gpx_solve_opts* opts, double* maxwell_out,
                         gpx_solve_report* report) {
    if (!ctx || !pb || !maxwell_out) return fail(ctx, GPX_ERR_INVALID_ARG, "null argument");
    if (report) std::memset(report, 0, sizeof(*report));
    CopyMeter meter(report);
    return guarded(ctx, [&] {
        Opts o = normalize(opts);
        cap_solve(ctx->impl, pb->n_panels, pb->verts, pb->conductor, pb->n_conductors, o, maxwell_out, report);
    });
}

gpx_status gpx_cap_solve_eps(gpx_ctx* ctx, const gpx_panel_problem* pb, const double* eps, const gpx_solve_opts* opts,
                             double* maxwell_out, gpx_solve_report* report) {
    if (!ctx || !pb || !eps || !maxwell_out) return fail(ctx, GPX_ERR_INVALID_ARG, "null argument");
    if (report) std::memset(report, 0, sizeof(*report));
    CopyMeter meter(report);
    return guarded(ctx, [&] {
        Opts o = normalize(opts);
        cap_solve(ctx->impl, pb->n_panels, pb->verts, pb->conductor, pb->n_conductors, o, maxwell_out, report, eps);
    });
}

// Windows are independent: a work queue, largest estimated cost first, is
// drained by batch_streams worker threads, each with its own stream (a
// private context on the same device), so small and large windows overlap on
// the GPU.  Every window runs the same code path as gpx_cap_solve, so its
// result is identical to a separate call.
gpx_status gpx_cap_solve_batched(gpx_ctx* ctx, const gpx_panel_problem* pbs, int32_t n, const gpx_solve_opts* opts,
                                 double* const* maxwell_out, gpx_solve_report* reports) {
    if (!ctx || n < 0 || (n > 0 && (!pbs || !maxwell_out))) return fail(ctx, GPX_ERR_INVALID_ARG, "null argument");
    return guarded(ctx, [&] {
        Opts o = normalize(opts);
        for (int32_t i = 0; i < n; ++i) {
            if (reports) std::memset(&reports[i], 0, sizeof(reports[i]));
            if (!maxwell_out[i]) throw Error(GPX_ERR_INVALID_ARG, "window " + std::to_string(i) + ": null output");
        }
        const int workers = std::max(1, std::min<int>(n, o.batch_streams > 0 ? std::min(o.batch_streams, 32) : 8));
        if (workers == 1 || ctx->impl.profile) {
            for (int32_t i = 0; i < n; ++i) {
                try {
                    cap_solve(ctx->impl, pbs[i].n_panels, pbs[i].verts, pbs[i].conductor, pbs[i].n_conductors, o,
                              maxwell_out[i], reports ? &reports[i] : nullptr);
                } catch (const Error& e) {
                    throw Error(e.status, "window " + std::to_string(i) + ": " + e.what(), e.polygon);
                }
            }
            return;
        }
        std::vector<int32_t> order(n);
        for (int32_t i = 0; i < n; ++i) order[i] = i;
        auto cost = [&](int32_t i) { return (double)pbs[i].n_panels * std::max(1, pbs[i].n_conductors); };
        std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return cost(a) > cost(b); });
        std::atomic<int32_t> next{0};
        std::atomic<int64_t> launches{0};
        std::vector<gpx_status> st(n, GPX_OK);
        std::vector<std::string> msg(n);
        const int device = ctx->impl.device;
        auto work = [&] {
            gpx_ctx* sub = nullptr;
            if (gpx_ctx_create(&sub, device) != GPX_OK) {
                for (int32_t k; (k = next.fetch_add(1)) < n;) {
                    st[order[k]] = GPX_ERR_CUDA;
                    msg[order[k]] = "could not create a worker stream";
                }
                return;
            }
            for (int32_t k; (k = next.fetch_add(1)) < n;) {
                const int32_t i = order[k];
                gpx_solve_report* r = reports ? &reports[i] : nullptr;
                CopyMeter meter(r);
                st[i] = guarded(sub, [&] {
                    cap_solve(sub->impl, pbs[i].n_panels, pbs[i].verts, pbs[i].conductor, pbs[i].n_conductors, o,
                              maxwell_out[i], r);
                });
                if (st[i] != GPX_OK) msg[i] = sub->impl.last_error;
            }
            launches += sub->impl.launches;
            gpx_ctx_destroy(sub);
        };
        std::vector<std::thread> pool;
        for (int w = 0; w < workers; ++w) pool.emplace_back(work);
        for (auto& t : pool) t.join();
        ctx->impl.launches += launches.load();
        GPX_CUDA(cudaSetDevice(device));
        for (int32_t i = 0; i < n; ++i)
            if (st[i] != GPX_OK) throw Error(st[i], "window " + std::to_string(i) + ": " + msg[i]);
    });
}

gpx_status gpx_cap_sensitivity(gpx_ctx* ctx, const gpx_panel_problem* pb, const gpx_solve_opts* opts, int32_t n_params,
                               const double* vert_velocity, double* maxwell_out, double* dmaxwell_out,
                               gpx_solve_report* report) {
    if (!ctx || !pb || !maxwell_out || (n_params > 0 && (!vert_velocity || !dmaxwell_out)))
        return fail(ctx, GPX_ERR_INVALID_ARG, "null argument");
    if (report) std::memset(report, 0, sizeof(*report));
    CopyMeter meter(report);
    return guarded(ctx, [&] {
        Opts o = normalize(opts);
        cap_sensitivity(ctx->impl, pb->n_panels, pb->verts, pb->conductor, pb->n_conductors, o, n_params,
                        vert_velocity, 0, nullptr, maxwell_out, dmaxwell_out, report);
    });
}

gpx_status gpx_cap_sensitivity_rows(gpx_ctx* ctx, const gpx_panel_problem* pb, const gpx_solve_opts* opts,
                                    int32_t n_params, const double* vert_velocity, int32_t n_rows,
                                    const int32_t* rows, double* maxwell_out, double* dmaxwell_out,
                                    gpx_solve_report* report) {
    if (!ctx || !pb || !maxwell_out || !rows || (n_params > 0 && (!vert_velocity || !dmaxwell_out)))
        return fail(ctx, GPX_ERR_INVALID_ARG, "null argument");
    if (report) std::memset(report, 0, sizeof(*report));
    CopyMeter meter(report);
    return guarded(ctx, [&] {
        Opts o = normalize(opts);
        cap_sensitivity(ctx->impl, pb->n_panels, pb->verts, pb->conductor, pb->n_conductors, o, n_params,
                        vert_velocity, n_rows, rows, maxwell_out, dmaxwell_out, report);
    });
}

gpx_status gpx_autotune(gpx_ctx* ctx, const gpx_panel_problem* pb, const gpx_solve_opts* base, double target_rel_err,
                        const char* cache_path, gpx_solve_opts* tuned, gpx_tune_report* report) {
    if (!ctx || !pb || !tuned) return fail(ctx, GPX_ERR_INVALID_ARG, "null argument");
    if (report) std::memset(report, 0, sizeof(*report));
    return guarded(ctx, [&] {
        Opts o = normalize(base);
        Opts t;
        autotune(ctx->impl, pb->n_panels, pb->verts, pb->conductor, pb->n_conductors, o, target_rel_err, cache_path,
                 t, report);
        gpx_solve_opts res{};
        if (base) res = *base;
        res.order = t.order;
        res.max_level = t.max_level;
        res.far_quad = t.far_quad;
        res.mixed_near = t.mixed_near;
        res.dense_below = -1;
        *tuned = res;
    });
}

gpx_status gpx_operator_apply(gpx_ctx* ctx, const gpx_panel_problem* pb, const gpx_solve_opts* opts, int32_t nrhs,
                              const double* sigma, double* y, gpx_solve_report* report) {
    if (!ctx || !pb || !sigma || !y) return fail(ctx, GPX_ERR_INVALID_ARG, "null argument");
    if (report) std::memset(report, 0, sizeof(*report));
    return guarded(ctx, [&] {
        Opts o = normalize(opts);
        operator_apply(ctx->impl, pb->n_panels, pb->verts, o, nrhs, sigma, y, report);
    });
}

gpx_status gpx_potential_matrix(gpx_ctx* ctx, int64_t n_src, const double* src_verts, int64_t n_tgt,
                                const double* tgt_points, double* out) {
    if (!ctx || (n_src > 0 && !src_verts) || (n_tgt > 0 && !tgt_points) || !out)
        return fail(ctx, GPX_ERR_INVALID_ARG, "null argument");
    return guarded(ctx, [&] { potential_matrix(ctx->impl, n_src, src_verts, n_tgt, tgt_points, out); });
}

gpx_status gpx_cap_solve_groups(gpx_ctx* ctx, const gpx_volume_group* groups, int64_t n_groups, const int32_t* rects,
                                double xy_scale_m, const gpx_solve_opts* opts, uint32_t* nets_out, double* cap_af_out,
                                int64_t nets_cap, int64_t* n_nets, double* maxwell_out, gpx_solve_report* report) {
    if (!ctx || (n_groups > 0 && (!groups || !rects)) || !n_nets) return fail(ctx, GPX_ERR_INVALID_ARG, "null argument");
    if (report) std::memset(report, 0, sizeof(*report));
    CopyMeter meter(report);
    return guarded(ctx, [&] {
        Opts o = normalize(opts);
        *n_nets = 0;
        if (n_groups == 0) return;
        auto gs = groups_from_abi(groups, n_groups, rects);
        thread_local PanelizeResult pr;  // buffers kept between calls of this thread
        const double t0 = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
        panelize_groups(gs, xy_scale_m, o.mesh_max_edge, o.max_panels, pr);
        const double t1 = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
        if ((int64_t)pr.nets.size() > nets_cap) throw Error(GPX_ERR_OUTPUT_CAPACITY, "nets_out too small");
        std::vector<double> C;
        solve_panelized(ctx->impl, pr, o, C, report);
        const size_t nc = pr.nets.size() + 1;
        for (size_t i = 0; i < pr.nets.size(); ++i) {
            if (nets_out) nets_out[i] = pr.nets[i];
            if (cap_af_out) cap_af_out[i] = C[i * nc + i] * 1.0e18;
        }
        if (maxwell_out) std::memcpy(maxwell_out, C.data(), C.size() * sizeof(double));
        *n_nets = (int64_t)pr.nets.size();
        if (report) {
            report->t_panelize_s = t1 - t0;
            report->t_total_s += t1 - t0;
        }
    });
}

gpx_status gpx_extract_quasistatic(gpx_ctx* ctx, const gpx_geometry_store* store, const gpx_deck* deck,
                                   const uint32_t* net_of_poly, int64_t n_nop, const gpx_solve_opts* opts,
                                   gpx_net_parasitics* out, int64_t out_cap, int64_t* n_out, uint32_t* err_polygon,
                                   gpx_solve_report* report) {
    if (!ctx || !store || !deck || !n_out) return fail(ctx, GPX_ERR_INVALID_ARG, "null argument");
    if (report) std::memset(report, 0, sizeof(*report));
    CopyMeter meter(report);
    return guarded(
        ctx,
        [&] {
            Opts o = normalize(opts);
            // The per-net result needs only the nets' diagonal entries: the
            // substrate right-hand side is skipped unless asked for.
            if (!opts) o.skip_ground_rhs = 1;
            *n_out = 0;
            thread_local PanelizeResult pr;  // buffers kept between calls of this thread
            const double t0 =
                std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
            panelize_store(*store, *deck, net_of_poly, n_nop, o.mesh_max_edge, o.max_panels, pr);
            const double t1 =
                std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
            if ((int64_t)pr.out_nets.size() > out_cap) throw Error(GPX_ERR_OUTPUT_CAPACITY, "out too small");
            std::vector<double> C;
            if (!pr.nets.empty()) solve_panelized(ctx->impl, pr, o, C, report);
            const size_t nc = pr.nets.size() + 1;
            for (size_t k = 0; k < pr.out_nets.size(); ++k) {
                const uint32_t net = pr.out_nets[k];
                out[k].net = net;
                out[k].r_ohm = pr.via_r[k];
                auto it = std::lower_bound(pr.nets.begin(), pr.nets.end(), net);
                out[k].cap_af = (it != pr.nets.end() && *it == net) ? C[(size_t)(it - pr.nets.begin()) * (nc + 1)] * 1.0e18
                                                                     : 0.0;
            }
            *n_out = (int64_t)pr.out_nets.size();
            if (report) {
                report->t_panelize_s = t1 - t0;
                report->t_total_s += t1 - t0;
            }
        },
        err_polygon);
}

gpx_status gpx_bridge_panelize(gpx_ctx* ctx, const gpx_geometry_store* store, const gpx_deck* deck,
                               const uint32_t* net_of_poly, int64_t n_nop, const gpx_solve_opts* opts,
                               double* verts_out, int32_t* cond_out, double* eps_out, int64_t cap, int64_t* n_panels,
                               uint32_t* nets_out, int64_t nets_cap, int64_t* n_nets, uint32_t* err_polygon) {
    if (!store || !deck || !n_panels || !n_nets) return fail(ctx, GPX_ERR_INVALID_ARG, "null argument");
    // Host-only: a NULL context is allowed (no device work).
    gpx_status st = guarded(
        nullptr,
        [&] {
            Opts o = normalize(opts);
            thread_local PanelizeResult pr;  // buffers kept between calls of this thread
            panelize_store(*store, *deck, net_of_poly, n_nop, o.mesh_max_edge, o.max_panels, pr);
            *n_panels = pr.panels.size();
            *n_nets = (int64_t)pr.nets.size();
            if (pr.panels.size() > cap) throw Error(GPX_ERR_OUTPUT_CAPACITY, "panel output too small");
            if ((int64_t)pr.nets.size() > nets_cap) throw Error(GPX_ERR_OUTPUT_CAPACITY, "nets_out too small");
            if (verts_out) std::memcpy(verts_out, pr.panels.verts.data(), pr.panels.verts.size() * sizeof(double));
            if (cond_out) std::memcpy(cond_out, pr.panels.cond.data(), pr.panels.cond.size() * sizeof(int32_t));
            if (eps_out) std::memcpy(eps_out, pr.panels.eps.data(), pr.panels.eps.size() * sizeof(double));
            if (nets_out) std::memcpy(nets_out, pr.nets.data(), pr.nets.size() * sizeof(uint32_t));
        },
        err_polygon);
    if (st != GPX_OK && ctx) ctx->impl.last_error = g_noctx_error;
    return st;
}

void* gpx_ctx_stream(gpx_ctx* ctx) { return ctx ? (void*)ctx->impl.stream : nullptr; }

gpx_status gpx_ctx_set_profiling(gpx_ctx* ctx, int32_t on) {
    if (!ctx) return GPX_ERR_INVALID_ARG;
    return guarded(ctx, [&] {
        ctx->impl.drain();
        ctx->impl.profile = on != 0;
    });
}

gpx_status gpx_ctx_kernel_stats(gpx_ctx* ctx, int32_t k, int64_t* launches, double* ms, double* bytes, double* flops,
                                int64_t* total) {
    if (!ctx || k < 0 || k >= K_NTAGS) return fail(ctx, GPX_ERR_INVALID_ARG, "bad kernel class");
    return guarded(ctx, [&] {
        ctx->impl.drain();
        const KStats& s = ctx->impl.kstats[k];
        if (launches) *launches = s.launches;
        if (ms) *ms = s.ms;
        if (bytes) *bytes = s.bytes;
        if (flops) *flops = s.flops;
        if (total) *total = ctx->impl.launches;
    });
}

gpx_status gpx_ctx_reset_stats(gpx_ctx* ctx) {
    if (!ctx) return GPX_ERR_INVALID_ARG;
    return guarded(ctx, [&] {
        ctx->impl.drain();
        for (auto& s : ctx->impl.kstats) s = KStats();
        ctx->impl.launches = 0;
    });
}

gpx_status gpx_plan_check(int64_t n_panels, const double* verts, int32_t order, int32_t depth, int64_t* stats) {
    if (!verts || !stats || n_panels <= 0 || depth < 1 || depth > 12 || order < 2 || order > 8)
        return fail(nullptr, GPX_ERR_INVALID_ARG, "bad argument");
    return guarded(nullptr, [&] {
        Plan p;
        build_plan(p, n_panels, verts, nullptr, 1, order, depth);
        auto bad = [](const std::string& what) { throw Error(GPX_ERR_INTERNAL, "plan invariant broken: " + what); };
        const int64_t nl = p.nleaf(), nb = p.nbox();
        if (p.leaf_begin.front() != 0 || p.leaf_begin.back() != n_panels) bad("leaf ranges");
        std::vector<char> seen(n_panels, 0);
        for (int32_t i : p.perm) {
            if (i < 0 || i >= n_panels || seen[i]) bad("perm");
            seen[i] = 1;
        }
        for (int64_t k = 0; k < nl; ++k) {
            if (p.near_off[k + 1] - p.near_off[k] > 27 || p.near_src[p.near_off[k]] != k) bad("near list");
            int64_t S = 0;
            for (int32_t e = p.near_off[k]; e < p.near_off[k + 1]; ++e) {
                if (p.near_src[e] < 0 || p.near_src[e] >= nl) bad("near source");
                S += p.leaf_begin[p.near_src[e] + 1] - p.leaf_begin[p.near_src[e]];
            }
            if (S != p.near_S[k]) bad("near S");
        }
        int64_t far_pairs = 0;
        for (int64_t b = 0; b < nb; ++b)
            for (int64_t e = p.m2l_off[b]; e < p.m2l_off[b + 1]; ++e) {
                if (p.m2l_src[e] < 0 || p.m2l_src[e] >= nb || p.m2l_slot[e] < 0 || p.m2l_slot[e] >= 343) bad("m2l");
                ++far_pairs;
            }
        for (int64_t b = 0; b < nb; ++b)
            if (p.child_count[b] > 8 || (p.child_count[b] && (p.child_first[b] < 0 || p.child_first[b] + p.child_count[b] > nb)))
                bad("children");
        // every ordered leaf pair is covered exactly once by near blocks or by
        // an M2L pair of some ancestor pair (checked by panel-pair counting)
        int64_t near_pairs = p.near_pairs();
        int64_t covered_far = 0;
        std::vector<int64_t> cnt(nb, 0);
        for (int64_t k = 0; k < nl; ++k) cnt[p.lvl_off[p.L] + k] = p.leaf_begin[k + 1] - p.leaf_begin[k];
        for (int l = p.L; l >= 1; --l)
            for (int32_t b = p.lvl_off[l]; b < p.lvl_off[l + 1]; ++b) cnt[p.box_parent[b]] += cnt[b];
        for (int64_t b = 0; b < nb; ++b)
            for (int64_t e = p.m2l_off[b]; e < p.m2l_off[b + 1]; ++e) covered_far += cnt[b] * cnt[p.m2l_src[e]];
        stats[0] = nl;
        stats[1] = nb;
        stats[2] = near_pairs;
        stats[3] = far_pairs;
        stats[4] = covered_far;
        stats[5] = p.max_leaf;
        stats[6] = p.max_S;
        // FNV-1a over every array the device kernels index, in a fixed order:
        // a plan built another way must reproduce it bit for bit
        uint64_t h = 1469598103934665603ull;
        auto mix = [&h](const void* d, size_t bytes) {
            const unsigned char* c = static_cast<const unsigned char*>(d);
            for (size_t i = 0; i < bytes; ++i) h = (h ^ c[i]) * 1099511628211ull;
        };
        auto vec = [&mix](const auto& v) { mix(v.data(), v.size() * sizeof(v[0])); };
        vec(p.perm);
        vec(p.verts);
        vec(p.cent);
        vec(p.area);
        vec(p.cond);
        vec(p.w1d);
        vec(p.lvl_off);
        vec(p.box_cell);
        vec(p.box_parent);
        vec(p.box_octant);
        vec(p.lvl_half);
        vec(p.child_first);
        vec(p.child_count);
        vec(p.leaf_begin);
        vec(p.leaf_of);
        vec(p.near_off);
        vec(p.near_src);
        vec(p.near_S);
        vec(p.nval_off);
        vec(p.item_leaf);
        vec(p.item_row0);
        vec(p.m2l_off);
        vec(p.m2l_src);
        vec(p.m2l_slot);
        vec(p.m2m1d);
        mix(p.origin, sizeof(p.origin));
        mix(&p.max_leaf, sizeof(p.max_leaf));
        mix(&p.max_S, sizeof(p.max_S));
        std::memcpy(&stats[7], &h, sizeof(h));
        if (near_pairs + covered_far != n_panels * n_panels) bad("pair coverage");
    });
}

}  // extern "C"
