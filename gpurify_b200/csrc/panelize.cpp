// Layout -> boundary-element panels, bit-exact with the reference bridge
// (crates/pex/src/bridge.rs:73-147, :307-386, :445-652,
//  crates/core/src/geometry/rects.rs:96-176, cap/mesh.rs:12-43,
//  analytical/process_stack.rs:31-76).  Coordinates use the same operation
// order as the reference and this file is compiled with -ffp-contract=off,
// so every vertex coordinate matches the reference bit for bit.
#include "panelize.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <set>
#include <string>

namespace gpx {

namespace {

constexpr double kMetresPerNm = 1.0e-9;
constexpr size_t kMaxGridCells = 262144;    // bridge.rs:28
constexpr int64_t kRefMaxPanels = 20000;    // bridge.rs:29

// Face subdivision count.  max_edge == 0: the reference rule (bridge.rs:559-563),
// aspect ratio at most 4:1 and at most 32 pieces.  max_edge > 0: pieces no
// longer than max_edge.
inline size_t pieces(double len, double transverse, double max_edge) {
    if (max_edge > 0.0) return (size_t)std::min(std::max(std::ceil(len / max_edge), 1.0), 1.0e6);
    double v = std::ceil(len / (4.0 * std::max(transverse, 2.2250738585072014e-308)));
    return (size_t)std::min(std::max(v, 1.0), 32.0);
}

struct Sink {
    PanelBuffer& b;
    void quad(const double (&v)[4][3], bool reverse, int32_t c) {
        size_t o = b.verts.size();
        b.verts.resize(o + 12);
        for (int i = 0; i < 4; ++i) {
            const double* src = v[reverse ? 3 - i : i];
            b.verts[o + 3 * i] = src[0];
            b.verts[o + 3 * i + 1] = src[1];
            b.verts[o + 3 * i + 2] = src[2];
        }
        b.cond.push_back(c);
    }
};

// Subdivision coordinate a + (b - a) * i / n, in the reference's order.
inline double lerp_at(double a, double b, size_t i, size_t n) { return a + (b - a) * (double)i / (double)n; }

void face_xy(Sink& s, double x0, double x1, double y0, double y1, double z, int32_t c, bool rev, double me) {
    size_t nx = pieces(x1 - x0, y1 - y0, me), ny = pieces(y1 - y0, x1 - x0, me);
    for (size_t i = 0; i < nx; ++i) {
        double xa = lerp_at(x0, x1, i, nx), xb = lerp_at(x0, x1, i + 1, nx);
        for (size_t j = 0; j < ny; ++j) {
            double ya = lerp_at(y0, y1, j, ny), yb = lerp_at(y0, y1, j + 1, ny);
            double v[4][3] = {{xa, ya, z}, {xb, ya, z}, {xb, yb, z}, {xa, yb, z}};
            s.quad(v, rev, c);
        }
    }
}

// Sidewall at constant x (bridge.rs:599-624); target-edge mode also splits z.
void face_yz(Sink& s, double x, double y0, double y1, double z0, double z1, int32_t c, bool rev, double me) {
    size_t ny = pieces(y1 - y0, z1 - z0, me);
    size_t nz = me > 0.0 ? pieces(z1 - z0, y1 - y0, me) : 1;
    for (size_t j = 0; j < ny; ++j) {
        double ya = lerp_at(y0, y1, j, ny), yb = lerp_at(y0, y1, j + 1, ny);
        for (size_t k = 0; k < nz; ++k) {
            double za = nz == 1 ? z0 : lerp_at(z0, z1, k, nz), zb = nz == 1 ? z1 : lerp_at(z0, z1, k + 1, nz);
            double v[4][3] = {{x, ya, za}, {x, yb, za}, {x, yb, zb}, {x, ya, zb}};
            s.quad(v, rev, c);
        }
    }
}

// Sidewall at constant y (bridge.rs:627-652).
void face_xz(Sink& s, double x0, double x1, double y, double z0, double z1, int32_t c, bool rev, double me) {
    size_t nx = pieces(x1 - x0, z1 - z0, me);
    size_t nz = me > 0.0 ? pieces(z1 - z0, x1 - x0, me) : 1;
    for (size_t i = 0; i < nx; ++i) {
        double xa = lerp_at(x0, x1, i, nx), xb = lerp_at(x0, x1, i + 1, nx);
        for (size_t k = 0; k < nz; ++k) {
            double za = nz == 1 ? z0 : lerp_at(z0, z1, k, nz), zb = nz == 1 ? z1 : lerp_at(z0, z1, k + 1, nz);
            double v[4][3] = {{xa, y, za}, {xb, y, za}, {xb, y, zb}, {xa, y, zb}};
            s.quad(v, rev, c);
        }
    }
}

// Union grid, greedy top/bottom merge, atomic sidewalls (bridge.rs:445-557).
void group_to_panels(const VolumeGroup& g, int32_t c, double xy, double me, Sink& s) {
    std::vector<int32_t> xs, ys;
    xs.reserve(2 * g.rects.size());
    ys.reserve(2 * g.rects.size());
    for (const RectI& r : g.rects) {
        xs.push_back(r.x0);
        xs.push_back(r.x1);
        ys.push_back(r.y0);
        ys.push_back(r.y1);
    }
    std::sort(xs.begin(), xs.end());
    xs.erase(std::unique(xs.begin(), xs.end()), xs.end());
    std::sort(ys.begin(), ys.end());
    ys.erase(std::unique(ys.begin(), ys.end()), ys.end());
    const size_t nx = xs.empty() ? 0 : xs.size() - 1, ny = ys.empty() ? 0 : ys.size() - 1;
    const size_t cells = nx * ny;
    if (cells > kMaxGridCells)
        throw Error(GPX_ERR_GRID_CAPACITY, "conductor union grid needs " + std::to_string(cells) +
                                               " cells; limit is " + std::to_string(kMaxGridCells));
    // Cell occupancy by rectangle rasterisation over the grid indices.
    std::vector<uint8_t> filled(cells, 0), used(cells, 0);
    for (const RectI& r : g.rects) {
        size_t ia = std::lower_bound(xs.begin(), xs.end(), r.x0) - xs.begin();
        size_t ib = std::lower_bound(xs.begin(), xs.end(), r.x1) - xs.begin();
        size_t ja = std::lower_bound(ys.begin(), ys.end(), r.y0) - ys.begin();
        size_t jb = std::lower_bound(ys.begin(), ys.end(), r.y1) - ys.begin();
        for (size_t i = ia; i < ib; ++i)
            for (size_t j = ja; j < jb; ++j) filled[i * ny + j] = 1;
    }
    auto at = [&](size_t i, size_t j) { return filled[i * ny + j] != 0; };
    for (size_t i = 0; i < nx; ++i)
        for (size_t j = 0; j < ny; ++j) {
            if (!at(i, j) || used[i * ny + j]) continue;
            size_t ie = i + 1;
            while (ie < nx && at(ie, j) && !used[ie * ny + j]) ++ie;
            size_t je = j + 1;
            for (;; ++je) {
                if (je >= ny) break;
                bool full = true;
                for (size_t x = i; x < ie && full; ++x) full = at(x, je) && !used[x * ny + je];
                if (!full) break;
            }
            for (size_t x = i; x < ie; ++x)
                for (size_t y = j; y < je; ++y) used[x * ny + y] = 1;
            double x0 = (double)xs[i] * xy, x1 = (double)xs[ie] * xy;
            double y0 = (double)ys[j] * xy, y1 = (double)ys[je] * xy;
            face_xy(s, x0, x1, y0, y1, g.z1, c, false, me);
            face_xy(s, x0, x1, y0, y1, g.z0, c, true, me);
        }
    for (size_t i = 0; i < nx; ++i)
        for (size_t j = 0; j < ny; ++j) {
            if (!at(i, j)) continue;
            double x0 = (double)xs[i] * xy, x1 = (double)xs[i + 1] * xy;
            double y0 = (double)ys[j] * xy, y1 = (double)ys[j + 1] * xy;
            if (i == 0 || !at(i - 1, j)) face_yz(s, x0, y0, y1, g.z0, g.z1, c, true, me);
            if (i + 1 == nx || !at(i + 1, j)) face_yz(s, x1, y0, y1, g.z0, g.z1, c, false, me);
            if (j == 0 || !at(i, j - 1)) face_xz(s, x0, x1, y0, g.z0, g.z1, c, false, me);
            if (j + 1 == ny || !at(i, j + 1)) face_xz(s, x0, x1, y1, g.z0, g.z1, c, true, me);
        }
}

bool volume_conductor(const gpx_layer_params& p) {  // bridge.rs:171-178
    return p.sheet_res_ohm_sq != 0.0 || p.area_cap_af_um2 != 0.0 || p.fringe_cap_af_um != 0.0 ||
           p.coupling_cap_af_um != 0.0 || p.interlayer_cap_af_um2 != 0.0 ||
           (p.thickness_nm > 0.0 && p.via_res_ohm == 0.0);
}

std::string fmt_g(double v) {
    char b[64];
    snprintf(b, sizeof b, "%g", v);
    return b;
}

}  // namespace

void decompose_ring(const int32_t* xs, const int32_t* ys, size_t n, uint32_t poly, std::vector<RectI>& out) {
    const std::string head = "polygon " + std::to_string(poly) + " cannot be extruded for quasi-static PEX: ";
    if (n < 4)
        throw Error(GPX_ERR_UNSUPPORTED_GEOMETRY,
                    head + "polygon " + std::to_string(poly) + " has " + std::to_string(n) +
                        " vertices, need >= 4 for rectilinear decomposition",
                    poly);
    struct HEdge {
        int32_t y, lo, hi;
    };
    std::vector<HEdge> h;
    std::vector<int32_t> bx;
    bx.reserve(n);
    for (size_t i = 0; i < n; ++i) {
        size_t k = (i + 1) % n;
        if (xs[i] != xs[k] && ys[i] != ys[k])
            throw Error(GPX_ERR_UNSUPPORTED_GEOMETRY,
                        head + "polygon " + std::to_string(poly) + ": non-rectilinear edge (" +
                            std::to_string(xs[i]) + "," + std::to_string(ys[i]) + ") -> (" + std::to_string(xs[k]) +
                            "," + std::to_string(ys[k]) + ")",
                        poly);
        if (ys[i] == ys[k]) h.push_back({ys[i], std::min(xs[i], xs[k]), std::max(xs[i], xs[k])});
        bx.push_back(xs[i]);
    }
    std::sort(bx.begin(), bx.end());
    bx.erase(std::unique(bx.begin(), bx.end()), bx.end());
    std::vector<int32_t> cross;
    for (size_t w = 0; w + 1 < bx.size(); ++w) {
        cross.clear();
        for (const HEdge& e : h)
            if (e.lo <= bx[w] && e.hi >= bx[w + 1]) cross.push_back(e.y);
        if (cross.size() & 1)
            throw Error(GPX_ERR_UNSUPPORTED_GEOMETRY,
                        head + "polygon " + std::to_string(poly) + ": odd crossing count " +
                            std::to_string(cross.size()) + " in slab [" + std::to_string(bx[w]) + ", " +
                            std::to_string(bx[w + 1]) + "] (self-intersecting?)",
                        poly);
        std::sort(cross.begin(), cross.end());
        for (size_t k = 0; k + 1 < cross.size(); k += 2)
            if (cross[k] < cross[k + 1]) out.push_back({bx[w], cross[k], bx[w + 1], cross[k + 1]});
    }
}

void panelize_groups(const std::vector<VolumeGroup>& groups, double xy, double me, int64_t max_panels_opt,
                     PanelizeResult& res) {
    const int64_t max_panels = max_panels_opt == 0 ? kRefMaxPanels : (max_panels_opt < 0 ? INT64_MAX : max_panels_opt);
    // cleared, not released: a result kept by the caller between calls keeps
    // its capacity (no fresh pages, no regrowth)
    res.panels.verts.clear();
    res.panels.cond.clear();
    res.panels.eps.clear();
    res.nets.clear();
    res.homogeneous = true;
    res.first_eps = 1.0;
    if (groups.empty()) return;
    std::set<uint32_t> netset;
    for (const auto& g : groups) netset.insert(g.net);
    res.nets.assign(netset.begin(), netset.end());
    auto index_of = [&](uint32_t net) {
        return (int32_t)(std::lower_bound(res.nets.begin(), res.nets.end(), net) - res.nets.begin());
    };
    Sink s{res.panels};
    double lo_x = INFINITY, lo_y = INFINITY, hi_x = -INFINITY, hi_y = -INFINITY, min_z = INFINITY, max_t = 0.0;
    for (const auto& g : groups) {
        group_to_panels(g, index_of(g.net), xy, me, s);
        res.panels.eps.resize(res.panels.cond.size(), g.k);
        if (res.panels.size() > max_panels)
            throw Error(GPX_ERR_PANEL_CAPACITY, "extruded layout needs " + std::to_string(res.panels.size()) +
                                                    " panels; limit is " + std::to_string(max_panels));
        for (const RectI& r : g.rects) {
            lo_x = std::min(lo_x, (double)r.x0 * xy);
            lo_y = std::min(lo_y, (double)r.y0 * xy);
            hi_x = std::max(hi_x, (double)r.x1 * xy);
            hi_y = std::max(hi_y, (double)r.y1 * xy);
        }
        min_z = std::min(min_z, g.z0);
        max_t = std::max(max_t, g.z1 - g.z0);
    }
    // Finite substrate reference plate (bridge.rs:346-379, cap/mesh.rs:12-43).
    const double gap = min_z > 0.0 ? min_z : std::max(max_t, 100.0 * kMetresPerNm);
    const double gz = min_z > 0.0 ? 0.0 : min_z - gap;
    const double sx = hi_x - lo_x, sy = hi_y - lo_y;
    const double pad = 0.5 * std::max(std::max(sx, sy), 8.0 * gap);
    const double lx = sx + 2.0 * pad, ly = sy + 2.0 * pad;
    double geps = 1.0, zbest = INFINITY;
    for (const auto& g : groups)
        if (g.z0 < zbest) {
            zbest = g.z0;
            geps = g.k;
        }
    // Reference rule: cells of 4 gap, 4..32 per side.  Target-edge mode: cells
    // of at most 4 max_edge and no cap, so plate panels stay small next to the
    // far-field boxes the wires' mesh size calls for.
    const double cap = me > 0.0 ? 4096.0 : 32.0;
    const double cell = me > 0.0 ? std::min(4.0 * gap, 4.0 * me) : 4.0 * gap;
    const size_t gnx = (size_t)std::min(std::max(std::ceil(lx / cell), 4.0), cap);
    const size_t gny = (size_t)std::min(std::max(std::ceil(ly / cell), 4.0), cap);
    const double cx = 0.5 * (lo_x + hi_x), cy = 0.5 * (lo_y + hi_y);
    const double x0 = cx - lx / 2.0, y0 = cy - ly / 2.0, dx = lx / (double)gnx, dy = ly / (double)gny;
    const int32_t gid = (int32_t)res.nets.size();
    for (size_t i = 0; i < gnx; ++i)
        for (size_t j = 0; j < gny; ++j) {
            double xa = x0 + (double)i * dx, xb = xa + dx, ya = y0 + (double)j * dy, yb = ya + dy;
            double v[4][3] = {{xa, ya, gz}, {xb, ya, gz}, {xb, yb, gz}, {xa, yb, gz}};
            s.quad(v, false, gid);
        }
    res.panels.eps.resize(res.panels.cond.size(), geps);
    if (res.panels.size() > max_panels)
        throw Error(GPX_ERR_PANEL_CAPACITY, "extruded layout needs " + std::to_string(res.panels.size()) +
                                                " panels; limit is " + std::to_string(max_panels));
    // Homogeneous dielectric test (bridge.rs:393-396).
    res.first_eps = res.panels.eps[0];
    res.homogeneous = true;
    for (double e : res.panels.eps)
        if (!(std::fabs(e - res.first_eps) <= std::max(std::fabs(res.first_eps), 1.0) * 1.0e-12)) {
            res.homogeneous = false;
            break;
        }
}

void panelize_store(const gpx_geometry_store& st, const gpx_deck& deck, const uint32_t* net_of_poly, int64_t n_nop,
                    double me, int64_t max_panels, PanelizeResult& res) {
    if (!std::isfinite(deck.dbu_nm) || deck.dbu_nm <= 0.0)
        throw Error(GPX_ERR_INVALID_DBU, "deck database unit must be finite and positive, got " + fmt_g(deck.dbu_nm) +
                                             " nm");
    // Process stack (analytical/process_stack.rs:31-76): layers ascending by id.
    struct Proc {
        double t, h, k;
        const gpx_layer_params* p;
    };
    std::map<uint16_t, Proc> stack;
    {
        std::vector<const gpx_layer_params*> ls;
        for (int64_t i = 0; i < deck.n_layers; ++i) ls.push_back(&deck.layers[i]);
        std::sort(ls.begin(), ls.end(), [](auto a, auto b) { return a->layer < b->layer; });
        double running = 0.0;
        for (auto p : ls) {
            double t = p->thickness_nm > 0.0 ? p->thickness_nm : 200.0;
            double h = (p->height_nm > 0.0 || p->thickness_nm > 0.0) ? p->height_nm : running;
            running = h + t + 100.0;
            stack[p->layer] = {t, h, p->dielectric_k > 0.0 ? p->dielectric_k : 3.9, p};
        }
    }
    for (auto& kv : stack) {  // validate_stack (bridge.rs:149-169)
        const struct {
            const char* f;
            double v;
            bool pos;
        } fs[3] = {{"thickness_nm", kv.second.t, true}, {"height_nm", kv.second.h, false},
                   {"dielectric_k", kv.second.k, true}};
        for (const auto& f : fs)
            if (!std::isfinite(f.v) || (f.pos && f.v <= 0.0) || (!f.pos && f.v < 0.0))
                throw Error(GPX_ERR_INVALID_PROCESS, "PEX layer " + std::to_string(kv.first) + " has invalid " + f.f +
                                                         " value " + fmt_g(f.v));
    }
    std::map<uint32_t, double> via;
    std::set<uint32_t> reported;
    std::map<std::pair<uint32_t, uint16_t>, VolumeGroup> grouped;
    std::vector<RectI> rects;
    for (int64_t poly = 0; poly < st.n_poly; ++poly) {
        auto it = stack.find(st.poly_layer[poly]);
        if (it == stack.end()) continue;
        const gpx_layer_params& p = *it->second.p;
        const uint32_t net = poly < n_nop ? net_of_poly[poly] : 0xFFFFFFFFu;
        if (p.via_res_ohm != 0.0) {
            via[net] += p.via_res_ohm;
            reported.insert(net);
        }
        if (!volume_conductor(p)) continue;
        reported.insert(net);
        rects.clear();
        decompose_ring(st.verts_x + st.poly_vert_start[poly], st.verts_y + st.poly_vert_start[poly],
                       st.poly_vert_len[poly], (uint32_t)poly, rects);
        if (rects.empty())
            throw Error(GPX_ERR_UNSUPPORTED_GEOMETRY,
                        "polygon " + std::to_string(poly) +
                            " cannot be extruded for quasi-static PEX: rectilinear decomposition produced no material",
                        (uint32_t)poly);
        auto key = std::make_pair(net, st.poly_layer[poly]);
        auto g = grouped.find(key);
        if (g == grouped.end()) {
            const Proc& pr = it->second;
            VolumeGroup vg{net, pr.h * kMetresPerNm, (pr.h + pr.t) * kMetresPerNm, pr.k, {}};
            g = grouped.emplace(key, std::move(vg)).first;
        }
        g->second.rects.insert(g->second.rects.end(), rects.begin(), rects.end());
    }
    std::vector<VolumeGroup> groups;
    groups.reserve(grouped.size());
    for (auto& kv : grouped) groups.push_back(std::move(kv.second));
    panelize_groups(groups, deck.dbu_nm * kMetresPerNm, me, max_panels, res);
    res.out_nets.assign(reported.begin(), reported.end());
    res.via_r.clear();
    for (uint32_t n : res.out_nets) res.via_r.push_back(via.count(n) ? via[n] : 0.0);
}

}  // namespace gpx
