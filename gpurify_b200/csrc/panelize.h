// Layout -> 3-D boundary-element panels (the bridge front end).
#pragma once
#include <cstdint>
#include <vector>

#include "gpx_common.h"

namespace gpx {

struct RectI {
    int32_t x0, y0, x1, y1;
};

// One extruded (net, layer) volume (bridge.rs:58-65).
struct VolumeGroup {
    uint32_t net;
    double z0, z1, k;
    std::vector<RectI> rects;
};

// Panels as one flat SoA-friendly set: 12 doubles per panel (4 vertices).
struct PanelBuffer {
    std::vector<double> verts;
    std::vector<int32_t> cond;
    std::vector<double> eps;
    int64_t size() const { return (int64_t)cond.size(); }
};

struct PanelizeResult {
    PanelBuffer panels;
    std::vector<uint32_t> nets;   // ascending; conductor i <-> nets[i]; ground = nets.size()
    std::vector<double> via_r;    // fixed via R per net, same order as `out_nets`
    std::vector<uint32_t> out_nets;  // every net the reference would report (volume or via)
    bool homogeneous = true;
    double first_eps = 1.0;
};

// Split one Manhattan polygon ring into disjoint rectangles (vertical slabs).
// Throws Error(GPX_ERR_UNSUPPORTED_GEOMETRY) with the reference's messages.
void decompose_ring(const int32_t* xs, const int32_t* ys, size_t n, uint32_t poly, std::vector<RectI>& out);

// Groups -> panels + ground plate (bridge.rs:307-386).
void panelize_groups(const std::vector<VolumeGroup>& groups, double xy_scale, double max_edge, int64_t max_panels,
                     PanelizeResult& res);

// Store + deck -> groups -> panels (bridge.rs:73-147 without the R solve).
void panelize_store(const gpx_geometry_store& store, const gpx_deck& deck, const uint32_t* net_of_poly,
                    int64_t n_nop, double max_edge, int64_t max_panels, PanelizeResult& res);

}  // namespace gpx
