// Closed-form Wilton integral of 1/|p - r'| over one flat panel
// (integrals/panel.rs:147-208), shared by the near-field assembly, the small
// dense solve and (on dual numbers, dual.cuh) the geometric sensitivities.
#pragma once
#include "dual.cuh"

namespace gpx {

template <class S>
struct SrcPanelT {
    S v[4][3];
    S n[3];
    S lh[4][3], uh[4][3];
    S el[4];
};
using SrcPanel = SrcPanelT<double>;

// Newell normal, unit edge tangents and in-plane edge normals of one panel.
template <class S>
__device__ __forceinline__ void prep_source_t(const S* g, SrcPanelT<S>& s) {
    using ::sqrt;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int d = 0; d < 3; ++d) s.v[i][d] = g[3 * i + d];
    S nx = 0.0, ny = 0.0, nz = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const S* c = s.v[i];
        const S* d = s.v[(i + 1) & 3];
        nx += (c[1] - d[1]) * (c[2] + d[2]);
        ny += (c[2] - d[2]) * (c[0] + d[0]);
        nz += (c[0] - d[0]) * (c[1] + d[1]);
    }
    S nn = sqrt(nx * nx + ny * ny + nz * nz);
    if (nn == 0.0) {
        s.n[0] = s.n[1] = s.n[2] = 0.0;
    } else {
        s.n[0] = nx / nn;
        s.n[1] = ny / nn;
        s.n[2] = nz / nn;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const S* a = s.v[i];
        const S* b = s.v[(i + 1) & 3];
        S e[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        S el = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        s.el[i] = el;
        S l[3] = {0.0, 0.0, 0.0};
        if (el != 0.0) {
            l[0] = e[0] / el;
            l[1] = e[1] / el;
            l[2] = e[2] / el;
        }
        s.lh[i][0] = l[0];
        s.lh[i][1] = l[1];
        s.lh[i][2] = l[2];
        s.uh[i][0] = l[1] * s.n[2] - l[2] * s.n[1];
        s.uh[i][1] = l[2] * s.n[0] - l[0] * s.n[2];
        s.uh[i][2] = l[0] * s.n[1] - l[1] * s.n[0];
    }
}

// Wilton integral of one prepared panel at point p (panel.rs:147-208).  A
// zero-length edge (the repeated vertex of a triangle) contributes nothing.
//
// The log term is evaluated in an algebraically identical, cancellation-free
// form: with r0^2 = pp^2 + d^2, num = r+ + s+ and den = r- + s- are formed as
// r0^2 / (r - s) when s < 0, and log(num/den) = log1p((num-den)/den) with
// num - den = el * (num + den) / (r+ + r-).  Where the reference's direct
// form rounds num or den to <= 0 it falls back to the asinh difference; the
// stable form needs no fallback, and a point on the edge line (r0 = 0)
// contributes 0 exactly as the reference's fallback does.
template <class S>
__device__ __forceinline__ S wilton_t(const SrcPanelT<S>& s, S px, S py, S pz) {
    using ::atan;
    using ::fabs;
    using ::log1p;
    using ::sqrt;
    const S d = (px - s.v[0][0]) * s.n[0] + (py - s.v[0][1]) * s.n[1] + (pz - s.v[0][2]) * s.n[2];
    const S p0[3] = {px - s.n[0] * d, py - s.n[1] * d, pz - s.n[2] * d};
    const S ad = fabs(d);
    S total = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (s.el[i] == 0.0) continue;
        const S* a = s.v[i];
        const S* b = s.v[(i + 1) & 3];
        const S am[3] = {a[0] - p0[0], a[1] - p0[1], a[2] - p0[2]};
        const S bm[3] = {b[0] - p0[0], b[1] - p0[1], b[2] - p0[2]};
        const S pp = am[0] * s.uh[i][0] + am[1] * s.uh[i][1] + am[2] * s.uh[i][2];
        const S sm = am[0] * s.lh[i][0] + am[1] * s.lh[i][1] + am[2] * s.lh[i][2];
        const S sp = bm[0] * s.lh[i][0] + bm[1] * s.lh[i][1] + bm[2] * s.lh[i][2];
        const S r0sq = pp * pp + d * d;
        const S rp = sqrt(sp * sp + r0sq);
        const S rm = sqrt(sm * sm + r0sq);
        const S num = sp >= 0.0 ? rp + sp : r0sq / (rp - sp);
        const S den = sm >= 0.0 ? rm + sm : r0sq / (rm - sm);
        S lt = 0.0;
        if (num > 0.0 && den > 0.0) lt = pp * log1p(s.el[i] * (num + den) / ((rp + rm) * den));
        S at = 0.0;
        if (ad > 0.0 && pp != 0.0) {
            const S tp = (pp * sp) / (r0sq + ad * rp);
            const S tm = (pp * sm) / (r0sq + ad * rm);
            at = ad * (atan(tp) - atan(tm));
        }
        total += lt - at;
    }
    return total;
}

__device__ __forceinline__ void prep_source(const double* g, SrcPanel& s) { prep_source_t<double>(g, s); }
__device__ __forceinline__ double wilton(const SrcPanel& s, double px, double py, double pz) {
    return wilton_t<double>(s, px, py, pz);
}

}  // namespace gpx
