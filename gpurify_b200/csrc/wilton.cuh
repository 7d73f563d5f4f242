// Closed-form Wilton integral of 1/|p - r'| over one flat panel
// (integrals/panel.rs:147-208), shared by the near-field assembly and the
// small dense solve.
#pragma once

namespace gpx {

struct SrcPanel {
    double v[4][3];
    double n[3];
    double lh[4][3], uh[4][3];
    double el[4];
};

// Newell normal, unit edge tangents and in-plane edge normals of one panel.
__device__ __forceinline__ void prep_source(const double* g, SrcPanel& s) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int d = 0; d < 3; ++d) s.v[i][d] = g[3 * i + d];
    double nx = 0.0, ny = 0.0, nz = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double* c = s.v[i];
        const double* d = s.v[(i + 1) & 3];
        nx += (c[1] - d[1]) * (c[2] + d[2]);
        ny += (c[2] - d[2]) * (c[0] + d[0]);
        nz += (c[0] - d[0]) * (c[1] + d[1]);
    }
    double nn = sqrt(nx * nx + ny * ny + nz * nz);
    if (nn == 0.0) {
        s.n[0] = s.n[1] = s.n[2] = 0.0;
    } else {
        s.n[0] = nx / nn;
        s.n[1] = ny / nn;
        s.n[2] = nz / nn;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double* a = s.v[i];
        const double* b = s.v[(i + 1) & 3];
        double e[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        double el = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        s.el[i] = el;
        double l[3] = {0.0, 0.0, 0.0};
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
__device__ __forceinline__ double wilton(const SrcPanel& s, double px, double py, double pz) {
    const double d = (px - s.v[0][0]) * s.n[0] + (py - s.v[0][1]) * s.n[1] + (pz - s.v[0][2]) * s.n[2];
    const double p0[3] = {px - s.n[0] * d, py - s.n[1] * d, pz - s.n[2] * d};
    const double ad = fabs(d);
    double total = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (s.el[i] == 0.0) continue;
        const double* a = s.v[i];
        const double* b = s.v[(i + 1) & 3];
        const double am[3] = {a[0] - p0[0], a[1] - p0[1], a[2] - p0[2]};
        const double bm[3] = {b[0] - p0[0], b[1] - p0[1], b[2] - p0[2]};
        const double pp = am[0] * s.uh[i][0] + am[1] * s.uh[i][1] + am[2] * s.uh[i][2];
        const double sm = am[0] * s.lh[i][0] + am[1] * s.lh[i][1] + am[2] * s.lh[i][2];
        const double sp = bm[0] * s.lh[i][0] + bm[1] * s.lh[i][1] + bm[2] * s.lh[i][2];
        const double r0sq = pp * pp + d * d;
        const double rp = sqrt(sp * sp + r0sq);
        const double rm = sqrt(sm * sm + r0sq);
        const double num = sp >= 0.0 ? rp + sp : r0sq / (rp - sp);
        const double den = sm >= 0.0 ? rm + sm : r0sq / (rm - sm);
        double lt = 0.0;
        if (num > 0.0 && den > 0.0) lt = pp * log1p(s.el[i] * (num + den) / ((rp + rm) * den));
        double at = 0.0;
        if (ad > 0.0 && pp != 0.0) {
            const double tp = (pp * sp) / (r0sq + ad * rp);
            const double tm = (pp * sm) / (r0sq + ad * rm);
            at = ad * (atan(tp) - atan(tm));
        }
        total += lt - at;
    }
    return total;
}

}  // namespace gpx
