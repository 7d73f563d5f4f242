// CPU oracle for the field-solver capacitance path — TEST INFRASTRUCTURE ONLY.
// A plain restatement of the reference's CPU algorithm; each function cites the
// reference file:line it follows.  Compiled with -ffp-contract=off so that, like
// the reference's Rust code, no multiply-add is fused.
#include "orc.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- constants
// quasistatic/constants.rs:13,20
const double kPi = 3.14159265358979323846;
const double EPS0 = 8.854187812800e-12;
const double ONE_OVER_4PI_EPS0 = 1.0 / (4.0 * kPi * EPS0);

// ---------------------------------------------------------------- Vec3
// quasistatic/geometry.rs:12-107
struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalized(V3 a) {
    double n = norm(a);
    if (n == 0.0) return {0.0, 0.0, 0.0};
    return a / n;
}

struct Quad {
    V3 v[4];
};
inline Quad load_quad(const double* p) {
    Quad q;
    for (int i = 0; i < 4; ++i) q.v[i] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
    return q;
}

// Number of distinct vertices: a triangle is stored with v3 == v2.
inline int quad_nv(const Quad& q) {
    return (q.v[3].x == q.v[2].x && q.v[3].y == q.v[2].y && q.v[3].z == q.v[2].z) ? 3 : 4;
}

// integrals/panel.rs:29-47 (fan-triangulated, area-weighted centroid)
V3 centroid(const Quad& q) {
    int nv = quad_nv(q);
    V3 v0 = q.v[0];
    double area_sum = 0.0;
    V3 c{0.0, 0.0, 0.0};
    for (int i = 1; i < nv - 1; ++i) {
        V3 v1 = q.v[i], v2 = q.v[i + 1];
        double a = norm(cross(v1 - v0, v2 - v0)) * 0.5;
        V3 tri_c = (v0 + v1 + v2) * (1.0 / 3.0);
        c = c + tri_c * a;
        area_sum += a;
    }
    if (area_sum == 0.0) return v0;
    return c * (1.0 / area_sum);
}

// integrals/panel.rs:58-67
double area(const Quad& q) {
    int nv = quad_nv(q);
    V3 v0 = q.v[0];
    double a = 0.0;
    for (int i = 1; i < nv - 1; ++i) {
        V3 v1 = q.v[i], v2 = q.v[i + 1];
        a += norm(cross(v1 - v0, v2 - v0)) * 0.5;
    }
    return a;
}

// integrals/panel.rs:256-269 (Newell normal)
V3 polygon_normal(const Quad& q, int nv) {
    double nx = 0.0, ny = 0.0, nz = 0.0;
    for (int i = 0; i < nv; ++i) {
        V3 c = q.v[i], d = q.v[(i + 1) % nv];
        nx += (c.y - d.y) * (c.z + d.z);
        ny += (c.z - d.z) * (c.x + d.x);
        nz += (c.x - d.x) * (c.y + d.y);
    }
    return normalized(V3{nx, ny, nz});
}

// integrals/panel.rs:272-286
inline double asinh_over(double s, double r0_sq) {
    double r0 = std::sqrt(r0_sq);
    if (r0 == 0.0) return 0.0;
    return std::asinh(s / r0);
}

// integrals/panel.rs:147-208 — closed-form Wilton integral of 1/|p - r'| over
// the flat polygon.
double potential_integral(const Quad& q, V3 p) {
    int nv = quad_nv(q);
    V3 n = polygon_normal(q, nv);
    V3 v0 = q.v[0];
    double d = dot(p - v0, n);
    V3 p0 = p - n * d;
    double absd = std::fabs(d);
    double total = 0.0;
    for (int i = 0; i < nv; ++i) {
        V3 a = q.v[i], b = q.v[(i + 1) % nv];
        V3 edge = b - a;
        double edge_len = norm(edge);
        if (edge_len == 0.0) continue;
        V3 lhat = edge / edge_len;
        V3 uhat = cross(lhat, n);
        double p0_perp = dot(a - p0, uhat);
        double s_minus = dot(a - p0, lhat);
        double s_plus = dot(b - p0, lhat);
        double r0_sq = p0_perp * p0_perp + d * d;
        double r_plus = std::sqrt(s_plus * s_plus + r0_sq);
        double r_minus = std::sqrt(s_minus * s_minus + r0_sq);
        double num = r_plus + s_plus;
        double den = r_minus + s_minus;
        double log_term;
        if (num > 0.0 && den > 0.0) {
            log_term = p0_perp * std::log(num / den);
        } else if (std::fabs(den) > 0.0) {
            log_term = p0_perp * (asinh_over(s_plus, r0_sq) - asinh_over(s_minus, r0_sq));
        } else {
            log_term = 0.0;
        }
        double atan_term = 0.0;
        if (absd > 0.0 && p0_perp != 0.0) {
            double t_plus = (p0_perp * s_plus) / (r0_sq + absd * r_plus);
            double t_minus = (p0_perp * s_minus) / (r0_sq + absd * r_minus);
            atan_term = absd * (std::atan(t_plus) - std::atan(t_minus));
        }
        total += log_term - atan_term;
    }
    return total;
}

// ---------------------------------------------------------------- PanelSet
// integrals/panel.rs:78-118
struct PanelSet {
    std::vector<double> cx, cy, cz, ar;
    std::vector<int32_t> cond;
    std::vector<Quad> quads;
    size_t size() const { return ar.size(); }
    V3 c(size_t i) const { return {cx[i], cy[i], cz[i]}; }
};
PanelSet build_set(int64_t n, const double* verts, const int32_t* cond) {
    PanelSet s;
    s.cx.resize(n);
    s.cy.resize(n);
    s.cz.resize(n);
    s.ar.resize(n);
    s.cond.assign(n, 0);
    s.quads.resize(n);
    for (int64_t i = 0; i < n; ++i) {
        Quad q = load_quad(verts + 12 * i);
        V3 c = centroid(q);
        s.cx[i] = c.x;
        s.cy[i] = c.y;
        s.cz[i] = c.z;
        s.ar[i] = area(q);
        if (cond) s.cond[i] = cond[i];
        s.quads[i] = q;
    }
    return s;
}

// ---------------------------------------------------------------- BLAS-1
// simd.rs:20-45: 4 vector accumulators x 4 lanes over 16-blocks, then 4-blocks
// into accumulator 0, horizontal reduce, scalar tail.
double dot16(const double* a, const double* b, size_t n) {
    double acc[4][4] = {{0}};
    size_t n16 = n & ~size_t(15), j = 0;
    for (; j < n16; j += 16)
        for (int v = 0; v < 4; ++v)
            for (int l = 0; l < 4; ++l) acc[v][l] = a[j + 4 * v + l] * b[j + 4 * v + l] + acc[v][l];
    size_t n4 = n & ~size_t(3);
    for (; j < n4; j += 4)
        for (int l = 0; l < 4; ++l) acc[0][l] = a[j + l] * b[j + l] + acc[0][l];
    double lane[4];
    for (int l = 0; l < 4; ++l) lane[l] = (acc[0][l] + acc[1][l]) + (acc[2][l] + acc[3][l]);
    double s = ((lane[0] + lane[1]) + lane[2]) + lane[3];
    for (; j < n; ++j) s += a[j] * b[j];
    return s;
}
inline double nrm2(const double* a, size_t n) { return std::sqrt(dot16(a, a, n)); }
// simd.rs:55-70
void axpy(double alpha, const double* x, double* y, size_t n) {
    for (size_t j = 0; j < n; ++j) y[j] = alpha * x[j] + y[j];
}

// ---------------------------------------------------------------- operators
struct Op {
    virtual ~Op() {}
    virtual size_t dim() const = 0;
    virtual void apply(const double* x, double* y) const = 0;
};

// krylov.rs:14-41
struct GmresOpts {
    double tol;
    size_t restart, max_restarts;
};
struct GmresResult {
    std::vector<double> x;
    size_t iterations;
    double residual;
    bool converged;
};

// krylov.rs:195-207
inline void givens(double a, double b, double& c, double& s) {
    if (b == 0.0) {
        c = 1.0;
        s = 0.0;
    } else if (std::fabs(b) > std::fabs(a)) {
        double t = a / b;
        s = 1.0 / std::sqrt(1.0 + t * t);
        c = t * s;
    } else {
        double t = b / a;
        c = 1.0 / std::sqrt(1.0 + t * t);
        s = t * c;
    }
}

// krylov.rs:50-191 — restarted right-preconditioned GMRES(m), MGS.
GmresResult gmres(const Op& a, const double* b, const Op* precond, GmresOpts opts) {
    size_t n = a.dim();
    double bnorm = std::max(nrm2(b, n), 2.2250738585072014e-308);
    std::vector<double> x(n, 0.0), z(n, 0.0), ax(n, 0.0);
    size_t total_iters = 0;
    for (size_t cycle = 0; cycle < opts.max_restarts; ++cycle) {
        a.apply(x.data(), ax.data());
        std::vector<double> r(n);
        for (size_t i = 0; i < n; ++i) r[i] = b[i] - ax[i];
        double beta = nrm2(r.data(), n);
        if (beta / bnorm <= opts.tol) return {x, total_iters, beta / bnorm, true};
        size_t m = opts.restart;
        std::vector<std::vector<double>> v;
        v.reserve(m + 1);
        for (auto& vi : r) vi /= beta;
        v.push_back(std::move(r));
        std::vector<std::vector<double>> h(m + 1, std::vector<double>(m, 0.0));
        std::vector<double> cs(m, 0.0), sn(m, 0.0), g(m + 1, 0.0);
        g[0] = beta;
        size_t k_used = 0;
        for (size_t k = 0; k < m; ++k) {
            const double* zk = v[k].data();
            if (precond) {
                precond->apply(v[k].data(), z.data());
                zk = z.data();
            }
            std::vector<double> w(n, 0.0);
            a.apply(zk, w.data());
            for (size_t i = 0; i <= k; ++i) {
                h[i][k] = dot16(w.data(), v[i].data(), n);
                axpy(-h[i][k], v[i].data(), w.data(), n);
            }
            h[k + 1][k] = nrm2(w.data(), n);
            if (h[k + 1][k] > 1e-14)
                for (auto& wj : w) wj /= h[k + 1][k];
            v.push_back(std::move(w));
            for (size_t i = 0; i < k; ++i) {
                double temp = cs[i] * h[i][k] + sn[i] * h[i + 1][k];
                h[i + 1][k] = -sn[i] * h[i][k] + cs[i] * h[i + 1][k];
                h[i][k] = temp;
            }
            double c, s;
            givens(h[k][k], h[k + 1][k], c, s);
            cs[k] = c;
            sn[k] = s;
            h[k][k] = c * h[k][k] + s * h[k + 1][k];
            h[k + 1][k] = 0.0;
            double temp = c * g[k] + s * g[k + 1];
            g[k + 1] = -s * g[k] + c * g[k + 1];
            g[k] = temp;
            total_iters += 1;
            k_used = k + 1;
            if (std::fabs(g[k + 1]) / bnorm <= opts.tol) break;
        }
        std::vector<double> y(k_used, 0.0);
        for (size_t ii = k_used; ii-- > 0;) {
            double sum = g[ii];
            for (size_t j = ii + 1; j < k_used; ++j) sum -= h[ii][j] * y[j];
            y[ii] = sum / h[ii][ii];
        }
        std::vector<double> dx(n, 0.0);
        for (size_t i = 0; i < k_used; ++i)
            for (size_t j = 0; j < n; ++j) dx[j] += y[i] * v[i][j];
        const double* dz = dx.data();
        if (precond) {
            precond->apply(dx.data(), z.data());
            dz = z.data();
        }
        for (size_t j = 0; j < n; ++j) x[j] += dz[j];
        double est = std::fabs(g[k_used]) / bnorm;
        if (est <= opts.tol * 10.0) {
            a.apply(x.data(), ax.data());
            std::vector<double> r2(n);
            for (size_t i = 0; i < n; ++i) r2[i] = b[i] - ax[i];
            double resid = nrm2(r2.data(), n) / bnorm;
            if (resid <= opts.tol) return {x, total_iters, resid, true};
        }
    }
    a.apply(x.data(), ax.data());
    std::vector<double> r(n);
    for (size_t i = 0; i < n; ++i) r[i] = b[i] - ax[i];
    return {x, total_iters, nrm2(r.data(), n) / bnorm, false};
}

// ---------------------------------------------------------------- dense LA
// linalg.rs:170-259 — LU with partial pivoting.
struct LU {
    std::vector<double> lu;
    std::vector<size_t> piv;
    size_t n;
    bool ok;
};
LU lu_factor(const std::vector<double>& a, size_t n) {
    LU f{a, {}, n, true};
    f.piv.resize(n);
    for (size_t i = 0; i < n; ++i) f.piv[i] = i;
    std::vector<double>& lu = f.lu;
    for (size_t k = 0; k < n; ++k) {
        size_t p = k;
        double mx = std::fabs(lu[k * n + k]);
        for (size_t i = k + 1; i < n; ++i) {
            double m = std::fabs(lu[i * n + k]);
            if (m > mx) {
                mx = m;
                p = i;
            }
        }
        if (mx == 0.0) {
            f.ok = false;
            return f;
        }
        if (p != k) {
            for (size_t j = 0; j < n; ++j) std::swap(lu[k * n + j], lu[p * n + j]);
            std::swap(f.piv[k], f.piv[p]);
        }
        double pivot = lu[k * n + k];
#pragma omp parallel for schedule(static) if ((n - k) * (n - k) > 4096)
        for (long long i = (long long)k + 1; i < (long long)n; ++i) {
            double* row = &lu[i * n];
            const double* prow = &lu[k * n];
            double factor = row[k] / pivot;
            row[k] = factor;
            for (size_t j = k + 1; j < n; ++j) row[j] = row[j] - factor * prow[j];
        }
    }
    return f;
}
std::vector<double> lu_solve(const LU& f, const std::vector<double>& b) {
    size_t n = f.n;
    std::vector<double> x(n);
    for (size_t i = 0; i < n; ++i) x[i] = b[f.piv[i]];
    for (size_t i = 0; i < n; ++i) {
        double sum = x[i];
        for (size_t j = 0; j < i; ++j) sum = sum - f.lu[i * n + j] * x[j];
        x[i] = sum;
    }
    for (size_t i = n; i-- > 0;) {
        double sum = x[i];
        for (size_t j = i + 1; j < n; ++j) sum = sum - f.lu[i * n + j] * x[j];
        x[i] = sum / f.lu[i * n + i];
    }
    return x;
}

// compiler-rt __powidf2 (what Rust's f64::powi lowers to).
double powi(double a, int b) {
    bool recip = b < 0;
    double r = 1.0;
    for (;;) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? 1.0 / r : r;
}

// linalg.rs:264-400 — column-pivoted MGS QR truncated low-rank approximation.
struct LowRank {
    std::vector<double> u, vt;
    size_t m = 0, n = 0, k = 0;
};
LowRank compress(const std::vector<double>& a, size_t m, size_t n, double eps) {
    std::vector<double> q(a.begin(), a.begin() + m * n), r(n * n, 0.0);
    std::vector<size_t> perm(n);
    for (size_t j = 0; j < n; ++j) perm[j] = j;
    std::vector<double> col(n);
    for (size_t j = 0; j < n; ++j) {
        double s = -0.0;
        for (size_t i = 0; i < m; ++i) s += a[i * n + j] * a[i * n + j];
        col[j] = s;
    }
    size_t max_k = std::min(m, n), k = 0;
    double mx = 0.0;
    for (double c : col) mx = std::fmax(mx, c);
    double thr = eps * mx;
    for (size_t step = 0; step < max_k; ++step) {
        size_t best = step;
        for (size_t j = step + 1; j < n; ++j)
            if (col[j] > col[best]) best = j;
        if (col[best] < thr) break;
        if (best != step) {
            std::swap(perm[step], perm[best]);
            std::swap(col[step], col[best]);
            for (size_t i = 0; i < m; ++i) std::swap(q[i * n + step], q[i * n + best]);
            for (size_t row = 0; row < step; ++row) std::swap(r[row * n + step], r[row * n + best]);
        }
        double nrm = 0.0;
        for (size_t i = 0; i < m; ++i) nrm += q[i * n + step] * q[i * n + step];
        nrm = std::sqrt(nrm);
        if (nrm < 1e-15) break;
        r[step * n + step] = nrm;
        double inv = 1.0 / nrm;
        for (size_t i = 0; i < m; ++i) q[i * n + step] *= inv;
        for (size_t j = step + 1; j < n; ++j) {
            double d = 0.0;
            for (size_t i = 0; i < m; ++i) d += q[i * n + step] * q[i * n + j];
            r[step * n + j] = d;
            for (size_t i = 0; i < m; ++i) q[i * n + j] -= d * q[i * n + step];
            col[j] -= d * d;
            if (col[j] < 0.0) col[j] = 0.0;
        }
        k = step + 1;
    }
    LowRank lr;
    lr.m = m;
    lr.n = n;
    lr.k = k;
    if (k == 0) return lr;
    lr.u.assign(m * k, 0.0);
    for (size_t i = 0; i < m; ++i)
        for (size_t j = 0; j < k; ++j) lr.u[i * k + j] = q[i * n + j];
    lr.vt.assign(k * n, 0.0);
    for (size_t i = 0; i < k; ++i)
        for (size_t j = 0; j < n; ++j) lr.vt[i * n + perm[j]] = r[i * n + j];
    return lr;
}
// linalg.rs:386-400
void lr_apply_add(const LowRank& lr, const double* x, double* y, double scale, double* t) {
    if (lr.k == 0) return;
    for (size_t i = 0; i < lr.k; ++i) {
        double s = -0.0;
        for (size_t l = 0; l < lr.n; ++l) s += lr.vt[i * lr.n + l] * x[l];
        t[i] = s;
    }
    for (size_t i = 0; i < lr.m; ++i) {
        double s = -0.0;
        for (size_t j = 0; j < lr.k; ++j) s += lr.u[i * lr.k + j] * t[j];
        y[i] += scale * s;
    }
}

// ---------------------------------------------------------------- Chebyshev
// fmm/chebyshev.rs:11-18
std::vector<double> cheb_nodes(int n) {
    std::vector<double> v(n);
    for (int m = 0; m < n; ++m) v[m] = std::cos((2.0 * m + 1.0) * kPi / (2.0 * n));
    return v;
}
// fmm/chebyshev.rs:41-74
void interp_weights(double x, int n, const std::vector<double>& nodes, double* out) {
    std::vector<double> tx(n, 0.0);
    tx[0] = 1.0;
    if (n > 1) {
        tx[1] = x;
        for (int k = 2; k < n; ++k) tx[k] = 2.0 * x * tx[k - 1] - tx[k - 2];
    }
    double inv_n = 1.0 / n;
    for (int m = 0; m < n; ++m) {
        double xm = nodes[m], sum = 0.5, tkm1 = 1.0, tk = xm;
        for (int k = 1; k < n; ++k) {
            double tkm;
            if (k == 1) {
                tkm = xm;
            } else {
                double t = 2.0 * xm * tk - tkm1;
                tkm1 = tk;
                tk = t;
                tkm = t;
            }
            sum += tkm * tx[k];
        }
        out[m] = 2.0 * inv_n * sum;
    }
}
// fmm/chebyshev.rs:78-93
void interp_weights_3d(const double p[3], int n, const std::vector<double>& nodes, double* w) {
    std::vector<double> w1(n), w2(n), w3(n);
    interp_weights(p[0], n, nodes, w1.data());
    interp_weights(p[1], n, nodes, w2.data());
    interp_weights(p[2], n, nodes, w3.data());
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) {
            double wab = w1[a] * w2[b];
            int base = (a * n + b) * n;
            for (int c = 0; c < n; ++c) w[base + c] = wab * w3[c];
        }
}

// ---------------------------------------------------------------- Octree
// fmm/tree.rs:11-37
struct Node {
    int level;
    uint32_t cell[3];
    double center[3];
    double half;
    long parent;
    std::vector<size_t> children, points, neighbors, interaction;
};
struct CellKey {
    uint32_t c[3];
    bool operator==(const CellKey& o) const { return c[0] == o.c[0] && c[1] == o.c[1] && c[2] == o.c[2]; }
};
struct CellHash {
    size_t operator()(const CellKey& k) const {
        return (size_t(k.c[0]) * 73856093u) ^ (size_t(k.c[1]) * 19349663u) ^ (size_t(k.c[2]) * 83492791u);
    }
};
struct Octree {
    std::vector<Node> nodes;
    int max_level;
    std::vector<std::vector<size_t>> levels;
    const std::vector<size_t>& leaves() const { return levels[max_level]; }
};

// fmm/tree.rs:109-151
size_t ensure_box(std::vector<Node>& nodes, std::vector<std::unordered_map<CellKey, size_t, CellHash>>& maps,
                  int level, const uint32_t cell[3], const double rc[3], double rh) {
    CellKey key{{cell[0], cell[1], cell[2]}};
    auto it = maps[level].find(key);
    if (it != maps[level].end()) return it->second;
    long parent = -1;
    if (level > 0) {
        uint32_t pc[3] = {cell[0] / 2, cell[1] / 2, cell[2] / 2};
        parent = (long)ensure_box(nodes, maps, level - 1, pc, rc, rh);
    }
    double half = rh / double(1u << level);
    double origin[3] = {rc[0] - rh, rc[1] - rh, rc[2] - rh};
    Node nd;
    nd.level = level;
    for (int d = 0; d < 3; ++d) {
        nd.cell[d] = cell[d];
        nd.center[d] = origin[d] + (double(cell[d]) + 0.5) * 2.0 * half;
    }
    nd.half = half;
    nd.parent = parent;
    size_t id = nodes.size();
    nodes.push_back(std::move(nd));
    maps[level][key] = id;
    if (parent >= 0) nodes[parent].children.push_back(id);
    return id;
}

// fmm/tree.rs:41-106 and :154-210
Octree build_tree(const std::vector<V3>& pts, int max_level) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (const V3& p : pts) {
        double a[3] = {p.x, p.y, p.z};
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::fmin(lo[d], a[d]);
            hi[d] = std::fmax(hi[d], a[d]);
        }
    }
    double half = 0.0, center[3];
    for (int d = 0; d < 3; ++d) {
        center[d] = 0.5 * (lo[d] + hi[d]);
        half = std::fmax(half, 0.5 * (hi[d] - lo[d]));
    }
    half *= 1.0 + 1e-6;
    if (half == 0.0) half = 1.0;
    Octree t;
    t.max_level = max_level;
    std::vector<std::unordered_map<CellKey, size_t, CellHash>> maps(max_level + 1);
    {
        Node root;
        root.level = 0;
        root.cell[0] = root.cell[1] = root.cell[2] = 0;
        for (int d = 0; d < 3; ++d) root.center[d] = center[d];
        root.half = half;
        root.parent = -1;
        t.nodes.push_back(root);
        maps[0][CellKey{{0, 0, 0}}] = 0;
    }
    uint32_t ncell = 1u << max_level;
    double leaf_size = 2.0 * half / double(ncell);
    double origin[3] = {center[0] - half, center[1] - half, center[2] - half};
    for (size_t pi = 0; pi < pts.size(); ++pi) {
        double a[3] = {pts[pi].x, pts[pi].y, pts[pi].z};
        uint32_t cell[3];
        for (int d = 0; d < 3; ++d) {
            long long idx = (long long)std::floor((a[d] - origin[d]) / leaf_size);
            if (idx < 0) idx = 0;
            if (idx > (long long)ncell - 1) idx = ncell - 1;
            cell[d] = (uint32_t)idx;
        }
        size_t leaf = ensure_box(t.nodes, maps, max_level, cell, center, half);
        t.nodes[leaf].points.push_back(pi);
    }
    t.levels.assign(max_level + 1, {});
    for (size_t id = 0; id < t.nodes.size(); ++id) t.levels[t.nodes[id].level].push_back(id);
    // neighbours
    for (size_t id = 0; id < t.nodes.size(); ++id) {
        int level = t.nodes[id].level;
        long long nc = 1ll << level;
        std::vector<size_t> nb;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    if (dx == 0 && dy == 0 && dz == 0) continue;
                    long long c[3] = {(long long)t.nodes[id].cell[0] + dx, (long long)t.nodes[id].cell[1] + dy,
                                      (long long)t.nodes[id].cell[2] + dz};
                    bool out = false;
                    for (int d = 0; d < 3; ++d) out |= (c[d] < 0 || c[d] >= nc);
                    if (out) continue;
                    auto it = maps[level].find(CellKey{{(uint32_t)c[0], (uint32_t)c[1], (uint32_t)c[2]}});
                    if (it != maps[level].end()) nb.push_back(it->second);
                }
        t.nodes[id].neighbors = nb;
    }
    // interaction lists
    for (size_t id = 0; id < t.nodes.size(); ++id) {
        if (t.nodes[id].level < 2) continue;
        size_t parent = (size_t)t.nodes[id].parent;
        std::set<size_t> own(t.nodes[id].neighbors.begin(), t.nodes[id].neighbors.end());
        std::vector<size_t> fam = t.nodes[parent].neighbors;
        fam.push_back(parent);
        std::vector<size_t> inter;
        for (size_t pn : fam)
            for (size_t ch : t.nodes[pn].children)
                if (ch != id && !own.count(ch)) inter.push_back(ch);
        t.nodes[id].interaction = inter;
    }
    return t;
}

// ---------------------------------------------------------------- bbFMM
inline int m2l_index(int ox, int oy, int oz) { return ((ox + 3) * 7 + oy + 3) * 7 + oz + 3; }

// fmm/bbfmm.rs:132-174 (operator for one offset, reference coordinates)
LowRank build_m2l(const std::vector<std::array<double, 3>>& ref3d, int n, int ox, int oy, int oz) {
    size_t n3 = ref3d.size();
    double eps = std::fmax(1e-3 * powi(0.1, n), 1e-14);
    std::vector<double> g(n3 * n3, 0.0);
    double shift[3] = {2.0 * ox, 2.0 * oy, 2.0 * oz};
    for (size_t m = 0; m < n3; ++m)
        for (size_t l = 0; l < n3; ++l) {
            double dx = ref3d[m][0] - ref3d[l][0] - shift[0];
            double dy = ref3d[m][1] - ref3d[l][1] - shift[1];
            double dz = ref3d[m][2] - ref3d[l][2] - shift[2];
            double r = std::sqrt(dx * dx + dy * dy + dz * dz);
            g[m * n3 + l] = r > 0.0 ? 1.0 / r : 0.0;
        }
    return compress(g, n3, n3, eps);
}

struct Fmm {
    Octree tree;
    int n;
    size_t n3;
    std::vector<std::array<double, 3>> ref3d;
    std::vector<V3> points;
    std::vector<std::vector<double>> pw;  // per point n^3 weights
    std::vector<std::vector<double>> m2m_1d;
    std::vector<LowRank> table;
    std::vector<bool> has;

    // fmm/bbfmm.rs:46-128
    Fmm(const std::vector<V3>& pts, int order, int max_level) : n(order) {
        tree = build_tree(pts, max_level);
        std::vector<double> nodes1d = cheb_nodes(n);
        n3 = size_t(n) * n * n;
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b)
                for (int c = 0; c < n; ++c) ref3d.push_back({nodes1d[a], nodes1d[b], nodes1d[c]});
        points = pts;
        pw.assign(pts.size(), {});
        for (size_t leaf : tree.leaves()) {
            const Node& nd = tree.nodes[leaf];
            for (size_t pi : nd.points) {
                double loc[3] = {(pts[pi].x - nd.center[0]) / nd.half, (pts[pi].y - nd.center[1]) / nd.half,
                                 (pts[pi].z - nd.center[2]) / nd.half};
                pw[pi].resize(n3);
                interp_weights_3d(loc, n, nodes1d, pw[pi].data());
            }
        }
        m2m_1d.assign(24, std::vector<double>(size_t(n) * n, 0.0));
        std::vector<double> w(n);
        for (int oz = 0; oz < 2; ++oz)
            for (int oy = 0; oy < 2; ++oy)
                for (int ox = 0; ox < 2; ++ox) {
                    int o = ox + 2 * oy + 4 * oz;
                    double cc[3] = {(2.0 * ox - 1.0) * 0.5, (2.0 * oy - 1.0) * 0.5, (2.0 * oz - 1.0) * 0.5};
                    for (int axis = 0; axis < 3; ++axis) {
                        auto& mat = m2m_1d[o * 3 + axis];
                        for (int k = 0; k < n; ++k) {
                            double child = cc[axis] + 0.5 * nodes1d[k];
                            interp_weights(child, n, nodes1d, w.data());
                            for (int m = 0; m < n; ++m) mat[m * n + k] = w[m];
                        }
                    }
                }
        // precompute_m2l over the offsets that occur
        table.assign(343, LowRank());
        has.assign(343, false);
        std::vector<int> offs;
        for (const Node& nd : tree.nodes)
            for (size_t c : nd.interaction) {
                const Node& cn = tree.nodes[c];
                int idx = m2l_index((int)cn.cell[0] - (int)nd.cell[0], (int)cn.cell[1] - (int)nd.cell[1],
                                    (int)cn.cell[2] - (int)nd.cell[2]);
                if (!has[idx]) {
                    has[idx] = true;
                    offs.push_back(idx);
                }
            }
#pragma omp parallel for schedule(dynamic)
        for (long i = 0; i < (long)offs.size(); ++i) {
            int idx = offs[i];
            int ox = idx / 49 - 3, oy = (idx / 7) % 7 - 3, oz = idx % 7 - 3;
            table[idx] = build_m2l(ref3d, n, ox, oy, oz);
        }
    }

    int octant(size_t child, size_t parent) const {
        const Node& c = tree.nodes[child];
        const Node& p = tree.nodes[parent];
        return int(c.cell[0] - 2 * p.cell[0]) + 2 * int(c.cell[1] - 2 * p.cell[1]) + 4 * int(c.cell[2] - 2 * p.cell[2]);
    }

    // fmm/bbfmm.rs:209-448
    std::vector<double> run(const double* q, bool with_p2p) const {
        size_t nb = tree.nodes.size();
        std::vector<std::vector<double>> w(nb, std::vector<double>(n3, 0.0)), loc(nb, std::vector<double>(n3, 0.0));
        for (size_t leaf : tree.leaves()) {
            auto& wl = w[leaf];
            for (size_t pi : tree.nodes[leaf].points) {
                double qi = q[pi];
                if (qi == 0.0) continue;
                const auto& p = pw[pi];
                for (size_t m = 0; m < n3; ++m) wl[m] += p[m] * qi;
            }
        }
        std::vector<double> t1(n3), t2(n3);
        for (int level = tree.max_level; level >= 1; --level)
            for (size_t id : tree.levels[level]) {
                long parent = tree.nodes[id].parent;
                if (parent < 0) continue;
                int o = octant(id, (size_t)parent);
                const auto& mx = m2m_1d[o * 3];
                const auto& my = m2m_1d[o * 3 + 1];
                const auto& mz = m2m_1d[o * 3 + 2];
                const auto& wc = w[id];
                auto& wp = w[parent];
                for (int a = 0; a < n; ++a)
                    for (int b = 0; b < n; ++b)
                        for (int cp = 0; cp < n; ++cp) {
                            double s = 0.0;
                            for (int c = 0; c < n; ++c) s += mz[cp * n + c] * wc[a * n * n + b * n + c];
                            t1[a * n * n + b * n + cp] = s;
                        }
                for (int a = 0; a < n; ++a)
                    for (int bp = 0; bp < n; ++bp)
                        for (int cp = 0; cp < n; ++cp) {
                            double s = 0.0;
                            for (int b = 0; b < n; ++b) s += my[bp * n + b] * t1[a * n * n + b * n + cp];
                            t2[a * n * n + bp * n + cp] = s;
                        }
                for (int ap = 0; ap < n; ++ap)
                    for (int bp = 0; bp < n; ++bp)
                        for (int cp = 0; cp < n; ++cp) {
                            double s = 0.0;
                            for (int a = 0; a < n; ++a) s += mx[ap * n + a] * t2[a * n * n + bp * n + cp];
                            wp[ap * n * n + bp * n + cp] += s;
                        }
            }
        for (int level = 2; level <= tree.max_level; ++level) {
            const auto& ids = tree.levels[level];
            if (ids.empty()) continue;
            double inv_half = 1.0 / tree.nodes[ids[0]].half;
#pragma omp parallel for schedule(dynamic, 16)
            for (long ii = 0; ii < (long)ids.size(); ++ii) {
                size_t id = ids[ii];
                const Node& nd = tree.nodes[id];
                std::vector<double> acc(n3, 0.0), scratch(n3, 0.0);
                for (size_t c : nd.interaction) {
                    const Node& cn = tree.nodes[c];
                    int idx = m2l_index((int)cn.cell[0] - (int)nd.cell[0], (int)cn.cell[1] - (int)nd.cell[1],
                                        (int)cn.cell[2] - (int)nd.cell[2]);
                    if (has[idx]) lr_apply_add(table[idx], w[c].data(), acc.data(), inv_half, scratch.data());
                }
                for (size_t m = 0; m < n3; ++m) loc[id][m] += acc[m];
            }
        }
        for (int level = 2; level < tree.max_level; ++level)
            for (size_t id : tree.levels[level])
                for (size_t child : tree.nodes[id].children) {
                    int o = octant(child, id);
                    const auto& mx = m2m_1d[o * 3];
                    const auto& my = m2m_1d[o * 3 + 1];
                    const auto& mz = m2m_1d[o * 3 + 2];
                    const auto& lp = loc[id];
                    auto& lc = loc[child];
                    for (int ap = 0; ap < n; ++ap)
                        for (int b = 0; b < n; ++b)
                            for (int c = 0; c < n; ++c) {
                                double s = 0.0;
                                for (int a = 0; a < n; ++a) s += mx[a * n + ap] * lp[a * n * n + b * n + c];
                                t1[ap * n * n + b * n + c] = s;
                            }
                    for (int a = 0; a < n; ++a)
                        for (int bp = 0; bp < n; ++bp)
                            for (int c = 0; c < n; ++c) {
                                double s = 0.0;
                                for (int b = 0; b < n; ++b) s += my[b * n + bp] * t1[a * n * n + b * n + c];
                                t2[a * n * n + bp * n + c] = s;
                            }
                    for (int a = 0; a < n; ++a)
                        for (int b = 0; b < n; ++b)
                            for (int cp = 0; cp < n; ++cp) {
                                double s = 0.0;
                                for (int c = 0; c < n; ++c) s += mz[c * n + cp] * t2[a * n * n + b * n + c];
                                lc[a * n * n + b * n + cp] += s;
                            }
                }
        std::vector<double> y(points.size(), 0.0);
        const auto& leaves = tree.leaves();
#pragma omp parallel for schedule(dynamic, 8)
        for (long li = 0; li < (long)leaves.size(); ++li) {
            size_t leaf = leaves[li];
            const auto& ll = loc[leaf];
            const Node& nd = tree.nodes[leaf];
            for (size_t pi : nd.points) {
                const auto& p = pw[pi];
                double acc = 0.0;
                for (size_t m = 0; m < n3; ++m) acc += p[m] * ll[m];
                if (with_p2p) {
                    V3 xi = points[pi];
                    auto visit = [&](size_t c) {
                        for (size_t sj : tree.nodes[c].points) {
                            if (sj == pi) continue;
                            double r = norm(xi - points[sj]);
                            if (r > 0.0) acc += q[sj] / r;
                        }
                    };
                    for (size_t c : nd.neighbors) visit(c);
                    visit(leaf);
                }
                y[pi] += acc;
            }
        }
        return y;
    }

    // fmm/bbfmm.rs:192-206
    std::vector<std::pair<std::vector<size_t>, std::vector<size_t>>> near_blocks() const {
        std::vector<std::pair<std::vector<size_t>, std::vector<size_t>>> out;
        for (size_t leaf : tree.leaves()) {
            const auto& targets = tree.nodes[leaf].points;
            if (targets.empty()) continue;
            std::vector<size_t> src = targets;
            for (size_t c : tree.nodes[leaf].neighbors)
                src.insert(src.end(), tree.nodes[c].points.begin(), tree.nodes[c].points.end());
            out.push_back({targets, src});
        }
        return out;
    }
};

// cap/fmm_solver.rs:23-129
struct FmmCapOp : Op {
    Fmm fmm;
    std::vector<double> areas;
    std::vector<size_t> off;
    std::vector<uint32_t> idx;
    std::vector<double> val;
    size_t n;
    static std::vector<V3> pts_of(const PanelSet& s) {
        std::vector<V3> p(s.size());
        for (size_t i = 0; i < s.size(); ++i) p[i] = s.c(i);
        return p;
    }
    FmmCapOp(const PanelSet& s, int order, int max_level)
        : fmm(pts_of(s), order, max_level), areas(s.ar), n(s.size()) {
        auto blocks = fmm.near_blocks();
        std::vector<std::vector<std::pair<uint32_t, double>>> rows(n);
        std::vector<std::pair<size_t, size_t>> work;
        for (size_t b = 0; b < blocks.size(); ++b)
            for (size_t t = 0; t < blocks[b].first.size(); ++t) work.push_back({b, t});
#pragma omp parallel for schedule(dynamic, 16)
        for (long wi = 0; wi < (long)work.size(); ++wi) {
            const auto& blk = blocks[work[wi].first];
            size_t i = blk.first[work[wi].second];
            V3 ri = s.c(i);
            std::vector<std::pair<uint32_t, double>> row;
            row.reserve(blk.second.size());
            for (size_t j : blk.second) row.push_back({(uint32_t)j, ONE_OVER_4PI_EPS0 * potential_integral(s.quads[j], ri)});
            rows[i] = std::move(row);
        }
        off.push_back(0);
        for (auto& r : rows) {
            for (auto& e : r) {
                idx.push_back(e.first);
                val.push_back(e.second);
            }
            off.push_back(idx.size());
        }
    }
    size_t dim() const override { return n; }
    void apply(const double* sigma, double* y) const override {
        std::vector<double> q(n);
        for (size_t j = 0; j < n; ++j) q[j] = areas[j] * sigma[j];
        std::vector<double> far = fmm.run(q.data(), false);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; ++i) {
            double acc = ONE_OVER_4PI_EPS0 * far[i];
            for (size_t e = off[i]; e < off[i + 1]; ++e) acc += val[e] * sigma[idx[e]];
            y[i] = acc;
        }
    }
    bool diagonal(size_t i, double& d) const {
        for (size_t e = off[i]; e < off[i + 1]; ++e)
            if (idx[e] == i) {
                d = val[e];
                return true;
            }
        return false;
    }
};

// cap/fmm_solver.rs:133-144
struct DiagJacobi : Op {
    std::vector<double> inv;
    size_t dim() const override { return inv.size(); }
    void apply(const double* x, double* y) const override {
        for (size_t i = 0; i < inv.size(); ++i) y[i] = x[i] * inv[i];
    }
};

struct DenseOp : Op {
    const std::vector<double>& p;
    size_t n;
    DenseOp(const std::vector<double>& pp, size_t nn) : p(pp), n(nn) {}
    size_t dim() const override { return n; }
    // operator.rs:13-35: SIMD dot per row
    void apply(const double* x, double* y) const override {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < (long)n; ++i) y[i] = dot16(&p[i * n], x, n);
    }
};

// cap/solver.rs:81-97
std::vector<double> assemble_p(const PanelSet& s) {
    size_t n = s.size();
    std::vector<double> p(n * n);
#pragma omp parallel for schedule(dynamic, 4)
    for (long k = 0; k < (long)n; ++k) {
        V3 rk = s.c(k);
        for (size_t l = 0; l < n; ++l) p[k * n + l] = ONE_OVER_4PI_EPS0 * potential_integral(s.quads[l], rk);
    }
    return p;
}

// cap/solver.rs:55-71
std::vector<double> rhs_unit(const PanelSet& s, int j) {
    std::vector<double> b(s.size(), 0.0);
    for (size_t k = 0; k < s.size(); ++k)
        if (s.cond[k] == j) b[k] = 1.0;
    return b;
}
void accumulate_c(const PanelSet& s, const std::vector<double>& sigma, int j, int ncond, double* C) {
    for (size_t k = 0; k < s.size(); ++k) C[(size_t)s.cond[k] * ncond + j] += sigma[k] * s.ar[k];
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------- meshes
void put_quad(double* out, V3 a, V3 b, V3 c, V3 d) {
    V3 v[4] = {a, b, c, d};
    for (int i = 0; i < 4; ++i) {
        out[3 * i] = v[i].x;
        out[3 * i + 1] = v[i].y;
        out[3 * i + 2] = v[i].z;
    }
}

struct PanelSink {
    std::vector<double> verts;
    std::vector<int32_t> cond;
    std::vector<double> eps;
    void push(V3 a, V3 b, V3 c, V3 d, bool reverse, int32_t conductor) {
        size_t o = verts.size();
        verts.resize(o + 12);
        if (reverse)
            put_quad(&verts[o], d, c, b, a);
        else
            put_quad(&verts[o], a, b, c, d);
        cond.push_back(conductor);
    }
    size_t size() const { return cond.size(); }
};

// cap/mesh.rs:12-43
void plate(PanelSink& s, double cx, double cy, double z0, double lx, double ly, size_t nx, size_t ny,
           int32_t conductor) {
    double x0 = cx - lx / 2.0, y0 = cy - ly / 2.0, dx = lx / (double)nx, dy = ly / (double)ny;
    for (size_t i = 0; i < nx; ++i)
        for (size_t j = 0; j < ny; ++j) {
            double xa = x0 + (double)i * dx, xb = xa + dx, ya = y0 + (double)j * dy, yb = ya + dy;
            s.push({xa, ya, z0}, {xb, ya, z0}, {xb, yb, z0}, {xa, yb, z0}, false, conductor);
        }
}

// ---------------------------------------------------------------- bridge
const size_t MAX_GRID_CELLS = 262144;
const size_t MAX_PANELS = 20000;

struct Rect {
    int32_t x0, y0, x1, y1;
};

// core/geometry/rects.rs:96-176
int decompose(const int32_t* xs_in, const int32_t* ys_in, size_t n, std::vector<Rect>& rects, std::string& msg) {
    if (n < 4) {
        msg = "has " + std::to_string(n) + " vertices, need >= 4 for rectilinear decomposition";
        return -1;
    }
    for (size_t i = 0; i < n; ++i) {
        int32_t x0 = xs_in[i], y0 = ys_in[i], x1 = xs_in[(i + 1) % n], y1 = ys_in[(i + 1) % n];
        if (x0 != x1 && y0 != y1) {
            msg = "non-rectilinear edge (" + std::to_string(x0) + "," + std::to_string(y0) + ") -> (" +
                  std::to_string(x1) + "," + std::to_string(y1) + ")";
            return -2;
        }
    }
    std::vector<int32_t> xs(xs_in, xs_in + n);
    std::sort(xs.begin(), xs.end());
    xs.erase(std::unique(xs.begin(), xs.end()), xs.end());
    if (xs.size() < 2) return 0;
    std::vector<int32_t> cr;
    for (size_t w = 0; w + 1 < xs.size(); ++w) {
        int32_t sx0 = xs[w], sx1 = xs[w + 1];
        cr.clear();
        for (size_t i = 0; i < n; ++i) {
            int32_t x0 = xs_in[i], y0 = ys_in[i], x1 = xs_in[(i + 1) % n], y1 = ys_in[(i + 1) % n];
            if (y0 != y1) continue;
            if (std::min(x0, x1) <= sx0 && std::max(x0, x1) >= sx1) cr.push_back(y0);
        }
        std::sort(cr.begin(), cr.end());
        if (cr.size() % 2 != 0) {
            msg = "odd crossing count " + std::to_string(cr.size()) + " in slab [" + std::to_string(sx0) + ", " +
                  std::to_string(sx1) + "] (self-intersecting?)";
            return -3;
        }
        for (size_t k = 0; k + 1 < cr.size(); k += 2)
            if (cr[k] < cr[k + 1]) rects.push_back({sx0, cr[k], sx1, cr[k + 1]});
    }
    return 0;
}

// bridge.rs:559-563 (reference rule) and the target-edge rule.
size_t subdivisions(double length, double transverse, double max_edge) {
    if (max_edge > 0.0) {
        double v = std::ceil(length / max_edge);
        return (size_t)std::fmin(std::fmax(v, 1.0), 1.0e6);
    }
    double v = std::ceil(length / (4.0 * std::fmax(transverse, 2.2250738585072014e-308)));
    return (size_t)std::fmin(std::fmax(v, 1.0), 32.0);
}

// bridge.rs:566-596
void xy_face(PanelSink& s, double x0, double x1, double y0, double y1, double z, int32_t c, bool rev, double me) {
    size_t nx = subdivisions(x1 - x0, y1 - y0, me), ny = subdivisions(y1 - y0, x1 - x0, me);
    for (size_t ix = 0; ix < nx; ++ix)
        for (size_t iy = 0; iy < ny; ++iy) {
            double xa = x0 + (x1 - x0) * (double)ix / (double)nx;
            double xb = x0 + (x1 - x0) * (double)(ix + 1) / (double)nx;
            double ya = y0 + (y1 - y0) * (double)iy / (double)ny;
            double yb = y0 + (y1 - y0) * (double)(iy + 1) / (double)ny;
            s.push({xa, ya, z}, {xb, ya, z}, {xb, yb, z}, {xa, yb, z}, rev, c);
        }
}
// bridge.rs:599-624
void yz_face(PanelSink& s, double x, double y0, double y1, double z0, double z1, int32_t c, bool rev, double me) {
    size_t ny = subdivisions(y1 - y0, z1 - z0, me);
    size_t nz = me > 0.0 ? subdivisions(z1 - z0, y1 - y0, me) : 1;
    for (size_t iy = 0; iy < ny; ++iy)
        for (size_t iz = 0; iz < nz; ++iz) {
            double ya = y0 + (y1 - y0) * (double)iy / (double)ny;
            double yb = y0 + (y1 - y0) * (double)(iy + 1) / (double)ny;
            double za = nz == 1 ? z0 : z0 + (z1 - z0) * (double)iz / (double)nz;
            double zb = nz == 1 ? z1 : z0 + (z1 - z0) * (double)(iz + 1) / (double)nz;
            s.push({x, ya, za}, {x, yb, za}, {x, yb, zb}, {x, ya, zb}, rev, c);
        }
}
// bridge.rs:627-652
void xz_face(PanelSink& s, double x0, double x1, double y, double z0, double z1, int32_t c, bool rev, double me) {
    size_t nx = subdivisions(x1 - x0, z1 - z0, me);
    size_t nz = me > 0.0 ? subdivisions(z1 - z0, x1 - x0, me) : 1;
    for (size_t ix = 0; ix < nx; ++ix)
        for (size_t iz = 0; iz < nz; ++iz) {
            double xa = x0 + (x1 - x0) * (double)ix / (double)nx;
            double xb = x0 + (x1 - x0) * (double)(ix + 1) / (double)nx;
            double za = nz == 1 ? z0 : z0 + (z1 - z0) * (double)iz / (double)nz;
            double zb = nz == 1 ? z1 : z0 + (z1 - z0) * (double)(iz + 1) / (double)nz;
            s.push({xa, y, za}, {xb, y, za}, {xb, y, zb}, {xa, y, zb}, rev, c);
        }
}

struct Group {
    uint32_t net;
    double z0, z1, k;
    std::vector<Rect> rects;
};

// bridge.rs:445-557
int group_panels(const Group& g, int32_t conductor, double xy, double me, size_t max_panels, PanelSink& s,
                 std::string& msg) {
    std::vector<int32_t> xs, ys;
    for (const Rect& r : g.rects) {
        xs.push_back(r.x0);
        xs.push_back(r.x1);
        ys.push_back(r.y0);
        ys.push_back(r.y1);
    }
    std::sort(xs.begin(), xs.end());
    xs.erase(std::unique(xs.begin(), xs.end()), xs.end());
    std::sort(ys.begin(), ys.end());
    ys.erase(std::unique(ys.begin(), ys.end()), ys.end());
    size_t nx = xs.empty() ? 0 : xs.size() - 1, ny = ys.empty() ? 0 : ys.size() - 1;
    size_t cells = nx * ny;
    if (cells > MAX_GRID_CELLS) {
        msg = "conductor union grid needs " + std::to_string(cells) + " cells; limit is " +
              std::to_string(MAX_GRID_CELLS);
        return -5;
    }
    std::vector<char> filled(cells, 0), consumed(cells, 0);
    for (size_t ix = 0; ix < nx; ++ix)
        for (size_t iy = 0; iy < ny; ++iy) {
            bool f = false;
            for (const Rect& r : g.rects)
                if (r.x0 <= xs[ix] && r.x1 >= xs[ix + 1] && r.y0 <= ys[iy] && r.y1 >= ys[iy + 1]) {
                    f = true;
                    break;
                }
            filled[ix * ny + iy] = f;
        }
    for (size_t ix = 0; ix < nx; ++ix)
        for (size_t iy = 0; iy < ny; ++iy) {
            size_t cell = ix * ny + iy;
            if (!filled[cell] || consumed[cell]) continue;
            size_t x_end = ix + 1;
            while (x_end < nx && filled[x_end * ny + iy] && !consumed[x_end * ny + iy]) ++x_end;
            size_t y_end = iy + 1;
            bool stop = false;
            while (y_end < ny && !stop) {
                for (size_t x = ix; x < x_end; ++x) {
                    size_t nxt = x * ny + y_end;
                    if (!filled[nxt] || consumed[nxt]) {
                        stop = true;
                        break;
                    }
                }
                if (!stop) ++y_end;
            }
            for (size_t x = ix; x < x_end; ++x)
                for (size_t y = iy; y < y_end; ++y) consumed[x * ny + y] = 1;
            double x0 = (double)xs[ix] * xy, x1 = (double)xs[x_end] * xy;
            double y0 = (double)ys[iy] * xy, y1 = (double)ys[y_end] * xy;
            xy_face(s, x0, x1, y0, y1, g.z1, conductor, false, me);
            xy_face(s, x0, x1, y0, y1, g.z0, conductor, true, me);
        }
    for (size_t ix = 0; ix < nx; ++ix)
        for (size_t iy = 0; iy < ny; ++iy) {
            if (!filled[ix * ny + iy]) continue;
            double x0 = (double)xs[ix] * xy, x1 = (double)xs[ix + 1] * xy;
            double y0 = (double)ys[iy] * xy, y1 = (double)ys[iy + 1] * xy;
            if (ix == 0 || !filled[(ix - 1) * ny + iy]) yz_face(s, x0, y0, y1, g.z0, g.z1, conductor, true, me);
            if (ix + 1 == nx || !filled[(ix + 1) * ny + iy]) yz_face(s, x1, y0, y1, g.z0, g.z1, conductor, false, me);
            if (iy == 0 || !filled[ix * ny + iy - 1]) xz_face(s, x0, x1, y0, g.z0, g.z1, conductor, false, me);
            if (iy + 1 == ny || !filled[ix * ny + iy + 1]) xz_face(s, x0, x1, y1, g.z0, g.z1, conductor, true, me);
        }
    s.eps.resize(s.size(), g.k);
    if (s.size() > max_panels) {
        msg = "extruded layout needs " + std::to_string(s.size()) + " panels; limit is " + std::to_string(max_panels);
        return -6;
    }
    return 0;
}

bool is_volume_conductor(const orc_layer_params& p) {  // bridge.rs:171-178
    return p.sheet_res_ohm_sq != 0.0 || p.area_cap_af_um2 != 0.0 || p.fringe_cap_af_um != 0.0 ||
           p.coupling_cap_af_um != 0.0 || p.interlayer_cap_af_um2 != 0.0 ||
           (p.thickness_nm > 0.0 && p.via_res_ohm == 0.0);
}

void set_err(char* buf, int64_t cap, const std::string& s) {
    if (!buf || cap <= 0) return;
    size_t n = std::min((size_t)cap - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
}

}  // namespace

// =====================================================================
// C API
// =====================================================================
extern "C" {

double orc_potential_integral(const double* verts12, const double* p3) {
    return potential_integral(load_quad(verts12), V3{p3[0], p3[1], p3[2]});
}

void orc_panel_props(const double* verts12, double* c3, double* a, double* n3) {
    Quad q = load_quad(verts12);
    V3 c = centroid(q);
    c3[0] = c.x;
    c3[1] = c.y;
    c3[2] = c.z;
    *a = area(q);
    V3 n = normalized(cross(q.v[1] - q.v[0], q.v[2] - q.v[0]));  // panel.rs:50-55
    n3[0] = n.x;
    n3[1] = n.y;
    n3[2] = n.z;
}

int64_t orc_plate(double cx, double cy, double z0, double lx, double ly, int64_t nx, int64_t ny, int32_t conductor,
                  double* verts_out, int32_t* cond_out, int64_t cap) {
    PanelSink s;
    plate(s, cx, cy, z0, lx, ly, (size_t)nx, (size_t)ny, conductor);
    if ((int64_t)s.size() > cap) return -4;
    std::memcpy(verts_out, s.verts.data(), s.verts.size() * sizeof(double));
    std::memcpy(cond_out, s.cond.data(), s.cond.size() * sizeof(int32_t));
    return (int64_t)s.size();
}

// cap/mesh.rs:48-114
int64_t orc_icosphere(double cx, double cy, double cz, double r, int32_t subdivisions, int32_t conductor,
                      double* verts_out, int32_t* cond_out, int64_t cap) {
    double t = (1.0 + std::sqrt(5.0)) / 2.0;
    std::vector<V3> v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                         {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& p : v) p = normalized(p);
    std::vector<std::array<size_t, 3>> f = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11},
                                            {1, 5, 9},  {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                                            {3, 9, 4},  {3, 4, 2},  {3, 2, 6},   {3, 6, 8},  {3, 8, 9},
                                            {4, 9, 5},  {2, 4, 11}, {6, 2, 10},  {8, 6, 7},  {9, 8, 1}};
    for (int s = 0; s < subdivisions; ++s) {
        std::map<std::pair<size_t, size_t>, size_t> cache;
        auto mid = [&](size_t a, size_t b) {
            auto key = a < b ? std::make_pair(a, b) : std::make_pair(b, a);
            auto it = cache.find(key);
            if (it != cache.end()) return it->second;
            V3 m = normalized((v[a] + v[b]) * 0.5);
            size_t idx = v.size();
            v.push_back(m);
            cache[key] = idx;
            return idx;
        };
        std::vector<std::array<size_t, 3>> nf;
        for (auto& fc : f) {
            size_t a = mid(fc[0], fc[1]), b = mid(fc[1], fc[2]), c = mid(fc[2], fc[0]);
            nf.push_back({fc[0], a, c});
            nf.push_back({fc[1], b, a});
            nf.push_back({fc[2], c, b});
            nf.push_back({a, b, c});
        }
        f = nf;
    }
    if ((int64_t)f.size() > cap) return -4;
    V3 ctr{cx, cy, cz};
    for (size_t i = 0; i < f.size(); ++i) {
        V3 a = ctr + v[f[i][0]] * r, b = ctr + v[f[i][1]] * r, c = ctr + v[f[i][2]] * r;
        put_quad(verts_out + 12 * i, a, b, c, c);
        cond_out[i] = conductor;
    }
    return (int64_t)f.size();
}

int64_t orc_decompose_rectilinear(const int32_t* xs, const int32_t* ys, int64_t nv, int32_t* out, int64_t cap) {
    std::vector<Rect> rects;
    std::string msg;
    int rc = decompose(xs, ys, (size_t)nv, rects, msg);
    if (rc < 0) return rc;
    if ((int64_t)rects.size() > cap) return -4;
    for (size_t i = 0; i < rects.size(); ++i) {
        out[4 * i] = rects[i].x0;
        out[4 * i + 1] = rects[i].y0;
        out[4 * i + 2] = rects[i].x1;
        out[4 * i + 3] = rects[i].y1;
    }
    return (int64_t)rects.size();
}

int64_t orc_bridge_panelize(const int32_t* vx, const int32_t* vy, const uint32_t* pstart, const uint32_t* plen,
                            const uint16_t* player, int64_t n_poly, const uint32_t* net_of_poly, int64_t n_nop,
                            const orc_layer_params* layers, int64_t n_layers, double dbu_nm, double me,
                            int64_t max_panels_in, double* verts_out, int32_t* cond_out, double* eps_out,
                            int64_t cap, uint32_t* nets_out, int64_t* n_nets_out, double* via_r_out, char* err,
                            int64_t err_cap) {
    const double M_PER_NM = 1.0e-9;
    size_t max_panels = max_panels_in == 0 ? MAX_PANELS : (max_panels_in < 0 ? SIZE_MAX : (size_t)max_panels_in);
    if (!std::isfinite(dbu_nm) || dbu_nm <= 0.0) {  // bridge.rs:78-80
        char b[128];
        snprintf(b, sizeof b, "deck database unit must be finite and positive, got %g nm", dbu_nm);
        set_err(err, err_cap, b);
        return -10;
    }
    // ProcessStack::from_deck (analytical/process_stack.rs:31-76)
    std::vector<orc_layer_params> sorted(layers, layers + n_layers);
    std::sort(sorted.begin(), sorted.end(), [](const orc_layer_params& a, const orc_layer_params& b) {
        return a.layer < b.layer;
    });
    struct Proc {
        double t, h, k;
    };
    std::map<uint16_t, Proc> stack;
    std::map<uint16_t, orc_layer_params> params;
    double next_z = 0.0;
    for (auto& p : sorted) {
        double th = p.thickness_nm > 0.0 ? p.thickness_nm : 200.0;
        double h = (p.height_nm > 0.0 || p.thickness_nm > 0.0) ? p.height_nm : next_z;
        next_z = h + th + 100.0;
        stack[p.layer] = {th, h, p.dielectric_k > 0.0 ? p.dielectric_k : 3.9};
        params[p.layer] = p;
    }
    // validate_stack (bridge.rs:149-169)
    for (auto& kv : stack) {
        struct {
            const char* f;
            double v;
            bool pos;
        } fs[3] = {{"thickness_nm", kv.second.t, true}, {"height_nm", kv.second.h, false},
                   {"dielectric_k", kv.second.k, true}};
        for (auto& f : fs)
            if (!std::isfinite(f.v) || (f.pos && f.v <= 0.0) || (std::string(f.f) == "height_nm" && f.v < 0.0)) {
                char b[160];
                snprintf(b, sizeof b, "PEX layer %u has invalid %s value %g", (unsigned)kv.first, f.f, f.v);
                set_err(err, err_cap, b);
                return -11;
            }
    }
    std::map<uint32_t, double> via_r;
    std::set<uint32_t> out_nets;
    std::map<std::pair<uint32_t, uint16_t>, Group> grouped;
    for (int64_t poly = 0; poly < n_poly; ++poly) {
        uint16_t layer = player[poly];
        auto pit = params.find(layer);
        if (pit == params.end()) continue;
        uint32_t net = poly < n_nop ? net_of_poly[poly] : 0xFFFFFFFFu;
        const orc_layer_params& p = pit->second;
        if (p.via_res_ohm != 0.0) via_r[net] += p.via_res_ohm;
        if (!is_volume_conductor(p)) continue;
        out_nets.insert(net);
        std::vector<Rect> rects;
        std::string msg;
        int rc = decompose(vx + pstart[poly], vy + pstart[poly], plen[poly], rects, msg);
        if (rc < 0) {
            set_err(err, err_cap,
                    "polygon " + std::to_string(poly) + " cannot be extruded for quasi-static PEX: polygon " +
                        std::to_string(poly) + ": " + msg);
            return -12;
        }
        if (rects.empty()) {
            set_err(err, err_cap,
                    "polygon " + std::to_string(poly) +
                        " cannot be extruded for quasi-static PEX: rectilinear decomposition produced no material");
            return -12;
        }
        auto key = std::make_pair(net, layer);
        auto git = grouped.find(key);
        if (git == grouped.end()) {
            const Proc& pr = stack[layer];
            Group g{net, pr.h * M_PER_NM, (pr.h + pr.t) * M_PER_NM, pr.k, {}};
            git = grouped.emplace(key, g).first;
        }
        git->second.rects.insert(git->second.rects.end(), rects.begin(), rects.end());
    }
    // solve_capacitance panelisation (bridge.rs:307-386)
    std::set<uint32_t> nets;
    for (auto& kv : grouped) nets.insert(kv.second.net);
    std::map<uint32_t, int32_t> net_index;
    {
        int32_t i = 0;
        for (uint32_t n : nets) net_index[n] = i++;
    }
    int64_t nn = 0;
    for (uint32_t n : nets) {
        nets_out[nn] = n;
        if (via_r_out) via_r_out[nn] = via_r.count(n) ? via_r[n] : 0.0;
        ++nn;
    }
    *n_nets_out = nn;
    if (grouped.empty()) return 0;
    double xy = dbu_nm * M_PER_NM;
    PanelSink s;
    double b[4] = {INFINITY, INFINITY, -INFINITY, -INFINITY}, min_z = INFINITY, max_t = 0.0;
    for (auto& kv : grouped) {
        const Group& g = kv.second;
        std::string msg;
        int rc = group_panels(g, net_index[g.net], xy, me, max_panels, s, msg);
        if (rc < 0) {
            set_err(err, err_cap, msg);
            return rc;
        }
        for (const Rect& r : g.rects) {
            b[0] = std::fmin(b[0], (double)r.x0 * xy);
            b[1] = std::fmin(b[1], (double)r.y0 * xy);
            b[2] = std::fmax(b[2], (double)r.x1 * xy);
            b[3] = std::fmax(b[3], (double)r.y1 * xy);
        }
        min_z = std::fmin(min_z, g.z0);
        max_t = std::fmax(max_t, g.z1 - g.z0);
    }
    double gap = min_z > 0.0 ? min_z : std::fmax(max_t, 100.0 * M_PER_NM);
    double gz = min_z > 0.0 ? 0.0 : min_z - gap;
    double sx = b[2] - b[0], sy = b[3] - b[1];
    double pad = 0.5 * std::fmax(std::fmax(sx, sy), 8.0 * gap);
    double lx = sx + 2.0 * pad, ly = sy + 2.0 * pad;
    int32_t gid = (int32_t)nets.size();
    // ground eps = k of the group with minimum z0 (first minimum in map order)
    double geps = 1.0, bestz = INFINITY;
    for (auto& kv : grouped)
        if (kv.second.z0 < bestz) {
            bestz = kv.second.z0;
            geps = kv.second.k;
        }
    // reference rule (cap/mesh.rs:12-43 via bridge.rs:346-379): cells of 4 gap,
    // 4..32 per side; target-edge mode: cells of at most 4 max_edge, no cap
    double plate_cap = me > 0.0 ? 4096.0 : 32.0;
    double cell = me > 0.0 ? std::fmin(4.0 * gap, 4.0 * me) : 4.0 * gap;
    size_t gnx = (size_t)std::fmin(std::fmax(std::ceil(lx / cell), 4.0), plate_cap);
    size_t gny = (size_t)std::fmin(std::fmax(std::ceil(ly / cell), 4.0), plate_cap);
    size_t before = s.size();
    plate(s, 0.5 * (b[0] + b[2]), 0.5 * (b[1] + b[3]), gz, lx, ly, gnx, gny, gid);
    s.eps.resize(s.size(), geps);
    (void)before;
    if (s.size() > max_panels) {
        set_err(err, err_cap,
                "extruded layout needs " + std::to_string(s.size()) + " panels; limit is " +
                    std::to_string(max_panels));
        return -6;
    }
    if ((int64_t)s.size() > cap) {
        set_err(err, err_cap, "output capacity exceeded");
        return -4;
    }
    std::memcpy(verts_out, s.verts.data(), s.verts.size() * sizeof(double));
    std::memcpy(cond_out, s.cond.data(), s.cond.size() * sizeof(int32_t));
    std::memcpy(eps_out, s.eps.data(), s.eps.size() * sizeof(double));
    return (int64_t)s.size();
}

int orc_dense_P(int64_t n, const double* verts, double* P_out) {
    PanelSet s = build_set(n, verts, nullptr);
    std::vector<double> p = assemble_p(s);
    std::memcpy(P_out, p.data(), p.size() * sizeof(double));
    return 0;
}

// cap/solver.rs:100-134 (Method::Direct)
int orc_cap_dense(int64_t n, const double* verts, const int32_t* cond, int32_t ncond, double* C) {
    if (n <= 0) return -1;
    PanelSet s = build_set(n, verts, cond);
    std::vector<double> p = assemble_p(s);
    LU f = lu_factor(p, (size_t)n);
    if (!f.ok) return -2;
    std::fill(C, C + (size_t)ncond * ncond, 0.0);
    for (int j = 0; j < ncond; ++j) {
        std::vector<double> x = lu_solve(f, rhs_unit(s, j));
        accumulate_c(s, x, j, ncond, C);
    }
    return 0;
}

// cap/dielectric.rs:76-150 with conductor roles only, as the bridge calls it
// for a stack of several k (bridge.rs:409-430): the same potential rows and
// unit-conductor right-hand sides as the homogeneous solve, but each panel's
// charge counts with its own surrounding permittivity,
// C[id][j] += eps_k * sigma_k * a_k.
int orc_cap_dense_eps(int64_t n, const double* verts, const int32_t* cond, int32_t ncond, const double* eps,
                      double* C) {
    if (n <= 0) return -1;
    PanelSet s = build_set(n, verts, cond);
    std::vector<double> p = assemble_p(s);
    LU f = lu_factor(p, (size_t)n);
    if (!f.ok) return -2;
    std::fill(C, C + (size_t)ncond * ncond, 0.0);
    for (int j = 0; j < ncond; ++j) {
        std::vector<double> x = lu_solve(f, rhs_unit(s, j));
        for (size_t k = 0; k < s.size(); ++k) C[(size_t)s.cond[k] * ncond + j] += eps[k] * x[k] * s.ar[k];
    }
    return 0;
}

// cap/solver.rs:118-125 (Method::Iterative)
int orc_cap_dense_gmres(int64_t n, const double* verts, const int32_t* cond, int32_t ncond, double* C) {
    if (n <= 0) return -1;
    PanelSet s = build_set(n, verts, cond);
    std::vector<double> p = assemble_p(s);
    DenseOp op(p, (size_t)n);
    std::fill(C, C + (size_t)ncond * ncond, 0.0);
    for (int j = 0; j < ncond; ++j) {
        std::vector<double> b = rhs_unit(s, j);
        GmresResult r = gmres(op, b.data(), nullptr, {1e-8, 100, 50});
        accumulate_c(s, r.x, j, ncond, C);
    }
    return 0;
}

// cap/fmm_solver.rs:147-172
int orc_cap_fmm(int64_t n, const double* verts, const int32_t* cond, int32_t ncond, const orc_fmm_opts* o,
                double* C, orc_fmm_report* rep) {
    if (n <= 0) return -1;
#ifdef _OPENMP
    int saved = omp_get_max_threads();
    if (o->threads > 0) omp_set_num_threads(o->threads);
#endif
    double t0 = now_s();
    PanelSet s = build_set(n, verts, cond);
    FmmCapOp op(s, o->order, o->max_level);
    DiagJacobi pc;
    pc.inv.resize((size_t)n);
    for (size_t i = 0; i < (size_t)n; ++i) {
        double d = 1.0;
        op.diagonal(i, d);
        pc.inv[i] = std::fabs(d) > 1e-30 ? 1.0 / d : 1.0;
    }
    double t1 = now_s();
    std::fill(C, C + (size_t)ncond * ncond, 0.0);
    orc_fmm_report r{};
    r.all_converged = 1;
    const int stride = o->rhs_stride > 1 ? o->rhs_stride : 1;
    const int avail = (ncond + stride - 1) / stride;
    const int nrhs = o->rhs_limit > 0 ? std::min(o->rhs_limit, avail) : avail;
    for (int q = 0; q < nrhs; ++q) {
        const int j = q * stride;
        std::vector<double> b = rhs_unit(s, j);
        GmresResult g = gmres(op, b.data(), &pc, {o->tol, (size_t)o->restart, (size_t)o->max_restarts});
        accumulate_c(s, g.x, j, ncond, C);
        r.total_iterations += (int64_t)g.iterations;
        r.max_iterations = std::max<int64_t>(r.max_iterations, (int64_t)g.iterations);
        r.max_residual = std::fmax(r.max_residual, g.residual);
        if (!g.converged) r.all_converged = 0;
    }
    double t2 = now_s();
    r.nnz_near = (int64_t)op.val.size();
    r.n_boxes = (int64_t)op.fmm.tree.nodes.size();
    r.t_setup_s = t1 - t0;
    r.t_solve_s = t2 - t1;
    if (rep) *rep = r;
#ifdef _OPENMP
    omp_set_num_threads(saved);
#endif
    return 0;
}

// The same solve split into its set-up and its per-conductor solves, so a
// caller can time one conductor's GMRES at a time (cap/fmm_solver.rs:147-172:
// the operator and the Jacobi preconditioner are built once, then each
// conductor is solved in turn).
struct OrcFmmHandle {
    PanelSet s;
    FmmCapOp op;
    DiagJacobi pc;
    int ncond;
    int threads;
    OrcFmmHandle(PanelSet&& set, int order, int level, int nc, int th)
        : s(std::move(set)), op(s, order, level), ncond(nc), threads(th) {}
};

void* orc_fmm_new(int64_t n, const double* verts, const int32_t* cond, int32_t ncond, int32_t order,
                  int32_t max_level, int32_t threads, double* t_setup_s) {
    if (n <= 0) return nullptr;
#ifdef _OPENMP
    int saved = omp_get_max_threads();
    if (threads > 0) omp_set_num_threads(threads);
#endif
    double t0 = now_s();
    OrcFmmHandle* h = new OrcFmmHandle(build_set(n, verts, cond), order, max_level, ncond, threads);
    h->pc.inv.resize((size_t)n);
    for (size_t i = 0; i < (size_t)n; ++i) {
        double d = 1.0;
        h->op.diagonal(i, d);
        h->pc.inv[i] = std::fabs(d) > 1e-30 ? 1.0 / d : 1.0;
    }
    if (t_setup_s) *t_setup_s = now_s() - t0;
#ifdef _OPENMP
    omp_set_num_threads(saved);
#endif
    return h;
}

// Column j of the Maxwell matrix: C_out[i] = C[i][j] for i < ncond.
int orc_fmm_solve_column(void* handle, int32_t j, double tol, int32_t restart, int32_t max_restarts,
                         double* C_col, int64_t* iterations, double* residual) {
    OrcFmmHandle* h = static_cast<OrcFmmHandle*>(handle);
    if (!h || j < 0 || j >= h->ncond) return -1;
#ifdef _OPENMP
    int saved = omp_get_max_threads();
    if (h->threads > 0) omp_set_num_threads(h->threads);
#endif
    std::vector<double> b = rhs_unit(h->s, j);
    GmresResult g = gmres(h->op, b.data(), &h->pc, {tol, (size_t)restart, (size_t)max_restarts});
    std::vector<double> C((size_t)h->ncond * h->ncond, 0.0);
    accumulate_c(h->s, g.x, j, h->ncond, C.data());
    for (int i = 0; i < h->ncond; ++i) C_col[i] = C[(size_t)i * h->ncond + j];
    if (iterations) *iterations = (int64_t)g.iterations;
    if (residual) *residual = g.residual;
#ifdef _OPENMP
    omp_set_num_threads(saved);
#endif
    return g.converged ? 0 : 1;
}

void orc_fmm_free(void* handle) { delete static_cast<OrcFmmHandle*>(handle); }

int orc_fmm_point_matvec(int64_t n, const double* pts3, const double* q, int32_t order, int32_t max_level,
                         int32_t with_p2p, double* y) {
    std::vector<V3> pts((size_t)n);
    for (int64_t i = 0; i < n; ++i) pts[i] = {pts3[3 * i], pts3[3 * i + 1], pts3[3 * i + 2]};
    Fmm f(pts, order, max_level);
    std::vector<double> out = f.run(q, with_p2p != 0);
    std::memcpy(y, out.data(), out.size() * sizeof(double));
    return 0;
}

int orc_fmm_cap_apply(int64_t n, const double* verts, int32_t order, int32_t max_level, const double* sigma,
                      double* y, int64_t* nnz_out) {
    PanelSet s = build_set(n, verts, nullptr);
    FmmCapOp op(s, order, max_level);
    op.apply(sigma, y);
    if (nnz_out) *nnz_out = (int64_t)op.val.size();
    return 0;
}

int orc_m2l_table(int32_t order, double* k_out, int32_t* rank_out) {
    int n = order;
    std::vector<double> nodes1d = cheb_nodes(n);
    std::vector<std::array<double, 3>> ref3d;
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b)
            for (int c = 0; c < n; ++c) ref3d.push_back({nodes1d[a], nodes1d[b], nodes1d[c]});
    size_t n3 = ref3d.size();
    for (int idx = 0; idx < 343; ++idx) rank_out[idx] = -1;
#pragma omp parallel for schedule(dynamic)
    for (int idx = 0; idx < 343; ++idx) {
        int ox = idx / 49 - 3, oy = (idx / 7) % 7 - 3, oz = idx % 7 - 3;
        if (std::max(std::abs(ox), std::max(std::abs(oy), std::abs(oz))) < 2) continue;
        LowRank lr = build_m2l(ref3d, n, ox, oy, oz);
        double* K = k_out + (size_t)idx * n3 * n3;
        for (size_t m = 0; m < n3; ++m)
            for (size_t l = 0; l < n3; ++l) {
                double s = 0.0;
                for (size_t i = 0; i < lr.k; ++i) s += lr.u[m * lr.k + i] * lr.vt[i * n3 + l];
                K[m * n3 + l] = s;
            }
        rank_out[idx] = (int32_t)lr.k;
    }
    return 0;
}

double orc_dot(const double* a, const double* b, int64_t n) { return dot16(a, b, (size_t)n); }

}  // extern "C"
