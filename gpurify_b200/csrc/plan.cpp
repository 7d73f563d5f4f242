// Host plan builder: bit-exact panel centroids/areas, the uniform octree of
// the reference (fmm/tree.rs:41-210), near-field blocks (bbfmm.rs:192-206),
// interaction lists and the M2L operator table (bbfmm.rs:132-174).
// Compiled with -ffp-contract=off: centroids, leaf cells and Chebyshev
// weights use the reference's operation order.
#include "plan.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <numeric>
#include <thread>
#include <unordered_map>

namespace gpx {

namespace {

struct P3 {
    double x, y, z;
};
inline P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline P3 add(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline P3 scl(P3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline P3 crs(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double len(P3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

inline uint64_t spread3(uint32_t v) {
    uint64_t x = v & 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}
inline uint64_t morton(uint32_t x, uint32_t y, uint32_t z) { return spread3(x) << 2 | spread3(y) << 1 | spread3(z); }
inline uint64_t cell_key(int64_t x, int64_t y, int64_t z) { return ((uint64_t)x << 42) | ((uint64_t)y << 21) | (uint64_t)z; }

// compiler-rt's repeated-squaring power, which Rust's f64::powi lowers to.
double powi_sq(double a, int b) {
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

// Column-pivoted modified Gram-Schmidt truncation of the m x m kernel matrix
// g (linalg.rs:277-381), returning the product Q_k * R_k (P^T applied):
// the operator the reference applies as U * (V^T x).
void qr_truncate_product(const std::vector<double>& g, int m, double eps, double* out, int32_t* rank, double* Uo,
                         double* Vto) {
    std::vector<double> q(g), r((size_t)m * m, 0.0), nrm(m);
    std::vector<int> perm(m);
    std::iota(perm.begin(), perm.end(), 0);
    for (int j = 0; j < m; ++j) {
        double s = -0.0;
        for (int i = 0; i < m; ++i) s += g[(size_t)i * m + j] * g[(size_t)i * m + j];
        nrm[j] = s;
    }
    double big = 0.0;
    for (double v : nrm) big = std::fmax(big, v);
    const double thr = eps * big;
    int k = 0;
    for (int st = 0; st < m; ++st) {
        int piv = st;
        for (int j = st + 1; j < m; ++j)
            if (nrm[j] > nrm[piv]) piv = j;
        if (nrm[piv] < thr) break;
        if (piv != st) {
            std::swap(perm[st], perm[piv]);
            std::swap(nrm[st], nrm[piv]);
            for (int i = 0; i < m; ++i) std::swap(q[(size_t)i * m + st], q[(size_t)i * m + piv]);
            for (int row = 0; row < st; ++row) std::swap(r[(size_t)row * m + st], r[(size_t)row * m + piv]);
        }
        double cn = 0.0;
        for (int i = 0; i < m; ++i) cn += q[(size_t)i * m + st] * q[(size_t)i * m + st];
        cn = std::sqrt(cn);
        if (cn < 1e-15) break;
        r[(size_t)st * m + st] = cn;
        const double inv = 1.0 / cn;
        for (int i = 0; i < m; ++i) q[(size_t)i * m + st] *= inv;
        for (int j = st + 1; j < m; ++j) {
            double d = 0.0;
            for (int i = 0; i < m; ++i) d += q[(size_t)i * m + st] * q[(size_t)i * m + j];
            r[(size_t)st * m + j] = d;
            for (int i = 0; i < m; ++i) q[(size_t)i * m + j] -= d * q[(size_t)i * m + st];
            nrm[j] -= d * d;
            if (nrm[j] < 0.0) nrm[j] = 0.0;
        }
        k = st + 1;
    }
    // V^T[i][perm[j]] = R[i][j]; product U * V^T.
    std::vector<double> vt((size_t)k * m);
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < m; ++j) vt[(size_t)i * m + perm[j]] = r[(size_t)i * m + j];
    for (int a = 0; a < m; ++a)
        for (int b = 0; b < m; ++b) {
            double s = 0.0;
            for (int i = 0; i < k; ++i) s += q[(size_t)a * m + i] * vt[(size_t)i * m + b];
            out[(size_t)a * m + b] = s;
        }
    for (int a = 0; a < m; ++a)
        for (int i = 0; i < m; ++i) Uo[(size_t)a * m + i] = i < k ? q[(size_t)a * m + i] : 0.0;
    for (int i = 0; i < m; ++i)
        for (int b = 0; b < m; ++b) Vto[(size_t)i * m + b] = i < k ? vt[(size_t)i * m + b] : 0.0;
    *rank = k;
}

}  // namespace

// Area-weighted fan centroid and area of a quad whose 4th vertex may repeat
// the 3rd (integrals/panel.rs:29-67).
void panel_centroid_area(const double* v, double* c, double* a) {
    P3 q[4];
    for (int i = 0; i < 4; ++i) q[i] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
    int nv = (q[3].x == q[2].x && q[3].y == q[2].y && q[3].z == q[2].z) ? 3 : 4;
    double asum = 0.0;
    P3 acc{0.0, 0.0, 0.0};
    for (int i = 1; i < nv - 1; ++i) {
        double t = len(crs(sub(q[i], q[0]), sub(q[i + 1], q[0]))) * 0.5;
        P3 tc = scl(add(add(q[0], q[i]), q[i + 1]), 1.0 / 3.0);
        acc = add(acc, scl(tc, t));
        asum += t;
    }
    P3 r = asum == 0.0 ? q[0] : scl(acc, 1.0 / asum);
    c[0] = r.x;
    c[1] = r.y;
    c[2] = r.z;
    *a = asum;
}


std::vector<double> cheb_roots(int n) {
    std::vector<double> v(n);
    for (int m = 0; m < n; ++m) v[m] = std::cos((2.0 * m + 1.0) * kPi / (2.0 * n));
    return v;
}

namespace {

// T_k(x_m) of the n roots, k = 0..n-1 (row m), by the recurrence
// cheb_weights runs: the same values, computed once per plan.
std::vector<double> cheb_root_table(int n, const double* roots) {
    std::vector<double> t((size_t)n * n);
    for (int m = 0; m < n; ++m) {
        const double xm = roots[m];
        double prev = 1.0, cur = xm;
        t[(size_t)m * n] = 1.0;
        for (int k = 1; k < n; ++k) {
            double tk;
            if (k == 1) {
                tk = xm;
            } else {
                tk = 2.0 * xm * cur - prev;
                prev = cur;
                cur = tk;
            }
            t[(size_t)m * n + k] = tk;
        }
    }
    return t;
}

// cheb_weights with the roots' T_k from cheb_root_table: identical sums in
// the identical order.
inline void cheb_weights_tab(double x, int n, const double* tab, double* out) {
    double tx[32];
    tx[0] = 1.0;
    if (n > 1) {
        tx[1] = x;
        for (int k = 2; k < n; ++k) tx[k] = 2.0 * x * tx[k - 1] - tx[k - 2];
    }
    const double inv_n = 1.0 / n;
    for (int m = 0; m < n; ++m) {
        const double* tm = tab + (size_t)m * n;
        double sum = 0.5;
        for (int k = 1; k < n; ++k) sum += tm[k] * tx[k];
        out[m] = 2.0 * inv_n * sum;
    }
}

constexpr unsigned kMaxChunks = 16;  // threads of one parallel_chunks call, the caller's included

// fn(chunk, begin, end) over [0, n) in contiguous chunks of at least
// min_chunk items, on up to kMaxChunks threads (the caller's among them).
// Returns the number of chunks.  Chunks are independent; fn must not throw.
template <class F>
int parallel_chunks(int64_t n, int64_t min_chunk, F&& fn) {
    const int64_t hw = std::max(1u, std::min(kMaxChunks, std::thread::hardware_concurrency()));
    const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(hw, n / std::max<int64_t>(1, min_chunk)));
    const int64_t per = (n + nt - 1) / nt;
    std::vector<std::thread> th;
    th.reserve(nt - 1);
    for (int t = 1; t < nt; ++t) {
        const int64_t b = std::min(n, t * per), e = std::min(n, b + per);
        th.emplace_back([&fn, t, b, e] { fn(t, b, e); });
    }
    fn(0, 0, std::min(n, per));
    for (auto& x : th) x.join();
    return nt;
}

}  // namespace

// S_n(x, x_m) = 1/n + 2/n sum_{k=1}^{n-1} T_k(x_m) T_k(x), by recurrence.
void cheb_weights(double x, int n, const double* roots, double* out) {
    double tx[32];
    tx[0] = 1.0;
    if (n > 1) {
        tx[1] = x;
        for (int k = 2; k < n; ++k) tx[k] = 2.0 * x * tx[k - 1] - tx[k - 2];
    }
    const double inv_n = 1.0 / n;
    for (int m = 0; m < n; ++m) {
        const double xm = roots[m];
        double sum = 0.5, prev = 1.0, cur = xm;
        for (int k = 1; k < n; ++k) {
            double tk;
            if (k == 1) {
                tk = xm;
            } else {
                tk = 2.0 * xm * cur - prev;
                prev = cur;
                cur = tk;
            }
            sum += tk * tx[k];
        }
        out[m] = 2.0 * inv_n * sum;
    }
}

void build_m2l_table(M2LTable& t, int n, int mode) {
    const int n3 = n * n * n;
    t.n = n;
    t.mode = mode;
    t.K.assign((size_t)343 * n3 * n3, 0.0);
    t.U.assign((size_t)343 * n3 * n3, 0.0);
    t.Vt.assign((size_t)343 * n3 * n3, 0.0);
    t.rank.assign(343, -1);
    std::vector<double> roots = cheb_roots(n);
    std::vector<double> ref((size_t)n3 * 3);
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b)
            for (int c = 0; c < n; ++c) {
                int m = (a * n + b) * n + c;
                ref[3 * m] = roots[a];
                ref[3 * m + 1] = roots[b];
                ref[3 * m + 2] = roots[c];
            }
    const double eps = std::fmax(1e-3 * powi_sq(0.1, n), 1e-14);
    std::vector<int> slots;
    for (int s = 0; s < 343; ++s) {
        int ox = s / 49 - 3, oy = (s / 7) % 7 - 3, oz = s % 7 - 3;
        if (std::max(std::abs(ox), std::max(std::abs(oy), std::abs(oz))) >= 2) slots.push_back(s);
    }
    auto work = [&](size_t lo, size_t hi) {
        std::vector<double> g((size_t)n3 * n3);
        for (size_t si = lo; si < hi; ++si) {
            int s = slots[si];
            double sh[3] = {2.0 * (s / 49 - 3), 2.0 * ((s / 7) % 7 - 3), 2.0 * (s % 7 - 3)};
            for (int m = 0; m < n3; ++m)
                for (int l = 0; l < n3; ++l) {
                    double dx = ref[3 * m] - ref[3 * l] - sh[0];
                    double dy = ref[3 * m + 1] - ref[3 * l + 1] - sh[1];
                    double dz = ref[3 * m + 2] - ref[3 * l + 2] - sh[2];
                    double r = std::sqrt(dx * dx + dy * dy + dz * dz);
                    g[(size_t)m * n3 + l] = r > 0.0 ? 1.0 / r : 0.0;
                }
            double* dst = &t.K[(size_t)s * n3 * n3];
            if (mode == GPX_M2L_EXACT) {
                std::copy(g.begin(), g.end(), dst);
                t.rank[s] = n3;
            } else {
                qr_truncate_product(g, n3, eps, dst, &t.rank[s], &t.U[(size_t)s * n3 * n3], &t.Vt[(size_t)s * n3 * n3]);
            }
        }
    };
    unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    size_t per = (slots.size() + nt - 1) / nt;
    for (unsigned i = 0; i < nt; ++i) {
        size_t lo = i * per, hi = std::min(slots.size(), lo + per);
        if (lo < hi) th.emplace_back(work, lo, hi);
    }
    for (auto& x : th) x.join();
}

namespace {

// Eigen-decomposition of a symmetric n x n matrix A (row-major, destroyed) by
// cyclic Jacobi rotations: eigenvalues in w, eigenvectors in the columns of Q.
void jacobi_eigen(std::vector<double>& A, int n, std::vector<double>& w, std::vector<double>& Q) {
    Q.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) Q[(size_t)i * n + i] = 1.0;
    double total = 0.0;
    for (double x : A) total += x * x;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) off += A[(size_t)p * n + q] * A[(size_t)p * n + q];
        if (off <= 1e-30 * total) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[(size_t)p * n + q];
                if (std::fabs(apq) <= 1e-300) continue;
                const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < n; ++k) {  // columns p, q
                    const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = c * akp - sn * akq;
                    A[(size_t)k * n + q] = sn * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {  // rows p, q
                    const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = c * apk - sn * aqk;
                    A[(size_t)q * n + k] = sn * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double qkp = Q[(size_t)k * n + p], qkq = Q[(size_t)k * n + q];
                    Q[(size_t)k * n + p] = c * qkp - sn * qkq;
                    Q[(size_t)k * n + q] = sn * qkp + c * qkq;
                }
            }
    }
    w.resize(n);
    for (int i = 0; i < n; ++i) w[i] = A[(size_t)i * n + i];
}

// The r leading eigenvectors (largest eigenvalues first) of the symmetric
// n x n matrix S, as the columns of an n x r row-major matrix.
std::vector<double> leading_eigenvectors(std::vector<double> S, int n, int r) {
    std::vector<double> w, Q;
    jacobi_eigen(S, n, w, Q);
    std::vector<int> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return w[a] > w[b]; });
    std::vector<double> B((size_t)n * r);
    for (int j = 0; j < r; ++j)
        for (int i = 0; i < n; ++i) B[(size_t)i * r + j] = Q[(size_t)i * n + idx[j]];
    return B;
}

}  // namespace

void build_shared_basis(const M2LTable& t, int r, SharedBasis& out) {
    const int n3 = t.n * t.n * t.n;
    out.n = t.n;
    out.mode = t.mode;
    out.r = r;
    std::vector<int> slots;
    for (int s = 0; s < 343; ++s)
        if (t.rank[s] >= 0) slots.push_back(s);
    // Gram sums of all offsets' operators
    std::vector<double> SU((size_t)n3 * n3, 0.0), SV((size_t)n3 * n3, 0.0);
    for (int s : slots) {
        const double* K = &t.K[(size_t)s * n3 * n3];
        for (int a = 0; a < n3; ++a)
            for (int b = 0; b < n3; ++b) {
                double u = 0.0, v = 0.0;
                for (int k = 0; k < n3; ++k) {
                    u += K[(size_t)a * n3 + k] * K[(size_t)b * n3 + k];
                    v += K[(size_t)k * n3 + a] * K[(size_t)k * n3 + b];
                }
                SU[(size_t)a * n3 + b] += u;
                SV[(size_t)a * n3 + b] += v;
            }
    }
    out.U = leading_eigenvectors(SU, n3, r);
    out.V = leading_eigenvectors(SV, n3, r);
    out.C.assign((size_t)343 * r * r, 0.0);
    double worst = 0.0;
    std::vector<double> KV((size_t)n3 * r), UC((size_t)n3 * r);
    for (int s : slots) {
        const double* K = &t.K[(size_t)s * n3 * n3];
        for (int a = 0; a < n3; ++a)
            for (int j = 0; j < r; ++j) {
                double acc = 0.0;
                for (int k = 0; k < n3; ++k) acc += K[(size_t)a * n3 + k] * out.V[(size_t)k * r + j];
                KV[(size_t)a * r + j] = acc;
            }
        double* C = &out.C[(size_t)s * r * r];
        for (int i = 0; i < r; ++i)
            for (int j = 0; j < r; ++j) {
                double acc = 0.0;
                for (int a = 0; a < n3; ++a) acc += out.U[(size_t)a * r + i] * KV[(size_t)a * r + j];
                C[(size_t)i * r + j] = acc;
            }
        // relative Frobenius error of (U C) V^T against K
        std::fill(UC.begin(), UC.end(), 0.0);
        for (int a = 0; a < n3; ++a)
            for (int i = 0; i < r; ++i) {
                const double u = out.U[(size_t)a * r + i];
                for (int j = 0; j < r; ++j) UC[(size_t)a * r + j] += u * C[(size_t)i * r + j];
            }
        double num = 0.0, den = 0.0;
        for (int a = 0; a < n3; ++a)
            for (int b = 0; b < n3; ++b) {
                double acc = 0.0;
                for (int j = 0; j < r; ++j) acc += UC[(size_t)a * r + j] * out.V[(size_t)b * r + j];
                const double k = K[(size_t)a * n3 + b];
                num += (k - acc) * (k - acc);
                den += k * k;
            }
        worst = std::max(worst, std::sqrt(num / std::max(den, 1e-300)));
    }
    out.rel_err = worst;
}

void build_plan(Plan& p, int64_t N, const double* verts, const int32_t* cond, int ncond, int order, int depth) {
    p.n = order;
    p.n3 = order * order * order;
    p.L = depth;
    p.N = N;
    p.ncond = ncond;
    p.far = depth >= 2;
    // centroids / areas in caller order
    // scratch of this thread, kept between calls (no fresh pages per solve)
    thread_local std::vector<double> c0, a0;
    c0.resize((size_t)N * 3);
    a0.resize((size_t)N);
    // the helper threads see this thread's scratch through plain pointers (a
    // thread_local named inside them would be their own, empty, instance)
    double* const cen = c0.data();
    double* const are = a0.data();
    // cubic bounding box (fmm/tree.rs:43-62), per chunk then combined (the
    // extremes of finite values do not depend on the order)
    constexpr int64_t kChunk = 8192;
    double clo[kMaxChunks][3], chi[kMaxChunks][3];
    const int nch = parallel_chunks(N, kChunk, [&](int t, int64_t b, int64_t e) {
        double l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int64_t i = b; i < e; ++i) {
            panel_centroid_area(verts + 12 * i, &cen[3 * i], &are[i]);
            for (int d = 0; d < 3; ++d) {
                l[d] = std::fmin(l[d], cen[3 * i + d]);
                h[d] = std::fmax(h[d], cen[3 * i + d]);
            }
        }
        for (int d = 0; d < 3; ++d) {
            clo[t][d] = l[d];
            chi[t][d] = h[d];
        }
    });
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int t = 0; t < nch; ++t)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::fmin(lo[d], clo[t][d]);
            hi[d] = std::fmax(hi[d], chi[t][d]);
        }
    double half = 0.0, center[3];
    for (int d = 0; d < 3; ++d) {
        center[d] = 0.5 * (lo[d] + hi[d]);
        half = std::fmax(half, 0.5 * (hi[d] - lo[d]));
    }
    half *= 1.0 + 1e-6;
    if (half == 0.0) half = 1.0;
    const uint32_t ncell = 1u << depth;
    const double leaf_size = 2.0 * half / (double)ncell;
    const double origin[3] = {center[0] - half, center[1] - half, center[2] - half};
    for (int dd = 0; dd < 3; ++dd) p.origin[dd] = origin[dd];
    // leaf cell per panel (fmm/tree.rs:86-95)
    thread_local std::vector<uint32_t> cell;
    thread_local std::vector<uint64_t> key;
    cell.resize((size_t)N * 3);
    key.resize((size_t)N);
    uint32_t* const cel = cell.data();
    uint64_t* const kys = key.data();
    parallel_chunks(N, kChunk, [&](int, int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            for (int d = 0; d < 3; ++d) {
                long long idx = (long long)std::floor((cen[3 * i + d] - origin[d]) / leaf_size);
                idx = std::max(0ll, std::min((long long)ncell - 1, idx));
                cel[3 * i + d] = (uint32_t)idx;
            }
            kys[i] = morton(cel[3 * i], cel[3 * i + 1], cel[3 * i + 2]);
        }
    });
    // leaf order: stable by key.  Up to depth 12 the key takes 36 bits, so
    // (key << 28 | caller index) sorts plainly into the same order (a merge
    // sort: bridge panels arrive in long runs of rising keys).
    p.perm.resize(N);
    if (depth <= 12 && N < (int64_t(1) << 28)) {
        thread_local std::vector<uint64_t> packed;
        packed.resize((size_t)N);
        for (int64_t i = 0; i < N; ++i) packed[i] = key[i] << 28 | (uint64_t)i;
        std::stable_sort(packed.begin(), packed.end());
        for (int64_t s = 0; s < N; ++s) p.perm[s] = (int32_t)(packed[s] & ((uint64_t(1) << 28) - 1));
    } else {
        std::iota(p.perm.begin(), p.perm.end(), 0);
        std::stable_sort(p.perm.begin(), p.perm.end(), [&](int32_t a, int32_t b) { return key[a] < key[b]; });
    }
    p.verts.resize((size_t)N * 12);
    p.cent.resize((size_t)N * 3);
    p.area.resize(N);
    p.cond.resize(N);
    parallel_chunks(N, kChunk, [&](int, int64_t b, int64_t e) {
        for (int64_t s = b; s < e; ++s) {
            int64_t i = p.perm[s];
            std::copy(verts + 12 * i, verts + 12 * i + 12, &p.verts[12 * s]);
            std::copy(&cen[3 * i], &cen[3 * i] + 3, &p.cent[3 * s]);
            p.area[s] = are[i];
            p.cond[s] = cond ? cond[i] : 0;
        }
    });
    // levels: leaf boxes in Morton order, then parents
    std::vector<std::vector<std::array<uint32_t, 3>>> cells(depth + 1);
    p.leaf_begin.clear();
    for (int64_t s = 0; s < N; ++s) {
        int64_t i = p.perm[s];
        std::array<uint32_t, 3> c = {cell[3 * i], cell[3 * i + 1], cell[3 * i + 2]};
        if (cells[depth].empty() || cells[depth].back() != c) {
            cells[depth].push_back(c);
            p.leaf_begin.push_back(s);
        }
    }
    p.leaf_begin.push_back(N);
    p.max_leaf = 0;
    for (size_t k = 0; k + 1 < p.leaf_begin.size(); ++k)
        p.max_leaf = std::max<int32_t>(p.max_leaf, (int32_t)(p.leaf_begin[k + 1] - p.leaf_begin[k]));
    for (int l = depth - 1; l >= 0; --l)
        for (auto& c : cells[l + 1]) {
            std::array<uint32_t, 3> pc = {c[0] / 2, c[1] / 2, c[2] / 2};
            if (cells[l].empty() || cells[l].back() != pc) cells[l].push_back(pc);
        }
    p.lvl_off.assign(depth + 2, 0);
    for (int l = 0; l <= depth; ++l) p.lvl_off[l + 1] = p.lvl_off[l] + (int32_t)cells[l].size();
    const int64_t nb = p.lvl_off[depth + 1];
    p.box_cell.resize(nb * 3);
    p.box_parent.assign(nb, -1);
    p.box_octant.assign(nb, 0);
    p.lvl_half.resize(depth + 1);
    std::vector<std::unordered_map<uint64_t, int32_t>> idx(depth + 1);
    for (int l = 0; l <= depth; ++l) {
        p.lvl_half[l] = half / (double)(1u << l);
        for (size_t k = 0; k < cells[l].size(); ++k) {
            int32_t b = p.lvl_off[l] + (int32_t)k;
            for (int d = 0; d < 3; ++d) p.box_cell[3 * b + d] = (int32_t)cells[l][k][d];
            idx[l][cell_key(cells[l][k][0], cells[l][k][1], cells[l][k][2])] = b;
        }
    }
    p.child_first.assign(nb, 0);
    p.child_count.assign(nb, 0);
    for (int l = 1; l <= depth; ++l)
        for (int32_t b = p.lvl_off[l]; b < p.lvl_off[l + 1]; ++b) {
            const int32_t* c = &p.box_cell[3 * b];
            const int32_t par = idx[l - 1].at(cell_key(c[0] / 2, c[1] / 2, c[2] / 2));
            p.box_parent[b] = par;
            p.box_octant[b] = (c[0] & 1) + 2 * (c[1] & 1) + 4 * (c[2] & 1);
            if (p.child_count[par] == 0) p.child_first[par] = b;
            p.child_count[par] += 1;
        }
    p.leaf_of.resize(N);
    for (int64_t k = 0; k + 1 < (int64_t)p.leaf_begin.size(); ++k)
        for (int64_t s = p.leaf_begin[k]; s < p.leaf_begin[k + 1]; ++s) p.leaf_of[s] = (int32_t)k;
    // 1-D Chebyshev weights of each panel in its leaf (bbfmm.rs:53-59).
    std::vector<double> roots = cheb_roots(order);
    const std::vector<double> troots = cheb_root_table(order, roots.data());
    p.w1d.resize((size_t)N * 3 * order);
    const double hl = p.lvl_half[depth];
    parallel_chunks(N, kChunk, [&](int, int64_t b, int64_t e) {
        for (int64_t s = b; s < e; ++s) {
            const int32_t bx = p.lvl_off[depth] + p.leaf_of[s];
            for (int d = 0; d < 3; ++d) {
                const double ctr = origin[d] + ((double)p.box_cell[3 * bx + d] + 0.5) * 2.0 * hl;
                cheb_weights_tab((p.cent[3 * s + d] - ctr) / hl, order, troots.data(), &p.w1d[(s * 3 + d) * order]);
            }
        }
    });
    // near blocks: self leaf first, then neighbours in dx,dy,dz order
    const int64_t nl = p.nleaf();
    p.near_off.assign(nl + 1, 0);
    p.near_src.clear();
    p.near_S.assign(nl, 0);
    p.nval_off.assign(nl + 1, 0);
    p.max_S = 0;
    const int64_t ncl = 1ll << depth;
    for (int64_t k = 0; k < nl; ++k) {
        int32_t b = p.lvl_off[depth] + (int32_t)k;
        const int32_t* c = &p.box_cell[3 * b];
        p.near_src.push_back((int32_t)k);
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    if (!dx && !dy && !dz) continue;
                    int64_t x = c[0] + dx, y = c[1] + dy, z = c[2] + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= ncl || y >= ncl || z >= ncl) continue;
                    auto it = idx[depth].find(cell_key(x, y, z));
                    if (it != idx[depth].end()) p.near_src.push_back(it->second - p.lvl_off[depth]);
                }
        p.near_off[k + 1] = (int32_t)p.near_src.size();
        int64_t S = 0;
        for (int32_t e = p.near_off[k]; e < p.near_off[k + 1]; ++e)
            S += p.leaf_begin[p.near_src[e] + 1] - p.leaf_begin[p.near_src[e]];
        p.near_S[k] = (int32_t)S;
        p.max_S = std::max<int32_t>(p.max_S, (int32_t)S);
        // rows are stored with a stride padded to 4 entries (16-byte aligned rows)
        p.nval_off[k + 1] = p.nval_off[k] + (p.leaf_begin[k + 1] - p.leaf_begin[k]) * ((S + 3) & ~int64_t(3));
    }
    p.item_leaf.clear();
    p.item_row0.clear();
    for (int64_t k = 0; k < nl; ++k)
        for (int64_t r = 0; r < p.leaf_begin[k + 1] - p.leaf_begin[k]; r += Plan::kRowsPerItem) {
            p.item_leaf.push_back((int32_t)k);
            p.item_row0.push_back((int32_t)r);
        }
    // interaction lists (fmm/tree.rs:188-209): children of the parent's
    // neighbourhood that are not neighbours of the box.
    // Boxes of level >= 2 are visited parent by parent: the parent's
    // existing neighbours are looked up once, and each neighbour's children
    // are taken by octant from its contiguous child range.
    p.m2l_off.assign(nb + 1, 0);
    p.m2l_src.clear();
    p.m2l_slot.clear();
    const int64_t first2 = depth >= 2 ? p.lvl_off[2] : nb;
    for (int64_t b = 0; b < first2; ++b) p.m2l_off[b + 1] = 0;
    int64_t next = first2;
    for (int l = 2; l <= depth; ++l) {
        const int64_t npc = 1ll << (l - 1);
        for (int32_t pb = p.lvl_off[l - 1]; pb < p.lvl_off[l]; ++pb) {
            const int32_t* pcell = &p.box_cell[3 * pb];
            int32_t nbr_child[27][8];
            int nn = 0;
            for (int dx = -1; dx <= 1; ++dx)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dz = -1; dz <= 1; ++dz) {
                        int64_t q[3] = {pcell[0] + dx, pcell[1] + dy, pcell[2] + dz};
                        if (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[0] >= npc || q[1] >= npc || q[2] >= npc) continue;
                        auto it = idx[l - 1].find(cell_key(q[0], q[1], q[2]));
                        if (it == idx[l - 1].end()) continue;
                        int32_t* slot = nbr_child[nn++];
                        for (int o = 0; o < 8; ++o) slot[o] = -1;
                        const int32_t qb = it->second;
                        for (int32_t ch = p.child_first[qb]; ch < p.child_first[qb] + p.child_count[qb]; ++ch)
                            slot[p.box_octant[ch]] = ch;
                    }
            for (int32_t b = p.child_first[pb]; b < p.child_first[pb] + p.child_count[pb]; ++b) {
                if (b != next) throw Error(GPX_ERR_INTERNAL, "octree children out of order");
                const int32_t* c = &p.box_cell[3 * b];
                for (int k = 0; k < nn; ++k)
                    for (int o = 0; o < 8; ++o) {
                        const int32_t src = nbr_child[k][o];
                        if (src < 0) continue;
                        const int32_t* ch = &p.box_cell[3 * src];
                        int64_t ox = ch[0] - c[0], oy = ch[1] - c[1], oz = ch[2] - c[2];
                        if (std::max(std::llabs(ox), std::max(std::llabs(oy), std::llabs(oz))) <= 1) continue;
                        p.m2l_src.push_back(src);
                        p.m2l_slot.push_back((int32_t)(((ox + 3) * 7 + oy + 3) * 7 + oz + 3));
                    }
                p.m2l_off[b + 1] = (int64_t)p.m2l_src.size();
                ++next;
            }
        }
    }
    if (next != nb) throw Error(GPX_ERR_INTERNAL, "octree boxes without a parent");
    // tensor-product M2M operators (bbfmm.rs:89-112)
    p.m2m1d.assign((size_t)24 * order * order, 0.0);
    std::vector<double> w(order);
    for (int o = 0; o < 8; ++o) {
        const int ob[3] = {o & 1, (o >> 1) & 1, (o >> 2) & 1};
        for (int axis = 0; axis < 3; ++axis) {
            const double cc = (2.0 * ob[axis] - 1.0) * 0.5;
            for (int k = 0; k < order; ++k) {
                cheb_weights(cc + 0.5 * roots[k], order, roots.data(), w.data());
                for (int m = 0; m < order; ++m) p.m2m1d[((size_t)(o * 3 + axis) * order + m) * order + k] = w[m];
            }
        }
    }
}

}  // namespace gpx
