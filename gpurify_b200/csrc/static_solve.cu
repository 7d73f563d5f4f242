// Maxwell matrix of a small panel problem whose panels already sit in device
// memory, computed without allocating memory: every intermediate lives in one
// file-scope device array of fixed size, g_small_scratch below.
//
// The algorithm is the reference's dense path (cap/solver.rs:100-134):
// assemble the potential-coefficient matrix P (Wilton closed form at panel
// centroids, cap/solver.rs:81-97), LU-factor it with partial pivoting, solve
// one unit-potential right-hand side per conductor (cap/solver.rs:55-63) and
// accumulate C[i][j] = sum over conductor i's panels of sigma * area
// (cap/solver.rs:64-71).  Here the right-hand sides are carried as extra
// columns of the factorised matrix, so the blocked LU leaves L^-1 P_perm B in
// them and only a back substitution with U remains.
//
// Limits: at most kMaxPanels panels and kMaxCond conductors.  Scratch layout
// (doubles, row stride kLd = kMaxPanels + kMaxCond):
//   [0, kMaxPanels * kLd)        augmented system [P | B], factorised in place
//   cen  3 per panel, area 1 per panel
//   piv  kMaxPanels int32 pivot rows
//   status int32 word: bit 0 zero pivot, bit 1 conductor index out of range
// Only the status word has to start at zero; the call clears it itself before
// its first launch.  Every other element the call reads it has written earlier
// in the same call.
#include <cstdint>
#include <mutex>
#include <string>

#include "gpx_common.h"
#include "wilton.cuh"

namespace gpx {

namespace {

constexpr int kMaxPanels = 512;
constexpr int kMaxCond = 64;
constexpr int kLd = kMaxPanels + kMaxCond;
constexpr int kNb = 32;  // LU column-block width
constexpr int kMaxDevices = 64;
constexpr size_t kOffCen = (size_t)kMaxPanels * kLd;
constexpr size_t kOffArea = kOffCen + 3 * kMaxPanels;
constexpr size_t kOffPiv = kOffArea + kMaxPanels;
constexpr size_t kOffStatus = kOffPiv + kMaxPanels / 2;
constexpr size_t kScratchDoubles = kOffStatus + 32;  // 297,248 doubles = 2,377,984 bytes
constexpr int kPanelSmem = kMaxPanels * (kNb + 1) * (int)sizeof(double);
constexpr int kStatusSingular = 1, kStatusBadConductor = 2;

static __device__ __align__(256) double g_small_scratch[kScratchDoubles];

__device__ __forceinline__ int* piv_of(double* S) { return reinterpret_cast<int*>(S + kOffPiv); }
__device__ __forceinline__ int* status_of(double* S) { return reinterpret_cast<int*>(S + kOffStatus); }

// Centroid and area (area-weighted triangle fan, integrals/panel.rs:29-67) of
// each panel, and row i of the right-hand sides: B[i][j] = 1 if panel i lies
// on conductor j.
__global__ void k_small_setup(double* __restrict__ S, const double* __restrict__ verts,
                              const int32_t* __restrict__ cond, int n, int ncond) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double q[4][3];
    for (int k = 0; k < 4; ++k)
        for (int d = 0; d < 3; ++d) q[k][d] = verts[12 * (int64_t)i + 3 * k + d];
    const int nv = (q[3][0] == q[2][0] && q[3][1] == q[2][1] && q[3][2] == q[2][2]) ? 3 : 4;
    double asum = 0.0, acc[3] = {0.0, 0.0, 0.0};
    for (int k = 1; k < nv - 1; ++k) {
        const double a[3] = {q[k][0] - q[0][0], q[k][1] - q[0][1], q[k][2] - q[0][2]};
        const double b[3] = {q[k + 1][0] - q[0][0], q[k + 1][1] - q[0][1], q[k + 1][2] - q[0][2]};
        const double c[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
        const double t = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]) * 0.5;
        for (int d = 0; d < 3; ++d) acc[d] += (q[0][d] + q[k][d] + q[k + 1][d]) * (1.0 / 3.0) * t;
        asum += t;
    }
    for (int d = 0; d < 3; ++d) S[kOffCen + 3 * i + d] = asum == 0.0 ? q[0][d] : acc[d] * (1.0 / asum);
    S[kOffArea + i] = asum;
    const int ci = cond[i];
    if (ci < 0 || ci >= ncond) atomicOr(status_of(S), kStatusBadConductor);
    double* row = S + (size_t)i * kLd + kMaxPanels;
    for (int j = 0; j < ncond; ++j) row[j] = j == ci ? 1.0 : 0.0;
}

// P[t][s] = coef * Wilton integral of source panel s at the centroid of t.
// Thread per source panel, 32 targets per CTA row.
__global__ void __launch_bounds__(128) k_small_assemble(double* __restrict__ S, const double* __restrict__ verts,
                                                        int n, double coef) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int t0 = blockIdx.y * 32;
    if (s >= n) return;
    SrcPanel sp;
    prep_source(verts + 12 * (int64_t)s, sp);
    const double* cen = S + kOffCen;
    const int t1 = min(n, t0 + 32);
    for (int t = t0; t < t1; ++t) S[(size_t)t * kLd + s] = coef * wilton(sp, cen[3 * t], cen[3 * t + 1], cen[3 * t + 2]);
}

// Unblocked LU with partial pivoting of the column panel rows [k0, n) x
// columns [k0, k0 + w), held in shared memory; one thread per panel row.
// Records the pivot row of each column in piv[k0 + c] (absolute row index).
__global__ void __launch_bounds__(kMaxPanels) k_small_panel(double* __restrict__ S, int n, int k0, int w) {
    constexpr int PW = kNb + 1;
    extern __shared__ double ps[];  // [m][PW]
    __shared__ double wbest[kMaxPanels / 32];
    __shared__ int wrow[kMaxPanels / 32];
    __shared__ int prow;
    const int m = n - k0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
    for (int e = tid; e < m * w; e += blockDim.x) ps[(e / w) * PW + e % w] = S[(size_t)(k0 + e / w) * kLd + k0 + e % w];
    for (int c = 0; c < w; ++c) {
        __syncthreads();
        double best = -1.0;
        int bi = c;
        for (int r = c + tid; r < m; r += blockDim.x) {
            const double a = fabs(ps[r * PW + c]);
            if (a > best) {
                best = a;
                bi = r;
            }
        }
        for (int off = 16; off > 0; off >>= 1) {
            const double ob = __shfl_down_sync(0xffffffffu, best, off);
            const int oi = __shfl_down_sync(0xffffffffu, bi, off);
            if (ob > best || (ob == best && oi < bi)) {
                best = ob;
                bi = oi;
            }
        }
        if (lane == 0) {
            wbest[warp] = best;
            wrow[warp] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            double b = wbest[0];
            int r = wrow[0];
            for (int k = 1; k < nwarp; ++k)
                if (wbest[k] > b || (wbest[k] == b && wrow[k] < r)) {
                    b = wbest[k];
                    r = wrow[k];
                }
            if (!(b > 0.0)) atomicOr(status_of(S), kStatusSingular);
            prow = r;
            piv_of(S)[k0 + c] = k0 + r;
        }
        __syncthreads();
        const int p = prow;
        if (p != c)
            for (int j = tid; j < w; j += blockDim.x) {
                const double t = ps[c * PW + j];
                ps[c * PW + j] = ps[p * PW + j];
                ps[p * PW + j] = t;
            }
        __syncthreads();
        const double d = ps[c * PW + c];
        const double inv = d != 0.0 ? 1.0 / d : 0.0;
        for (int r = c + 1 + tid; r < m; r += blockDim.x) {
            const double l = ps[r * PW + c] * inv;
            ps[r * PW + c] = l;
            for (int j = c + 1; j < w; ++j) ps[r * PW + j] -= l * ps[c * PW + j];
        }
    }
    __syncthreads();
    for (int e = tid; e < m * w; e += blockDim.x) S[(size_t)(k0 + e / w) * kLd + k0 + e % w] = ps[(e / w) * PW + e % w];
}

// Column q of the columns right of the panel: P columns [c0, c0 + nq1), then
// the right-hand-side columns.
__device__ __forceinline__ int right_col(int q, int c0, int nq1) {
    return q < nq1 ? c0 + q : kMaxPanels + (q - nq1);
}

// For each column right of the panel: apply the panel's row interchanges,
// then U12 = L11^-1 A12 (L11 unit lower triangular); thread per column.
__global__ void __launch_bounds__(128) k_small_swap_trsm(double* __restrict__ S, int n, int ncond, int k0, int w) {
    __shared__ double Ls[kNb][kNb + 1];
    for (int e = threadIdx.x; e < kNb * kNb; e += blockDim.x) {
        const int r = e / kNb, c = e % kNb;
        Ls[r][c] = (r < w && c < w) ? S[(size_t)(k0 + r) * kLd + k0 + c] : 0.0;
    }
    __syncthreads();
    const int nq1 = n - k0 - w;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq1 + ncond) return;
    const int j = right_col(q, k0 + w, nq1);
    const int* piv = piv_of(S);
    for (int c = 0; c < w; ++c) {
        const int p = piv[k0 + c];
        if (p != k0 + c) {
            double* a = S + (size_t)(k0 + c) * kLd + j;
            double* b = S + (size_t)p * kLd + j;
            const double t = *a;
            *a = *b;
            *b = t;
        }
    }
    double x[kNb];
#pragma unroll
    for (int r = 0; r < kNb; ++r) x[r] = r < w ? S[(size_t)(k0 + r) * kLd + j] : 0.0;
#pragma unroll
    for (int r = 1; r < kNb; ++r) {
        double a = x[r];
#pragma unroll
        for (int c = 0; c < r; ++c) a -= Ls[r][c] * x[c];
        x[r] = a;
    }
#pragma unroll
    for (int r = 0; r < kNb; ++r)
        if (r < w) S[(size_t)(k0 + r) * kLd + j] = x[r];
}

// C -= A B on 64 x 64 tiles with a contraction of w <= kNb:
//   rows i in [r0, r0 + nr), columns right_col(q, c0, nq1) for q < nq,
//   A[i][kc0 + c], B[kr0 + c][col].  The three regions never overlap.
__global__ void __launch_bounds__(256) k_small_gemm(double* __restrict__ S, int r0, int nr, int kc0, int kr0, int w,
                                                    int c0, int nq1, int nq) {
    __shared__ double As[kNb][65];  // [c][i]
    __shared__ double Bs[kNb][65];  // [c][q]
    const int i0 = blockIdx.y * 64, q0 = blockIdx.x * 64;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    for (int e = tid; e < kNb * 64; e += 256) {
        const int ii = e / kNb, c = e % kNb;
        As[c][ii] = (i0 + ii < nr && c < w) ? S[(size_t)(r0 + i0 + ii) * kLd + kc0 + c] : 0.0;
    }
    for (int e = tid; e < kNb * 64; e += 256) {
        const int c = e / 64, qq = e % 64;
        Bs[c][qq] = (q0 + qq < nq && c < w) ? S[(size_t)(kr0 + c) * kLd + right_col(q0 + qq, c0, nq1)] : 0.0;
    }
    __syncthreads();
    double acc[4][4] = {};
#pragma unroll 8
    for (int c = 0; c < kNb; ++c) {
        double a[4], b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) a[u] = As[c][ty + 16 * u];
#pragma unroll
        for (int v = 0; v < 4; ++v) b[v] = Bs[c][tx + 16 * v];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] += a[u] * b[v];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int ii = i0 + ty + 16 * u;
        if (ii >= nr) continue;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int qq = q0 + tx + 16 * v;
            if (qq < nq) S[(size_t)(r0 + ii) * kLd + right_col(qq, c0, nq1)] -= acc[u][v];
        }
    }
}

// Back substitution with the diagonal block U11 (rows/columns [k0, k0 + w))
// on every right-hand-side column; thread per column.
__global__ void __launch_bounds__(kMaxCond) k_small_diag_back(double* __restrict__ S, int ncond, int k0, int w) {
    __shared__ double Us[kNb][kNb + 1];
    for (int e = threadIdx.x; e < kNb * kNb; e += blockDim.x) {
        const int r = e / kNb, c = e % kNb;
        Us[r][c] = (r < w && c < w) ? S[(size_t)(k0 + r) * kLd + k0 + c] : 0.0;
    }
    __syncthreads();
    if ((int)threadIdx.x >= ncond) return;
    const int j = kMaxPanels + threadIdx.x;
    double x[kNb];
#pragma unroll
    for (int r = 0; r < kNb; ++r) x[r] = r < w ? S[(size_t)(k0 + r) * kLd + j] : 0.0;
#pragma unroll
    for (int r = kNb - 1; r >= 0; --r) {
        if (r >= w) continue;
        double a = x[r];
#pragma unroll
        for (int c = r + 1; c < kNb; ++c) a -= Us[r][c] * x[c];  // Us[r][c] = 0 for c >= w
        const double d = Us[r][r];
        x[r] = d != 0.0 ? a / d : 0.0;
    }
#pragma unroll
    for (int r = 0; r < kNb; ++r)
        if (r < w) S[(size_t)(k0 + r) * kLd + j] = x[r];
}

// C[i][j] = sum over panels k of conductor i of sigma_j[k] * area[k], panels
// in ascending order (cap/solver.rs:64-71).
__global__ void k_small_maxwell(double* __restrict__ S, const int32_t* __restrict__ cond, int n, int ncond,
                                double* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ncond * ncond) return;
    const int i = e / ncond, j = e % ncond;
    const double* area = S + kOffArea;
    double acc = 0.0;
    for (int k = 0; k < n; ++k)
        if (cond[k] == i) acc += S[(size_t)k * kLd + kMaxPanels + j] * area[k];
    out[e] = acc;
}

std::mutex g_small_mu[kMaxDevices];
double* g_small_ptr[kMaxDevices] = {};

// Device address of this device's scratch array.  The first call on a device
// (made with that device current and its lock held) looks the address up,
// loads every kernel this entry point launches and raises the panel kernel's
// dynamic shared-memory limit.  With CUDA's lazy module loading a kernel is
// otherwise loaded, and its device memory taken, on its first launch: a later
// call that reaches a kernel the earlier calls did not (k_small_gemm runs
// only above 32 panels) would then allocate.  Querying each kernel's
// attributes here loads them all up front.
double* small_scratch(int dev) {
    if (!g_small_ptr[dev]) {
        void* p = nullptr;
        GPX_CUDA(cudaGetSymbolAddress(&p, g_small_scratch));
        const void* kernels[] = {(const void*)k_small_setup,     (const void*)k_small_assemble,
                                 (const void*)k_small_panel,     (const void*)k_small_swap_trsm,
                                 (const void*)k_small_gemm,      (const void*)k_small_diag_back,
                                 (const void*)k_small_maxwell};
        for (const void* k : kernels) {
            cudaFuncAttributes fa{};
            GPX_CUDA(cudaFuncGetAttributes(&fa, k));
        }
        GPX_CUDA(cudaFuncSetAttribute(k_small_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPanelSmem));
        g_small_ptr[dev] = static_cast<double*>(p);
    }
    return g_small_ptr[dev];
}

// Rejects a pointer that is not device or managed memory usable on `dev`, or
// that is misaligned for its element type.
void check_device_ptr(const void* p, size_t align, int dev, const char* what) {
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(GPX_ERR_INVALID_ARG, std::string(what) + " is not a CUDA pointer");
    }
    const bool ok = (a.type == cudaMemoryTypeDevice && a.device == dev) || a.type == cudaMemoryTypeManaged;
    if (!ok)
        throw Error(GPX_ERR_INVALID_ARG,
                    std::string(what) + " must be device (or managed) memory of the context's device");
    if (reinterpret_cast<uintptr_t>(p) % align != 0)
        throw Error(GPX_ERR_INVALID_ARG, std::string(what) + " is misaligned");
}

inline unsigned cdiv(int a, int b) { return (unsigned)((a + b - 1) / b); }

void small_solve(Ctx& c, int64_t n_panels, const double* verts, const int32_t* cond, int ncond, double* out) {
    if (n_panels < 1 || n_panels > kMaxPanels)
        throw Error(GPX_ERR_INVALID_ARG, "n_panels = " + std::to_string(n_panels) +
                                             " is outside [1, 512], the static-scratch limit; use gpx_cap_solve");
    const int n = (int)n_panels;
    if (ncond < 1 || ncond > kMaxCond)
        throw Error(GPX_ERR_INVALID_ARG, "n_conductors = " + std::to_string(ncond) +
                                             " is outside [1, 64], the static-scratch limit; use gpx_cap_solve");
    if (!verts || !cond || !out) throw Error(GPX_ERR_INVALID_ARG, "null pointer");
    const int dev = c.device;
    if (dev < 0 || dev >= kMaxDevices) throw Error(GPX_ERR_INVALID_ARG, "device index above 63");
    GPX_CUDA(cudaSetDevice(dev));
    check_device_ptr(verts, alignof(double), dev, "d_verts");
    check_device_ptr(cond, alignof(int32_t), dev, "d_conductor");
    check_device_ptr(out, alignof(double), dev, "d_maxwell_out");
    std::lock_guard<std::mutex> lock(g_small_mu[dev]);
    double* S = small_scratch(dev);
    cudaStream_t s = c.stream;
    int* status = reinterpret_cast<int*>(S + kOffStatus);
    GPX_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
    int64_t launches = 0;
    k_small_setup<<<cdiv(n, 128), 128, 0, s>>>(S, verts, cond, n, ncond);
    GPX_LAUNCH_CHECK();
    k_small_assemble<<<dim3(cdiv(n, 128), cdiv(n, 32)), 128, 0, s>>>(S, verts, n, kCoulomb);
    GPX_LAUNCH_CHECK();
    launches += 2;
    for (int k0 = 0; k0 < n; k0 += kNb) {
        const int w = std::min(kNb, n - k0);
        const int m = n - k0;
        k_small_panel<<<1, kMaxPanels, (size_t)m * (kNb + 1) * sizeof(double), s>>>(S, n, k0, w);
        GPX_LAUNCH_CHECK();
        const int nq1 = n - k0 - w, nq = nq1 + ncond;
        k_small_swap_trsm<<<cdiv(nq, 128), 128, 0, s>>>(S, n, ncond, k0, w);
        GPX_LAUNCH_CHECK();
        launches += 2;
        if (nq1 > 0) {
            k_small_gemm<<<dim3(cdiv(nq, 64), cdiv(nq1, 64)), 256, 0, s>>>(S, k0 + w, nq1, k0, k0, w, k0 + w, nq1,
                                                                             nq);
            GPX_LAUNCH_CHECK();
            launches += 1;
        }
    }
    const int nblk = (n + kNb - 1) / kNb;
    for (int b = nblk - 1; b >= 0; --b) {
        const int k0 = b * kNb, w = std::min(kNb, n - k0);
        k_small_diag_back<<<1, kMaxCond, 0, s>>>(S, ncond, k0, w);
        GPX_LAUNCH_CHECK();
        launches += 1;
        if (k0 > 0) {
            k_small_gemm<<<dim3(cdiv(ncond, 64), cdiv(k0, 64)), 256, 0, s>>>(S, 0, k0, k0, k0, w, 0, 0, ncond);
            GPX_LAUNCH_CHECK();
            launches += 1;
        }
    }
    k_small_maxwell<<<cdiv(ncond * ncond, 128), 128, 0, s>>>(S, cond, n, ncond, out);
    GPX_LAUNCH_CHECK();
    launches += 1;
    int hstatus = 0;
    GPX_CUDA(cudaMemcpyAsync(&hstatus, status, sizeof(int), cudaMemcpyDeviceToHost, s));
    GPX_CUDA(cudaStreamSynchronize(s));
    c.launches += launches;
    if (hstatus & kStatusBadConductor)
        throw Error(GPX_ERR_INVALID_ARG, "a conductor index is outside [0, n_conductors)");
    if (hstatus & kStatusSingular) throw Error(GPX_ERR_CAPACITANCE, "singular potential matrix (zero LU pivot)");
}

}  // namespace

}  // namespace gpx

extern "C" gpx_status gpx_cap_solve_small_static(gpx_ctx* ctx, int64_t n_panels, const double* d_verts,
                                                 const int32_t* d_conductor, int32_t n_conductors,
                                                 double* d_maxwell_out) {
    if (!ctx) return GPX_ERR_INVALID_ARG;
    ctx->impl.last_error.clear();
    try {
        gpx::small_solve(ctx->impl, n_panels, d_verts, d_conductor, n_conductors, d_maxwell_out);
        return GPX_OK;
    } catch (const gpx::Error& e) {
        ctx->impl.last_error = e.what();
        return e.status;
    } catch (const std::exception& e) {
        ctx->impl.last_error = e.what();
        return GPX_ERR_INTERNAL;
    } catch (...) {
        ctx->impl.last_error = "unknown error";
        return GPX_ERR_INTERNAL;
    }
}
