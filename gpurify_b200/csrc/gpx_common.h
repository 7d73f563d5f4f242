// Shared internals of the gpx-pex library: error handling, device buffers,
// the context, and the host-side problem description the kernels consume.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <mutex>
#include <utility>

#include <cstdint>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/gpx_pex.h"

namespace gpx {

// Vacuum permittivity and Coulomb constant (quasistatic/constants.rs:13,20).
constexpr double kPi = 3.14159265358979323846;
constexpr double kEps0 = 8.854187812800e-12;
constexpr double kCoulomb = 1.0 / (4.0 * kPi * kEps0);

// Error carried from the point of failure to the C ABI.
struct Error : std::runtime_error {
    gpx_status status;
    uint32_t polygon;
    Error(gpx_status s, const std::string& m, uint32_t poly = 0xFFFFFFFFu)
        : std::runtime_error(m), status(s), polygon(poly) {}
};

#define GPX_CUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            throw ::gpx::Error(e_ == cudaErrorMemoryAllocation ? GPX_ERR_OUT_OF_MEMORY        \
                                                               : GPX_ERR_CUDA,                \
                               std::string(#call) + ": " + cudaGetErrorString(e_));           \
    } while (0)

// Host<->device bytes copied by the library on the calling thread (a call's
// copies all happen on the thread that made it, so a per-thread count gives
// each call's own bytes even while other threads solve concurrently).
inline int64_t& h2d_counter() {
    static thread_local int64_t c = 0;
    return c;
}
inline int64_t& d2h_counter() {
    static thread_local int64_t c = 0;
    return c;
}

// Stream-ordered device buffer (cudaMallocAsync pool of the context stream).
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p; n = o.n; s = o.s;
            o.p = nullptr; o.n = 0;
        }
        return *this;
    }
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count, cudaStream_t stream) {
        if (count == n && p) return;
        release();
        s = stream;
        n = count;
        if (count) GPX_CUDA(cudaMallocAsync((void**)&p, count * sizeof(T), stream));
    }
    void zero() {
        if (n) GPX_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    }
    void upload(const T* h, size_t count, cudaStream_t stream) {
        alloc(count, stream);
        if (count) GPX_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, stream));
        h2d_counter() += (int64_t)(count * sizeof(T));
    }
    void upload(const std::vector<T>& v, cudaStream_t stream) { upload(v.data(), v.size(), stream); }
    void download(T* h, size_t count) const {
        if (count) GPX_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
        d2h_counter() += (int64_t)(count * sizeof(T));
    }
};

struct DevM2L;  // device M2L operator table, cached per (order, mode)

// An iteration index held in device memory, for kernels replayed by a
// device-side loop: the kernel reads k = *k at run time and offsets a vector
// pointer by (k + add) * stride.  k == nullptr: no offset (host-known index).
struct DevIndex {
    const int32_t* k = nullptr;
    int64_t stride = 0;
    int add = 0;
};
#ifdef __CUDACC__
template <class T>
__device__ __forceinline__ T* dev_offset(T* p, const DevIndex& di) {
    return di.k ? p + (int64_t)(*di.k + di.add) * di.stride : p;
}
#endif

// Kernel classes timed by the optional per-kernel event timer.
// The operator's kernel classes are split by precision: the plain names hold
// the FP32 / TF32 launches of the mixed path's inner operator, the *64 names
// the FP64 launches (the plain path, and the mixed path's refinement
// residuals).
enum KTag {
    K_NEAR_ASSEMBLE = 0, K_NEAR_APPLY, K_P2M, K_M2M, K_M2L, K_L2L, K_L2P, K_GS_DOT, K_GS_AXPY, K_VEC, K_SMALL,
    K_NEAR_APPLY64, K_P2M64, K_M2M64, K_M2L64, K_L2L64, K_L2P64, K_NTAGS
};
// The FP64 class of an operator kernel class.
constexpr int f64_tag(int tag) { return tag >= K_NEAR_APPLY && tag <= K_L2P ? tag + (K_NEAR_APPLY64 - K_NEAR_APPLY) : tag; }
template <class T>
constexpr int prec_tag(int tag) { return sizeof(T) == 8 ? f64_tag(tag) : tag; }

struct KStats {
    int64_t launches = 0;
    double ms = 0.0;
    double bytes = 0.0;  // algorithmic bytes moved (minimum DRAM traffic)
    double flops = 0.0;  // algorithmic flops
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    int64_t launches = 0;  // kernel launches issued by this context
    int sm_count = 148;
    std::vector<std::shared_ptr<DevM2L>> m2l_cache;
    // per-kernel timing (enabled by gpx_ctx_set_profiling)
    bool profile = false;
    // true while a device-side GMRES loop is being captured: operator applies
    // launch their kernels into the capture instead of replaying their own graphs
    bool capturing = false;
    KStats kstats[K_NTAGS];
    struct Pending {
        int tag;
        cudaEvent_t a, b;
        double bytes, flops;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    cudaEvent_t take_event() {
        if (!event_pool.empty()) {
            cudaEvent_t e = event_pool.back();
            event_pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    // Fold recorded event pairs into kstats (synchronises on the last event).
    void drain() {
        for (auto& p : pending) {
            float ms = 0.f;
            cudaEventSynchronize(p.b);
            cudaEventElapsedTime(&ms, p.a, p.b);
            KStats& k = kstats[p.tag];
            k.launches += 1;
            k.ms += ms;
            k.bytes += p.bytes;
            k.flops += p.flops;
            event_pool.push_back(p.a);
            event_pool.push_back(p.b);
        }
        pending.clear();
    }
    ~Ctx() {
        for (auto e : event_pool) cudaEventDestroy(e);
        for (auto& p : pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
    }
};

// RAII bracket around one kernel launch: records an event pair on the
// context stream when profiling is on, with the launch's algorithmic work.
struct KTimer {
    Ctx& c;
    int tag;
    double bytes, flops;
    cudaEvent_t a = nullptr;
    KTimer(Ctx& ctx, int t, double by = 0.0, double fl = 0.0) : c(ctx), tag(t), bytes(by), flops(fl) {
        if (c.profile) {
            a = c.take_event();
            cudaEventRecord(a, c.stream);
        }
    }
    ~KTimer() {
        if (a) {
            cudaEvent_t b = c.take_event();
            cudaEventRecord(b, c.stream);
            c.pending.push_back({tag, a, b, bytes, flops});
        }
    }
};

inline void count_launch(Ctx& c, int k = 1) { c.launches += k; }

// Raises a kernel's dynamic shared-memory limit on the current device, once
// per (kernel, device, size) in the process: the attribute call is a host
// API call that must not run while a stream is being captured into a graph,
// so launches inside a capture find it already set.
template <class K>
inline void set_smem_once(K* kernel, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> done;
    int dev = 0;
    GPX_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    int& have = done[{reinterpret_cast<const void*>(kernel), dev}];
    if (have >= bytes) return;
    GPX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    have = bytes;
}

#define GPX_LAUNCH_CHECK() GPX_CUDA(cudaGetLastError())

}  // namespace gpx

struct gpx_ctx {
    gpx::Ctx impl;
};
