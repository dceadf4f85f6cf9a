// sm_common.cuh -- shared device helpers of libseismod_gpu (sm_100a).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "../host/sm_host.h"

#define SM_CUDA_TRY(expr)                                                              \
    do {                                                                               \
        cudaError_t sm_e_ = (expr);                                                    \
        if (sm_e_ != cudaSuccess)                                                      \
            return sm_fail(SM_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #expr,        \
                           cudaGetErrorString(sm_e_));                                 \
    } while (0)

namespace sm {

// ---------------------------------------------------------------------------
// storage types.  A field is held in S and updated in C = Store<S>::C.  16-bit
// types carry one power-of-two scale per field: stored = value * 2^e, so
// load/store multiply by exact powers of two (no rounding beyond the 16-bit
// conversion itself).
// ---------------------------------------------------------------------------
template <typename S>
struct Store;

template <>
struct Store<float> {
    using C = float;
    static __device__ __forceinline__ float ld(const float *p, float) { return *p; }
    static __device__ __forceinline__ void st(float *p, float v, float) { *p = v; }
    static __device__ __forceinline__ float ldg(const float *p, float) { return __ldg(p); }
};

template <>
struct Store<double> {
    using C = double;
    static __device__ __forceinline__ double ld(const double *p, double) { return *p; }
    static __device__ __forceinline__ void st(double *p, double v, double) { *p = v; }
    static __device__ __forceinline__ double ldg(const double *p, double) { return __ldg(p); }
};

// 16-bit: `s` passed to ld is 2^-e (unscale), to st is 2^e (scale)
template <>
struct Store<__half> {
    using C = float;
    static __device__ __forceinline__ float ld(const __half *p, float inv) {
        return __half2float(*p) * inv;
    }
    static __device__ __forceinline__ void st(__half *p, float v, float sc) {
        *p = __float2half_rn(v * sc);
    }
    static __device__ __forceinline__ float ldg(const __half *p, float inv) {
        return __half2float(__ldg(p)) * inv;
    }
};

template <>
struct Store<__nv_bfloat16> {
    using C = float;
    static __device__ __forceinline__ float ld(const __nv_bfloat16 *p, float inv) {
        return __bfloat162float(*p) * inv;
    }
    static __device__ __forceinline__ void st(__nv_bfloat16 *p, float v, float sc) {
        *p = __float2bfloat16_rn(v * sc);
    }
    static __device__ __forceinline__ float ldg(const __nv_bfloat16 *p, float inv) {
        return __bfloat162float(__ldg(p)) * inv;
    }
};

inline size_t storage_bytes(int precision) {
    switch (precision) {
    case SM_FP64: return 8;
    case SM_FP16:
    case SM_BF16: return 2;
    default: return 4;
    }
}

// ---------------------------------------------------------------------------
// owning device buffer
// ---------------------------------------------------------------------------
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    int alloc(size_t n) {
        release();
        if (n == 0) return SM_OK;
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return sm_fail(SM_ENOMEM, "cudaMalloc(%zu bytes) failed: %s", n,
                           cudaGetErrorString(e));
        }
        bytes = n;
        return SM_OK;
    }
    int zero(cudaStream_t s) {
        if (!p) return SM_OK;
        SM_CUDA_TRY(cudaMemsetAsync(p, 0, bytes, s));
        return SM_OK;
    }
    template <typename T>
    T *as() const { return static_cast<T *>(p); }
};

// device scoped switch that restores the caller's current device
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// copy host doubles into a device array of T (converting)
template <typename T>
int upload_convert(void *dst, const double *src, size_t n, cudaStream_t s) {
    std::vector<T> tmp(n);
    for (size_t i = 0; i < n; ++i) tmp[i] = static_cast<T>(src[i]);
    if (cudaMemcpyAsync(dst, tmp.data(), n * sizeof(T), cudaMemcpyHostToDevice, s) !=
        cudaSuccess)
        return sm_fail(SM_ECUDA, "upload failed: %s", cudaGetErrorString(cudaGetLastError()));
    if (cudaStreamSynchronize(s) != cudaSuccess)
        return sm_fail(SM_ECUDA, "upload sync failed: %s",
                       cudaGetErrorString(cudaGetLastError()));
    return SM_OK;
}

inline size_t round_up(size_t a, size_t b) { return (a + b - 1) / b * b; }

// receiver sampling plan shared by both paths: receivers with the same
// (t0, rdt) share one step -> slot table.
struct SamplePlan {
    size_t nsteps_max = 0;
    size_t nrec = 0;
    size_t max_samples = 0;
    std::vector<int32_t> group_of;      // per receiver
    std::vector<int32_t> table;         // ngroups * nsteps_max, slot or -1
    std::vector<size_t> count_total;    // per group: samples over nsteps_max
    int build(size_t n, const double *t0, const double *rdt, double dt, size_t nsteps) {
        nrec = n;
        nsteps_max = nsteps;
        group_of.assign(n, 0);
        table.clear();
        count_total.clear();
        std::vector<std::pair<double, double>> keys;
        for (size_t r = 0; r < n; ++r) {
            int g = -1;
            for (size_t k = 0; k < keys.size(); ++k)
                if (keys[k].first == t0[r] && keys[k].second == rdt[r]) { g = (int)k; break; }
            if (g < 0) {
                g = (int)keys.size();
                keys.emplace_back(t0[r], rdt[r]);
                size_t c = 0;
                for (size_t it = 0; it < nsteps; ++it) {
                    int take = sm_sample_predicate(it, dt, t0[r], rdt[r]);
                    table.push_back(take ? (int32_t)c : -1);
                    if (take) ++c;
                }
                count_total.push_back(c);
            }
            group_of[r] = g;
        }
        max_samples = 0;
        for (size_t c : count_total) max_samples = c > max_samples ? c : max_samples;
        return SM_OK;
    }
};

}  // namespace sm
