// sm_common.cuh -- shared device helpers of libseismod_gpu (sm_100a).
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <type_traits>
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
    case SM_BF16:
    case SM_BFP16: return 2;
    default: return 4;
    }
}

// ---------------------------------------------------------------------------
// 16-bit block floating point (SM_BFP16; no counterpart in the reference).
// A block of values shares one 8-bit exponent byte e8; each value is a
// 16-bit two's-complement mantissa m with value m * 2^(e8 - 126).  The
// encoder takes e8 from the FP32 bits of the block's largest magnitude M,
// so that M maps into [2^14, 2^15) (15 significant bits and a sign for the
// largest value; a block whose M would round up to 2^15 takes the next
// exponent); e8 = 0 is the finest scale, 2^-126, which also stands for a
// block of zeros (the zero fill of an out-of-grid TMA read decodes to 0).
// Arithmetic stays FP32.  Decoding and encoding use the float magic
// constant 1.5 * 2^23, whose ulp is 1: adding it to an integer or rounding
// a product onto it is exact, so no conversion instruction is needed.
// ---------------------------------------------------------------------------
struct Bfp16 {};     // storage tag of the block-floating-point kernels
struct BDec {
    float sc, off;   // value = (1.5 * 2^23 + m) * sc + off
};
__device__ __forceinline__ BDec bfp_dec(unsigned e8) {
    const float sc = __int_as_float((int)((e8 + 1u) << 23));   // 2^(e8 - 126)
    return BDec{sc, __fmul_rn(-12582912.0f, sc)};
}
// m: the mantissa, sign-extended
__device__ __forceinline__ float bfp_val(int m, BDec d) {
    return __fmaf_rn(__int_as_float(m + 0x4B400000), d.sc, d.off);
}
// e8 of a block from the largest |value|'s bits (sign cleared); *over is set
// when the block exceeds the format's range (|value| >= 2^114)
__device__ __forceinline__ unsigned bfp_e8(unsigned mxbits, bool *over) {
    int eb = (int)((mxbits + 0x100u) >> 23);   // the next exponent from M >= 2^E (1 - 2^-16)
    *over = eb > 240;
    eb = eb < 15 ? 15 : (eb > 240 ? 240 : eb);
    return (unsigned)(eb - 15);
}
// 2^(126 - e8): value * scale lies in (-32767.5, 32767.5)
__device__ __forceinline__ float bfp_escale(unsigned e8) {
    return __int_as_float((int)((253u - e8) << 23));
}
// round-half-even mantissa of value * scale (the low 16 bits of the sum)
__device__ __forceinline__ short bfp_man(float v, float esc) {
    return (short)__float_as_int(__fmaf_rn(v, esc, 12582912.0f));
}
__device__ __forceinline__ unsigned bfp_absbits(float v) { return __float_as_uint(v) & 0x7fffffffu; }

// host-side counterparts (the same rules, for field reads and writes)
inline unsigned bfp_e8_host(float mx) {
    unsigned b;
    std::memcpy(&b, &mx, 4);
    b &= 0x7fffffffu;
    int eb = (int)((b + 0x100u) >> 23);
    eb = eb < 15 ? 15 : (eb > 240 ? 240 : eb);
    return (unsigned)(eb - 15);
}
inline double bfp_value_host(int16_t m, unsigned e8) { return std::ldexp((double)m, (int)e8 - 126); }
inline int16_t bfp_man_host(float v, unsigned e8) {
    const float x = std::ldexp(v, 126 - (int)e8);   // exact (power-of-two scale)
    float r = std::nearbyint(x);                     // round half even
    if (r > 32767.f) r = 32767.f;
    if (r < -32768.f) r = -32768.f;
    return (int16_t)r;
}

// ---------------------------------------------------------------------------
// cache of large device blocks and pinned host blocks (sm_pool.cu)
// ---------------------------------------------------------------------------
int pool_get(int device, size_t bytes, void **out);
void pool_put(int device, void *ptr, size_t bytes);
int pinned_get(size_t bytes, void **out);
void pinned_put(void *ptr, size_t bytes);

// pinned host staging block, given back to the cache on scope exit
struct PinnedBuf {
    void *p = nullptr;
    size_t bytes = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf &) = delete;
    PinnedBuf &operator=(const PinnedBuf &) = delete;
    ~PinnedBuf() { pinned_put(p, bytes); }
    int get(size_t n) {
        bytes = n;
        return pinned_get(n, &p);
    }
    template <typename T>
    T *as() const { return static_cast<T *>(p); }
};

// ---------------------------------------------------------------------------
// owning device buffer.  alloc: cudaMalloc / cudaFree.  alloc_pooled: a block
// of the device cache, given back on release, which the owner may only do
// when no work in flight uses it (handle teardown after its streams finished)
// ---------------------------------------------------------------------------
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int pool_dev = -1;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) {
            if (pool_dev >= 0) pool_put(pool_dev, p, bytes);
            else cudaFree(p);
        }
        p = nullptr;
        bytes = 0;
        pool_dev = -1;
    }
    int alloc_pooled(size_t n, int device) {
        release();
        if (n == 0) return SM_OK;
        if (int rc = pool_get(device, n, &p)) return rc;
        bytes = n;
        pool_dev = device;
        return SM_OK;
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

// CUDA-event timing of the update kernel(s) plus launch counters
// begin/end event pairs of the launches timed inside one captured CUDA graph
using EventPairs = std::vector<std::pair<cudaEvent_t, cudaEvent_t>>;

struct KernelTimer {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    EventPairs pending;
    // set while a graph is captured with timing on: begin() and end() then
    // record external event nodes, which every replay of the graph records
    // again, and the pairs go to the graph's list instead of `pending`
    EventPairs *capture = nullptr;
    double ms = 0.0;
    size_t timed = 0;
    size_t launches = 0;        // every kernel this handle launched
    ~KernelTimer() {
        for (auto e : pool) cudaEventDestroy(e);
        for (auto &p : pending) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
    }
    cudaEvent_t get() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    // switch per-launch timing on or off; on: events for n timed launches are
    // created up front, so no event creation falls inside a timed pass
    void set(bool v, size_t n = 512) {
        on = v;
        if (!v) return;
        while (pool.size() < 2 * n) {
            cudaEvent_t e = nullptr;
            if (cudaEventCreate(&e) != cudaSuccess) break;
            pool.push_back(e);
        }
    }
    cudaEvent_t begin(cudaStream_t s) {
        if (!on) return nullptr;
        cudaEvent_t a = get();
        if (capture) cudaEventRecordWithFlags(a, s, cudaEventRecordExternal);
        else cudaEventRecord(a, s);
        return a;
    }
    void end(cudaEvent_t a, cudaStream_t s) {
        if (!a) return;
        cudaEvent_t b = get();
        if (capture) {
            cudaEventRecordWithFlags(b, s, cudaEventRecordExternal);
            capture->emplace_back(a, b);
            return;
        }
        cudaEventRecord(b, s);
        pending.emplace_back(a, b);
        if (pending.size() > 4096) collect();
    }
    // one replay of a graph captured with timing was launched: wait for its
    // last event (the next replay records the same events) and add the
    // durations of its timed launches
    void replayed(const EventPairs &ev) {
        if (ev.empty()) return;
        cudaEventSynchronize(ev.back().second);
        for (auto &p : ev) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, p.first, p.second) != cudaSuccess) continue;
            ms += t;
            ++timed;
        }
    }
    // a timed graph was destroyed: its events back to the pool
    void release(EventPairs &ev) {
        for (auto &p : ev) {
            pool.push_back(p.first);
            pool.push_back(p.second);
        }
        ev.clear();
    }
    void collect() {
        for (auto &p : pending) {
            cudaEventSynchronize(p.second);
            float t = 0.f;
            cudaEventElapsedTime(&t, p.first, p.second);
            ms += t;
            ++timed;
            pool.push_back(p.first);
            pool.push_back(p.second);
        }
        pending.clear();
    }
    int stats(int reset, double *out_ms, size_t *out_timed, size_t *out_all) {
        collect();
        if (out_ms) *out_ms = ms;
        if (out_timed) *out_timed = timed;
        if (out_all) *out_all = launches;
        if (reset) { ms = 0.0; timed = 0; launches = 0; }
        return SM_OK;
    }
};

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

// ---------------------------------------------------------------------------
// arithmetic with fixed rounding: no contraction is left to the compiler, so
// the same formula evaluated in two code paths (a cell and its recomputed
// halo copy) rounds identically, and results do not depend on the launch
// configuration
// ---------------------------------------------------------------------------
__device__ __forceinline__ float r_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float r_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float r_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float r_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
// 2 dt / (a + b): in FP32 the numerator times the hardware's approximate
// reciprocal (PTX rcp.approx.ftz.f32, within 1 ulp; the denominators here are
// sums of densities, far from the denormal and overflow ranges), exact in FP64
__device__ __forceinline__ float r_quot(float num, float den) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(den));
    return __fmul_rn(num, r);
}
__device__ __forceinline__ double r_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double r_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double r_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double r_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double r_quot(double num, double den) { return __ddiv_rn(num, den); }

// ---------------------------------------------------------------------------
// TMA tile loads (cp.async.bulk.tensor, no multicast) completing on an
// mbarrier, and bounded waits on it
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// hint: bring the line holding p into L2 (p must be a valid global address)
__device__ __forceinline__ void prefetch_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, int c3, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
        "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// try_wait with a suspend-time hint (ns): the thread sleeps until the phase
// completes or the hint runs out, instead of spinning on the issue slots
__device__ __forceinline__ bool mbar_try_wait_for(uint64_t *bar, unsigned parity, unsigned ns) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}
// Wait for the phase with this parity; gives up after 2^18 tries of up to
// 10 us each (at least ~26 ms even if no try suspends), records `code` in
// *err and returns false.  A normal load lands within microseconds.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int *err, int code) {
    for (int n = 0; n < (1 << 18); ++n)
        if (mbar_try_wait_for(bar, parity, 10000u)) return true;
    atomicExch(err, code);
    return false;
}

// ---------------------------------------------------------------------------
// per-array power-of-two scaling of 16-bit storage
// ---------------------------------------------------------------------------
template <typename S>
__global__ void amax_kernel(const S *p, size_t n, unsigned *out) {
    float m = 0.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float v = fabsf(static_cast<float>(p[i]));
        m = (v > m || v != v) ? v : m;   // a NaN wins, so overflow is seen
    }
    for (int o = 16; o > 0; o >>= 1) {
        const float t = __shfl_xor_sync(0xffffffffu, m, o);
        m = (t > m || t != t) ? t : m;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

template <typename S>
__global__ void rescale_kernel(S *p, size_t n, float factor) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        p[i] = static_cast<S>(static_cast<float>(p[i]) * factor);
}

}  // namespace sm

// ---------------------------------------------------------------------------
// host: TMA descriptors through the driver entry point (no -lcuda needed)
// ---------------------------------------------------------------------------
namespace sm {

inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 3-D tiled map over a padded array [n2][n1][pitch] of `elem`-byte values
// whose valid extent is n0 x n1 x n2; box b0 x b1 x 1.  Loads outside the
// extent read zeros.  The box row must be a multiple of 16 bytes and every
// load's first coordinate a multiple of 16 bytes / elem (callers ensure it).
inline int make_map_3d(CUtensorMap *m, const void *base, CUtensorMapDataType dt, size_t elem,
                       size_t n0, size_t n1, size_t n2, size_t pitch, unsigned b0, unsigned b1) {
    auto enc = tensor_map_encoder();
    if (!enc) return sm_fail(SM_ECUDA, "cuTensorMapEncodeTiled is not available");
    if ((b0 * elem) % 16 || (pitch * elem) % 16 || (reinterpret_cast<uintptr_t>(base) % 16))
        return sm_fail(SM_EINVAL, "tensor map: 16-byte alignment rule violated");
    cuuint64_t dims[3] = {n0, n1, n2};
    cuuint64_t strides[2] = {pitch * elem, n1 * pitch * elem};
    cuuint32_t box[3] = {b0, b1, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(m, dt, 3, const_cast<void *>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return sm_fail(SM_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return SM_OK;
}

// general tiled map: dims / box innermost first, strides (bytes) of dims 1..
inline int make_map_nd(CUtensorMap *m, const void *base, CUtensorMapDataType dt, size_t elem,
                       int rank, const size_t *dims, const size_t *strides, const unsigned *box) {
    auto enc = tensor_map_encoder();
    if (!enc) return sm_fail(SM_ECUDA, "cuTensorMapEncodeTiled is not available");
    if (rank < 1 || rank > 5) return sm_fail(SM_EINVAL, "tensor map: rank %d", rank);
    if ((box[0] * elem) % 16 || (reinterpret_cast<uintptr_t>(base) % 16))
        return sm_fail(SM_EINVAL, "tensor map: 16-byte alignment rule violated");
    cuuint64_t d[5], st[4];
    cuuint32_t b[5], es[5];
    for (int i = 0; i < rank; ++i) {
        d[i] = dims[i];
        b[i] = box[i];
        es[i] = 1;
        if (i > 0) {
            if (strides[i - 1] % 16) return sm_fail(SM_EINVAL, "tensor map: stride not a multiple of 16");
            st[i - 1] = strides[i - 1];
        }
    }
    CUresult r = enc(m, dt, (cuuint32_t)rank, const_cast<void *>(base), d, st, b, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return sm_fail(SM_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return SM_OK;
}

// Keeps each 16-bit array group's largest stored magnitude near 2^11..2^12
// by power-of-two rescaling (exact unless a value under- or overflows):
// stored = value * 2^expo[group].  check() measures every array (device
// max-abs reduction), rescales the groups whose maximum left [2^9, 2^13],
// and returns SM_ESTATE if any array already holds Inf/NaN.  A group is
// scaled down whenever it grows, but scaled up at most to ceil[group] (set
// from an upper estimate of its amplitude): while a wave is still arriving a
// field's maximum is tiny, and scaling it up to match would overflow once
// the wave arrives.
struct Scaler16 {
    int ngroups = 0;
    std::vector<int> expo;   // per group
    std::vector<int> ceil;   // largest exponent a group may be raised to
    DevBuf d_amax;
    unsigned *h_amax = nullptr;
    int cap = 0;
    ~Scaler16() {
        if (h_amax) cudaFreeHost(h_amax);
    }
    int init(int groups, int max_arrays) {
        ngroups = groups;
        cap = max_arrays;
        expo.assign(groups, 0);
        ceil.assign(groups, 0);
        if (int rc = d_amax.alloc(max_arrays * sizeof(unsigned))) return rc;
        if (cudaMallocHost(&h_amax, max_arrays * sizeof(unsigned)) != cudaSuccess)
            return sm_fail(SM_ENOMEM, "cudaMallocHost failed");
        return SM_OK;
    }
    static int expo_for(double maxval) {   // exponent putting maxval near 2^11
        if (!(maxval > 0.0) || !std::isfinite(maxval)) return 0;
        int e = 11 - std::ilogb(maxval);
        if (e > 100) e = 100;
        if (e < -100) e = -100;
        return e;
    }
    // arrays [0, narr): device pointers, element counts, group of each
    template <typename S>
    int check(cudaStream_t st, int narr, void *const *ptrs, const size_t *ns, const int *group,
              const char *const *gnames) {
        if (narr > cap) return sm_fail(SM_EINVAL, "Scaler16: too many arrays");
        SM_CUDA_TRY(cudaMemsetAsync(d_amax.p, 0, narr * sizeof(unsigned), st));
        for (int a = 0; a < narr; ++a) {
            if (!ns[a]) continue;
            unsigned blocks = (unsigned)std::min<size_t>((ns[a] + 255) / 256, 1184);
            amax_kernel<S><<<blocks, 256, 0, st>>>(static_cast<const S *>(ptrs[a]), ns[a],
                                                   d_amax.as<unsigned>() + a);
        }
        SM_CUDA_TRY(cudaMemcpyAsync(h_amax, d_amax.p, narr * sizeof(unsigned),
                                    cudaMemcpyDeviceToHost, st));
        SM_CUDA_TRY(cudaStreamSynchronize(st));
        std::vector<float> gmax(ngroups, 0.f);
        for (int a = 0; a < narr; ++a) {
            float m;
            std::memcpy(&m, &h_amax[a], sizeof m);
            if (!std::isfinite(m))
                return sm_fail(SM_ESTATE, "16-bit storage of %s overflowed (scale 2^%d)",
                               gnames[group[a]], expo[group[a]]);
            gmax[group[a]] = std::max(gmax[group[a]], m);
        }
        for (int g = 0; g < ngroups; ++g) {
            if (gmax[g] == 0.f) continue;
            const int ex = std::ilogb(gmax[g]);
            if (ex <= 13 && ex >= 9) continue;
            int shift = 11 - ex;
            if (shift > 0) shift = std::min(shift, ceil[g] - expo[g]);
            if (shift == 0) continue;
            for (int a = 0; a < narr; ++a) {
                if (group[a] != g || !ns[a]) continue;
                unsigned blocks = (unsigned)std::min<size_t>((ns[a] + 255) / 256, 4736);
                rescale_kernel<S><<<blocks, 256, 0, st>>>(static_cast<S *>(ptrs[a]), ns[a],
                                                          std::ldexp(1.0f, shift));
            }
            expo[g] += shift;
        }
        SM_CUDA_TRY(cudaGetLastError());
        return SM_OK;
    }
};

template <typename T>
struct MapType;
template <>
struct MapType<float> { static constexpr CUtensorMapDataType v = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; };
template <>
struct MapType<double> { static constexpr CUtensorMapDataType v = CU_TENSOR_MAP_DATA_TYPE_FLOAT64; };
template <>
struct MapType<__half> { static constexpr CUtensorMapDataType v = CU_TENSOR_MAP_DATA_TYPE_FLOAT16; };
template <>
struct MapType<__nv_bfloat16> { static constexpr CUtensorMapDataType v = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; };

}  // namespace sm
