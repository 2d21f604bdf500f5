// Shared helpers of the libpcb200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cmath>
#include <utility>

#include "../../include/pcb200.h"

namespace pcb {

// Records a message as the calling thread's last error and returns `code`.
int set_error(int code, const char* fmt, ...);

// Checks the launch that was just issued; returns PCB_OK or PCB_E_LAUNCH.
int check_launch(const char* what);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

__device__ __forceinline__ float neg_inf() { return -INFINITY; }

// 4 consecutive samples of row `row`: vectorised when the row start is 16-byte aligned
// and all 4 samples are in range, scalar (with `fill` beyond B) otherwise.
__device__ __forceinline__ float4 load4(const float* __restrict__ base, int64_t row, int64_t ld, int b, int B,
                                        bool vec, float fill) {
    const float* p = base + row * ld + b;
    if (vec && b + 3 < B) {
        return __ldg(reinterpret_cast<const float4*>(p));
    }
    float4 v;
    v.x = (b + 0 < B) ? __ldg(p + 0) : fill;
    v.y = (b + 1 < B) ? __ldg(p + 1) : fill;
    v.z = (b + 2 < B) ? __ldg(p + 2) : fill;
    v.w = (b + 3 < B) ? __ldg(p + 3) : fill;
    return v;
}

__device__ __forceinline__ void store4(float* __restrict__ base, int64_t row, int64_t ld, int b, int B, bool vec,
                                       float4 v) {
    float* p = base + row * ld + b;
    if (vec && b + 3 < B) {
        *reinterpret_cast<float4*>(p) = v;
        return;
    }
    if (b + 0 < B) p[0] = v.x;
    if (b + 1 < B) p[1] = v.y;
    if (b + 2 < B) p[2] = v.z;
    if (b + 3 < B) p[3] = v.w;
}

__device__ __forceinline__ float get(const float4& v, int j) {
    return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}

__device__ __forceinline__ void set(float4& v, int j, float x) {
    if (j == 0) v.x = x; else if (j == 1) v.y = x; else if (j == 2) v.z = x; else v.w = x;
}

// log(a) + log(b) combined in log space: log(exp(a) + exp(b)).
__device__ __forceinline__ float logaddexp(float a, float b) {
    if (a == -INFINITY) return b;
    if (b == -INFINITY) return a;
    float m = fmaxf(a, b);
    return m + log1pf(expf(-fabsf(a - b)));
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Asynchronous global -> shared copies (no register round trip, so a thread can have many
// in flight). 16-byte copies need 16-byte aligned addresses on both sides.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Programmatic dependent launch. pdl_trigger() lets the next kernel of the stream be
// scheduled as soon as every CTA of this grid has executed it; pdl_wait() blocks until the
// previous grid has completed and its memory is visible. Kernels launched without the
// attribute pass through both instructions at once. Most kernels start with both
// (pdl_begin). A kernel may do work between the two, overlapping the previous kernel's
// tail, only on memory that no early-triggering kernel writes: the compiled tables, data
// written by other libraries' kernels (which never trigger early), and the parameters,
// whose writers (the EM kernels) call pdl_wait() alone, so that their successors start
// only after they have completed. Such reads bypass L1 (cp.async.cg, ld.global.cg).
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

__device__ __forceinline__ void pdl_begin() {
    pdl_trigger();
    pdl_wait();
}

// Whether launches carry the programmatic-stream-serialization attribute (on unless the
// environment sets PCB_NO_PDL=1).
bool pdl_enabled();

// Launch with the programmatic-stream-serialization attribute (and an optional cluster
// size along x); returns the launch status.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                            unsigned cluster_x, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    unsigned n = 0;
    if (pdl_enabled()) {
        attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[n].val.programmaticStreamSerializationAllowed = 1;
        ++n;
    }
    if (cluster_x > 1) {
        attr[n].id = cudaLaunchAttributeClusterDimension;
        attr[n].val.clusterDim.x = cluster_x;
        attr[n].val.clusterDim.y = 1;
        attr[n].val.clusterDim.z = 1;
        ++n;
    }
    cfg.attrs = attr;
    cfg.numAttrs = n;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Status of a launch_k call: PCB_OK, or PCB_E_LAUNCH with the message recorded.
int launch_status(cudaError_t e, const char* what);

// Device address of the library's status word on the current device (a __device__ int32 in
// capi_common.cu, looked up once per device; nullptr if the look-up failed). Kernels OR
// PCB_STATUS_* bits into it when they detect a fault; pcb_device_status reads it.
int32_t* status_word();

__device__ __forceinline__ void report_status(int32_t* status, int32_t bits) {
    if (status) atomicOr(status, bits);
}

// Natural logarithm and exponential on the hardware base-2 approximations (MUFU lg2 / ex2,
// flush-to-zero forms): ln x = log2(x) ln 2 with subnormal x rescaled by 2^24 first, and
// e^x = 2^(x log2 e), whose results below the smallest normal float are 0. For the BF16
// contraction forms, whose operand rounding is far coarser than these approximations.
__device__ __forceinline__ float fast_log(float x) {
    const bool sub = x < 1.17549435e-38f;
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(sub ? x * 16777216.f : x));
    return (r - (sub ? 24.f : 0.f)) * 0.6931471805599453f;
}

__device__ __forceinline__ float fast_exp(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x * 1.4426950408889634f));
    return r;
}

// Vectorised access needs ld % 4 == 0 and a 16-byte aligned base.
inline bool vec_ok(const void* p, int64_t ld) {
    return (ld % 4 == 0) && ((reinterpret_cast<uintptr_t>(p) & 15) == 0);
}

}  // namespace pcb
