// Library-level entry points and error reporting.
#include <cstdarg>
#include <cstring>

#include <atomic>
#include <cstdlib>

#include "common.cuh"

namespace pcb {

static thread_local char g_last_error[512] = {0};

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

bool pdl_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("PCB_NO_PDL");
        return !(v && v[0] == '1');
    }();
    return on;
}

int launch_status(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(PCB_E_LAUNCH, "%s: launch failed: %s", what, cudaGetErrorString(e));
    }
    return PCB_OK;
}

namespace {
// One status word per device (the runtime instantiates __device__ variables per device).
__device__ int32_t g_status_word = 0;
constexpr int kMaxDevices = 64;
std::atomic<int32_t*> g_status_addr[kMaxDevices];
}  // namespace

int32_t* status_word() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    int32_t* p = g_status_addr[dev].load(std::memory_order_acquire);
    if (p == nullptr) {
        void* a = nullptr;
        if (cudaGetSymbolAddress(&a, g_status_word) != cudaSuccess || a == nullptr) {
            cudaGetLastError();
            return nullptr;
        }
        p = static_cast<int32_t*>(a);
        g_status_addr[dev].store(p, std::memory_order_release);
    }
    return p;
}

int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        return set_error(PCB_E_LAUNCH, "%s: launch failed: %s", what, cudaGetErrorString(e));
    }
    return PCB_OK;
}

}  // namespace pcb

namespace {

__global__ void fill_rows_kernel(float* __restrict__ mat, int64_t n, float value) {
    pcb::pdl_begin();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) mat[i] = value;
}

__global__ void ll_sum_kernel(const float* __restrict__ lls, int B, double* __restrict__ out) {
    pcb::pdl_begin();
    __shared__ double part[8];
    double s = 0.0;
    for (int b = threadIdx.x; b < B; b += blockDim.x) s += (double)lls[b];
    s = pcb::warp_sum(s);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = (threadIdx.x < (blockDim.x >> 5)) ? part[threadIdx.x] : 0.0;
        t = pcb::warp_sum(t);
        if (threadIdx.x == 0) out[0] += t;
    }
}

// One CTA waits, with a bounded number of polls, on an mbarrier that nothing completes (the
// same bounded wait the tcgen05 contraction uses for its weight copy and MMAs), then reports
// the timeout in the status word and returns.
__global__ void status_selftest_kernel(int spin_limit, int32_t* status) {
    __shared__ __align__(8) uint64_t bar;
    const unsigned b = (unsigned)__cvta_generic_to_shared(&bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(b), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int i = 0; i < spin_limit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(b), "r"(0)
            : "memory");
        if (ok) return;
    }
    pcb::report_status(status, PCB_STATUS_WAIT_TIMEOUT);
}

__global__ void pflow_accum_kernel(float* __restrict__ pf, int64_t dst, int64_t n, const int64_t* __restrict__ srcs,
                                   int nsrc) {
    pcb::pdl_begin();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.f;
    for (int j = 0; j < nsrc; ++j) s += pf[srcs[j] + i];
    pf[dst + i] = s;
}

}  // namespace

extern "C" {

int pcb_version(void) { return 1; }

const char* pcb_last_error(void) { return pcb::g_last_error; }

int pcb_num_sms(void) {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "cudaGetDevice failed");
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return pcb::set_error(PCB_E_CUDA, "cudaDeviceGetAttribute failed");
    return n;
}

int pcb_fill_rows(float* mat, int64_t ld, int64_t row0, int64_t row1, float value, void* stream) {
    if (!mat || ld <= 0 || row0 < 0 || row1 < row0) return pcb::set_error(PCB_E_ARG, "pcb_fill_rows: bad arguments");
    int64_t n = (row1 - row0) * ld;
    if (n == 0) return PCB_OK;
    int64_t blocks = pcb::cdiv(n, 256);
    if (blocks > 4 * 148 * 8) blocks = 4 * 148 * 8;
    return pcb::launch_status(pcb::launch_k(fill_rows_kernel, dim3((unsigned)blocks), dim3(256), 0,
                                            pcb::as_stream(stream), 1u, mat + row0 * ld, n, value),
                              "pcb_fill_rows");
}

int pcb_ll_sum_f64(const float* lls, int64_t ld, int32_t B, int64_t row, double* out, void* stream) {
    if (!lls || !out || B <= 0 || row < 0) return pcb::set_error(PCB_E_ARG, "pcb_ll_sum_f64: bad arguments");
    return pcb::launch_status(pcb::launch_k(ll_sum_kernel, dim3(1), dim3(256), 0, pcb::as_stream(stream), 1u,
                                            lls + row * ld, B, out), "pcb_ll_sum_f64");
}

int pcb_device_status(int32_t* out, int32_t clear, void* stream) {
    if (!out) return pcb::set_error(PCB_E_ARG, "pcb_device_status: bad arguments");
    int32_t* w = pcb::status_word();
    if (!w) return pcb::set_error(PCB_E_CUDA, "pcb_device_status: status word look-up failed");
    cudaStream_t s = pcb::as_stream(stream);
    cudaError_t e = cudaMemcpyAsync(out, w, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && clear) e = cudaMemsetAsync(w, 0, sizeof(int32_t), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_device_status: %s", cudaGetErrorString(e));
    return PCB_OK;
}

int pcb_status_selftest(int32_t spin_limit, void* stream) {
    if (spin_limit < 0) return pcb::set_error(PCB_E_ARG, "pcb_status_selftest: bad arguments");
    status_selftest_kernel<<<1, 32, 0, pcb::as_stream(stream)>>>(spin_limit, pcb::status_word());
    return pcb::check_launch("pcb_status_selftest");
}

int pcb_pflow_accum(float* param_flows, int64_t dst, int64_t n, const int64_t* srcs, int32_t nsrc, void* stream) {
    if (!param_flows || !srcs || n < 0 || nsrc <= 0) return pcb::set_error(PCB_E_ARG, "pcb_pflow_accum: bad arguments");
    if (n == 0) return PCB_OK;
    return pcb::launch_status(pcb::launch_k(pflow_accum_kernel, dim3((unsigned)pcb::cdiv(n, 256)), dim3(256), 0,
                                            pcb::as_stream(stream), 1u, param_flows, dst, n, srcs, nsrc),
                              "pcb_pflow_accum");
}

}  // extern "C"
