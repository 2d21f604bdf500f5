// EM parameter updates and sum-to-one normalisation, accumulated in FP64.
//
// A sum node block's parameters form a contiguous [nch x bs] slab (child-major, node
// index fastest), and so do its parameter flows. One CTA owns one node block: it reads
// the slab with coalesced row loads, reduces each column (node) in FP64 and rewrites
// the slab. No atomics, no second pass over a per-node scratch buffer.
#include "common.cuh"

namespace {

// Column sums of a [nch x bs] slab for columns [c0, c0 + 256/ROWS...]: thread layout
// (row group rg, column c); partial sums in shared memory.
template <bool EM, bool KEEP_ZERO, typename FT>
__global__ void __launch_bounds__(256)
sum_em_kernel(float* __restrict__ params, const FT* __restrict__ pflows, const int64_t* __restrict__ pbase,
              const int64_t* __restrict__ pfbase, const int* __restrict__ nchs, const int* __restrict__ bss,
              double step, double pc) {
    // No early trigger: kernels after this one may read the parameters before their own wait.
    pcb::pdl_wait();
    __shared__ double part[256];
    const int g = blockIdx.x;
    const int64_t pb = pbase[g];
    const int64_t fb = EM ? pfbase[g] : 0;
    const int nch = nchs[g];
    const int bs = bss[g];
    const int cols = bs < 256 ? bs : 256;       // columns handled per pass
    const int rgs = 256 / cols;                 // row groups
    const int c = threadIdx.x % cols;
    const int rg = threadIdx.x / cols;
    const double pcn = pc / (double)nch;

    // Update of one entry with the column's scale: inv = step / (tot + pc) (EM), 1 / (tot + pc)
    // (normalisation); one FP64 reciprocal per column instead of a division per entry.
    auto update = [&](double p, double f, double inv) -> float {
        double np;
        if (EM) {
            if (KEEP_ZERO) np = (p < 1e-12) ? 0.0 : (1.0 - step) * p + (f + pcn) * inv;
            else np = (1.0 - step) * p + (f + pcn) * inv;
        } else {
            np = (p + pcn) * inv;
        }
        return (float)np;
    };
    constexpr int R = 16;  // entries per thread held in registers (nch <= rgs * R)
    for (int c0 = 0; c0 < bs; c0 += cols) {
        const int col = c0 + c;
        const bool reg = nch <= rgs * R;
        float pv[R];
        FT fv[R];
        double s = 0.0;
        if (rg < rgs) {
            if (reg) {
#pragma unroll
                for (int j = 0; j < R; ++j) {
                    const int k = rg + j * rgs;
                    const int64_t off = (int64_t)k * bs + col;
                    pv[j] = (k < nch) ? params[pb + off] : 0.f;
                    fv[j] = (EM && k < nch) ? pflows[fb + off] : FT(0);
                }
#pragma unroll
                for (int j = 0; j < R; ++j) {
                    if (rg + j * rgs >= nch) continue;
                    if (EM) {
                        if (KEEP_ZERO) s += (pv[j] < 1e-12f) ? 0.0 : ((double)fv[j] + pcn);
                        else s += (double)fv[j];
                    } else {
                        s += (double)pv[j];
                    }
                }
            } else {
                for (int k = rg; k < nch; k += rgs) {
                    const int64_t off = (int64_t)k * bs + col;
                    if (EM) {
                        const double f = (double)pflows[fb + off];
                        if (KEEP_ZERO) {
                            const float p = params[pb + off];
                            s += (p < 1e-12f) ? 0.0 : (f + pcn);
                        } else {
                            s += f;
                        }
                    } else {
                        s += (double)params[pb + off];
                    }
                }
            }
        }
        part[threadIdx.x] = s;
        __syncthreads();
        double tot = 0.0;
        for (int r = 0; r < rgs; ++r) tot += part[r * cols + c];
        __syncthreads();
        const double inv = EM ? (KEEP_ZERO ? step / tot : step / (tot + pc)) : 1.0 / (tot + pc);
        if (rg < rgs) {
            if (reg) {
#pragma unroll
                for (int j = 0; j < R; ++j) {
                    const int k = rg + j * rgs;
                    if (k < nch) params[pb + (int64_t)k * bs + col] = update((double)pv[j], (double)fv[j], inv);
                }
            } else {
                for (int k = rg; k < nch; k += rgs) {
                    const int64_t off = (int64_t)k * bs + col;
                    params[pb + off] = update((double)params[pb + off], EM ? (double)pflows[fb + off] : 0.0, inv);
                }
            }
        }
    }
}

// One warp per source input node, categories strided over the lanes. Nodes of up to 256
// categories keep their flows and parameters in registers (all loads of a node issued at
// once, one pass over memory); larger ones take two passes.
template <bool KEEP_ZERO, typename FT>
__global__ void __launch_bounds__(256)
input_em_kernel(float* __restrict__ params, const FT* __restrict__ pflows, const int* __restrict__ s_pids,
                const int* __restrict__ s_pfids, const int* __restrict__ ncats, const int* __restrict__ source_nids,
                int num_src, double step, double pc) {
    pcb::pdl_wait();  // no early trigger, as in sum_em_kernel
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= num_src) return;
    const int n = source_nids[w];
    const int K = ncats[n];
    const int64_t sp = s_pids[n];
    const int64_t sf = s_pfids[n];
    const double pcn = pc / (double)K;
    // one FP64 reciprocal per node: inv = step / s (keep-zero form) or step / (s + pc)
    auto scale = [&](double s) -> double { return KEEP_ZERO ? step / s : step / (s + pc); };
    auto update = [&](double p, double f, double inv) -> float {
        double np;
        if (KEEP_ZERO) np = (p < 1e-12) ? 0.0 : (1.0 - step) * p + (f + pcn) * inv;
        else np = (1.0 - step) * p + (f + pcn) * inv;
        return (float)np;
    };
    constexpr int R = 8;
    if (K <= 32 * R) {
        FT f[R];
        float p[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int k = lane + 32 * j;
            f[j] = k < K ? pflows[sf + k] : FT(0);
            p[j] = k < K ? params[sp + k] : 0.f;
        }
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < R; ++j) {
            if (lane + 32 * j >= K) continue;
            if (KEEP_ZERO) s += (p[j] < 1e-12f) ? 0.0 : (double)f[j] + pcn;
            else s += (double)f[j];
        }
        s = pcb::warp_sum(s);
        const double inv = scale(s);
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int k = lane + 32 * j;
            if (k < K) params[sp + k] = update((double)p[j], (double)f[j], inv);
        }
        return;
    }
    double s = 0.0;
    for (int k = lane; k < K; k += 32) {
        const double f = (double)pflows[sf + k];
        if (KEEP_ZERO) s += (params[sp + k] < 1e-12f) ? 0.0 : f + pcn;
        else s += f;
    }
    s = pcb::warp_sum(s);
    const double inv = scale(s);
    for (int k = lane; k < K; k += 32) params[sp + k] = update((double)params[sp + k], (double)pflows[sf + k], inv);
}

template <typename FT>
int sum_em_launch(float* params, const FT* param_flows, const int64_t* blk_pbase, const int64_t* blk_pfbase,
                  const int32_t* blk_nch, const int32_t* blk_bs, int32_t num_blocks, double step_size,
                  double pseudocount, int32_t keep_zero_params, void* stream, const char* name) {
    if (!params || !param_flows || !blk_pbase || !blk_pfbase || !blk_nch || !blk_bs || num_blocks < 0)
        return pcb::set_error(PCB_E_ARG, "%s: bad arguments", name);
    if (!(step_size > 0.0 && step_size <= 1.0)) return pcb::set_error(PCB_E_ARG, "%s: step_size must be in (0, 1]", name);
    if (num_blocks == 0) return PCB_OK;
    cudaStream_t s = pcb::as_stream(stream);
    if (keep_zero_params) {
        return pcb::launch_status(pcb::launch_k(sum_em_kernel<true, true, FT>, dim3(num_blocks), dim3(256), 0, s, 1u,
                                                params, param_flows, blk_pbase, blk_pfbase, blk_nch, blk_bs,
                                                step_size, pseudocount), name);
    }
    return pcb::launch_status(pcb::launch_k(sum_em_kernel<true, false, FT>, dim3(num_blocks), dim3(256), 0, s, 1u,
                                            params, param_flows, blk_pbase, blk_pfbase, blk_nch, blk_bs, step_size,
                                            pseudocount), name);
}

template <typename FT>
int input_em_launch(float* params, const FT* param_flows, const int32_t* s_pids, const int32_t* s_pfids,
                    const int32_t* ncats, const int32_t* source_nids, int32_t num_source_nodes, double step_size,
                    double pseudocount, int32_t keep_zero_params, void* stream, const char* name) {
    if (!params || !param_flows || !s_pids || !s_pfids || !ncats || !source_nids || num_source_nodes < 0)
        return pcb::set_error(PCB_E_ARG, "%s: bad arguments", name);
    if (!(step_size > 0.0 && step_size <= 1.0)) return pcb::set_error(PCB_E_ARG, "%s: step_size must be in (0, 1]", name);
    if (num_source_nodes == 0) return PCB_OK;
    const unsigned grid = (unsigned)pcb::cdiv((int64_t)num_source_nodes * 32, 256);
    cudaStream_t s = pcb::as_stream(stream);
    if (keep_zero_params) {
        return pcb::launch_status(pcb::launch_k(input_em_kernel<true, FT>, dim3(grid), dim3(256), 0, s, 1u, params,
                                                param_flows, s_pids, s_pfids, ncats, source_nids, num_source_nodes,
                                                step_size, pseudocount), name);
    }
    return pcb::launch_status(pcb::launch_k(input_em_kernel<false, FT>, dim3(grid), dim3(256), 0, s, 1u, params,
                                            param_flows, s_pids, s_pfids, ncats, source_nids, num_source_nodes,
                                            step_size, pseudocount), name);
}

// acc[i] += flows[i]: 4 elements per thread, grid-stride.
__global__ void flows_accumulate_f64_kernel(double* __restrict__ acc, const float* __restrict__ flows, int64_t n) {
    pcb::pdl_begin();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) acc[i] += (double)flows[i];
}

__global__ void pflow_accum_f64_kernel(double* __restrict__ pf, int64_t dst, int64_t n,
                                       const int64_t* __restrict__ srcs, int nsrc) {
    pcb::pdl_begin();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int j = 0; j < nsrc; ++j) s += pf[srcs[j] + i];
    pf[dst + i] = s;
}

// Gradient of the scaled log-likelihood with respect to softmax logits of the weights:
// per node i of a block, grad[k, i] = scale * (pf[k, i] - theta[k, i] * sum_k' pf[k', i]),
// where pf are the parameter flows (theta times the derivative with respect to theta).
__global__ void __launch_bounds__(256)
sum_logit_grad_kernel(const float* __restrict__ params, const float* __restrict__ pflows,
                      const int64_t* __restrict__ pbase, const int64_t* __restrict__ pfbase,
                      const int* __restrict__ nchs, const int* __restrict__ bss, double scale,
                      float* __restrict__ grad) {
    pcb::pdl_begin();
    const int g = blockIdx.x;
    const int64_t pb = pbase[g], fb = pfbase[g];
    const int nch = nchs[g], bs = bss[g];
    for (int i = threadIdx.x; i < bs; i += blockDim.x) {
        double tot = 0.0;
        for (int k = 0; k < nch; ++k) tot += (double)pflows[fb + (int64_t)k * bs + i];
        for (int k = 0; k < nch; ++k) {
            const int64_t o = (int64_t)k * bs + i;
            grad[pb + o] = (float)(scale * ((double)pflows[fb + o] - (double)params[pb + o] * tot));
        }
    }
}

// Weights from softmax logits: per node i of a block, theta[k, i] = exp(z[k, i] - m) / sum_k' exp(z[k', i] - m),
// m = max_k z[k, i] (FP64 sum).
__global__ void __launch_bounds__(128)
sum_softmax_kernel(const float* __restrict__ logits, float* __restrict__ params, const int64_t* __restrict__ pbase,
                   const int* __restrict__ nchs, const int* __restrict__ bss) {
    pcb::pdl_begin();
    const int g = blockIdx.x;
    const int64_t pb = pbase[g];
    const int nch = nchs[g], bs = bss[g];
    for (int i = threadIdx.x; i < bs; i += blockDim.x) {
        float m = -INFINITY;
        for (int k = 0; k < nch; ++k) m = fmaxf(m, logits[pb + (int64_t)k * bs + i]);
        double tot = 0.0;
        for (int k = 0; k < nch; ++k) tot += exp((double)logits[pb + (int64_t)k * bs + i] - (double)m);
        const double inv = 1.0 / tot;
        for (int k = 0; k < nch; ++k) {
            const int64_t o = pb + (int64_t)k * bs + i;
            params[o] = (float)(exp((double)logits[o] - (double)m) * inv);
        }
    }
}

// The same for Categorical input nodes: one warp per source node.
__global__ void __launch_bounds__(256)
input_logit_grad_kernel(const float* __restrict__ params, const float* __restrict__ pflows,
                        const int* __restrict__ s_pids, const int* __restrict__ s_pfids, const int* __restrict__ ncats,
                        const int* __restrict__ source_nids, int num_src, double scale, float* __restrict__ grad) {
    pcb::pdl_begin();
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= num_src) return;
    const int n = source_nids[w];
    const int K = ncats[n];
    const int64_t sp = s_pids[n], sf = s_pfids[n];
    double tot = 0.0;
    for (int k = lane; k < K; k += 32) tot += (double)pflows[sf + k];
    tot = pcb::warp_sum(tot);
    for (int k = lane; k < K; k += 32)
        grad[sp + k] = (float)(scale * ((double)pflows[sf + k] - (double)params[sp + k] * tot));
}

}  // namespace

extern "C" int pcb_sum_logit_grad(const float* params, const float* param_flows, const int64_t* blk_pbase,
                                  const int64_t* blk_pfbase, const int32_t* blk_nch, const int32_t* blk_bs,
                                  int32_t num_blocks, double scale, float* grad, void* stream) {
    if (!params || !param_flows || !blk_pbase || !blk_pfbase || !blk_nch || !blk_bs || !grad || num_blocks < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_sum_logit_grad: bad arguments");
    if (num_blocks == 0) return PCB_OK;
    return pcb::launch_status(pcb::launch_k(sum_logit_grad_kernel, dim3(num_blocks), dim3(128), 0,
                                            pcb::as_stream(stream), 1u, params, param_flows, blk_pbase, blk_pfbase,
                                            blk_nch, blk_bs, scale, grad), "pcb_sum_logit_grad");
}

extern "C" int pcb_sum_softmax(const float* logits, float* params, const int64_t* blk_pbase, const int32_t* blk_nch,
                               const int32_t* blk_bs, int32_t num_blocks, void* stream) {
    if (!logits || !params || !blk_pbase || !blk_nch || !blk_bs || num_blocks < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_sum_softmax: bad arguments");
    if (num_blocks == 0) return PCB_OK;
    return pcb::launch_status(pcb::launch_k(sum_softmax_kernel, dim3(num_blocks), dim3(128), 0, pcb::as_stream(stream),
                                            1u, logits, params, blk_pbase, blk_nch, blk_bs), "pcb_sum_softmax");
}

extern "C" int pcb_input_cat_logit_grad(const float* params, const float* param_flows, const int32_t* s_pids,
                                        const int32_t* s_pfids, const int32_t* ncats, const int32_t* source_nids,
                                        int32_t num_source_nodes, double scale, float* grad, void* stream) {
    if (!params || !param_flows || !s_pids || !s_pfids || !ncats || !source_nids || !grad || num_source_nodes < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_input_cat_logit_grad: bad arguments");
    if (num_source_nodes == 0) return PCB_OK;
    return pcb::launch_status(pcb::launch_k(input_logit_grad_kernel,
                                            dim3((unsigned)pcb::cdiv((int64_t)num_source_nodes * 32, 256)), dim3(256),
                                            0, pcb::as_stream(stream), 1u, params, param_flows, s_pids, s_pfids, ncats,
                                            source_nids, num_source_nodes, scale, grad), "pcb_input_cat_logit_grad");
}

extern "C" int pcb_sum_em(float* params, const float* param_flows, const int64_t* blk_pbase, const int64_t* blk_pfbase,
                          const int32_t* blk_nch, const int32_t* blk_bs, int32_t num_blocks, double step_size,
                          double pseudocount, int32_t keep_zero_params, void* stream) {
    return sum_em_launch<float>(params, param_flows, blk_pbase, blk_pfbase, blk_nch, blk_bs, num_blocks, step_size,
                                pseudocount, keep_zero_params, stream, "pcb_sum_em");
}

extern "C" int pcb_sum_em_f64flows(float* params, const double* param_flows, const int64_t* blk_pbase,
                                   const int64_t* blk_pfbase, const int32_t* blk_nch, const int32_t* blk_bs,
                                   int32_t num_blocks, double step_size, double pseudocount, int32_t keep_zero_params,
                                   void* stream) {
    return sum_em_launch<double>(params, param_flows, blk_pbase, blk_pfbase, blk_nch, blk_bs, num_blocks, step_size,
                                 pseudocount, keep_zero_params, stream, "pcb_sum_em_f64flows");
}

extern "C" int pcb_sum_normalize(float* params, const int64_t* blk_pbase, const int32_t* blk_nch, const int32_t* blk_bs,
                                 int32_t num_blocks, double pseudocount, void* stream) {
    if (!params || !blk_pbase || !blk_nch || !blk_bs || num_blocks < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_sum_normalize: bad arguments");
    if (num_blocks == 0) return PCB_OK;
    return pcb::launch_status(pcb::launch_k(sum_em_kernel<false, false, float>, dim3(num_blocks), dim3(256), 0,
                                            pcb::as_stream(stream), 1u, params, nullptr, blk_pbase, nullptr, blk_nch,
                                            blk_bs, 1.0, pseudocount), "pcb_sum_normalize");
}

extern "C" int pcb_input_cat_em(float* params, const float* param_flows, const int32_t* s_pids, const int32_t* s_pfids,
                                const int32_t* ncats, const int32_t* source_nids, int32_t num_source_nodes,
                                double step_size, double pseudocount, int32_t keep_zero_params, void* stream) {
    return input_em_launch<float>(params, param_flows, s_pids, s_pfids, ncats, source_nids, num_source_nodes,
                                  step_size, pseudocount, keep_zero_params, stream, "pcb_input_cat_em");
}

extern "C" int pcb_input_cat_em_f64flows(float* params, const double* param_flows, const int32_t* s_pids,
                                         const int32_t* s_pfids, const int32_t* ncats, const int32_t* source_nids,
                                         int32_t num_source_nodes, double step_size, double pseudocount,
                                         int32_t keep_zero_params, void* stream) {
    return input_em_launch<double>(params, param_flows, s_pids, s_pfids, ncats, source_nids, num_source_nodes,
                                   step_size, pseudocount, keep_zero_params, stream, "pcb_input_cat_em_f64flows");
}

extern "C" int pcb_flows_accumulate_f64(double* acc, const float* flows, int64_t n, void* stream) {
    if (!acc || !flows || n < 0) return pcb::set_error(PCB_E_ARG, "pcb_flows_accumulate_f64: bad arguments");
    if (n == 0) return PCB_OK;
    int64_t blocks = pcb::cdiv(n, 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    return pcb::launch_status(pcb::launch_k(flows_accumulate_f64_kernel, dim3((unsigned)blocks), dim3(256), 0,
                                            pcb::as_stream(stream), 1u, acc, flows, n), "pcb_flows_accumulate_f64");
}

extern "C" int pcb_pflow_accum_f64(double* param_flows, int64_t dst, int64_t n, const int64_t* srcs, int32_t nsrc,
                                   void* stream) {
    if (!param_flows || !srcs || n < 0 || nsrc <= 0) return pcb::set_error(PCB_E_ARG, "pcb_pflow_accum_f64: bad arguments");
    if (n == 0) return PCB_OK;
    return pcb::launch_status(pcb::launch_k(pflow_accum_f64_kernel, dim3((unsigned)pcb::cdiv(n, 256)), dim3(256), 0,
                                            pcb::as_stream(stream), 1u, param_flows, dst, n, srcs, nsrc),
                              "pcb_pflow_accum_f64");
}
