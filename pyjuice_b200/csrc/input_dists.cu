// Bernoulli and Gaussian input layers: forward log-probabilities, parameter flows (the
// distributions' sufficient statistics weighted by node flows) and the EM update.
//   Bernoulli (kind 1): one parameter p per node; x > 0 has probability p. Flows: slot 0
//     collects the flow of samples with x > 0, slot 1 the others
//     (src/pyjuice/nodes/distributions/bernoulli.py:64-102).
//   Gaussian (kind 2): parameters (mu, sigma) per node, log N(x; mu, sigma). Flows: slots
//     (sum f x, sum f x^2, sum f); a missing value contributes its expectation (mu f,
//     (sigma^2 + mu^2) f, f). EM moment-matches the updated expectation parameters, with
//     sigma clamped below at min_sigma (gaussian.py:87-170).
// Data: FP32 [num_vars, data_ld] (Bernoulli reads x > 0). Missing values (mask as in
// pcb_input_cat_fwd) give log 1 in the forward pass.
#include <algorithm>

#include "common.cuh"

namespace {

constexpr float kLog2Pi = 1.8378770664093453f;

__global__ void __launch_bounds__(256)
dist_fwd_kernel(int kind, const float* __restrict__ data, int64_t data_ld, const float* __restrict__ params,
                const int* __restrict__ vids, const int* __restrict__ s_pids, int num_nodes, int node_offset,
                float* __restrict__ nm, int64_t ld, int B, const uint8_t* __restrict__ miss, int64_t m_sb,
                int64_t m_sv) {
    pcb::pdl_begin();
    for (int n = blockIdx.y; n < num_nodes; n += gridDim.y) {
    const int64_t v = vids[n];
    const int64_t sp = s_pids[n];
    const float a = params[sp];
    const float s = kind == 2 ? params[sp + 1] : 0.f;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
        float r;
        if (miss && miss[(int64_t)b * m_sb + v * m_sv]) {
            r = 0.f;
        } else {
            const float x = data[v * data_ld + b];
            if (kind == 1) {
                r = logf(x > 0.f ? a : 1.f - a);
            } else {
                const float c = (x - a) / s;
                r = -0.5f * c * c - 0.5f * kLog2Pi - logf(s);
            }
        }
        nm[((int64_t)node_offset + n) * ld + b] = r;
    }
    }
}

// One warp per node: the statistics summed over the batch, then added to the node's slots.
__global__ void __launch_bounds__(256)
dist_bwd_kernel(int kind, const float* __restrict__ data, int64_t data_ld, const float* __restrict__ nf, int64_t ld,
                int B, const float* __restrict__ params, const int* __restrict__ vids, const int* __restrict__ s_pids,
                const int* __restrict__ s_pfids, int num_nodes, int node_offset, float* __restrict__ pf,
                bool logspace, const uint8_t* __restrict__ miss, int64_t m_sb, int64_t m_sv, bool atomic) {
    pcb::pdl_begin();
    const int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (n >= num_nodes) return;
    const int64_t v = vids[n];
    const int64_t sp = s_pids[n];
    const float mu = params[sp];
    const float sg = kind == 2 ? params[sp + 1] : 0.f;
    const float* row = nf + ((int64_t)node_offset + n) * ld;
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    for (int b = lane; b < B; b += 32) {
        float f = row[b];
        if (logspace) f = expf(f);
        const bool missing = miss && miss[(int64_t)b * m_sb + v * m_sv];
        if (kind == 1) {
            if (missing) continue;  // the Bernoulli layer has no missing-value flows (bernoulli.py)
            if (data[v * data_ld + b] > 0.f) s0 += f;
            else s1 += f;
        } else if (missing) {
            s0 += mu * f;
            s1 += (sg * sg + mu * mu) * f;
            s2 += f;
        } else {
            const float x = data[v * data_ld + b];
            s0 += x * f;
            s1 += x * x * f;
            s2 += f;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
        const int64_t sf = s_pfids[n];
        const int ns = kind == 1 ? 2 : 3;
        const float st[3] = {s0, s1, s2};
        for (int j = 0; j < ns; ++j) {
            if (atomic) atomicAdd(pf + sf + j, st[j]);
            else pf[sf + j] += st[j];
        }
    }
}

__global__ void __launch_bounds__(256)
dist_em_kernel(int kind, float* __restrict__ params, const float* __restrict__ pf, const int* __restrict__ s_pids,
               const int* __restrict__ s_pfids, const float* __restrict__ min_sigma,
               const int* __restrict__ source_nids, int num_src, double step, double pc) {
    pcb::pdl_wait();  // parameter writer: no early trigger
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= num_src) return;
    const int n = source_nids[i];
    const int64_t sp = s_pids[n], sf = s_pfids[n];
    if (kind == 1) {
        const double f1 = pf[sf], f0 = pf[sf + 1];
        const double upd = (f1 + 0.5 * pc) / (f1 + f0 + pc);
        params[sp] = (float)((1.0 - step) * (double)params[sp] + step * upd);
    } else {
        const double mu = params[sp], sg = params[sp + 1];
        const double t1 = pf[sf] / ((double)pf[sf + 2] + 1e-10);
        const double t2 = pf[sf + 1] / ((double)pf[sf + 2] + 1e-10);
        const double u1 = (1.0 - step) * mu + step * t1;
        const double u2 = (1.0 - step) * (sg * sg + mu * mu) + step * t2;
        const double var = u2 - u1 * u1;
        const double ms = min_sigma[n];
        params[sp] = (float)u1;
        params[sp + 1] = (float)(var < ms * ms ? ms : sqrt(var));
    }
}

}  // namespace

extern "C" int pcb_input_dist_fwd(int32_t kind, const float* data, int64_t data_ld, const float* params,
                                  const int32_t* vids, const int32_t* s_pids, int32_t num_nodes, int32_t node_offset,
                                  float* node_mars, int64_t ld, int32_t B, const uint8_t* missing, int64_t miss_sb,
                                  int64_t miss_sv, void* stream) {
    if ((kind != 1 && kind != 2) || !data || !params || !vids || !s_pids || !node_mars || B <= 0 || ld < B ||
        data_ld < B || num_nodes < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_input_dist_fwd: bad arguments");
    if (num_nodes == 0) return PCB_OK;
    const unsigned gx = (unsigned)std::min<int64_t>(pcb::cdiv(B, 256), 64);
    const unsigned gy = (unsigned)std::min<int64_t>(num_nodes, 65535);
    return pcb::launch_status(pcb::launch_k(dist_fwd_kernel, dim3(gx, gy), dim3(256), 0,
                                            pcb::as_stream(stream), 1u, (int)kind, data, data_ld, params, vids, s_pids,
                                            num_nodes, node_offset, node_mars, ld, B, missing, miss_sb, miss_sv),
                              "pcb_input_dist_fwd");
}

extern "C" int pcb_input_dist_bwd(int32_t kind, const float* data, int64_t data_ld, const float* node_flows, int64_t ld,
                                  int32_t B, const float* params, const int32_t* vids, const int32_t* s_pids,
                                  const int32_t* s_pfids, int32_t num_nodes, int32_t node_offset, float* param_flows,
                                  int32_t logspace_flows, const uint8_t* missing, int64_t miss_sb, int64_t miss_sv,
                                  int32_t atomic, void* stream) {
    if ((kind != 1 && kind != 2) || !data || !node_flows || !params || !vids || !s_pids || !s_pfids || !param_flows ||
        B <= 0 || ld < B || data_ld < B || num_nodes < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_input_dist_bwd: bad arguments");
    if (num_nodes == 0) return PCB_OK;
    return pcb::launch_status(pcb::launch_k(dist_bwd_kernel, dim3((unsigned)pcb::cdiv((int64_t)num_nodes * 32, 256)),
                                            dim3(256), 0, pcb::as_stream(stream), 1u, (int)kind, data, data_ld,
                                            node_flows, ld, B, params, vids, s_pids, s_pfids, num_nodes, node_offset,
                                            param_flows, logspace_flows != 0, missing, miss_sb, miss_sv, atomic != 0),
                              "pcb_input_dist_bwd");
}

extern "C" int pcb_input_dist_em(int32_t kind, float* params, const float* param_flows, const int32_t* s_pids,
                                 const int32_t* s_pfids, const float* min_sigma, const int32_t* source_nids,
                                 int32_t num_source_nodes, double step_size, double pseudocount, void* stream) {
    if ((kind != 1 && kind != 2) || !params || !param_flows || !s_pids || !s_pfids || !source_nids ||
        (kind == 2 && !min_sigma) || num_source_nodes < 0 || !(step_size > 0.0 && step_size <= 1.0))
        return pcb::set_error(PCB_E_ARG, "pcb_input_dist_em: bad arguments");
    if (num_source_nodes == 0) return PCB_OK;
    return pcb::launch_status(pcb::launch_k(dist_em_kernel, dim3((unsigned)pcb::cdiv(num_source_nodes, 256)),
                                            dim3(256), 0, pcb::as_stream(stream), 1u, (int)kind, params, param_flows,
                                            s_pids, s_pfids, min_sigma, source_nids, num_source_nodes, step_size,
                                            pseudocount), "pcb_input_dist_em");
}
