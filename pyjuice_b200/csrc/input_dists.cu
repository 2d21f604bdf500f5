// Bernoulli and Gaussian input layers: forward log-probabilities, parameter flows (the
// distributions' sufficient statistics weighted by node flows) and the EM update.
//   Bernoulli (kind 1): one parameter p per node; x > 0 has probability p. Flows: slot 0
//     collects the flow of samples with x > 0, slot 1 the others
//     (src/pyjuice/nodes/distributions/bernoulli.py:64-102).
//   Gaussian (kind 2): parameters (mu, sigma) per node, log N(x; mu, sigma). Flows: slots
//     (sum f x, sum f x^2, sum f); a missing value contributes its expectation (mu f,
//     (sigma^2 + mu^2) f, f). EM moment-matches the updated expectation parameters, with
//     sigma clamped below at min_sigma (gaussian.py:87-170).
//   DiscreteLogistic (kind 3): parameters (mu, s) per node; x is a bin index of num_cats
//     equal bins of [lo, hi) (the outer bins open to -inf / +inf), probability
//     sigma((x + 1) w + lo) - sigma(x w + lo) with sigma(v) = 1 / (1 + exp((mu - v) / s)),
//     log clamped at -1000. Flows: slots (sum f m, sum f m^2, sum f) with m the bin's
//     midpoint; a missing value contributes (mu f, (s^2 pi^2 / 3 + mu^2) f, f). EM as for
//     the Gaussian on the standard deviation s pi / sqrt(3), at least min_std
//     (discrete_logistic.py:81-202).
// Data: FP32 [num_vars, data_ld] (Bernoulli reads x > 0). Missing values (mask as in
// pcb_input_cat_fwd) give log 1 in the forward pass. Per-node metadata (meta, indexed by
// the node's layer-local id): Gaussian min_sigma (one float, EM only); DiscreteLogistic
// (lo, hi, num_cats, min_std) (four floats).
#include <algorithm>

#include "common.cuh"

namespace {

constexpr float kLog2Pi = 1.8378770664093453f;
constexpr double kPiSq3 = 3.289868133696453;        // pi^2 / 3: variance of the unit logistic
constexpr double kStdPerScale = 1.8137993642342178;  // pi / sqrt(3)

__device__ __forceinline__ float logistic_cdf(float mu, float s, float v) { return 1.f / (1.f + expf((mu - v) / s)); }

__global__ void __launch_bounds__(256)
dist_fwd_kernel(int kind, const float* __restrict__ data, int64_t data_ld, const float* __restrict__ params,
                const int* __restrict__ vids, const int* __restrict__ s_pids, const float* __restrict__ meta,
                int num_nodes, int node_offset, float* __restrict__ nm, int64_t ld, int B,
                const uint8_t* __restrict__ miss, int64_t m_sb, int64_t m_sv) {
    pcb::pdl_begin();
    for (int n = blockIdx.y; n < num_nodes; n += gridDim.y) {
    const int64_t v = vids[n];
    const int64_t sp = s_pids[n];
    const float a = params[sp];
    const float s = kind >= 2 ? params[sp + 1] : 0.f;
    float lo = 0.f, w = 0.f, last = 0.f;
    if (kind == 3) {
        lo = meta[4 * (int64_t)n];
        last = meta[4 * (int64_t)n + 2] - 1.f;
        w = (meta[4 * (int64_t)n + 1] - lo) / meta[4 * (int64_t)n + 2];
    }
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
        float r;
        if (miss && miss[(int64_t)b * m_sb + v * m_sv]) {
            r = 0.f;
        } else {
            const float x = data[v * data_ld + b];
            if (kind == 1) {
                r = logf(x > 0.f ? a : 1.f - a);
            } else if (kind == 3) {
                const float vlow = x * w + lo;
                const float hi_cdf = x == last ? 1.f : logistic_cdf(a, s, vlow + w);
                const float lo_cdf = x == 0.f ? 0.f : logistic_cdf(a, s, vlow);
                r = fmaxf(logf(hi_cdf - lo_cdf), -1000.f);
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
                const int* __restrict__ s_pfids, const float* __restrict__ meta, int num_nodes, int node_offset,
                float* __restrict__ pf, bool logspace, const uint8_t* __restrict__ miss, int64_t m_sb, int64_t m_sv,
                bool atomic) {
    pcb::pdl_begin();
    const int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (n >= num_nodes) return;
    const int64_t v = vids[n];
    const int64_t sp = s_pids[n];
    const float mu = params[sp];
    const float sg = kind >= 2 ? params[sp + 1] : 0.f;
    // the missing-value second moment, and the bin midpoint as mid0 + x w
    const float m2 = kind == 3 ? (float)(sg * sg * kPiSq3) + mu * mu : sg * sg + mu * mu;
    float mid0 = 0.f, w = 0.f;
    if (kind == 3) {
        w = (meta[4 * (int64_t)n + 1] - meta[4 * (int64_t)n]) / meta[4 * (int64_t)n + 2];
        mid0 = meta[4 * (int64_t)n] + 0.5f * w;
    }
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
            s1 += m2 * f;
            s2 += f;
        } else {
            float x = data[v * data_ld + b];
            if (kind == 3) x = x * w + mid0;
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
               const int* __restrict__ s_pfids, const float* __restrict__ meta,
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
        const double scale = kind == 3 ? kStdPerScale : 1.0;  // standard deviation per unit of parameter 2
        const double mu = params[sp], sg = params[sp + 1] * scale;
        const double t1 = pf[sf] / ((double)pf[sf + 2] + 1e-10);
        const double t2 = pf[sf + 1] / ((double)pf[sf + 2] + 1e-10);
        const double u1 = (1.0 - step) * mu + step * t1;
        const double u2 = (1.0 - step) * (sg * sg + mu * mu) + step * t2;
        const double var = u2 - u1 * u1;
        const double ms = kind == 3 ? meta[4 * (int64_t)n + 3] : meta[n];
        params[sp] = (float)u1;
        params[sp + 1] = (float)((var < ms * ms ? ms : sqrt(var)) / scale);
    }
}

}  // namespace

extern "C" int pcb_input_dist_fwd(int32_t kind, const float* data, int64_t data_ld, const float* params,
                                  const int32_t* vids, const int32_t* s_pids, const float* meta, int32_t num_nodes,
                                  int32_t node_offset, float* node_mars, int64_t ld, int32_t B, const uint8_t* missing,
                                  int64_t miss_sb, int64_t miss_sv, void* stream) {
    if (kind < 1 || kind > 3 || (kind == 3 && !meta) || !data || !params || !vids || !s_pids || !node_mars || B <= 0 ||
        ld < B || data_ld < B || num_nodes < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_input_dist_fwd: bad arguments");
    if (num_nodes == 0) return PCB_OK;
    const unsigned gx = (unsigned)std::min<int64_t>(pcb::cdiv(B, 256), 64);
    const unsigned gy = (unsigned)std::min<int64_t>(num_nodes, 65535);
    return pcb::launch_status(pcb::launch_k(dist_fwd_kernel, dim3(gx, gy), dim3(256), 0,
                                            pcb::as_stream(stream), 1u, (int)kind, data, data_ld, params, vids, s_pids,
                                            meta, num_nodes, node_offset, node_mars, ld, B, missing, miss_sb, miss_sv),
                              "pcb_input_dist_fwd");
}

extern "C" int pcb_input_dist_bwd(int32_t kind, const float* data, int64_t data_ld, const float* node_flows, int64_t ld,
                                  int32_t B, const float* params, const int32_t* vids, const int32_t* s_pids,
                                  const int32_t* s_pfids, const float* meta, int32_t num_nodes, int32_t node_offset,
                                  float* param_flows, int32_t logspace_flows, const uint8_t* missing, int64_t miss_sb,
                                  int64_t miss_sv, int32_t atomic, void* stream) {
    if (kind < 1 || kind > 3 || (kind == 3 && !meta) || !data || !node_flows || !params || !vids || !s_pids || !s_pfids || !param_flows ||
        B <= 0 || ld < B || data_ld < B || num_nodes < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_input_dist_bwd: bad arguments");
    if (num_nodes == 0) return PCB_OK;
    return pcb::launch_status(pcb::launch_k(dist_bwd_kernel, dim3((unsigned)pcb::cdiv((int64_t)num_nodes * 32, 256)),
                                            dim3(256), 0, pcb::as_stream(stream), 1u, (int)kind, data, data_ld,
                                            node_flows, ld, B, params, vids, s_pids, s_pfids, meta, num_nodes, node_offset,
                                            param_flows, logspace_flows != 0, missing, miss_sb, miss_sv, atomic != 0),
                              "pcb_input_dist_bwd");
}

extern "C" int pcb_input_dist_em(int32_t kind, float* params, const float* param_flows, const int32_t* s_pids,
                                 const int32_t* s_pfids, const float* meta, const int32_t* source_nids,
                                 int32_t num_source_nodes, double step_size, double pseudocount, void* stream) {
    if (kind < 1 || kind > 3 || !params || !param_flows || !s_pids || !s_pfids || !source_nids ||
        (kind >= 2 && !meta) || num_source_nodes < 0 || !(step_size > 0.0 && step_size <= 1.0))
        return pcb::set_error(PCB_E_ARG, "pcb_input_dist_em: bad arguments");
    if (num_source_nodes == 0) return PCB_OK;
    return pcb::launch_status(pcb::launch_k(dist_em_kernel, dim3((unsigned)pcb::cdiv(num_source_nodes, 256)),
                                            dim3(256), 0, pcb::as_stream(stream), 1u, (int)kind, params, param_flows,
                                            s_pids, s_pfids, meta, source_nids, num_source_nodes, step_size,
                                            pseudocount), "pcb_input_dist_em");
}
