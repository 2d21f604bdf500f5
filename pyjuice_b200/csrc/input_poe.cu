// SoftEvidenceCategorical input layers: categorical nodes whose distribution is multiplied by
// per-sample external evidence (a product of experts), with the evidence given as log-weights
// L[b, u, k] over categories (u = the variable's index among the layer's variables):
//   node_mars[n, b] = log theta[n, x] + L[b, u, x] - log Z[n, b],
//   Z[n, b] = sum_{k < K} theta[n, k] exp(L[b, u, k]),
// and the gradient of the node values with respect to the evidence, weighted by node flows f
// (linear or log space):
//   G[b, u, k] += sum_n f[n, b] ([k == x] - theta[n, k] exp(L[b, u, k]) / Z[n, b]).
// Dense evidence covers categories 0..K-1; sparse evidence gives, per (b, u), K category ids
// with their log-weights. Replaces the fw_kernel, bk_params_kernel and bk_softevi_kernel of
// src/pyjuice/nodes/distributions/softevi_categorical.py:21-661 (the parameter flows are the
// categorical flow histogram, pcb_input_cat_bwd).
//
// Dense forward: per variable, 64 nodes x 64 samples per CTA, the contraction over categories
// staged through shared memory in chunks of 32 with the per-sample maximum of L subtracted
// before the exponential (so Z never overflows). Dense backward: per variable, 64 samples x
// 64 categories per CTA, contracting over the variable's nodes with weights
// exp(log f - log Z - m_b) <= 1 (m_b: the per-sample maximum of log f - log Z over the nodes);
// log Z is recovered from the forward values as log theta[n, x] + L[b, u, x] - node_mars.
// Each output element has one writer (one CTA per variable and tile), so G is accumulated
// without atomics. Sparse forms: one thread per (node, sample), resp. one CTA per (variable,
// sample) with the nodes' weights in shared memory.
#include "common.cuh"

namespace {

constexpr int kT = 64;   // output tile (rows and columns)
constexpr int kC = 32;   // contraction chunk

struct PoeArgs {
    const int64_t* data;     // [num_vars, data_ld] category of each (variable, sample)
    int64_t data_ld;
    const float* logp;       // evidence log-weights [B, U, K] (k contiguous)
    const int64_t* cat_ids;  // sparse evidence: category ids [B, U, K], or NULL (dense)
    int64_t e_sb, e_su;
    int K;
    const float* params;
    const int* grp_var;      // per group (run of nodes of one variable): the variable
    const int* grp_lvid;     //   its index u in the evidence
    const int* grp_node0;    //   first node (layer-local)
    const int* grp_count;    //   number of nodes
    const int* s_pids;
    const int* ncats;        // per node
    int node_offset;
    int64_t ld;
    int B;
};

__device__ __forceinline__ float safe_log_theta(const PoeArgs& a, int n, int64_t x) {
    return (x >= 0 && x < a.ncats[n]) ? logf(a.params[(int64_t)a.s_pids[n] + x]) : -INFINITY;
}

// Log-weight of category x in the evidence of (b, u): dense L[b, u, x] (x < K), or the entry
// whose id is x (last match), else -inf.
__device__ __forceinline__ float evidence_of(const PoeArgs& a, int b, int u, int64_t x) {
    const int64_t row = (int64_t)b * a.e_sb + (int64_t)u * a.e_su;
    if (!a.cat_ids) return (x >= 0 && x < a.K) ? a.logp[row + x] : NAN;
    float r = -INFINITY;
    for (int j = 0; j < a.K; ++j)
        if (a.cat_ids[row + j] == x) r = a.logp[row + j];
    return r;
}

__global__ void __launch_bounds__(256)
poe_fwd_dense_kernel(PoeArgs a, float* __restrict__ nm, const uint8_t* __restrict__ miss, int64_t m_sb,
                     int64_t m_sv) {
    pcb::pdl_begin();
    __shared__ float sT[kC][kT + 1];  // [k][node]
    __shared__ float sE[kC][kT + 1];  // [k][sample]
    __shared__ float sM[kT];          // per-sample maximum of L
    const int g = blockIdx.x;
    const int n0 = blockIdx.y * kT;
    const int b0 = blockIdx.z * kT;
    const int cnt = a.grp_count[g];
    if (n0 >= cnt) return;
    const int64_t v = a.grp_var[g];
    const int u = a.grp_lvid[g];
    const int node0 = a.grp_node0[g];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int c = warp; c < kT; c += 8) {  // one warp per sample column
        const int b = b0 + c;
        float m = -INFINITY;
        if (b < a.B) {
            const float* row = a.logp + (int64_t)b * a.e_sb + (int64_t)u * a.e_su;
            for (int k = lane; k < a.K; k += 32) m = fmaxf(m, row[k]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) sM[c] = m;
    }
    __syncthreads();
    const int tx = tid & 15, ty = tid >> 4;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < a.K; k0 += kC) {
        for (int idx = tid; idx < kT * kC; idx += 256) {
            const int r = idx / kC, kk = idx % kC;
            const int n = n0 + r, b = b0 + r, k = k0 + kk;
            sT[kk][r] = (n < cnt && k < a.K) ? a.params[(int64_t)a.s_pids[node0 + n] + k] : 0.f;
            float e = 0.f;
            if (b < a.B && k < a.K && sM[r] != -INFINITY)
                e = expf(a.logp[(int64_t)b * a.e_sb + (int64_t)u * a.e_su + k] - sM[r]);
            sE[kk][r] = e;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < kC; ++kk) {
            float t[4], e[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) t[i] = sT[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) e[j] = sE[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(t[i], e[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int n = n0 + ty * 4 + i;
        if (n >= cnt) continue;
        float* row = nm + ((int64_t)a.node_offset + node0 + n) * a.ld;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int b = b0 + tx * 4 + j;
            if (b >= a.B) continue;
            if (miss && miss[(int64_t)b * m_sb + v * m_sv]) {
                row[b] = 0.f;
                continue;
            }
            const int64_t x = a.data[v * a.data_ld + b];
            const float lz = logf(acc[i][j]) + sM[tx * 4 + j];
            row[b] = safe_log_theta(a, node0 + n, x) + evidence_of(a, b, u, x) - lz;
        }
    }
}

__global__ void __launch_bounds__(256)
poe_fwd_sparse_kernel(PoeArgs a, const int* __restrict__ node_grp, int num_nodes, float* __restrict__ nm,
                      const uint8_t* __restrict__ miss, int64_t m_sb, int64_t m_sv) {
    pcb::pdl_begin();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)num_nodes * a.B) return;
    const int n = (int)(i / a.B), b = (int)(i % a.B);
    const int g = node_grp[n];
    const int64_t v = a.grp_var[g];
    const int u = a.grp_lvid[g];
    float* out = nm + ((int64_t)a.node_offset + n) * a.ld + b;
    if (miss && miss[(int64_t)b * m_sb + v * m_sv]) {
        *out = 0.f;
        return;
    }
    const int64_t row = (int64_t)b * a.e_sb + (int64_t)u * a.e_su;
    float m = -INFINITY, s = 0.f;  // online log-sum-exp of log theta[n, id_j] + L_j
    for (int j = 0; j < a.K; ++j) {
        const float t = safe_log_theta(a, n, a.cat_ids[row + j]) + a.logp[row + j];
        if (t == -INFINITY) continue;
        if (t > m) {
            s = s * expf(m - t) + 1.f;
            m = t;
        } else {
            s += expf(t - m);
        }
    }
    const int64_t x = a.data[v * a.data_ld + b];
    *out = safe_log_theta(a, n, x) + evidence_of(a, b, u, x) - (logf(s) + m);
}

// log Z[n, b] from the forward values, and the node flow in log space.
__device__ __forceinline__ void flow_terms(const PoeArgs& a, const float* nf, const float* nm, bool logspace, int n,
                                           int b, int64_t x, float lex, float& log_f, float& log_z) {
    const int64_t o = ((int64_t)a.node_offset + n) * a.ld + b;
    const float f = nf[o];
    log_f = logspace ? f : logf(f);
    log_z = safe_log_theta(a, n, x) + lex - nm[o];
}

__global__ void __launch_bounds__(256)
poe_bwd_dense_kernel(PoeArgs a, const float* __restrict__ nf, const float* __restrict__ nm, bool logspace,
                     float* __restrict__ grad, int64_t g_sb, int64_t g_su) {
    pcb::pdl_begin();
    __shared__ float sW[kC][kT + 1];  // [node][sample]
    __shared__ float sT[kC][kT + 1];  // [node][category]
    __shared__ float sMax[kT], sFsum[kT], sLex[kT];
    __shared__ int64_t sX[kT];
    const int g = blockIdx.x;
    const int b0 = blockIdx.y * kT;
    const int k0 = blockIdx.z * kT;
    const int64_t v = a.grp_var[g];
    const int u = a.grp_lvid[g];
    const int node0 = a.grp_node0[g], cnt = a.grp_count[g];
    const int tid = threadIdx.x;
    // per sample: its category, its evidence, the maximum of log f - log Z over the nodes and
    // the sum of the flows
    if (tid < kT) {
        const int b = b0 + tid;
        float mx = -INFINITY, fs = 0.f, lex = 0.f;
        int64_t x = -1;
        if (b < a.B) {
            x = a.data[v * a.data_ld + b];
            lex = evidence_of(a, b, u, x);
            for (int c = 0; c < cnt; ++c) {
                float lf, lz;
                flow_terms(a, nf, nm, logspace, node0 + c, b, x, lex, lf, lz);
                if (lf != -INFINITY) {
                    mx = fmaxf(mx, lf - lz);
                    fs += expf(lf);
                }
            }
        }
        sMax[tid] = mx;
        sFsum[tid] = fs;
        sLex[tid] = lex;
        sX[tid] = x;
    }
    __syncthreads();
    const int tx = tid & 15, ty = tid >> 4;  // tx: 4 categories, ty: 4 samples
    float acc[4][4] = {};
    for (int c0 = 0; c0 < cnt; c0 += kC) {
        for (int idx = tid; idx < kT * kC; idx += 256) {
            const int r = idx / kT, col = idx % kT;  // r: node of the chunk, col: sample / category
            const int c = c0 + r;
            float w = 0.f, th = 0.f;
            if (c < cnt) {
                const int n = node0 + c;
                const int b = b0 + col, k = k0 + col;
                if (b < a.B && sMax[col] != -INFINITY) {
                    float lf, lz;
                    flow_terms(a, nf, nm, logspace, n, b, sX[col], sLex[col], lf, lz);
                    w = lf == -INFINITY ? 0.f : expf(lf - lz - sMax[col]);
                }
                if (k < a.K) th = a.params[(int64_t)a.s_pids[n] + k];
            }
            sW[r][col] = w;
            sT[r][col] = th;
        }
        __syncthreads();
#pragma unroll 8
        for (int r = 0; r < kC; ++r) {
            float w[4], t[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) w[i] = sW[r][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) t[j] = sT[r][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(w[i], t[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int bl = ty * 4 + i, b = b0 + bl;
        if (b >= a.B) continue;
        const float* lrow = a.logp + (int64_t)b * a.e_sb + (int64_t)u * a.e_su;
        float* grow = grad + (int64_t)b * g_sb + (int64_t)u * g_su;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k = k0 + tx * 4 + j;
            if (k >= a.K) continue;
            float d = sMax[bl] == -INFINITY ? 0.f : -acc[i][j] * expf(sMax[bl] + lrow[k]);
            if (k == sX[bl]) d += sFsum[bl];
            grow[k] += d;
        }
    }
}

__global__ void __launch_bounds__(256)
poe_bwd_sparse_kernel(PoeArgs a, const float* __restrict__ nf, const float* __restrict__ nm, bool logspace,
                      float* __restrict__ grad, int64_t g_sb, int64_t g_su) {
    pcb::pdl_begin();
    extern __shared__ float sW[];  // [nodes of the variable]
    __shared__ float sMax, sFsum;
    const int g = blockIdx.x, b = blockIdx.y;
    const int64_t v = a.grp_var[g];
    const int u = a.grp_lvid[g];
    const int node0 = a.grp_node0[g], cnt = a.grp_count[g];
    const int64_t x = a.data[v * a.data_ld + b];
    const float lex = evidence_of(a, b, u, x);
    const int tid = threadIdx.x;
    if (tid == 0) {
        float mx = -INFINITY, fs = 0.f;
        for (int c = 0; c < cnt; ++c) {
            float lf, lz;
            flow_terms(a, nf, nm, logspace, node0 + c, b, x, lex, lf, lz);
            if (lf != -INFINITY) {
                mx = fmaxf(mx, lf - lz);
                fs += expf(lf);
            }
        }
        sMax = mx;
        sFsum = fs;
    }
    __syncthreads();
    for (int c = tid; c < cnt; c += blockDim.x) {
        float lf, lz;
        flow_terms(a, nf, nm, logspace, node0 + c, b, x, lex, lf, lz);
        sW[c] = (lf == -INFINITY || sMax == -INFINITY) ? 0.f : expf(lf - lz - sMax);
    }
    __syncthreads();
    const int64_t row = (int64_t)b * a.e_sb + (int64_t)u * a.e_su;
    float* grow = grad + (int64_t)b * g_sb + (int64_t)u * g_su;
    for (int j = tid; j < a.K; j += blockDim.x) {
        const int64_t id = a.cat_ids[row + j];
        float s = 0.f;
        for (int c = 0; c < cnt; ++c) {
            const int n = node0 + c;
            if (id >= 0 && id < a.ncats[n]) s = fmaf(sW[c], a.params[(int64_t)a.s_pids[n] + id], s);
        }
        float d = sMax == -INFINITY ? 0.f : -s * expf(sMax + a.logp[row + j]);
        if (id == x) d += sFsum;
        grow[j] += d;
    }
}

bool poe_args_ok(const PoeArgs& a) {
    return a.data && a.data_ld >= a.B && a.logp && a.e_sb >= 0 && a.e_su >= 0 && a.K > 0 && a.params && a.grp_var &&
           a.grp_lvid && a.grp_node0 && a.grp_count && a.s_pids && a.ncats && a.B > 0 && a.ld >= a.B;
}

}  // namespace

extern "C" int pcb_input_poe_fwd(const int64_t* data, int64_t data_ld, const float* evidence_logp,
                                 const int64_t* cat_ids, int64_t e_sb, int64_t e_su, int32_t K, const float* params,
                                 const int32_t* grp_var, const int32_t* grp_lvid, const int32_t* grp_node0,
                                 const int32_t* grp_count, int32_t num_groups, int32_t max_group_nodes,
                                 const int32_t* node_grp, int32_t num_nodes, const int32_t* s_pids,
                                 const int32_t* ncats, int32_t node_offset, float* node_mars, int64_t ld, int32_t B,
                                 const uint8_t* missing, int64_t miss_sb, int64_t miss_sv, void* stream) {
    const PoeArgs a{data, data_ld, evidence_logp, cat_ids, e_sb, e_su, K, params, grp_var, grp_lvid, grp_node0,
                    grp_count, s_pids, ncats, node_offset, ld, B};
    if (!poe_args_ok(a) || !node_mars || num_groups < 0 || max_group_nodes < 0 || num_nodes < 0 ||
        (cat_ids && !node_grp))
        return pcb::set_error(PCB_E_ARG, "pcb_input_poe_fwd: bad arguments");
    if (num_groups == 0 || max_group_nodes == 0) return PCB_OK;
    if (cat_ids) {
        const int64_t total = (int64_t)num_nodes * B;
        return pcb::launch_status(
            pcb::launch_k(poe_fwd_sparse_kernel, dim3((unsigned)pcb::cdiv(total, 256)), dim3(256), 0,
                          pcb::as_stream(stream), 1u, a, node_grp, num_nodes, node_mars, missing, miss_sb, miss_sv),
            "pcb_input_poe_fwd");
    }
    const int64_t gy = pcb::cdiv(max_group_nodes, kT), gz = pcb::cdiv(B, kT);
    if (gy > 65535 || gz > 65535) return pcb::set_error(PCB_E_ARG, "pcb_input_poe_fwd: grid too large");
    return pcb::launch_status(
        pcb::launch_k(poe_fwd_dense_kernel, dim3((unsigned)num_groups, (unsigned)gy, (unsigned)gz), dim3(256), 0,
                      pcb::as_stream(stream), 1u, a, node_mars, missing, miss_sb, miss_sv),
        "pcb_input_poe_fwd");
}

extern "C" int pcb_input_poe_evidence_bwd(const int64_t* data, int64_t data_ld, const float* node_flows,
                                          const float* node_mars, int64_t ld, int32_t B, int32_t logspace_flows,
                                          const float* evidence_logp, const int64_t* cat_ids, int64_t e_sb,
                                          int64_t e_su, int32_t K, float* evidence_grad, int64_t g_sb, int64_t g_su,
                                          const float* params, const int32_t* grp_var, const int32_t* grp_lvid,
                                          const int32_t* grp_node0, const int32_t* grp_count, int32_t num_groups,
                                          int32_t max_group_nodes, const int32_t* s_pids, const int32_t* ncats,
                                          int32_t node_offset, void* stream) {
    const PoeArgs a{data, data_ld, evidence_logp, cat_ids, e_sb, e_su, K, params, grp_var, grp_lvid, grp_node0,
                    grp_count, s_pids, ncats, node_offset, ld, B};
    if (!poe_args_ok(a) || !node_flows || !node_mars || !evidence_grad || g_sb < 0 || g_su < 0 || num_groups < 0 ||
        max_group_nodes < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_input_poe_evidence_bwd: bad arguments");
    if (num_groups == 0 || max_group_nodes == 0) return PCB_OK;
    if (cat_ids) {
        const size_t smem = (size_t)max_group_nodes * sizeof(float);
        if (smem > 48 * 1024 || B > 65535)
            return pcb::set_error(PCB_E_ARG, "pcb_input_poe_evidence_bwd: too many nodes per variable or samples");
        return pcb::launch_status(
            pcb::launch_k(poe_bwd_sparse_kernel, dim3((unsigned)num_groups, (unsigned)B), dim3(256), smem,
                          pcb::as_stream(stream), 1u, a, node_flows, node_mars, logspace_flows != 0, evidence_grad,
                          g_sb, g_su),
            "pcb_input_poe_evidence_bwd");
    }
    const int64_t gy = pcb::cdiv(B, kT), gz = pcb::cdiv(K, kT);
    if (gy > 65535 || gz > 65535) return pcb::set_error(PCB_E_ARG, "pcb_input_poe_evidence_bwd: grid too large");
    return pcb::launch_status(
        pcb::launch_k(poe_bwd_dense_kernel, dim3((unsigned)num_groups, (unsigned)gy, (unsigned)gz), dim3(256), 0,
                      pcb::as_stream(stream), 1u, a, node_flows, node_mars, logspace_flows != 0, evidence_grad, g_sb,
                      g_su),
        "pcb_input_poe_evidence_bwd");
}
