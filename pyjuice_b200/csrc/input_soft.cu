// Categorical input layers with soft evidence, and the backward contractions that turn node
// flows into per-category quantities:
//   * soft-evidence forward: node_mars[n, b] = min(log sum_k E[b, v, k] theta[n, k], 0)
//     (src/pyjuice/queries/conditional.py:25-68, 108-111);
//   * evidence backward: out[b, t, k] = sum_{n over the nodes of variable v_t} W[n, b] theta[n, k]
//     with W = node flows (the reference's conditional query, conditional.py:241-336, before its
//     normalisation over k), or W = node flows / exp(node_mars) (the adjoint
//     d LL / d E[b, v, k] of the soft-evidence forward; no reference counterpart).
// Both are small dense contractions per variable, over the categories (forward) or the
// variable's nodes (backward): 64 x 64 output tiles, operands staged through shared memory
// in chunks of 32, FP32 FMA with 4 x 4 register tiles per thread.
#include "common.cuh"

namespace {

constexpr int kT = 64;   // output tile (rows and columns)
constexpr int kC = 32;   // contraction chunk

__global__ void __launch_bounds__(256)
soft_fwd_kernel(const float* __restrict__ evid, int64_t e_sb, int64_t e_sv, int64_t e_sk,
                const float* __restrict__ params, const int* __restrict__ grp_var, const int* __restrict__ grp_node0,
                const int* __restrict__ grp_count, const int* __restrict__ grp_ncats, const int* __restrict__ s_pids,
                int node_offset, float* __restrict__ nm, int64_t ld, int B, const uint8_t* __restrict__ miss,
                int64_t m_sb, int64_t m_sv) {
    pcb::pdl_begin();
    __shared__ float sT[kC][kT + 1];  // [k][node]
    __shared__ float sE[kC][kT + 1];  // [k][sample]
    const int g = blockIdx.x;
    const int n0 = blockIdx.y * kT;
    const int b0 = blockIdx.z * kT;
    const int cnt = grp_count[g];
    if (n0 >= cnt) return;
    const int K = grp_ncats[g];
    const int64_t v = grp_var[g];
    const int node0 = grp_node0[g];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += kC) {
        for (int idx = tid; idx < kT * kC; idx += 256) {
            const int r = idx / kC, kk = idx % kC;
            const int n = n0 + r, b = b0 + r, k = k0 + kk;
            sT[kk][r] = (n < cnt && k < K) ? params[(int64_t)s_pids[node0 + n] + k] : 0.f;
            sE[kk][r] = (b < B && k < K) ? evid[(int64_t)b * e_sb + v * e_sv + (int64_t)k * e_sk] : 0.f;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < kC; ++kk) {
            float a[4], e[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sT[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) e[j] = sE[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], e[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int n = n0 + ty * 4 + i;
        if (n >= cnt) continue;
        float* row = nm + ((int64_t)node_offset + node0 + n) * ld;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int b = b0 + tx * 4 + j;
            if (b >= B) continue;
            const bool missing = miss && miss[(int64_t)b * m_sb + v * m_sv];
            row[b] = missing ? 0.f : fminf(logf(acc[i][j]), 0.f);
        }
    }
}

__global__ void __launch_bounds__(256)
evidence_bwd_kernel(const float* __restrict__ nf, const float* __restrict__ nm, int64_t ld, int B,
                    const float* __restrict__ params, const int* __restrict__ tgt_ptr, const int* __restrict__ tgt_nodes,
                    const int* __restrict__ s_pids, const int* __restrict__ ncats, int node_offset, int T, int Kmax,
                    int mode, float* __restrict__ out) {
    pcb::pdl_begin();
    __shared__ float sW[kC][kT + 1];  // [node][sample]
    __shared__ float sT[kC][kT + 1];  // [node][category]
    const int t = blockIdx.x;
    const int b0 = blockIdx.y * kT;
    const int k0 = blockIdx.z * kT;
    const int p0 = tgt_ptr[t], p1 = tgt_ptr[t + 1];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;  // tx: 4 categories, ty: 4 samples
    float acc[4][4] = {};
    for (int c0 = p0; c0 < p1; c0 += kC) {
        for (int idx = tid; idx < kT * kC; idx += 256) {
            const int r = idx / kT, col = idx % kT;  // r: node of the chunk, col: sample / category
            const int p = c0 + r;
            float w = 0.f, th = 0.f;
            if (p < p1) {
                const int n = tgt_nodes[p];
                const int b = b0 + col, k = k0 + col;
                if (b < B) {
                    const int64_t o = ((int64_t)node_offset + n) * ld + b;
                    w = nf[o];
                    if (mode == 1) {
                        const float m = nm[o];
                        w = (m == -INFINITY) ? 0.f : w * expf(-m);
                    }
                }
                if (k < ncats[n]) th = params[(int64_t)s_pids[n] + k];
            }
            sW[r][col] = w;
            sT[r][col] = th;
        }
        __syncthreads();
#pragma unroll 8
        for (int r = 0; r < kC; ++r) {
            float a[4], c[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sW[r][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) c[j] = sT[r][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], c[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int b = b0 + ty * 4 + i;
        if (b >= B) continue;
        float* row = out + ((int64_t)b * T + t) * Kmax;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k = k0 + tx * 4 + j;
            if (k < Kmax) row[k] = acc[i][j];
        }
    }
}

}  // namespace

extern "C" int pcb_input_cat_soft_fwd(const float* evidence, int64_t e_sb, int64_t e_sv, int64_t e_sk,
                                      const float* params, const int32_t* grp_var, const int32_t* grp_node0,
                                      const int32_t* grp_count, const int32_t* grp_ncats, int32_t num_groups,
                                      int32_t max_group_nodes, const int32_t* s_pids, int32_t node_offset,
                                      float* node_mars, int64_t ld, int32_t B, const uint8_t* missing, int64_t miss_sb,
                                      int64_t miss_sv, void* stream) {
    if (!evidence || !params || !grp_var || !grp_node0 || !grp_count || !grp_ncats || !s_pids || !node_mars || B <= 0 ||
        ld < B || num_groups < 0 || max_group_nodes < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_input_cat_soft_fwd: bad arguments");
    if (num_groups == 0 || max_group_nodes == 0) return PCB_OK;
    const int64_t gy = pcb::cdiv(max_group_nodes, kT), gz = pcb::cdiv(B, kT);
    if (gy > 65535 || gz > 65535) return pcb::set_error(PCB_E_ARG, "pcb_input_cat_soft_fwd: grid too large");
    return pcb::launch_status(
        pcb::launch_k(soft_fwd_kernel, dim3((unsigned)num_groups, (unsigned)gy, (unsigned)gz), dim3(256), 0,
                      pcb::as_stream(stream), 1u, evidence, e_sb, e_sv, e_sk, params, grp_var, grp_node0, grp_count,
                      grp_ncats, s_pids, node_offset, node_mars, ld, B, missing, miss_sb, miss_sv),
        "pcb_input_cat_soft_fwd");
}

extern "C" int pcb_input_cat_evidence_bwd(const float* node_flows, const float* node_mars, int64_t ld, int32_t B,
                                          const float* params, const int32_t* tgt_ptr, const int32_t* tgt_nodes,
                                          int32_t num_targets, const int32_t* s_pids, const int32_t* ncats,
                                          int32_t node_offset, int32_t max_ncats, int32_t mode, float* out,
                                          void* stream) {
    if (!node_flows || !params || !tgt_ptr || !tgt_nodes || !s_pids || !ncats || !out || B <= 0 || ld < B ||
        num_targets < 0 || max_ncats <= 0 || mode < 0 || mode > 1 || (mode == 1 && !node_mars))
        return pcb::set_error(PCB_E_ARG, "pcb_input_cat_evidence_bwd: bad arguments");
    if (num_targets == 0) return PCB_OK;
    const int64_t gy = pcb::cdiv(B, kT), gz = pcb::cdiv(max_ncats, kT);
    if (gy > 65535 || gz > 65535) return pcb::set_error(PCB_E_ARG, "pcb_input_cat_evidence_bwd: grid too large");
    return pcb::launch_status(
        pcb::launch_k(evidence_bwd_kernel, dim3((unsigned)num_targets, (unsigned)gy, (unsigned)gz), dim3(256), 0,
                      pcb::as_stream(stream), 1u, node_flows, node_mars, ld, B, params, tgt_ptr, tgt_nodes, s_pids,
                      ncats, node_offset, num_targets, max_ncats, mode, out),
        "pcb_input_cat_evidence_bwd");
}
