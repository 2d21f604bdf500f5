// Sum layers under the MPE and GeneralLL propagation algorithms, and the backward pass in
// log-space, with negated parameter flows or with accumulated child flows: plain FP32
// kernels over the same tile tables as the log-likelihood kernels. These modes serve
// queries (most probable explanations, tempered likelihoods, log-space flows for
// gradients) rather than the EM training step, so the kernels favour exactness over
// throughput: one thread per (row, sample), the 32 lanes of a warp on consecutive samples
// (coalesced row reads), accurate expf / logf.
//
// Propagation algorithms (alg): 0 LL, 1 MPE, 2 GeneralLL(alpha):
//   forward   LL         nm = log sum_k w_k exp(e_k)
//             MPE        nm = max_k (log w_k + e_k)
//             GeneralLL  nm = (log(sum_k w_k^alpha exp(alpha (e_k - m)) + 1e-24) + alpha m) / alpha,  m = max_k e_k
//   element flows of child c (parents n, weight w = theta[n, c], f = flow of n, m = its value):
//             LL         sum_n f w exp(e_c - m_n)                 (log space: logsumexp_n (f + log w + e_c - m_n))
//             MPE        sum_n [|log w + e_c - m_n| < 1e-6] f     (log space: logsumexp over the same parents)
//             GeneralLL  sum_n f w^alpha exp(alpha (e_c - m_n))   (log space: logsumexp_n (f + alpha (log w + e_c - m_n)))
//   parameter flows of edge (n, c), summed over the batch:
//             LL, GeneralLL  w sum_b f exp(e_c - m_n)             (log space: w sum_b exp(f + e_c - m_n), exp(f) where m_n = -inf)
//             MPE            sum_b [|log w + e_c - m_n| < 1e-6] f (log space: exp(f))
// Reference: src/pyjuice/layer/sum_layer.py:454-568 (forward), 1572-1730 (element flows),
// 2052-2169 and 2795-2902 (parameter flows), 3068-3127 (the PyTorch restatement).
#include "common.cuh"

namespace {

constexpr int kRowsPerCta = 8;  // one row per warp

__device__ __forceinline__ float lae(float a, float b) {  // log(exp(a) + exp(b))
    if (a == -INFINITY) return b;
    if (b == -INFINITY) return a;
    const float m = fmaxf(a, b);
    return m + log1pf(expf(-fabsf(a - b)));
}

__device__ __forceinline__ float tile_weight(const float* __restrict__ params, const int* __restrict__ kw,
                                             const PcbLseTile& t, int k, int r, int rpb_log2, int w_stride) {
    const int64_t idx = (int64_t)kw[t.k_off + k] + t.w_add + (int64_t)(r >> rpb_log2) * t.g_stride +
                        (int64_t)(r & ((1 << rpb_log2) - 1)) * w_stride;
    return params[idx];
}

__global__ void __launch_bounds__(32 * kRowsPerCta)
sum_fwd_generic_kernel(const float* __restrict__ em, float* __restrict__ nm, int64_t ld, int B,
                       const float* __restrict__ params, const PcbLseTile* __restrict__ tiles, int rpb_log2,
                       const int* __restrict__ krow, const int* __restrict__ kw, int w_stride, int alg, float alpha) {
    pcb::pdl_begin();
    const PcbLseTile t = tiles[blockIdx.x];
    const int r = blockIdx.z * kRowsPerCta + threadIdx.y;
    const int b = blockIdx.y * 32 + threadIdx.x;
    if (r >= t.n_rows || b >= B) return;
    float out;
    if (alg == 1) {
        out = -INFINITY;
        for (int k = 0; k < t.k_cnt; ++k) {
            const float e = em[(int64_t)krow[t.k_off + k] * ld + b];
            const float w = tile_weight(params, kw, t, k, r, rpb_log2, w_stride);
            out = fmaxf(out, logf(w) + e);
        }
    } else {
        float m = -INFINITY;
        for (int k = 0; k < t.k_cnt; ++k) m = fmaxf(m, em[(int64_t)krow[t.k_off + k] * ld + b]);
        if (m == -INFINITY) {
            out = -INFINITY;
        } else {
            float s = 0.f;
            for (int k = 0; k < t.k_cnt; ++k) {
                const float e = em[(int64_t)krow[t.k_off + k] * ld + b];
                const float w = tile_weight(params, kw, t, k, r, rpb_log2, w_stride);
                s += (alg == 2) ? expf(alpha * logf(w)) * expf(alpha * (e - m)) : w * expf(e - m);
            }
            out = (alg == 2) ? (logf(s + 1e-24f) + alpha * m) / alpha : logf(s) + m;
        }
    }
    nm[((int64_t)t.out_row + r) * ld + b] = out;
}

// Element flows: tile rows are child (element) rows, terms are parent node rows.
__global__ void __launch_bounds__(32 * kRowsPerCta)
sum_ele_generic_kernel(const float* __restrict__ nf, const float* __restrict__ nm, const float* __restrict__ em,
                       float* __restrict__ ef, int64_t ld, int B, const float* __restrict__ params,
                       const PcbLseTile* __restrict__ tiles, int rpb_log2, const int* __restrict__ krow,
                       const int* __restrict__ kw, int w_stride, int alg, float alpha, int logspace, int accumulate) {
    pcb::pdl_begin();
    const PcbLseTile t = tiles[blockIdx.x];
    const int r = blockIdx.z * kRowsPerCta + threadIdx.y;
    const int b = blockIdx.y * 32 + threadIdx.x;
    if (r >= t.n_rows || b >= B) return;
    const float e = em[((int64_t)t.aux_row + r) * ld + b];
    float acc = logspace ? -INFINITY : 0.f;
    for (int k = 0; k < t.k_cnt; ++k) {
        const int64_t n = (int64_t)krow[t.k_off + k] * ld + b;
        const float f = nf[n], m = nm[n];
        if (m == -INFINITY) continue;
        const float lw = logf(tile_weight(params, kw, t, k, r, rpb_log2, w_stride));
        if (alg == 1) {
            if (fabsf(lw + e - m) < 1e-6f) acc = logspace ? lae(acc, f) : acc + f;
        } else {
            const float x = (alg == 2) ? alpha * (lw + e - m) : lw + e - m;
            acc = logspace ? lae(acc, f + x) : acc + f * expf(x);
        }
    }
    float* dst = ef + ((int64_t)t.out_row + r) * ld + b;
    if (accumulate) acc = logspace ? lae(*dst, acc) : *dst + acc;
    *dst = acc;
}

// Parameter flows: one warp per (node row, child) pair of a tile, lanes over the batch.
__global__ void __launch_bounds__(256)
sum_par_generic_kernel(const float* __restrict__ nf, const float* __restrict__ nm, const float* __restrict__ em,
                       int64_t ld, int B, const float* __restrict__ params, float* __restrict__ pflows,
                       const PcbPflowTile* __restrict__ tiles, int rpb_log2, const int* __restrict__ cids,
                       const int* __restrict__ pids, const int* __restrict__ pfids, int alg, int logspace,
                       float sign) {
    pcb::pdl_begin();
    const PcbPflowTile t = tiles[blockIdx.x];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int pairs = t.n_rows * t.k_cnt;
    for (int p = blockIdx.y * 8 + warp; p < pairs; p += gridDim.y * 8) {
        const int r = p / t.k_cnt, k = p % t.k_cnt;
        const int blk = r >> rpb_log2, i = r & ((1 << rpb_log2) - 1);
        const float w = params[(int64_t)pids[t.k_off + k] + t.p_add + (int64_t)blk * t.gs_p + i];
        const float lw = logf(w);
        const int64_t nrow = ((int64_t)t.nid + r) * ld;
        const int64_t crow = (int64_t)cids[t.k_off + k] * ld;
        float s = 0.f;
        for (int b = lane; b < B; b += 32) {
            const float f = nf[nrow + b], m = nm[nrow + b], e = em[crow + b];
            if (alg == 1) {
                if (fabsf(lw + e - m) < 1e-6f) s += logspace ? expf(f) : f;
            } else if (logspace) {
                s += (m == -INFINITY) ? expf(f) : expf(f + e - m);
            } else if (m != -INFINITY) {
                s += f * expf(e - m);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            const float v = (alg == 1) ? s : s * w;
            atomicAdd(pflows + (int64_t)pfids[t.k_off + k] + t.p_add + (int64_t)blk * t.gs_pf + i, sign * v);
        }
    }
}

int log2_pow2(int v) {
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}

}  // namespace

extern "C" int pcb_sum_fwd_generic(const float* element_mars, float* node_mars, int64_t ld, int32_t B,
                                   const float* params, const PcbLseTile* tiles, int32_t num_tiles,
                                   int32_t rows_per_block, const int32_t* krow, const int32_t* kw, int32_t w_stride,
                                   int32_t alg, float alpha, void* stream) {
    if (!element_mars || !node_mars || !params || !tiles || !krow || !kw || B <= 0 || ld < B || num_tiles < 0 ||
        rows_per_block <= 0 || (rows_per_block & (rows_per_block - 1)) || alg < 0 || alg > 2 ||
        (alg == 2 && !(alpha > 0.f)))
        return pcb::set_error(PCB_E_ARG, "pcb_sum_fwd_generic: bad arguments");
    if (num_tiles == 0) return PCB_OK;
    const int64_t gy = pcb::cdiv(B, 32);
    if (gy > 65535) return pcb::set_error(PCB_E_ARG, "pcb_sum_fwd_generic: batch too large");
    return pcb::launch_status(
        pcb::launch_k(sum_fwd_generic_kernel, dim3((unsigned)num_tiles, (unsigned)gy, 128 / kRowsPerCta),
                      dim3(32, kRowsPerCta), 0, pcb::as_stream(stream), 1u, element_mars, node_mars, ld, B, params,
                      tiles, log2_pow2(rows_per_block), krow, kw, w_stride, alg, alpha),
        "pcb_sum_fwd_generic");
}

extern "C" int pcb_sum_ele_generic(const float* node_flows, const float* node_mars, const float* element_mars,
                                   float* element_flows, int64_t ld, int32_t B, const float* params,
                                   const PcbLseTile* tiles, int32_t num_tiles, int32_t rows_per_block,
                                   const int32_t* krow, const int32_t* kw, int32_t w_stride, int32_t alg, float alpha,
                                   int32_t logspace, int32_t accumulate, void* stream) {
    if (!node_flows || !node_mars || !element_mars || !element_flows || !params || !tiles || !krow || !kw || B <= 0 ||
        ld < B || num_tiles < 0 || rows_per_block <= 0 || (rows_per_block & (rows_per_block - 1)) || alg < 0 ||
        alg > 2 || (alg == 2 && !(alpha > 0.f)))
        return pcb::set_error(PCB_E_ARG, "pcb_sum_ele_generic: bad arguments");
    if (num_tiles == 0) return PCB_OK;
    const int64_t gy = pcb::cdiv(B, 32);
    if (gy > 65535) return pcb::set_error(PCB_E_ARG, "pcb_sum_ele_generic: batch too large");
    return pcb::launch_status(
        pcb::launch_k(sum_ele_generic_kernel, dim3((unsigned)num_tiles, (unsigned)gy, 128 / kRowsPerCta),
                      dim3(32, kRowsPerCta), 0, pcb::as_stream(stream), 1u, node_flows, node_mars, element_mars,
                      element_flows, ld, B, params, tiles, log2_pow2(rows_per_block), krow, kw, w_stride, alg, alpha,
                      logspace, accumulate),
        "pcb_sum_ele_generic");
}

extern "C" int pcb_sum_par_generic(const float* node_flows, const float* node_mars, const float* element_mars,
                                   int64_t ld, int32_t B, const float* params, float* param_flows,
                                   const PcbPflowTile* tiles, int32_t num_tiles, int32_t rows_per_block,
                                   const int32_t* cids, const int32_t* pids, const int32_t* pfids, int32_t alg,
                                   int32_t logspace, int32_t negate, void* stream) {
    if (!node_flows || !node_mars || !element_mars || !params || !param_flows || !tiles || !cids || !pids || !pfids ||
        B <= 0 || ld < B || num_tiles < 0 || rows_per_block <= 0 || (rows_per_block & (rows_per_block - 1)) ||
        alg < 0 || alg > 2)
        return pcb::set_error(PCB_E_ARG, "pcb_sum_par_generic: bad arguments");
    if (num_tiles == 0) return PCB_OK;
    return pcb::launch_status(
        pcb::launch_k(sum_par_generic_kernel, dim3((unsigned)num_tiles, 16), dim3(256), 0, pcb::as_stream(stream), 1u,
                      node_flows, node_mars, element_mars, ld, B, params, param_flows, tiles,
                      log2_pow2(rows_per_block), cids, pids, pfids, alg, logspace, negate ? -1.f : 1.f),
        "pcb_sum_par_generic");
}
