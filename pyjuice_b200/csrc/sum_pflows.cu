// Sum-layer parameter flows (plain FP32 path): a contraction over the batch.
//
// For a tile of up to 32 nodes (rows nid + i) and up to 64 children (element rows
// cids[k]) of one node block:
//   pf[pfids[k] + i] += params[pids[k] + i] * sum_b A[i, b] * C[k, b]
//   A[i, b] = exp(lf[nid + i, b] - M_b),  C[k, b] = exp(em[cids[k], b] + M_b)
// with lf = log(node flow) - log(node mar) and M_b = max_i lf[nid + i, b]. The batch
// is staged in chunks of 32 samples; exponentials are taken once per staged value.
// Each (node, child) flow slot is owned by one CTA, so the update is a plain
// read-modify-write unless slots are shared by tied nodes (atomic = 1).
#include "common.cuh"

namespace {

constexpr int TMN = 32;   // nodes per tile
constexpr int TKC = 64;   // children per tile
constexpr int KB = 32;    // samples per staged chunk

template <bool MODIFIED, bool ATOMIC>
__global__ void __launch_bounds__(256)
sum_pflows_kernel(const float* __restrict__ nf, const float* __restrict__ nm, const float* __restrict__ em,
                  int64_t ld, int B, const float* __restrict__ params, float* __restrict__ pf,
                  const PcbPflowTile* __restrict__ tiles, const int* __restrict__ cids, const int* __restrict__ pids,
                  const int* __restrict__ pfids) {
    __shared__ float sA[TMN][KB + 1];
    __shared__ float sC[TKC][KB + 1];
    __shared__ float sM[KB];
    __shared__ int sCid[TKC];

    const PcbPflowTile t = tiles[blockIdx.x];
    const int tid = threadIdx.x;
    // thread -> (2 nodes, 4 children): nodes ty*2 + {0,1}, children tx + 16*q
    const int tx = tid % 16;
    const int ty = tid / 16;

    if (tid < TKC) sCid[tid] = (tid < t.k_cnt) ? cids[t.k_off + tid] : 0;

    float acc[2][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[a][q] = 0.f;
    __syncthreads();

    for (int b0 = 0; b0 < B; b0 += KB) {
        for (int idx = tid; idx < TMN * KB; idx += 256) {
            const int i = idx / KB;
            const int b = idx % KB;
            float v = -INFINITY;
            if (i < t.n_rows && b0 + b < B) {
                const int64_t off = ((int64_t)t.nid + i) * ld + b0 + b;
                if (MODIFIED) {
                    v = __ldg(nf + off);
                } else {
                    const float m = __ldg(nm + off);
                    v = (m == -INFINITY) ? -INFINITY : logf(__ldg(nf + off)) - m;
                }
            }
            sA[i][b] = v;
        }
        __syncthreads();
        if (tid < KB) {
            float m = -INFINITY;
            for (int i = 0; i < TMN; ++i) m = fmaxf(m, sA[i][tid]);
            sM[tid] = m;
        }
        __syncthreads();
        for (int idx = tid; idx < TMN * KB; idx += 256) {
            const int i = idx / KB;
            const int b = idx % KB;
            const float m = sM[b];
            sA[i][b] = (m == -INFINITY) ? 0.f : __expf(sA[i][b] - m);
        }
        for (int idx = tid; idx < TKC * KB; idx += 256) {
            const int k = idx / KB;
            const int b = idx % KB;
            float v = 0.f;
            const float m = sM[b];
            if (k < t.k_cnt && b0 + b < B && m != -INFINITY) {
                v = __expf(__ldg(em + (int64_t)sCid[k] * ld + b0 + b) + m);
            }
            sC[k][b] = v;
        }
        __syncthreads();
#pragma unroll 8
        for (int b = 0; b < KB; ++b) {
            const float a0 = sA[ty * 2 + 0][b];
            const float a1 = sA[ty * 2 + 1][b];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float c = sC[tx + 16 * q][b];
                acc[0][q] = fmaf(a0, c, acc[0][q]);
                acc[1][q] = fmaf(a1, c, acc[1][q]);
            }
        }
        __syncthreads();
    }

#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const int i = ty * 2 + a;
        if (i >= t.n_rows) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = tx + 16 * q;
            if (k >= t.k_cnt) continue;
            const float w = __ldg(params + (int64_t)pids[t.k_off + k] + t.p_add + i);
            const int64_t slot = (int64_t)pfids[t.k_off + k] + t.p_add + i;
            const float v = acc[a][q] * w;
            if (ATOMIC) atomicAdd(pf + slot, v);
            else pf[slot] += v;
        }
    }
}

}  // namespace

extern "C" int pcb_sum_pflows(const float* node_flows, const float* node_mars, const float* element_mars, int64_t ld,
                              int32_t B, const float* params, float* param_flows, const PcbPflowTile* tiles,
                              int32_t num_tiles, const int32_t* cids, const int32_t* pids, const int32_t* pfids,
                              int32_t modified, int32_t atomic, void* stream) {
    if (!node_flows || !node_mars || !element_mars || !params || !param_flows || !tiles || !cids || !pids || !pfids ||
        B <= 0 || ld < B || num_tiles < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_sum_pflows: bad arguments");
    if (num_tiles == 0) return PCB_OK;
    cudaStream_t s = pcb::as_stream(stream);
    if (modified && atomic)
        sum_pflows_kernel<true, true><<<num_tiles, 256, 0, s>>>(node_flows, node_mars, element_mars, ld, B, params, param_flows, tiles, cids, pids, pfids);
    else if (modified)
        sum_pflows_kernel<true, false><<<num_tiles, 256, 0, s>>>(node_flows, node_mars, element_mars, ld, B, params, param_flows, tiles, cids, pids, pfids);
    else if (atomic)
        sum_pflows_kernel<false, true><<<num_tiles, 256, 0, s>>>(node_flows, node_mars, element_mars, ld, B, params, param_flows, tiles, cids, pids, pfids);
    else
        sum_pflows_kernel<false, false><<<num_tiles, 256, 0, s>>>(node_flows, node_mars, element_mars, ld, B, params, param_flows, tiles, cids, pids, pfids);
    return pcb::check_launch("pcb_sum_pflows");
}
