// Sum-layer parameter flows (plain FP32 path): a contraction over the batch.
//
// A tile covers up to 128 nodes (rows nid + r: consecutive node blocks that share their
// children) and up to 64 children (element rows cids[k]):
//   pf(r, k) += params(r, k) * sum_b A[r, b] * C[k, b]
//   A[r, b] = exp(lf[nid + r, b] - M_b),  C[k, b] = exp(em[cids[k], b] + M_b)
// with lf = log(node flow) - log(node mar) and M_b = max_r lf[nid + r, b].
//
// The batch is split over a thread-block cluster of CS CTAs (one batch slice each). Each
// CTA stages its slice in chunks of 32 samples (every exponential taken once) and keeps
// an 8 x 4 register tile per thread. At the end the CTAs exchange their partial tiles
// through distributed shared memory and each adds the CS partials of its share of the
// outputs in rank order: the result does not depend on timing (no float atomics), and no
// global scratch is needed. Each (node, child) flow slot is owned by one tile, so the
// final update is a plain read-modify-write unless slots are shared by tied nodes
// (atomic = 1).
#include <cooperative_groups.h>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int TMN = 128;  // nodes per tile
constexpr int TKC = 64;   // children per tile
constexpr int KB = 32;    // samples per staged chunk
constexpr int AS = TMN + 4;
constexpr int CSS = TKC + 4;

template <bool MODIFIED, bool ATOMIC>
__global__ void __launch_bounds__(256)
sum_pflows_kernel(const float* __restrict__ nf, const float* __restrict__ nm, const float* __restrict__ em,
                  int64_t ld, int B, const float* __restrict__ params, float* __restrict__ pf,
                  const PcbPflowTile* __restrict__ tiles, int rpb_log2, const int* __restrict__ cids,
                  const int* __restrict__ pids, const int* __restrict__ pfids, int slice) {
    // staging buffers during the loop; the partial-result tile [TMN][TKC] afterwards
    __shared__ __align__(16) float smem[TMN * TKC];
    float* sA = smem;                       // [KB][AS]   exp(lf - M), sample-major
    float* sC = smem + KB * AS;             // [KB][CSS]  exp(em + M)
    float* sM = sC + KB * CSS;              // [KB]
    float* sPart = sM + KB;                 // [8][KB]
    __shared__ int sCid[TKC];

    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank();
    const int csize = (int)cluster.num_blocks();
    const PcbPflowTile t = tiles[blockIdx.x / csize];
    const int tid = threadIdx.x;
    const int tx = tid % 16;   // children tx*4 .. +4
    const int ty = tid / 16;   // nodes ty*8 .. +8
    const int rpb_mask = (1 << rpb_log2) - 1;

    if (tid < TKC) sCid[tid] = (tid < t.k_cnt) ? cids[t.k_off + tid] : 0;

    float acc[8][4];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[a][q] = 0.f;
    __syncthreads();

    const int bs0 = crank * slice;
    const int bs1 = min(B, bs0 + slice);
    for (int b0 = bs0; b0 < bs1; b0 += KB) {
        for (int idx = tid; idx < TMN * KB; idx += 256) {
            const int i = idx / KB;
            const int b = idx % KB;
            float v = -INFINITY;
            if (i < t.n_rows && b0 + b < bs1) {
                const int64_t off = ((int64_t)t.nid + i) * ld + b0 + b;
                if (MODIFIED) {
                    v = __ldg(nf + off);
                } else {
                    const float m = __ldg(nm + off);
                    v = (m == -INFINITY) ? -INFINITY : logf(__ldg(nf + off)) - m;
                }
            }
            sA[b * AS + i] = v;
        }
        __syncthreads();
        {
            const int b = tid % KB;
            const int part = tid / KB;      // 8 parts of 16 rows
            float m = -INFINITY;
#pragma unroll 4
            for (int i = part * 16; i < part * 16 + 16; ++i) m = fmaxf(m, sA[b * AS + i]);
            sPart[part * KB + b] = m;
        }
        __syncthreads();
        if (tid < KB) {
            float m = -INFINITY;
#pragma unroll
            for (int p = 0; p < 8; ++p) m = fmaxf(m, sPart[p * KB + tid]);
            sM[tid] = m;
        }
        __syncthreads();
        for (int idx = tid; idx < TMN * KB; idx += 256) {
            const int b = idx / TMN;
            const int i = idx % TMN;
            const float m = sM[b];
            sA[b * AS + i] = (m == -INFINITY) ? 0.f : __expf(sA[b * AS + i] - m);
        }
        for (int idx = tid; idx < TKC * KB; idx += 256) {
            const int k = idx / KB;
            const int b = idx % KB;
            float v = 0.f;
            const float m = sM[b];
            if (k < t.k_cnt && b0 + b < bs1 && m != -INFINITY) {
                v = __expf(__ldg(em + (int64_t)sCid[k] * ld + b0 + b) + m);
            }
            sC[b * CSS + k] = v;
        }
        __syncthreads();
#pragma unroll 4
        for (int b = 0; b < KB; ++b) {
            const float4 a0 = *reinterpret_cast<const float4*>(&sA[b * AS + ty * 8]);
            const float4 a1 = *reinterpret_cast<const float4*>(&sA[b * AS + ty * 8 + 4]);
            const float4 c = *reinterpret_cast<const float4*>(&sC[b * CSS + tx * 4]);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[a][q] = fmaf(av[a], cv[q], acc[a][q]);
        }
        __syncthreads();
    }

    // partial tile -> shared memory; cluster-wide exchange; fixed-order sum
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        float4 v = make_float4(acc[a][0], acc[a][1], acc[a][2], acc[a][3]);
        *reinterpret_cast<float4*>(&smem[(ty * 8 + a) * TKC + tx * 4]) = v;
    }
    cluster.sync();
    const int per = (TMN * TKC) / csize;
    for (int idx = crank * per + tid; idx < (crank + 1) * per; idx += 256) {
        const int i = idx / TKC;
        const int k = idx % TKC;
        if (i >= t.n_rows || k >= t.k_cnt) continue;
        float s = 0.f;
        for (int r = 0; r < csize; ++r) s += cluster.map_shared_rank(smem, r)[idx];
        const int64_t roff = (int64_t)t.p_add + (int64_t)(i & rpb_mask);
        const int blk = i >> rpb_log2;
        const float w = __ldg(params + (int64_t)pids[t.k_off + k] + roff + (int64_t)blk * t.gs_p);
        const int64_t slot = (int64_t)pfids[t.k_off + k] + roff + (int64_t)blk * t.gs_pf;
        if (ATOMIC) atomicAdd(pf + slot, s * w);
        else pf[slot] += s * w;
    }
    cluster.sync();  // keep every CTA's shared memory alive until all reads are done
}

template <bool MODIFIED, bool ATOMIC>
int launch(int cs, const float* nf, const float* nm, const float* em, int64_t ld, int B, const float* params,
           float* pf, const PcbPflowTile* tiles, int num_tiles, int rpb_log2, const int* cids, const int* pids,
           const int* pfids, cudaStream_t s) {
    const int slice = (int)pcb::cdiv(pcb::cdiv(B, cs), KB) * KB;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)num_tiles * cs);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, sum_pflows_kernel<MODIFIED, ATOMIC>, nf, nm, em, ld, B, params, pf, tiles,
                                       rpb_log2, cids, pids, pfids, slice);
    if (e != cudaSuccess) return pcb::set_error(PCB_E_LAUNCH, "pcb_sum_pflows: %s", cudaGetErrorString(e));
    return pcb::check_launch("pcb_sum_pflows");
}

}  // namespace

extern "C" int pcb_sum_pflows(const float* node_flows, const float* node_mars, const float* element_mars, int64_t ld,
                              int32_t B, const float* params, float* param_flows, const PcbPflowTile* tiles,
                              int32_t num_tiles, int32_t rows_per_block, const int32_t* cids, const int32_t* pids,
                              const int32_t* pfids, int32_t modified, int32_t atomic, void* stream) {
    if (!node_flows || !node_mars || !element_mars || !params || !param_flows || !tiles || !cids || !pids || !pfids ||
        B <= 0 || ld < B || num_tiles < 0 || rows_per_block <= 0 || (rows_per_block & (rows_per_block - 1)))
        return pcb::set_error(PCB_E_ARG, "pcb_sum_pflows: bad arguments");
    if (num_tiles == 0) return PCB_OK;
    int rpb_log2 = 0;
    while ((1 << rpb_log2) < rows_per_block) ++rpb_log2;
    // batch slices of >= 128 samples, up to 4 CTAs per cluster
    const int cs = B >= 512 ? 4 : (B >= 256 ? 2 : 1);
    if ((int64_t)num_tiles * cs > 2147483647) return pcb::set_error(PCB_E_ARG, "pcb_sum_pflows: too many tiles");
    cudaStream_t s = pcb::as_stream(stream);
    const float *nf = node_flows, *nm = node_mars, *em = element_mars;
    if (modified && atomic) return launch<true, true>(cs, nf, nm, em, ld, B, params, param_flows, tiles, num_tiles, rpb_log2, cids, pids, pfids, s);
    if (modified) return launch<true, false>(cs, nf, nm, em, ld, B, params, param_flows, tiles, num_tiles, rpb_log2, cids, pids, pfids, s);
    if (atomic) return launch<false, true>(cs, nf, nm, em, ld, B, params, param_flows, tiles, num_tiles, rpb_log2, cids, pids, pfids, s);
    return launch<false, false>(cs, nf, nm, em, ld, B, params, param_flows, tiles, num_tiles, rpb_log2, cids, pids, pfids, s);
}
