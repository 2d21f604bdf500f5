// Sum-layer parameter flows (plain FP32 path): a contraction over the batch.
//
// A tile covers up to 128 nodes (rows nid + r: consecutive node blocks that share their
// children) and up to 64 children (element rows cids[k]):
//   pf(r, k) += params(r, k) * sum_b A[r, b] * C[k, b]
//   A[r, b] = exp(lf[nid + r, b] - M_b),  C[k, b] = exp(em[cids[k], b] + M_b)
// with lf = log(node flow) - log(node mar) and M_b = max_r lf[nid + r, b].
//
// The batch is split over a thread-block cluster of CS CTAs (one batch slice each). Each
// CTA stages its slice in chunks of 32 samples with asynchronous copies into two shared
// buffers (the next chunk's copies fly while the current one is reduced), takes every
// exponential once, and keeps an 8 x 4 register tile per thread. At the end the CTAs
// exchange their partial tiles through distributed shared memory and each adds the CS
// partials of its share of the outputs in rank order: the result does not depend on
// timing (no float atomics) and no global scratch is needed. Each (node, child) flow slot
// is owned by one tile, so the final update is a plain read-modify-write unless slots are
// shared by tied nodes (atomic = 1).
#include <cooperative_groups.h>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int TMN = 128;  // nodes per tile
constexpr int TKC = 64;   // children per tile
constexpr int KB = 32;    // samples per staged chunk
constexpr int RS = KB + 4;  // shared row stride (floats): 16-byte rows, conflict-free float4 reads

template <bool MODIFIED>
struct PfStage {
    static constexpr int kA = TMN * RS;
    static constexpr int kC = TKC * RS;
    static constexpr int kPer = kA * (MODIFIED ? 1 : 2) + kC;
    static constexpr size_t bytes() { return sizeof(float) * (2 * kPer + KB + 8 * KB) + sizeof(int) * TKC; }
    float* base;
    __device__ explicit PfStage(float* p) : base(p) {}
    __device__ float* A(int s) { return base + s * kPer; }
    __device__ float* A2(int s) { return base + s * kPer + kA; }
    __device__ float* C(int s) { return base + s * kPer + kA * (MODIFIED ? 1 : 2); }
    __device__ float* M() { return base + 2 * kPer; }
    __device__ float* Part() { return base + 2 * kPer + KB; }
    __device__ int* Cid() { return reinterpret_cast<int*>(base + 2 * kPer + KB + 8 * KB); }
};

__device__ __forceinline__ void stage_row(float* d, const float* g, int b, int bend, bool vec, float fill) {
    // 32 samples of one row, copied by the calling thread in 8 pieces of 4
#pragma unroll
    for (int j4 = 0; j4 < KB / 4; ++j4) {
        const int bb = b + j4 * 4;
        if (vec && bb + 3 < bend) {
            pcb::cp_async16(d + j4 * 4, g + j4 * 4);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (bb + j < bend) pcb::cp_async4(d + j4 * 4 + j, g + j4 * 4 + j);
                else d[j4 * 4 + j] = fill;
            }
        }
    }
}

template <bool MODIFIED, bool ATOMIC>
__global__ void __launch_bounds__(256)
sum_pflows_kernel(const float* __restrict__ nf, const float* __restrict__ nm, const float* __restrict__ em,
                  int64_t ld, int B, const float* __restrict__ params, float* __restrict__ pf,
                  const PcbPflowTile* __restrict__ tiles, int rpb_log2, const int* __restrict__ cids,
                  const int* __restrict__ pids, const int* __restrict__ pfids, int slice, bool vec) {
    extern __shared__ __align__(16) float dsm[];
    PfStage<MODIFIED> st(dsm);
    float* sM = st.M();
    float* sPart = st.Part();
    int* sCid = st.Cid();

    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank();
    const int csize = (int)cluster.num_blocks();
    const PcbPflowTile t = tiles[blockIdx.x / csize];
    const int tid = threadIdx.x;
    const int tx = tid % 16;   // children tx + 16 * kk, kk < 4
    const int ty = tid / 16;   // nodes ty * 8 .. + 8
    const int rpb_mask = (1 << rpb_log2) - 1;

    if (tid < TKC) sCid[tid] = (tid < t.k_cnt) ? cids[t.k_off + tid] : -1;
    __syncthreads();

    float acc[8][4];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[a][q] = 0.f;

    const int bs0 = crank * slice;
    const int bs1 = min(B, bs0 + slice);
    const int nchunks = bs1 > bs0 ? (bs1 - bs0 + KB - 1) / KB : 0;

    auto issue = [&](int c, int s) {
        const int b0 = bs0 + c * KB;
        // 128 node rows (+ mars rows), 64 child rows: one row per thread-iteration
        for (int i = tid; i < TMN; i += 256) {
            float* dA = st.A(s) + i * RS;
            if (i < t.n_rows) {
                const int64_t off = ((int64_t)t.nid + i) * ld + b0;
                stage_row(dA, nf + off, b0, bs1, vec, -INFINITY);
                if (!MODIFIED) stage_row(st.A2(s) + i * RS, nm + off, b0, bs1, vec, -INFINITY);
            } else {
#pragma unroll
                for (int j = 0; j < KB; ++j) dA[j] = -INFINITY;
                if (!MODIFIED)
#pragma unroll
                    for (int j = 0; j < KB; ++j) st.A2(s)[i * RS + j] = -INFINITY;
            }
        }
        for (int k = tid; k < TKC; k += 256) {
            float* dC = st.C(s) + k * RS;
            const int row = sCid[k];
            if (row >= 0) {
                stage_row(dC, em + (int64_t)row * ld + b0, b0, bs1, vec, -INFINITY);
            } else {
#pragma unroll
                for (int j = 0; j < KB; ++j) dC[j] = -INFINITY;
            }
        }
        pcb::cp_async_commit();
    };

    if (nchunks > 0) issue(0, 0);
    for (int c = 0; c < nchunks; ++c) {
        const int s = c & 1;
        if (c + 1 < nchunks) {
            issue(c + 1, s ^ 1);
            pcb::cp_async_wait<1>();
        } else {
            pcb::cp_async_wait<0>();
        }
        __syncthreads();
        float* sA = st.A(s);
        float* sC = st.C(s);
        if (!MODIFIED) {
            float* sA2 = st.A2(s);
            for (int idx = tid; idx < TMN * KB; idx += 256) {
                const int i = idx / KB;
                const int b = idx % KB;
                const float m = sA2[i * RS + b];
                sA[i * RS + b] = (m == -INFINITY) ? -INFINITY : logf(sA[i * RS + b]) - m;
            }
            __syncthreads();
        }
        {
            const int b = tid % KB;
            const int part = tid / KB;  // 8 parts of 16 rows
            float m = -INFINITY;
#pragma unroll 4
            for (int i = part * 16; i < part * 16 + 16; ++i) m = fmaxf(m, sA[i * RS + b]);
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
            const int i = idx / KB;
            const int b = idx % KB;
            const float m = sM[b];
            sA[i * RS + b] = (m == -INFINITY) ? 0.f : __expf(sA[i * RS + b] - m);
        }
        for (int idx = tid; idx < TKC * KB; idx += 256) {
            const int k = idx / KB;
            const int b = idx % KB;
            const float m = sM[b];
            sC[k * RS + b] = (m == -INFINITY) ? 0.f : __expf(sC[k * RS + b] + m);
        }
        __syncthreads();
#pragma unroll 2
        for (int b = 0; b < KB; b += 4) {
            float4 cv[4];
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) cv[kk] = *reinterpret_cast<const float4*>(&sC[(tx + 16 * kk) * RS + b]);
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                const float4 av = *reinterpret_cast<const float4*>(&sA[(ty * 8 + a) * RS + b]);
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    acc[a][kk] = fmaf(av.x, cv[kk].x, acc[a][kk]);
                    acc[a][kk] = fmaf(av.y, cv[kk].y, acc[a][kk]);
                    acc[a][kk] = fmaf(av.z, cv[kk].z, acc[a][kk]);
                    acc[a][kk] = fmaf(av.w, cv[kk].w, acc[a][kk]);
                }
            }
        }
        __syncthreads();
    }

    // partial tile -> shared memory (aliases the stage buffers); cluster-wide fixed-order sum
    float* red = dsm;  // [TMN][TKC]
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) red[(ty * 8 + a) * TKC + tx + 16 * kk] = acc[a][kk];
    cluster.sync();
    const int per = (TMN * TKC) / csize;
    for (int idx = crank * per + tid; idx < (crank + 1) * per; idx += 256) {
        const int i = idx / TKC;
        const int k = idx % TKC;
        if (i >= t.n_rows || k >= t.k_cnt) continue;
        float s = 0.f;
        for (int r = 0; r < csize; ++r) s += cluster.map_shared_rank(red, r)[idx];
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
           const int* pfids, cudaStream_t s, bool vec) {
    const int slice = (int)pcb::cdiv(pcb::cdiv(B, cs), KB) * KB;
    constexpr size_t smem = PfStage<MODIFIED>::bytes();
    static_assert(PfStage<MODIFIED>::bytes() >= sizeof(float) * TMN * TKC, "reduction tile must fit");
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    dev = dev < 0 ? 0 : (dev > 63 ? 63 : dev);
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(sum_pflows_kernel<MODIFIED, ATOMIC>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_sum_pflows: %s", cudaGetErrorString(e));
        configured[dev] = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)num_tiles * cs);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, sum_pflows_kernel<MODIFIED, ATOMIC>, nf, nm, em, ld, B, params, pf, tiles,
                                       rpb_log2, cids, pids, pfids, slice, vec);
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
    const bool vec = pcb::vec_ok(node_flows, ld) && pcb::vec_ok(node_mars, ld) && pcb::vec_ok(element_mars, ld);
    cudaStream_t s = pcb::as_stream(stream);
    const float *nf = node_flows, *nm = node_mars, *em = element_mars;
    if (modified && atomic) return launch<true, true>(cs, nf, nm, em, ld, B, params, param_flows, tiles, num_tiles, rpb_log2, cids, pids, pfids, s, vec);
    if (modified) return launch<true, false>(cs, nf, nm, em, ld, B, params, param_flows, tiles, num_tiles, rpb_log2, cids, pids, pfids, s, vec);
    if (atomic) return launch<false, true>(cs, nf, nm, em, ld, B, params, param_flows, tiles, num_tiles, rpb_log2, cids, pids, pfids, s, vec);
    return launch<false, false>(cs, nf, nm, em, ld, B, params, param_flows, tiles, num_tiles, rpb_log2, cids, pids, pfids, s, vec);
}
