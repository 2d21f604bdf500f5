// Categorical input layer: forward lookup and deterministic parameter-flow histogram.
#include "common.cuh"

namespace {

// node_mars[node_offset + n, b] = log(params[s_pids[n] + x]) with x = data[vids[n], b], or
// 0 (log 1: the variable is summed out) where the missing mask is set,
// miss[b * m_sb + vids[n] * m_sv] != 0. A category outside [0, ncats) yields NaN (no
// out-of-range read).
// A CTA covers kFwdNodes consecutive nodes over 512 samples (4 per thread): the logs of
// the nodes' parameter slabs (up to kFwdSlab categories) are taken once into shared
// memory, each thread loads its 4 category values once and reuses them for every node of
// the same variable, and each node row is written with 16-byte stores.
constexpr int kFwdNodes = 8;
constexpr int kFwdSlab = 256;

constexpr int kFwdThreads = 128;
constexpr int kFwdSamples = 4 * kFwdThreads;

__global__ void __launch_bounds__(kFwdThreads)
input_cat_fwd_kernel(const int64_t* __restrict__ data, int64_t data_ld, const float* __restrict__ params,
                     const int* __restrict__ vids, const int* __restrict__ s_pids, const int* __restrict__ ncats,
                     int num_nodes, int node_offset, float* __restrict__ nm, int64_t ld, int B, bool vec,
                     const uint8_t* __restrict__ miss, int64_t m_sb, int64_t m_sv, int32_t* __restrict__ status) {
    // The node tables and the parameter logs are read before the wait for the previous kernel
    // (the parameters' writers do not trigger early); the samples and outputs after it.
    pcb::pdl_trigger();
    __shared__ float slab[kFwdNodes][kFwdSlab];
    __shared__ int sV[kFwdNodes], sK[kFwdNodes], sP[kFwdNodes];
    const int n0 = blockIdx.x * kFwdNodes;
    const int tid = threadIdx.x;
    if (tid < kFwdNodes) {
        const int n = n0 + tid;
        sV[tid] = n < num_nodes ? __ldg(vids + n) : -1;
        sK[tid] = n < num_nodes ? __ldg(ncats + n) : 0;
        sP[tid] = n < num_nodes ? __ldg(s_pids + n) : 0;
    }
    __syncthreads();
    for (int i = tid; i < kFwdNodes * kFwdSlab; i += blockDim.x) {
        const int j = i / kFwdSlab, k = i % kFwdSlab;
        if (k < sK[j] && sK[j] <= kFwdSlab) slab[j][k] = __logf(__ldcg(params + sP[j] + k));
    }
    __syncthreads();
    pcb::pdl_wait();
    const int b = blockIdx.y * kFwdSamples + tid * 4;
    if (b >= B) return;
    const int v0 = sV[0];
    int64_t x0[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) x0[q] = (b + q < B) ? __ldg(data + (int64_t)v0 * data_ld + b + q) : 0;
    for (int j = 0; j < kFwdNodes && n0 + j < num_nodes; ++j) {
        const int v = sV[j], K = sK[j];
        float4 o;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float r = 0.f;
            if (b + q < B && miss && miss[(int64_t)(b + q) * m_sb + (int64_t)v * m_sv]) {
                r = 0.f;
            } else if (b + q < B) {
                const int64_t x = (v == v0) ? x0[q] : __ldg(data + (int64_t)v * data_ld + b + q);
                if (x >= 0 && x < K) r = (K <= kFwdSlab) ? slab[j][x] : __logf(__ldcg(params + sP[j] + x));
                else {
                    r = NAN;
                    pcb::report_status(status, PCB_STATUS_BAD_CATEGORY);
                }
            }
            pcb::set(o, q, r);
        }
        pcb::store4(nm, (int64_t)node_offset + n0 + j, ld, b, B, vec, o);
    }
}

// One CTA per variable group: stable counting sort of the batch by category (chunks of
// up to CB samples; warp-parallel prefix sum of the category counts), then one warp per
// node copies the node's flow row into shared memory with coalesced loads and sums it per
// category in sample order, adding the sums to the node's flow slots. Deterministic: no
// float atomics (unless flow slots are shared by tied nodes of different variables:
// atomic = 1 adds with atomics). Samples whose variable is missing (miss[b * m_sb + v * m_sv] != 0) form
// their own segment: their flow sum M is spread over the categories as M * params[k]
// (input_layer.py:537-571, categorical.py:102-134).
__global__ void __launch_bounds__(256)
input_cat_bwd_kernel(const int64_t* __restrict__ data, int64_t data_ld, const float* __restrict__ nf, int64_t ld,
                     int B, const int* __restrict__ grp_var, const int* __restrict__ grp_node0,
                     const int* __restrict__ grp_count, const int* __restrict__ grp_ncats,
                     const int* __restrict__ s_pfids, int node_offset, float* __restrict__ pf, bool logspace, int CB,
                     const uint8_t* __restrict__ miss, int64_t m_sb, int64_t m_sv, const int* __restrict__ s_pids,
                     const float* __restrict__ params, bool atomic) {
    pcb::pdl_begin();
    extern __shared__ int smem[];
    const int g = blockIdx.x;
    const int K = grp_ncats[g];
    const int64_t v = grp_var[g];
    const int node0 = grp_node0[g];
    const int cnt = grp_count[g];
    int* keys = smem;              // [CB]
    int* perm = keys + CB;         // [CB]
    float* rows = reinterpret_cast<float*>(perm + CB);  // [warps][CB]
    int* seg = perm + CB + (blockDim.x >> 5) * CB;      // [K + 3]: categories, dropped, missing
    int* ucat = seg + K + 3;                            // [CB]: the categories present in the chunk
    __shared__ int sU;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;

    for (int c0 = 0; c0 < B; c0 += CB) {
        const int nb = min(CB, B - c0);
        for (int i = tid; i < K + 3; i += blockDim.x) seg[i] = 0;
        __syncthreads();
        for (int i = tid; i < nb; i += blockDim.x) {
            int key;
            if (miss && miss[(int64_t)(c0 + i) * m_sb + v * m_sv]) {
                key = K + 1;  // missing: spread over the categories below
            } else {
                const int64_t x = data[v * data_ld + c0 + i];
                key = (x >= 0 && x < K) ? (int)x : K;  // out-of-range samples are dropped
            }
            keys[i] = key;
            atomicAdd(&seg[key + 1], 1);
        }
        __syncthreads();
        if (warp == 0) {
            int carry = 0;
            for (int base = 0; base < K + 3; base += 32) {
                const int i = base + lane;
                int v = (i < K + 3) ? seg[i] : 0;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, v, o);
                    if (lane >= o) v += t;
                }
                v += carry;
                if (i < K + 3) seg[i] = v;
                carry = __shfl_sync(0xffffffffu, v, 31);
            }
        }
        __syncthreads();
        // Stable scatter by warp 0: 32 samples at a time, ranks from lane matching.
        if (warp == 0) {
            for (int i0 = 0; i0 < nb; i0 += 32) {
                const int i = i0 + lane;
                const bool act = i < nb;
                const int key = act ? keys[i] : -1;
                const unsigned same = __match_any_sync(0xffffffffu, key);
                const int rank = __popc(same & ((1u << lane) - 1u));
                int pos = 0;
                if (act) pos = seg[key] + rank;
                __syncwarp();
                if (act) perm[pos] = i;
                // The highest lane of each key group advances the cursor.
                const bool leader = act && ((same >> lane) == 1u);
                __syncwarp();
                if (leader) seg[key] += __popc(same);
                __syncwarp();
            }
        }
        __syncthreads();
        // seg[k] now holds the end of category k; its start is the end of category k-1. The
        // categories that occur in this chunk, in order (at most one per sample): without
        // missing values only their slots change, so the nodes' loops run over them instead
        // of all K categories (a vocabulary of thousands against a batch of tens).
        if (warp == 0) {
            int nu = 0;
            for (int base = 0; base < K; base += 32) {
                const int k = base + lane;
                const bool present = k < K && seg[k] > (k == 0 ? 0 : seg[k - 1]);
                const unsigned bal = __ballot_sync(0xffffffffu, present);
                if (present) ucat[nu + __popc(bal & ((1u << lane) - 1u))] = k;
                nu += __popc(bal);
            }
            if (lane == 0) sU = nu;
        }
        __syncthreads();
        const bool dense = seg[K + 1] > seg[K];  // missing samples: every category gets flow
        const int L = dense ? K : sU;
        float* wrow = rows + warp * CB;
        const bool vec4 = ((ld & 3) == 0) && ((c0 & 3) == 0) && ((reinterpret_cast<uintptr_t>(nf) & 15) == 0);
        for (int n = warp; n < cnt; n += (blockDim.x >> 5)) {
            const int64_t row = (int64_t)node_offset + node0 + n;
            const float* frow = nf + row * ld + c0;
            const int64_t sf = s_pfids[node0 + n];
            if (vec4 && (nb & 3) == 0) {
                for (int i = lane; i < nb / 4; i += 32)
                    reinterpret_cast<float4*>(wrow)[i] = __ldg(reinterpret_cast<const float4*>(frow) + i);
            } else {
                for (int i = lane; i < nb; i += 32) wrow[i] = __ldg(frow + i);
            }
            __syncwarp();
            // flow of the samples with this variable missing (segment K + 1)
            float msum = 0.f;
            if (miss) {
                for (int p = seg[K] + lane; p < seg[K + 1]; p += 32) {
                    const float f = wrow[perm[p]];
                    msum += logspace ? __expf(f) : f;
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) msum += __shfl_xor_sync(0xffffffffu, msum, o);
            }
            const int64_t sp = miss ? s_pids[node0 + n] : 0;
            // list entries lane, lane + 32, ... (all categories, or the present ones): the
            // slots' old values are loaded for a batch of kR entries at once (one round trip),
            // then summed and stored
            constexpr int kR = 8;
            for (int k0 = 0; k0 < L; k0 += 32 * kR) {
                float old[kR];
#pragma unroll
                for (int j = 0; j < kR; ++j) {
                    const int idx = k0 + lane + 32 * j;
                    old[j] = (idx < L && !atomic) ? pf[sf + (dense ? idx : ucat[idx])] : 0.f;
                }
#pragma unroll
                for (int j = 0; j < kR; ++j) {
                    const int idx = k0 + lane + 32 * j;
                    if (idx >= L) continue;
                    const int k = dense ? idx : ucat[idx];
                    const int s = (k == 0) ? 0 : seg[k - 1];
                    const int e = seg[k];
                    if (e == s && msum == 0.f) continue;
                    float acc = (msum != 0.f) ? msum * params[sp + k] : 0.f;
                    for (int p = s; p < e; ++p) {
                        const float f = wrow[perm[p]];
                        acc += logspace ? __expf(f) : f;
                    }
                    if (atomic) atomicAdd(pf + sf + k, acc);  // slot shared by tied nodes
                    else pf[sf + k] = old[j] + acc;
                }
            }
            __syncwarp();  // the next node overwrites this warp's row
        }
        __syncthreads();
    }
}

}  // namespace

extern "C" int pcb_input_cat_fwd(const int64_t* data, int64_t data_ld, const float* params, const int32_t* vids,
                                 const int32_t* s_pids, const int32_t* ncats, int32_t num_nodes, int32_t node_offset,
                                 float* node_mars, int64_t ld, int32_t B, const uint8_t* missing, int64_t miss_sb,
                                 int64_t miss_sv, void* stream) {
    if (!data || !params || !vids || !s_pids || !ncats || !node_mars || B <= 0 || ld < B || data_ld < B || num_nodes < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_input_cat_fwd: bad arguments");
    if (num_nodes == 0) return PCB_OK;
    const bool vec = pcb::vec_ok(node_mars, ld);
    const int64_t gy = pcb::cdiv(B, kFwdSamples);
    if (gy > 65535) return pcb::set_error(PCB_E_ARG, "pcb_input_cat_fwd: batch too large");
    return pcb::launch_status(pcb::launch_k(input_cat_fwd_kernel, dim3((unsigned)pcb::cdiv(num_nodes, kFwdNodes),
                                                                       (unsigned)gy),
                                            dim3(kFwdThreads), 0, pcb::as_stream(stream), 1u, data, data_ld, params, vids,
                                            s_pids, ncats, num_nodes, node_offset, node_mars, ld, B, vec, missing,
                                            miss_sb, miss_sv, pcb::status_word()),
                              "pcb_input_cat_fwd");
}

extern "C" int pcb_input_cat_bwd(const int64_t* data, int64_t data_ld, const float* node_flows, int64_t ld, int32_t B,
                                 const int32_t* grp_var, const int32_t* grp_node0, const int32_t* grp_count,
                                 const int32_t* grp_ncats, int32_t num_groups, int32_t max_ncats,
                                 const int32_t* s_pfids, int32_t node_offset, float* param_flows,
                                 int32_t logspace_flows, const uint8_t* missing, int64_t miss_sb, int64_t miss_sv,
                                 const int32_t* s_pids, const float* params, int32_t atomic, void* stream) {
    if (!data || !node_flows || !grp_var || !grp_node0 || !grp_count || !grp_ncats || !s_pfids || !param_flows ||
        B <= 0 || ld < B || data_ld < B || num_groups < 0 || max_ncats <= 0 || (missing && (!s_pids || !params)))
        return pcb::set_error(PCB_E_ARG, "pcb_input_cat_bwd: bad arguments");
    if (num_groups == 0) return PCB_OK;
    const int CB = B < 1024 ? B : 1024;
    const size_t smem = (size_t)(2 * CB + 8 * CB + max_ncats + 3 + CB) * sizeof(int);
    if (smem > 200 * 1024) return pcb::set_error(PCB_E_ARG, "pcb_input_cat_bwd: too many categories (%d)", max_ncats);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(input_cat_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_input_cat_bwd: %s", cudaGetErrorString(e));
    }
    return pcb::launch_status(pcb::launch_k(input_cat_bwd_kernel, dim3(num_groups), dim3(256), smem,
                                            pcb::as_stream(stream), 1u, data, data_ld, node_flows, ld, B, grp_var,
                                            grp_node0, grp_count, grp_ncats, s_pfids, node_offset, param_flows,
                                            logspace_flows != 0, CB, missing, miss_sb, miss_sv, s_pids, params,
                                            atomic != 0),
                              "pcb_input_cat_bwd");
}
