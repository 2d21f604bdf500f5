// Sum-layer parameter flows: a contraction over the batch.
//
// A tile covers up to 128 nodes (rows nid + r: consecutive node blocks that share their
// children) and up to TKC children (element rows cids[k], TKC = 32, 64 or 128):
//   pf(r, k) += params(r, k) * sum_b A[r, b] * C[k, b]
//   A[r, b] = exp(lf[nid + r, b] - M_b),  C[k, b] = exp(em[cids[k], b] + M_b)
// with lf = log(node flow) - log(node mar) and M_b = max_r lf[nid + r, b]: every
// exponential is taken once per (row, sample), not once per (node, child, sample).
//
// The batch is split over a thread-block cluster of up to 8 CTAs (fewer when the layer's
// tiles alone give about two CTAs per SM; a CTA then walks several chunks). A CTA copies 64
// samples of its slice at a time (all node rows and child rows in one batch of
// asynchronous copies), forms A and C, and contracts them either with FP32 FMA (prec 0)
// or on the tensor cores (prec 1: bf16 operands; prec 2: both operands split into
// bf16 hi + lo, three MMAs, FP32 accumulators). At the end the CTAs exchange their
// partial tiles through distributed shared memory and each adds the partials of its
// share of the outputs in rank order: the result does not depend on timing (no float
// atomics) and no global scratch is needed. Each (node, child) flow slot is owned by one
// tile, so the final update is a plain read-modify-write unless slots are shared by tied
// nodes (atomic = 1).
#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int kThreads = 256;
constexpr int TMN = 128;      // nodes per tile
constexpr int KB = 64;        // samples per staged chunk
constexpr int RS = KB + 4;    // fp32 staging row stride (16-byte rows)
constexpr int PS = KB / 2 + 4;  // packed bf16-pair row stride (conflict-free fragment loads)
constexpr int kMaxCluster = 8;

__device__ __forceinline__ void split_bf16(float lo_k, float hi_k, uint32_t& h, uint32_t& l) {
    __nv_bfloat162 hv = __floats2bfloat162_rn(lo_k, hi_k);
    const float2 hf = __bfloat1622float2(hv);
    __nv_bfloat162 lv = __floats2bfloat162_rn(lo_k - hf.x, hi_k - hf.y);
    h = *reinterpret_cast<uint32_t*>(&hv);
    l = *reinterpret_cast<uint32_t*>(&lv);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Shared-memory plan in 4-byte words (16-byte aligned arrays).
template <int TKC, bool MODIFIED, int PREC>
struct Plan {
    static constexpr int NB = PREC == 2 ? 2 : (PREC == 1 ? 1 : 0);
    static constexpr int oA = 0;
    static constexpr int oA2 = oA + TMN * RS;
    static constexpr int oC = oA2 + (MODIFIED ? 0 : TMN * RS);
    static constexpr int oPA = oC + TKC * RS;
    static constexpr int oPC = oPA + NB * TMN * PS;
    static constexpr int oPart = oPC + NB * TKC * PS;
    static constexpr int oM = oPart + kThreads;
    static constexpr int oCid = oM + KB;
    static constexpr int words = oCid + TKC;
    static_assert(words >= TMN * TKC, "the partial tile aliases the staging area");
    static constexpr size_t bytes() { return 4ull * words; }
};

template <int TKC, bool MODIFIED, bool ATOMIC, int PREC>
__global__ void __launch_bounds__(kThreads)
sum_pflows_kernel(const float* __restrict__ nf, const float* __restrict__ nm, const float* __restrict__ em,
                  int64_t ld, int B, const float* __restrict__ params, float* __restrict__ pf,
                  const PcbPflowTile* __restrict__ tiles, int rpb_log2, const int* __restrict__ cids,
                  const int* __restrict__ pids, const int* __restrict__ pfids, int slice, bool vec) {
    pcb::pdl_begin();
    using P = Plan<TKC, MODIFIED, PREC>;
    extern __shared__ __align__(16) float dsm[];
    float(*sA)[RS] = reinterpret_cast<float(*)[RS]>(dsm + P::oA);
    float(*sA2)[RS] = reinterpret_cast<float(*)[RS]>(dsm + P::oA2);
    float(*sC)[RS] = reinterpret_cast<float(*)[RS]>(dsm + P::oC);
    uint32_t* pA = reinterpret_cast<uint32_t*>(dsm + P::oPA);
    uint32_t* pC = reinterpret_cast<uint32_t*>(dsm + P::oPC);
    float* sPart = dsm + P::oPart;
    float* sM = dsm + P::oM;
    int* sCid = reinterpret_cast<int*>(dsm + P::oCid);

    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank();
    const int csize = (int)cluster.num_blocks();
    const PcbPflowTile t = tiles[blockIdx.x / csize];
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int rpb_mask = (1 << rpb_log2) - 1;

    if (tid < TKC) sCid[tid] = (tid < t.k_cnt) ? __ldg(cids + t.k_off + tid) : -1;
    __syncthreads();

    // FP32: thread (ty, tx) owns nodes ty * 8 .. + 8 and children tx + 16 * j.
    // Tensor cores: warp w owns nodes 16 w .. 16 w + 15 and all TKC children.
    constexpr int FJ = TKC / 16;
    constexpr int NT = TKC / 8;
    float acc[PREC == 0 ? 8 : NT][PREC == 0 ? FJ : 4];
#pragma unroll
    for (int a = 0; a < (PREC == 0 ? 8 : NT); ++a)
#pragma unroll
        for (int j = 0; j < (PREC == 0 ? FJ : 4); ++j) acc[a][j] = 0.f;

    const int bs0 = crank * slice;
    const int bs1 = min(B, bs0 + slice);
    for (int b0 = bs0; b0 < bs1; b0 += KB) {
        // ---- one batch of asynchronous copies: node rows (flows, mars) and child rows ----
        {
            constexpr int NX = KB / 4;
#pragma unroll
            for (int it = 0; it < TMN * NX / kThreads; ++it) {
                const int idx = tid + it * kThreads;
                const int r = idx / NX;
                const int c4 = (idx % NX) * 4;
                const int b = b0 + c4;
#pragma unroll
                for (int h = 0; h < (MODIFIED ? 1 : 2); ++h) {
                    float* d = h == 0 ? &sA[r][c4] : &sA2[r][c4];
                    if (r < t.n_rows) {
                        const float* g = (h == 0 ? nf : nm) + ((int64_t)t.nid + r) * ld + b;
                        if (vec && b + 3 < bs1) {
                            pcb::cp_async16(d, g);
                        } else {
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                if (b + j < bs1) pcb::cp_async4(d + j, g + j);
                                else d[j] = -INFINITY;
                            }
                        }
                    } else {
                        *reinterpret_cast<float4*>(d) = make_float4(-INFINITY, -INFINITY, -INFINITY, -INFINITY);
                    }
                }
            }
#pragma unroll
            for (int it = 0; it < TKC * NX / kThreads; ++it) {
                const int idx = tid + it * kThreads;
                const int k = idx / NX;
                const int c4 = (idx % NX) * 4;
                const int b = b0 + c4;
                float* d = &sC[k][c4];
                const int row = sCid[k];
                if (row >= 0) {
                    const float* g = em + (int64_t)row * ld + b;
                    if (vec && b + 3 < bs1) {
                        pcb::cp_async16(d, g);
                    } else {
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            if (b + j < bs1) pcb::cp_async4(d + j, g + j);
                            else d[j] = -INFINITY;
                        }
                    }
                } else {
                    *reinterpret_cast<float4*>(d) = make_float4(-INFINITY, -INFINITY, -INFINITY, -INFINITY);
                }
            }
            pcb::cp_async_commit();
            pcb::cp_async_wait<0>();
        }
        __syncthreads();

        // ---- lf = log f - log m (unmodified flows), then M_b = max over the tile's nodes ----
        {
            const int b = tid % KB;
            const int part = tid / KB;  // 4 parts of 32 rows
            float mx = -INFINITY;
            for (int r = part * (TMN / 4); r < (part + 1) * (TMN / 4); ++r) {
                float v = sA[r][b];
                if (!MODIFIED) {
                    const float m2 = sA2[r][b];
                    v = (m2 == -INFINITY) ? -INFINITY : logf(v) - m2;
                    sA[r][b] = v;
                }
                mx = fmaxf(mx, v);
            }
            sPart[part * KB + b] = mx;
        }
        __syncthreads();
        if (tid < KB) sM[tid] = fmaxf(fmaxf(sPart[tid], sPart[KB + tid]), fmaxf(sPart[2 * KB + tid], sPart[3 * KB + tid]));
        __syncthreads();

        if constexpr (PREC == 0) {
            for (int idx = tid; idx < TMN * KB; idx += kThreads) {
                const int r = idx / KB, b = idx % KB;
                const float m = sM[b];
                sA[r][b] = (m == -INFINITY) ? 0.f : __expf(sA[r][b] - m);
            }
            for (int idx = tid; idx < TKC * KB; idx += kThreads) {
                const int k = idx / KB, b = idx % KB;
                const float m = sM[b];
                sC[k][b] = (m == -INFINITY) ? 0.f : __expf(sC[k][b] + m);
            }
            __syncthreads();
            const int tx = tid % 16;
            const int ty = tid / 16;
#pragma unroll 2
            for (int b = 0; b < KB; b += 4) {
                float4 cv[FJ];
#pragma unroll
                for (int j = 0; j < FJ; ++j) cv[j] = *reinterpret_cast<const float4*>(&sC[tx + 16 * j][b]);
#pragma unroll
                for (int a = 0; a < 8; ++a) {
                    const float4 av = *reinterpret_cast<const float4*>(&sA[ty * 8 + a][b]);
#pragma unroll
                    for (int j = 0; j < FJ; ++j) {
                        acc[a][j] = fmaf(av.x, cv[j].x, acc[a][j]);
                        acc[a][j] = fmaf(av.y, cv[j].y, acc[a][j]);
                        acc[a][j] = fmaf(av.z, cv[j].z, acc[a][j]);
                        acc[a][j] = fmaf(av.w, cv[j].w, acc[a][j]);
                    }
                }
            }
        } else {
            constexpr bool SPLIT = PREC == 2;
            // ---- exponentiate and pack sample pairs as bf16 (hi, lo) ----
            for (int idx = tid; idx < TMN * (KB / 2); idx += kThreads) {
                const int r = idx / (KB / 2), j = idx % (KB / 2);
                const float2 v = *reinterpret_cast<const float2*>(&sA[r][2 * j]);
                const float m0 = sM[2 * j], m1 = sM[2 * j + 1];
                const float e0 = (m0 == -INFINITY) ? 0.f : __expf(v.x - m0);
                const float e1 = (m1 == -INFINITY) ? 0.f : __expf(v.y - m1);
                if (SPLIT) split_bf16(e0, e1, pA[r * PS + j], pA[TMN * PS + r * PS + j]);
                else pA[r * PS + j] = pack_bf16(e0, e1);
            }
            for (int idx = tid; idx < TKC * (KB / 2); idx += kThreads) {
                const int k = idx / (KB / 2), j = idx % (KB / 2);
                const float2 v = *reinterpret_cast<const float2*>(&sC[k][2 * j]);
                const float m0 = sM[2 * j], m1 = sM[2 * j + 1];
                const float e0 = (m0 == -INFINITY) ? 0.f : __expf(v.x + m0);
                const float e1 = (m1 == -INFINITY) ? 0.f : __expf(v.y + m1);
                if (SPLIT) split_bf16(e0, e1, pC[k * PS + j], pC[TKC * PS + k * PS + j]);
                else pC[k * PS + j] = pack_bf16(e0, e1);
            }
            __syncthreads();
            const int g = lane >> 2, q = lane & 3;
            const int mr = warp * 16 + g;
#pragma unroll
            for (int kk = 0; kk < KB / 2; kk += 8) {
                const uint32_t a0 = pA[mr * PS + kk + q], a1 = pA[(mr + 8) * PS + kk + q];
                const uint32_t a2 = pA[mr * PS + kk + 4 + q], a3 = pA[(mr + 8) * PS + kk + 4 + q];
                uint32_t l0 = 0, l1 = 0, l2 = 0, l3 = 0;
                if (SPLIT) {
                    l0 = pA[TMN * PS + mr * PS + kk + q];
                    l1 = pA[TMN * PS + (mr + 8) * PS + kk + q];
                    l2 = pA[TMN * PS + mr * PS + kk + 4 + q];
                    l3 = pA[TMN * PS + (mr + 8) * PS + kk + 4 + q];
                }
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) {
                    const int n = nt * 8 + g;
                    const uint32_t b0v = pC[n * PS + kk + q], b1v = pC[n * PS + kk + 4 + q];
                    mma_bf16(acc[nt], a0, a1, a2, a3, b0v, b1v);
                    if (SPLIT) {
                        mma_bf16(acc[nt], l0, l1, l2, l3, b0v, b1v);
                        mma_bf16(acc[nt], a0, a1, a2, a3, pC[TKC * PS + n * PS + kk + q],
                                 pC[TKC * PS + n * PS + kk + 4 + q]);
                    }
                }
            }
        }
        __syncthreads();  // the next chunk (or the partial tile) overwrites the staging area
    }

    // ---- partial tile -> shared memory; cluster-wide fixed-order sum ----
    float* red = dsm;  // [TMN][TKC]
    if constexpr (PREC == 0) {
        const int tx = tid % 16, ty = tid / 16;
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int j = 0; j < FJ; ++j) red[(ty * 8 + a) * TKC + tx + 16 * j] = acc[a][j];
    } else {
        const int g = lane >> 2, q = lane & 3;
        const int mr = warp * 16 + g;
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const int n = nt * 8 + 2 * q;
            red[mr * TKC + n] = acc[nt][0];
            red[mr * TKC + n + 1] = acc[nt][1];
            red[(mr + 8) * TKC + n] = acc[nt][2];
            red[(mr + 8) * TKC + n + 1] = acc[nt][3];
        }
    }
    cluster.sync();
    const int per = (TMN * TKC + csize - 1) / csize;
    const int end = min(TMN * TKC, (crank + 1) * per);
    for (int idx = crank * per + tid; idx < end; idx += kThreads) {
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

template <int TKC, bool MODIFIED, bool ATOMIC, int PREC>
int launch(int cs, const float* nf, const float* nm, const float* em, int64_t ld, int B, const float* params,
           float* pf, const PcbPflowTile* tiles, int num_tiles, int rpb_log2, const int* cids, const int* pids,
           const int* pfids, cudaStream_t s, bool vec) {
    const int slice = (int)pcb::cdiv(pcb::cdiv(B, cs), KB) * KB;
    using P = Plan<TKC, MODIFIED, PREC>;
    constexpr size_t smem = P::bytes();
    static_assert(P::bytes() <= 227 * 1024, "shared memory");
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    dev = dev < 0 ? 0 : (dev > 63 ? 63 : dev);
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(sum_pflows_kernel<TKC, MODIFIED, ATOMIC, PREC>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_sum_pflows: %s", cudaGetErrorString(e));
        configured[dev] = true;
    }
    return pcb::launch_status(pcb::launch_k(sum_pflows_kernel<TKC, MODIFIED, ATOMIC, PREC>, dim3((unsigned)num_tiles * cs),
                                            dim3(kThreads), smem, s, (unsigned)cs, nf, nm, em, ld, B, params, pf,
                                            tiles, rpb_log2, cids, pids, pfids, slice, vec),
                              "pcb_sum_pflows");
}

template <int TKC, int PREC>
int launch_flags(int cs, bool modified, bool atomic, const float* nf, const float* nm, const float* em, int64_t ld,
                 int B, const float* params, float* pf, const PcbPflowTile* tiles, int num_tiles, int rpb_log2,
                 const int* cids, const int* pids, const int* pfids, cudaStream_t s, bool vec) {
#define PCB_PF(M, A) \
    launch<TKC, M, A, PREC>(cs, nf, nm, em, ld, B, params, pf, tiles, num_tiles, rpb_log2, cids, pids, pfids, s, vec)
    if (modified) return atomic ? PCB_PF(true, true) : PCB_PF(true, false);
    return atomic ? PCB_PF(false, true) : PCB_PF(false, false);
#undef PCB_PF
}

}  // namespace

extern "C" int pcb_sum_pflows(const float* node_flows, const float* node_mars, const float* element_mars, int64_t ld,
                              int32_t B, const float* params, float* param_flows, const PcbPflowTile* tiles,
                              int32_t num_tiles, int32_t rows_per_block, const int32_t* cids, const int32_t* pids,
                              const int32_t* pfids, int32_t modified, int32_t atomic, int32_t tile_children,
                              int32_t prec, void* stream) {
    if (!node_flows || !node_mars || !element_mars || !params || !param_flows || !tiles || !cids || !pids || !pfids ||
        B <= 0 || ld < B || num_tiles < 0 || rows_per_block <= 0 || (rows_per_block & (rows_per_block - 1)) ||
        (tile_children != 32 && tile_children != 64 && tile_children != 128) || prec < 0 || prec > 2)
        return pcb::set_error(PCB_E_ARG, "pcb_sum_pflows: bad arguments");
    if (num_tiles == 0) return PCB_OK;
    int rpb_log2 = 0;
    while ((1 << rpb_log2) < rows_per_block) ++rpb_log2;
    // one CTA per 64-sample slice, up to 8 CTAs per cluster (a power of two); layers with many
    // tiles take smaller clusters (each CTA then walks several 64-sample chunks) so that the
    // launch stays within about two CTAs per SM instead of adding waves of short CTAs
    int cs = 1;
    while (cs < kMaxCluster && (int64_t)cs * KB < B) cs *= 2;
    static int sms_of[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64) {
        if (sms_of[dev] == 0) cudaDeviceGetAttribute(&sms_of[dev], cudaDevAttrMultiProcessorCount, dev);
        while (cs > 1 && (int64_t)num_tiles * cs > 2 * (int64_t)sms_of[dev]) cs /= 2;
    }
    if ((int64_t)num_tiles * cs > 2147483647) return pcb::set_error(PCB_E_ARG, "pcb_sum_pflows: too many tiles");
    const bool vec = pcb::vec_ok(node_flows, ld) && pcb::vec_ok(node_mars, ld) && pcb::vec_ok(element_mars, ld);
    cudaStream_t s = pcb::as_stream(stream);
    const bool mod = modified != 0, at = atomic != 0;
#define PCB_PK(T, P) \
    launch_flags<T, P>(cs, mod, at, node_flows, node_mars, element_mars, ld, B, params, param_flows, tiles, num_tiles, rpb_log2, cids, pids, pfids, s, vec)
    if (tile_children == 32) return prec == 0 ? PCB_PK(32, 0) : (prec == 1 ? PCB_PK(32, 1) : PCB_PK(32, 2));
    if (tile_children == 64) return prec == 0 ? PCB_PK(64, 0) : (prec == 1 ? PCB_PK(64, 1) : PCB_PK(64, 2));
    return prec == 0 ? PCB_PK(128, 0) : (prec == 1 ? PCB_PK(128, 1) : PCB_PK(128, 2));
#undef PCB_PK
}
