// Sum-layer parameter flows: a contraction over the batch.
//
// A tile covers up to 128 nodes (rows nid + r: consecutive node blocks that share their
// children) and up to TKC children (element rows cids[k], TKC = 32, 64 or 128):
//   pf(r, k) += params(r, k) * sum_b A[r, b] * C[k, b]
//   A[r, b] = exp(lf[nid + r, b] - M_b),  C[k, b] = exp(em[cids[k], b] + M_b)
// with lf = log(node flow) - log(node mar) and M_b = max_r lf[nid + r, b]: every
// exponential is taken once per (row, sample), not once per (node, child, sample).
//
// The batch is split over a thread-block cluster of up to 8 CTAs, one per 64-sample slice
// (fewer when the layer's tiles alone give about two CTAs per SM; a CTA then walks a longer
// slice). A CTA walks its slice in chunks of 32 samples, double-buffered: the copies of the
// next chunk (all node rows and child rows in one batch of asynchronous copies) are in
// flight while the current one is reduced. It forms A and C (4 samples per thread and
// step), and contracts them either with FP32 FMA (prec 0) or on the tensor cores (prec 1: bf16 operands; prec 2: both operands split into
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

constexpr int kThreads = 512;
constexpr int TMN = 128;      // nodes per tile
constexpr int KB = 32;        // samples per staged chunk (two chunks in flight)
constexpr int kSliceUnit = 64;  // cluster sizing: one CTA per 64-sample slice
constexpr int RS = KB + 4;    // fp32 staging row stride (16-byte rows)
constexpr int PS = KB / 2 + 4;  // packed bf16-pair row stride (conflict-free fragment loads)
constexpr int kParts = kThreads / KB;  // row parts of the max pass
constexpr int RT = TMN + 4;   // partial-tile row stride (child-major; conflict-free fragment stores)
constexpr int kMaxCluster = 8;
constexpr float kLog2e = 1.4426950408889634f;  // log2(e): exp(x) = 2^(x log2 e)

// 2^x with the hardware approximation (flushes subnormal results to zero).
__device__ __forceinline__ float ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

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

// Shared-memory plan in 4-byte words (16-byte aligned arrays). Two staging buffers (chunk
// c + 1 is copied while chunk c is reduced), each holding the node rows (flows, and mars
// for unmodified flows) and the child rows of one chunk.
template <int TKC, bool MODIFIED, int PREC>
struct Plan {
    static constexpr int NB = PREC == 2 ? 2 : (PREC == 1 ? 1 : 0);
    static constexpr int sA = 0;
    static constexpr int sA2 = sA + TMN * RS;
    static constexpr int sC = sA2 + (MODIFIED ? 0 : TMN * RS);
    static constexpr int kStage = sC + TKC * RS;
    static constexpr int oPA = 2 * kStage;
    static constexpr int oPC = oPA + NB * TMN * PS;
    static constexpr int oPart = oPC + NB * TKC * PS;
    static constexpr int oM = oPart + kThreads;   // [2][KB]: -M_b for A, +M_b for C
    static constexpr int oCid = oM + 2 * KB;
    static constexpr int oPid = oCid + TKC;
    static constexpr int oPfid = oPid + TKC;
    static constexpr int words = oPfid + TKC;
    static_assert(2 * kStage >= TKC * RT, "the partial tile aliases the staging area");
    static constexpr size_t bytes() { return 4ull * words; }
};

template <int TKC, bool MODIFIED, bool ATOMIC, int PREC>
__global__ void __launch_bounds__(kThreads, (PREC == 0 && TKC == 128) ? 1 : 2)
sum_pflows_kernel(const float* __restrict__ nf, const float* __restrict__ nm, const float* __restrict__ em,
                  int64_t ld, int B, const float* __restrict__ params, float* __restrict__ pf,
                  const PcbPflowTile* __restrict__ tiles, int rpb_log2, const int* __restrict__ cids,
                  const int* __restrict__ pids, const int* __restrict__ pfids, int slice, bool vec) {
    // The tile and its child indices (compiled tables) are read before the wait for the
    // previous kernel; the flows and values after it.
    pcb::pdl_trigger();
    using P = Plan<TKC, MODIFIED, PREC>;
    extern __shared__ __align__(16) float dsm[];
    uint32_t* pA = reinterpret_cast<uint32_t*>(dsm + P::oPA);
    uint32_t* pC = reinterpret_cast<uint32_t*>(dsm + P::oPC);
    float* sPart = dsm + P::oPart;
    float* sM = dsm + P::oM;
    int* sCid = reinterpret_cast<int*>(dsm + P::oCid);
    int* sPid = reinterpret_cast<int*>(dsm + P::oPid);
    int* sPfid = reinterpret_cast<int*>(dsm + P::oPfid);

    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank();
    const int csize = (int)cluster.num_blocks();
    const PcbPflowTile t = tiles[blockIdx.x / csize];
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int rpb_mask = (1 << rpb_log2) - 1;

    if (tid < TKC) {
        const bool in = tid < t.k_cnt;
        sCid[tid] = in ? __ldg(cids + t.k_off + tid) : -1;
        sPid[tid] = in ? __ldg(pids + t.k_off + tid) : 0;
        sPfid[tid] = in ? __ldg(pfids + t.k_off + tid) : 0;
    }
    __syncthreads();
    pcb::pdl_wait();

    // FP32: thread (ty, tx) owns nodes ty * FR .. + FR and children tx + 16 * j.
    // Tensor cores: warp w owns nodes 16 (w % 8) .. + 15 and children half w / 8.
    constexpr int FR = TMN * 16 / kThreads;
    constexpr int FJ = TKC / 16;
    constexpr int NT = TKC / 16;
    static_assert(kThreads == 512 && FR >= 1 && NT >= 1, "thread layout");
    float acc[PREC == 0 ? FR : NT][PREC == 0 ? FJ : 4];
#pragma unroll
    for (int a = 0; a < (PREC == 0 ? FR : NT); ++a)
#pragma unroll
        for (int j = 0; j < (PREC == 0 ? FJ : 4); ++j) acc[a][j] = 0.f;

    const int bs0 = crank * slice;
    const int bs1 = min(B, bs0 + slice);
    const int nch = bs1 > bs0 ? (bs1 - bs0 + KB - 1) / KB : 0;

    // one batch of asynchronous copies per chunk: node rows (flows, mars) and child rows
    auto issue = [&](int b0, int st) {
        float* stage = dsm + st * P::kStage;
        constexpr int NX = KB / 4;
#pragma unroll
        for (int it = 0; it < TMN * NX / kThreads; ++it) {
            const int idx = tid + it * kThreads;
            const int r = idx / NX;
            const int c4 = (idx % NX) * 4;
            const int b = b0 + c4;
#pragma unroll
            for (int h = 0; h < (MODIFIED ? 1 : 2); ++h) {
                float* d = stage + (h == 0 ? P::sA : P::sA2) + r * RS + c4;
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
        for (int it = 0; it < (TKC * NX + kThreads - 1) / kThreads; ++it) {
            const int idx = tid + it * kThreads;
            if (idx >= TKC * NX) break;
            const int k = idx / NX;
            const int c4 = (idx % NX) * 4;
            const int b = b0 + c4;
            float* d = stage + P::sC + k * RS + c4;
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
    };

    if (nch > 0) issue(bs0, 0);
    for (int c = 0; c < nch; ++c) {
        const int st = c & 1;
        // the other buffer was last read before the previous chunk's contraction barrier
        if (c + 1 < nch) {
            issue(bs0 + (c + 1) * KB, st ^ 1);
            pcb::cp_async_wait<1>();
        } else {
            pcb::cp_async_wait<0>();
        }
        __syncthreads();
        float(*sA)[RS] = reinterpret_cast<float(*)[RS]>(dsm + st * P::kStage + P::sA);
        float(*sA2)[RS] = reinterpret_cast<float(*)[RS]>(dsm + st * P::kStage + P::sA2);
        float(*sC)[RS] = reinterpret_cast<float(*)[RS]>(dsm + st * P::kStage + P::sC);

        // ---- lf = log f - log m (unmodified flows), then M_b = max over the tile's nodes ----
        {
            const int b = tid % KB;
            const int part = tid / KB;
            float mx = -INFINITY;
#pragma unroll 4
            for (int r = part * (TMN / kParts); r < (part + 1) * (TMN / kParts); ++r) {
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
        if (tid < KB) {
            float m = sPart[tid];
#pragma unroll
            for (int p = 1; p < kParts; ++p) m = fmaxf(m, sPart[p * KB + tid]);
            // A = 2^((lf - M) log2e), C = 2^((em + M) log2e); a sample whose rows are all -inf
            // gets A = 0 (M taken as +inf there) and C = 0 (M as -inf). The sums are formed
            // before scaling: lf and M (em and -M) are close, so the difference is exact.
            sM[tid] = (m == -INFINITY) ? -INFINITY : -m;
            sM[KB + tid] = m;
        }
        __syncthreads();

        if constexpr (PREC == 0) {
            for (int idx = tid; idx < TMN * KB; idx += kThreads) {
                const int r = idx / KB, b = idx % KB;
                sA[r][b] = ex2((sA[r][b] + sM[b]) * kLog2e);
            }
            for (int idx = tid; idx < TKC * KB; idx += kThreads) {
                const int k = idx / KB, b = idx % KB;
                sC[k][b] = ex2((sC[k][b] + sM[KB + b]) * kLog2e);
            }
            __syncthreads();
            const int tx = tid % 16;
            const int ty = tid / 16;
#pragma unroll 1
            for (int b = 0; b < KB; b += 4) {
                float4 cv[FJ];
#pragma unroll
                for (int j = 0; j < FJ; ++j) cv[j] = *reinterpret_cast<const float4*>(&sC[tx + 16 * j][b]);
#pragma unroll
                for (int a = 0; a < FR; ++a) {
                    const float4 av = *reinterpret_cast<const float4*>(&sA[ty * FR + a][b]);
#pragma unroll
                    for (int j = 0; j < FJ; ++j) {
                        acc[a][j] = fmaf(av.x, cv[j].x, acc[a][j]);
                        acc[a][j] = fmaf(av.y, cv[j].y, acc[a][j]);
                        acc[a][j] = fmaf(av.z, cv[j].z, acc[a][j]);
                        acc[a][j] = fmaf(av.w, cv[j].w, acc[a][j]);
                    }
                }
            }
            __syncthreads();  // the next chunk's copies overwrite this buffer
        } else {
            constexpr bool SPLIT = PREC == 2;
            // ---- exponentiate and pack sample pairs as bf16 (hi, lo), 4 samples per step ----
            constexpr int NX = KB / 4;
            for (int idx = tid; idx < TMN * NX; idx += kThreads) {
                const int r = idx / NX, c4 = (idx % NX) * 4;
                const float4 v = *reinterpret_cast<const float4*>(&sA[r][c4]);
                const float4 m = *reinterpret_cast<const float4*>(&sM[c4]);
                const float e0 = ex2((v.x + m.x) * kLog2e);
                const float e1 = ex2((v.y + m.y) * kLog2e);
                const float e2 = ex2((v.z + m.z) * kLog2e);
                const float e3 = ex2((v.w + m.w) * kLog2e);
                uint2 h, l;
                if (SPLIT) {
                    split_bf16(e0, e1, h.x, l.x);
                    split_bf16(e2, e3, h.y, l.y);
                    *reinterpret_cast<uint2*>(&pA[TMN * PS + r * PS + c4 / 2]) = l;
                } else {
                    h.x = pack_bf16(e0, e1);
                    h.y = pack_bf16(e2, e3);
                }
                *reinterpret_cast<uint2*>(&pA[r * PS + c4 / 2]) = h;
            }
            for (int idx = tid; idx < TKC * NX; idx += kThreads) {
                const int k = idx / NX, c4 = (idx % NX) * 4;
                const float4 v = *reinterpret_cast<const float4*>(&sC[k][c4]);
                const float4 m = *reinterpret_cast<const float4*>(&sM[KB + c4]);
                const float e0 = ex2((v.x + m.x) * kLog2e);
                const float e1 = ex2((v.y + m.y) * kLog2e);
                const float e2 = ex2((v.z + m.z) * kLog2e);
                const float e3 = ex2((v.w + m.w) * kLog2e);
                uint2 h, l;
                if (SPLIT) {
                    split_bf16(e0, e1, h.x, l.x);
                    split_bf16(e2, e3, h.y, l.y);
                    *reinterpret_cast<uint2*>(&pC[TKC * PS + k * PS + c4 / 2]) = l;
                } else {
                    h.x = pack_bf16(e0, e1);
                    h.y = pack_bf16(e2, e3);
                }
                *reinterpret_cast<uint2*>(&pC[k * PS + c4 / 2]) = h;
            }
            __syncthreads();
            const int g = lane >> 2, q = lane & 3;
            const int mr = (warp % 8) * 16 + g;
            const int nw = (warp / 8) * (TKC / 2);
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
                    const int n = nw + nt * 8 + g;
                    const uint32_t b0v = pC[n * PS + kk + q], b1v = pC[n * PS + kk + 4 + q];
                    mma_bf16(acc[nt], a0, a1, a2, a3, b0v, b1v);
                    if (SPLIT) {
                        mma_bf16(acc[nt], l0, l1, l2, l3, b0v, b1v);
                        mma_bf16(acc[nt], a0, a1, a2, a3, pC[TKC * PS + n * PS + kk + q],
                                 pC[TKC * PS + n * PS + kk + 4 + q]);
                    }
                }
            }
            // The packed operands are rewritten only after the next chunk's first barrier, and
            // this chunk's staging buffer was last read before the barrier above.
        }
    }
    __syncthreads();  // the partial tile overwrites the staging area

    // ---- partial tile -> shared memory (child-major); cluster-wide fixed-order sum ----
    float* red = dsm;  // [TKC][RT]
    if constexpr (PREC == 0) {
        const int tx = tid % 16, ty = tid / 16;
#pragma unroll
        for (int a = 0; a < FR; ++a)
#pragma unroll
            for (int j = 0; j < FJ; ++j) red[(tx + 16 * j) * RT + ty * FR + a] = acc[a][j];
    } else {
        const int g = lane >> 2, q = lane & 3;
        const int mr = (warp % 8) * 16 + g;
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const int n = (warp / 8) * (TKC / 2) + nt * 8 + 2 * q;
            red[n * RT + mr] = acc[nt][0];
            red[(n + 1) * RT + mr] = acc[nt][1];
            red[n * RT + mr + 8] = acc[nt][2];
            red[(n + 1) * RT + mr + 8] = acc[nt][3];
        }
    }
    cluster.sync();
    // Outputs (child k, node i) with the node fastest, so that consecutive threads touch
    // consecutive parameters and flow slots; U outputs per thread at a time, all loads of a
    // round issued before any of its stores.
    constexpr int U = 8;
    const int per = (TMN * TKC + csize - 1) / csize;
    const int beg = crank * per;
    const int end = min(TMN * TKC, beg + per);
    for (int base = beg; base < end; base += kThreads * U) {
        float sv[U], wv[U], old[U];
        int64_t slot[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = base + u * kThreads + tid;
            const int k = idx / TMN;
            const int i = idx % TMN;
            ok[u] = idx < end && i < t.n_rows && k < t.k_cnt;
            sv[u] = 0.f;
            wv[u] = 0.f;
            slot[u] = 0;
            if (ok[u]) {
                for (int r = 0; r < csize; ++r) sv[u] += cluster.map_shared_rank(red, r)[k * RT + i];
                const int64_t roff = (int64_t)t.p_add + (int64_t)(i & rpb_mask);
                const int64_t blk = i >> rpb_log2;
                wv[u] = __ldg(params + (int64_t)sPid[k] + roff + blk * t.gs_p);
                slot[u] = (int64_t)sPfid[k] + roff + blk * t.gs_pf;
            }
        }
        if (!ATOMIC) {
#pragma unroll
            for (int u = 0; u < U; ++u) old[u] = ok[u] ? pf[slot[u]] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!ok[u]) continue;
            if (ATOMIC) atomicAdd(pf + slot[u], sv[u] * wv[u]);
            else pf[slot[u]] = old[u] + sv[u] * wv[u];
        }
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
    while (cs < kMaxCluster && (int64_t)cs * kSliceUnit < B) cs *= 2;
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
