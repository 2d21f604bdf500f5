// Sum-layer parameter flows on the tcgen05 tensor cores: the same contraction over the batch
// as sum_pflows.cu,
//   pf(r, k) += params(r, k) * sum_b A[r, b] * C[k, b],
//   A[r, b] = exp(lf[nid + r, b] - M_b),  C[k, b] = exp(em[cids[k], b] + M_b),
// with the accumulator D[128 nodes x TKC children] held in tensor memory for the whole
// batch slice. Per 32-sample chunk (double-buffered cp.async staging as in sum_pflows.cu)
// the CTA forms A and C in FP32, rounds them to bf16 (split into hi + lo parts for the
// accurate form) and writes them as K-major operands (K = samples); one thread then issues
// 2 K-steps of 16 x (1 or 3) tcgen05.mma into D and commits them to an mbarrier. The MMAs
// of chunk c run while chunk c + 1 is exponentiated; an operand buffer is rewritten only
// after the MMAs that read it have completed (double-buffered operands). At the end the
// accumulator is read back with tcgen05.ld and reduced across the cluster in rank order
// exactly as in sum_pflows.cu (deterministic, no float atomics for untied slots).
//
// Shared-memory operand layout (no swizzle, K-major): an operand of R rows x 32 samples is
// R/8 x 4 core matrices of 8 rows x 8 bf16 (16 bytes per row, 128 bytes per core matrix),
// core matrices 128 bytes apart along K and 512 bytes apart along the rows.
#include <cooperative_groups.h>

#include "tc05.cuh"

namespace cg = cooperative_groups;

namespace {

using namespace pcb::tc05;

constexpr int kThreads = 512;
constexpr int TMN = 128;       // nodes per tile (the MMA's M)
constexpr int KB = 32;         // samples per staged chunk
constexpr int kSliceUnit = 64;
constexpr int RS = KB + 4;     // fp32 staging row stride
constexpr int kParts = kThreads / KB;
constexpr int RT = TMN + 4;    // partial-tile row stride
constexpr int kMaxCluster = 8;
constexpr float kLog2e = 1.4426950408889634f;
constexpr uint32_t kLBO = 128;            // core matrices adjacent along K
constexpr uint32_t kSBO = (KB / 8) * 128;  // 8-row groups

__device__ __forceinline__ float ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// byte offset of (row r, sample k) in a K-major operand of 32 samples
__device__ __forceinline__ uint32_t op_off(int r, int k) {
    return (uint32_t)(r >> 3) * kSBO + (uint32_t)(k >> 3) * kLBO + (uint32_t)(r & 7) * 16 + (uint32_t)(k & 7) * 2;
}

template <int TKC, bool MODIFIED>
struct Plan {
    // fp32 staging, in words: node rows (flows [, mars]) and child rows of one chunk; two buffers
    static constexpr int sA = 0;
    static constexpr int sA2 = sA + TMN * RS;
    static constexpr int sC = sA2 + (MODIFIED ? 0 : TMN * RS);
    static constexpr int kStage = sC + TKC * RS;
    // bf16 operands, in bytes: per buffer A hi, A lo, C hi, C lo
    static constexpr uint32_t kA = TMN * KB * 2, kC = TKC * KB * 2;
    static constexpr uint32_t kOpBuf = 2 * kA + 2 * kC;
    static constexpr uint32_t oOp = ((2u * kStage * 4u) + 1023u) & ~1023u;
    static constexpr uint32_t oPart = oOp + 2 * kOpBuf;            // [kThreads] floats
    static constexpr uint32_t oM = oPart + kThreads * 4;           // [2][KB] floats
    static constexpr uint32_t oIdx = oM + 2 * KB * 4;              // cids, pids, pfids: [3][TKC] ints
    static constexpr uint32_t oBar = (oIdx + 3 * TKC * 4 + 7u) & ~7u;  // two mbarriers
    static constexpr uint32_t oSlot = oBar + 16;                   // tensor-memory address, fail flag
    static constexpr size_t bytes() { return oSlot + 16; }
    static_assert(2 * kStage >= TKC * RT, "the partial tile aliases the staging area");
};

template <int TKC, bool MODIFIED, bool ATOMIC, bool SPLIT>
__global__ void __launch_bounds__(kThreads, MODIFIED ? 2 : 1)
sum_pflows_tc05_kernel(const float* __restrict__ nf, const float* __restrict__ nm, const float* __restrict__ em,
                       int64_t ld, int B, const float* __restrict__ params, float* __restrict__ pf,
                       const PcbPflowTile* __restrict__ tiles, int rpb_log2, const int* __restrict__ cids,
                       const int* __restrict__ pids, const int* __restrict__ pfids, int slice, bool vec,
                       const int* __restrict__ deltas, int nlay, int32_t* __restrict__ status) {
    pcb::pdl_trigger();
    using P = Plan<TKC, MODIFIED>;
    static_assert(TKC == 64 || TKC == 128, "children per tile");
    extern __shared__ __align__(1024) uint8_t smem[];
    float* dsm = reinterpret_cast<float*>(smem);
    float* sPart = reinterpret_cast<float*>(smem + P::oPart);
    float* sM = reinterpret_cast<float*>(smem + P::oM);
    int* sCid = reinterpret_cast<int*>(smem + P::oIdx);
    int* sPid = sCid + TKC;
    int* sPfid = sPid + TKC;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + P::oBar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + P::oSlot);

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
    if (warp == 0) {
        tmem_alloc(slot, TKC);
        fence_before_sync();
    }
    if (tid == 32) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        slot[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    fence_after_sync();
    const uint32_t taddr = slot[0];
    pcb::pdl_wait();

    const int bs0 = crank * slice;
    const int bs1 = min(B, bs0 + slice);
    // chunks of this CTA's batch slice, for each of the nlay layers that share the tile's
    // parameters and flow slots (a tied set; layer i's node rows and child rows are the
    // tile's shifted by deltas[2 i] and deltas[2 i + 1]): all accumulate into D
    const int nchl = bs1 > bs0 ? (bs1 - bs0 + KB - 1) / KB : 0;
    const int nch = nchl * nlay;

    auto issue = [&](int cidx, int st) {
        const int li = nchl > 0 ? cidx / nchl : 0;
        const int b0 = bs0 + (cidx - li * nchl) * KB;
        const int dn = deltas ? __ldg(deltas + 2 * li) : 0;
        const int de = deltas ? __ldg(deltas + 2 * li + 1) : 0;
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
                    const float* g = (h == 0 ? nf : nm) + ((int64_t)t.nid + dn + r) * ld + b;
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
                const float* g = em + (int64_t)(row + de) * ld + b;
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

    // exponentiate 4 samples of one row and store them (hi [, lo]) into a K-major operand
    auto put4 = [&](uint8_t* hi, uint8_t* lo, int r, int k, float4 v, float4 m) {
        const float e0 = ex2((v.x + m.x) * kLog2e), e1 = ex2((v.y + m.y) * kLog2e);
        const float e2 = ex2((v.z + m.z) * kLog2e), e3 = ex2((v.w + m.w) * kLog2e);
        const __nv_bfloat162 h01 = __floats2bfloat162_rn(e0, e1), h23 = __floats2bfloat162_rn(e2, e3);
        const uint32_t off = op_off(r, k);
        *reinterpret_cast<uint2*>(hi + off) =
            make_uint2(*reinterpret_cast<const uint32_t*>(&h01), *reinterpret_cast<const uint32_t*>(&h23));
        if (SPLIT) {
            const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
            const __nv_bfloat162 l01 = __floats2bfloat162_rn(e0 - f01.x, e1 - f01.y);
            const __nv_bfloat162 l23 = __floats2bfloat162_rn(e2 - f23.x, e3 - f23.y);
            *reinterpret_cast<uint2*>(lo + off) =
                make_uint2(*reinterpret_cast<const uint32_t*>(&l01), *reinterpret_cast<const uint32_t*>(&l23));
        }
    };

    bool fail = false;
    if (nch > 0) issue(0, 0);
    for (int c = 0; c < nch; ++c) {
        const int st = c & 1;
        if (c + 1 < nch) {
            issue(c + 1, st ^ 1);
            pcb::cp_async_wait<1>();
        } else {
            pcb::cp_async_wait<0>();
        }
        __syncthreads();
        float(*sA)[RS] = reinterpret_cast<float(*)[RS]>(dsm + st * P::kStage + P::sA);
        float(*sA2)[RS] = reinterpret_cast<float(*)[RS]>(dsm + st * P::kStage + P::sA2);
        float(*sC)[RS] = reinterpret_cast<float(*)[RS]>(dsm + st * P::kStage + P::sC);
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
            sM[tid] = (m == -INFINITY) ? -INFINITY : -m;
            sM[KB + tid] = m;
        }
        // operand buffer ob was last read by the MMAs of chunk c - 2
        const int ob = c & 1;
        if (c >= 2 && !mbar_wait_bounded(&bar[ob], (uint32_t)(((c - 2) >> 1) & 1))) fail = true;
        __syncthreads();
        uint8_t* aHi = smem + P::oOp + ob * P::kOpBuf;
        uint8_t* aLo = aHi + P::kA;
        uint8_t* cHi = aLo + P::kA;
        uint8_t* cLo = cHi + P::kC;
        // items (row group of 8, half of the chunk's samples, 8 rows x 4 samples per warp):
        // each warp writes two whole adjacent core matrices (256 contiguous bytes)
        for (int i = tid; i < TMN * (KB / 4); i += kThreads) {
            const int w = i >> 5, q = i & 31;
            const int r = (w >> 1) * 8 + (q & 7), k = (w & 1) * 16 + (q >> 3) * 4;
            put4(aHi, aLo, r, k, *reinterpret_cast<const float4*>(&sA[r][k]),
                 *reinterpret_cast<const float4*>(&sM[k]));
        }
        for (int i = tid; i < TKC * (KB / 4); i += kThreads) {
            const int w = i >> 5, q = i & 31;
            const int r = (w >> 1) * 8 + (q & 7), k = (w & 1) * 16 + (q >> 3) * 4;
            put4(cHi, cLo, r, k, *reinterpret_cast<const float4*>(&sC[r][k]),
                 *reinterpret_cast<const float4*>(&sM[KB + k]));
        }
        fence_smem_async();
        __syncthreads();
        fence_after_sync();
        if (tid == 0) {
            constexpr uint32_t idesc = idesc_kk<TKC>();
            const uint32_t ah = smem_u32(aHi), al = smem_u32(aLo), ch = smem_u32(cHi), cl = smem_u32(cLo);
#pragma unroll
            for (int s = 0; s < KB / 16; ++s) {
                const uint32_t o = (uint32_t)s * 2 * kLBO;
                mma_bf16(taddr, desc(ah + o, kLBO, kSBO), desc(ch + o, kLBO, kSBO), idesc, (c > 0 || s > 0) ? 1u : 0u);
                if (SPLIT) {
                    mma_bf16(taddr, desc(al + o, kLBO, kSBO), desc(ch + o, kLBO, kSBO), idesc, 1u);
                    mma_bf16(taddr, desc(ah + o, kLBO, kSBO), desc(cl + o, kLBO, kSBO), idesc, 1u);
                }
            }
            commit(&bar[ob]);
        }
        // the staging buffer st is refilled by the next iteration's copies: its reads (the
        // operand writes above) completed before the barrier
    }
    // all MMAs done: the last commit tracks every earlier MMA of the issuing thread
    if (nch > 0 && !mbar_wait_bounded(&bar[(nch - 1) & 1], (uint32_t)(((nch - 1) >> 1) & 1))) fail = true;
    __syncthreads();
    fence_after_sync();

    // ---- accumulator -> partial tile in shared memory (child-major) ----
    float* red = dsm;  // [TKC][RT]
    {
        const int q = warp & 3;                   // lane quarter: rows 32 q .. + 31
        constexpr int CW = TKC / 4;               // columns per warp
        const int cb = (warp >> 2) * CW;
        const int r = q * 32 + lane;
#pragma unroll
        for (int c16 = 0; c16 < CW / 16; ++c16) {
            float v[16];
            tmem_ld16(taddr + ((uint32_t)(q * 32) << 16) + (uint32_t)(cb + c16 * 16), v);
            wait_ld();
#pragma unroll
            for (int j = 0; j < 16; ++j)
                red[(cb + c16 * 16 + j) * RT + r] = (nch > 0 && !fail) ? v[j] : (nch > 0 ? __int_as_float(0x7fc00000) : 0.f);
        }
    }
    if (fail) pcb::report_status(status, PCB_STATUS_WAIT_TIMEOUT);
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr, TKC);
    cluster.sync();
    constexpr int U = 8;
    const int per = (TMN * TKC + csize - 1) / csize;
    const int beg = crank * per;
    const int end = min(TMN * TKC, beg + per);
    for (int base = beg; base < end; base += kThreads * U) {
        float sv[U], wv[U], old[U];
        int64_t slot_[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = base + u * kThreads + tid;
            const int k = idx / TMN;
            const int i = idx % TMN;
            ok[u] = idx < end && i < t.n_rows && k < t.k_cnt;
            sv[u] = 0.f;
            wv[u] = 0.f;
            slot_[u] = 0;
            if (ok[u]) {
                for (int rr = 0; rr < csize; ++rr) sv[u] += cluster.map_shared_rank(red, rr)[k * RT + i];
                const int64_t roff = (int64_t)t.p_add + (int64_t)(i & rpb_mask);
                const int64_t blk = i >> rpb_log2;
                wv[u] = __ldg(params + (int64_t)sPid[k] + roff + blk * t.gs_p);
                slot_[u] = (int64_t)sPfid[k] + roff + blk * t.gs_pf;
            }
        }
        if (!ATOMIC) {
#pragma unroll
            for (int u = 0; u < U; ++u) old[u] = ok[u] ? pf[slot_[u]] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!ok[u]) continue;
            if (ATOMIC) atomicAdd(pf + slot_[u], sv[u] * wv[u]);
            else pf[slot_[u]] = old[u] + sv[u] * wv[u];
        }
    }
    cluster.sync();
}

template <int TKC, bool MODIFIED, bool ATOMIC, bool SPLIT>
int launch(int cs, const float* nf, const float* nm, const float* em, int64_t ld, int B, const float* params,
           float* pf, const PcbPflowTile* tiles, int num_tiles, int rpb_log2, const int* cids, const int* pids,
           const int* pfids, cudaStream_t s, bool vec, const int* deltas, int nlay) {
    const int slice = (int)pcb::cdiv(pcb::cdiv(B, cs), KB) * KB;
    using P = Plan<TKC, MODIFIED>;
    constexpr size_t smem = P::bytes();
    static_assert(smem <= 227 * 1024, "shared memory");
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    dev = dev < 0 ? 0 : (dev > 63 ? 63 : dev);
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(sum_pflows_tc05_kernel<TKC, MODIFIED, ATOMIC, SPLIT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_sum_pflows_tc05: %s", cudaGetErrorString(e));
        configured[dev] = true;
    }
    return pcb::launch_status(
        pcb::launch_k(sum_pflows_tc05_kernel<TKC, MODIFIED, ATOMIC, SPLIT>, dim3((unsigned)num_tiles * cs),
                      dim3(kThreads), smem, s, (unsigned)cs, nf, nm, em, ld, B, params, pf, tiles, rpb_log2, cids,
                      pids, pfids, slice, vec, deltas, nlay, pcb::status_word()),
        "pcb_sum_pflows_tc05");
}

template <int TKC, bool SPLIT>
int launch_flags(int cs, bool modified, bool atomic, const float* nf, const float* nm, const float* em, int64_t ld,
                 int B, const float* params, float* pf, const PcbPflowTile* tiles, int num_tiles, int rpb_log2,
                 const int* cids, const int* pids, const int* pfids, cudaStream_t s, bool vec, const int* deltas,
                 int nlay) {
#define PCB_PF(M, A) \
    launch<TKC, M, A, SPLIT>(cs, nf, nm, em, ld, B, params, pf, tiles, num_tiles, rpb_log2, cids, pids, pfids, s, vec, \
                             deltas, nlay)
    if (modified) return atomic ? PCB_PF(true, true) : PCB_PF(true, false);
    return atomic ? PCB_PF(false, true) : PCB_PF(false, false);
#undef PCB_PF
}

}  // namespace

namespace {

int pflows_tc05_impl(const float* node_flows, const float* node_mars, const float* element_mars, int64_t ld, int32_t B,
                     const float* params, float* param_flows, const PcbPflowTile* tiles, int32_t num_tiles,
                     int32_t rows_per_block, const int32_t* cids, const int32_t* pids, const int32_t* pfids,
                     int32_t modified, int32_t atomic, int32_t tile_children, int32_t prec, const int32_t* deltas,
                     int32_t nlay, void* stream) {
    if (!node_flows || !node_mars || !element_mars || !params || !param_flows || !tiles || !cids || !pids || !pfids ||
        B <= 0 || ld < B || num_tiles < 0 || rows_per_block <= 0 || (rows_per_block & (rows_per_block - 1)) ||
        (tile_children != 64 && tile_children != 128) || prec < 1 || prec > 2 || nlay < 1 || (nlay > 1 && !deltas))
        return pcb::set_error(PCB_E_ARG, "pcb_sum_pflows_tc05: bad arguments");
    if (num_tiles == 0) return PCB_OK;
    int rpb_log2 = 0;
    while ((1 << rpb_log2) < rows_per_block) ++rpb_log2;
    int cs = 1;
    while (cs < kMaxCluster && (int64_t)cs * kSliceUnit < B) cs *= 2;
    static int sms_of[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64) {
        if (sms_of[dev] == 0) cudaDeviceGetAttribute(&sms_of[dev], cudaDevAttrMultiProcessorCount, dev);
        const int per_sm = modified ? 2 : 1;
        while (cs > 1 && (int64_t)num_tiles * cs > (int64_t)per_sm * sms_of[dev]) cs /= 2;
    }
    if ((int64_t)num_tiles * cs > 2147483647) return pcb::set_error(PCB_E_ARG, "pcb_sum_pflows_tc05: too many tiles");
    const bool vec = pcb::vec_ok(node_flows, ld) && pcb::vec_ok(node_mars, ld) && pcb::vec_ok(element_mars, ld);
    cudaStream_t s = pcb::as_stream(stream);
    const bool mod = modified != 0, at = atomic != 0, split = prec == 2;
#define PCB_PK(T, S) \
    launch_flags<T, S>(cs, mod, at, node_flows, node_mars, element_mars, ld, B, params, param_flows, tiles, num_tiles, rpb_log2, cids, pids, pfids, s, vec, deltas, nlay)
    if (tile_children == 64) return split ? PCB_PK(64, true) : PCB_PK(64, false);
    return split ? PCB_PK(128, true) : PCB_PK(128, false);
#undef PCB_PK
}

}  // namespace

extern "C" int pcb_sum_pflows_tc05(const float* node_flows, const float* node_mars, const float* element_mars,
                                   int64_t ld, int32_t B, const float* params, float* param_flows,
                                   const PcbPflowTile* tiles, int32_t num_tiles, int32_t rows_per_block,
                                   const int32_t* cids, const int32_t* pids, const int32_t* pfids, int32_t modified,
                                   int32_t atomic, int32_t tile_children, int32_t prec, void* stream) {
    return pflows_tc05_impl(node_flows, node_mars, element_mars, ld, B, params, param_flows, tiles, num_tiles,
                            rows_per_block, cids, pids, pfids, modified, atomic, tile_children, prec, nullptr, 1,
                            stream);
}

extern "C" int pcb_sum_pflows_tc05_tied(const float* node_flows, const float* node_mars, const float* element_mars,
                                        int64_t ld, int32_t B, const float* params, float* param_flows,
                                        const PcbPflowTile* tiles, int32_t num_tiles, int32_t rows_per_block,
                                        const int32_t* cids, const int32_t* pids, const int32_t* pfids,
                                        int32_t modified, int32_t atomic, int32_t tile_children, int32_t prec,
                                        const int32_t* row_deltas, int32_t num_layers, void* stream) {
    return pflows_tc05_impl(node_flows, node_mars, element_mars, ld, B, params, param_flows, tiles, num_tiles,
                            rows_per_block, cids, pids, pfids, modified, atomic, tile_children, prec, row_deltas,
                            num_layers, stream);
}
