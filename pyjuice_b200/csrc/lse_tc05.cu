// Log-sum-exp contractions on the 5th-generation tensor cores (tcgen05, accumulators in
// tensor memory), for tiles of at most 128 terms.
//
// Same result as pcb_lse_contract in its BF16 forms:
//   acc[r, b] = sum_k W(k, r) * exp(src[krow[k], b] - m_b),  m_b = max_k src[krow[k], b]
// with mode 0 writing log(acc) + m (sum forward) and modes 1/2 writing acc * exp(aux + m)
// (element flows; mode 2 first turns node flows into log f - log m).
//
// Two kernels:
//  * pack: W(k, r) of every tile, rounded to bf16 (hi) plus the bf16 rounding of the
//    remainder (lo), written once per pass in the canonical no-swizzle K-major layout of a
//    128 x 128 UMMA operand (8 x 8 core matrices of 128 contiguous bytes; adjacent core
//    matrices 128 bytes apart along K and 2048 bytes apart along the rows).
//  * contract: one CTA of 512 threads (256 for 32-sample slices) per tile and run of
//    consecutive N-sample slices. One thread starts a bulk copy of the packed weights into
//    shared memory (mbarrier completion, once per CTA). Per slice, all threads hold their
//    source values in registers (the next slice's values are loaded while this one is
//    processed), reduce the per-sample max, exponentiate and write the B operand (bf16 hi
//    and lo) in the canonical no-swizzle MN-major layout. One thread then issues the MMAs
//    (M = 128 rows, N samples, K = 16 per instruction; three per step in the split form:
//    hi*hi + lo*hi + hi*lo) and commits them to an mbarrier. Every warp then reads its
//    accumulator rows and columns back from tensor memory for the epilogue. Every wait is
//    bounded; a CTA whose wait runs out writes NaN rows and reports PCB_STATUS_WAIT_TIMEOUT in
//    the device status word.
//
// These kernels serve the BF16 forms only: their logarithms use the hardware approximation
// (__logf, absolute error ~1e-6, far below the bf16 operand rounding), which halves the
// instruction count of the epilogue.
#include <cuda_bf16.h>

#include "common.cuh"

namespace {

constexpr int KT = 128;                      // terms per tile (zero padded)
constexpr uint32_t kHalfBytes = 128 * KT * 2;  // one bf16 copy of a 128 x 128 operand
constexpr uint32_t kTileBytes = 2 * kHalfBytes;  // hi + lo
constexpr uint32_t kLBO = 128;               // bytes between core matrices along K
constexpr uint32_t kSBO = (KT / 8) * 128;    // bytes between 8-row (8-column) groups
constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle (sm_100 descriptor version 1).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(kLBO >> 4) << 16) | ((uint64_t)(kSBO >> 4) << 32) |
           (1ull << 46);
}

// Instruction descriptor: D f32, A and B bf16, A K-major, B MN-major, M = 128, N.
template <int N>
__device__ __forceinline__ constexpr uint32_t make_idesc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16_ss(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(m)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* m, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* m, uint32_t parity) {
    for (int i = 0; i < kSpinLimit; ++i)
        if (mbar_try_wait(m, parity)) return true;
    return false;
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(mbar))
        : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

// hi = bf16(x), lo = bf16(x - hi), packed in pairs
__device__ __forceinline__ void split8(const float (&x)[8], uint4& h, uint4& l) {
    uint32_t hh[4], ll[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        __nv_bfloat162 hv = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
        const float2 hf = __bfloat1622float2(hv);
        __nv_bfloat162 lv = __floats2bfloat162_rn(x[2 * i] - hf.x, x[2 * i + 1] - hf.y);
        hh[i] = *reinterpret_cast<uint32_t*>(&hv);
        ll[i] = *reinterpret_cast<uint32_t*>(&lv);
    }
    h = make_uint4(hh[0], hh[1], hh[2], hh[3]);
    l = make_uint4(ll[0], ll[1], ll[2], ll[3]);
}

// ---------------------------------------------------------------------------------------
// Weight packing: 8 CTAs per tile, one 16-byte chunk (8 terms of one row) per thread;
// consecutive threads take consecutive rows, so each weight load is coalesced along the
// rows of the forward tables.
constexpr int kPackSplit = (128 * (KT / 8)) / 256;

__device__ __forceinline__ void pack_tile_part(const float* __restrict__ params, const PcbLseTile& t, int rpb_log2,
                                               const int* __restrict__ kw, int w_stride, uint8_t* __restrict__ dst,
                                               int part) {
    const int rpb_mask = (1 << rpb_log2) - 1;
    const int nk = min(t.k_cnt, KT);
    {
        const int c = part * 256 + threadIdx.x;
        const int r = c % 128;
        const int kg = c / 128;
        float w[8];
        const int64_t rb = (int64_t)t.w_add + (int64_t)(r >> rpb_log2) * t.g_stride + (int64_t)(r & rpb_mask) * w_stride;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int k = kg * 8 + j;
            w[j] = (r < t.n_rows && k < nk) ? __ldg(params + (int64_t)__ldg(kw + t.k_off + k) + rb) : 0.f;
        }
        uint4 h, l;
        split8(w, h, l);
        const uint32_t off = (uint32_t)(r >> 3) * kSBO + (uint32_t)kg * kLBO + (uint32_t)(r & 7) * 16;
        *reinterpret_cast<uint4*>(dst + off) = h;
        *reinterpret_cast<uint4*>(dst + kHalfBytes + off) = l;
    }
}

__global__ void __launch_bounds__(256)
pack_weights_kernel(const float* __restrict__ params, const PcbLseTile* __restrict__ tiles, int rpb_log2,
                    const int* __restrict__ kw, int w_stride, uint8_t* __restrict__ packed) {
    pcb::pdl_begin();
    const int tile = blockIdx.x / kPackSplit;
    pack_tile_part(params, tiles[tile], rpb_log2, kw, w_stride, packed + (size_t)tile * kTileBytes,
                   blockIdx.x % kPackSplit);
}

// All tiles of several tile tables in one launch: global tile g is tile tile_index[g] of
// job tile_job[g].
__global__ void __launch_bounds__(256)
pack_weights_multi_kernel(const float* __restrict__ params, const PcbPackJob* __restrict__ jobs,
                          const int* __restrict__ tile_job, const int* __restrict__ tile_index) {
    pcb::pdl_begin();
    const int g = blockIdx.x / kPackSplit;
    const PcbPackJob jb = jobs[tile_job[g]];
    const int ti = tile_index[g];
    pack_tile_part(params, jb.tiles[ti], jb.rows_per_block_log2, jb.kw, jb.w_stride,
                   jb.packed + (size_t)ti * kTileBytes, blockIdx.x % kPackSplit);
}

// ---------------------------------------------------------------------------------------
// Threads of the contraction kernel: 16 warps for 64-sample slices, 8 for 32 (two CTAs per
// SM by shared memory; each warp's epilogue reads 16 accumulator columns).
template <int N>
constexpr int tc05_threads() { return N == 64 ? 512 : 256; }

template <int N>
struct Tc05Smem {
    static constexpr int W = tc05_threads<N>() / 32;
    static constexpr uint32_t oW = 0;                       // packed weights (hi, lo)
    static constexpr uint32_t oE = kTileBytes;              // B operand (hi, lo): N x 128 bf16 each
    static constexpr uint32_t kEHalf = (uint32_t)N * KT * 2;
    static constexpr uint32_t oPart = oE + 2 * kEHalf;      // [W][N] partial maxima
    static constexpr uint32_t oMax = oPart + W * N * 4;     // [N]
    static constexpr uint32_t oRow = oMax + N * 4;          // [128] source rows
    static constexpr uint32_t oBar = oRow + KT * 4;         // two mbarriers
    static constexpr uint32_t oSlot = oBar + 16;            // tensor-memory address, failure flag
    static constexpr size_t bytes() { return oSlot + 16; }
};

__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

// One CTA per tile and run of up to spc consecutive N-sample slices. The packed weights are
// copied once per CTA; the source values (and epilogue element values) of slice s + 1 are
// prefetched into L2 while slice s is reduced, exponentiated, contracted and written out.
template <int N, int MODE, bool SPLIT>
__global__ void __launch_bounds__(tc05_threads<N>(), 2)
lse_tc05_kernel(const float* __restrict__ src, const float* __restrict__ src2, const float* __restrict__ aux,
                float* __restrict__ out, int64_t ld, int B, const uint8_t* __restrict__ packed,
                const PcbLseTile* __restrict__ tiles, const int* __restrict__ krow, int spc, bool vec,
                int32_t* __restrict__ status) {
    // tile and term indices (compiled tables) before the wait for the previous kernel
    pcb::pdl_trigger();
    static_assert(N == 32 || N == 64, "sample slice");
    using S = Tc05Smem<N>;
    constexpr int W = S::W;             // warps
    constexpr int NQ = N / 32;          // groups of 4 x 8 samples
    constexpr int WPQ = W / NQ;         // warps per group
    constexpr int ITER = KT / (8 * WPQ);  // 8-term groups (16-byte chunks) per thread
    constexpr int CW = N / (W / 4);     // accumulator columns per warp in the epilogue
    constexpr int NH = MODE == 2 ? 2 : 1;  // source arrays (flows and mars in mode 2)
    static_assert(ITER >= 1 && CW % 16 == 0, "thread layout");
    extern __shared__ __align__(1024) uint8_t sm[];
    float* sPart = reinterpret_cast<float*>(sm + S::oPart);
    float* sMax = reinterpret_cast<float*>(sm + S::oMax);
    int* sRow = reinterpret_cast<int*>(sm + S::oRow);
    uint64_t* barW = reinterpret_cast<uint64_t*>(sm + S::oBar);
    uint64_t* barM = barW + 1;
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + S::oSlot);

    const int tile_id = blockIdx.x;
    const PcbLseTile t = tiles[tile_id];
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const bool bad = t.k_cnt > KT;
    const int nk = bad ? 0 : t.k_cnt;
    const int s0 = blockIdx.y * spc;
    const int nsl = min(spc, (B + N - 1) / N - s0);
    if (tid < nk) sRow[tid] = __ldg(krow + t.k_off + tid);
    pcb::pdl_wait();

    if (warp == 0) {
        tmem_alloc(slot, N);
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(barW, 1);
        mbar_init(barM, 1);
        slot[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t taddr = slot[0];
    if (tid == 0) {
        const uint32_t wbytes = SPLIT ? kTileBytes : kHalfBytes;
        mbar_expect_tx(barW, wbytes);
        bulk_copy_g2s(sm + S::oW, packed + (size_t)tile_id * kTileBytes, wbytes, barW);
    }

    // thread layout of the source values: term chunk (k, 8 samples) per thread and step
    const int nq = warp % NQ;
    const int n8 = nq * 4 + (lane >> 3);      // this thread's 8-sample group
    const int kl = lane & 7;
    // epilogue: warp w owns accumulator rows 32 (w % 4) .. + 31 (its lane quarter) and
    // columns (w / 4) CW .. + CW
    const int q = warp & 3;
    const int cb = (warp >> 2) * CW;
    const int r = q * 32 + lane;

    auto load_slice = [&](int sl, float (&v)[NH][ITER][8]) {
        const int bb = (s0 + sl) * N + n8 * 8;
#pragma unroll
        for (int it = 0; it < ITER; ++it) {
            const int k = ((warp / NQ) + it * WPQ) * 8 + kl;
#pragma unroll
            for (int h = 0; h < NH; ++h) {
                if (k < nk) {
                    const float* g = (h == 0 ? src : src2) + (int64_t)sRow[k] * ld + bb;
                    if (vec && bb + 7 < B) {
                        const float4 a = __ldg(reinterpret_cast<const float4*>(g));
                        const float4 c = __ldg(reinterpret_cast<const float4*>(g + 4));
                        v[h][it][0] = a.x; v[h][it][1] = a.y; v[h][it][2] = a.z; v[h][it][3] = a.w;
                        v[h][it][4] = c.x; v[h][it][5] = c.y; v[h][it][6] = c.z; v[h][it][7] = c.w;
                    } else {
#pragma unroll
                        for (int j = 0; j < 8; ++j) v[h][it][j] = (bb + j < B) ? __ldg(g + j) : -INFINITY;
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 8; ++j) v[h][it][j] = -INFINITY;
                }
            }
        }
    };

    // the next slice's rows into L2 (one prefetch per 32-byte sector this thread will read)
    auto prefetch_slice = [&](int sl) {
        const int bb = (s0 + sl) * N + n8 * 8;
        if (bb < B) {
#pragma unroll
            for (int it = 0; it < ITER; ++it) {
                const int k = ((warp / NQ) + it * WPQ) * 8 + kl;
                if (k < nk) {
#pragma unroll
                    for (int h = 0; h < NH; ++h) prefetch_l2((h == 0 ? src : src2) + (int64_t)sRow[k] * ld + bb);
                }
            }
        }
        if (MODE != 0 && r < t.n_rows) {
            const int b = (s0 + sl) * N + cb;
#pragma unroll
            for (int c8 = 0; c8 < CW / 8; ++c8)
                if (b + c8 * 8 < B) prefetch_l2(aux + ((int64_t)t.aux_row + r) * ld + b + c8 * 8);
        }
    };

    float cur[NH][ITER][8];
    bool fail = bad;
    for (int sl = 0; sl < nsl; ++sl) {
        const int b0 = (s0 + sl) * N;
        if (sl == 0) prefetch_slice(0);
        load_slice(sl, cur);
        if (sl + 1 < nsl) prefetch_slice(sl + 1);
        // mode 2: node flows -> log f - log m
        float v[ITER][8];
#pragma unroll
        for (int it = 0; it < ITER; ++it)
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (MODE == 2) {
                    const float m2 = cur[NH - 1][it][j];
                    v[it][j] = (m2 == -INFINITY) ? -INFINITY : __logf(cur[0][it][j]) - m2;
                } else {
                    v[it][j] = cur[0][it][j];
                }
            }
        // per-sample max: over this thread's terms, the 8 lanes of the group, then the warps
        float m[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float x = v[0][j];
#pragma unroll
            for (int it = 1; it < ITER; ++it) x = fmaxf(x, v[it][j]);
            x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, 1));
            x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, 2));
            x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, 4));
            m[j] = x;
        }
        if (kl == 0) {
#pragma unroll
            for (int j = 0; j < 8; ++j) sPart[(warp / NQ) * N + n8 * 8 + j] = m[j];
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float x = sPart[n8 * 8 + j];
#pragma unroll
            for (int w = 1; w < WPQ; ++w) x = fmaxf(x, sPart[w * N + n8 * 8 + j]);
            m[j] = x;
        }
        if (warp / NQ == 0 && kl == 0) {
#pragma unroll
            for (int j = 0; j < 8; ++j) sMax[n8 * 8 + j] = m[j];
        }
        // exponentiate; B operand in the MN-major core-matrix layout (the previous slice's
        // MMAs have completed: its epilogue waited for them)
        uint8_t* eh = sm + S::oE;
        uint8_t* el = eh + S::kEHalf;
#pragma unroll
        for (int it = 0; it < ITER; ++it) {
            const int k = ((warp / NQ) + it * WPQ) * 8 + kl;
            float e[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) e[j] = (m[j] == -INFINITY) ? 0.f : __expf(v[it][j] - m[j]);
            const uint32_t off = (uint32_t)n8 * kSBO + (uint32_t)(k >> 3) * kLBO + (uint32_t)(k & 7) * 16;
            if (SPLIT) {
                uint4 h, l;
                split8(e, h, l);
                *reinterpret_cast<uint4*>(eh + off) = h;
                *reinterpret_cast<uint4*>(el + off) = l;
            } else {
                *reinterpret_cast<uint4*>(eh + off) =
                    make_uint4(pack2(e[0], e[1]), pack2(e[2], e[3]), pack2(e[4], e[5]), pack2(e[6], e[7]));
            }
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

        // ---- one thread issues the MMAs ----
        if (tid == 0) {
            if (sl == 0 && !mbar_wait_bounded(barW, 0)) slot[1] = 1;
            if (slot[1] == 0) {
                constexpr uint32_t idesc = make_idesc<N>();
                const uint32_t aw = smem_u32(sm + S::oW);
                const uint32_t ae = smem_u32(eh);
                const int ks = (nk + 15) / 16;
                for (int s = 0; s < ks; ++s) {
                    const uint32_t o = (uint32_t)s * 2 * kLBO;
                    mma_bf16_ss(taddr, make_desc(aw + o), make_desc(ae + o), idesc, s > 0 ? 1u : 0u);
                    if (SPLIT) {
                        mma_bf16_ss(taddr, make_desc(aw + kHalfBytes + o), make_desc(ae + o), idesc, 1u);
                        mma_bf16_ss(taddr, make_desc(aw + o), make_desc(ae + S::kEHalf + o), idesc, 1u);
                    }
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(barM))
                         : "memory");
        }
        const bool mok = mbar_wait_bounded(barM, (uint32_t)(sl & 1));
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        fail = fail || !mok || slot[1] != 0;

        // ---- epilogue ----
        float a[CW];  // element values of this slice (modes 1/2; in L2 by the prefetch)
        if (MODE != 0) {
            const float* ax = aux + ((int64_t)t.aux_row + (r < t.n_rows ? r : 0)) * ld + b0 + cb;
#pragma unroll
            for (int c4 = 0; c4 < CW / 4; ++c4) {
                const int b = b0 + cb + c4 * 4;
                if (vec && b + 3 < B) {
                    const float4 av = __ldg(reinterpret_cast<const float4*>(ax + c4 * 4));
                    a[c4 * 4] = av.x; a[c4 * 4 + 1] = av.y; a[c4 * 4 + 2] = av.z; a[c4 * 4 + 3] = av.w;
                } else {
#pragma unroll
                    for (int j = 0; j < 4; ++j) a[c4 * 4 + j] = (b + j < B) ? __ldg(ax + c4 * 4 + j) : 0.f;
                }
            }
        }
        float acc[CW];
#pragma unroll
        for (int c = 0; c < CW / 16; ++c) {
            float x[16];
            tmem_ld16(taddr + ((uint32_t)(q * 32) << 16) + (uint32_t)(cb + c * 16), x);
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[c * 16 + i] = x[i];
        }
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (r < t.n_rows) {
            float* dst = out + ((int64_t)t.out_row + r) * ld + b0 + cb;
#pragma unroll
            for (int c4 = 0; c4 < CW / 4; ++c4) {
                float o[4];
                const int b = b0 + cb + c4 * 4;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float mm = sMax[cb + c4 * 4 + j];
                    const float val = acc[c4 * 4 + j];
                    if (fail) o[j] = __int_as_float(0x7fc00000);
                    else if (MODE == 0) o[j] = (mm == -INFINITY) ? -INFINITY : __logf(val) + mm;
                    else o[j] = (mm == -INFINITY) ? 0.f : val * __expf(a[c4 * 4 + j] + mm);
                }
                if (vec && b + 3 < B) {
                    *reinterpret_cast<float4*>(dst + c4 * 4) = make_float4(o[0], o[1], o[2], o[3]);
                } else {
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (b + j < B) dst[c4 * 4 + j] = o[j];
                }
            }
        }
        // the next slice rewrites the partial maxima, the B operand and the accumulators
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
    }
    if (fail) pcb::report_status(status, bad ? PCB_STATUS_TILE_TOO_LONG : PCB_STATUS_WAIT_TIMEOUT);
    if (warp == 0) tmem_dealloc(taddr, N);
}

int current_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d < 0 ? 0 : (d > 63 ? 63 : d);
}

template <int N, int MODE, bool SPLIT>
int launch(int num_tiles, int spc, const float* src, const float* src2, const float* aux, float* out, int64_t ld,
           int B, const uint8_t* packed, const PcbLseTile* tiles, const int* krow, cudaStream_t s, bool vec) {
    constexpr size_t smem = Tc05Smem<N>::bytes();
    static_assert(smem <= 227 * 1024, "shared memory");
    static bool configured[64] = {false};
    const int dev = current_device();
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(lse_tc05_kernel<N, MODE, SPLIT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_lse_contract_tc05: %s", cudaGetErrorString(e));
        configured[dev] = true;
    }
    const int64_t gy = pcb::cdiv(pcb::cdiv(B, N), spc);
    if (gy > 65535) return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_tc05: batch too large");
    return pcb::launch_status(pcb::launch_k(lse_tc05_kernel<N, MODE, SPLIT>,
                                            dim3((unsigned)num_tiles, (unsigned)gy), dim3(tc05_threads<N>()), smem, s,
                                            1u, src, src2, aux, out, ld, B, packed, tiles, krow, spc, vec,
                                            pcb::status_word()),
                              "pcb_lse_contract_tc05");
}

template <int N>
int launch_n(int mode, bool split, int num_tiles, int spc, const float* src, const float* src2, const float* aux,
             float* out, int64_t ld, int B, const uint8_t* packed, const PcbLseTile* tiles, const int* krow,
             cudaStream_t s, bool vec) {
#define PCB_TC(M, SP) launch<N, M, SP>(num_tiles, spc, src, src2, aux, out, ld, B, packed, tiles, krow, s, vec)
    if (split) return mode == 0 ? PCB_TC(0, true) : (mode == 1 ? PCB_TC(1, true) : PCB_TC(2, true));
    return mode == 0 ? PCB_TC(0, false) : (mode == 1 ? PCB_TC(1, false) : PCB_TC(2, false));
#undef PCB_TC
}

}  // namespace

extern "C" int pcb_pack_weights(const float* params, const PcbLseTile* tiles, int32_t num_tiles,
                                int32_t rows_per_block, const int32_t* kw, int32_t w_stride, uint8_t* packed,
                                void* stream) {
    if (!params || !tiles || !kw || !packed || num_tiles < 0 || rows_per_block <= 0 ||
        (rows_per_block & (rows_per_block - 1)) || (reinterpret_cast<uintptr_t>(packed) & 15) != 0)
        return pcb::set_error(PCB_E_ARG, "pcb_pack_weights: bad arguments");
    if (num_tiles == 0) return PCB_OK;
    int rpb_log2 = 0;
    while ((1 << rpb_log2) < rows_per_block) ++rpb_log2;
    if ((int64_t)num_tiles * kPackSplit > 2147483647) return pcb::set_error(PCB_E_ARG, "pcb_pack_weights: too many tiles");
    return pcb::launch_status(pcb::launch_k(pack_weights_kernel, dim3((unsigned)(num_tiles * kPackSplit)), dim3(256),
                                            0, pcb::as_stream(stream), 1u, params, tiles, rpb_log2, kw, w_stride,
                                            packed), "pcb_pack_weights");
}

extern "C" int pcb_pack_weights_multi(const float* params, const PcbPackJob* jobs, const int32_t* tile_job,
                                      const int32_t* tile_index, int32_t total_tiles, void* stream) {
    if (!params || !jobs || !tile_job || !tile_index || total_tiles < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_pack_weights_multi: bad arguments");
    if (total_tiles == 0) return PCB_OK;
    if ((int64_t)total_tiles * kPackSplit > 2147483647)
        return pcb::set_error(PCB_E_ARG, "pcb_pack_weights_multi: too many tiles");
    return pcb::launch_status(pcb::launch_k(pack_weights_multi_kernel, dim3((unsigned)(total_tiles * kPackSplit)),
                                            dim3(256), 0, pcb::as_stream(stream), 1u, params, jobs, tile_job,
                                            tile_index), "pcb_pack_weights_multi");
}

extern "C" int pcb_lse_contract_tc05(const float* src, const float* src2, const float* aux, float* out, int64_t ld,
                                     int32_t B, const uint8_t* packed, const PcbLseTile* tiles, int32_t num_tiles,
                                     const int32_t* krow, int32_t mode, int32_t prec, int32_t batch_tile,
                                     int32_t slices_per_cta, void* stream) {
    if (!src || !out || !packed || !tiles || !krow || B <= 0 || ld < B || num_tiles < 0 || mode < 0 || mode > 2 ||
        (mode == 2 && !src2) || (mode >= 1 && !aux) || prec < 1 || prec > 2 ||
        (batch_tile != 32 && batch_tile != 64) || slices_per_cta < 1 || (reinterpret_cast<uintptr_t>(packed) & 15) != 0)
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_tc05: bad arguments");
    if (num_tiles == 0) return PCB_OK;
    const bool vec = pcb::vec_ok(src, ld) && pcb::vec_ok(out, ld) && (!src2 || pcb::vec_ok(src2, ld)) &&
                     (!aux || pcb::vec_ok(aux, ld));
    cudaStream_t s = pcb::as_stream(stream);
    const bool split = prec == 2;
    const int spc = slices_per_cta;
    if (batch_tile == 32)
        return launch_n<32>(mode, split, num_tiles, spc, src, src2, aux, out, ld, B, packed, tiles, krow, s, vec);
    return launch_n<64>(mode, split, num_tiles, spc, src, src2, aux, out, ld, B, packed, tiles, krow, s, vec);
}
