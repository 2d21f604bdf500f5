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
// These kernels serve the BF16 forms only: their logarithms and exponentials are the
// hardware base-2 approximations (pcb::fast_log / fast_exp, relative error ~1e-7, far below
// the bf16 operand rounding), a few instructions each.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>

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

// E4M3 form: a tile's weights as e4m3 bytes in the K-major no-swizzle layout (8 rows x 16
// terms per core matrix, 128 bytes along K between core matrices, 1024 bytes between 8-row
// groups), each row scaled by 448 / (its largest weight), followed by 128 FP32 unscale
// factors (largest weight / 448^2, applied to the accumulator with the B operand's 448).
constexpr uint32_t kF8Bytes = 128 * KT;
constexpr uint32_t kF8SBO = (KT / 16) * 128;
constexpr uint32_t kF8TileBytes = kF8Bytes + 128 * 4;

__device__ __forceinline__ uint64_t make_desc_sbo(uint32_t saddr, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(kLBO >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}

// Instruction descriptor of kind::f8f6f4: D f32, A and B e4m3, both K-major, M = 128, N.
template <int N>
__device__ __forceinline__ constexpr uint32_t make_idesc_f8() {
    return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_f8_ss(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Two floats as e4m3 (round to nearest, saturating): a in the low byte, b in the high byte.
__device__ __forceinline__ uint32_t e4m3x2(float a, float b) {
    uint16_t r;
    asm("cvt.rn.satfinite.e4m3x2.f32 %0, %1, %2;" : "=h"(r) : "f"(b), "f"(a));
    return r;
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

// E4M3 packing of one tile by a CTA of 256 threads: thread (r, h) takes row r and terms
// 64 h .. 64 h + 63; the row's largest weight (over both halves) sets its scale.
__device__ __forceinline__ void pack_tile_fp8(const float* __restrict__ params, const PcbLseTile& t, int rpb_log2,
                                              const int* __restrict__ kw, int w_stride, uint8_t* __restrict__ dst,
                                              float (*smax)[128]) {
    const int rpb_mask = (1 << rpb_log2) - 1;
    const int nk = min(t.k_cnt, KT);
    const int r = threadIdx.x & 127, h = threadIdx.x >> 7;
    const bool row_ok = r < t.n_rows;
    const int64_t rb = (int64_t)t.w_add + (int64_t)(r >> rpb_log2) * t.g_stride + (int64_t)(r & rpb_mask) * w_stride;
    float mx = 0.f;
    for (int j = 0; j < 64; ++j) {
        const int k = h * 64 + j;
        if (row_ok && k < nk) mx = fmaxf(mx, __ldg(params + (int64_t)__ldg(kw + t.k_off + k) + rb));
    }
    smax[h][r] = mx;
    __syncthreads();
    mx = fmaxf(smax[0][r], smax[1][r]);
    const float sc = mx > 0.f ? 448.f / mx : 0.f;
#pragma unroll 1
    for (int g = 0; g < 4; ++g) {
        uint32_t wd[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float w[4];
#pragma unroll
            for (int z = 0; z < 4; ++z) {
                const int k = h * 64 + g * 16 + q * 4 + z;
                w[z] = (row_ok && k < nk) ? __ldg(params + (int64_t)__ldg(kw + t.k_off + k) + rb) * sc : 0.f;
            }
            wd[q] = e4m3x2(w[0], w[1]) | (e4m3x2(w[2], w[3]) << 16);
        }
        *reinterpret_cast<uint4*>(dst + (uint32_t)(r >> 3) * kF8SBO + (uint32_t)(h * 4 + g) * kLBO +
                                  (uint32_t)(r & 7) * 16) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
    }
    if (h == 0) reinterpret_cast<float*>(dst + kF8Bytes)[r] = mx / (448.f * 448.f);
}

__global__ void __launch_bounds__(256)
pack_weights_fp8_kernel(const float* __restrict__ params, const PcbLseTile* __restrict__ tiles, int rpb_log2,
                        const int* __restrict__ kw, int w_stride, uint8_t* __restrict__ packed) {
    pcb::pdl_begin();
    __shared__ float smax[2][128];
    pack_tile_fp8(params, tiles[blockIdx.x], rpb_log2, kw, w_stride, packed + (size_t)blockIdx.x * kTileBytes, smax);
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
    __shared__ float smax[2][128];
    const int g = blockIdx.x / kPackSplit;
    const PcbPackJob jb = jobs[tile_job[g]];
    const int ti = tile_index[g];
    if (jb.format == 1) {  // e4m3: the whole tile in the first of its CTAs (row maxima)
        if (blockIdx.x % kPackSplit == 0)
            pack_tile_fp8(params, jb.tiles[ti], jb.rows_per_block_log2, jb.kw, jb.w_stride,
                          jb.packed + (size_t)ti * kTileBytes, smax);
        return;
    }
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

// log(e^a + e^b) (-inf + -inf = -inf), with the hardware base-2 approximations.
__device__ __forceinline__ float log_add(float a, float b) {
    const float hi = fmaxf(a, b), lo = fminf(a, b);
    return hi == -INFINITY ? -INFINITY : hi + pcb::fast_log(1.f + pcb::fast_exp(lo - hi));
}

// One CTA per tile and run of up to spc consecutive N-sample slices. The packed weights are
// copied once per CTA; the source values (and epilogue element values) of slice s + 1 are
// prefetched into L2 while slice s is reduced, exponentiated, contracted and written out.
template <int N, int MODE, int PREC>
__global__ void __launch_bounds__(tc05_threads<N>(), 2)
lse_tc05_kernel(const float* __restrict__ src, const float* __restrict__ src2, const float* __restrict__ aux,
                float* __restrict__ out, int64_t ld, int B, const uint8_t* __restrict__ packed,
                const PcbLseTile* __restrict__ tiles, const int* __restrict__ krow, int spc, bool vec,
                bool accum, int32_t* __restrict__ status) {
    // tile and term indices (compiled tables) before the wait for the previous kernel
    pcb::pdl_trigger();
    static_assert(N == 32 || N == 64, "sample slice");
    constexpr bool SPLIT = PREC == 2;
    constexpr bool FP8 = PREC == 3;
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
        const uint32_t wbytes = FP8 ? kF8TileBytes : (SPLIT ? kTileBytes : kHalfBytes);
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
                    v[it][j] = (m2 == -INFINITY) ? -INFINITY : pcb::fast_log(cur[0][it][j]) - m2;
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
            for (int j = 0; j < 8; ++j) e[j] = (m[j] == -INFINITY) ? 0.f : pcb::fast_exp(v[it][j] - m[j]);
            const uint32_t off = (uint32_t)n8 * kSBO + (uint32_t)(k >> 3) * kLBO + (uint32_t)(k & 7) * 16;
            if (FP8) {
                // K-major e4m3 B operand: sample n's 16 terms k & ~15 .. per 16-byte row;
                // values scaled by 448 (the largest finite e4m3) before rounding
                uint8_t* row = eh + (uint32_t)n8 * kF8SBO + (uint32_t)(k >> 4) * kLBO + (uint32_t)(k & 15);
#pragma unroll
                for (int j = 0; j < 8; j += 2) {
                    const uint32_t two = e4m3x2(e[j] * 448.f, e[j + 1] * 448.f);
                    row[j * 16] = (uint8_t)(two & 0xFF);
                    row[(j + 1) * 16] = (uint8_t)(two >> 8);
                }
            } else if (SPLIT) {
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
            if (slot[1] == 0 && FP8) {
                constexpr uint32_t idesc = make_idesc_f8<N>();
                const uint32_t aw = smem_u32(sm + S::oW);
                const uint32_t ae = smem_u32(eh);
                for (int s = 0; s < (nk + 31) / 32; ++s) {
                    const uint32_t o = (uint32_t)s * 2 * kLBO;
                    mma_f8_ss(taddr, make_desc_sbo(aw + o, kF8SBO), make_desc_sbo(ae + o, kF8SBO), idesc,
                              s > 0 ? 1u : 0u);
                }
            } else if (slot[1] == 0) {
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
        if (FP8) {  // undo the row's weight scale and the 448 of the B operand
            const float us = reinterpret_cast<const float*>(sm + S::oW + kF8Bytes)[r];
#pragma unroll
            for (int i = 0; i < CW; ++i) acc[i] *= us;
        }
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
                    else if (MODE == 0) o[j] = (mm == -INFINITY) ? -INFINITY : pcb::fast_log(val) + mm;
                    else o[j] = (mm == -INFINITY) ? 0.f : val * pcb::fast_exp(a[c4 * 4 + j] + mm);
                }
                if (accum && !fail) {  // a later chunk of the tile's terms: combine with the output
                    float old[4];
                    if (vec && b + 3 < B) {
                        const float4 ov = *reinterpret_cast<const float4*>(dst + c4 * 4);
                        old[0] = ov.x; old[1] = ov.y; old[2] = ov.z; old[3] = ov.w;
                    } else {
#pragma unroll
                        for (int j = 0; j < 4; ++j) old[j] = (b + j < B) ? dst[c4 * 4 + j] : 0.f;
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j) o[j] = MODE == 0 ? log_add(old[j], o[j]) : old[j] + o[j];
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

// ---------------------------------------------------------------------------------------
// Warp-specialised persistent form. A CTA owns a contiguous run of work units (tile,
// N-sample slice), tile-major, so consecutive units share the tile's packed weights (copied
// again only when the tile changes). Roles:
//   warp 0      producer: one bulk copy (cp.async.bulk, mbarrier completion) per source row
//               and unit into a ring of NS stages; the packed weights once per tile;
//   warp 1      one thread issues the MMAs of a unit into one of two tensor-memory
//               accumulators and commits them to the accumulator-full, B-free and (last
//               unit of a tile) weights-free barriers;
//   warps 2-9   converters: load a stage into registers and free it, per-sample max over the
//               tile's terms (warp shuffles, then partial maxima of the 8 warps through
//               shared memory), exponentiate, write the B operand (double buffered);
//   warps 10-13 epilogue: one accumulator row per thread (warp w reads tensor-memory lanes
//               32 (w % 4) .. + 31), log + max (mode 0) or value * exp(element + max)
//               (modes 1/2), stored straight to global memory.
// Every wait is bounded; on a timeout the CTA records a failure, writes NaN rows, keeps
// its barrier arrivals going so that every role ends, waits (bounded) for its own copies in
// flight and releases its tensor memory.
constexpr int kWsThreads = 448;
constexpr int kWsConverters = 8;  // warps

template <int N, int MODE, bool SPLIT>
struct WsSmem {
    static constexpr int NH = MODE == 2 ? 2 : 1;                       // source arrays
    static constexpr uint32_t kStage = (uint32_t)NH * KT * N * 4;       // FP32 rows of one unit
    static constexpr uint32_t kW = SPLIT ? kTileBytes : kHalfBytes;     // packed weights
    static constexpr uint32_t kBHalf = (uint32_t)N * KT * 2;            // one bf16 copy of B
    static constexpr uint32_t kB = SPLIT ? 2 * kBHalf : kBHalf;
    static constexpr uint32_t oW = 0;
    static constexpr uint32_t oB = oW + kW;                             // [2] B operands
    static constexpr uint32_t oEpi = oB + 2 * kB;                       // [4 warps] 32 x 32 output boxes
    static constexpr uint32_t oMax = oEpi + 4 * 4096;                   // [4][N] per-sample maxima
    static constexpr uint32_t oPart = oMax + 4 * N * 4;                 // [2][8][N] partial maxima
    static constexpr uint32_t oBar = oPart + 2 * kWsConverters * N * 4; // mbarriers, TMEM address
    static constexpr uint32_t oStage = (oBar + 256 + 1023) / 1024 * 1024;  // [NS] stages (1 KB aligned)
    static constexpr uint32_t kBudget = 227u * 1024u;
    static constexpr int kFit = (int)((kBudget - oStage) / kStage);
    static constexpr int NS = kFit > 6 ? 6 : kFit;
    static constexpr size_t bytes() { return oStage + (size_t)NS * kStage; }
};

// 2-D tiled TMA store of one box from shared memory (bulk async-group completion).
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, const void* src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];\n"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(src))
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}

// 2-D tiled TMA load of one box (32 samples x box rows, 128-byte swizzle) into shared memory.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* mbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(mbar))
        : "memory");
}

// Epilogue of 4 samples: log(acc) + max (mode 0) or acc * exp(element + max) (modes 1/2);
// -inf maxima give -inf / 0, a failed CTA NaN.
template <int MODE>
__device__ __forceinline__ float4 finish4(float4 x, float4 m, float4 e, bool fail) {
    float o[4] = {x.x, x.y, x.z, x.w};
    const float mm[4] = {m.x, m.y, m.z, m.w};
    const float ee[4] = {e.x, e.y, e.z, e.w};
#pragma unroll
    for (int z = 0; z < 4; ++z) {
        if (fail) o[z] = __int_as_float(0x7fc00000);
        else if (MODE == 0) o[z] = (mm[z] == -INFINITY) ? -INFINITY : pcb::fast_log(o[z]) + mm[z];
        else o[z] = (mm[z] == -INFINITY) ? 0.f : o[z] * pcb::fast_exp(ee[z] + mm[z]);
    }
    return make_float4(o[0], o[1], o[2], o[3]);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* m) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(m)) : "memory");
}

__device__ __forceinline__ void commit_to(uint64_t* m) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(m))
                 : "memory");
}

// 8 samples (8-sample group g4 of a 32-sample row) of one 128-byte line written by a TMA box
// with 128-byte swizzle: 16-byte chunk c of the line sits at chunk c ^ (line % 8), and
// line % 8 == kl here, so the 8 lanes of a phase (kl = 0..7) hit distinct banks.
__device__ __forceinline__ void load8_sw(const uint8_t* line, int g4, int kl, float (&v)[8]) {
    const float4 a = *reinterpret_cast<const float4*>(line + (((2 * g4) ^ kl) << 4));
    const float4 c = *reinterpret_cast<const float4*>(line + (((2 * g4 + 1) ^ kl) << 4));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = c.x; v[5] = c.y; v[6] = c.z; v[7] = c.w;
}

// 8 consecutive floats of shared memory as two 16-byte loads, the half hs first (threads
// of one 8-lane phase alternate halves, so that their loads fall into distinct banks)
__device__ __forceinline__ void load8(const float* p, int hs, float (&v)[8]) {
    const float4 a = *reinterpret_cast<const float4*>(p + hs * 4);
    const float4 c = *reinterpret_cast<const float4*>(p + (hs ^ 1) * 4);
    const float4 lo = hs ? c : a, hi = hs ? a : c;
    v[0] = lo.x; v[1] = lo.y; v[2] = lo.z; v[3] = lo.w;
    v[4] = hi.x; v[5] = hi.y; v[6] = hi.z; v[7] = hi.w;
}

__device__ __forceinline__ void converters_sync() {
    asm volatile("bar.sync 1, %0;\n" ::"n"(kWsConverters * 32) : "memory");
}

template <int N, int MODE, bool SPLIT>
__global__ void __launch_bounds__(kWsThreads, 1)
lse_tc05_ws_kernel(const __grid_constant__ CUtensorMap map_src, const __grid_constant__ CUtensorMap map_src2,
                   const __grid_constant__ CUtensorMap map_out, const float* __restrict__ aux, float* __restrict__ out, int64_t ld, int B, int run_log2,
                   const uint8_t* __restrict__ packed, const PcbLseTile* __restrict__ tiles, int num_tiles,
                   const int* __restrict__ krow, int32_t* __restrict__ status) {
    pcb::pdl_trigger();
    static_assert(N == 32 || N == 64, "sample slice");
    using S = WsSmem<N, MODE, SPLIT>;
    constexpr int NS = S::NS;
    constexpr int NH = S::NH;
    static_assert(NS >= 1, "shared memory");
    extern __shared__ __align__(1024) uint8_t sm[];
    uint64_t* fullS = reinterpret_cast<uint64_t*>(sm + S::oBar);  // [NS] stage loaded
    uint64_t* emptyS = fullS + NS;                                 // [NS] stage free
    uint64_t* wfull = fullS + 2 * NS;                              // weights loaded
    uint64_t* wempty = wfull + 1;                                  // weights free
    uint64_t* bfull = wfull + 2;                                   // [2] B operand written
    uint64_t* bempty = wfull + 4;                                  // [2] B operand consumed
    uint64_t* afull = wfull + 6;                                   // [2] accumulator ready
    uint64_t* aempty = wfull + 8;                                  // [2] accumulator drained
    uint64_t* mfull = wfull + 10;                                  // [4] maxima written
    uint64_t* mempty = wfull + 14;                                 // [4] maxima read
    volatile uint32_t* slot = reinterpret_cast<volatile uint32_t*>(wfull + 18);  // TMEM address, failure
    float* sMax = reinterpret_cast<float*>(sm + S::oMax);
    float* sPart = reinterpret_cast<float*>(sm + S::oPart);
    static_assert((2 * NS + 18) * 8 + 8 <= 256, "barrier area");

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nsl = (B + N - 1) / N;
    const int64_t units = (int64_t)num_tiles * nsl;
    const int64_t u0 = units * blockIdx.x / gridDim.x, u1 = units * (blockIdx.x + 1) / gridDim.x;

    if (warp == 1) {
        tmem_alloc(const_cast<uint32_t*>(slot), 2 * N);
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(fullS + s, 1);
            mbar_init(emptyS + s, kWsConverters);
        }
        mbar_init(wfull, 1);
        mbar_init(wempty, 1);
        for (int j = 0; j < 2; ++j) {
            mbar_init(bfull + j, kWsConverters);
            mbar_init(bempty + j, 1);
            mbar_init(afull + j, 1);
            mbar_init(aempty + j, 4);
        }
        for (int j = 0; j < 4; ++j) {
            mbar_init(mfull + j, N / 8);
            mbar_init(mempty + j, 4);
        }
        slot[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t taddr = slot[0];
    pcb::pdl_wait();

    if (warp == 0) {
        // ---- producer ----
        // A tile's terms come in runs of run_rows consecutive source rows (8 or 32, checked by
        // the caller), so one box of run_rows rows x 32 samples per run, source array and
        // 32-sample half covers the unit: at most 128 / 8 x 2 x 2 = 64 TMA loads.
        constexpr int NHALF = N / 32;
        const int run_rows = 1 << run_log2;
        int cur = -1, nk = 0;
        int run_row = 0;  // lane m < runs: first source row of run m
        int tcount = 0;
        for (int64_t u = u0; u < u1; ++u) {
            const int tile = (int)(u / nsl), sl = (int)(u % nsl);
            const int64_t i = u - u0;
            const bool new_tile = tile != cur;
            if (new_tile) {
                const PcbLseTile t = tiles[tile];
                nk = t.k_cnt > KT ? 0 : t.k_cnt;
                run_row = (lane * run_rows < nk) ? __ldg(krow + t.k_off + lane * run_rows) : 0;
                cur = tile;
            }
            const int st = (int)(i % NS);
            const uint32_t ph = (uint32_t)((i / NS) & 1);
            const int b0 = sl * N;
            const int runs = (nk + run_rows - 1) / run_rows;
            const uint32_t box_bytes = (uint32_t)run_rows * 128u;
            uint8_t* stg = sm + S::oStage + (uint32_t)st * S::kStage;
            // a swizzled box needs a 1 KB aligned destination: otherwise load nothing, fail
            const bool aligned = (smem_u32(stg) & 1023u) == 0;
            if (lane == 0) {
                if (!mbar_wait_bounded(emptyS + st, ph ^ 1u)) slot[1] = 1;
                if (!aligned) slot[1] = 1;
                mbar_expect_tx(fullS + st, aligned ? (uint32_t)(NH * runs * NHALF) * box_bytes : 0u);
            }
            __syncwarp();
            if (aligned && lane < runs) {
#pragma unroll
                for (int h = 0; h < NH; ++h)
#pragma unroll
                    for (int hf = 0; hf < NHALF; ++hf)
                        tma_load_2d(stg + ((uint32_t)((h * KT + lane * run_rows) * NHALF + hf * run_rows)) * 128u,
                                    h == 0 ? &map_src : &map_src2, b0 + hf * 32, run_row, fullS + st);
            }
            // the tile's weights once the previous tile's MMAs are done (after this unit's
            // source loads, so that the converters are not held up meanwhile)
            if (new_tile) {
                if (lane == 0) {
                    if (tcount > 0 && !mbar_wait_bounded(wempty, (uint32_t)((tcount - 1) & 1))) slot[1] = 1;
                    mbar_expect_tx(wfull, S::kW);
                    bulk_copy_g2s(sm + S::oW, packed + (size_t)tile * kTileBytes, S::kW, wfull);
                }
                ++tcount;
            }
        }
        // copies still in flight into this CTA's stages (none unless a consumer gave up)
        if (lane == 0) {
            const int64_t n = u1 - u0;
            for (int64_t i = (n > NS ? n - NS : 0); i < n; ++i)
                if (!mbar_wait_bounded(fullS + (int)(i % NS), (uint32_t)((i / NS) & 1))) slot[1] = 1;
        }
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            int cur = -1, nk = 0, tcount = 0;
            constexpr uint32_t idesc = make_idesc<N>();
            const uint32_t aw = smem_u32(sm + S::oW);
            for (int64_t u = u0; u < u1; ++u) {
                const int tile = (int)(u / nsl);
                const int64_t i = u - u0;
                const int j = (int)(i & 1);
                if (tile != cur) {
                    if (!mbar_wait_bounded(wfull, (uint32_t)(tcount & 1))) slot[1] = 1;
                    const int kc = tiles[tile].k_cnt;
                    nk = kc > KT ? 0 : kc;
                    cur = tile;
                    ++tcount;
                }
                if (!mbar_wait_bounded(bfull + j, (uint32_t)((i >> 1) & 1))) slot[1] = 1;
                if (!mbar_wait_bounded(aempty + j, (uint32_t)(((i >> 1) & 1) ^ 1))) slot[1] = 1;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                if (slot[1] == 0) {
                    const uint32_t ab = smem_u32(sm + S::oB + (uint32_t)j * S::kB);
                    const uint32_t d = taddr + (uint32_t)(j * N);
                    const int ks = (nk + 15) / 16;
                    for (int s = 0; s < ks; ++s) {
                        const uint32_t o = (uint32_t)s * 2 * kLBO;
                        mma_bf16_ss(d, make_desc(aw + o), make_desc(ab + o), idesc, s > 0 ? 1u : 0u);
                        if (SPLIT) {
                            mma_bf16_ss(d, make_desc(aw + kHalfBytes + o), make_desc(ab + o), idesc, 1u);
                            mma_bf16_ss(d, make_desc(aw + o), make_desc(ab + S::kBHalf + o), idesc, 1u);
                        }
                    }
                }
                commit_to(afull + j);
                commit_to(bempty + j);
                if (u + 1 == u1 || (int)((u + 1) / nsl) != tile) commit_to(wempty);
            }
            // the last MMAs have completed before the tensor memory is released
            const int64_t n = u1 - u0;
            for (int64_t i = (n > 2 ? n - 2 : 0); i < n; ++i)
                if (!mbar_wait_bounded(afull + (int)(i & 1), (uint32_t)((i >> 1) & 1))) slot[1] = 1;
        }
        __syncwarp();
    } else if (warp < 2 + kWsConverters) {
        // ---- converters ----
        // Chunk = 8 samples of one term. Lanes take consecutive terms of one 8-term block
        // (k = 8 kb + kl, kl = lane % 8): the 16-byte B-operand stores of an 8-lane phase
        // are contiguous, and the 128-byte swizzle of the stage boxes puts the phase's stage
        // loads into distinct banks. A thread keeps one 8-sample group g over its R rounds.
        const int cw = warp - 2;
        constexpr int G8 = N / 8;                 // 8-sample groups
        constexpr int NPG = 32 / G8;              // term-block groups per round (partial maxima)
        constexpr int R = G8 / 2;                 // rounds: 128 terms x G8 groups / 256 threads
        const int c0 = cw * 32 + lane;
        const int kl = lane & 7;
        const int g = (c0 >> 3) % G8, pg = (c0 >> 3) / G8;
        constexpr int NHALF = N / 32;
        int cur = -1, nk = 0;
        for (int64_t u = u0; u < u1; ++u) {
            const int tile = (int)(u / nsl);
            const int64_t i = u - u0;
            const int j = (int)(i & 1);
            if (tile != cur) {
                const int kc = tiles[tile].k_cnt;
                nk = kc > KT ? 0 : kc;
                cur = tile;
            }
            const int st = (int)(i % NS);
            if (!mbar_wait_bounded(fullS + st, (uint32_t)((i / NS) & 1))) slot[1] = 1;
            const uint8_t* stg = sm + S::oStage + (uint32_t)st * S::kStage;
            float v[R][8];
#pragma unroll
            for (int it = 0; it < R; ++it) {
                const int k = (it * NPG + pg) * 8 + kl;
                // 128-byte line of term k in its box (run k >> run_log2, 32-sample half g / 4)
                const int line = (((k >> run_log2) * NHALF + (g >> 2)) << run_log2) + (k & ((1 << run_log2) - 1));
                if (k < nk) {
                    load8_sw(stg + (uint32_t)line * 128u, g & 3, kl, v[it]);
                    if (MODE == 2) {
                        float y[8];
                        load8_sw(stg + (uint32_t)(line + KT * NHALF) * 128u, g & 3, kl, y);
#pragma unroll
                        for (int q = 0; q < 8; ++q)
                            v[it][q] = (y[q] == -INFINITY) ? -INFINITY : pcb::fast_log(v[it][q]) - y[q];
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < 8; ++q) v[it][q] = -INFINITY;
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(emptyS + st);  // one arrival per warp: the stage is read
            // per-sample max: this thread's rounds, the 8 term lanes, the NPG block groups
            float m[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                float x = v[0][q];
#pragma unroll
                for (int it = 1; it < R; ++it) x = fmaxf(x, v[it][q]);
                x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, 1));
                x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, 2));
                x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, 4));
                m[q] = x;
            }
            float* part = sPart + j * NPG * N;
            if (kl == 0) {
                *reinterpret_cast<float4*>(part + pg * N + g * 8) = make_float4(m[0], m[1], m[2], m[3]);
                *reinterpret_cast<float4*>(part + pg * N + g * 8 + 4) = make_float4(m[4], m[5], m[6], m[7]);
            }
            converters_sync();
#pragma unroll
            for (int w = 0; w < NPG; ++w) {
                float y[8];
                load8(part + w * N + g * 8, 0, y);
#pragma unroll
                for (int q = 0; q < 8; ++q) m[q] = w == 0 ? y[q] : fmaxf(m[q], y[q]);
            }
            if (pg == 0 && kl == 0) {  // one thread per 8-sample group publishes the maxima
                const int mb = (int)(i & 3);
                if (!mbar_wait_bounded(mempty + mb, (uint32_t)(((i >> 2) & 1) ^ 1))) slot[1] = 1;
                *reinterpret_cast<float4*>(sMax + mb * N + g * 8) = make_float4(m[0], m[1], m[2], m[3]);
                *reinterpret_cast<float4*>(sMax + mb * N + g * 8 + 4) = make_float4(m[4], m[5], m[6], m[7]);
                mbar_arrive(mfull + mb);
            }
            // exponentiate into the B operand once the MMAs of unit i - 2 have read it
            if (!mbar_wait_bounded(bempty + j, (uint32_t)(((i >> 1) & 1) ^ 1))) slot[1] = 1;
            uint8_t* eh = sm + S::oB + (uint32_t)j * S::kB;
#pragma unroll
            for (int it = 0; it < R; ++it) {
                const int kb = it * NPG + pg;
                float e[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) e[q] = (m[q] == -INFINITY) ? 0.f : pcb::fast_exp(v[it][q] - m[q]);
                const uint32_t off = (uint32_t)g * kSBO + (uint32_t)kb * kLBO + (uint32_t)kl * 16;
                if (SPLIT) {
                    uint4 h, l;
                    split8(e, h, l);
                    *reinterpret_cast<uint4*>(eh + off) = h;
                    *reinterpret_cast<uint4*>(eh + S::kBHalf + off) = l;
                } else {
                    *reinterpret_cast<uint4*>(eh + off) =
                        make_uint4(pack2(e[0], e[1]), pack2(e[2], e[3]), pack2(e[4], e[5]), pack2(e[6], e[7]));
                }
            }
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(bfull + j);
        }
    } else {
        // ---- epilogue ----
        // Per 32-sample chunk: the warp's 32 accumulator rows (tensor-memory lanes
        // 32 (warp % 4) ..) go, row per lane, into the warp's 4 KB output box in shared memory
        // (128-byte swizzle: 16-byte chunk c of row r at c ^ (r % 8), conflict-free both
        // ways). Each lane then finishes 4 samples of 8 rows in place (log + max, or
        // value * exp(element + max) with the element values loaded row-contiguously), and
        // one lane stores the box with a TMA store. Row blocks that end inside the tile are
        // stored with plain stores instead (a box would write rows of the next tile).
        const int q = warp & 3;
        uint8_t* box = sm + S::oEpi + (uint32_t)q * 4096u;
        int cur = -1;
        PcbLseTile t = {};
        bool bad = false;
        for (int64_t u = u0; u < u1; ++u) {
            const int tile = (int)(u / nsl), sl = (int)(u % nsl);
            const int64_t i = u - u0;
            const int a = (int)(i & 1);
            const int b0 = sl * N;
            if (tile != cur) {
                t = tiles[tile];
                cur = tile;
                bad = bad || t.k_cnt > KT;
            }
            const bool full_box = q * 32 + 32 <= t.n_rows;
            if (MODE != 0) {  // this unit's element values into L2 while the MMAs run
#pragma unroll
                for (int it = 0; it < 8; ++it) {
                    const int r = q * 32 + it * 4 + (lane >> 3);
                    const int b = b0 + (lane & 7) * 8;
                    if (r < t.n_rows && b < B) prefetch_l2(aux + ((int64_t)t.aux_row + r) * ld + b);
                }
            }
            const int mb = (int)(i & 3);
            if (!mbar_wait_bounded(mfull + mb, (uint32_t)((i >> 2) & 1))) slot[1] = 1;
            if (!mbar_wait_bounded(afull + a, (uint32_t)((i >> 1) & 1))) slot[1] = 1;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const bool fail = slot[1] != 0 || t.k_cnt > KT;
#pragma unroll 1
            for (int cc = 0; cc < N / 32; ++cc) {  // rolled: a compact loop stays in the instruction cache
                const int c4 = lane & 7;
                const int b = b0 + cc * 32 + c4 * 4;  // B % 4 == 0: a 4-sample group is all in or all out
                float4 e[8];                           // element values (modes 1/2), loaded first
                if (MODE != 0) {
#pragma unroll
                    for (int it = 0; it < 8; ++it) {
                        const int r = q * 32 + it * 4 + (lane >> 3);
                        e[it] = (r < t.n_rows && b < B)
                                    ? __ldg(reinterpret_cast<const float4*>(aux + ((int64_t)t.aux_row + r) * ld + b))
                                    : make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                }
                float acc[32];
                {
                    float x0[16], x1[16];
                    const uint32_t ta = taddr + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * N + cc * 32);
                    tmem_ld16(ta, x0);
                    tmem_ld16(ta + 16, x1);
                    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
                    for (int z = 0; z < 16; ++z) {
                        acc[z] = x0[z];
                        acc[16 + z] = x1[z];
                    }
                }
                if (cc == N / 32 - 1) {  // the accumulator is free for the MMAs of unit i + 2
                    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
                    __syncwarp();
                    if (lane == 0) mbar_arrive(aempty + a);
                }
                // the previous box store has read the staging block
                if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
                __syncwarp();
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    *reinterpret_cast<float4*>(box + lane * 128 + ((c ^ (lane & 7)) << 4)) =
                        make_float4(acc[c * 4], acc[c * 4 + 1], acc[c * 4 + 2], acc[c * 4 + 3]);
                __syncwarp();
                const float4 mm = *reinterpret_cast<const float4*>(sMax + mb * N + cc * 32 + c4 * 4);
                float4 x[8];
#pragma unroll
                for (int it = 0; it < 8; ++it) {
                    const int rr = it * 4 + (lane >> 3);  // row within the warp's 32
                    x[it] = *reinterpret_cast<const float4*>(box + rr * 128 + ((c4 ^ (rr & 7)) << 4));
                }
#pragma unroll
                for (int it = 0; it < 8; ++it) x[it] = finish4<MODE>(x[it], mm, e[it], fail);
#pragma unroll
                for (int it = 0; it < 8; ++it) {
                    const int rr = it * 4 + (lane >> 3);
                    if (full_box) {
                        *reinterpret_cast<float4*>(box + rr * 128 + ((c4 ^ (rr & 7)) << 4)) = x[it];
                    } else {
                        const int r = q * 32 + rr;
                        if (r < t.n_rows && b < B)
                            *reinterpret_cast<float4*>(out + ((int64_t)t.out_row + r) * ld + b) = x[it];
                    }
                }
                if (full_box) {
                    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                    __syncwarp();
                    if (lane == 0 && b0 + cc * 32 < B) tma_store_2d(&map_out, b0 + cc * 32, t.out_row + q * 32, box);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(mempty + mb);
        }
        // every box store has completed its writes
        if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
        __syncwarp();
        if (bad) pcb::report_status(status, PCB_STATUS_TILE_TOO_LONG);
    }
    __syncthreads();
    if (tid == 0 && slot[1] != 0) pcb::report_status(status, PCB_STATUS_WAIT_TIMEOUT);
    if (warp == 1) tmem_dealloc(taddr, 2 * N);
}

// Tensor map of a row-major FP32 matrix [rows, ld] read in boxes of 32 samples x box_rows
// rows with 128-byte swizzle; samples >= B and rows >= rows read as zero.
int encode_rows_map(CUtensorMap* map, const float* base, int64_t ld, int64_t rows, int B, int box_rows) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return pcb::set_error(PCB_E_CUDA, "pcb_lse_contract_tc05_ws: cuTensorMapEncodeTiled unavailable");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[2] = {(cuuint64_t)B, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
    const cuuint32_t box[2] = {32, (cuuint32_t)box_rows};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, es,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_tc05_ws: tensor map rejected (%d)", (int)r);
    return PCB_OK;
}

template <int N, int MODE, bool SPLIT>
int launch_ws(int num_tiles, int num_ctas, const CUtensorMap& m1, const CUtensorMap& m2, const CUtensorMap& mo,
              const float* aux, float* out,
              int64_t ld, int B, int run_log2, const uint8_t* packed, const PcbLseTile* tiles, const int* krow,
              cudaStream_t s) {
    constexpr size_t smem = WsSmem<N, MODE, SPLIT>::bytes();
    static_assert(smem <= 227 * 1024, "shared memory");
    static bool configured[64] = {false};
    const int dev = current_device();
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(lse_tc05_ws_kernel<N, MODE, SPLIT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return pcb::set_error(PCB_E_CUDA, "pcb_lse_contract_tc05_ws: %s", cudaGetErrorString(e));
        configured[dev] = true;
    }
    const int64_t units = (int64_t)num_tiles * pcb::cdiv(B, N);
    const int grid = (int)std::min<int64_t>(units, num_ctas);
    return pcb::launch_status(pcb::launch_k(lse_tc05_ws_kernel<N, MODE, SPLIT>, dim3((unsigned)grid),
                                            dim3(kWsThreads), smem, s, 1u, m1, m2, mo, aux, out, ld, B, run_log2, packed,
                                            tiles, num_tiles, krow, pcb::status_word()),
                              "pcb_lse_contract_tc05_ws");
}

template <int N>
int launch_ws_n(int mode, bool split, int num_tiles, int num_ctas, const CUtensorMap& m1, const CUtensorMap& m2,
                const CUtensorMap& mo, const float* aux, float* out, int64_t ld, int B, int run_log2, const uint8_t* packed,
                const PcbLseTile* tiles, const int* krow, cudaStream_t s) {
#define PCB_WS(M, SP) \
    launch_ws<N, M, SP>(num_tiles, num_ctas, m1, m2, mo, aux, out, ld, B, run_log2, packed, tiles, krow, s)
    if (split) return mode == 0 ? PCB_WS(0, true) : (mode == 1 ? PCB_WS(1, true) : PCB_WS(2, true));
    return mode == 0 ? PCB_WS(0, false) : (mode == 1 ? PCB_WS(1, false) : PCB_WS(2, false));
#undef PCB_WS
}

template <int N, int MODE, int PREC>
int launch(int num_tiles, int spc, const float* src, const float* src2, const float* aux, float* out, int64_t ld,
           int B, const uint8_t* packed, const PcbLseTile* tiles, const int* krow, cudaStream_t s, bool vec, bool accum) {
    constexpr size_t smem = Tc05Smem<N>::bytes();
    static_assert(smem <= 227 * 1024, "shared memory");
    static bool configured[64] = {false};
    const int dev = current_device();
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(lse_tc05_kernel<N, MODE, PREC>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_lse_contract_tc05: %s", cudaGetErrorString(e));
        configured[dev] = true;
    }
    const int64_t gy = pcb::cdiv(pcb::cdiv(B, N), spc);
    if (gy > 65535) return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_tc05: batch too large");
    return pcb::launch_status(pcb::launch_k(lse_tc05_kernel<N, MODE, PREC>,
                                            dim3((unsigned)num_tiles, (unsigned)gy), dim3(tc05_threads<N>()), smem, s,
                                            1u, src, src2, aux, out, ld, B, packed, tiles, krow, spc, vec, accum,
                                            pcb::status_word()),
                              "pcb_lse_contract_tc05");
}

template <int N>
int launch_n(int mode, int prec, int num_tiles, int spc, const float* src, const float* src2, const float* aux,
             float* out, int64_t ld, int B, const uint8_t* packed, const PcbLseTile* tiles, const int* krow,
             cudaStream_t s, bool vec, bool accum) {
#define PCB_TC(M, P) launch<N, M, P>(num_tiles, spc, src, src2, aux, out, ld, B, packed, tiles, krow, s, vec, accum)
    if (prec == 3) return mode == 0 ? PCB_TC(0, 3) : (mode == 1 ? PCB_TC(1, 3) : PCB_TC(2, 3));
    if (prec == 2) return mode == 0 ? PCB_TC(0, 2) : (mode == 1 ? PCB_TC(1, 2) : PCB_TC(2, 2));
    return mode == 0 ? PCB_TC(0, 1) : (mode == 1 ? PCB_TC(1, 1) : PCB_TC(2, 1));
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

extern "C" int pcb_pack_weights_fp8(const float* params, const PcbLseTile* tiles, int32_t num_tiles,
                                    int32_t rows_per_block, const int32_t* kw, int32_t w_stride, uint8_t* packed,
                                    void* stream) {
    if (!params || !tiles || !kw || !packed || num_tiles < 0 || rows_per_block <= 0 ||
        (rows_per_block & (rows_per_block - 1)) || (reinterpret_cast<uintptr_t>(packed) & 15) != 0)
        return pcb::set_error(PCB_E_ARG, "pcb_pack_weights_fp8: bad arguments");
    if (num_tiles == 0) return PCB_OK;
    int rpb_log2 = 0;
    while ((1 << rpb_log2) < rows_per_block) ++rpb_log2;
    return pcb::launch_status(pcb::launch_k(pack_weights_fp8_kernel, dim3((unsigned)num_tiles), dim3(256), 0,
                                            pcb::as_stream(stream), 1u, params, tiles, rpb_log2, kw, w_stride, packed),
                              "pcb_pack_weights_fp8");
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

static int tc05_entry(const float* src, const float* src2, const float* aux, float* out, int64_t ld,
                                     int32_t B, const uint8_t* packed, const PcbLseTile* tiles, int32_t num_tiles,
                                     const int32_t* krow, int32_t mode, int32_t prec, int32_t batch_tile,
                                     int32_t slices_per_cta, void* stream, bool accum) {
    if (!src || !out || !packed || !tiles || !krow || B <= 0 || ld < B || num_tiles < 0 || mode < 0 || mode > 2 ||
        (mode == 2 && !src2) || (mode >= 1 && !aux) || prec < 1 || prec > 3 ||
        (batch_tile != 32 && batch_tile != 64) || slices_per_cta < 1 || (reinterpret_cast<uintptr_t>(packed) & 15) != 0)
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_tc05: bad arguments");
    if (num_tiles == 0) return PCB_OK;
    const bool vec = pcb::vec_ok(src, ld) && pcb::vec_ok(out, ld) && (!src2 || pcb::vec_ok(src2, ld)) &&
                     (!aux || pcb::vec_ok(aux, ld));
    cudaStream_t s = pcb::as_stream(stream);
    const int spc = slices_per_cta;
    if (batch_tile == 32)
        return launch_n<32>(mode, prec, num_tiles, spc, src, src2, aux, out, ld, B, packed, tiles, krow, s, vec,
                            accum);
    return launch_n<64>(mode, prec, num_tiles, spc, src, src2, aux, out, ld, B, packed, tiles, krow, s, vec, accum);
}

extern "C" int pcb_lse_contract_tc05(const float* src, const float* src2, const float* aux, float* out, int64_t ld,
                                     int32_t B, const uint8_t* packed, const PcbLseTile* tiles, int32_t num_tiles,
                                     const int32_t* krow, int32_t mode, int32_t prec, int32_t batch_tile,
                                     int32_t slices_per_cta, void* stream) {
    return tc05_entry(src, src2, aux, out, ld, B, packed, tiles, num_tiles, krow, mode, prec, batch_tile,
                      slices_per_cta, stream, false);
}

extern "C" int pcb_lse_contract_tc05_accum(const float* src, const float* src2, const float* aux, float* out,
                                           int64_t ld, int32_t B, const uint8_t* packed, const PcbLseTile* tiles,
                                           int32_t num_tiles, const int32_t* krow, int32_t mode, int32_t prec,
                                           int32_t batch_tile, int32_t slices_per_cta, void* stream) {
    return tc05_entry(src, src2, aux, out, ld, B, packed, tiles, num_tiles, krow, mode, prec, batch_tile,
                      slices_per_cta, stream, true);
}

namespace {

// Long tiles as 128-term chunks contracted in one launch into partial rows, then combined:
// out[dst_rows[r], b] = log sum_j exp(part[j S + r, b]) (mode 0) or sum_j part[j S + r, b]
// (modes 1/2), j < nch[r], in a fixed order. One thread per (row, sample), samples fastest.
__global__ void __launch_bounds__(256)
chunk_combine_kernel(const float* __restrict__ part, int64_t ld, int B, int S, const int* __restrict__ dst_rows,
                     const int* __restrict__ nch, float* __restrict__ out, int mode) {
    pcb::pdl_begin();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)S * B) return;
    const int r = (int)(i / B), b = (int)(i % B);
    const int n = nch[r];
    const float* p = part + (int64_t)r * ld + b;
    const int64_t js = (int64_t)S * ld;
    float res;
    if (mode == 0) {
        float m = -INFINITY;
        for (int j = 0; j < n; ++j) m = fmaxf(m, p[j * js]);
        float sum = 0.f;
        if (m != -INFINITY)
            for (int j = 0; j < n; ++j) sum += expf(p[j * js] - m);
        res = m == -INFINITY ? -INFINITY : m + logf(sum);
    } else {
        res = 0.f;
        for (int j = 0; j < n; ++j) res += p[j * js];
    }
    out[(int64_t)dst_rows[r] * ld + b] = res;
}

}  // namespace

extern "C" int pcb_chunk_combine(const float* partials, int64_t ld, int32_t B, int32_t num_rows,
                                 const int32_t* dst_rows, const int32_t* chunks_per_row, float* out, int32_t mode,
                                 void* stream) {
    if (!partials || !dst_rows || !chunks_per_row || !out || B <= 0 || ld < B || num_rows < 0 || mode < 0 || mode > 2)
        return pcb::set_error(PCB_E_ARG, "pcb_chunk_combine: bad arguments");
    if (num_rows == 0) return PCB_OK;
    const int64_t total = (int64_t)num_rows * B;
    return pcb::launch_status(pcb::launch_k(chunk_combine_kernel, dim3((unsigned)pcb::cdiv(total, 256)), dim3(256), 0,
                                            pcb::as_stream(stream), 1u, partials, ld, (int)B, (int)num_rows, dst_rows,
                                            chunks_per_row, out, (int)mode),
                              "pcb_chunk_combine");
}

extern "C" int pcb_lse_contract_tc05_ws(const float* src, const float* src2, const float* aux, float* out,
                                        int64_t ld, int32_t B, int64_t src_rows, int64_t out_rows, const uint8_t* packed,
                                        const PcbLseTile* tiles, int32_t num_tiles, const int32_t* krow, int32_t mode,
                                        int32_t prec, int32_t batch_tile, int32_t run_rows, int32_t num_ctas,
                                        void* stream) {
    if (!src || !out || !packed || !tiles || !krow || B <= 0 || ld < B || src_rows <= 0 || out_rows <= 0 || num_tiles < 0 ||
        mode < 0 || mode > 2 || (mode == 2 && !src2) || (mode >= 1 && !aux) || prec < 1 || prec > 2 ||
        (batch_tile != 32 && batch_tile != 64) || (run_rows != 8 && run_rows != 32) || num_ctas < 0 ||
        (reinterpret_cast<uintptr_t>(packed) & 15) != 0)
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_tc05_ws: bad arguments");
    // TMA boxes of 32 samples: 16-byte aligned rows (ld % 4 == 0) and whole 4-sample groups
    if (B % 4 != 0 || !pcb::vec_ok(src, ld) || !pcb::vec_ok(out, ld) || (src2 && !pcb::vec_ok(src2, ld)) ||
        (aux && !pcb::vec_ok(aux, ld)))
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_tc05_ws: needs B %% 4 == 0, ld %% 4 == 0 and 16-byte "
                                         "aligned rows");
    if (num_tiles == 0) return PCB_OK;
    int ctas = num_ctas;
    if (ctas == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&ctas, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return pcb::set_error(PCB_E_CUDA, "pcb_lse_contract_tc05_ws: device query failed");
    }
    CUtensorMap m1, m2, mo;
    int rc = encode_rows_map(&m1, src, ld, src_rows, B, run_rows);
    if (rc != PCB_OK) return rc;
    rc = encode_rows_map(&m2, src2 ? src2 : src, ld, src_rows, B, run_rows);
    if (rc != PCB_OK) return rc;
    rc = encode_rows_map(&mo, out, ld, out_rows, B, 32);
    if (rc != PCB_OK) return rc;
    const int run_log2 = run_rows == 8 ? 3 : 5;
    cudaStream_t s = pcb::as_stream(stream);
    const bool split = prec == 2;
    if (batch_tile == 32)
        return launch_ws_n<32>(mode, split, num_tiles, ctas, m1, m2, mo, aux, out, ld, B, run_log2, packed, tiles, krow,
                               s);
    return launch_ws_n<64>(mode, split, num_tiles, ctas, m1, m2, mo, aux, out, ld, B, run_log2, packed, tiles, krow, s);
}
