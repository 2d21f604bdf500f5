// Log-sum-exp contractions with at most 128 terms per output row, built for latency.
//
// Same result as the chunked kernels (lse_contract.cu, lse_contract_tc.cu):
//   acc[r, b] = sum_k W(k, r) * exp(src[krow[k], b] - m_b),  m_b = max_k src[krow[k], b]
//   W(k, r) = params[kw[k] + w_add + (r >> rpb_log2) * g_stride + (r & (rpb - 1)) * w_stride]
// A CTA first reads the tile's term indices into shared memory, then issues ALL its
// copies (up to 128 source rows over TB samples, and the RM x 128 weights of its rows) as
// one batch of asynchronous copies with no dependent global load in between, waits once,
// takes the exact per-sample max, exponentiates and contracts: four barriers per CTA and
// no online rescaling. A tile of up to 128 rows is split into row slices of RM and the
// batch into TB-sample slices, so a layer of two or three regions still launches enough
// CTAs to cover the GPU.
//
// Contraction forms: FP32 FMA (prec 0) or the BF16 tensor cores (prec 1: one bf16
// operand pair; prec 2: both operands split into bf16 hi + lo, three MMAs).
//
// Weight copies are 16 bytes wide when the host has checked that groups of 4 weights are
// contiguous and aligned: along the rows (wlayout 1, the forward: node-fastest parameter
// blocks) or along the terms (wlayout 2, element flows: a child's weights over the
// parents of one block are consecutive). wlayout 0 copies every weight on its own. In the
// BF16 forms the weights can instead come already rounded and split (pcb_pack_weights):
// the CTA then copies its rows of the packed tile as they are and reads the A fragments
// straight from that core-matrix layout (no per-CTA conversion of the weights).
//
// Epilogues: mode 0 writes log(acc) + m (sum forward); modes 1/2 write
// acc * exp(aux + m) (element flows; mode 2 first turns node flows into log f - log m).
#include <cuda_bf16.h>

#include "common.cuh"

namespace {

constexpr int kThreads = 128;

int current_device_ls() {
    int d = 0;
    cudaGetDevice(&d);
    return d < 0 ? 0 : (d > 63 ? 63 : d);
}
constexpr int KMAX = 128;
constexpr int kFuse = 4;  // children per element of a fused product layer (table stride)

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void split_bf16(float lo_k, float hi_k, uint32_t& h, uint32_t& l) {
    __nv_bfloat162 hv = __floats2bfloat162_rn(lo_k, hi_k);
    const float2 hf = __bfloat1622float2(hv);
    __nv_bfloat162 lv = __floats2bfloat162_rn(lo_k - hf.x, hi_k - hf.y);
    h = *reinterpret_cast<uint32_t*>(&hv);
    l = *reinterpret_cast<uint32_t*>(&lv);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Shared-memory plan (offsets in 4-byte words; every array starts 16-byte aligned).
// PREC: 0 = FP32, 1 = bf16, 2 = split bf16.
template <int RM, int TB, int MODE, int PREC, bool WK, bool FUSE = false>
struct Smem {
    static constexpr int ES = TB + 8;            // packed row strides: conflict-free fragment loads
    static constexpr int WS = RM + 8;
    static constexpr int NB = PREC == 2 ? 2 : (PREC == 1 ? 1 : 0);
    static constexpr int WROW = WK ? KMAX + 4 : RM + 4;   // fp32 weight staging row
    static constexpr int kE = KMAX * TB;
    // second staging set: node mars (mode 2) or children 1 .. kFuse - 1 (fused forward)
    static constexpr int kE2 = MODE == 2 ? KMAX * TB : ((MODE == 0 && FUSE) ? (kFuse - 1) * KMAX * TB : 0);
    static constexpr int kW = WK ? RM * WROW : KMAX * WROW;
    static constexpr int kPE = NB * (KMAX / 2) * ES;
    static constexpr int kPW = NB * (KMAX / 2) * WS;
    static constexpr int AS = TB + 4;            // epilogue rows (modes 1/2), 16-byte rows
    static constexpr int kA = MODE >= 1 ? RM * AS : 0;
    static constexpr int oE = 0, oE2 = oE + kE, oW = oE2 + kE2, oPE = oW + kW, oPW = oPE + kPE;
    static constexpr int oA = oPW + kPW, oPart = oA + kA, oMax = oPart + kThreads, oIdx = oMax + TB;
    static constexpr size_t bytes() { return 4ull * (oIdx + (2 + kFuse) * KMAX); }
};

// One work item of the single-stage contraction: rows r0 .. r0 + RM - 1 of tile t (number
// tile_index of its table, for the packed weights) for samples b0 .. b0 + TB - 1. With pdl,
// the source rows are read after the programmatic-launch wait.
template <int RM, int TB, int MODE, int PREC, bool WK, bool FUSE>
__device__ __forceinline__ void short_item(const float* __restrict__ src, const float* __restrict__ src2,
                                           const float* __restrict__ aux, float* __restrict__ out, int64_t ld, int B,
                                           const float* __restrict__ params, const PcbLseTile t, int tile_index, int r0,
                                           int b0, const int* __restrict__ krow, const int* __restrict__ kw,
                                           int w_stride, int rpb_log2, bool vec, bool wvec,
                                           const uint8_t* __restrict__ packed, const PcbShortFusion& fu,
                                           int32_t* __restrict__ status, bool pdl, const int* wait_ctr = nullptr,
                                           int wait_need = 0) {
    using S = Smem<RM, TB, MODE, PREC, WK, FUSE>;
    constexpr int ES = S::ES, WS = S::WS, WROW = S::WROW;
    constexpr int PARTS = kThreads / TB;  // threads per sample column in the max / exp passes
    static_assert(kThreads % TB == 0 && RM % 16 == 0 && TB % 8 == 0, "tile shape");
    extern __shared__ __align__(16) float sm[];
    float(*sE)[TB] = reinterpret_cast<float(*)[TB]>(sm + S::oE);
    float(*sE2)[TB] = reinterpret_cast<float(*)[TB]>(sm + S::oE2);
    float(*sW)[WROW] = reinterpret_cast<float(*)[WROW]>(sm + S::oW);
    uint32_t* pE = reinterpret_cast<uint32_t*>(sm + S::oPE);
    uint32_t* pW = reinterpret_cast<uint32_t*>(sm + S::oPW);
    float(*sAux)[S::AS] = reinterpret_cast<float(*)[S::AS]>(sm + S::oA);
    float* sPart = sm + S::oPart;
    float* sMax = sm + S::oMax;
    int* sRow = reinterpret_cast<int*>(sm + S::oIdx);
    int* sKw = sRow + KMAX;

    const int tid = threadIdx.x;
    const int nrows = min(RM, t.n_rows - r0);
    if (nrows <= 0) return;
    const bool bad = t.k_cnt > KMAX;  // the host only sends tiles of <= 128 terms; never read past them
    const int nk = bad ? 0 : t.k_cnt;
    if (bad && tid == 0) pcb::report_status(status, PCB_STATUS_TILE_TOO_LONG);
    const int rpb_mask = (1 << rpb_log2) - 1;

    // ---- term indices, then one batch of asynchronous copies ----
    int* sCh = sKw + KMAX;  // fused forward: [KMAX][kFuse] child node rows of each term
    if (tid < nk) {
        sRow[tid] = __ldg(krow + t.k_off + tid);
        sKw[tid] = __ldg(kw + t.k_off + tid);
        if (MODE == 0 && FUSE) {
#pragma unroll
            for (int j = 0; j < kFuse; ++j)
                sCh[kFuse * tid + j] = __ldg(fu.term_children + (int64_t)kFuse * (t.k_off + tid) + j);
        }
    }
    __syncthreads();
    constexpr int kPackHalf = RM * 256;
    const bool pk = PREC > 0 && packed != nullptr;
    auto wbase = [&](int r) -> int64_t {
        const int rr = r0 + r;
        return (int64_t)t.w_add + (int64_t)(rr >> rpb_log2) * t.g_stride + (int64_t)(rr & rpb_mask) * w_stride;
    };
    if (pk) {
    } else if (WK) {
        // sW[r][k]: each thread copies groups of 4 consecutive terms of one row
        constexpr int IT = RM * (KMAX / 4) / kThreads;
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int idx = tid + it * kThreads;
            const int r = idx / (KMAX / 4);
            const int k = (idx % (KMAX / 4)) * 4;
            if (r < nrows && k < nk) {
                const int64_t base = wbase(r);
                if (wvec && k + 3 < nk) {
                    pcb::cp_async16(&sW[r][k], params + base + sKw[k]);
                } else {
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (k + j < nk) sW[r][k + j] = __ldcg(params + base + sKw[k + j]);
                }
            }
        }
    } else {
        // sW[k][r]: each thread copies groups of 4 consecutive rows of one term
        constexpr int IT = KMAX * (RM / 4) / kThreads;
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int idx = tid + it * kThreads;
            const int k = idx / (RM / 4);
            const int r = (idx % (RM / 4)) * 4;
            if (k < nk && r < nrows) {
                const int64_t kb = sKw[k];
                if (wvec && r + 3 < nrows) {
                    pcb::cp_async16(&sW[k][r], params + kb + wbase(r));
                } else {
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (r + j < nrows) sW[k][r + j] = __ldcg(params + kb + wbase(r + j));
                }
            }
        }
    }
    pcb::cp_async_commit();
    if constexpr (PREC > 0) {
        // weights -> bf16 pairs along the terms (split: hi, then lo), still before the wait
        if (!pk) {
            pcb::cp_async_wait<0>();
            __syncthreads();
            for (int idx = tid; idx < (KMAX / 2) * RM; idx += kThreads) {
                const int kk = idx / RM;
                const int r = idx % RM;
                float w0 = 0.f, w1 = 0.f;
                if (r < nrows) {
                    if (2 * kk < nk) w0 = WK ? sW[r][2 * kk] : sW[2 * kk][r];
                    if (2 * kk + 1 < nk) w1 = WK ? sW[r][2 * kk + 1] : sW[2 * kk + 1][r];
                }
                if (PREC == 2) split_bf16(w0, w1, pW[kk * WS + r], pW[(KMAX / 2) * WS + kk * WS + r]);
                else pW[kk * WS + r] = pack_bf16(w0, w1);
            }
        }
    }

    if (pdl) pcb::pdl_wait();
    if (wait_ctr != nullptr && wait_need > 0) {
        // the node rows this item reads are written by earlier items (persistent launch)
        if (tid == 0) {
            const volatile int* done = wait_ctr;
            int i = 0;
            while (*done < wait_need && ++i < (1 << 20)) {
            }
            if (*done < wait_need) pcb::report_status(status, PCB_STATUS_WAIT_TIMEOUT);
            __threadfence();
        }
        __syncthreads();
    }
    {
        constexpr int NX = TB / 4;
        constexpr int IT = KMAX * NX / kThreads;
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int idx = tid + it * kThreads;
            const int k = idx / NX;
            const int c4 = idx % NX;
            const int b = b0 + c4 * 4;
            if (k < nk) {
                constexpr bool F0 = MODE == 0 && FUSE;
#pragma unroll
                for (int h = 0; h < (MODE == 2 ? 2 : (F0 ? kFuse : 1)); ++h) {
                    // fused forward: the term's element value is the sum of its child node
                    // rows (staged in set h = child h; a missing child reads as 0)
                    float* d = h == 0 ? &sE[k][c4 * 4] : &sE2[(h - 1) * KMAX + k][c4 * 4];
                    const int row = F0 ? sCh[kFuse * k + h] : sRow[k];
                    if (F0 && row < 0) {
                        *reinterpret_cast<float4*>(d) = make_float4(0.f, 0.f, 0.f, 0.f);
                        continue;
                    }
                    const float* g = (h == 0 || F0 ? src : src2) + (int64_t)row * ld + b;
                    if (vec && b + 3 < B) {
                        pcb::cp_async16(d, g);
                    } else {
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            if (b + j < B) pcb::cp_async4(d + j, g + j);
                            else d[j] = -INFINITY;
                        }
                    }
                }
            }
        }
    }
    // packed bf16 weights (hi, then lo): rows r0 .. r0 + RM - 1 are RM / 8 core-matrix row
    // groups of 2048 bytes in each half of the tile's 64 KB block
    if (pk) {
        const uint8_t* srcp = packed + (size_t)tile_index * 65536 + (size_t)(r0 / 8) * 2048;
        uint8_t* dstp = reinterpret_cast<uint8_t*>(pW);
        constexpr int CH = kPackHalf / 16;
        constexpr int IT = (PREC == 2 ? 2 : 1) * CH / kThreads;
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int i = tid + it * kThreads;
            const int h = i / CH, c = i % CH;
            pcb::cp_async16(dstp + h * kPackHalf + c * 16, srcp + (size_t)h * 32768 + c * 16);
        }
    }
    if constexpr (MODE >= 1) {
        // the epilogue's element values: RM rows x TB samples, in the same batch of copies
        constexpr int NX = TB / 4;
        for (int idx = tid; idx < RM * NX; idx += kThreads) {
            const int r = idx / NX;
            const int c4 = (idx % NX) * 4;
            const int b = b0 + c4;
            if (r >= nrows) continue;
            float* d = &sAux[r][c4];
            const float* g = aux + ((int64_t)t.aux_row + r0 + r) * ld + b;
            if (vec && b + 3 < B) {
                pcb::cp_async16(d, g);
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (b + j < B) pcb::cp_async4(d + j, g + j);
                    else d[j] = 0.f;
                }
            }
        }
    }
    pcb::cp_async_commit();
    pcb::cp_async_wait<0>();
    __syncthreads();

    // ---- exact per-sample max (mode 2: node flows -> log f - log m first) ----
    const int cb = tid % TB;  // this thread's sample column in the max and exp passes
    const int part = tid / TB;
    {
        float mx = -INFINITY;
        const bool write_em = MODE == 0 && FUSE && r0 == 0 && b0 + cb < B;
        for (int k = part; k < nk; k += PARTS) {
            float v = sE[k][cb];
            if (MODE == 2) {
                const float m2 = sE2[k][cb];
                v = (m2 == -INFINITY) ? -INFINITY : logf(v) - m2;
                sE[k][cb] = v;
            }
            if (MODE == 0 && FUSE) {
#pragma unroll
                for (int j = 1; j < kFuse; ++j) v = v + sE2[(j - 1) * KMAX + k][cb];
                sE[k][cb] = v;
                if (write_em) fu.element_out[(int64_t)sRow[k] * ld + b0 + cb] = v;
            }
            mx = fmaxf(mx, v);
        }
        sPart[part * TB + cb] = mx;
    }
    __syncthreads();
    float m = -INFINITY;
#pragma unroll
    for (int p = 0; p < PARTS; ++p) m = fmaxf(m, sPart[p * TB + cb]);
    if (part == 0) sMax[cb] = m;

    const int warp = tid >> 5;
    const int lane = tid & 31;

    if constexpr (PREC == 0) {
        // ---- FP32: exponentiate in place, then FMA with an RN x 4 register tile per thread ----
        for (int k = part; k < nk; k += PARTS) sE[k][cb] = (m == -INFINITY) ? 0.f : __expf(sE[k][cb] - m);
        __syncthreads();
        constexpr int NX = TB / 4;
        constexpr int NY = kThreads / NX;
        constexpr int RN = RM / NY;
        static_assert(RN >= 1 && RM % NY == 0, "fp32 tile shape");
        const int tx = tid % NX;
        const int ty = tid / NX;
        float acc[RN][4];
#pragma unroll
        for (int r = 0; r < RN; ++r)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[r][j] = 0.f;
        for (int k = 0; k < nk; ++k) {
            const float4 e = *reinterpret_cast<const float4*>(&sE[k][tx * 4]);
#pragma unroll
            for (int r = 0; r < RN; ++r) {
                const int rr = ty * RN + r;
                const float w = (rr < nrows) ? (WK ? sW[rr][k] : sW[k][rr]) : 0.f;
                acc[r][0] = fmaf(w, e.x, acc[r][0]);
                acc[r][1] = fmaf(w, e.y, acc[r][1]);
                acc[r][2] = fmaf(w, e.z, acc[r][2]);
                acc[r][3] = fmaf(w, e.w, acc[r][3]);
            }
        }
        const int bb = b0 + tx * 4;
#pragma unroll
        for (int r = 0; r < RN; ++r) {
            const int rr = ty * RN + r;
            if (rr >= nrows) continue;
            const int row = r0 + rr;
            float4 o;
            if (bad) {
                o = make_float4(__int_as_float(0x7fc00000), __int_as_float(0x7fc00000), __int_as_float(0x7fc00000),
                                __int_as_float(0x7fc00000));
            } else if (MODE == 0) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float mm = sMax[tx * 4 + j];
                    pcb::set(o, j, (mm == -INFINITY) ? -INFINITY : logf(acc[r][j]) + mm);
                }
            } else {
                const float4 a = *reinterpret_cast<const float4*>(&sAux[rr][tx * 4]);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float mm = sMax[tx * 4 + j];
                    pcb::set(o, j, (mm == -INFINITY) ? 0.f : acc[r][j] * __expf(pcb::get(a, j) + mm));
                }
            }
            if (MODE != 0 && FUSE) {
                const int64_t e = (int64_t)t.out_row + row;
#pragma unroll
                for (int h = 0; h < kFuse; ++h) {
                    const int c = __ldg(fu.out_children + kFuse * e + h);
                    if (c >= 0) pcb::store4(out, c, ld, bb, B, vec, o);
                }
            } else {
                pcb::store4(out, (int64_t)t.out_row + row, ld, bb, B, vec, o);
            }
        }
    } else {
        constexpr bool SPLIT = PREC == 2;
        constexpr int WM = (RM / 16) < 4 ? (RM / 16) : 4;  // warps along rows
        constexpr int WN = 4 / WM;                          // warps along samples
        constexpr int MT = RM / 16 / WM;                    // m16 tiles per warp
        constexpr int NTL = TB / 8 / WN;                    // n8 tiles per warp
        static_assert(NTL >= 1 && MT >= 1, "mma tile shape");
        // ---- exponentiate and repack both operands as bf16 pairs along the terms ----
        for (int kk = part; kk < KMAX / 2; kk += PARTS) {
            float e0 = 0.f, e1 = 0.f;
            if (m != -INFINITY) {
                if (2 * kk < nk) e0 = __expf(sE[2 * kk][cb] - m);
                if (2 * kk + 1 < nk) e1 = __expf(sE[2 * kk + 1][cb] - m);
            }
            if (SPLIT) split_bf16(e0, e1, pE[kk * ES + cb], pE[(KMAX / 2) * ES + kk * ES + cb]);
            else pE[kk * ES + cb] = pack_bf16(e0, e1);
        }
        __syncthreads();

        // ---- tensor-core contraction ----
        const int g = lane >> 2;
        const int q = lane & 3;
        const int mw = (warp % WM) * MT * 16;
        const int nw = (warp / WM) * NTL * 8;
        float acc[MT][NTL][4];
#pragma unroll
        for (int a = 0; a < MT; ++a)
#pragma unroll
            for (int c = 0; c < NTL; ++c)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[a][c][j] = 0.f;
        const int kend = (nk + 15) & ~15;
        for (int k0 = 0; k0 < kend; k0 += 16) {
            const int kk = k0 >> 1;
            uint32_t bh[NTL][2], bl[NTL][2];
#pragma unroll
            for (int c = 0; c < NTL; ++c) {
                const int col = nw + c * 8 + g;
                bh[c][0] = pE[(kk + q) * ES + col];
                bh[c][1] = pE[(kk + 4 + q) * ES + col];
                if (SPLIT) {
                    bl[c][0] = pE[(KMAX / 2) * ES + (kk + q) * ES + col];
                    bl[c][1] = pE[(KMAX / 2) * ES + (kk + 4 + q) * ES + col];
                }
            }
#pragma unroll
            for (int a = 0; a < MT; ++a) {
                const int mr = mw + a * 16 + g;
                uint32_t a0, a1, a2, a3, l0 = 0, l1 = 0, l2 = 0, l3 = 0;
                if (pk) {
                    // word of (row group G, k group kg, row g of the group, pair q): G*512 + kg*32 + g*4 + q
                    const int w0 = ((mw + a * 16) >> 3) * 512 + (k0 >> 3) * 32 + g * 4 + q;
                    a0 = pW[w0]; a1 = pW[w0 + 512]; a2 = pW[w0 + 32]; a3 = pW[w0 + 544];
                    if (SPLIT) {
                        const int w1 = w0 + kPackHalf / 4;
                        l0 = pW[w1]; l1 = pW[w1 + 512]; l2 = pW[w1 + 32]; l3 = pW[w1 + 544];
                    }
                } else {
                    a0 = pW[(kk + q) * WS + mr]; a1 = pW[(kk + q) * WS + mr + 8];
                    a2 = pW[(kk + 4 + q) * WS + mr]; a3 = pW[(kk + 4 + q) * WS + mr + 8];
                    if (SPLIT) {
                        const int o = (KMAX / 2) * WS;
                        l0 = pW[o + (kk + q) * WS + mr]; l1 = pW[o + (kk + q) * WS + mr + 8];
                        l2 = pW[o + (kk + 4 + q) * WS + mr]; l3 = pW[o + (kk + 4 + q) * WS + mr + 8];
                    }
                }
#pragma unroll
                for (int c = 0; c < NTL; ++c) mma_bf16(acc[a][c], a0, a1, a2, a3, bh[c][0], bh[c][1]);
                if (SPLIT) {
#pragma unroll
                    for (int c = 0; c < NTL; ++c) {
                        mma_bf16(acc[a][c], l0, l1, l2, l3, bh[c][0], bh[c][1]);
                        mma_bf16(acc[a][c], a0, a1, a2, a3, bl[c][0], bl[c][1]);
                    }
                }
            }
        }

        // ---- epilogue ----
#pragma unroll
        for (int a = 0; a < MT; ++a) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = mw + a * 16 + g + h * 8;
                if (r >= nrows) continue;
                const int row = r0 + r;
#pragma unroll
                for (int c = 0; c < NTL; ++c) {
                    const int col = nw + c * 8 + 2 * q;
                    const int b = b0 + col;
                    float o[2];
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const float mm = sMax[col + j];
                        const float v = acc[a][c][h * 2 + j];
                        if (bad) {
                            o[j] = __int_as_float(0x7fc00000);
                        } else if (MODE == 0) {
                            o[j] = (mm == -INFINITY) ? -INFINITY : __logf(v) + mm;
                        } else {
                            const float x = sAux[r][col + j];
                            o[j] = (mm == -INFINITY) ? 0.f : v * __expf(x + mm);
                        }
                    }
#pragma unroll
                    for (int hh = 0; hh < ((MODE != 0 && FUSE) ? kFuse : 1); ++hh) {
                        int64_t orow = (int64_t)t.out_row + row;
                        if (MODE != 0 && FUSE) {
                            // fused backward: the element's flow is the flow of its child rows
                            const int c = __ldg(fu.out_children + kFuse * orow + hh);
                            if (c < 0) continue;
                            orow = c;
                        }
                        float* dst = out + orow * ld + b;
                        if (vec && b + 1 < B) {
                            *reinterpret_cast<float2*>(dst) = make_float2(o[0], o[1]);
                        } else {
                            if (b < B) dst[0] = o[0];
                            if (b + 1 < B) dst[1] = o[1];
                        }
                    }
                }
            }
        }
    }
}

template <int RM, int TB, int MODE, int PREC, bool WK, bool FUSE>
__global__ void __launch_bounds__(kThreads)
lse_short_kernel(const float* __restrict__ src, const float* __restrict__ src2, const float* __restrict__ aux,
                 float* __restrict__ out, int64_t ld, int B, const float* __restrict__ params,
                 const PcbLseTile* __restrict__ tiles, const int* __restrict__ krow, const int* __restrict__ kw,
                 int w_stride, int rpb_log2, int row_splits, bool vec, bool wvec,
                 const uint8_t* __restrict__ packed, PcbShortFusion fu, int32_t* __restrict__ status) {
    // The term indices and the weights (compiled tables and parameters) are read before the
    // wait for the previous kernel; only the source rows and the packed weights after it.
    pcb::pdl_trigger();
    const int ti = blockIdx.x / row_splits;
    short_item<RM, TB, MODE, PREC, WK, FUSE>(src, src2, aux, out, ld, B, params, tiles[ti], ti,
                                             (blockIdx.x % row_splits) * RM, blockIdx.y * TB, krow, kw, w_stride,
                                             rpb_log2, vec, wvec, packed, fu, status, true);
}

// ---------------------------------------------------------------------------------------
// A run of small levels (fused product + sum forward) in one persistent launch. Work items
// (level, slice, tile, row split) are numbered level by level; every CTA takes the next
// item from a global counter, waits until its sample slice has finished all items of the
// earlier levels (a per-slice completion counter), runs the item and counts it done.
// Samples are independent, so no other synchronisation is needed. Items are handed out in
// level order to running CTAs only, so an item waits only for items that running CTAs
// hold: the wait always ends (and is bounded in any case).
template <int RM, int TB, int PREC, bool WK>
__global__ void __launch_bounds__(kThreads)
short_levels_kernel(float* __restrict__ nm, int64_t ld, int B, const float* __restrict__ params,
                    const PcbLseTile* __restrict__ tiles, const int* __restrict__ krow, const int* __restrict__ kw,
                    const int* __restrict__ term_children, const PcbShortLevel* __restrict__ levels, int num_levels,
                    int total_items, int* __restrict__ counters, bool vec, int32_t* __restrict__ status) {
    pcb::pdl_trigger();
    pcb::pdl_wait();
    __shared__ int s_item;
    int lv = 0;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counters, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= total_items) break;
        while (lv + 1 < num_levels && levels[lv + 1].item0 <= item) ++lv;
        const PcbShortLevel L = levels[lv];
        const int local = item - L.item0;
        const int split = local % L.row_splits;
        const int ts = local / L.row_splits;
        const int tile = ts % L.num_tiles;
        const int slice = ts / L.num_tiles;
        PcbShortFusion fu;
        fu.term_children = term_children;
        fu.element_out = L.element_out;
        fu.out_children = nullptr;
        short_item<RM, TB, 0, PREC, WK, true>(nm, nullptr, nullptr, nm, ld, B, params, tiles[L.tile0 + tile], tile,
                                              split * RM, slice * TB, krow, kw, L.w_stride, L.rpb_log2, vec,
                                              L.wvec != 0, nullptr, fu, status, false, counters + 1 + slice, L.need);
        __syncthreads();  // the item's stores, then the next item reuses the shared memory
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(counters + 1 + slice, 1);
        }
    }
}

template <int TB, int PREC, bool WK>
int launch_levels(float* nm, int64_t ld, int B, const float* params, const PcbLseTile* tiles, const int* krow,
                  const int* kw, const int* term_children, const PcbShortLevel* levels, int num_levels,
                  int total_items, int* counters, int num_ctas, cudaStream_t s, bool vec) {
    constexpr int RM = 64;
    constexpr size_t smem = Smem<RM, TB, 0, PREC, WK, true>::bytes();
    static_assert(smem <= 227 * 1024, "shared memory");
    static bool configured[64] = {false};
    const int dev = current_device_ls();
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(short_levels_kernel<RM, TB, PREC, WK>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_lse_levels_short: %s", cudaGetErrorString(e));
        configured[dev] = true;
    }
    return pcb::launch_status(pcb::launch_k(short_levels_kernel<RM, TB, PREC, WK>, dim3((unsigned)num_ctas),
                                            dim3(kThreads), smem, s, 1u, nm, ld, B, params, tiles, krow, kw,
                                            term_children, levels, num_levels, total_items, counters, vec,
                                            pcb::status_word()),
                              "pcb_lse_levels_short");
}

int current_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d < 0 ? 0 : (d > 63 ? 63 : d);
}

template <int RM, int TB, int MODE, int PREC, bool WK, bool FUSE>
int launch_one(int num_tiles, int row_splits, const float* src, const float* src2, const float* aux, float* out,
               int64_t ld, int B, const float* params, const PcbLseTile* tiles, const int* krow, const int* kw,
               int w_stride, int rpb_log2, cudaStream_t s, bool vec, bool wvec, const uint8_t* packed,
               const PcbShortFusion& fu) {
    constexpr size_t smem = Smem<RM, TB, MODE, PREC, WK, FUSE>::bytes();
    static_assert(smem <= 227 * 1024, "shared memory");
    static bool configured[64] = {false};
    const int dev = current_device();
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(lse_short_kernel<RM, TB, MODE, PREC, WK, FUSE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_lse_contract_short: %s", cudaGetErrorString(e));
        configured[dev] = true;
    }
    const int64_t gx = (int64_t)num_tiles * row_splits;
    const int64_t gy = pcb::cdiv(B, TB);
    if (gx > 2147483647 || gy > 65535) return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_short: grid too large");
    return pcb::launch_status(pcb::launch_k(lse_short_kernel<RM, TB, MODE, PREC, WK, FUSE>,
                                            dim3((unsigned)gx, (unsigned)gy), dim3(kThreads), smem, s, 1u, src,
                                            src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2,
                                            row_splits, vec, wvec, packed, fu, pcb::status_word()),
                              "pcb_lse_contract_short");
}

template <int RM, int TB, int PREC>
int launch_prec(int num_tiles, int row_splits, const float* src, const float* src2, const float* aux, float* out,
                int64_t ld, int B, const float* params, const PcbLseTile* tiles, const int* krow, const int* kw,
                int w_stride, int rpb_log2, int mode, bool wk, cudaStream_t s, bool vec, bool wvec,
                const uint8_t* packed, const PcbShortFusion& fu) {
    // fusion: forward (mode 0) with term_children, element flows (mode 2) with out_children
    const bool f = mode == 0 ? fu.term_children != nullptr : (mode == 2 && fu.out_children != nullptr);
#define PCB_LS(M, W, F) \
    launch_one<RM, TB, M, PREC, W, F>(num_tiles, row_splits, src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2, s, vec, wvec, packed, fu)
    if (f) {
        // fused forms stage up to four child rows per term: batch tiles of at most 32 samples
        if constexpr (TB <= 32) {
            if (wk) return mode == 0 ? PCB_LS(0, true, true) : PCB_LS(2, true, true);
            return mode == 0 ? PCB_LS(0, false, true) : PCB_LS(2, false, true);
        } else {
            return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_short: product fusion needs batch_tile <= 32");
        }
    }
    if (wk) return mode == 0 ? PCB_LS(0, true, false) : (mode == 1 ? PCB_LS(1, true, false) : PCB_LS(2, true, false));
    return mode == 0 ? PCB_LS(0, false, false) : (mode == 1 ? PCB_LS(1, false, false) : PCB_LS(2, false, false));
#undef PCB_LS
}

template <int RM, int TB>
int launch_shape(int num_tiles, int row_splits, const float* src, const float* src2, const float* aux, float* out,
                 int64_t ld, int B, const float* params, const PcbLseTile* tiles, const int* krow, const int* kw,
                 int w_stride, int rpb_log2, int mode, int prec, bool wk, cudaStream_t s, bool vec, bool wvec,
                 const uint8_t* packed, const PcbShortFusion& fu) {
#define PCB_LP(P) \
    launch_prec<RM, TB, P>(num_tiles, row_splits, src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2, mode, wk, s, vec, wvec, packed, fu)
    if (prec == 0) return PCB_LP(0);
    if (prec == 1) return PCB_LP(1);
    return PCB_LP(2);
#undef PCB_LP
}

}  // namespace

extern "C" int pcb_lse_contract_short(const float* src, const float* src2, const float* aux, float* out, int64_t ld,
                                      int32_t B, const float* params, const PcbLseTile* tiles, int32_t num_tiles,
                                      int32_t tile_rows, int32_t rows_per_block, const int32_t* krow,
                                      const int32_t* kw, int32_t w_stride, int32_t mode, int32_t prec,
                                      const uint8_t* packed, int32_t wlayout, int32_t batch_tile,
                                      const PcbShortFusion* fusion, void* stream) {
    if (!src || !out || !params || !tiles || !krow || !kw || B <= 0 || ld < B || num_tiles < 0 || mode < 0 ||
        mode > 2 || (mode == 2 && !src2) || (mode >= 1 && !aux) || rows_per_block <= 0 ||
        (rows_per_block & (rows_per_block - 1)) || tile_rows < 1 || tile_rows > 128 || prec < 0 || prec > 2 ||
        wlayout < 0 || wlayout > 2 || (batch_tile != 16 && batch_tile != 32 && batch_tile != 64))
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_short: bad arguments");
    if (num_tiles == 0) return PCB_OK;
    if (packed && (prec == 0 || (reinterpret_cast<uintptr_t>(packed) & 15) != 0))
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_short: packed weights need a BF16 form and 16-byte alignment");
    if (wlayout != 0 && (reinterpret_cast<uintptr_t>(params) & 15) != 0)
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_short: 16-byte weight copies need an aligned params base");
    PcbShortFusion fu = {nullptr, nullptr, nullptr};
    if (fusion) fu = *fusion;
    if ((fu.term_children && (mode != 0 || !fu.element_out)) || (fu.out_children && mode != 2))
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract_short: product fusion needs mode 0 (with element_out) or mode 2");
    if (mode != 0) fu.term_children = nullptr;
    if (mode != 2) fu.out_children = nullptr;
    int rpb_log2 = 0;
    while ((1 << rpb_log2) < rows_per_block) ++rpb_log2;
    const bool vec = pcb::vec_ok(src, ld) && pcb::vec_ok(out, ld) && (!src2 || pcb::vec_ok(src2, ld)) &&
                     (!aux || pcb::vec_ok(aux, ld));
    const bool wk = wlayout == 2;
    const bool wvec = wlayout != 0;
    cudaStream_t s = pcb::as_stream(stream);
    const int rm = tile_rows <= 32 ? 32 : 64;
    const int row_splits = (tile_rows + rm - 1) / rm;
#define PCB_SH(RM, TB) \
    launch_shape<RM, TB>(num_tiles, row_splits, src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2, mode, prec, wk, s, vec, wvec, packed, fu)
    if (rm == 32) {
        if (batch_tile == 16) return PCB_SH(32, 16);
        if (batch_tile == 32) return PCB_SH(32, 32);
        return PCB_SH(32, 64);
    }
    if (batch_tile == 16) return PCB_SH(64, 16);
    if (batch_tile == 32) return PCB_SH(64, 32);
    return PCB_SH(64, 64);
#undef PCB_SH
}

extern "C" int pcb_lse_levels_short(float* node_mars, int64_t ld, int32_t B, const float* params,
                                    const PcbLseTile* tiles, const int32_t* krow, const int32_t* kw,
                                    const int32_t* term_children, const PcbShortLevel* levels, int32_t num_levels,
                                    int32_t total_items, int32_t num_slices, int32_t* counters, int32_t prec,
                                    int32_t batch_tile, int32_t wk, int32_t num_ctas, void* stream) {
    if (!node_mars || !params || !tiles || !krow || !kw || !term_children || !levels || !counters || B <= 0 ||
        ld < B || num_levels <= 0 || total_items < 0 || num_slices <= 0 || prec < 0 || prec > 2 ||
        (batch_tile != 16 && batch_tile != 32) || num_ctas <= 0 || (int64_t)num_slices * batch_tile < B)
        return pcb::set_error(PCB_E_ARG, "pcb_lse_levels_short: bad arguments");
    cudaStream_t s = pcb::as_stream(stream);
    cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(int32_t) * (size_t)(1 + num_slices), s);
    if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_lse_levels_short: %s", cudaGetErrorString(e));
    if (total_items == 0) return PCB_OK;
    const bool vec = pcb::vec_ok(node_mars, ld);
    const int ctas = num_ctas < total_items ? num_ctas : total_items;
#define PCB_LV(TBV, P, W) \
    launch_levels<TBV, P, W>(node_mars, ld, B, params, tiles, krow, kw, term_children, levels, num_levels, total_items, counters, ctas, s, vec)
    if (batch_tile == 16) {
        if (prec == 0) return wk ? PCB_LV(16, 0, true) : PCB_LV(16, 0, false);
        if (prec == 1) return wk ? PCB_LV(16, 1, true) : PCB_LV(16, 1, false);
        return wk ? PCB_LV(16, 2, true) : PCB_LV(16, 2, false);
    }
    if (prec == 0) return wk ? PCB_LV(32, 0, true) : PCB_LV(32, 0, false);
    if (prec == 1) return wk ? PCB_LV(32, 1, true) : PCB_LV(32, 1, false);
    return wk ? PCB_LV(32, 2, true) : PCB_LV(32, 2, false);
#undef PCB_LV
}
