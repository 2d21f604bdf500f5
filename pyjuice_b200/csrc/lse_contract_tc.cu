// BF16 tensor-core form of the log-sum-exp contraction (see lse_contract.cu).
//
// Same tiles and online-max scheme as the FP32 kernel; each staged chunk is contracted on
// the tensor cores: A = W (rows x K, rounded to bf16), B = exp(src - m) (K x samples,
// rounded to bf16), FP32 accumulators; max / exp / log stay in FP32.
// Operands are kept in shared memory as packed bf16 pairs along K, so every mma fragment
// register is one 32-bit shared load. Tile: TM (16..128) rows x 128 samples, 8 warps:
// TM/16 warps along the rows, the rest along the samples.
//
// SPLIT: each operand x is held as hi = bf16(x) plus lo = bf16(x - hi) and the product is
// accumulated as hi*hi + lo*hi + hi*lo (three bf16 MMAs). This keeps the contraction on
// the bf16 tensor cores while removing the bf16 rounding of the weights, whose per-node
// sums would otherwise drift from one and bias every sample's log-likelihood the same way.
#include <cuda_bf16.h>

#include "common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int TB = 128;
constexpr int KC = 32;

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

__device__ __forceinline__ void split_bf16(float lo_k, float hi_k, uint32_t& h, uint32_t& l) {
    __nv_bfloat162 hv = __floats2bfloat162_rn(lo_k, hi_k);
    const float2 hf = __bfloat1622float2(hv);
    __nv_bfloat162 lv = __floats2bfloat162_rn(lo_k - hf.x, hi_k - hf.y);
    h = *reinterpret_cast<uint32_t*>(&hv);
    l = *reinterpret_cast<uint32_t*>(&lv);
}

template <int TM, int MODE, bool SPLIT>
__global__ void __launch_bounds__(kThreads)
lse_bf16_kernel(const float* __restrict__ src, const float* __restrict__ src2, const float* __restrict__ aux,
                float* __restrict__ out, int64_t ld, int B, const float* __restrict__ params,
                const PcbLseTile* __restrict__ tiles, const int* __restrict__ krow, const int* __restrict__ kw,
                int w_stride, int rpb_log2, bool vec) {
    constexpr int WM = TM / 16;          // warps along rows
    constexpr int WN = 8 / WM;           // warps along samples
    constexpr int NT = TB / 8 / WN;      // n8 tiles per warp
    constexpr int ES = TB + 8;           // packed row strides (conflict-free fragment loads)
    constexpr int WS = TM + 8;
    extern __shared__ __align__(16) unsigned char dsm[];
    float (*sE)[TB] = reinterpret_cast<float (*)[TB]>(dsm);
    uint32_t (*sE2)[ES] = reinterpret_cast<uint32_t (*)[ES]>(dsm + sizeof(float) * KC * TB);
    uint32_t (*sW2)[WS] = reinterpret_cast<uint32_t (*)[WS]>(reinterpret_cast<unsigned char*>(sE2) + 4 * (KC / 2) * ES);
    uint32_t (*sE2l)[ES] = reinterpret_cast<uint32_t (*)[ES]>(reinterpret_cast<unsigned char*>(sW2) + 4 * (KC / 2) * WS);
    uint32_t (*sW2l)[WS] = reinterpret_cast<uint32_t (*)[WS]>(reinterpret_cast<unsigned char*>(sE2l) + (SPLIT ? 4 * (KC / 2) * ES : 0));
    float* sMax = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(sW2l) + (SPLIT ? 4 * (KC / 2) * WS : 0));
    float* sScale = sMax + TB;

    const PcbLseTile t = tiles[blockIdx.x];
    const int b0 = blockIdx.y * TB;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int g = lane >> 2;
    const int q = lane & 3;
    const int wm = warp % WM;
    const int wn = warp / WM;
    const int m0 = wm * 16;
    const int nb = wn * (TB / WN);
    const int rpb_mask = (1 << rpb_log2) - 1;

    for (int i = tid; i < TB; i += kThreads) sMax[i] = -INFINITY;

    float acc[NT][4];
#pragma unroll
    for (int a = 0; a < NT; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] = 0.f;

    for (int kc = 0; kc < t.k_cnt; kc += KC) {
        const int n = min(KC, t.k_cnt - kc);
        for (int idx = tid; idx < KC * (TB / 4); idx += kThreads) {
            const int k = idx / (TB / 4);
            const int c4 = idx % (TB / 4);
            float4 v = make_float4(-INFINITY, -INFINITY, -INFINITY, -INFINITY);
            if (k < n) {
                const int row = krow[t.k_off + kc + k];
                v = pcb::load4(src, row, ld, b0 + c4 * 4, B, vec, -INFINITY);
                if (MODE == 2) {
                    const float4 m = pcb::load4(src2, row, ld, b0 + c4 * 4, B, vec, -INFINITY);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float mm = pcb::get(m, j);
                        pcb::set(v, j, (mm == -INFINITY) ? -INFINITY : logf(pcb::get(v, j)) - mm);
                    }
                }
            }
            *reinterpret_cast<float4*>(&sE[k][c4 * 4]) = v;
        }
        // weights, packed along K: sW2[k/2][r] = (W(k, r), W(k + 1, r))
        for (int idx = tid; idx < (KC / 2) * TM; idx += kThreads) {
            const int kk = idx / TM;
            const int r = idx % TM;
            float w0 = 0.f, w1 = 0.f;
            if (r < t.n_rows) {
                const int64_t roff = (int64_t)t.w_add + (int64_t)(r >> rpb_log2) * t.g_stride +
                                     (int64_t)(r & rpb_mask) * w_stride;
                if (2 * kk < n) w0 = __ldg(params + (int64_t)kw[t.k_off + kc + 2 * kk] + roff);
                if (2 * kk + 1 < n) w1 = __ldg(params + (int64_t)kw[t.k_off + kc + 2 * kk + 1] + roff);
            }
            if (SPLIT) split_bf16(w0, w1, sW2[kk][r], sW2l[kk][r]);
            else sW2[kk][r] = pack_bf16(w0, w1);
        }
        __syncthreads();
        for (int b = tid; b < TB; b += kThreads) {
            float cm = -INFINITY;
            for (int k = 0; k < n; ++k) cm = fmaxf(cm, sE[k][b]);
            const float old = sMax[b];
            const float nm = fmaxf(old, cm);
            sScale[b] = (nm == -INFINITY) ? 1.f : __expf(old - nm);
            sMax[b] = nm;
        }
        __syncthreads();
        for (int idx = tid; idx < (KC / 2) * TB; idx += kThreads) {
            const int kk = idx / TB;
            const int b = idx % TB;
            const float m = sMax[b];
            float e0 = 0.f, e1 = 0.f;
            if (m != -INFINITY) {
                if (2 * kk < n) e0 = __expf(sE[2 * kk][b] - m);
                if (2 * kk + 1 < n) e1 = __expf(sE[2 * kk + 1][b] - m);
            }
            if (SPLIT) split_bf16(e0, e1, sE2[kk][b], sE2l[kk][b]);
            else sE2[kk][b] = pack_bf16(e0, e1);
        }
        __syncthreads();
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const float s0 = sScale[nb + nt * 8 + 2 * q];
            const float s1 = sScale[nb + nt * 8 + 2 * q + 1];
            acc[nt][0] *= s0;
            acc[nt][1] *= s1;
            acc[nt][2] *= s0;
            acc[nt][3] *= s1;
        }
        const int kend = (n + 15) & ~15;
        for (int k0 = 0; k0 < kend; k0 += 16) {
            const int kk = k0 >> 1;
            const uint32_t a0 = sW2[kk + q][m0 + g];
            const uint32_t a1 = sW2[kk + q][m0 + g + 8];
            const uint32_t a2 = sW2[kk + 4 + q][m0 + g];
            const uint32_t a3 = sW2[kk + 4 + q][m0 + g + 8];
            if (SPLIT) {
                const uint32_t l0 = sW2l[kk + q][m0 + g];
                const uint32_t l1 = sW2l[kk + q][m0 + g + 8];
                const uint32_t l2 = sW2l[kk + 4 + q][m0 + g];
                const uint32_t l3 = sW2l[kk + 4 + q][m0 + g + 8];
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) {
                    const int col = nb + nt * 8 + g;
                    const uint32_t bh0 = sE2[kk + q][col], bh1 = sE2[kk + 4 + q][col];
                    mma_bf16(acc[nt], a0, a1, a2, a3, bh0, bh1);
                    mma_bf16(acc[nt], l0, l1, l2, l3, bh0, bh1);
                    mma_bf16(acc[nt], a0, a1, a2, a3, sE2l[kk + q][col], sE2l[kk + 4 + q][col]);
                }
            } else {
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) {
                    const int col = nb + nt * 8 + g;
                    mma_bf16(acc[nt], a0, a1, a2, a3, sE2[kk + q][col], sE2[kk + 4 + q][col]);
                }
            }
        }
        __syncthreads();
    }

#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int row = m0 + g + h * 8;
        if (row >= t.n_rows) continue;
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int col = nb + nt * 8 + 2 * q + j;
                const int b = b0 + col;
                if (b >= B) continue;
                const float m = sMax[col];
                const float v = acc[nt][h * 2 + j];
                float o;
                if (MODE == 0) {
                    o = (m == -INFINITY) ? -INFINITY : logf(v) + m;
                } else {
                    const float x = __ldg(aux + ((int64_t)t.aux_row + row) * ld + b);
                    o = (m == -INFINITY) ? 0.f : v * __expf(x + m);
                }
                out[((int64_t)t.out_row + row) * ld + b] = o;
            }
        }
    }
}

template <int TM, int MODE, bool SPLIT>
int launch_one(dim3 grid, const float* src, const float* src2, const float* aux, float* out, int64_t ld, int B,
               const float* params, const PcbLseTile* tiles, const int* krow, const int* kw, int w_stride,
               int rpb_log2, cudaStream_t s, bool vec) {
    constexpr int ES = TB + 8, WS = TM + 8;
    constexpr size_t smem = sizeof(float) * KC * TB + 4 * (KC / 2) * (ES + WS) * (SPLIT ? 2 : 1) + 2 * sizeof(float) * TB;
    static bool configured = false;  // per instantiation; the attribute is per function, not per device state
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(lse_bf16_kernel<TM, MODE, SPLIT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_lse_contract(bf16): %s", cudaGetErrorString(e));
        configured = true;
    }
    lse_bf16_kernel<TM, MODE, SPLIT><<<grid, kThreads, smem, s>>>(src, src2, aux, out, ld, B, params, tiles, krow, kw,
                                                                  w_stride, rpb_log2, vec);
    return pcb::check_launch("pcb_lse_contract(bf16)");
}

template <int TM>
int launch(const float* src, const float* src2, const float* aux, float* out, int64_t ld, int B, const float* params,
           const PcbLseTile* tiles, int num_tiles, const int* krow, const int* kw, int w_stride, int rpb_log2,
           int mode, bool split, cudaStream_t s, bool vec) {
    dim3 grid((unsigned)num_tiles, (unsigned)pcb::cdiv(B, TB));
    if (grid.y > 65535) return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: batch too large");
#define PCB_L1(M, S) launch_one<TM, M, S>(grid, src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2, s, vec)
    if (split) {
        if (mode == 0) return PCB_L1(0, true);
        if (mode == 1) return PCB_L1(1, true);
        return PCB_L1(2, true);
    }
    if (mode == 0) return PCB_L1(0, false);
    if (mode == 1) return PCB_L1(1, false);
    return PCB_L1(2, false);
#undef PCB_L1
}

}  // namespace

int pcb_lse_contract_bf16(const float* src, const float* src2, const float* aux, float* out, int64_t ld, int B,
                          const float* params, const PcbLseTile* tiles, int num_tiles, int tile_rows, int rpb_log2,
                          const int* krow, const int* kw, int w_stride, int mode, bool split, cudaStream_t s) {
    const bool vec = pcb::vec_ok(src, ld) && (!src2 || pcb::vec_ok(src2, ld));
    switch (tile_rows) {
        case 16: return launch<16>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, rpb_log2, mode, split, s, vec);
        case 32: return launch<32>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, rpb_log2, mode, split, s, vec);
        case 64: return launch<64>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, rpb_log2, mode, split, s, vec);
        case 128: return launch<128>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, rpb_log2, mode, split, s, vec);
        default:
            return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: the bf16 form needs tile_rows 16..128, got %d", tile_rows);
    }
}
