// Log-sum-exp contractions: sum-layer forward and element flows (plain FP32 path).
//
// One CTA computes a tile of up to TM output rows x TB samples:
//   acc[r, b] = sum_k W(k, r) * exp(src[krow[k], b] - m_b)
// where m_b is the running max over the contraction terms seen so far (online
// rescaling, one max per sample, shared by all rows of the tile). A tile spans several
// node blocks that share their children (a whole region of a structured circuit), so
// every staged child value is exponentiated once and reused by up to 128 output rows.
// Terms are staged in shared memory in chunks of KC rows.
//   W(k, r) = params[kw[k] + w_add + (r >> rpb_log2) * g_stride + (r & (rpb - 1)) * w_stride]
//
// Epilogues: mode 0 writes log(acc) + m (sum forward); modes 1/2 write
// acc * exp(aux + m) (element flows; mode 2 first turns node flows into log f - log m).
#include "common.cuh"

namespace {

constexpr int kThreads = 256;

template <int TM, int TB, int KC, int MODE>
__global__ void __launch_bounds__(kThreads)
lse_f32_kernel(const float* __restrict__ src, const float* __restrict__ src2, const float* __restrict__ aux,
               float* __restrict__ out, int64_t ld, int B, const float* __restrict__ params,
               const PcbLseTile* __restrict__ tiles, const int* __restrict__ krow, const int* __restrict__ kw,
               int w_stride, int rpb_log2, bool vec) {
    constexpr int NX = TB / 4;           // threads along the batch (4 samples each)
    constexpr int NY = kThreads / NX;    // threads along rows
    constexpr int RN = TM / NY;          // rows per thread
    static_assert(NY * RN == TM && RN >= 1, "tile shape");

    __shared__ __align__(16) float sE[KC][TB];
    __shared__ __align__(16) float sW[KC][TM];
    __shared__ float sMax[TB];
    __shared__ float sScale[TB];

    const PcbLseTile t = tiles[blockIdx.x];
    const int b0 = blockIdx.y * TB;
    const int tid = threadIdx.x;
    const int tx = tid % NX;
    const int ty = tid / NX;
    const int rpb_mask = (1 << rpb_log2) - 1;

    for (int i = tid; i < TB; i += kThreads) sMax[i] = -INFINITY;

    float acc[RN][4];
#pragma unroll
    for (int r = 0; r < RN; ++r)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[r][j] = 0.f;

    for (int kc = 0; kc < t.k_cnt; kc += KC) {
        const int n = min(KC, t.k_cnt - kc);
        for (int idx = tid; idx < KC * NX; idx += kThreads) {
            const int k = idx / NX;
            const int c4 = idx % NX;
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
        for (int idx = tid; idx < KC * TM; idx += kThreads) {
            const int k = idx / TM;
            const int r = idx % TM;
            float w = 0.f;
            if (k < n && r < t.n_rows) {
                const int64_t wi = (int64_t)kw[t.k_off + kc + k] + t.w_add + (int64_t)(r >> rpb_log2) * t.g_stride +
                                   (int64_t)(r & rpb_mask) * w_stride;
                w = __ldg(params + wi);
            }
            sW[k][r] = w;
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
        for (int idx = tid; idx < n * TB; idx += kThreads) {
            const int k = idx / TB;
            const int b = idx % TB;
            const float m = sMax[b];
            sE[k][b] = (m == -INFINITY) ? 0.f : __expf(sE[k][b] - m);
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float s = sScale[tx * 4 + j];
#pragma unroll
            for (int r = 0; r < RN; ++r) acc[r][j] *= s;
        }
        for (int k = 0; k < n; ++k) {
            const float4 e = *reinterpret_cast<const float4*>(&sE[k][tx * 4]);
            float w[RN];
            if constexpr (RN % 4 == 0) {
#pragma unroll
                for (int r4 = 0; r4 < RN / 4; ++r4) {
                    const float4 wv = *reinterpret_cast<const float4*>(&sW[k][ty * RN + r4 * 4]);
                    w[r4 * 4 + 0] = wv.x; w[r4 * 4 + 1] = wv.y; w[r4 * 4 + 2] = wv.z; w[r4 * 4 + 3] = wv.w;
                }
            } else {
#pragma unroll
                for (int r = 0; r < RN; ++r) w[r] = sW[k][ty * RN + r];
            }
#pragma unroll
            for (int r = 0; r < RN; ++r) {
                acc[r][0] = fmaf(w[r], e.x, acc[r][0]);
                acc[r][1] = fmaf(w[r], e.y, acc[r][1]);
                acc[r][2] = fmaf(w[r], e.z, acc[r][2]);
                acc[r][3] = fmaf(w[r], e.w, acc[r][3]);
            }
        }
        __syncthreads();
    }

    const int bb = b0 + tx * 4;
#pragma unroll
    for (int r = 0; r < RN; ++r) {
        const int row = ty * RN + r;
        if (row >= t.n_rows) continue;
        float4 o;
        if (MODE == 0) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float m = sMax[tx * 4 + j];
                pcb::set(o, j, (m == -INFINITY) ? -INFINITY : logf(acc[r][j]) + m);
            }
        } else {
            const float4 a = pcb::load4(aux, (int64_t)t.aux_row + row, ld, bb, B, vec, 0.f);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float m = sMax[tx * 4 + j];
                pcb::set(o, j, (m == -INFINITY) ? 0.f : acc[r][j] * __expf(pcb::get(a, j) + m));
            }
        }
        pcb::store4(out, (int64_t)t.out_row + row, ld, bb, B, vec, o);
    }
}

template <int TM, int TB, int KC>
int launch_cfg(const float* src, const float* src2, const float* aux, float* out, int64_t ld, int B,
               const float* params, const PcbLseTile* tiles, int num_tiles, const int* krow, const int* kw,
               int w_stride, int rpb_log2, int mode, cudaStream_t s, bool vec) {
    dim3 grid((unsigned)num_tiles, (unsigned)pcb::cdiv(B, TB));
    if (grid.y > 65535) return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: batch too large");
    if (mode == 0)
        lse_f32_kernel<TM, TB, KC, 0><<<grid, kThreads, 0, s>>>(src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2, vec);
    else if (mode == 1)
        lse_f32_kernel<TM, TB, KC, 1><<<grid, kThreads, 0, s>>>(src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2, vec);
    else
        lse_f32_kernel<TM, TB, KC, 2><<<grid, kThreads, 0, s>>>(src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2, vec);
    return pcb::check_launch("pcb_lse_contract");
}

int ilog2(int v) {
    int l = 0;
    while ((1 << l) < v) ++l;
    return (1 << l) == v ? l : -1;
}

}  // namespace

// Tensor-core (BF16) variant, defined in lse_contract_tc.cu.
int pcb_lse_contract_bf16(const float* src, const float* src2, const float* aux, float* out, int64_t ld, int B,
                          const float* params, const PcbLseTile* tiles, int num_tiles, int tile_rows, int rpb_log2,
                          const int* krow, const int* kw, int w_stride, int mode, bool split, cudaStream_t s);

extern "C" int pcb_lse_contract(const float* src, const float* src2, const float* aux, float* out, int64_t ld,
                                int32_t B, const float* params, const PcbLseTile* tiles, int32_t num_tiles,
                                int32_t tile_rows, int32_t rows_per_block, const int32_t* krow, const int32_t* kw,
                                int32_t w_stride, int32_t mode, int32_t prec, void* stream) {
    if (!src || !out || !params || !tiles || !krow || !kw || B <= 0 || ld < B || num_tiles < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: bad arguments");
    if (mode < 0 || mode > 2 || (mode >= 1 && !aux) || (mode == 2 && !src2))
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: bad mode %d", mode);
    const int rpb_log2 = ilog2(rows_per_block);
    if (rpb_log2 < 0) return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: rows_per_block must be a power of 2");
    if (num_tiles == 0) return PCB_OK;
    cudaStream_t s = pcb::as_stream(stream);
    if (prec == 1 || prec == 2) {
        return pcb_lse_contract_bf16(src, src2, aux, out, ld, B, params, tiles, num_tiles, tile_rows, rpb_log2, krow, kw,
                                     w_stride, mode, prec == 2, s);
    }
    if (prec != 0) return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: prec must be 0, 1 or 2");
    const bool vec = pcb::vec_ok(src, ld) && pcb::vec_ok(out, ld) && (!aux || pcb::vec_ok(aux, ld)) &&
                     (!src2 || pcb::vec_ok(src2, ld));
#define PCB_LSE(TM, TB, KC) launch_cfg<TM, TB, KC>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, rpb_log2, mode, s, vec)
    switch (tile_rows) {
        case 1: return PCB_LSE(1, 1024, 8);
        case 2: return PCB_LSE(2, 1024, 8);
        case 4: return PCB_LSE(4, 1024, 8);
        case 8: return PCB_LSE(8, 512, 16);
        case 16: return PCB_LSE(16, 256, 32);
        case 32: return PCB_LSE(32, 128, 64);
        case 64: return PCB_LSE(64, 128, 32);
        case 128: return PCB_LSE(128, 128, 32);
        default:
            return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: tile_rows must be a power of 2 <= 128, got %d", tile_rows);
    }
#undef PCB_LSE
}
