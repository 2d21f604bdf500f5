// Log-sum-exp contractions: sum-layer forward and element flows (plain FP32 path).
//
// One CTA computes a tile of `TM` output rows x `TB` samples:
//   acc[r, b] = sum_k W(k, r) * exp(src[krow[k], b] - m_b)
// where m_b is the running max over the contraction terms seen so far (online
// rescaling, one max per sample, shared by all rows of the tile). Terms are staged in
// shared memory in chunks of KC rows; each staged value is exponentiated once and
// reused by all TM output rows. Weights W(k, r) = params[kw[k] + w_add + r * w_stride].
//
// Epilogues: mode 0 writes log(acc) + m (sum forward); modes 1/2 write
// acc * exp(aux + m) (element flows; mode 2 first turns node flows into log f - log m).
#include "common.cuh"

namespace {

constexpr int kThreads = 256;

template <int TM, int RN, int MODE>
__global__ void __launch_bounds__(kThreads)
lse_f32_kernel(const float* __restrict__ src, const float* __restrict__ src2, const float* __restrict__ aux,
               float* __restrict__ out, int64_t ld, int B, const float* __restrict__ params,
               const PcbLseTile* __restrict__ tiles, const int* __restrict__ krow, const int* __restrict__ kw,
               int w_stride, bool vec) {
    constexpr int TB = 4 * kThreads * RN / TM;  // samples per CTA
    constexpr int NX = TB / 4;                  // threads along the batch (4 samples each)
    constexpr int NY = kThreads / NX;           // threads along rows (RN rows each)
    static_assert(NY * RN == TM, "tile shape");
    constexpr int KC = 8192 / TB;               // contraction terms per staged chunk

    __shared__ __align__(16) float sE[KC][TB];
    __shared__ __align__(16) float sW[KC][TM];
    __shared__ float sMax[TB];
    __shared__ float sScale[TB];

    const PcbLseTile t = tiles[blockIdx.x];
    const int b0 = blockIdx.y * TB;
    const int tid = threadIdx.x;
    const int tx = tid % NX;
    const int ty = tid / NX;

    for (int i = tid; i < TB; i += kThreads) sMax[i] = -INFINITY;

    float acc[RN][4];
#pragma unroll
    for (int r = 0; r < RN; ++r)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[r][j] = 0.f;

    for (int kc = 0; kc < t.k_cnt; kc += KC) {
        const int n = min(KC, t.k_cnt - kc);
        // Stage the source rows of this chunk.
        for (int idx = tid; idx < KC * NX; idx += kThreads) {
            const int k = idx / NX;
            const int c4 = idx % NX;
            float4 v = make_float4(-INFINITY, -INFINITY, -INFINITY, -INFINITY);
            if (k < n) {
                const int row = krow[t.k_off + kc + k];
                v = pcb::load4(src, row, ld, b0 + c4 * 4, B, vec, -INFINITY);
                if (MODE == 2) {
                    float4 m = pcb::load4(src2, row, ld, b0 + c4 * 4, B, vec, -INFINITY);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        float mm = pcb::get(m, j);
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
            if (k < n && r < t.n_rows) w = __ldg(params + (int64_t)kw[t.k_off + kc + k] + t.w_add + (int64_t)r * w_stride);
            sW[k][r] = w;
        }
        __syncthreads();
        // Per-sample running max and rescale factor.
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
            const float v = sE[k][b];
            sE[k][b] = (m == -INFINITY) ? 0.f : __expf(v - m);
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
#pragma unroll
            for (int r = 0; r < RN; ++r) w[r] = sW[k][ty * RN + r];
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

template <int TM, int RN>
int launch_tm(const float* src, const float* src2, const float* aux, float* out, int64_t ld, int B,
              const float* params, const PcbLseTile* tiles, int num_tiles, const int* krow, const int* kw,
              int w_stride, int mode, cudaStream_t s, bool vec) {
    constexpr int TB = 4 * kThreads * RN / TM;
    dim3 grid((unsigned)num_tiles, (unsigned)pcb::cdiv(B, TB));
    if (mode == 0)
        lse_f32_kernel<TM, RN, 0><<<grid, kThreads, 0, s>>>(src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, vec);
    else if (mode == 1)
        lse_f32_kernel<TM, RN, 1><<<grid, kThreads, 0, s>>>(src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, vec);
    else
        lse_f32_kernel<TM, RN, 2><<<grid, kThreads, 0, s>>>(src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, vec);
    return pcb::check_launch("pcb_lse_contract");
}

}  // namespace

// Tensor-core (BF16) variant, defined in lse_contract_tc.cu.
int pcb_lse_contract_bf16(const float* src, const float* src2, const float* aux, float* out, int64_t ld, int B,
                          const float* params, const PcbLseTile* tiles, int num_tiles, int tile_rows,
                          const int* krow, const int* kw, int w_stride, int mode, cudaStream_t s);

extern "C" int pcb_lse_contract(const float* src, const float* src2, const float* aux, float* out, int64_t ld,
                                int32_t B, const float* params, const PcbLseTile* tiles, int32_t num_tiles,
                                int32_t tile_rows, const int32_t* krow, const int32_t* kw, int32_t w_stride,
                                int32_t mode, int32_t prec, void* stream) {
    if (!src || !out || !params || !tiles || !krow || !kw || B <= 0 || ld < B || num_tiles < 0)
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: bad arguments");
    if (mode < 0 || mode > 2 || (mode >= 1 && !aux) || (mode == 2 && !src2))
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: bad mode %d", mode);
    if (num_tiles == 0) return PCB_OK;
    if (num_tiles > 2147483647 || pcb::cdiv(B, 128) > 65535)
        return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: grid too large");
    cudaStream_t s = pcb::as_stream(stream);
    if (prec == 1) {
        return pcb_lse_contract_bf16(src, src2, aux, out, ld, B, params, tiles, num_tiles, tile_rows, krow, kw,
                                     w_stride, mode, s);
    }
    const bool vec = pcb::vec_ok(src, ld) && pcb::vec_ok(out, ld) && (!aux || pcb::vec_ok(aux, ld)) &&
                     (!src2 || pcb::vec_ok(src2, ld));
    switch (tile_rows) {
        case 1: return launch_tm<1, 1>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, mode, s, vec);
        case 2: return launch_tm<2, 2>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, mode, s, vec);
        case 4: return launch_tm<4, 4>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, mode, s, vec);
        case 8: return launch_tm<8, 4>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, mode, s, vec);
        case 16: return launch_tm<16, 4>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, mode, s, vec);
        case 32: return launch_tm<32, 4>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, mode, s, vec);
        default: return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: tile_rows must be a power of 2 <= 32, got %d", tile_rows);
    }
}
