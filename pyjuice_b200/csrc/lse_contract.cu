// Log-sum-exp contractions: sum-layer forward and element flows (plain FP32 path).
//
// One CTA computes a tile of up to TM output rows x TB samples:
//   acc[r, b] = sum_k W(k, r) * exp(src[krow[k], b] - m_b)
// where m_b is the running max over the contraction terms seen so far (online
// rescaling, one max per sample, shared by all rows of the tile). A tile spans several
// node blocks that share their children (a whole region of a structured circuit), so
// every staged child value is exponentiated once and reused by up to 128 output rows.
//   W(k, r) = params[kw[k] + w_add + (r >> rpb_log2) * g_stride + (r & (rpb - 1)) * w_stride]
//
// Terms are staged in chunks of KC with asynchronous copies (cp.async) into two shared
// buffers: the copies of chunk c + 1 are in flight while chunk c is reduced, so a CTA
// pays one memory latency per tile rather than one per staged value.
//
// Epilogues: mode 0 writes log(acc) + m (sum forward); modes 1/2 write
// acc * exp(aux + m) (element flows; mode 2 first turns node flows into log f - log m).
#include "lse_stage.cuh"

namespace {

template <int TM, int TB, int RN, int MODE>
__global__ void __launch_bounds__(TB / 4 * (TM / RN))
lse_f32_kernel(const float* __restrict__ src, const float* __restrict__ src2, const float* __restrict__ aux,
               float* __restrict__ out, int64_t ld, int B, const float* __restrict__ params,
               const PcbLseTile* __restrict__ tiles, const int* __restrict__ krow, const int* __restrict__ kw,
               int w_stride, int rpb_log2, bool vec) {
    pcb::pdl_begin();
    constexpr int NX = TB / 4;           // threads along the batch (4 samples each)
    constexpr int NY = TM / RN;          // threads along rows
    constexpr int NT = NX * NY;
    using St = pcb::LseStage<TM, TB, MODE == 2>;
    extern __shared__ __align__(16) unsigned char dsm[];
    St st(dsm);
    float* sMax = st.end();
    float* sScale = sMax + TB;

    const PcbLseTile t = tiles[blockIdx.x];
    const int b0 = blockIdx.y * TB;
    const int tid = threadIdx.x;
    const int tx = tid % NX;
    const int ty = tid / NX;

    for (int i = tid; i < TB; i += NT) sMax[i] = -INFINITY;

    float acc[RN][4];
#pragma unroll
    for (int r = 0; r < RN; ++r)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[r][j] = 0.f;

    const int nchunks = (t.k_cnt + pcb::kLseKC - 1) / pcb::kLseKC;
    st.template issue<NT>(0, 0, t, src, src2, params, krow, kw, ld, B, b0, w_stride, rpb_log2, vec, tid);
    for (int c = 0; c < nchunks; ++c) {
        const int s = c & 1;
        if (c + 1 < nchunks) {
            st.template issue<NT>(c + 1, s ^ 1, t, src, src2, params, krow, kw, ld, B, b0, w_stride, rpb_log2, vec, tid);
            pcb::cp_async_wait<1>();
        } else {
            pcb::cp_async_wait<0>();
        }
        __syncthreads();
        const int n = min(pcb::kLseKC, t.k_cnt - c * pcb::kLseKC);
        float (*sE)[TB] = st.E(s);
        float (*sW)[TM] = st.W(s);
        st.transform_and_max(s, n, sMax, sScale, tid, NT);
        __syncthreads();
        for (int idx = tid; idx < n * TB; idx += NT) {
            const int k = idx / TB;
            const int b = idx % TB;
            const float m = sMax[b];
            sE[k][b] = (m == -INFINITY) ? 0.f : __expf(sE[k][b] - m);
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float sc = sScale[tx * 4 + j];
#pragma unroll
            for (int r = 0; r < RN; ++r) acc[r][j] *= sc;
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

// Forward of tiles of one row (sum layers of block size 1, e.g. a root over thousands of
// children): out[row, b] = log sum_k w_k exp(src[krow[k], b]). Lane = sample (32 consecutive
// samples per CTA, coalesced rows), warp = every 32nd term; each thread keeps an online
// (max, scaled sum) over its terms, and the 32 warps' pairs are combined through shared
// memory. Weight of term k: params[kw[k_off + k] + w_add].
constexpr int kRowWarps = 32;

__global__ void __launch_bounds__(32 * kRowWarps)
lse_row_kernel(const float* __restrict__ src, float* __restrict__ out, int64_t ld, int B,
               const float* __restrict__ params, const PcbLseTile* __restrict__ tiles, const int* __restrict__ krow,
               const int* __restrict__ kw) {
    pcb::pdl_begin();
    __shared__ float sM[kRowWarps][32], sS[kRowWarps][32];
    const PcbLseTile t = tiles[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int b = blockIdx.y * 32 + lane;
    float m = -INFINITY, sum = 0.f;
    if (b < B) {
#pragma unroll 4
        for (int k = warp; k < t.k_cnt; k += kRowWarps) {
            const float e = __ldg(src + (int64_t)__ldg(krow + t.k_off + k) * ld + b);
            const float w = __ldg(params + (int64_t)__ldg(kw + t.k_off + k) + t.w_add);
            if (e == -INFINITY) continue;
            if (e > m) {
                sum = sum * expf(m - e) + w;
                m = e;
            } else {
                sum = fmaf(w, expf(e - m), sum);
            }
        }
    }
    sM[warp][lane] = m;
    sS[warp][lane] = sum;
    __syncthreads();
    if (warp == 0 && b < B && t.n_rows > 0) {
        float mm = -INFINITY;
#pragma unroll
        for (int w = 0; w < kRowWarps; ++w) mm = fmaxf(mm, sM[w][lane]);
        float ss = 0.f;
#pragma unroll
        for (int w = 0; w < kRowWarps; ++w)
            if (sM[w][lane] != -INFINITY) ss = fmaf(sS[w][lane], expf(sM[w][lane] - mm), ss);
        out[(int64_t)t.out_row * ld + b] = mm == -INFINITY ? -INFINITY : logf(ss) + mm;
    }
}

template <int TM, int TB, int RN, int MODE>
int launch_mode(dim3 grid, const float* src, const float* src2, const float* aux, float* out, int64_t ld, int B,
                const float* params, const PcbLseTile* tiles, const int* krow, const int* kw, int w_stride,
                int rpb_log2, cudaStream_t s, bool vec) {
    constexpr int threads = TB / 4 * (TM / RN);
    constexpr size_t smem = pcb::LseStage<TM, TB, MODE == 2>::bytes() + 2 * sizeof(float) * TB;
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    dev = dev < 0 ? 0 : (dev > 63 ? 63 : dev);
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(lse_f32_kernel<TM, TB, RN, MODE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_lse_contract: %s", cudaGetErrorString(e));
        configured[dev] = true;
    }
    return pcb::launch_status(pcb::launch_k(lse_f32_kernel<TM, TB, RN, MODE>, dim3(grid), dim3(threads), smem, s, 1u,
                                            src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2,
                                            vec), "pcb_lse_contract");
}

template <int TM, int TB, int RN>
int launch_cfg(const float* src, const float* src2, const float* aux, float* out, int64_t ld, int B,
               const float* params, const PcbLseTile* tiles, int num_tiles, const int* krow, const int* kw,
               int w_stride, int rpb_log2, int mode, cudaStream_t s, bool vec) {
    dim3 grid((unsigned)num_tiles, (unsigned)pcb::cdiv(B, TB));
    if (grid.y > 65535) return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: batch too large");
    if (mode == 0) return launch_mode<TM, TB, RN, 0>(grid, src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2, s, vec);
    if (mode == 1) return launch_mode<TM, TB, RN, 1>(grid, src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2, s, vec);
    return launch_mode<TM, TB, RN, 2>(grid, src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2, s, vec);
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
    if (tile_rows == 1 && mode == 0) {
        const dim3 grid((unsigned)num_tiles, (unsigned)pcb::cdiv(B, 32));
        if (grid.y > 65535) return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: batch too large");
        return pcb::launch_status(pcb::launch_k(lse_row_kernel, grid, dim3(32 * kRowWarps), 0, s, 1u, src, out, ld,
                                                B, params, tiles, krow, kw), "pcb_lse_contract");
    }
    const bool vec = pcb::vec_ok(src, ld) && pcb::vec_ok(out, ld) && (!aux || pcb::vec_ok(aux, ld)) &&
                     (!src2 || pcb::vec_ok(src2, ld));
#define PCB_LSE(TM, TB, RN) launch_cfg<TM, TB, RN>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, rpb_log2, mode, s, vec)
    switch (tile_rows) {
        case 1: return PCB_LSE(1, 128, 1);
        case 2: return PCB_LSE(2, 128, 1);
        case 4: return PCB_LSE(4, 128, 1);
        case 8: return PCB_LSE(8, 128, 1);
        case 16: return PCB_LSE(16, 128, 2);
        case 32: return PCB_LSE(32, 128, 4);
        case 64: return PCB_LSE(64, 64, 4);
        case 128: return PCB_LSE(128, 32, 4);
        default:
            return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: tile_rows must be a power of 2 <= 128, got %d", tile_rows);
    }
#undef PCB_LSE
}
