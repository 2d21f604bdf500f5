// BF16 tensor-core form of the log-sum-exp contraction (see lse_contract.cu).
//
// Same tiles, asynchronous double-buffered staging (lse_stage.cuh) and online-max scheme
// as the FP32 kernel; each staged chunk is contracted on the tensor cores: A = W (rows x K)
// and B = exp(src - m) (K x samples) in bf16, FP32 accumulators; max / exp / log stay in
// FP32. Operands are repacked in shared memory as bf16 pairs along K, so every mma
// fragment register is one 32-bit shared load. 8 warps: TM/16 along the rows, the rest
// along the samples.
//
// SPLIT: each operand x is held as hi = bf16(x) plus lo = bf16(x - hi) and the product is
// accumulated as hi*hi + lo*hi + hi*lo (three bf16 MMAs). This keeps the contraction on
// the bf16 tensor cores while removing the bf16 rounding of the weights, whose per-node
// sums would otherwise drift from one and bias every sample's log-likelihood the same way.
#include <cuda_bf16.h>

#include "lse_stage.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int KC = pcb::kLseKC;

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

template <int TM, int TB, bool SPLIT>
struct Packed {
    static constexpr int ES = TB + 8;  // packed row strides: conflict-free fragment loads
    static constexpr int WS = TM + 8;
    static constexpr int NB = SPLIT ? 2 : 1;
    static constexpr size_t bytes() { return 4ull * (KC / 2) * (ES + WS) * NB; }
    uint32_t* p;
    __device__ explicit Packed(float* base) : p(reinterpret_cast<uint32_t*>(base)) {}
    __device__ uint32_t (*E(int h))[ES] { return reinterpret_cast<uint32_t(*)[ES]>(p + h * (KC / 2) * ES); }
    __device__ uint32_t (*W(int h))[WS] {
        return reinterpret_cast<uint32_t(*)[WS]>(p + NB * (KC / 2) * ES + h * (KC / 2) * WS);
    }
    __device__ float* end() { return reinterpret_cast<float*>(p + NB * (KC / 2) * (ES + WS)); }
};

template <int TM, int TB, int MODE, bool SPLIT>
__global__ void __launch_bounds__(kThreads)
lse_bf16_kernel(const float* __restrict__ src, const float* __restrict__ src2, const float* __restrict__ aux,
                float* __restrict__ out, int64_t ld, int B, const float* __restrict__ params,
                const PcbLseTile* __restrict__ tiles, const int* __restrict__ krow, const int* __restrict__ kw,
                int w_stride, int rpb_log2, bool vec) {
    pcb::pdl_begin();
    constexpr int WM = TM / 16;          // warps along rows
    constexpr int WN = 8 / WM;           // warps along samples
    constexpr int NT = TB / 8 / WN;      // n8 tiles per warp
    using St = pcb::LseStage<TM, TB, MODE == 2>;
    using Pk = Packed<TM, TB, SPLIT>;
    extern __shared__ __align__(16) unsigned char dsm[];
    St st(dsm);
    Pk pk(st.end());
    float* sMax = pk.end();
    float* sScale = sMax + TB;

    const PcbLseTile t = tiles[blockIdx.x];
    const int b0 = blockIdx.y * TB;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int g = lane >> 2;
    const int q = lane & 3;
    const int m0 = (warp % WM) * 16;
    const int nb = (warp / WM) * (TB / WN);

    for (int i = tid; i < TB; i += kThreads) sMax[i] = -INFINITY;

    float acc[NT][4];
#pragma unroll
    for (int a = 0; a < NT; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] = 0.f;

    const int nchunks = (t.k_cnt + KC - 1) / KC;
    st.template issue<kThreads>(0, 0, t, src, src2, params, krow, kw, ld, B, b0, w_stride, rpb_log2, vec, tid);
    for (int c = 0; c < nchunks; ++c) {
        const int s = c & 1;
        if (c + 1 < nchunks) {
            st.template issue<kThreads>(c + 1, s ^ 1, t, src, src2, params, krow, kw, ld, B, b0, w_stride, rpb_log2,
                                        vec, tid);
            pcb::cp_async_wait<1>();
        } else {
            pcb::cp_async_wait<0>();
        }
        __syncthreads();
        const int n = min(KC, t.k_cnt - c * KC);
        float(*sE)[TB] = st.E(s);
        float(*sW)[TM] = st.W(s);
        st.transform_and_max(s, n, sMax, sScale, tid, kThreads);
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
            if (SPLIT) split_bf16(e0, e1, pk.E(0)[kk][b], pk.E(1)[kk][b]);
            else pk.E(0)[kk][b] = pack_bf16(e0, e1);
        }
        for (int idx = tid; idx < (KC / 2) * TM; idx += kThreads) {
            const int kk = idx / TM;
            const int r = idx % TM;
            const float w0 = sW[2 * kk][r];
            const float w1 = sW[2 * kk + 1][r];
            if (SPLIT) split_bf16(w0, w1, pk.W(0)[kk][r], pk.W(1)[kk][r]);
            else pk.W(0)[kk][r] = pack_bf16(w0, w1);
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
            const uint32_t a0 = pk.W(0)[kk + q][m0 + g];
            const uint32_t a1 = pk.W(0)[kk + q][m0 + g + 8];
            const uint32_t a2 = pk.W(0)[kk + 4 + q][m0 + g];
            const uint32_t a3 = pk.W(0)[kk + 4 + q][m0 + g + 8];
            if (SPLIT) {
                const uint32_t l0 = pk.W(1)[kk + q][m0 + g];
                const uint32_t l1 = pk.W(1)[kk + q][m0 + g + 8];
                const uint32_t l2 = pk.W(1)[kk + 4 + q][m0 + g];
                const uint32_t l3 = pk.W(1)[kk + 4 + q][m0 + g + 8];
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) {
                    const int col = nb + nt * 8 + g;
                    const uint32_t bh0 = pk.E(0)[kk + q][col], bh1 = pk.E(0)[kk + 4 + q][col];
                    mma_bf16(acc[nt], a0, a1, a2, a3, bh0, bh1);
                    mma_bf16(acc[nt], l0, l1, l2, l3, bh0, bh1);
                    mma_bf16(acc[nt], a0, a1, a2, a3, pk.E(1)[kk + q][col], pk.E(1)[kk + 4 + q][col]);
                }
            } else {
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) {
                    const int col = nb + nt * 8 + g;
                    mma_bf16(acc[nt], a0, a1, a2, a3, pk.E(0)[kk + q][col], pk.E(0)[kk + 4 + q][col]);
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
            const int col = nb + nt * 8 + 2 * q;
            const int b = b0 + col;
            float o[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const float m = sMax[col + j];
                const float v = acc[nt][h * 2 + j];
                if (MODE == 0) {
                    o[j] = (m == -INFINITY) ? -INFINITY : logf(v) + m;
                } else {
                    const float x = (b + j < B) ? __ldg(aux + ((int64_t)t.aux_row + row) * ld + b + j) : 0.f;
                    o[j] = (m == -INFINITY) ? 0.f : v * __expf(x + m);
                }
            }
            float* dst = out + ((int64_t)t.out_row + row) * ld + b;
            if (vec && b + 1 < B) {
                *reinterpret_cast<float2*>(dst) = make_float2(o[0], o[1]);
            } else {
                if (b < B) dst[0] = o[0];
                if (b + 1 < B) dst[1] = o[1];
            }
        }
    }
}

int current_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d < 0 ? 0 : (d > 63 ? 63 : d);
}

template <int TM, int TB, int MODE, bool SPLIT>
int launch_one(dim3 grid, const float* src, const float* src2, const float* aux, float* out, int64_t ld, int B,
               const float* params, const PcbLseTile* tiles, const int* krow, const int* kw, int w_stride,
               int rpb_log2, cudaStream_t s, bool vec) {
    constexpr size_t smem = pcb::LseStage<TM, TB, MODE == 2>::bytes() + Packed<TM, TB, SPLIT>::bytes() +
                            2 * sizeof(float) * TB;
    static bool configured[64] = {false};
    const int dev = current_device();
    if (!configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(lse_bf16_kernel<TM, TB, MODE, SPLIT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return pcb::set_error(PCB_E_CUDA, "pcb_lse_contract(bf16): %s", cudaGetErrorString(e));
        configured[dev] = true;
    }
    return pcb::launch_status(pcb::launch_k(lse_bf16_kernel<TM, TB, MODE, SPLIT>, dim3(grid), dim3(kThreads), smem, s,
                                            1u, src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride,
                                            rpb_log2, vec), "pcb_lse_contract(bf16)");
}

template <int TM, int TB>
int launch(const float* src, const float* src2, const float* aux, float* out, int64_t ld, int B, const float* params,
           const PcbLseTile* tiles, int num_tiles, const int* krow, const int* kw, int w_stride, int rpb_log2,
           int mode, bool split, cudaStream_t s, bool vec) {
    dim3 grid((unsigned)num_tiles, (unsigned)pcb::cdiv(B, TB));
    if (grid.y > 65535) return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: batch too large");
#define PCB_L1(M, S) launch_one<TM, TB, M, S>(grid, src, src2, aux, out, ld, B, params, tiles, krow, kw, w_stride, rpb_log2, s, vec)
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
    const bool vec = pcb::vec_ok(src, ld) && pcb::vec_ok(out, ld) && (!src2 || pcb::vec_ok(src2, ld));
#define PCB_LB(TM, TB) launch<TM, TB>(src, src2, aux, out, ld, B, params, tiles, num_tiles, krow, kw, w_stride, rpb_log2, mode, split, s, vec)
    switch (tile_rows) {
        case 16: return PCB_LB(16, 128);
        case 32: return PCB_LB(32, 128);
        case 64: return PCB_LB(64, 64);
        case 128: return PCB_LB(128, 64);
        default:
            return pcb::set_error(PCB_E_ARG, "pcb_lse_contract: the bf16 form needs tile_rows 16..128, got %d", tile_rows);
    }
#undef PCB_LB
}
