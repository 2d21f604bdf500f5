// Double-buffered staging of LSE-contraction chunks (shared by the FP32 and BF16 kernels).
//
// A chunk is kLseKC contraction terms of one tile: the source rows krow[k] over the
// tile's samples, and the weights W(k, r) of the tile's rows. Both are copied with
// cp.async into one of two stage buffers; the issue loops have compile-time trip counts
// and are fully unrolled, so every thread issues all its index loads and copies back to
// back instead of waiting on each in turn.
#pragma once

#include "common.cuh"

namespace pcb {

constexpr int kLseKC = 32;

template <int TM, int TB, bool SRC2>
struct LseStage {
    static constexpr size_t kE = (size_t)kLseKC * TB;
    static constexpr size_t kW = (size_t)kLseKC * TM;
    static constexpr size_t kPer = kE * (SRC2 ? 2 : 1) + kW;
    static constexpr size_t bytes() { return sizeof(float) * 2 * kPer; }

    float* base;
    __device__ explicit LseStage(unsigned char* p) : base(reinterpret_cast<float*>(p)) {}
    __device__ float (*E(int s))[TB] { return reinterpret_cast<float(*)[TB]>(base + s * kPer); }
    __device__ float (*E2(int s))[TB] { return reinterpret_cast<float(*)[TB]>(base + s * kPer + kE); }
    __device__ float (*W(int s))[TM] { return reinterpret_cast<float(*)[TM]>(base + s * kPer + kE * (SRC2 ? 2 : 1)); }
    __device__ float* end() { return base + 2 * kPer; }

    __device__ __forceinline__ static void copy4(float* d, const float* g, int b, int B, bool vec) {
        if (vec && b + 3 < B) {
            cp_async16(d, g);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (b + j < B) cp_async4(d + j, g + j);
                else d[j] = -INFINITY;
            }
        }
    }

    // Issue the copies of chunk c into stage s (and commit them as one group).
    template <int NT>
    __device__ __forceinline__ void issue(int c, int s, const PcbLseTile& t, const float* __restrict__ src,
                                          const float* __restrict__ src2, const float* __restrict__ params,
                                          const int* __restrict__ krow, const int* __restrict__ kw, int64_t ld, int B,
                                          int b0, int w_stride, int rpb_log2, bool vec, int tid) {
        constexpr int NX = TB / 4;
        constexpr int E_IT = (kLseKC * NX + NT - 1) / NT;
        constexpr int W_IT = (kLseKC * TM + NT - 1) / NT;
        const int k0 = c * kLseKC;
        const int n = min(kLseKC, t.k_cnt - k0);
        float(*sE)[TB] = E(s);
        float(*sE2)[TB] = E2(s);
        float(*sW)[TM] = W(s);
        int rows[E_IT];
#pragma unroll
        for (int it = 0; it < E_IT; ++it) {
            const int idx = tid + it * NT;
            const int k = idx / NX;
            rows[it] = (idx < kLseKC * NX && k < n) ? __ldg(krow + t.k_off + k0 + k) : -1;
        }
#pragma unroll
        for (int it = 0; it < E_IT; ++it) {
            const int idx = tid + it * NT;
            if (idx >= kLseKC * NX) break;
            const int k = idx / NX;
            const int c4 = idx % NX;
            const int b = b0 + c4 * 4;
            if (rows[it] >= 0) {
                copy4(&sE[k][c4 * 4], src + (int64_t)rows[it] * ld + b, b, B, vec);
                if (SRC2) copy4(&sE2[k][c4 * 4], src2 + (int64_t)rows[it] * ld + b, b, B, vec);
            } else {
                *reinterpret_cast<float4*>(&sE[k][c4 * 4]) = make_float4(-INFINITY, -INFINITY, -INFINITY, -INFINITY);
                if (SRC2)
                    *reinterpret_cast<float4*>(&sE2[k][c4 * 4]) = make_float4(-INFINITY, -INFINITY, -INFINITY, -INFINITY);
            }
        }
        const int rpb_mask = (1 << rpb_log2) - 1;
        // forward weights are contiguous along rows, element-flow weights along terms
        const bool rows_fast = (w_stride == 1);
        int wk[W_IT];
#pragma unroll
        for (int it = 0; it < W_IT; ++it) {
            const int idx = tid + it * NT;
            const int k = rows_fast ? idx / TM : idx % kLseKC;
            const int r = rows_fast ? idx % TM : idx / kLseKC;
            wk[it] = (idx < kLseKC * TM && k < n && r < t.n_rows) ? __ldg(kw + t.k_off + k0 + k) : -1;
        }
#pragma unroll
        for (int it = 0; it < W_IT; ++it) {
            const int idx = tid + it * NT;
            if (idx >= kLseKC * TM) break;
            const int k = rows_fast ? idx / TM : idx % kLseKC;
            const int r = rows_fast ? idx % TM : idx / kLseKC;
            if (wk[it] >= 0) {
                const int64_t wi = (int64_t)wk[it] + t.w_add + (int64_t)(r >> rpb_log2) * t.g_stride +
                                   (int64_t)(r & rpb_mask) * w_stride;
                cp_async4(&sW[k][r], params + wi);
            } else {
                sW[k][r] = 0.f;
            }
        }
        cp_async_commit();
    }

    // After the chunk landed: mode-2 transform (log f - log m) and the per-sample running max.
    __device__ __forceinline__ void transform_and_max(int s, int n, float* sMax, float* sScale, int tid, int nt) {
        float(*sE)[TB] = E(s);
        if (SRC2) {
            float(*sE2)[TB] = E2(s);
            for (int idx = tid; idx < n * TB; idx += nt) {
                const int k = idx / TB;
                const int b = idx % TB;
                const float m = sE2[k][b];
                sE[k][b] = (m == -INFINITY) ? -INFINITY : logf(sE[k][b]) - m;
            }
            __syncthreads();
        }
        for (int b = tid; b < TB; b += nt) {
            float cm = -INFINITY;
            for (int k = 0; k < n; ++k) cm = fmaxf(cm, sE[k][b]);
            const float old = sMax[b];
            const float nm = fmaxf(old, cm);
            sScale[b] = (nm == -INFINITY) ? 1.f : __expf(old - nm);
            sMax[b] = nm;
        }
    }
};

}  // namespace pcb
