// Product-layer gather-add (forward) and flow scatter (backward) plus the
// sum-layer "modify flows" pass. All are HBM-bound row gathers along the batch:
// one thread handles 4 consecutive samples of one output row (16-byte accesses).
#include "common.cuh"

namespace {

// MOD (overwrite, linear flows only): the rows of blocks g with mod_blk[g] != 0 are written as
// log(sum) - nm, the sum layer's "modified" node flows (log f - log m), instead of the sum.
template <bool ACCUM, bool LSE, bool MOD = false>
__global__ void __launch_bounds__(256)
prod_kernel(const float* __restrict__ in, float* __restrict__ out, int64_t ld, int B, const int* __restrict__ blk_row,
            const int* __restrict__ blk_off, const int* __restrict__ blk_cnt, const int* __restrict__ chs,
            int blk_size, int ngrp, int64_t total, bool vec, const float* __restrict__ nm,
            const int* __restrict__ mod_blk) {
    // The block tables (and the first 8 child indices) are read before the wait for the
    // previous kernel: they are compiled once and never written by a pass.
    pcb::pdl_trigger();
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int grp = (int)(idx % ngrp);
    const int64_t rowi = idx / ngrp;
    const int g = (int)(rowi / blk_size);
    const int i = (int)(rowi % blk_size);
    const int b = grp * 4;
    const int off = __ldg(blk_off + g);
    const int cnt = __ldg(blk_cnt + g);
    const int64_t row = (int64_t)__ldg(blk_row + g) + i;
    const bool rewrite = MOD && __ldg(mod_blk + g) != 0;
    int c[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) c[j] = (j < cnt) ? __ldg(chs + off + j) : -1;
    pcb::pdl_wait();
    float4 acc;
    if (!LSE) {
        acc = make_float4(0.f, 0.f, 0.f, 0.f);
        // 8 children at a time: all index loads, then all row loads, are independent
        for (int j0 = 0; j0 < cnt; j0 += 8) {
            if (j0 > 0) {
#pragma unroll
                for (int j = 0; j < 8; ++j) c[j] = (j0 + j < cnt) ? __ldg(chs + off + j0 + j) : -1;
            }
            float4 v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j)
                v[j] = (c[j] >= 0) ? pcb::load4(in, (int64_t)c[j] + i, ld, b, B, vec, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                acc.x += v[j].x; acc.y += v[j].y; acc.z += v[j].z; acc.w += v[j].w;
            }
        }
    } else {
        float4 m = make_float4(-INFINITY, -INFINITY, -INFINITY, -INFINITY);
        for (int j = 0; j < cnt; ++j) {
            const int c = __ldg(chs + off + j);
            const float4 v = pcb::load4(in, (int64_t)c + i, ld, b, B, vec, -INFINITY);
            m.x = fmaxf(m.x, v.x); m.y = fmaxf(m.y, v.y); m.z = fmaxf(m.z, v.z); m.w = fmaxf(m.w, v.w);
        }
        float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int j = 0; j < cnt; ++j) {
            const int c = __ldg(chs + off + j);
            const float4 v = pcb::load4(in, (int64_t)c + i, ld, b, B, vec, -INFINITY);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float mq = pcb::get(m, q);
                pcb::set(s, q, pcb::get(s, q) + (mq == -INFINITY ? 0.f : __expf(pcb::get(v, q) - mq)));
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float mq = pcb::get(m, q);
            pcb::set(acc, q, mq == -INFINITY ? -INFINITY : logf(pcb::get(s, q)) + mq);
        }
    }
    if (rewrite) {
        const float4 m = pcb::load4(nm, row, ld, b, B, vec, 0.f);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float mq = pcb::get(m, q);
            pcb::set(acc, q, mq == -INFINITY ? -INFINITY : logf(pcb::get(acc, q)) - mq);
        }
    }
    if (ACCUM) {
        const float4 old = pcb::load4(out, row, ld, b, B, vec, 0.f);
        if (!LSE) {
            acc.x += old.x; acc.y += old.y; acc.z += old.z; acc.w += old.w;
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) pcb::set(acc, q, pcb::logaddexp(pcb::get(old, q), pcb::get(acc, q)));
        }
    }
    pcb::store4(out, row, ld, b, B, vec, acc);
}

__global__ void __launch_bounds__(256)
modify_flows_kernel(float* __restrict__ nf, const float* __restrict__ nm, int64_t ld, int B, int64_t row0, int ngrp,
                    int64_t total, bool vec) {
    pcb::pdl_begin();
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int b = (int)(idx % ngrp) * 4;
    const int64_t row = row0 + idx / ngrp;
    float4 f = pcb::load4(nf, row, ld, b, B, vec, 0.f);
    const float4 m = pcb::load4(nm, row, ld, b, B, vec, 0.f);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float mq = pcb::get(m, q);
        pcb::set(f, q, mq == -INFINITY ? -INFINITY : logf(pcb::get(f, q)) - mq);
    }
    pcb::store4(nf, row, ld, b, B, vec, f);
}

}  // namespace

extern "C" int pcb_prod_gather_sum(const float* in, float* out, int64_t ld, int32_t B, const int32_t* blk_row,
                                   const int32_t* blk_off, const int32_t* blk_cnt, const int32_t* chs,
                                   int32_t num_blocks, int32_t blk_size, int32_t accum, int32_t logsumexp,
                                   void* stream) {
    if (!in || !out || !blk_row || !blk_off || !blk_cnt || !chs || B <= 0 || ld < B || num_blocks < 0 || blk_size <= 0)
        return pcb::set_error(PCB_E_ARG, "pcb_prod_gather_sum: bad arguments");
    if (num_blocks == 0) return PCB_OK;
    const int ngrp = (int)pcb::cdiv(B, 4);
    const int64_t total = (int64_t)num_blocks * blk_size * ngrp;
    const bool vec = pcb::vec_ok(in, ld) && pcb::vec_ok(out, ld);
    const unsigned grid = (unsigned)pcb::cdiv(total, 256);
    cudaStream_t s = pcb::as_stream(stream);
    if (!accum && !logsumexp) {
        return pcb::launch_status(pcb::launch_k(prod_kernel<false, false>, dim3(grid), dim3(256), 0, s, 1u, in, out,
                                                ld, B, blk_row, blk_off, blk_cnt, chs, blk_size, ngrp, total, vec,
                                                static_cast<const float*>(nullptr), static_cast<const int*>(nullptr)),
                                  "pcb_prod_gather_sum");
    } else if (accum && !logsumexp) {
        return pcb::launch_status(pcb::launch_k(prod_kernel<true, false>, dim3(grid), dim3(256), 0, s, 1u, in, out,
                                                ld, B, blk_row, blk_off, blk_cnt, chs, blk_size, ngrp, total, vec,
                                                static_cast<const float*>(nullptr), static_cast<const int*>(nullptr)),
                                  "pcb_prod_gather_sum");
    } else if (!accum && logsumexp) {
        return pcb::launch_status(pcb::launch_k(prod_kernel<false, true>, dim3(grid), dim3(256), 0, s, 1u, in, out,
                                                ld, B, blk_row, blk_off, blk_cnt, chs, blk_size, ngrp, total, vec,
                                                static_cast<const float*>(nullptr), static_cast<const int*>(nullptr)),
                                  "pcb_prod_gather_sum");
    } else {
        return pcb::launch_status(pcb::launch_k(prod_kernel<true, true>, dim3(grid), dim3(256), 0, s, 1u, in, out, ld,
                                                B, blk_row, blk_off, blk_cnt, chs, blk_size, ngrp, total, vec,
                                                static_cast<const float*>(nullptr), static_cast<const int*>(nullptr)),
                                  "pcb_prod_gather_sum");
    }
}

extern "C" int pcb_prod_gather_sum_modify(const float* in, float* out, int64_t ld, int32_t B, const int32_t* blk_row,
                                          const int32_t* blk_off, const int32_t* blk_cnt, const int32_t* chs,
                                          int32_t num_blocks, int32_t blk_size, const float* node_mars,
                                          const int32_t* block_rewrite, void* stream) {
    if (!in || !out || !blk_row || !blk_off || !blk_cnt || !chs || !node_mars || !block_rewrite || B <= 0 || ld < B ||
        num_blocks < 0 || blk_size <= 0)
        return pcb::set_error(PCB_E_ARG, "pcb_prod_gather_sum_modify: bad arguments");
    if (num_blocks == 0) return PCB_OK;
    const int ngrp = (int)pcb::cdiv(B, 4);
    const int64_t total = (int64_t)num_blocks * blk_size * ngrp;
    const bool vec = pcb::vec_ok(in, ld) && pcb::vec_ok(out, ld) && pcb::vec_ok(node_mars, ld);
    return pcb::launch_status(pcb::launch_k(prod_kernel<false, false, true>, dim3((unsigned)pcb::cdiv(total, 256)),
                                            dim3(256), 0, pcb::as_stream(stream), 1u, in, out, ld, B, blk_row, blk_off,
                                            blk_cnt, chs, blk_size, ngrp, total, vec, node_mars, block_rewrite),
                              "pcb_prod_gather_sum_modify");
}

extern "C" int pcb_modify_flows(float* node_flows, const float* node_mars, int64_t ld, int32_t B, int64_t row0,
                                int64_t row1, void* stream) {
    if (!node_flows || !node_mars || B <= 0 || ld < B || row0 < 0 || row1 < row0)
        return pcb::set_error(PCB_E_ARG, "pcb_modify_flows: bad arguments");
    if (row1 == row0) return PCB_OK;
    const int ngrp = (int)pcb::cdiv(B, 4);
    const int64_t total = (row1 - row0) * ngrp;
    const bool vec = pcb::vec_ok(node_flows, ld) && pcb::vec_ok(node_mars, ld);
    return pcb::launch_status(pcb::launch_k(modify_flows_kernel, dim3((unsigned)pcb::cdiv(total, 256)), dim3(256), 0,
                                            pcb::as_stream(stream), 1u, node_flows, node_mars, ld, B, row0, ngrp,
                                            total, vec), "pcb_modify_flows");
}
