// Ancestral sampling, entirely on the device.
//
// Every sample keeps two short lists: the active nodes (input / sum node ids still to be
// expanded) and the active elements (product node ids chosen by the last sum layer
// group). Layer groups are visited top-down:
//   sum layer:  each active node of the layer picks one child element (first child k with
//               u < cumsum_k of its weights); other nodes stay in the list;
//   prod group: each active element appends all its children to the node list;
//   inputs:     each remaining input node draws a category (first k with u <= cumsum_k,
//               0 if none) into samples[s, var].
// Uniforms come from pcb_uniform(seed, node_id, sample) (SplitMix64 of a counter), so a
// CPU restatement with the same seed reproduces every draw bit for bit, or from a caller
// table uniforms[node_id * u_ld + sample] (the draws of another sampler, e.g. the
// reference's, replayed exactly).
#include "common.cuh"

namespace {

__device__ __forceinline__ float uniform(uint64_t seed, uint32_t node, uint32_t sample) {
    uint64_t z = seed + (((uint64_t)node << 32) | (uint64_t)sample) * 0x9E3779B97F4A7C15ull + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (float)(z >> 40) * (1.0f / 16777216.0f);
}

// One thread per sample; processes the nodes of one sum layer ([lo, hi)).
__global__ void sample_sum_kernel(int* __restrict__ nlist, int* __restrict__ ncnt, int* __restrict__ elist,
                                  int* __restrict__ ecnt, int S, int cap_n, int cap_e, int lo, int hi, int bs,
                                  const int* __restrict__ node2blk, const int* __restrict__ blk_nid,
                                  const int* __restrict__ blk_koff, const int* __restrict__ blk_kcnt,
                                  const int* __restrict__ krow, const int* __restrict__ kw,
                                  const float* __restrict__ params, const float* __restrict__ uniforms, int64_t u_ld,
                                  uint64_t seed, int* __restrict__ err) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    int* nl = nlist + (int64_t)s * cap_n;
    int* el = elist + (int64_t)s * cap_e;
    const int n = ncnt[s];
    int keep = 0;
    int ne = ecnt[s];
    for (int j = 0; j < n; ++j) {
        const int id = nl[j];
        if (id < lo || id >= hi) {
            nl[keep++] = id;
            continue;
        }
        const int g = node2blk[(id - lo) / bs];
        const int i = id - blk_nid[g];
        const int off = blk_koff[g];
        const int cnt = blk_kcnt[g];
        const float u = uniforms ? uniforms[(int64_t)id * u_ld + s] : uniform(seed, (uint32_t)id, (uint32_t)s);
        float cum = 0.f;
        int pick = -1, last_nz = 0;
        for (int k = 0; k < cnt; ++k) {
            const float w = params[(int64_t)kw[off + k] + i];
            cum += w;
            if (w > 0.f) last_nz = k;
            if (u < cum) { pick = k; break; }
        }
        if (pick < 0) pick = last_nz;
        if (ne < cap_e) el[ne++] = krow[off + pick];
        else atomicExch(err, 1);
    }
    ncnt[s] = keep;
    ecnt[s] = ne;
}

// One thread per sample: expand the active elements of one product layer ([elo, ehi));
// elements of other layers of the group stay in the list.
__global__ void sample_prod_kernel(int* __restrict__ nlist, int* __restrict__ ncnt, int* __restrict__ elist,
                                   int* __restrict__ ecnt, int S, int cap_n, int cap_e, int elo, int ehi,
                                   const int* __restrict__ elem2blk, const int* __restrict__ blk_row,
                                   const int* __restrict__ blk_off, const int* __restrict__ blk_cnt,
                                   const int* __restrict__ chs, int* __restrict__ err) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    int* nl = nlist + (int64_t)s * cap_n;
    int* el = elist + (int64_t)s * cap_e;
    int n = ncnt[s];
    const int ne = ecnt[s];
    int keep = 0;
    for (int j = 0; j < ne; ++j) {
        const int id = el[j];
        if (id < elo || id >= ehi) { el[keep++] = id; continue; }
        const int g = elem2blk[id - elo];
        if (g < 0) { atomicExch(err, 2); continue; }
        const int i = id - blk_row[g];
        const int off = blk_off[g];
        const int cnt = blk_cnt[g];
        for (int c = 0; c < cnt; ++c) {
            if (n < cap_n) nl[n++] = chs[off + c] + i;
            else atomicExch(err, 1);
        }
    }
    ncnt[s] = n;
    ecnt[s] = keep;
}

// One thread per (sample, list slot): draw a category for every active input node.
__global__ void sample_input_kernel(const int* __restrict__ nlist, const int* __restrict__ ncnt, int S, int cap_n,
                                    int lo, int hi, const int* __restrict__ vids, const int* __restrict__ s_pids,
                                    const int* __restrict__ ncats, const float* __restrict__ params,
                                    int64_t* __restrict__ samples, int64_t sld, const float* __restrict__ uniforms,
                                    int64_t u_ld, uint64_t seed) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= (int64_t)S * cap_n) return;
    const int s = (int)(idx / cap_n);
    const int j = (int)(idx % cap_n);
    if (j >= ncnt[s]) return;
    const int id = nlist[idx];
    if (id < lo || id >= hi) return;
    const int n = id - lo;
    const int K = ncats[n];
    const int64_t sp = s_pids[n];
    const float u = uniforms ? uniforms[(int64_t)id * u_ld + s] : uniform(seed, (uint32_t)id, (uint32_t)s);
    float cum = 0.f;
    int pick = -1;
    for (int k = 0; k < K; ++k) {
        cum += params[sp + k];
        if (cum >= u) { pick = k; break; }
    }
    if (pick < 0) pick = 0;
    samples[(int64_t)s * sld + vids[n]] = pick;
}

// SoftEvidenceCategorical inputs: category k with probability theta[n, k] exp(L[s, u, k]) / Z
// over k < K (the evidence of sample s for the node's variable u), the first category whose
// cumulative probability exceeds the uniform (softevi_categorical.py:683-761); the last
// category when rounding leaves the uniform above the total.
__global__ void sample_input_poe_kernel(const int* __restrict__ nlist, const int* __restrict__ ncnt, int S, int cap_n,
                                        int lo, int hi, const int* __restrict__ vids, const int* __restrict__ s_pids,
                                        const int* __restrict__ node_lvid, const float* __restrict__ params,
                                        const float* __restrict__ logp, int64_t e_sb, int64_t e_su, int K,
                                        int64_t* __restrict__ samples, int64_t sld, const float* __restrict__ uniforms,
                                        int64_t u_ld, uint64_t seed) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= (int64_t)S * cap_n) return;
    const int s = (int)(idx / cap_n);
    const int j = (int)(idx % cap_n);
    if (j >= ncnt[s]) return;
    const int id = nlist[idx];
    if (id < lo || id >= hi) return;
    const int n = id - lo;
    const int64_t sp = s_pids[n];
    const float* L = logp + (int64_t)s * e_sb + (int64_t)node_lvid[n] * e_su;
    float m = -INFINITY;
    for (int k = 0; k < K; ++k) m = fmaxf(m, L[k]);
    float z = 0.f;
    for (int k = 0; k < K; ++k) z += params[sp + k] * expf(L[k] - m);
    const float u = (uniforms ? uniforms[(int64_t)id * u_ld + s] : uniform(seed, (uint32_t)id, (uint32_t)s)) * z;
    float cum = 0.f;
    int pick = K - 1;
    for (int k = 0; k < K; ++k) {
        cum += params[sp + k] * expf(L[k] - m);
        if (cum > u) { pick = k; break; }
    }
    samples[(int64_t)s * sld + vids[n]] = pick;
}

// Bernoulli (kind 1), Gaussian (kind 2) and DiscreteLogistic (kind 3) inputs, one uniform u
// per (node, sample): Bernoulli 1 if u < p else 0 (bernoulli.py:79-88); Gaussian
// mu + sigma Phi^-1(u') with u' = u + 2^-25 inside (0, 1) (the reference draws a Box-Muller
// normal, gaussian.py:114-125: same distribution, other draws); DiscreteLogistic the bin of
// mu + s log(u / (1 - u)) among num_cats bins of [lo, hi), clamped to the first and last
// (discrete_logistic.py:157-181). Values are written as FP32.
__global__ void sample_input_dist_kernel(int kind, const int* __restrict__ nlist, const int* __restrict__ ncnt, int S,
                                         int cap_n, int lo, int hi, const int* __restrict__ vids,
                                         const int* __restrict__ s_pids, const float* __restrict__ meta,
                                         const float* __restrict__ params, float* __restrict__ samples, int64_t sld,
                                         const float* __restrict__ uniforms, int64_t u_ld, uint64_t seed) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= (int64_t)S * cap_n) return;
    const int s = (int)(idx / cap_n);
    const int j = (int)(idx % cap_n);
    if (j >= ncnt[s]) return;
    const int id = nlist[idx];
    if (id < lo || id >= hi) return;
    const int n = id - lo;
    const int64_t sp = s_pids[n];
    const float u = uniforms ? uniforms[(int64_t)id * u_ld + s] : uniform(seed, (uint32_t)id, (uint32_t)s);
    float r;
    if (kind == 1) {
        r = u < params[sp] ? 1.f : 0.f;
    } else if (kind == 2) {
        r = params[sp] + params[sp + 1] * normcdfinvf(fminf(u + 2.98023224e-8f, 0.99999994f));
    } else {
        const float lo_v = meta[4 * (int64_t)n], hi_v = meta[4 * (int64_t)n + 1], nc = meta[4 * (int64_t)n + 2];
        const float x = params[sp] + params[sp + 1] * logf(u / (1.f - u));
        const float bin = (x - lo_v) / ((hi_v - lo_v) / nc);
        r = bin < 0.f ? 0.f : (bin > nc - 1.f ? nc - 1.f : floorf(bin));
    }
    samples[(int64_t)s * sld + vids[n]] = r;
}

}  // namespace

extern "C" {

int pcb_sample_sum(int32_t* nlist, int32_t* ncnt, int32_t* elist, int32_t* ecnt, int32_t S, int32_t cap_n,
                   int32_t cap_e, int32_t lo, int32_t hi, int32_t bs, const int32_t* node2blk, const int32_t* blk_nid,
                   const int32_t* blk_koff, const int32_t* blk_kcnt, const int32_t* krow, const int32_t* kw,
                   const float* params, const float* uniforms, int64_t u_ld, uint64_t seed, int32_t* err,
                   void* stream) {
    if (!nlist || !ncnt || !elist || !ecnt || !node2blk || !blk_nid || !blk_koff || !blk_kcnt || !krow || !kw ||
        !params || !err || S < 0 || cap_n <= 0 || cap_e <= 0 || hi < lo || bs <= 0 || (uniforms && u_ld < S))
        return pcb::set_error(PCB_E_ARG, "pcb_sample_sum: bad arguments");
    if (S == 0) return PCB_OK;
    sample_sum_kernel<<<(unsigned)pcb::cdiv(S, 128), 128, 0, pcb::as_stream(stream)>>>(
        nlist, ncnt, elist, ecnt, S, cap_n, cap_e, lo, hi, bs, node2blk, blk_nid, blk_koff, blk_kcnt, krow, kw, params,
        uniforms, u_ld, seed, err);
    return pcb::check_launch("pcb_sample_sum");
}

int pcb_sample_prod(int32_t* nlist, int32_t* ncnt, int32_t* elist, int32_t* ecnt, int32_t S, int32_t cap_n,
                    int32_t cap_e, int32_t elo, int32_t ehi, const int32_t* elem2blk, const int32_t* blk_row,
                    const int32_t* blk_off, const int32_t* blk_cnt, const int32_t* chs, int32_t* err, void* stream) {
    if (!nlist || !ncnt || !elist || !ecnt || !elem2blk || !blk_row || !blk_off || !blk_cnt || !chs || !err || S < 0 ||
        cap_n <= 0 || cap_e <= 0 || ehi < elo)
        return pcb::set_error(PCB_E_ARG, "pcb_sample_prod: bad arguments");
    if (S == 0) return PCB_OK;
    sample_prod_kernel<<<(unsigned)pcb::cdiv(S, 128), 128, 0, pcb::as_stream(stream)>>>(
        nlist, ncnt, elist, ecnt, S, cap_n, cap_e, elo, ehi, elem2blk, blk_row, blk_off, blk_cnt, chs, err);
    return pcb::check_launch("pcb_sample_prod");
}

int pcb_sample_input(const int32_t* nlist, const int32_t* ncnt, int32_t S, int32_t cap_n, int32_t lo, int32_t hi,
                     const int32_t* vids, const int32_t* s_pids, const int32_t* ncats, const float* params,
                     int64_t* samples, int64_t sld, const float* uniforms, int64_t u_ld, uint64_t seed, void* stream) {
    if (!nlist || !ncnt || !vids || !s_pids || !ncats || !params || !samples || S < 0 || cap_n <= 0 || hi < lo ||
        (uniforms && u_ld < S))
        return pcb::set_error(PCB_E_ARG, "pcb_sample_input: bad arguments");
    if (S == 0) return PCB_OK;
    const int64_t total = (int64_t)S * cap_n;
    sample_input_kernel<<<(unsigned)pcb::cdiv(total, 256), 256, 0, pcb::as_stream(stream)>>>(
        nlist, ncnt, S, cap_n, lo, hi, vids, s_pids, ncats, params, samples, sld, uniforms, u_ld, seed);
    return pcb::check_launch("pcb_sample_input");
}

int pcb_sample_input_poe(const int32_t* nlist, const int32_t* ncnt, int32_t S, int32_t cap_n, int32_t lo, int32_t hi,
                         const int32_t* vids, const int32_t* s_pids, const int32_t* node_lvid, const float* params,
                         const float* evidence_logp, int64_t e_sb, int64_t e_su, int32_t K, int64_t* samples,
                         int64_t sld, const float* uniforms, int64_t u_ld, uint64_t seed, void* stream) {
    if (!nlist || !ncnt || !vids || !s_pids || !node_lvid || !params || !evidence_logp || K <= 0 || !samples ||
        S < 0 || cap_n <= 0 || hi < lo || (uniforms && u_ld < S))
        return pcb::set_error(PCB_E_ARG, "pcb_sample_input_poe: bad arguments");
    if (S == 0) return PCB_OK;
    const int64_t total = (int64_t)S * cap_n;
    sample_input_poe_kernel<<<(unsigned)pcb::cdiv(total, 256), 256, 0, pcb::as_stream(stream)>>>(
        nlist, ncnt, S, cap_n, lo, hi, vids, s_pids, node_lvid, params, evidence_logp, e_sb, e_su, K, samples, sld,
        uniforms, u_ld, seed);
    return pcb::check_launch("pcb_sample_input_poe");
}

int pcb_sample_input_dist(int32_t kind, const int32_t* nlist, const int32_t* ncnt, int32_t S, int32_t cap_n, int32_t lo,
                          int32_t hi, const int32_t* vids, const int32_t* s_pids, const float* meta,
                          const float* params, float* samples, int64_t sld, const float* uniforms, int64_t u_ld,
                          uint64_t seed, void* stream) {
    if (kind < 1 || kind > 3 || (kind == 3 && !meta) || !nlist || !ncnt || !vids || !s_pids || !params || !samples ||
        S < 0 || cap_n <= 0 || hi < lo || (uniforms && u_ld < S))
        return pcb::set_error(PCB_E_ARG, "pcb_sample_input_dist: bad arguments");
    if (S == 0) return PCB_OK;
    const int64_t total = (int64_t)S * cap_n;
    sample_input_dist_kernel<<<(unsigned)pcb::cdiv(total, 256), 256, 0, pcb::as_stream(stream)>>>(
        kind, nlist, ncnt, S, cap_n, lo, hi, vids, s_pids, meta, params, samples, sld, uniforms, u_ld, seed);
    return pcb::check_launch("pcb_sample_input_dist");
}

}  // extern "C"
