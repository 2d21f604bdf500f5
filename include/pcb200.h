/*
 * pcb200.h -- C ABI of libpcb200.so, the sm_100a kernels behind pyjuice_b200.
 *
 * Every entry point takes device pointers, sizes and a cudaStream_t (passed as
 * void*), launches asynchronously on that stream and returns 0 on success or a
 * negative PCB_E* code; pcb_last_error() then describes the failure. No entry point
 * allocates device memory: every buffer, including workspaces, is owned by the
 * caller. Index tables are int32 unless stated otherwise.
 *
 * Matrices of per-node values ("rows x batch") are row-major with leading
 * dimension `ld` (>= B): value (row r, sample b) lives at base[r * ld + b].
 *
 * The reference (SimonHaepers/pyjuice) is Python + Triton. Each entry point below
 * replaces the Triton launch(es) cited in its comment; paths are relative to the
 * reference project root.
 */
#ifndef PCB200_H
#define PCB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PCB_OK 0
#define PCB_E_ARG -1       /* bad size / pointer / unsupported configuration */
#define PCB_E_LAUNCH -2    /* CUDA launch error */
#define PCB_E_CUDA -3      /* other CUDA runtime error */

/* Bits of the device status word (pcb_device_status): faults that kernels detect on the
 * device, where they cannot return an error code. The affected outputs are NaN. */
#define PCB_STATUS_WAIT_TIMEOUT 1   /* a bounded wait (mbarrier: bulk copy or MMA completion) ran out */
#define PCB_STATUS_TILE_TOO_LONG 2  /* a contraction tile had more terms than the kernel handles */
#define PCB_STATUS_BAD_CATEGORY 4   /* an input value outside [0, num_cats) */

/*
 * One tile of an LSE contraction (sum forward / element flows). A tile covers n_rows
 * consecutive output rows made of consecutive blocks of `rows_per_block` rows (the
 * launch argument) that share the same contraction terms; row r of the tile uses weight
 *   params[kw[k] + w_add + (r / rows_per_block) * g_stride + (r % rows_per_block) * w_stride].
 */
typedef struct {
    int32_t out_row;   /* first output row of the tile */
    int32_t n_rows;    /* rows in the tile (<= tile height of the launch) */
    int32_t k_off;     /* offset into krow[] / kw[] */
    int32_t k_cnt;     /* number of contraction terms */
    int32_t w_add;     /* added to kw[k] for tile row 0 */
    int32_t aux_row;   /* element-flow epilogue: first element_mars row of the tile */
    int32_t g_stride;  /* weight offset between consecutive blocks of the tile */
    int32_t reserved;
} PcbLseTile;

/*
 * One tile of the sum-parameter-flow contraction (contraction over the batch): nodes
 * nid + r (r < n_rows, consecutive blocks of `rows_per_block` nodes sharing children)
 * and children k_off .. k_off + k_cnt - 1. Node r of child k uses
 *   weight  params[pids[k] + p_add + (r / rows_per_block) * gs_p + r % rows_per_block]
 *   flow    param_flows[pfids[k] + p_add + (r / rows_per_block) * gs_pf + r % rows_per_block].
 */
typedef struct {
    int32_t nid;       /* first node row of the tile */
    int32_t n_rows;    /* nodes in the tile (<= 128) */
    int32_t k_off;     /* offset into cids[] / pids[] / pfids[] of the tile's first child */
    int32_t k_cnt;     /* children in the tile (<= the launch's tile_children) */
    int32_t p_add;     /* added to pids / pfids for tile row 0 */
    int32_t gs_p;      /* parameter offset between consecutive blocks of the tile */
    int32_t gs_pf;     /* flow offset between consecutive blocks of the tile */
    int32_t reserved;
} PcbPflowTile;

/* Version of the library ABI (currently 1). No counterpart in the reference (library utility). */
int pcb_version(void);

/* Last error message of the calling host thread ("" if none). No counterpart in the reference (library utility). */
const char* pcb_last_error(void);

/* Number of SMs of the current device (for grid sizing on the host). No counterpart in the reference (library utility). */
int pcb_num_sms(void);

/*
 * Device status word of the current device: waits for `stream`, writes the OR of all
 * PCB_STATUS_* bits reported by kernels since the last clear to *out (host memory) and,
 * if clear != 0, resets it (on `stream`). Synchronises the stream. The word is per device
 * and shared by all streams and callers on it.
 * No counterpart in the reference (its Triton kernels have no device-side error channel;
 * the host asserts before launch, e.g. src/pyjuice/layer/sum_layer.py:819, 842-844).
 */
int pcb_device_status(int32_t* out, int32_t clear, void* stream);

/*
 * Test of the device error channel: one CTA polls an mbarrier that nothing completes at
 * most spin_limit times (the bounded wait of pcb_lse_contract_tc05), then reports
 * PCB_STATUS_WAIT_TIMEOUT and returns; the context stays usable.
 * No counterpart in the reference (library self-test).
 */
int pcb_status_selftest(int32_t spin_limit, void* stream);

/*
 * Fill rows [row0, row1) of a rows x ld matrix with `value` (all ld columns).
 * Replaces the buffer initialisations of TensorCircuit.forward / backward
 * (src/pyjuice/model/tensorcircuit.py:240-241, 394-395) for the rows that are read
 * before being written (dummy rows).
 */
int pcb_fill_rows(float* mat, int64_t ld, int64_t row0, int64_t row1, float value, void* stream);

/*
 * Categorical input layer forward: node_mars[node_offset + n, b] =
 *   log(params[s_pids[n] + data[vids[n] * data_ld + b]]) for n < num_nodes, b < B
 * (NaN where the category is outside [0, ncats[n]), reported as PCB_STATUS_BAD_CATEGORY),
 * or 0 where `missing` (may be NULL) marks the variable as missing in that sample:
 * missing[b * miss_sb + vids[n] * miss_sv] != 0 (miss_sb = 0 for a per-variable mask).
 * data is int64 [num_vars, data_ld]. The missing-mask form replaces
 * InputLayer._fw_missing_mask_kernel (src/pyjuice/layer/input_layer.py:1059-1095).
 * Replaces InputLayer._mars_kernel_template + Categorical.fw_mar_fn
 * (src/pyjuice/layer/input_layer.py:1016-1054, src/pyjuice/nodes/distributions/categorical.py:83-91).
 */
int pcb_input_cat_fwd(const int64_t* data, int64_t data_ld, const float* params,
                      const int32_t* vids, const int32_t* s_pids, const int32_t* ncats, int32_t num_nodes,
                      int32_t node_offset, float* node_mars, int64_t ld, int32_t B, const uint8_t* missing,
                      int64_t miss_sb, int64_t miss_sv, void* stream);

/*
 * Categorical input layer backward (parameter flows), deterministic:
 * param_flows[s_pfids[n] + k] += sum_{b : data[v, b] == k} node_flows[node_offset + n, b]
 * for every node n of every variable group. Groups are runs of nodes over the same
 * variable: group g covers nodes [grp_node0[g], grp_node0[g] + grp_count[g]) of
 * variable grp_var[g], with grp_ncats[g] categories; samples whose category is outside
 * [0, ncats) are skipped. logspace_flows: node flows hold log flows. Where `missing`
 * (may be NULL; same indexing as pcb_input_cat_fwd) marks the variable as missing, the
 * node's flow f goes to every category k as f * params[s_pids[n] + k] (s_pids and params
 * are read only then; categorical.py:102-134). atomic = 1 when several nodes share flow
 * slots (tied nodes; the sums are then added with float atomics, as the reference does).
 * Replaces InputLayer._flows_kernel_template + Categorical.bk_flow_fn
 * (src/pyjuice/layer/input_layer.py:1098-1155, categorical.py:94-100), whose atomic
 * scatter this replaces with a per-variable counting sort of the batch.
 */
int pcb_input_cat_bwd(const int64_t* data, int64_t data_ld, const float* node_flows, int64_t ld, int32_t B,
                      const int32_t* grp_var, const int32_t* grp_node0, const int32_t* grp_count,
                      const int32_t* grp_ncats, int32_t num_groups, int32_t max_ncats,
                      const int32_t* s_pfids, int32_t node_offset, float* param_flows,
                      int32_t logspace_flows, const uint8_t* missing, int64_t miss_sb, int64_t miss_sv,
                      const int32_t* s_pids, const float* params, int32_t atomic, void* stream);

/*
 * Categorical EM update of the source nodes (in FP64):
 *   theta' = (1 - s) * theta + s * (f + pc / K) / (sum_k f + pc)
 * (keep_zero_params: zero parameters stay zero and the normaliser excludes them).
 * Replaces InputLayer._em_kernel_template + Categorical.{small,large}_ncats_em_fn
 * (src/pyjuice/layer/input_layer.py:1275-1296, categorical.py:164-244).
 */
int pcb_input_cat_em(float* params, const float* param_flows, const int32_t* s_pids, const int32_t* s_pfids,
                     const int32_t* ncats, const int32_t* source_nids, int32_t num_source_nodes,
                     double step_size, double pseudocount, int32_t keep_zero_params, void* stream);

/*
 * Bernoulli (kind 1), Gaussian (kind 2) and DiscreteLogistic (kind 3) input layers; data is
 * FP32 [num_vars, data_ld] (Bernoulli reads x > 0; DiscreteLogistic reads bin indices),
 * missing values indexed as in pcb_input_cat_fwd. meta: per-node metadata indexed by the
 * node's layer-local id, Gaussian min_sigma[n] (EM only), DiscreteLogistic
 * (lo, hi, num_cats, min_std) at meta[4 n .. 4 n + 3] (all three calls); NULL otherwise.
 * pcb_input_dist_fwd: node_mars = log p (Bernoulli: p = params[s_pid] for x > 0, else 1 - p;
 *   Gaussian: log N(x; params[s_pid], params[s_pid + 1]); DiscreteLogistic with
 *   (mu, s) = params[s_pid ..] and w = (hi - lo) / num_cats: log(F(lo + (x + 1) w) - F(lo + x w)),
 *   F(v) = 1 / (1 + exp((mu - v) / s)), F = 1 above the last bin and 0 below the first,
 *   clamped at -1000), 0 where missing.
 * pcb_input_dist_bwd: per node, the batch sums of the flow-weighted sufficient statistics
 *   added to its flow slots: Bernoulli (x > 0, x <= 0) (missing samples add nothing);
 *   Gaussian (f x, f x^2, f), a missing value contributing (f mu, f (sigma^2 + mu^2), f);
 *   DiscreteLogistic the same with the bin midpoint m = lo + (x + 1/2) w for x and the
 *   variance s^2 pi^2 / 3 for sigma^2.
 *   atomic = 1 when tied nodes share slots. logspace_flows: node flows hold log flows.
 * pcb_input_dist_em: Bernoulli p' = (1 - s) p + s (f1 + pc / 2) / (f1 + f0 + pc); Gaussian
 *   moment matching of the step-interpolated expectation parameters, sigma >= min_sigma[n];
 *   DiscreteLogistic the same on the standard deviation s pi / sqrt(3) >= min_std.
 * Replace the fw_mar_fn / bk_flow_fn / bk_flow_mask_fn / em_fn kernels of
 * src/pyjuice/nodes/distributions/bernoulli.py:64-102, gaussian.py:87-170 and
 * discrete_logistic.py:81-202.
 */
int pcb_input_dist_fwd(int32_t kind, const float* data, int64_t data_ld, const float* params, const int32_t* vids,
                       const int32_t* s_pids, const float* meta, int32_t num_nodes, int32_t node_offset,
                       float* node_mars, int64_t ld, int32_t B, const uint8_t* missing, int64_t miss_sb,
                       int64_t miss_sv, void* stream);
int pcb_input_dist_bwd(int32_t kind, const float* data, int64_t data_ld, const float* node_flows, int64_t ld, int32_t B,
                       const float* params, const int32_t* vids, const int32_t* s_pids, const int32_t* s_pfids,
                       const float* meta, int32_t num_nodes, int32_t node_offset, float* param_flows,
                       int32_t logspace_flows, const uint8_t* missing, int64_t miss_sb, int64_t miss_sv,
                       int32_t atomic, void* stream);
int pcb_input_dist_em(int32_t kind, float* params, const float* param_flows, const int32_t* s_pids,
                      const int32_t* s_pfids, const float* meta, const int32_t* source_nids,
                      int32_t num_source_nodes, double step_size, double pseudocount, void* stream);

/*
 * SoftEvidenceCategorical input layers (categorical nodes times per-sample evidence over the
 * categories). Evidence: log-weights L[b, u, j] at evidence_logp + b e_sb + u e_su + j, j < K,
 * u = grp_lvid[g] for the group's variable; dense (cat_ids NULL: j is the category, K <= every
 * node's num_cats) or sparse (cat_ids at the same offsets give the category of entry j).
 * Groups: runs of consecutive nodes over one variable (grp_var, grp_node0 layer-local,
 * grp_count); node_grp: the group of each node (sparse forward only).
 * pcb_input_poe_fwd: node_mars[n, b] = log theta[n, x] + L[b, u, x] - log Z[n, b],
 *   Z = sum_j theta[n, cat_j] exp(L[b, u, j]), with x = data[v, b]; 0 where missing; a
 *   category outside the node's or the evidence's range gives -inf (sparse: no entry) or NaN
 *   (dense).
 * pcb_input_poe_evidence_bwd: evidence_grad[b, u, j] += sum_n f[n, b] ([cat_j == x] -
 *   theta[n, cat_j] exp(L[b, u, j]) / Z[n, b]) over the variable's nodes, f the node flows
 *   (logspace_flows: node_flows hold log f); Z recovered from node_mars of the forward.
 * Replace fw_kernel, bk_softevi_kernel (softevi_categorical.py:310-462, 502-681); the
 * parameter flows (bk_params_kernel, 464-500) are pcb_input_cat_bwd's.
 */
int pcb_input_poe_fwd(const int64_t* data, int64_t data_ld, const float* evidence_logp, const int64_t* cat_ids,
                      int64_t e_sb, int64_t e_su, int32_t K, const float* params, const int32_t* grp_var,
                      const int32_t* grp_lvid, const int32_t* grp_node0, const int32_t* grp_count,
                      int32_t num_groups, int32_t max_group_nodes, const int32_t* node_grp, int32_t num_nodes,
                      const int32_t* s_pids, const int32_t* ncats, int32_t node_offset, float* node_mars,
                      int64_t ld, int32_t B, const uint8_t* missing, int64_t miss_sb, int64_t miss_sv,
                      void* stream);
int pcb_input_poe_evidence_bwd(const int64_t* data, int64_t data_ld, const float* node_flows, const float* node_mars,
                               int64_t ld, int32_t B, int32_t logspace_flows, const float* evidence_logp,
                               const int64_t* cat_ids, int64_t e_sb, int64_t e_su, int32_t K, float* evidence_grad,
                               int64_t g_sb, int64_t g_su, const float* params, const int32_t* grp_var,
                               const int32_t* grp_lvid, const int32_t* grp_node0, const int32_t* grp_count,
                               int32_t num_groups, int32_t max_group_nodes, const int32_t* s_pids,
                               const int32_t* ncats, int32_t node_offset, void* stream);

/*
 * Sum of tied input-node flow slots into the source slot:
 * param_flows[dst + i] = sum_j param_flows[srcs[j] + i], i < n.
 * Replaces InputLayer._pflow_accum_kernel (src/pyjuice/layer/input_layer.py:1254-1272)
 * and cum_par_flows_kernel (src/pyjuice/model/backend/parflow_fusing.py:81-99).
 */
int pcb_pflow_accum(float* param_flows, int64_t dst, int64_t n, const int64_t* srcs, int32_t nsrc, void* stream);

/*
 * Product layer, forward (accum=0): out[r0 + i, b] = sum_j in[c_j + i, b], or
 * backward (accum=1): out[r0 + i, b] += sum_j in[c_j + i, b], where the block list
 * gives for block g: r0 = blk_row[g], its children c_j = chs[blk_off[g] + j],
 * j < blk_cnt[g] (zero entries are padding and skipped), and blk_size rows.
 * logsumexp=1 combines in log space (logspace flows).
 * Replaces ProdLayer._forward_backward_kernel_2d / _large
 * (src/pyjuice/layer/prod_layer.py:398-555).
 */
int pcb_prod_gather_sum(const float* in, float* out, int64_t ld, int32_t B,
                        const int32_t* blk_row, const int32_t* blk_off, const int32_t* blk_cnt, const int32_t* chs,
                        int32_t num_blocks, int32_t blk_size, int32_t accum, int32_t logsumexp, void* stream);

/*
 * pcb_prod_gather_sum backward in overwrite mode (accum = 0, linear flows) fused with
 * pcb_modify_flows: the rows of blocks g with block_rewrite[g] != 0 (device array, one entry
 * per block) receive log(sum) - node_mars (-inf where node_mars is -inf) instead of the sum,
 * other rows the sum. Valid when this launch is the only writer of the flagged rows (their
 * flows are complete when written). Replaces the same reference kernels as the two
 * launches it combines.
 */
int pcb_prod_gather_sum_modify(const float* in, float* out, int64_t ld, int32_t B, const int32_t* blk_row,
                               const int32_t* blk_off, const int32_t* blk_cnt, const int32_t* chs, int32_t num_blocks,
                               int32_t blk_size, const float* node_mars, const int32_t* block_rewrite, void* stream);

/*
 * Log-sum-exp contraction over tiles, FP32 FMA (plain) or BF16 tensor-core (prec=1):
 *   acc[r, b] = sum_k W(k, r) * exp(src[krow[k], b] - m_b),  m_b = max_k src[krow[k], b]
 *   W(k, r)   = params[kw[k] + w_add + (r / rows_per_block) * g_stride + (r % rows_per_block) * w_stride]
 * tile_rows (power of 2, <= 128) is the launch's tile height; rows_per_block a power of 2.
 * mode 0 (sum forward):    out[out_row + r, b] = log(acc) + m_b
 * mode 1 (element flows):  out[out_row + r, b] = acc * exp(aux[aux_row + r, b] + m_b)
 * mode 2 (element flows, unmodified node flows): as mode 1 with src = log(src) - src2.
 * FP32 forward of one-row tiles (tile_rows 1, mode 0: sum layers of block size 1): lanes over
 * 32 samples, 32 warps over the terms, online log-sum-exp, for roots over thousands of
 * children.
 * Replaces SumLayer._fw_triton_block_sparse_*_kernel, _fw_triton_sparse_kernel,
 * _fw_triton_large_sparse_kernel (src/pyjuice/layer/sum_layer.py:454-1104) and
 * _bk_triton_block_sparse_ele_kernel / _csmm2 / sparse element-flow kernels
 * (sum_layer.py:1572-1889, 2466-2666).
 */
int pcb_lse_contract(const float* src, const float* src2, const float* aux, float* out, int64_t ld, int32_t B,
                     const float* params, const PcbLseTile* tiles, int32_t num_tiles, int32_t tile_rows,
                     int32_t rows_per_block, const int32_t* krow, const int32_t* kw, int32_t w_stride, int32_t mode,
                     int32_t prec, void* stream);

/*
 * Product layer fused into a pcb_lse_contract_short launch (replaces the
 * pcb_prod_gather_sum launch of the product layer below / above the sum layer):
 *  - forward (mode 0): term_children[4 k + j], j < 4, are the node rows whose sum is term
 *    k's element value (-1: no such child). src is then node_mars; the kernel also writes
 *    the element values to element_out row krow[k] (the product layer's output).
 *  - element flows (mode 2): out_children[4 e + j], j < 4, are the node rows that receive
 *    output row e's flow (-1: none); out is then node_flows. Valid when those children
 *    have no other parent and nothing else writes their rows.
 * Fused launches need batch_tile <= 32. NULL (or null members) leaves the kernel unfused.
 */
typedef struct {
    const int32_t* term_children;
    float* element_out;
    const int32_t* out_children;
} PcbShortFusion;

/*
 * Same contraction, epilogues and precision forms (prec 0 FP32, 1 bf16, 2 split bf16) as
 * pcb_lse_contract for tiles of at most 128 terms, built for latency: each CTA stages all
 * its terms at once and computes a slice of RM rows (32 when tile_rows <= 32, else 64) by
 * batch_tile samples (16, 32 or 64), so small layers launch many CTAs.
 * wlayout: 0 = weights copied one by one; 1 = groups of 4 consecutive rows have
 * consecutive, 16-byte aligned weights (forward tables); 2 = groups of 4 consecutive terms
 * do (element-flow tables). packed (BF16 forms only, may be NULL): the same tiles' weights
 * as written by pcb_pack_weights; the kernel then copies them instead of reading params.
 * The caller guarantees k_cnt <= 128 and the wlayout property; a tile with more terms
 * produces NaN rows and reports PCB_STATUS_TILE_TOO_LONG.
 * Replaces the same sum-layer kernels as pcb_lse_contract (small-K case).
 */
int pcb_lse_contract_short(const float* src, const float* src2, const float* aux, float* out, int64_t ld, int32_t B,
                           const float* params, const PcbLseTile* tiles, int32_t num_tiles, int32_t tile_rows,
                           int32_t rows_per_block, const int32_t* krow, const int32_t* kw, int32_t w_stride,
                           int32_t mode, int32_t prec, const uint8_t* packed, int32_t wlayout, int32_t batch_tile,
                           const PcbShortFusion* fusion, void* stream);

/*
 * One level of a pcb_lse_levels_short launch: a sum layer with the product layer below it
 * fused (the forward form of PcbShortFusion), its tiles being tiles[tile0 ..
 * tile0 + num_tiles) of the launch's concatenated tables.
 */
typedef struct {
    const uint8_t* packed;   /* reserved, NULL: each item converts its FP32 weights itself */
    float* element_out;      /* the product layer's element values (written as a side output) */
    int32_t tile0;
    int32_t num_tiles;
    int32_t rpb_log2;        /* rows per block of the level's tiles, base-2 logarithm */
    int32_t w_stride;
    int32_t row_splits;      /* 64-row items per tile: (tile rows + 63) / 64 */
    int32_t need;            /* items per sample slice of all earlier levels */
    int32_t wvec;            /* the weight layout of pcb_lse_contract_short's wlayout 1 */
    int32_t item0;           /* first work item of the level */
} PcbShortLevel;

/*
 * The forward of a run of consecutive small levels (each a product layer fused into the sum
 * layer above it, as pcb_lse_contract_short with PcbShortFusion.term_children) in one
 * persistent launch over node_mars. Work items (level, sample slice of batch_tile, tile,
 * 64-row split) are numbered level by level (item0 and need as in PcbShortLevel); num_ctas
 * CTAs take items from a counter in that order, and an item first waits (bounded) until
 * its sample slice has finished every item of the earlier levels: no grid-wide
 * synchronisation, since samples are independent. Same results as one
 * pcb_lse_contract_short launch per level (prec 0 FP32, 1 bf16, 2 split bf16). krow, kw and
 * term_children are the levels' tables concatenated (tile k_off indexing all three).
 * counters: a caller-owned int32 workspace of 1 + num_slices entries (zeroed here). A wait
 * that runs out reports PCB_STATUS_WAIT_TIMEOUT.
 * Replaces the reference's per-layer launches of the product and sum forward kernels
 * (prod_layer.py:160-204, sum_layer.py:454-568) for those levels.
 */
int pcb_lse_levels_short(float* node_mars, int64_t ld, int32_t B, const float* params, const PcbLseTile* tiles,
                         const int32_t* krow, const int32_t* kw, const int32_t* term_children,
                         const PcbShortLevel* levels, int32_t num_levels, int32_t total_items, int32_t num_slices,
                         int32_t* counters, int32_t prec, int32_t batch_tile, int32_t wk, int32_t num_ctas,
                         void* stream);

/*
 * Weights of LSE-contraction tiles (at most 128 rows x 128 terms each, same tile table,
 * kw, rows_per_block and w_stride as pcb_lse_contract) packed for
 * pcb_lse_contract_tc05: for tile t, 65536 bytes at packed + t * 65536 hold W(k, r)
 * rounded to bf16 (first 32 KB) and the bf16 rounding of the remainder (next 32 KB), in
 * the canonical no-swizzle K-major layout of a 128 x 128 tensor-core operand; rows and
 * terms beyond the tile are zero. packed must be 16-byte aligned.
 * No counterpart in the reference: its Triton kernels convert the weights inside each
 * contraction (sum_layer.py:534-541).
 */
int pcb_pack_weights(const float* params, const PcbLseTile* tiles, int32_t num_tiles, int32_t rows_per_block,
                     const int32_t* kw, int32_t w_stride, uint8_t* packed, void* stream);

/*
 * The same weights packed for the E4M3 form of pcb_lse_contract_tc05 (prec 3): for tile t,
 * at packed + t * 65536, 16384 bytes of e4m3 values W(k, r) * 448 / max_k W(k, r) in the
 * K-major no-swizzle layout of a 128 x 128 8-bit operand (core matrices of 8 rows x 16
 * terms; 128 bytes between core matrices along K, 1024 bytes between 8-row groups),
 * followed by 128 FP32 factors max_k W(k, r) / 448^2 (per-row scaling; rows and terms
 * beyond the tile are zero). packed must be 16-byte aligned.
 * No counterpart in the reference (its sum layers have no 8-bit form).
 */
int pcb_pack_weights_fp8(const float* params, const PcbLseTile* tiles, int32_t num_tiles, int32_t rows_per_block,
                         const int32_t* kw, int32_t w_stride, uint8_t* packed, void* stream);

/*
 * One tile table of a pcb_pack_weights_multi launch: the arguments of one
 * pcb_pack_weights call (rows_per_block as its base-2 logarithm).
 * No counterpart in the reference (see pcb_pack_weights).
 */
typedef struct {
    const PcbLseTile* tiles;
    const int32_t* kw;
    uint8_t* packed;             /* 16-byte aligned */
    int32_t num_tiles;
    int32_t rows_per_block_log2;
    int32_t w_stride;
    int32_t format;              /* 0: bf16 hi + lo (pcb_pack_weights), 1: e4m3 (pcb_pack_weights_fp8) */
} PcbPackJob;

/*
 * pcb_pack_weights for several tile tables in one launch (device arrays): global tile g
 * (g < total_tiles) is tile tile_index[g] of jobs[tile_job[g]]. The caller guarantees
 * tile_index[g] < that job's num_tiles. Same output as one pcb_pack_weights (format 0) or
 * pcb_pack_weights_fp8 (format 1) per job.
 * No counterpart in the reference (see pcb_pack_weights).
 */
int pcb_pack_weights_multi(const float* params, const PcbPackJob* jobs, const int32_t* tile_job,
                           const int32_t* tile_index, int32_t total_tiles, void* stream);

/*
 * Same contraction and epilogues as pcb_lse_contract (BF16 forms, prec 1 or 2) on the
 * tcgen05 tensor cores with tensor-memory accumulators, for tiles of at most 128 terms,
 * using the weights packed by pcb_pack_weights from the same tile table; prec 3 is the
 * E4M3 form (kind::f8f6f4 MMAs, FP32 accumulation) on weights packed by
 * pcb_pack_weights_fp8, with the exponentials scaled by 448 into e4m3. One CTA per tile
 * and run of slices_per_cta consecutive batch_tile-sample slices (batch_tile 32 or 64):
 * the packed weights are copied once per CTA, and the next slice's source values are
 * loaded while the current slice is processed. A tile with more terms produces NaN rows
 * (PCB_STATUS_TILE_TOO_LONG); a bounded wait that runs out NaN rows and
 * PCB_STATUS_WAIT_TIMEOUT.
 * Replaces the same reference kernels as pcb_lse_contract.
 */
int pcb_lse_contract_tc05(const float* src, const float* src2, const float* aux, float* out, int64_t ld, int32_t B,
                          const uint8_t* packed, const PcbLseTile* tiles, int32_t num_tiles, const int32_t* krow,
                          int32_t mode, int32_t prec, int32_t batch_tile, int32_t slices_per_cta, void* stream);

/*
 * pcb_lse_contract_tc05 for a later chunk of the tiles' terms: the tile table holds the
 * next (at most 128) terms of each tile, and the result is combined with out instead of
 * overwriting it: log(e^out + e^result) for the sum forward (mode 0), out + result for
 * the element flows (modes 1/2). A tile of more than 128 terms is contracted exactly by one
 * pcb_lse_contract_tc05 launch over its first 128 terms and one accumulating launch per
 * further 128 terms (each chunk with its own per-sample max).
 * Replaces the same reference kernels as pcb_lse_contract (sum_layer.py:454-568,
 * 1572-1730) for tiles of any length.
 */
int pcb_lse_contract_tc05_accum(const float* src, const float* src2, const float* aux, float* out, int64_t ld,
                                int32_t B, const uint8_t* packed, const PcbLseTile* tiles, int32_t num_tiles,
                                const int32_t* krow, int32_t mode, int32_t prec, int32_t batch_tile,
                                int32_t slices_per_cta, void* stream);

/*
 * Combine of long tiles contracted as chunks in one launch: every 128-term chunk j of the
 * tile holding output row dst_rows[r] wrote its partial result to row j * num_rows + r of
 * partials (pcb_lse_contract_tc05 on a table whose out_row fields point there);
 * out[dst_rows[r], b] = log sum_j exp(partial) (mode 0) or sum_j partial (modes 1/2), over
 * j < chunks_per_row[r], in that order.
 */
int pcb_chunk_combine(const float* partials, int64_t ld, int32_t B, int32_t num_rows, const int32_t* dst_rows,
                      const int32_t* chunks_per_row, float* out, int32_t mode, void* stream);

/*
 * pcb_lse_contract_tc05 as a persistent, warp-specialised kernel: num_ctas CTAs (0: one
 * per SM) each own a contiguous run of (tile, batch_tile-sample slice) work units. One warp
 * stages a unit's source rows in shared memory with 2-D TMA loads (a box of 32 samples x
 * run_rows rows, 128-byte swizzle) into a ring of stages, eight warps exponentiate into a
 * double-buffered B operand, one thread issues the MMAs into two tensor-memory
 * accumulators, and four warps run the epilogue, which writes 32-row x 32-sample blocks of
 * out through shared memory with TMA stores; loads, conversion, MMAs and stores of
 * consecutive units overlap, and the packed weights are copied once per tile and CTA.
 * The caller guarantees that every tile's terms form runs of run_rows (8 or 32) consecutive
 * source rows: krow[k_off + k] == krow[k_off + (k / run_rows) * run_rows] + k % run_rows
 * for k < k_cnt. src (and src2) have src_rows rows, out has out_rows rows. Same results and fault reporting as
 * pcb_lse_contract_tc05; additionally B % 4 == 0, ld % 4 == 0 and 16-byte aligned
 * src / src2 / aux / out (PCB_E_ARG otherwise).
 * Replaces the same reference kernels as pcb_lse_contract (sum_layer.py:454-568,
 * 1572-1730).
 */
int pcb_lse_contract_tc05_ws(const float* src, const float* src2, const float* aux, float* out, int64_t ld,
                             int32_t B, int64_t src_rows, int64_t out_rows, const uint8_t* packed, const PcbLseTile* tiles,
                             int32_t num_tiles, const int32_t* krow, int32_t mode, int32_t prec, int32_t batch_tile,
                             int32_t run_rows, int32_t num_ctas, void* stream);

/*
 * Sum layers under the MPE / GeneralLL propagation algorithms and the backward pass in
 * log space, with negated parameter flows or accumulated child flows (plain FP32; these
 * serve queries, not the EM step). alg: 0 LL, 1 MPE, 2 GeneralLL (alpha > 0).
 * pcb_sum_fwd_generic: forward over the forward tile table (same tiles, kw, rows_per_block
 *   and w_stride as pcb_lse_contract mode 0):
 *   LL log sum w exp(e); MPE max (log w + e);
 *   GeneralLL (log(sum w^alpha exp(alpha (e - m)) + 1e-24) + alpha m) / alpha, m = max e.
 *   Replaces the propagation_alg_id 1/2 branches of _fw_triton_block_sparse_*_kernel and
 *   _fw_triton_sparse_kernel (src/pyjuice/layer/sum_layer.py:454-568, 970-1037).
 * pcb_sum_ele_generic: element flows over an element-flow tile table (rows = child rows,
 *   krow = parent node rows, aux_row = the child's element_mars row):
 *   LL sum f w exp(e - m); MPE sum over parents with |log w + e - m| < 1e-6 of f;
 *   GeneralLL sum f w^alpha exp(alpha (e - m)); logspace = 1: flows are log flows and the
 *   sums are log-sum-exps; accumulate = 1 adds to (log-adds to) the existing flows.
 *   Replaces _bk_triton_block_sparse_ele_kernel / _bk_triton_sparse_ele_kernel in those
 *   modes (sum_layer.py:1572-1889, 2466-2666).
 * pcb_sum_par_generic: parameter flows over a parameter-flow tile table, summed over the
 *   batch and added (negate = 1: subtracted) with float atomics:
 *   LL / GeneralLL w sum_b f exp(e - m) (logspace: w sum_b exp(f + e - m), exp(f) where
 *   m = -inf); MPE sum_b [|log w + e - m| < 1e-6] f (logspace: exp(f)).
 *   Replaces _bk_triton_block_sparse_par_kernel / _bk_triton_sparse_par_kernel in those
 *   modes (sum_layer.py:2052-2169, 2795-2902).
 */
int pcb_sum_fwd_generic(const float* element_mars, float* node_mars, int64_t ld, int32_t B, const float* params,
                        const PcbLseTile* tiles, int32_t num_tiles, int32_t rows_per_block, const int32_t* krow,
                        const int32_t* kw, int32_t w_stride, int32_t alg, float alpha, void* stream);
int pcb_sum_ele_generic(const float* node_flows, const float* node_mars, const float* element_mars,
                        float* element_flows, int64_t ld, int32_t B, const float* params, const PcbLseTile* tiles,
                        int32_t num_tiles, int32_t rows_per_block, const int32_t* krow, const int32_t* kw,
                        int32_t w_stride, int32_t alg, float alpha, int32_t logspace, int32_t accumulate,
                        void* stream);
int pcb_sum_par_generic(const float* node_flows, const float* node_mars, const float* element_mars, int64_t ld,
                        int32_t B, const float* params, float* param_flows, const PcbPflowTile* tiles,
                        int32_t num_tiles, int32_t rows_per_block, const int32_t* cids, const int32_t* pids,
                        const int32_t* pfids, int32_t alg, int32_t logspace, int32_t negate, void* stream);

/*
 * In place on rows [row0, row1) of node_flows: f <- (m == -inf) ? -inf : log(f) - m.
 * Replaces SumLayer._bk_triton_modify_flow_kernel (src/pyjuice/layer/sum_layer.py:1355-1515).
 */
int pcb_modify_flows(float* node_flows, const float* node_mars, int64_t ld, int32_t B,
                     int64_t row0, int64_t row1, void* stream);

/*
 * Sum-layer parameter flows, contraction over the batch (see PcbPflowTile for the ids):
 *   pf(r, k) += params(r, k) * sum_b exp(lf[nid + r, b] - M_b) * exp(em[cids[k], b] + M_b)
 * with lf = node_flows already in "log f - log m" form (modified=1) or computed as
 * log(node_flows) - node_mars (modified=0), M_b the max over the tile's nodes.
 * The batch is split over a cluster of up to 8 CTAs (64-sample staged chunks; fewer CTAs
 * per cluster when the tiles alone fill the GPU) whose partial sums are added in a fixed order through distributed shared memory
 * (deterministic, no scratch memory). Tiles hold at most tile_children (32, 64 or 128)
 * children. prec: 0 = FP32 FMA, 1 = bf16 tensor cores, 2 = split bf16 (hi + lo, three
 * MMAs). atomic=1 when flow slots are shared by tied nodes.
 * Replaces SumLayer._bk_triton_block_sparse_par_kernel / _csmm2 / sparse par kernel
 * (src/pyjuice/layer/sum_layer.py:2052-2282, 2795-2902).
 */
int pcb_sum_pflows(const float* node_flows, const float* node_mars, const float* element_mars, int64_t ld, int32_t B,
                   const float* params, float* param_flows, const PcbPflowTile* tiles, int32_t num_tiles,
                   int32_t rows_per_block, const int32_t* cids, const int32_t* pids, const int32_t* pfids,
                   int32_t modified, int32_t atomic, int32_t tile_children, int32_t prec, void* stream);

/*
 * pcb_sum_pflows on the tcgen05 tensor cores (prec 1: bf16 operands, 2: split bf16 hi + lo,
 * three MMAs; tile_children 64 or 128): the [128 x tile_children] accumulator of a tile stays
 * in tensor memory over the CTA's batch slice; each 32-sample chunk is exponentiated into
 * K-major bf16 operands (K = samples) while the previous chunk's MMAs run. Same tiles,
 * results (up to the FP32 summation order), cluster reduction and flow-slot update as
 * pcb_sum_pflows. A bounded wait that runs out reports PCB_STATUS_WAIT_TIMEOUT (NaN flows).
 * Replaces the same reference kernels as pcb_sum_pflows.
 */
int pcb_sum_pflows_tc05(const float* node_flows, const float* node_mars, const float* element_mars, int64_t ld,
                        int32_t B, const float* params, float* param_flows, const PcbPflowTile* tiles,
                        int32_t num_tiles, int32_t rows_per_block, const int32_t* cids, const int32_t* pids,
                        const int32_t* pfids, int32_t modified, int32_t atomic, int32_t tile_children, int32_t prec,
                        void* stream);

/*
 * pcb_sum_pflows_tc05 over a tied set of sum layers (the time steps of a homogeneous HMM):
 * layers that share the tiles' parameters and flow slots, layer i's node rows and child
 * rows being the tiles' (tiles[].nid, cids[]) shifted by row_deltas[2 i] and
 * row_deltas[2 i + 1]. All num_layers layers' samples accumulate into one tensor-memory
 * tile per CTA and the flow slots are updated once, instead of once per layer.
 */
int pcb_sum_pflows_tc05_tied(const float* node_flows, const float* node_mars, const float* element_mars, int64_t ld,
                             int32_t B, const float* params, float* param_flows, const PcbPflowTile* tiles,
                             int32_t num_tiles, int32_t rows_per_block, const int32_t* cids, const int32_t* pids,
                             const int32_t* pfids, int32_t modified, int32_t atomic, int32_t tile_children,
                             int32_t prec, const int32_t* row_deltas, int32_t num_layers, void* stream);

/*
 * Sum-parameter EM update, per node block (FP64 normalisation):
 *   for node i < bs, child k < nch:   p = params[pbase + k * bs + i], f = pflows[pfbase + k * bs + i]
 *   theta' = (1 - s) * p + s * (f + pc / nch) / (sum_k f + pc)
 * keep_zero_params: zero parameters stay zero; the normaliser then counts pc / nch
 * only for non-zero parameters and adds no extra pc.
 * Replaces cum_pflow_kernel + em_par_update_kernel
 * (src/pyjuice/model/backend/par_update.py:174-256).
 */
int pcb_sum_em(float* params, const float* param_flows, const int64_t* blk_pbase, const int64_t* blk_pfbase,
               const int32_t* blk_nch, const int32_t* blk_bs, int32_t num_blocks,
               double step_size, double pseudocount, int32_t keep_zero_params, void* stream);

/*
 * FP64 epoch-level parameter flows. pcb_flows_accumulate_f64: acc[i] += flows[i] (i < n),
 * after each batch's FP32 parameter flows; pcb_pflow_accum_f64: pcb_pflow_accum on FP64
 * flows (tied slots summed into the source slot); pcb_sum_em_f64flows /
 * pcb_input_cat_em_f64flows: pcb_sum_em / pcb_input_cat_em reading FP64 flows.
 * The reference accumulates parameter flows over batches in FP32 with atomics
 * (src/pyjuice/layer/sum_layer.py:2167-2169, TensorCircuit.cumulate_flows
 * src/pyjuice/model/tensorcircuit.py:592-595) and runs the same EM update
 * (par_update.py:174-256, categorical.py:164-244); these keep the epoch's sum in FP64.
 */
int pcb_flows_accumulate_f64(double* acc, const float* flows, int64_t n, void* stream);
int pcb_pflow_accum_f64(double* param_flows, int64_t dst, int64_t n, const int64_t* srcs, int32_t nsrc, void* stream);
int pcb_sum_em_f64flows(float* params, const double* param_flows, const int64_t* blk_pbase, const int64_t* blk_pfbase,
                        const int32_t* blk_nch, const int32_t* blk_bs, int32_t num_blocks, double step_size,
                        double pseudocount, int32_t keep_zero_params, void* stream);
int pcb_input_cat_em_f64flows(float* params, const double* param_flows, const int32_t* s_pids,
                              const int32_t* s_pfids, const int32_t* ncats, const int32_t* source_nids,
                              int32_t num_source_nodes, double step_size, double pseudocount,
                              int32_t keep_zero_params, void* stream);

/*
 * Gradients with respect to softmax logits of the parameters (one softmax per node over
 * its children / categories), from parameter flows pf (theta times dLL/dtheta, as the
 * backward pass accumulates them with root weights dLoss/dLL):
 *   grad = scale * (pf - theta * sum_children pf)
 * written in the parameters' layout. pcb_sum_logit_grad uses the pcb_sum_em block table
 * (tied flow slots must be summed into the source slot first, pcb_pflow_accum);
 * pcb_input_cat_logit_grad the pcb_input_cat_em node table.
 * No counterpart in the reference (its parameters carry no autograd; the formula is the
 * softmax chain rule applied to its parameter flows, sum_layer.py:2052-2169).
 */
int pcb_sum_logit_grad(const float* params, const float* param_flows, const int64_t* blk_pbase,
                       const int64_t* blk_pfbase, const int32_t* blk_nch, const int32_t* blk_bs, int32_t num_blocks,
                       double scale, float* grad, void* stream);
/* Sum weights from logits: softmax over each node's children (pcb_sum_em block table; FP64
 * normaliser). No counterpart in the reference (its weights are not parameterised by logits). */
int pcb_sum_softmax(const float* logits, float* params, const int64_t* blk_pbase, const int32_t* blk_nch,
                    const int32_t* blk_bs, int32_t num_blocks, void* stream);
int pcb_input_cat_logit_grad(const float* params, const float* param_flows, const int32_t* s_pids,
                             const int32_t* s_pfids, const int32_t* ncats, const int32_t* source_nids,
                             int32_t num_source_nodes, double scale, float* grad, void* stream);

/*
 * Categorical input layer with soft evidence E (FP32, element (b, v, k) at
 * evidence[b * e_sb + v * e_sv + k * e_sk]):
 *   node_mars[node_offset + n, b] = min(log sum_{k < ncats} E[b, vids[n], k] params[s_pids[n] + k], 0)
 * (0 where `missing`, indexed as in pcb_input_cat_fwd, is set), over the variable-run
 * table of pcb_input_cat_bwd (max_group_nodes = the largest grp_count).
 * Replaces _soft_evi_categorical_fw_kernel and the clip that follows it
 * (src/pyjuice/queries/conditional.py:25-68, 108-111).
 */
int pcb_input_cat_soft_fwd(const float* evidence, int64_t e_sb, int64_t e_sv, int64_t e_sk, const float* params,
                           const int32_t* grp_var, const int32_t* grp_node0, const int32_t* grp_count,
                           const int32_t* grp_ncats, int32_t num_groups, int32_t max_group_nodes,
                           const int32_t* s_pids, int32_t node_offset, float* node_mars, int64_t ld, int32_t B,
                           const uint8_t* missing, int64_t miss_sb, int64_t miss_sv, void* stream);

/*
 * Per-category evidence quantities from the node flows of an input layer, for target
 * variable t (its nodes: tgt_nodes[tgt_ptr[t] .. tgt_ptr[t + 1]), layer-local ids):
 *   out[(b * num_targets + t) * max_ncats + k] = sum_n W[n, b] params[s_pids[n] + k]
 * mode 0: W = node flows (the conditional query's category weights before their
 * normalisation over k; replaces _categorical_backward_kernel, conditional.py:241-336,
 * which adds the same terms with float atomics);
 * mode 1: W = node flows / exp(node_mars) (0 where node_mars = -inf): the derivative of the
 * weighted log-likelihood with respect to the soft evidence E[b, v, k] of the
 * soft-evidence forward (no reference counterpart).
 * Deterministic (every output is one sum in node order); entries k >= a node's ncats
 * receive no term.
 */
int pcb_input_cat_evidence_bwd(const float* node_flows, const float* node_mars, int64_t ld, int32_t B,
                               const float* params, const int32_t* tgt_ptr, const int32_t* tgt_nodes,
                               int32_t num_targets, const int32_t* s_pids, const int32_t* ncats, int32_t node_offset,
                               int32_t max_ncats, int32_t mode, float* out, void* stream);

/*
 * Sum-parameter normalisation (FP64), same block table as pcb_sum_em:
 *   theta' = (p + pc / nch) / (sum_k p + pc)
 * Replaces cum_par_kernel + par_update_kernel (src/pyjuice/model/backend/normalize.py:13-68).
 */
int pcb_sum_normalize(float* params, const int64_t* blk_pbase, const int32_t* blk_nch, const int32_t* blk_bs,
                      int32_t num_blocks, double pseudocount, void* stream);

/*
 * Log-likelihood reduction in FP64: out[0] += sum_b lls[row * ld + b] for b < B.
 * Dataset-level LL accumulation.
 * No kernel counterpart in the reference (its callers sum log-likelihoods with torch).
 */
int pcb_ll_sum_f64(const float* lls, int64_t ld, int32_t B, int64_t row, double* out, void* stream);

/*
 * Ancestral sampling (replaces queries.sample: sample_sum_layer_kernel, count_prod_nch_kernel,
 * sample_prod_layer_kernel and the Categorical sample kernel; src/pyjuice/queries/sample.py:38-474,
 * src/pyjuice/layer/input_layer.py:1222-1249, categorical.py:137-161).
 * Per sample s, nlist[s * cap_n + j] (j < ncnt[s]) are its active node ids and
 * elist[s * cap_e + j] (j < ecnt[s]) its active element ids. Uniform draws are
 * u(seed, id, s) = top 24 bits of SplitMix64(seed + ((id << 32) | s + 1) * 0x9E3779B97F4A7C15) / 2^24,
 * or, when `uniforms` is not NULL, uniforms[id * u_ld + s] (a [num_nodes, u_ld >= S] FP32
 * table, so that the draws of another sampler, e.g. the reference's tl.rand draws as
 * recorded per node and sample, are replayed exactly; seed is then unused).
 * *err is set to 1 on list overflow, 2 on an element outside the product group.
 *
 * pcb_sample_sum: nodes of the sum layer [lo, hi) (block size bs) choose the first child
 * k with u < cumsum_k(params[kw[k] + i]) (the last non-zero child if rounding leaves none);
 * the node's block is node2blk[(id - lo) / bs] in the forward tables (blk_nid, blk_koff,
 * blk_kcnt, krow = child element ids, kw = parameter bases).
 * pcb_sample_prod: active elements in [elo, ehi) append their children (chs[blk_off[g] + c] + i);
 * elements of other product layers stay in the element list.
 * pcb_sample_input: active input nodes in [lo, hi) draw category k = first k with
 * u <= cumsum_k (0 if none) into samples[s * sld + vids[id - lo]].
 */
int pcb_sample_sum(int32_t* nlist, int32_t* ncnt, int32_t* elist, int32_t* ecnt, int32_t S, int32_t cap_n,
                   int32_t cap_e, int32_t lo, int32_t hi, int32_t bs, const int32_t* node2blk, const int32_t* blk_nid,
                   const int32_t* blk_koff, const int32_t* blk_kcnt, const int32_t* krow, const int32_t* kw,
                   const float* params, const float* uniforms, int64_t u_ld, uint64_t seed, int32_t* err,
                   void* stream);
int pcb_sample_prod(int32_t* nlist, int32_t* ncnt, int32_t* elist, int32_t* ecnt, int32_t S, int32_t cap_n,
                    int32_t cap_e, int32_t elo, int32_t ehi, const int32_t* elem2blk, const int32_t* blk_row,
                    const int32_t* blk_off, const int32_t* blk_cnt, const int32_t* chs, int32_t* err, void* stream);
int pcb_sample_input(const int32_t* nlist, const int32_t* ncnt, int32_t S, int32_t cap_n, int32_t lo, int32_t hi,
                     const int32_t* vids, const int32_t* s_pids, const int32_t* ncats, const float* params,
                     int64_t* samples, int64_t sld, const float* uniforms, int64_t u_ld, uint64_t seed, void* stream);
/*
 * pcb_sample_input for a SoftEvidenceCategorical layer: node n of sample s draws category k
 * with probability theta[n, k] exp(L[s, u, k]) / sum_k' (...) over k < K, L the evidence
 * log-weights at evidence_logp + s e_sb + u e_su + k and u = node_lvid[n] (layer-local n);
 * the first k whose cumulative probability exceeds the uniform (the last category if rounding
 * leaves none). Replaces sample_kernel (softevi_categorical.py:683-761).
 */
int pcb_sample_input_poe(const int32_t* nlist, const int32_t* ncnt, int32_t S, int32_t cap_n, int32_t lo, int32_t hi,
                         const int32_t* vids, const int32_t* s_pids, const int32_t* node_lvid, const float* params,
                         const float* evidence_logp, int64_t e_sb, int64_t e_su, int32_t K, int64_t* samples,
                         int64_t sld, const float* uniforms, int64_t u_ld, uint64_t seed, void* stream);
/*
 * pcb_sample_input for Bernoulli (kind 1), Gaussian (kind 2) and DiscreteLogistic (kind 3)
 * layers, one uniform u per (node, sample) as for pcb_sample_input, values written as FP32
 * into samples[s * sld + var]: Bernoulli 1 if u < p else 0; Gaussian mu + sigma Phi^-1(u)
 * (u moved inside (0, 1)); DiscreteLogistic the bin of mu + s log(u / (1 - u)) among the
 * num_cats bins of [lo, hi), clamped to the first and last bin; meta as for
 * pcb_input_dist_fwd (kind 3 only). Replaces the sample_fn of bernoulli.py:79-88,
 * gaussian.py:114-125 and discrete_logistic.py:157-181.
 */
int pcb_sample_input_dist(int32_t kind, const int32_t* nlist, const int32_t* ncnt, int32_t S, int32_t cap_n, int32_t lo,
                          int32_t hi, const int32_t* vids, const int32_t* s_pids, const float* meta,
                          const float* params, float* samples, int64_t sld, const float* uniforms, int64_t u_ld,
                          uint64_t seed, void* stream);

/*
 * Whole-circuit sampling that allocates nothing. No counterpart in the reference: the
 * reference samples layer by layer with host-side tensors; this entry point exists for
 * callers that may not allocate device memory when they sample (a fixed pre-reserved
 * memory pool, a plugin inside another framework's allocator, a loop that must not call
 * cudaMalloc because it can synchronise the device). Neither this function nor its
 * kernel allocates; the caller passes only inputs and outputs.
 *
 * One step per layer, in the order the per-layer entry points above would be called
 * (sum and product layers top-down, then the input layers); the table lives in device
 * memory the caller owns. Draws are the same as pcb_sample_sum / pcb_sample_prod /
 * pcb_sample_input with the same seed, so the samples are identical.
 *   kind 0 (sum layer, nodes [lo, hi), block size bs): node2blk, blk_first (= blk_nid),
 *          blk_off, blk_cnt, children (= krow), weight_base (= kw), params.
 *   kind 1 (product layer, elements [lo, hi)): node2blk (= elem2blk), blk_first (= blk_row),
 *          blk_off, blk_cnt, children (= chs).
 *   kind 2 (input layer, nodes [lo, hi)): vids, s_pids, ncats, params.
 *
 * Working lists: S * (cap_n + cap_e) int32 in a fixed 8 MiB device array inside the
 * library (PCB_SAMPLE_NOALLOC_MAX_INTS entries); larger requests are rejected with
 * PCB_E_ARG before anything is launched (sample in smaller batches). The array is per
 * device and shared by all calls: two calls that overlap in time on the same device
 * (two streams, two host threads) overwrite each other's lists, so serialise them.
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress; with lazy module loading the runtime loads the module and
 * reserves the array at that point); make that first call before any stream capture.
 * *err is set to zero by the call (cudaMemsetAsync on `stream`), then to 1 on list
 * overflow, 2 on an element outside its product layer, 3 on a malformed step (kind not
 * 0, 1 or 2, or a sum step with bs <= 0; that sample stops there). samples[s * sld + v]
 * is written for every variable v that sample s draws; other entries are left as they are.
 * The kernel runs on the current device, which must be the device that holds the step
 * table, the tables it points to and the buffers.
 */
#define PCB_SAMPLE_NOALLOC_MAX_INTS (1 << 21)
typedef struct {
    int32_t kind, lo, hi, bs;
    const int32_t* node2blk;
    const int32_t* blk_first;
    const int32_t* blk_off;
    const int32_t* blk_cnt;
    const int32_t* children;
    const int32_t* weight_base;
    const float* params;
    const int32_t* vids;
    const int32_t* s_pids;
    const int32_t* ncats;
} PcbSampleStep;
int pcb_sample_circuit_noalloc(const PcbSampleStep* steps, int32_t num_steps, int32_t root_id, int32_t S,
                               int32_t cap_n, int32_t cap_e, int64_t* samples, int64_t sld, uint64_t seed,
                               int32_t* err, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PCB200_H */
