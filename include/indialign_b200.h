/* indialign_b200 -- B200 (sm_100a) implementation of INDIalign's RNA TM-score
 * superposition search, behind the reference's C ABI.
 *
 * The first four entry points and the three structs are drop-ins for the
 * reference's (indialign_c/api.h:10-46): same names, field order and sizes
 * (x86-64: 56 / 56 / 104 bytes), same argument meaning and return codes.
 * Differences a caller can see:
 *   - the search runs on the GPU; request_cuda and backend_mode are ignored
 *     (there is no CPU path and no CPU fallback);
 *   - a CUDA failure returns a negative code (INDIALIGN_E_*) instead of
 *     silently falling back; the reference has no such case.
 * Ownership is unchanged: all pointers are caller-owned host memory, the
 * library reads 3N doubles per coordinate array and N bytes per mask and
 * writes only *out / outputs[].  Calls are thread-safe (each call takes its
 * own stream and workspace from an internal pool).
 */
#ifndef INDIALIGN_B200_H
#define INDIALIGN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces NativeConfig (indialign_c/api.h:10-20). */
typedef struct {
    int backend_mode;        /* ignored (the reference ignores it too) */
    int use_fragment_search;
    int max_iter;
    int dp_iter;
    double max_mem_gb;       /* device workspace budget per call */
    int request_cuda;        /* ignored: always CUDA */
    double rescue_score_1;   /* trigger rescue if score < this (default 0.5) */
    double rescue_score_2;   /* trigger dense rescue if score < this (default 0.3) */
    double early_term_score; /* skip remaining seeds if score >= this (default 0.99) */
} NativeConfig;

/* Replaces NativePairInput (indialign_c/api.h:22-30). */
typedef struct {
    int length;
    const double *pred_xyz;          /* 3*length, xyz interleaved */
    const double *native_xyz;        /* 3*length */
    const uint8_t *valid_mask;       /* length; expected pred_valid & native_valid */
    const uint8_t *pred_valid_mask;  /* length */
    const uint8_t *native_valid_mask;/* length */
    double lnorm;                    /* TM normalisation length */
} NativePairInput;

/* Replaces NativePairResult (indialign_c/api.h:32-36).  aligned_d =
 * sum_k pred_k * rotation[3k+d] + translation[d]. */
typedef struct {
    double score;
    double rotation[9];
    double translation[3];
} NativePairResult;

enum {
    INDIALIGN_OK = 0,
    INDIALIGN_E_LENGTH = -1,   /* length <= 0 (reference behaviour) */
    INDIALIGN_E_NODEVICE = -2, /* no usable CUDA device */
    INDIALIGN_E_CUDA = -3,     /* CUDA runtime error (see indialign_last_error) */
    INDIALIGN_E_INPUT = -4,    /* null pointer or length above 65535 */
    INDIALIGN_E_DEVICE = -5,   /* device-side error flag (bounded wait / capacity) */
    INDIALIGN_E_INJECTED = -6  /* failure injected by the test hook */
};

/* Replaces indialign_default_config (indialign_c/indialign.cpp:272-282). */
void indialign_default_config(NativeConfig *cfg);

/* Replaces indialign_tmscore_search (indialign_c/indialign.cpp:284-303).
 * Returns -1 iff length <= 0 (out untouched), 0 on success, another
 * negative INDIALIGN_E_* code on a CUDA failure (out untouched). */
int indialign_tmscore_search(const NativePairInput *inp, const NativeConfig *cfg,
                             NativePairResult *out);

/* Replaces indialign_tmscore_search_batch (indialign_c/indialign.cpp:305-313).
 * All pairs run in one device pass.  Pairs with length <= 0 are skipped and
 * their outputs left untouched, as the reference does.  Returns 0, or a
 * negative code on a CUDA failure (then no output is written). */
int indialign_tmscore_search_batch(int n_pairs, const NativePairInput *inputs,
                                   const NativeConfig *cfg, NativePairResult *outputs);

/* Replaces indialign_cuda_available (indialign_c/indialign.cpp:315-321):
 * 1 when a CUDA device of compute capability 10.x is usable, else 0. */
int indialign_cuda_available(void);

/* ---- extensions (no counterpart in the reference's api.h) -------------- */

/* Per-call options for the batched entry points.  Zero-initialise. */
typedef struct {
    void *stream;            /* cudaStream_t to run on (NULL: library stream) */
    int device;              /* CUDA device ordinal (-1: current) */
    int use_graph;           /* reserved: accepted and ignored (the stage kernels are persistent) */
    int profile;             /* 1: print per-stage device times to stderr */
    double *stage_ms;        /* optional [INDIALIGN_STAGES] per-stage device ms:
                                seeds, seed bank, SS, gapless, local fragment,
                                threading DP, dense local fragment, top-k, DP
                                refinement, offset DP, weighted, total */
    long long *counters;     /* optional [INDIALIGN_COUNTERS] work counters: NW cells,
                                chain residue visits, bank residue visits, bank
                                items, chains, NW-chain kernel launches, bank
                                kernel launches, all kernel launches, then SM
                                cycles summed over warps in NW fill, traceback,
                                detailed refinement, alignment Kabsch */
    double *kernel_ms;       /* optional [6]: summed device ms of the NW-chain
                                kernel and of the bank kernel, their launch counts,
                                then ms and launches of the window-ranker kernel */
    double *stage_best;      /* optional [n_pairs*INDIALIGN_TRACE_STAGES*13]: running
                                best {score,R,t} after each search stage */
    /* ---- learned candidate ranker ----
     * The local-fragment, threading-DP and dense local-fragment passes
     * (rescue.h) each refine a list of candidate starts per pair (windows /
     * offsets), and every detailed search (align.h:15-50, in the SS seeds
     * and in dp_refine) refines a list of fragment seeds of an alignment
     * (INDIALIGN_CAND_*).  LEARNED mode scores them with the ranker and
     * refines the top_k of each pair (of each alignment for detailed
     * searches); the main seed bank's seeds can be ranked too
     * (INDIALIGN_RANK_MAIN).  Per-candidate arrays below hold the five kinds
     * back to back, each kind pair by pair, pair p with
     * indialign_candidate_count(plen_p, nlen_p, kind) entries (detailed
     * searches: two alignment slots of equal size; COLLECT keeps the last
     * detailed search that ran on a slot, normally dp_refine's). */
    int mode;                /* INDIALIGN_MODE_PLAIN (0), _LEARNED or _COLLECT */
    const float *ranker;     /* LEARNED (or COLLECT with predictions): host FP32
                                parameter blob of INDIALIGN_RANKER_FLOATS floats */
    int top_k;               /* LEARNED: candidates refined per pair (1..32; 0: 8) */
    double margin;           /* LEARNED: refine all candidates when the predicted
                                top-1 minus top-k score is below this */
    double audit_rate;       /* LEARNED: fraction of pairs refined on all candidates */
    unsigned long long seed; /* LEARNED: audit draw */
    long long *rank_stats;   /* LEARNED: optional [INDIALIGN_RANK_STATS] out, per kind
                                10 counts summed over the batch's searches: lists
                                ranked, margin fallbacks, audits, pruned lists,
                                candidates, candidates refined, audit misses (the
                                top_k's best refined score below the list's best),
                                lists with at most top_k candidates, audit misses by
                                more than 1e-4, by more than 1e-3 */
    float *win_feat;         /* COLLECT: out [candidates][16] raw features */
    float *win_label;        /* COLLECT: out [candidates] refined score, NaN where
                                the pair's pass did not run */
    long long win_cap;       /* COLLECT, or with win_score: capacity of the
                                per-candidate outputs */
    float *win_score;        /* optional out [candidates] (LEARNED, or COLLECT with a
                                ranker): predicted score of every candidate */
    int rank_mask;           /* LEARNED / COLLECT: INDIALIGN_RANK_* bits of the lists
                                to rank (0: INDIALIGN_RANK_DEFAULT) */
    int rank_min_len;        /* LEARNED: pairs with fewer valid pred or native
                                residues refine every candidate (0:
                                INDIALIGN_RANK_MIN_LEN; negative: rank all) */
    int *win_select;         /* optional out [6*n_pairs][33] (LEARNED): rows per kind
                                back to back (n_pairs each, 2*n_pairs alignment
                                slots for detailed searches, the batch's last one):
                                candidates refined (-1: all, margin fallback, not
                                run or at most top_k; -2: all, audit), then the
                                top_k candidates ascending */
} IndialignBatchOptions;

#define INDIALIGN_MODE_PLAIN 0   /* the reference's search, every candidate refined */
#define INDIALIGN_MODE_LEARNED 1 /* rescue passes refine the ranker's top-k candidates */
#define INDIALIGN_MODE_COLLECT 2 /* plain search + per-candidate features and labels */
#define INDIALIGN_CAND_LOCAL 0   /* local-fragment windows (rescue.h:50-117) */
#define INDIALIGN_CAND_THREAD 1  /* threading-DP offsets (rescue.h:121-190) */
#define INDIALIGN_CAND_DENSE 2   /* dense local-fragment windows */
#define INDIALIGN_CAND_DET 3     /* detailed-search fragment seeds (align.h:15-50) */
#define INDIALIGN_CAND_MAIN 4    /* main seed-bank seeds (windows + anchors, seeds.h:41-283) */
#define INDIALIGN_RANK_LOCAL 1   /* local-fragment windows */
#define INDIALIGN_RANK_THREAD 2  /* threading-DP offsets */
#define INDIALIGN_RANK_DENSE 4   /* dense local-fragment windows */
#define INDIALIGN_RANK_DET_SS 8  /* detailed searches of the SS seeds (ss.h:87-164) */
#define INDIALIGN_RANK_DET_DP 16 /* detailed searches of the final dp_refine (indialign.cpp:188-193) */
#define INDIALIGN_RANK_MAIN 32   /* the main seed bank (indialign.cpp:90-104); not in the
                                    default: pruning it measured worst TM changes ~1e-2 */
/* default: every list but the final dp_refine's detailed searches, which
 * stay exhaustive so that the final refinement of the best transform is the
 * plain search's (measured: pruning them too costs most of the worst-case
 * TM-score loss for a few percent of speed) */
#define INDIALIGN_RANK_DEFAULT (INDIALIGN_RANK_LOCAL | INDIALIGN_RANK_THREAD | INDIALIGN_RANK_DENSE | \
                                INDIALIGN_RANK_DET_SS)
/* short pairs cost little and lose most from pruning (measured on the hard
 * workload: the worst TM-score changes were pairs of L < 50) */
#define INDIALIGN_RANK_MIN_LEN 100
#define INDIALIGN_RANKER_FLOATS 18849
#define INDIALIGN_RANK_STATS 50

/* Stages recorded in stage_best, in search order: seed bank, SS seeds,
 * gapless threading, local fragment DP, threading DP, dense local fragment
 * DP, top-k seed, DP refinement, offset DP, weighted refinement. */
#define INDIALIGN_TRACE_STAGES 10

#define INDIALIGN_STAGES 12
#define INDIALIGN_COUNTERS 12

/* Batched search with per-call options.  Same inputs and outputs as
 * indialign_tmscore_search_batch. */
int indialign_tmscore_search_batch_ex(int n_pairs, const NativePairInput *inputs,
                                      const NativeConfig *cfg,
                                      const IndialignBatchOptions *opts,
                                      NativePairResult *outputs);

/* Device-resident batch: pairs packed back to back on the device.
 * off[n+1] residue offsets (host array), d_pred/d_nat [3*total] doubles,
 * d_v/d_pv/d_nv [total] bytes, lnorm[n] (host array); results written to
 * d_out [n*13] doubles on the device ({score, R[9], t[3]} per pair).  Used by
 * the torch shim; every pointer named d_* is device memory. */
int indialign_tmscore_search_device(int n_pairs, const int *off, const double *d_pred,
                                    const double *d_nat, const uint8_t *d_v,
                                    const uint8_t *d_pv, const uint8_t *d_nv,
                                    const double *lnorm, const NativeConfig *cfg,
                                    const IndialignBatchOptions *opts, double *d_out);

/* Padded device batch, the (B, N, 3) shape of the reference's torch scorer
 * (scoring/_tmscore_gpu/search.py:492-540): row p of d_pred / d_nat [B*N*3]
 * and of the masks d_v / d_pv / d_nv [B*N] holds pair p in its first
 * lengths[p] (host array, 1..N) residues; lnorm[B] host array; results
 * {score, R[9], t[3]} to d_out [B*13] on the device.  The search of each pair
 * is the reference's (only the first lengths[p] residues take part). */
int indialign_tmscore_search_padded(int n_pairs, int N, const int *lengths, const double *d_pred,
                                    const double *d_nat, const uint8_t *d_v, const uint8_t *d_pv,
                                    const uint8_t *d_nv, const double *lnorm, const NativeConfig *cfg,
                                    const IndialignBatchOptions *opts, double *d_out);

/* Needleman-Wunsch alignment of one explicit score matrix; replaces the
 * reference's nw_dp + nw_traceback pair (indialign_c/nw.h:10-68): zero
 * boundaries, a gap move out of a diagonally reached cell pays `gap`, ties
 * prefer diag, then left, then up; the traceback starts at (np, nn).
 * d_smat: np*nn doubles, row-major, device memory.  Writes the aligned
 * (pred, native) index pairs in ascending order to d_ap/d_an (device,
 * min(np,nn) ints each) and their count to *d_na (device int).  Synchronous
 * on `stream` (NULL: the library's stream).  1 <= np, nn <= 65535. */
int indialign_nw_align(const double *d_smat, int np, int nn, double gap, int *d_ap, int *d_an,
                       int *d_na, void *stream);

/* indialign_nw_align without any device allocation (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc when they align: hosts
 * whose device memory belongs to a framework's pool allocator, or paths that
 * forbid driver allocations.  Same arguments, kernel and outputs
 * as indialign_nw_align; the caller passes device inputs and outputs, the
 * scratch lives in a fixed device array of about 1.1 MB that every GPU using
 * the library keeps until exit.  Limit: 1 <= np, nn <= 2048, else
 * INDIALIGN_E_INPUT.  The first call on a device looks the array up with
 * cudaGetSymbolAddress.  All calls share
 * the array: calls whose work overlaps on the GPU race.  stream NULL is the
 * legacy default stream; the call returns after the stream synchronizes. */
int indialign_nw_align_noalloc(const double *d_smat, int np, int nn, double gap, int *d_ap,
                               int *d_an, int *d_na, void *stream);

/* ---- one batch over several GPUs of this process (no counterpart in the
 * reference, which parallelises over pairs with OpenMP only,
 * indialign_c/indialign.cpp:305-313).  Pairs are independent, so the split
 * needs no collective. */

/* Estimated device work of every pair (NW-cell units): the always-run passes
 * and the seed bank, plus the rescue passes' NW cells (windows and offsets
 * from rescue.h:12-46, 136-142) weighted by how likely they run, judged from
 * the pair's TM-score under one Kabsch superposition of all valid residues
 * (written to tm0[n] when tm0 is not NULL).  Host only, no device work. */
int indialign_pair_costs(int n_pairs, const NativePairInput *inputs, double *cost, double *tm0);

/* shard_of[p] in 0..n_shards-1: longest-processing-time split of the batch
 * by indialign_pair_costs (costliest pair first onto the least-loaded shard;
 * ties to the lower index).  Deterministic, so every rank of a multi-process
 * job computes the same split.  Host only. */
int indialign_shard_pairs(int n_pairs, const NativePairInput *inputs, int n_shards, int *shard_of);

/* indialign_tmscore_search_batch_ex over devices[0..n_devices-1] (a device
 * may be listed more than once): indialign_shard_pairs split, one host thread
 * and library context per shard, results in batch order.  opts may carry the
 * search mode and the aggregate outputs (stage_ms: the slowest shard's;
 * counters, kernel_ms, rank_stats: summed); a caller stream and the
 * per-pair outputs (stage_best, win_*) are per-device and rejected with
 * INDIALIGN_E_INPUT.  The first failing shard's code is returned. */
int indialign_tmscore_search_multi(int n_pairs, const NativePairInput *inputs, const NativeConfig *cfg,
                                   const IndialignBatchOptions *opts, const int *devices, int n_devices,
                                   NativePairResult *outputs);

/* Candidates of kind INDIALIGN_CAND_* of a pair with plen / nlen valid pred /
 * native residues (the schedules of rescue.h:12-46 and :136-142; for
 * detailed searches the room of both alignment slots). */
int indialign_candidate_count(int plen, int nlen, int kind);

/* ---- ranker training on caller-owned device buffers (no counterpart in the
 * reference, which has no learned component).  The parameter blob is FP32:
 * mean[16] std[16] W1[16][128] b1[128] W2[128][128] b2[128] w3[128] b3, weights
 * [in][out]; mean/std standardise the raw features and are not trained.  The
 * network runs on BF16 tensor cores with FP32 accumulation.  All calls are
 * asynchronous on `stream` (NULL: legacy default stream). */
size_t indialign_mlp_packed_bytes(void);
/* BF16 / layout copy of a device blob, read by the forward and backward. */
int indialign_mlp_pack(const float *d_blob, void *d_packed, void *stream);
size_t indialign_mlp_save_bytes(int n);
/* y[n] = MLP(x[n][16]); with d_save (indialign_mlp_save_bytes(n) bytes) the
 * activations the backward needs are kept. */
int indialign_mlp_forward(const void *d_packed, const float *d_x, int n, float *d_y,
                          void *d_save, void *stream);
/* Loss = mean squared error + lambda * mean logistic ranking loss over the
 * row pairs (2i, 2i+1); writes d_dy[n] = dLoss/dy and d_loss[0]. */
int indialign_mlp_loss(const float *d_y, const float *d_t, int n, float lambda, float *d_dy,
                       float *d_loss, void *stream);
size_t indialign_mlp_work_bytes(int n);
/* Gradients of sum_i dy[i] y[i] w.r.t. the blob, written to d_grad
 * (INDIALIGN_RANKER_FLOATS floats; the mean/std entries are zeroed).  d_save
 * from the forward on the same rows; d_work of indialign_mlp_work_bytes(n). */
int indialign_mlp_backward(const void *d_packed, const float *d_dy, int n, const void *d_save,
                           float *d_grad, void *d_work, void *stream);
/* C[m][n] = A . B^T on the tcgen05 tensor cores (BF16 in, FP32 out), the
 * product the backward's three weight/activation gradients use.  A is K-major
 * ([m][lda] row-major, a_mn = 0) or MN-major ([k][lda], a_mn = 1, m <= 128);
 * B is K-major ([n][ldb]) or MN-major ([k][ldb]), n <= 256; lda, ldb multiples
 * of 8 elements, 16-byte aligned device pointers.  C has row stride ldc, or is
 * written transposed (C[j][i] at j * ldc + i) with c_trans.  splits > 1 splits
 * k over partial tiles in d_partial (splits x m x n floats), added in a fixed
 * order.  INDIALIGN_E_INPUT on a shape it does not take. */
int indialign_gemm_bf16(const void *d_a, int lda, int a_mn, const void *d_b, int ldb, int b_mn, int m, int n,
                        int k, float *d_c, int ldc, int c_trans, float *d_partial, int splits, void *stream);
/* One Adam step (bias-corrected, step >= 1) on the trained blob entries. */
int indialign_mlp_adam(float *d_blob, const float *d_grad, float *d_m, float *d_v, int step,
                       float lr, float beta1, float beta2, float eps, void *stream);

/* Measured FP64 FMA throughput of the device in TFLOP/s (the roofline
 * denominator for the FP64 SIMT kernels: NW chains, Kabsch). */
int indialign_fp64_peak(int device, double *tflops);

/* Measured FP32 FMA throughput of the device in TFLOP/s (the roofline
 * denominator for the seed-bank kernel, whose residue visits run in FP32). */
int indialign_fp32_peak(int device, double *tflops);

/* Diagnostic: y[i] = the search kernels' Newton-Raphson reciprocal of x[i],
 * computed on the device (host arrays of n doubles). */
int indialign_selftest_rcp(int n, const double *x, double *y);

/* Diagnostic: R[9i..9i+8] = the search kernels' rotation (Horn quaternion,
 * aligned_d = sum_k p_k R[3k+d]) for the 3x3 covariance H[9i..9i+8] (row
 * major, sum of p q^T), computed on the device (host arrays of n matrices);
 * the counterpart of the reference's cov_to_rotation (indialign_c/core.h:64-90). */
int indialign_selftest_rotation(int n, const double *H, double *R);

/* ---- length buckets and kernel shapes (no counterpart in the reference,
 * whose only shape choice is the block size of its GPU seed-bank kernel by
 * N, indialign_c/gpu_kernels.cu:227-229).  Every pair's work runs with the
 * kernel shapes of its length bucket; with split = 1 a batch whose pairs
 * span buckets runs as one sub-batch per bucket, side by side on the device.
 * Results are those of one call either way.  The table comes from
 * tune_b200.txt beside the library (or the file named by
 * INDIALIGN_TUNE_TABLE), written by indialign_b200/autotune.py.
 * Rows: {max_len, bank_chunk (items per CTA chunk, multiple of 32, 32..4096),
 * bank_cutoff_major (0/1: item order), chain_chunk (NW chains per CTA chunk,
 * 1..256), chain_smem_trace (0/1: NW traces in shared memory when they fit
 * without losing occupancy)}, max_len ascending (the last bucket takes every
 * longer pair). */
#define INDIALIGN_TUNE_BUCKETS 3
#define INDIALIGN_TUNE_FIELDS 5
/* The table in use: split (0/1), min_pairs (batches with fewer pairs are not
 * split), rows [INDIALIGN_TUNE_BUCKETS][INDIALIGN_TUNE_FIELDS]. */
int indialign_get_tuning(int *split, int *min_pairs, int *table);
/* Replace the table for this process (table NULL: reload it from its file);
 * INDIALIGN_E_INPUT on an invalid row. */
int indialign_set_tuning(int split, int min_pairs, const int *table);

/* Text of the last error on this thread ("" if none). */
const char *indialign_last_error(void);

/* Test hook: make the next `count` calls fail with INDIALIGN_E_INJECTED
 * before any device work, to exercise callers' failure paths without a GPU
 * fault.  0 disarms. */
void indialign_inject_failure(int count);

#ifdef __cplusplus
}
#endif

#endif
