// Launch wrappers of the search kernels (host-callable, C++).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "pipeline.h"

namespace ia {

constexpr size_t kBankSmemMax = 200 * 1024;
constexpr size_t kChainSmemMax = 220 * 1024;

// Packed batch in device memory (see pipeline.h).  All arrays carry >= 64
// bytes of tail padding so rounded-up bulk copies stay inside them.
struct DevBatch {
    int n;
    const int *off;        // [n+1] residue offsets (even)
    const int *len;        // [n]
    const double *lnorm;   // [n]
    const double *pred, *nat;             // [3*total]
    const uint8_t *v, *pv, *nv;           // [total]
    PairInfo *info;        // [n]
    PairState *state;      // [n]
    int *pmap, *nmap, *vmap;              // [total]
    int *scratch;          // [total + n] per-residue ints
    double *dscr;          // [total] per-residue doubles
    double *predc, *natc;  // [3*total] compacted coordinates
    char *sspc, *ssnc;     // [total] compact SS labels
    int2 *seeds;           // [n*kMaxSeeds]
    int2 *topk_seed;       // [n]
    uint32_t *bits;        // bitmask seeds
    const int *bitoff;     // [n] first word of a pair's bitmask block
    uint64_t *hashes;      // [n*kMaxSeeds] seed hashes (dedup)
    int *kv;               // [2*total] sort records / SS partners
    const uint64_t *fnv_pow;  // [maxN+1] FNV prime powers
    int *err;              // device error word
    unsigned long long *ctr;  // [kCounters] work counters (see enum Counter)
    const int *gidx;       // [n] index of each pair in the caller's batch (a
                           // length bucket's sub-batch), or null: p itself
    const int *out_map;    // [n] result row of each pair in the caller's
                           // output (sub-batch), or null: p itself
};

// Work counters, accumulated on device per batch.
enum Counter {
    CTR_NW_CELLS = 0,     // Needleman-Wunsch cells (score + DP)
    CTR_CHAIN_RES,        // residue visits of Kabsch / refine passes in chains
    CTR_BANK_RES,         // residue visits of bank refine + score passes
    CTR_BANK_ITEMS,       // (seed, cutoff) items refined
    CTR_CHAINS,           // NW chains run
    CTR_CHAIN_LAUNCHES,   // k_chain launches (host-counted)
    CTR_BANK_LAUNCHES,    // k_bank launches (host-counted)
    CTR_LAUNCHES,         // all kernel launches (host-counted)
    CTR_CYC_NW,           // SM cycles (summed over warps) in NW fill
    CTR_CYC_TRACE,        // ... in traceback
    CTR_CYC_DETAIL,       // ... in the lite detailed search
    CTR_CYC_KABSCH,       // ... in window / alignment Kabsch + compact score
    kCounters
};

// search.cu: text returned by indialign_last_error on this thread
void set_last_error_text(const char *msg);

// k_misc.cu
void launch_prep(const DevBatch &b, int use_frag, cudaStream_t st);
void launch_anchor(const DevBatch &b, cudaStream_t st);
void launch_ss(const DevBatch &b, cudaStream_t st);
void launch_topk(const DevBatch &b, cudaStream_t st);
void launch_weighted(const DevBatch &b, cudaStream_t st);
void launch_rescore(const DevBatch &b, int slot, int need_flag, cudaStream_t st);
void launch_rescore_list(const DevBatch &b, double *recs, const int *rec_pair, int nrec,
                         cudaStream_t st);
void launch_offset_starts(const DevBatch &b, double *starts, const int *slot_pair,
                          const int *slot_idx, int nslots, cudaStream_t st);
void launch_repack(const DevBatch &b, const int *off_in, const double *pred, const double *nat,
                   const uint8_t *v, const uint8_t *pv, const uint8_t *nv, cudaStream_t st);
void launch_snapshot(const DevBatch &b, double *snap, int stage, int stages, cudaStream_t st);
void launch_export(const DevBatch &b, double *out, cudaStream_t st);
void launch_scan(const int *counts, int *begins, int ntasks, ScanOut *out, int *counter,
                 cudaStream_t st);

// k_bank.cu
size_t bank_smem_bytes(int nmax);
void launch_bank(const BankTask *tasks, const int *chunk_begin, int ntasks, const ScanOut *scan,
                 int *counter, double *item_res, int *err, int nmax, int grid,
                 unsigned long long *ctr, cudaStream_t st);
void launch_reduce_bank(const BankTask *tasks, int ntasks, const double *item_res,
                        PairState *state, cudaStream_t st);
cudaError_t bank_set_attributes();
const void *bank_kernel_ptr(bool smem);

// k_chain.cu
size_t chain_smem_bytes(int pmax, int nmax, int flags);
void launch_chain(const DevBatch &b, const ChainTask *tasks, const int *chunk_begin, int ntasks,
                  const ScanOut *scan, int *counter, uint32_t *gtrace, size_t trace_words,
                  double *gbh, uint32_t *gal, int pmax, int nmax, int flags, int grid, bool emit,
                  cudaStream_t st);
cudaError_t chain_set_attributes();
const void *chain_kernel_ptr();
size_t nw_trace_words(int np, int nn);
// NW trace words of an np x nn problem in k_chain.cu's layout: per 64-row
// stripe a block of G step words x 64 rows, G = (P + 127) / 16 with period
// P = max(nn + 1, 64).
constexpr size_t nw_trace_words_for(int np, int nn) {
    return (size_t)((np + 63) / 64) * 64 * (size_t)(((nn + 1 > 64 ? nn + 1 : 64) + 127) / 16);
}
void launch_nw_explicit(const double *smat, int np, int nn, double gap, uint32_t *trace,
                        double *bH, uint32_t *al, int *ap, int *an, int *na,
                        unsigned long long *ctr, cudaStream_t st);

// k_learn.cu -------------------------------------------------------------------
// Ranker parameters on device: FP32 biases / standardisation and BF16 weight
// copies in the layouts the tensor-core fragments read (built from a blob by
// launch_mlp_pack).
struct MlpPacked {
    float mean[kFeatures], inv_std[kFeatures];
    float b1[kHidden], b2[kHidden], w3[kHidden];
    float b3, pad_[3];
    uint16_t W1T[kHidden * kFeatures];  // bf16 [out][in]
    uint16_t W2T[kHidden * kHidden];    // bf16 [out][in]
    uint16_t W2[kHidden * kHidden];     // bf16 [in][out]
};

// Per-sample activations kept by a training forward pass.
struct MlpSave {
    uint16_t *xn;  // bf16 [n][16] standardised inputs
    float *z1;     // [n][128] layer-1 pre-activations
    uint16_t *h1;  // bf16 [n][128] gelu(z1)
    float *z2;     // [n][128] layer-2 pre-activations
};

struct RankArgs {
    const MlpPacked *mlp;      // nullptr: features only
    const long long *wbase;    // [ntasks] first candidate of a task in the candidate arrays
    float *score;              // [candidates] predicted refined score
    float *feat;               // optional [candidates][16] raw features
    int kind;                  // CandKind
    int ntasks;                // pairs, or pairs x kDetSlots for CAND_DET
    int det_ss;                // CAND_DET: the SS detailed search (slot 0 under the
                               // stage flag) instead of dp_refine's (active slots)
    const double *alP, *alQ;   // CAND_DET: aligned coordinates (2 slots per pair)
    int min_len;               // LEARNED: pairs with min(plen, nlen) below this refine
                               // every candidate (not ranked); 0 in COLLECT
};

struct SelectArgs {
    RankArgs task;              // candidate sets (kind, tasks, aligned sets)
    const long long *wbase;
    const float *score;
    int *wcount;               // [n] selected windows, -1 = all
    int *wlist;                // [n][kMaxTopK]
    int top_k;
    float margin;
    double audit_rate;
    unsigned long long seed;
    int kind;                   // CandKind
    unsigned long long *stats;  // [kRankStats] of this kind
};

// Where the refined results of a stage's candidates live: two gap-chain
// records per candidate (chain_res + chain_base[p]), and for threading
// offsets also the detailed-search record (det + det_base[p] + offset); for
// detailed-search seeds the bank items (kDetC cutoffs per seed) of the bank
// task of each (pair, slot).
struct CandRes {
    const double *chain_res;
    const long long *chain_base;
    const double *det;
    const int *det_base;
    const double *item_res;
    const BankTask *btasks;
    int bank_per_pair;  // detailed-search items: 1 one bank task per pair (the SS
                        // seeds' detailed search), 0 one per alignment slot
};

void launch_plan_rank(const DevBatch &b, const RankArgs &a, int *counts, cudaStream_t st);
void launch_rank(const DevBatch &b, const RankArgs &a, const int *chunk_begin, const ScanOut *scan,
                 int *counter, int grid, cudaStream_t st);
cudaError_t rank_set_attributes();
size_t rank_smem_bytes();
const void *rank_kernel_ptr();
void launch_select(const DevBatch &b, const SelectArgs &a, cudaStream_t st);
void launch_audit(const DevBatch &b, const SelectArgs &a, const CandRes &r, cudaStream_t st);
void launch_collect_labels(const DevBatch &b, const RankArgs &a, const CandRes &r, float *label,
                           cudaStream_t st);
void launch_mlp_pack(const float *blob, MlpPacked *out, cudaStream_t st);
void launch_mlp_forward(const MlpPacked *mlp, const float *x, int n, float *y, const MlpSave *save,
                        cudaStream_t st);
void launch_mlp_loss(const float *y, const float *t, int n, float lambda, float *dy, float *loss,
                     cudaStream_t st);
// dZ = dH (or dy x w3) * gelu'(Z) as bf16, with column sums (bias gradients)
// and, for the head, the w3 / b3 gradients.  Rows are split into up to
// kBwdBlocksMax blocks of >= kBwdRows rows whose partial sums go to `red`
// (kBwdBlocksMax x kBwdRedStride floats) and are added in block order.
constexpr int kBwdRows = 128, kBwdBlocksMax = 64, kBwdRedStride = 2 * kHidden + 4;
int bwd_row_blocks(int n);
void launch_mlp_head_bwd(const MlpPacked *mlp, const float *dy, const float *z2, int n, uint16_t *dz2,
                         float *red, float *grad, cudaStream_t st);
void launch_mlp_act_bwd(const float *dh, const float *z, int n, uint16_t *dz, float *red, float *dbias,
                        cudaStream_t st);
// k_tcgen05.cu: C[M][N] = A[M][K] . B[N][K]^T on the tcgen05 tensor cores,
// BF16 in, FP32 out.  A is K-major ([M][lda], a_mn = 0) or MN-major
// ([K][lda], a_mn = 1, M <= 128); B likewise with N (N <= 256); lda, ldb
// multiples of 8 elements, 16-byte aligned pointers.  C has row stride ldc,
// or is written transposed (C[n][m], c_trans = 1).  K is split over `splits`
// partial tiles in `partial` (splits x M x N floats) summed in a fixed order.
// Returns 0, -1 (arguments), -2 (tensor map) or -3 (launch).
int launch_gemm_tc(const uint16_t *A, int lda, int a_mn, const uint16_t *B, int ldb, int b_mn, int M, int N,
                   int K, float *C, int ldc, int c_trans, float *partial, int splits, int *err, cudaStream_t st);
void launch_adam(float *w, const float *g, float *m, float *v, int n, int first, float lr, float b1,
                 float b2, float eps, float bc1, float bc2, cudaStream_t st);

// k_plan.cu
void launch_plan_bank(const DevBatch &b, const PlanCtx &c, cudaStream_t st);
void launch_plan_chain(const DevBatch &b, const PlanCtx &c, cudaStream_t st);
void launch_reduce_chain(const DevBatch &b, const PlanCtx &c, cudaStream_t st);
void launch_glue(const DevBatch &b, const GlueArgs &a, cudaStream_t st);

}  // namespace ia
