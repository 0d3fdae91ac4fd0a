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
void launch_nw_explicit(const double *smat, int np, int nn, double gap, uint32_t *trace,
                        double *bH, uint32_t *al, int *ap, int *an, int *na,
                        unsigned long long *ctr, cudaStream_t st);

// k_plan.cu
void launch_plan_bank(const DevBatch &b, const PlanCtx &c, cudaStream_t st);
void launch_plan_chain(const DevBatch &b, const PlanCtx &c, cudaStream_t st);
void launch_reduce_chain(const DevBatch &b, const PlanCtx &c, cudaStream_t st);
void launch_glue(const DevBatch &b, const GlueArgs &a, cudaStream_t st);

}  // namespace ia
