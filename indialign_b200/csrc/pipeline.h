// Device-resident layout of a batch of pairs and the descriptors that the
// search's kernels consume.  Shared by host (search.cu) and device code.
//
// Residue data of all pairs is packed back to back in HBM; pair p owns
// residues [off[p], off[p]+N) (off[] padded to even counts so that every
// pair's xyz block starts on a 16-byte boundary for bulk copies).
//
// Every stage is a fixed launch sequence
//   plan kernel (per task slot: work count, 0 when gated off)
//   -> scan (chunk begins + total, on device)
//   -> persistent work kernel pulling chunks from a device counter
//   -> reduce / per-pair glue kernels that apply the reference's
//      first-max / strict-'>' update rules,
// so no host round trip is needed between stages.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define IA_HD_INLINE __host__ __device__ inline
#else
#define IA_HD_INLINE inline
#endif

namespace ia {

constexpr int kMaxC = 11;          // d0 cutoffs of the main seed bank
constexpr int kDetC = 6;           // cutoffs of the detailed searches
constexpr int kMaxSeeds = 1024;    // fragment windows (<= 1+9*101) + anchors
constexpr int kMaxBitSeeds = 32;   // anchor masks (<= 6 radii x 5) + top-k mask
constexpr int kRec = 13;           // {score, R[9], t[3]}
constexpr int kBankChunk = 128;    // threads of a bank CTA (4 warps x 32)
// Kernel shape knobs of one length bucket (tuning table, search.cu).
struct Tune {
    int bank_chunk = 256;       // bank items per CTA chunk (multiple of 32)
    int bank_cutoff_major = 1;  // bank item order: 1 cutoff major, 0 seed major
    int chain_chunk = 16;       // NW chains per CTA chunk
    int chain_smem_trace = 1;   // NW traces in shared memory when they fit
};
constexpr int kTuneBuckets = 3;
// The rows the plan kernels read: a task takes the shape of its pair's
// length bucket (N <= max_len[0], <= max_len[1], longer).
struct TuneRows {
    int max_len[kTuneBuckets];
    Tune t[kTuneBuckets];
    IA_HD_INLINE const Tune &of(int N) const {
        return N <= max_len[0] ? t[0] : (N <= max_len[1] ? t[1] : t[2]);
    }
};
constexpr int kChainWarps = 4;     // warps per NW-chain CTA

constexpr double kNegInf = -1e300; // "no candidate" marker
constexpr double kScoreInit = -1e30;

// Per-pair facts derived on device by k_prep / k_anchor.
struct PairInfo {
    int N, off;              // residues, offset in packed arrays
    int plen, nlen;          // nonzero pred / native valid entries
    int vsum, pvsum, nvsum;  // byte sums of the masks (reference semantics)
    int has_cross;           // some pv[i] != nv[i]
    int K;                   // seeds in the seed table (fragments + anchors)
    int nbits;               // bitmask seeds in use
    int bitoff, words;       // bitmask storage: first word, words per mask
    int C;                   // main-bank cutoffs
    int status;              // 0 search runs, 1 degenerate (score 0, identity)
    int vcount;              // nonzero valid entries
    double lnorm, d0, d0s, sd8;
    double cut[kMaxC];
    double dcut[kDetC];      // d0s x {2,1.5,1,.75,.5,.25}
};

// Per-pair records used by the stage glue (each record: {score,R,t}).
enum RecSlot {
    REC_BEST = 0,   // running best of the search
    REC_SS,         // best of the SS seeds
    REC_DET0, REC_DET1,   // detailed-search results (one per dp chain)
    REC_NEW0, REC_NEW1,   // Kabsch on the NW alignment + compact score
    REC_CUR0, REC_CUR1,   // current transform of a dp_refine chain
    REC_DPB0, REC_DPB1,   // best of a dp_refine chain
    REC_DP,         // dp_refine result
    REC_STAGE,      // result of the stage in flight
    REC_START,      // start transform handed to chains
    REC_START2,
    REC_TMP,
    REC_COUNT
};

struct PairState {
    double rec[REC_COUNT][kRec];
    int na[2];          // aligned pairs of the two NW tasks in flight
    int active[2];      // dp_refine chain still iterating
    int flag;           // stage-local condition
    int dp_on;          // a dp_refine is in flight for this pair
    int topk_ok;
    double seed_score, dp_id;
};

// ---- seed bank / detailed search tasks ---------------------------------
enum SeedMode { SEED_TABLE = 0, SEED_ARITH = 1, SEED_SHIFT = 2 };

// A set of n corresponding points (P[i] <-> Q[i]) refined from K seeds x C
// cutoffs.  Arrays are contiguous FP64 xyz; V == nullptr means all valid.
struct BankTask {
    const double *P, *Q;
    const uint8_t *V, *PV, *NV;
    const int2 *table;
    const int *slist;    // SEED_ARITH: the K seed indices to refine (nullptr: 0..K-1)
    const uint32_t *bits;
    const double *cut;
    int n, K, C, mode, ms, max_iter, use_d8, words;
    int shift_lo, shift_stride, shift_min;  // SEED_SHIFT: offsets
    double d0, sd8, lnorm, early_term;
    int pair;
    int out_rec;         // record slot for the reduced result (or -1)
    double *out;         // explicit output record (used when out_rec < 0)
    int n_items;         // K*C (0 = task inactive)
    int item_base;       // first item in the launch's item space (set by scan)
    int chunk;           // items per CTA chunk (the pair's length bucket)
    int cutoff_major;    // item order: 1 cutoff major, 0 seed major
};

// ---- NW chains ---------------------------------------------------------
enum ChainStart { START_WINDOW = 0, START_RT = 1 };
enum ChainMode { CHAIN_LITE = 0, CHAIN_EMIT = 1 };
enum ScoreMode { SMAT_DP = 0, SMAT_SS2 = 1, SMAT_SS4 = 2, SMAT_EXPLICIT = 3 };

// One task = all chains of one pair in one stage (windows x 2 gaps, or
// RT starts x 2 gaps, or single EMIT NW alignments).
struct ChainTask {
    int pair;
    int start;           // ChainStart
    int dense;           // window schedule (START_WINDOW)
    int n_starts;        // windows or RT starts
    int gaps;            // 2: both gap penalties per start, 1: gap0 only
    int max_iter;
    int smode;           // ScoreMode (EMIT tasks)
    double gap0, gap1;
    double sd8;          // score-matrix cutoff and detailed d8 cutoff
    const double *rt;    // START_RT: n_starts x 12 doubles (R,t)
    double *res;         // LITE: n_starts*gaps records; EMIT: see below
    int *na_out;         // EMIT: aligned pair count per start
    const int *live;     // optional per-start on/off flags
    const int *wlist;    // START_WINDOW: window index of start si (nullptr: si)
    double *alP, *alQ;   // EMIT: aligned coordinates (contiguous)
    int al_cap;          // capacity per EMIT start
    int n_chains;        // n_starts*gaps (0 = inactive)
    int chunk;           // chains per CTA chunk (the pair's length bucket)
    int chain_base;      // first chain in the launch's chain space
};

// Plan kinds: one per bank / chain stage flavour (k_plan.cu).
enum BankKind { BK_MAIN = 0, BK_DET_SS, BK_DET_DP, BK_GAPLESS, BK_THREAD, BK_TOPK };
enum ChainKind { CH_SS2 = 0, CH_SS4, CH_DP_EMIT, CH_LOCAL, CH_THREAD, CH_SINGLE, CH_OFFDP };

// Per-pair glue operations (k_plan.cu: k_glue).
enum GlueOp {
    G_GATE = 0, G_STAGE_UPDATE, G_SS_BEGIN, G_SS_DET, G_DP_STEP, G_DP_END, G_SS_DP,
    G_SS4_START, G_SS_FINISH, G_DPF_BEGIN, G_DPF_UPDATE, G_TMP_UPDATE, G_IDP_START,
    G_EXTRA_START, G_FLAG_ON, G_OFFDP_UPDATE
};

struct PlanCtx {
    int kind, ntasks;
    const int *pair;        // slot -> pair (nullptr: slot == pair)
    const int *aux;         // slot -> stage-specific index
    const long long *base;  // slot -> first result record / item
    BankTask *btasks;
    ChainTask *ctasks;
    int *counts;            // slot -> work chunks
    double *alP, *alQ;      // aligned sets (2 per pair)
    double *chain_res;      // LITE chain results
    double *recs, *recs2;   // stage record arrays (threading det, offset starts/results)
    const int *wcount;      // CH_LOCAL: per pair selected windows (-1: all), or nullptr
    const int *wlist;       // CH_LOCAL: per pair kMaxTopK selected windows, ascending
    int max_iter, iters;
    double early_term;
    TuneRows tune;          // kernel shapes per length bucket
};

struct GlueArgs {
    int op;
    double thr;
    int dp_iter;
    const double *recs;
    const int *idx;         // per pair first record of `recs`
};

struct ScanOut {
    int total_chunks;
    int error;           // device-side error flags (bounded waits, caps)
};

// ---- learned window ranker ---------------------------------------------------
// A 16 -> 128 -> 128 -> 1 GELU MLP predicts each rescue window's refined
// dp_refine score from cheap features; the search refines only the top-k
// windows of a pair (k_learn.cu).
constexpr int kFeatures = 16;
constexpr int kHidden = 128;
constexpr int kMaxTopK = 32;
constexpr int kRankChunk = 64;  // candidates per CTA chunk of the ranker (4 warps x 16)

// Candidate starts the ranker scores: local-fragment windows
// (rescue.h:50-117, dense = false), threading-DP offsets (rescue.h:121-190),
// dense local-fragment windows -- each a segment (flen, ps, ns) of compact
// pred / native positions of a pair -- and the seeds of the detailed searches
// on an NW alignment (align.h:15-50, fragments of the aligned set, two
// alignment slots per pair) and the seeds of the main seed bank (fragment
// windows and anchor bitmasks of the full pair, seeds.h:41-283).
enum CandKind { CAND_LOCAL = 0, CAND_THREAD = 1, CAND_DENSE = 2, CAND_DET = 3, CAND_MAIN = 4, kCandKinds = 5 };
constexpr int kDetSlots = 2;  // detailed-search alignment slots per pair (gap chains)

// FP32 parameter blob: mean[16] std[16] W1[16][128] b1[128] W2[128][128]
// b2[128] w3[128] b3, weights stored [in][out] row-major.  mean/std
// standardise the raw features and are not trained.
constexpr int kBlobMean = 0;
constexpr int kBlobStd = kBlobMean + kFeatures;
constexpr int kBlobW1 = kBlobStd + kFeatures;
constexpr int kBlobB1 = kBlobW1 + kFeatures * kHidden;
constexpr int kBlobW2 = kBlobB1 + kHidden;
constexpr int kBlobB2 = kBlobW2 + kHidden * kHidden;
constexpr int kBlobW3 = kBlobB2 + kHidden;
constexpr int kBlobB3 = kBlobW3 + kHidden;
constexpr int kBlobSize = kBlobB3 + 1;

// Ranker statistics of one batch per candidate kind (IndialignBatchOptions.rank_stats).
enum RankStat {
    RS_GATED = 0,      // pairs that reached the ranked stage
    RS_FALLBACK,       // ... refined on all windows: predicted margin below threshold
    RS_AUDIT,          // ... refined on all windows: random audit
    RS_PRUNED,         // ... refined on the top-k windows only
    RS_WINDOWS,        // windows of the gated pairs
    RS_REFINED,        // windows refined
    RS_AUDIT_MISS,     // audited pairs whose top-k windows miss the best window score
    RS_SMALL,          // gated lists with at most k candidates or of a pair shorter than
                       // the ranking length threshold (all refined)
    RS_AUDIT_MISS_1E4, // audited pairs whose top-k best is more than 1e-4 below the best
    RS_AUDIT_MISS_1E3, // ... more than 1e-3 below
    kRankStats
};

// Error bits reported through ScanOut.error / the batch status word.
enum DevError {
    DERR_TMA_TIMEOUT = 1,
    DERR_CAPACITY = 2,
    DERR_TRACE_CAP = 4,
};

}  // namespace ia
