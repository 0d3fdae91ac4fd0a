/* CPU restatement of INDIalign's TM-score superposition search, used ONLY as
 * test infrastructure: tests/, __graft_entry__.smoke() and bench.py's CPU
 * legs call it as the checker.  The product library never links it.
 *
 * Every function cites the reference file:line it restates (paths inside the
 * reference project).  Arithmetic is FP64 throughout, like the reference.
 * Parity of this restatement is pinned against the reference's own build
 * (oracle/_ref, compiled from the reference sources by oracle/Makefile) and
 * against the committed golden fixtures in tests/golden/.
 */
#ifndef INDIALIGN_ORACLE_H
#define INDIALIGN_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The reference ABI structs, field for field (indialign_c/api.h:10-36). */
typedef struct {
    int backend_mode;
    int use_fragment_search;
    int max_iter;
    int dp_iter;
    double max_mem_gb;
    int request_cuda;
    double rescue_score_1;
    double rescue_score_2;
    double early_term_score;
} OraConfig;

typedef struct {
    int length;
    const double *pred_xyz;
    const double *native_xyz;
    const uint8_t *valid_mask;
    const uint8_t *pred_valid_mask;
    const uint8_t *native_valid_mask;
    double lnorm;
} OraPairInput;

typedef struct {
    double score;
    double rotation[9];
    double translation[3];
} OraPairResult;

typedef struct { double R[9], t[3], score; } OraSeed;

void ora_default_config(OraConfig *cfg);
int ora_tmscore_search(const OraPairInput *in, const OraConfig *cfg, OraPairResult *out);
/* OpenMP over pairs; each pair runs the serial search (the reference's batch
 * entry runs every inner stage serially, indialign_c/search.h:16). */
int ora_tmscore_search_batch(int n, const OraPairInput *in, const OraConfig *cfg,
                     OraPairResult *out);
/* Same as ora_search, also writes the running best {score,R,t} after each of
 * the ORA_STAGES stages (13 doubles each; -2e30 score = stage skipped). */
int ora_trace_search(const OraPairInput *in, const OraConfig *cfg,
                     double *stage_best, OraPairResult *out);
#define ORA_STAGES 10

/* stage functions exposed for unit parity */
void ora_d0(double L, double *d0, double *d0s, double *sd8);
int ora_d0_candidates(double d0, double d0s, double *cand);
void ora_kabsch(const double *P, const double *Q, const uint8_t *mask, int N,
                double *R, double *t);
void ora_cov_to_rotation(const double *H9, double *R);
double ora_tm_score(const double *p, const double *q, const uint8_t *v,
                    const double *R, const double *t, double d0, double Lnorm,
                    double sd8, int N, int use_d8);
void ora_nw_dp(const double *smat, int Np, int Nn, double gap, double *H,
               int8_t *trace);
int ora_nw_align(const double *smat, int Np, int Nn, double gap, int *ap,
                 int *an);
int ora_seed_masks(int N, const uint8_t *valid, int use_frag, int max_starts,
                   uint8_t *masks_out, int max_K);
int ora_all_seeds(const double *p, const double *q, const uint8_t *valid,
                  int N, double d0s, double d0, int use_frag,
                  uint8_t *masks_out, int max_K);
void ora_seed_refine(const double *p, const double *q, const uint8_t *valid,
                     const uint8_t *seed, double d0s, int N, int max_iter,
                     double *R, double *t);
void ora_seed_bank(const double *p, const double *q, const uint8_t *valid,
                   const uint8_t *seeds, int K, const double *cands, int C,
                   double d0, double sd8, double Lnorm, int N, int max_iter,
                   int use_d8, double early_term, double *out13);
void ora_detailed_search(const double *p, const double *q, const int *ap,
                         const int *an, int na, double d0, double d0s,
                         double sd8, double Lnorm, int use_frag,
                         int max_iter_override, int max_starts, double *out13);
void ora_dp_refine(const double *p, const double *q, const uint8_t *pv,
                   const uint8_t *nv, const double *R0, const double *t0,
                   double d0, double d0s, double sd8, double Lnorm, int N,
                   int max_iter, int lite, double *out13);
void ora_assign_ss(const double *xyz, const uint8_t *v, int N, char *ss);
void ora_gapless(const double *p, const double *q, const uint8_t *pv,
                 const uint8_t *nv, const uint8_t *v, double d0, double d0s,
                 double Lnorm, int N, double *out13);
void ora_local_fragment_dp(const double *p, const double *q, const uint8_t *pv,
                           const uint8_t *nv, double d0, double d0s,
                           double Lnorm, int N, int dense, double *out13);
void ora_threading_dp(const double *p, const double *q, const uint8_t *pv,
                      const uint8_t *nv, double d0, double d0s, double Lnorm,
                      int N, double *out13);
void ora_topk_seed(const double *d2, const uint8_t *valid, int N, double frac,
                   uint8_t *mask);
void ora_weighted_refine(const double *p, const double *q, const uint8_t *v,
                         double d0, double Lnorm, int N, int n_iters,
                         double *R, double *t, double *score);
/* Sort (key,idx) records by key descending with the element order that the
 * reference's std::sort call produces (libstdc++ introsort). */
void ora_introsort_desc(int *keys, int *idx, int n);
uint64_t ora_fnv1a(const uint8_t *mask, int N);

#ifdef __cplusplus
}
#endif
#endif
