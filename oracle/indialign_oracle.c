/* CPU restatement of INDIalign's TM-score superposition search.
 *
 * TEST INFRASTRUCTURE ONLY.  tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs use it as the checker; the product
 * library (indialign_b200/) never links, loads or calls it.
 *
 * Each function names the reference file:line it restates (paths are inside
 * the reference project).  The restatement keeps the reference's FP64
 * arithmetic, loop orders and tie rules: first-max with strict '>' in serial
 * item order, the same early-termination points, the same NW tie-break.
 * Parity: pinned against the reference build (oracle/_ref) and the committed
 * golden fixtures (tests/golden/), see tests/test_oracle.py.
 */
#include "indialign_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAX_FRAG_STARTS 50
static const double D0_MULTS[6] = {2.0, 1.5, 1.0, 0.75, 0.5, 0.25};
static const double IDENT[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};

static double dmax(double a, double b) { return a > b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }

static void seed_ident(OraSeed *r, double score) {
    memcpy(r->R, IDENT, sizeof IDENT);
    r->t[0] = r->t[1] = r->t[2] = 0;
    r->score = score;
}
static void seed_out(const OraSeed *r, double *o13) {
    o13[0] = r->score;
    memcpy(o13 + 1, r->R, 72);
    memcpy(o13 + 10, r->t, 24);
}

/* ---- core math (indialign_c/core.h) ---------------------------------- */

/* core.h:12-25 */
void ora_d0(double L, double *d0, double *d0s, double *sd8) {
    double Lc = dmax(L, 1.0);
    double v;
    if (Lc <= 11.0) *d0 = 0.3;
    else if (Lc <= 15.0) *d0 = 0.4;
    else if (Lc <= 19.0) *d0 = 0.5;
    else if (Lc <= 23.0) *d0 = 0.6;
    else *d0 = 0.7;
    if (Lc >= 30.0) *d0 = 0.6 * sqrt(Lc - 0.5) - 2.5;
    if (*d0 < 0.3) *d0 = 0.3;
    v = 1.24 * cbrt(dmax(Lc - 15.0, 0.0)) - 1.8;
    *d0s = v < 4.5 ? 4.5 : (v > 8.0 ? 8.0 : v);
    *sd8 = 1.5 * pow(Lc, 0.3) + 3.5;
}

/* d0 search list: d0s x {2,1.5,1,.75,.5,.25} then d0+{1..5} unless within
 * 0.01 of an earlier entry (indialign.cpp:54-67). */
int ora_d0_candidates(double d0, double d0s, double *cand) {
    int C = 0;
    for (int c = 0; c < 6; c++) cand[C++] = d0s * D0_MULTS[c];
    for (int c = 1; c <= 5; c++) {
        double v = d0 + (double)c;
        int dup = 0;
        for (int e = 0; e < C && !dup; e++) dup = fabs(cand[e] - v) < 0.01;
        if (!dup) cand[C++] = v;
    }
    return C;
}

/* Cyclic Jacobi on a symmetric 4x4, 8 sweeps, pair order (0,1)(0,2)(0,3)
 * (1,2)(1,3)(2,3), skip |apq|<1e-15 (core.h:29-60). */
static void jacobi4(double A[4][4], double V[4][4]) {
    static const int P[6] = {0, 0, 0, 1, 1, 2}, Qi[6] = {1, 2, 3, 2, 3, 3};
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) V[i][j] = i == j ? 1.0 : 0.0;
    for (int sw = 0; sw < 8; sw++) {
        for (int k = 0; k < 6; k++) {
            int p = P[k], q = Qi[k];
            double apq = A[p][q];
            if (fabs(apq) < 1e-15) continue;
            double tau = (A[q][q] - A[p][p]) / (2.0 * apq);
            double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
            A[p][p] -= t * apq;
            A[q][q] += t * apq;
            A[p][q] = A[q][p] = 0.0;
            for (int r = 0; r < 4; r++) {
                if (r == p || r == q) continue;
                double rp = A[r][p], rq = A[r][q];
                A[r][p] = A[p][r] = c * rp - s * rq;
                A[r][q] = A[q][r] = s * rp + c * rq;
            }
            for (int r = 0; r < 4; r++) {
                double vp = V[r][p], vq = V[r][q];
                V[r][p] = c * vp - s * vq;
                V[r][q] = s * vp + c * vq;
            }
        }
    }
}

/* Horn's quaternion matrix from the 3x3 covariance, dominant eigenvector ->
 * rotation with aligned_d = sum_k p_k R[3k+d] (core.h:64-90). */
static void cov_to_rotation(const double H[3][3], double *R) {
    double F[4][4], V[4][4], q[4], qn;
    int best = 0;
    F[0][0] = H[0][0] + H[1][1] + H[2][2];
    F[0][1] = F[1][0] = H[1][2] - H[2][1];
    F[0][2] = F[2][0] = H[2][0] - H[0][2];
    F[0][3] = F[3][0] = H[0][1] - H[1][0];
    F[1][1] = H[0][0] - H[1][1] - H[2][2];
    F[1][2] = F[2][1] = H[0][1] + H[1][0];
    F[1][3] = F[3][1] = H[2][0] + H[0][2];
    F[2][2] = -H[0][0] + H[1][1] - H[2][2];
    F[2][3] = F[3][2] = H[1][2] + H[2][1];
    F[3][3] = -H[0][0] - H[1][1] + H[2][2];
    jacobi4(F, V);
    for (int i = 1; i < 4; i++)
        if (F[i][i] > F[best][best]) best = i;
    for (int i = 0; i < 4; i++) q[i] = V[i][best];
    qn = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    if (qn < 1e-12) { q[0] = 1; q[1] = q[2] = q[3] = 0; }
    else for (int i = 0; i < 4; i++) q[i] /= qn;
    {
        double q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
        R[0] = q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3;
        R[1] = 2 * (q1 * q2 + q0 * q3);
        R[2] = 2 * (q1 * q3 - q0 * q2);
        R[3] = 2 * (q1 * q2 - q0 * q3);
        R[4] = q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3;
        R[5] = 2 * (q2 * q3 + q0 * q1);
        R[6] = 2 * (q1 * q3 + q0 * q2);
        R[7] = 2 * (q2 * q3 - q0 * q1);
        R[8] = q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3;
    }
}

void ora_cov_to_rotation(const double *H9, double *R) {
    double H[3][3];
    for (int i = 0; i < 9; i++) H[i / 3][i % 3] = H9[i];
    cov_to_rotation(H, R);
}

/* Masked Kabsch, centroid pass then centred covariance pass; identity when
 * fewer than 3 points (core.h:94-123). */
void ora_kabsch(const double *P, const double *Q, const uint8_t *mask, int N,
                double *R, double *t) {
    double w = 0, cP[3] = {0, 0, 0}, cQ[3] = {0, 0, 0}, H[3][3];
    for (int i = 0; i < N; i++) {
        if (!mask[i]) continue;
        for (int d = 0; d < 3; d++) { cP[d] += P[i * 3 + d]; cQ[d] += Q[i * 3 + d]; }
        w += 1.0;
    }
    if (w < 3.0) {
        memcpy(R, IDENT, sizeof IDENT);
        t[0] = t[1] = t[2] = 0;
        return;
    }
    for (int d = 0; d < 3; d++) { cP[d] /= w; cQ[d] /= w; }
    memset(H, 0, sizeof H);
    for (int i = 0; i < N; i++) {
        double dp[3], dq[3];
        if (!mask[i]) continue;
        for (int d = 0; d < 3; d++) { dp[d] = P[i * 3 + d] - cP[d]; dq[d] = Q[i * 3 + d] - cQ[d]; }
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) H[r][c] += dp[r] * dq[c];
    }
    cov_to_rotation((const double(*)[3])H, R);
    for (int d = 0; d < 3; d++)
        t[d] = cQ[d] - (cP[0] * R[0 * 3 + d] + cP[1] * R[1 * 3 + d] + cP[2] * R[2 * 3 + d]);
}

static inline double dist2_at(const double *p, const double *q, const double *R,
                              const double *t) {
    double mx = p[0] * R[0] + p[1] * R[3] + p[2] * R[6] + t[0];
    double my = p[0] * R[1] + p[1] * R[4] + p[2] * R[7] + t[1];
    double mz = p[0] * R[2] + p[1] * R[5] + p[2] * R[8] + t[2];
    double dx = mx - q[0], dy = my - q[1], dz = mz - q[2];
    return dx * dx + dy * dy + dz * dz;
}

/* tm_score (d8 filter) / tm_score_no_d8 (core.h:134-166) */
double ora_tm_score(const double *p, const double *q, const uint8_t *v,
                    const double *R, const double *t, double d0, double Lnorm,
                    double sd8, int N, int use_d8) {
    double d0sq = dmax(d0 * d0, 1e-12), sd8sq = sd8 * sd8, sum = 0;
    for (int i = 0; i < N; i++) {
        double d2;
        if (!v[i]) continue;
        d2 = dist2_at(p + 3 * i, q + 3 * i, R, t);
        if (!use_d8 || d2 <= sd8sq) sum += 1.0 / (1.0 + d2 / d0sq);
    }
    return sum / dmax(Lnorm, 1.0);
}

/* kabsch_weighted (core.h:183-214) */
static void kabsch_weighted(const double *P, const double *Q, const uint8_t *v,
                            const double *w, int N, double *R, double *t) {
    double ws = 0, cP[3] = {0, 0, 0}, cQ[3] = {0, 0, 0}, H[3][3];
    for (int i = 0; i < N; i++) {
        if (!v[i] || w[i] <= 0) continue;
        for (int d = 0; d < 3; d++) { cP[d] += w[i] * P[i * 3 + d]; cQ[d] += w[i] * Q[i * 3 + d]; }
        ws += w[i];
    }
    if (ws < 1e-12) {
        memcpy(R, IDENT, sizeof IDENT);
        t[0] = t[1] = t[2] = 0;
        return;
    }
    for (int d = 0; d < 3; d++) { cP[d] /= ws; cQ[d] /= ws; }
    memset(H, 0, sizeof H);
    for (int i = 0; i < N; i++) {
        double dp[3], dq[3];
        if (!v[i] || w[i] <= 0) continue;
        for (int d = 0; d < 3; d++) { dp[d] = P[i * 3 + d] - cP[d]; dq[d] = Q[i * 3 + d] - cQ[d]; }
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) H[r][c] += w[i] * dp[r] * dq[c];
    }
    cov_to_rotation((const double(*)[3])H, R);
    for (int d = 0; d < 3; d++)
        t[d] = cQ[d] - (cP[0] * R[0 * 3 + d] + cP[1] * R[1 * 3 + d] + cP[2] * R[2 * 3 + d]);
}

/* weighted_tm_refine (core.h:218-237) */
void ora_weighted_refine(const double *p, const double *q, const uint8_t *v,
                         double d0, double Lnorm, int N, int n_iters,
                         double *R, double *t, double *score) {
    double d0sq = dmax(d0 * d0, 1e-12);
    double *w = (double *)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
    for (int it = 0; it < n_iters; it++) {
        for (int i = 0; i < N; i++)
            w[i] = v[i] ? 1.0 / (1.0 + dist2_at(p + 3 * i, q + 3 * i, R, t) / d0sq) : 0.0;
        kabsch_weighted(p, q, v, w, N, R, t);
    }
    *score = ora_tm_score(p, q, v, R, t, d0, Lnorm, 0, N, 0);
    free(w);
}

/* ---- seeds (indialign_c/seeds.h) ------------------------------------- */

/* fragment_lengths: {L, L/2, L/4, L/8, 64, 32, 16, 8, 4} within [4, L],
 * distinct, descending (seeds.h:15-22).  Returns count, writes <= 9. */
static int fragment_lengths(int L, int *out) {
    int vals[9] = {L, L / 2, L / 4, L / 8, 64, 32, 16, 8, 4}, n = 0;
    if (L < 4) return 0;
    for (int a = 0; a < 9; a++) {
        int v = vals[a], seen = 0;
        if (v < 4 || v > L) continue;
        for (int b = 0; b < n; b++) seen |= out[b] == v;
        if (!seen) out[n++] = v;
    }
    for (int a = 1; a < n; a++) /* descending */
        for (int b = a; b > 0 && out[b] > out[b - 1]; b--) {
            int tmp = out[b]; out[b] = out[b - 1]; out[b - 1] = tmp;
        }
    return n;
}

/* start_positions (seeds.h:24-37); out must hold n-frag+2 entries (between
 * ms and 2ms starts the step is 1, so the list can exceed ms) */
static int start_positions(int n, int frag, int ms, int *out) {
    int total = n - frag + 1, cnt = 0, step;
    if (total <= 0) return 0;
    if (total <= ms) {
        for (int i = 0; i < total; i++) out[i] = i;
        return total;
    }
    step = imax(1, total / ms);
    for (int i = 0; i < total; i += step) out[cnt++] = i;
    if (out[cnt - 1] != total - 1) out[cnt++] = total - 1;
    return cnt;
}

/* Growable mask list. */
typedef struct { uint8_t *m; int K, cap, N; } masklist;
static uint8_t *ml_push(masklist *L) {
    if (L->K == L->cap) {
        L->cap = L->cap ? 2 * L->cap : 64;
        L->m = (uint8_t *)realloc(L->m, (size_t)L->cap * (size_t)L->N);
    }
    if (L->N > 0) memset(L->m + (size_t)L->K * (size_t)L->N, 0, (size_t)L->N);
    return L->m + (size_t)(L->K++) * L->N;
}

/* build_seed_masks: global seed + fragment windows, byte-sum >= 3 filter
 * (seeds.h:41-82). */
static void build_seed_masks(int N, const uint8_t *valid, int use_frag,
                             int max_starts, masklist *out) {
    int vc = 0, fl[9], nf, *st = (int *)malloc(sizeof(int) * (size_t)(N + 2));
    masklist raw = {0, 0, 0, N};
    for (int i = 0; i < N; i++) vc += valid[i];
    memcpy(ml_push(&raw), valid, (size_t)N);
    if (use_frag) {
        nf = fragment_lengths(vc, fl);
        for (int a = 0; a < nf; a++) {
            int ns = start_positions(N, fl[a], max_starts, st);
            for (int b = 0; b < ns; b++) {
                int s = st[b], cnt = 0;
                for (int i = s; i < s + fl[a] && i < N; i++) cnt += valid[i];
                if (cnt < 3) continue;
                uint8_t *m = ml_push(&raw);
                for (int i = s; i < s + fl[a] && i < N; i++) m[i] = valid[i];
            }
        }
    }
    out->N = N;
    for (int k = 0; k < raw.K; k++) {
        int cnt = 0;
        const uint8_t *m = raw.m + (size_t)k * N;
        for (int i = 0; i < N; i++) cnt += m[i];
        if (cnt >= 3) memcpy(ml_push(out), m, (size_t)N);
    }
    free(raw.m);
    free(st);
}

int ora_seed_masks(int N, const uint8_t *valid, int use_frag, int max_starts,
                   uint8_t *masks_out, int max_K) {
    masklist L = {0, 0, 0, N};
    int K;
    build_seed_masks(N, valid, use_frag, max_starts, &L);
    K = L.K;
    if (K <= max_K) memcpy(masks_out, L.m, (size_t)K * N);
    free(L.m);
    return K <= max_K ? K : -1;
}

/* build_topk_seed: the max(3, floor(vc*frac)) residues with the smallest
 * (d2, index) among valid ones (seeds.h:85-98). */
void ora_topk_seed(const double *d2, const uint8_t *valid, int N, double frac,
                   uint8_t *mask) {
    int vc = 0, k, m = 0;
    for (int i = 0; i < N; i++) vc += valid[i];
    k = imax(3, (int)(vc * frac));
    k = imin(k, N);
    for (int i = 0; i < N; i++) mask[i] = 0;
    for (int i = 0; i < N; i++) {
        int rank = 0;
        if (!valid[i]) continue;
        m++;
        for (int j = 0; j < N; j++)
            if (valid[j] && (d2[j] < d2[i] || (d2[j] == d2[i] && j < i))) rank++;
        if (rank < k) mask[i] = 1;
    }
    (void)m;
}

/* FNV-1a 64 over the mask bytes (seeds.h:102-109) */
uint64_t ora_fnv1a(const uint8_t *mask, int N) {
    uint64_t h = 14695981039346656037ULL;
    for (int i = 0; i < N; i++) { h ^= mask[i]; h *= 1099511628211ULL; }
    return h;
}

/* Introsort with the exact element movements of the std::sort call at
 * seeds.h:237-238 (libstdc++: depth limit 2*floor(log2 n), median-of-three
 * moved to the front from (first+1, mid, last-1), unguarded Hoare partition,
 * runs of <= 16 left for a final insertion sort, heapsort on depth overflow).
 * The comparator orders by key only, so the order of equal keys is whatever
 * these movements produce; the anchor seeds depend on it. */
typedef struct { int key, idx; } kv_t;
#define KV_LESS(x, y) ((x).key > (y).key)
static void kv_swap(kv_t *a, kv_t *b) { kv_t t = *a; *a = *b; *b = t; }

static void kv_adjust_heap(kv_t *f, long hole, long len, kv_t v) {
    long top = hole, child = hole, parent;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (KV_LESS(f[child], f[child - 1])) child--;
        f[hole] = f[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        f[hole] = f[child - 1];
        hole = child - 1;
    }
    parent = (hole - 1) / 2;
    while (hole > top && KV_LESS(f[parent], v)) {
        f[hole] = f[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    f[hole] = v;
}

static void kv_heapsort(kv_t *f, long len) {
    if (len >= 2) {
        long parent = (len - 2) / 2;
        for (;;) {
            kv_adjust_heap(f, parent, len, f[parent]);
            if (parent == 0) break;
            parent--;
        }
    }
    while (len > 1) {
        kv_t v;
        len--;
        v = f[len];
        f[len] = f[0];
        kv_adjust_heap(f, 0, len, v);
    }
}

static void kv_introsort_loop(kv_t *f, long lo, long hi, int depth) {
    while (hi - lo > 16) {
        long mid, a, b;
        if (depth == 0) { kv_heapsort(f + lo, hi - lo); return; }
        depth--;
        mid = lo + (hi - lo) / 2;
        a = lo + 1; b = hi - 1;
        if (KV_LESS(f[a], f[mid])) {
            if (KV_LESS(f[mid], f[b])) kv_swap(&f[lo], &f[mid]);
            else if (KV_LESS(f[a], f[b])) kv_swap(&f[lo], &f[b]);
            else kv_swap(&f[lo], &f[a]);
        } else if (KV_LESS(f[a], f[b])) kv_swap(&f[lo], &f[a]);
        else if (KV_LESS(f[mid], f[b])) kv_swap(&f[lo], &f[b]);
        else kv_swap(&f[lo], &f[mid]);
        a = lo + 1; b = hi;
        for (;;) {
            while (KV_LESS(f[a], f[lo])) a++;
            b--;
            while (KV_LESS(f[lo], f[b])) b--;
            if (!(a < b)) break;
            kv_swap(&f[a], &f[b]);
            a++;
        }
        kv_introsort_loop(f, a, hi, depth);
        hi = a;
    }
}

static void kv_linear_insert(kv_t *f, long i) {
    kv_t v = f[i];
    long j = i - 1;
    while (KV_LESS(v, f[j])) { f[i] = f[j]; i = j; j--; }
    f[i] = v;
}

static void kv_insertion_sort(kv_t *f, long lo, long hi) {
    if (lo == hi) return;
    for (long i = lo + 1; i < hi; i++) {
        if (KV_LESS(f[i], f[lo])) {
            kv_t v = f[i];
            memmove(f + lo + 1, f + lo, sizeof(kv_t) * (size_t)(i - lo));
            f[lo] = v;
        } else {
            kv_linear_insert(f, i);
        }
    }
}

static void kv_sort(kv_t *f, long n) {
    int lg = 0;
    if (n <= 0) return;
    while ((1L << (lg + 1)) <= n) lg++;
    kv_introsort_loop(f, 0, n, 2 * lg);
    if (n > 16) {
        kv_insertion_sort(f, 0, 16);
        for (long i = 16; i < n; i++) kv_linear_insert(f, i);
    } else {
        kv_insertion_sort(f, 0, n);
    }
}

void ora_introsort_desc(int *keys, int *idx, int n) {
    kv_t *f = (kv_t *)malloc(sizeof(kv_t) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) { f[i].key = keys[i]; f[i].idx = idx[i]; }
    kv_sort(f, n);
    for (int i = 0; i < n; i++) { keys[i] = f[i].key; idx[i] = f[i].idx; }
    free(f);
}

/* Consistent-contact neighbour test of build_anchor_contact_seeds: both the
 * pred and the native distance within rad and |dp - dn| <= tol
 * (seeds.h:216-229).  The reference's spatial grid only accelerates the
 * search over valid residues; an exhaustive scan visits the same set. */
static int contact_ok(const double *p, const double *q, int i, int j,
                      double rad_sq, double tol) {
    double pdx = p[i * 3] - p[j * 3], pdy = p[i * 3 + 1] - p[j * 3 + 1], pdz = p[i * 3 + 2] - p[j * 3 + 2];
    double pd2 = pdx * pdx + pdy * pdy + pdz * pdz, ndx, ndy, ndz, nd2;
    if (pd2 > rad_sq) return 0;
    ndx = q[i * 3] - q[j * 3]; ndy = q[i * 3 + 1] - q[j * 3 + 1]; ndz = q[i * 3 + 2] - q[j * 3 + 2];
    nd2 = ndx * ndx + ndy * ndy + ndz * ndz;
    if (nd2 > rad_sq) return 0;
    return fabs(sqrt(pd2) - sqrt(nd2)) <= tol;
}

/* build_anchor_contact_seeds (seeds.h:164-283) */
static void anchor_seeds(const double *p, const double *q, const uint8_t *valid,
                         int N, double d0s, double d0, int max_anchors,
                         masklist *L) {
    double radii[8], mr[3] = {d0s, d0s * 1.5, d0s * 2.0}, ar[3] = {d0 + 1.0, d0 + 2.0, d0 + 3.0};
    int nrad = 0, V = 0, *vidx, *cnt, *keys, *ids;
    uint64_t *seen;
    int nseen = 0;
    for (int i = 0; i < 3; i++) radii[nrad++] = mr[i];
    for (int i = 0; i < 3; i++) {
        int dup = 0;
        for (int j = 0; j < nrad && !dup; j++) dup = fabs(radii[j] - ar[i]) < 0.01;
        if (!dup) radii[nrad++] = ar[i];
    }
    vidx = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    for (int i = 0; i < N; i++) if (valid[i]) vidx[V++] = i;
    if (V < 3) { free(vidx); return; }
    cnt = (int *)malloc(sizeof(int) * (size_t)V);
    keys = (int *)malloc(sizeof(int) * (size_t)V);
    ids = (int *)malloc(sizeof(int) * (size_t)V);
    seen = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(L->K + nrad * max_anchors + 1));
    for (int k = 0; k < L->K; k++) seen[nseen++] = ora_fnv1a(L->m + (size_t)k * N, N);
    for (int ri = 0; ri < nrad; ri++) {
        double rad = radii[ri], rad_sq, tol;
        int nc = 0, added = 0;
        if (rad <= 0) continue;
        rad_sq = rad * rad;
        tol = dmax(0.5, rad * 0.25);
        for (int a = 0; a < V; a++) {
            int i = vidx[a];
            cnt[a] = 1;
            for (int b = 0; b < V; b++) {
                int j = vidx[b];
                if (j != i && contact_ok(p, q, i, j, rad_sq, tol)) cnt[a]++;
            }
        }
        for (int a = 0; a < V; a++)
            if (cnt[a] >= 3) { keys[nc] = cnt[a]; ids[nc] = a; nc++; }
        ora_introsort_desc(keys, ids, nc);
        for (int c = 0; c < nc; c++) {
            int i = vidx[ids[c]], mc = 1, dup = 0;
            uint8_t *m;
            uint64_t h;
            if (added >= max_anchors) break;
            m = (uint8_t *)calloc((size_t)N, 1);
            m[i] = 1;
            for (int b = 0; b < V; b++) {
                int j = vidx[b];
                if (j != i && contact_ok(p, q, i, j, rad_sq, tol)) { m[j] = 1; mc++; }
            }
            if (mc < 3) { free(m); continue; }
            h = ora_fnv1a(m, N);
            for (int s = 0; s < nseen && !dup; s++) dup = seen[s] == h;
            if (dup) { free(m); continue; }
            seen[nseen++] = h;
            memcpy(ml_push(L), m, (size_t)N);
            free(m);
            added++;
        }
    }
    free(vidx); free(cnt); free(keys); free(ids); free(seen);
}

int ora_all_seeds(const double *p, const double *q, const uint8_t *valid,
                  int N, double d0s, double d0, int use_frag,
                  uint8_t *masks_out, int max_K) {
    masklist L = {0, 0, 0, N};
    int K;
    build_seed_masks(N, valid, use_frag, MAX_FRAG_STARTS, &L);
    anchor_seeds(p, q, valid, N, d0s, d0, 5, &L);
    K = L.K;
    if (K <= max_K) memcpy(masks_out, L.m, (size_t)K * N);
    free(L.m);
    return K <= max_K ? K : -1;
}

/* ---- seed refinement and seed bank (indialign_c/search.h) ------------- */

/* iterative_seed_refine: Kabsch on seed&valid, then up to max_iter rounds of
 * {select d2 <= d0s^2 among valid; Kabsch if >= 3 selected}, stopping when
 * the selected count repeats (search.h:28-56). */
static void seed_refine(const double *p, const double *q, const uint8_t *valid,
                        const uint8_t *seed, double d0s, int N, int max_iter,
                        double *R, double *t, uint8_t *work, uint8_t *sel) {
    double cut = d0s * d0s;
    int prev = -1;
    for (int i = 0; i < N; i++) work[i] = seed[i] & valid[i];
    ora_kabsch(p, q, work, N, R, t);
    for (int it = 0; it < max_iter; it++) {
        int c = 0;
        for (int i = 0; i < N; i++) {
            if (!valid[i]) { sel[i] = 0; continue; }
            sel[i] = dist2_at(p + 3 * i, q + 3 * i, R, t) <= cut;
            c += sel[i];
        }
        if (c >= 3) ora_kabsch(p, q, sel, N, R, t);
        if (c == prev) break;
        prev = c;
    }
}

void ora_seed_refine(const double *p, const double *q, const uint8_t *valid,
                     const uint8_t *seed, double d0s, int N, int max_iter,
                     double *R, double *t) {
    uint8_t *w = (uint8_t *)malloc((size_t)N + 1), *s = (uint8_t *)malloc((size_t)N + 1);
    seed_refine(p, q, valid, seed, d0s, N, max_iter, R, t, w, s);
    free(w); free(s);
}

/* evaluate_seed_bank, serial path: seeds outer, cutoffs inner, first max
 * wins, stop before a seed once best >= early_term (search.h:62-98). */
static OraSeed seed_bank(const double *p, const double *q, const uint8_t *valid,
                         const uint8_t *seeds, int K, const double *cands,
                         int C, double d0, double sd8, double Lnorm, int N,
                         int max_iter, int use_d8, double early_term) {
    OraSeed best;
    double R[9], t[3];
    uint8_t *w = (uint8_t *)malloc((size_t)N + 1), *s = (uint8_t *)malloc((size_t)N + 1);
    memset(&best, 0, sizeof best);
    best.score = -1e30;
    for (int k = 0; k < K; k++) {
        if (best.score >= early_term) break;
        for (int c = 0; c < C; c++) {
            double sc;
            seed_refine(p, q, valid, seeds + (size_t)k * N, cands[c], N, max_iter, R, t, w, s);
            sc = ora_tm_score(p, q, valid, R, t, d0, Lnorm, sd8, N, use_d8);
            if (sc > best.score) {
                best.score = sc;
                memcpy(best.R, R, 72);
                memcpy(best.t, t, 24);
            }
        }
    }
    free(w); free(s);
    return best;
}

void ora_seed_bank(const double *p, const double *q, const uint8_t *valid,
                   const uint8_t *seeds, int K, const double *cands, int C,
                   double d0, double sd8, double Lnorm, int N, int max_iter,
                   int use_d8, double early_term, double *out13) {
    OraSeed r = seed_bank(p, q, valid, seeds, K, cands, C, d0, sd8, Lnorm, N,
                          max_iter, use_d8, early_term);
    seed_out(&r, out13);
}

/* ---- Needleman-Wunsch (indialign_c/nw.h) ------------------------------ */

/* nw_dp: zero boundaries, anti-diagonal order, a gap move pays gap_open only
 * when the cell it leaves was reached diagonally; ties prefer diag, then
 * left, then up.  trace: -1 boundary, 0 diag, 1 up, 2 left (nw.h:10-38).
 * The order of cell evaluation does not change the values: every cell reads
 * only its three finished neighbours. */
void ora_nw_dp(const double *smat, int Np, int Nn, double gap, double *H,
               int8_t *tr) {
    int Hn = Nn + 1;
    for (long i = 0; i < (long)(Np + 1) * Hn; i++) { H[i] = 0.0; tr[i] = -1; }
    for (int i = 1; i <= Np; i++)
        for (int j = 1; j <= Nn; j++) {
            double diag = H[(i - 1) * Hn + (j - 1)] + smat[(i - 1) * Nn + (j - 1)];
            double up = H[(i - 1) * Hn + j], left = H[i * Hn + (j - 1)];
            if (tr[(i - 1) * Hn + j] == 0) up += gap;
            if (tr[i * Hn + (j - 1)] == 0) left += gap;
            if (diag >= up && diag >= left) { H[i * Hn + j] = diag; tr[i * Hn + j] = 0; }
            else if (left >= up) { H[i * Hn + j] = left; tr[i * Hn + j] = 2; }
            else { H[i * Hn + j] = up; tr[i * Hn + j] = 1; }
        }
}

/* nw_traceback from (Np, Nn): diag emits a pair, up steps i, anything else
 * steps j; pairs returned in ascending order (nw.h:42-68). */
static int nw_traceback(const int8_t *tr, int Np, int Nn, int *ap, int *an) {
    int Hn = Nn + 1, i = Np, j = Nn, cnt = 0;
    int *tp = (int *)malloc(sizeof(int) * (size_t)(imin(Np, Nn) + 1));
    int *tn = (int *)malloc(sizeof(int) * (size_t)(imin(Np, Nn) + 1));
    while (i > 0 && j > 0) {
        int8_t d = tr[i * Hn + j];
        if (d == 0) { tp[cnt] = i - 1; tn[cnt] = j - 1; cnt++; i--; j--; }
        else if (d == 1) i--;
        else j--;
    }
    for (int k = 0; k < cnt; k++) { ap[k] = tp[cnt - 1 - k]; an[k] = tn[cnt - 1 - k]; }
    free(tp); free(tn);
    return cnt;
}

int ora_nw_align(const double *smat, int Np, int Nn, double gap, int *ap,
                 int *an) {
    size_t cells = (size_t)(Np + 1) * (size_t)(Nn + 1);
    double *H = (double *)malloc(sizeof(double) * cells);
    int8_t *tr = (int8_t *)malloc(cells);
    int na;
    ora_nw_dp(smat, Np, Nn, gap, H, tr);
    na = nw_traceback(tr, Np, Nn, ap, an);
    free(H); free(tr);
    return na;
}

/* ---- DP refinement (indialign_c/align.h) ------------------------------ */

/* alignment_detailed_search: seed bank over the aligned pairs with all-ones
 * validity, cutoffs d0s x D0_MULTS, d8-filtered scoring (align.h:15-50). */
static OraSeed detailed_search(const double *p, const double *q, const int *ap,
                               const int *an, int na, double d0, double d0s,
                               double sd8, double Lnorm, int use_frag,
                               int max_iter_override, int max_starts) {
    OraSeed r;
    double *P, *Q, cand[6];
    uint8_t *ones;
    masklist L = {0, 0, 0, na};
    int mi;
    if (na < 3) { seed_ident(&r, -1e30); return r; }
    P = (double *)malloc(sizeof(double) * 3 * (size_t)na);
    Q = (double *)malloc(sizeof(double) * 3 * (size_t)na);
    ones = (uint8_t *)malloc((size_t)na);
    for (int i = 0; i < na; i++) {
        memcpy(P + 3 * i, p + 3 * ap[i], 24);
        memcpy(Q + 3 * i, q + 3 * an[i], 24);
        ones[i] = 1;
    }
    build_seed_masks(na, ones, use_frag, max_starts, &L);
    if (L.K == 0) {
        seed_ident(&r, -1e30);
    } else {
        for (int c = 0; c < 6; c++) cand[c] = d0s * D0_MULTS[c];
        mi = max_iter_override >= 0 ? max_iter_override : (use_frag ? 20 : 8);
        r = seed_bank(P, Q, ones, L.m, L.K, cand, 6, d0, sd8, Lnorm, na, mi, 1, 1.0);
    }
    free(L.m); free(P); free(Q); free(ones);
    return r;
}

void ora_detailed_search(const double *p, const double *q, const int *ap,
                         const int *an, int na, double d0, double d0s,
                         double sd8, double Lnorm, int use_frag,
                         int max_iter_override, int max_starts, double *out13) {
    OraSeed r = detailed_search(p, q, ap, an, na, d0, d0s, sd8, Lnorm, use_frag,
                                max_iter_override, max_starts);
    seed_out(&r, out13);
}

/* Compact index map of the nonzero entries of a mask. */
static int compact(const uint8_t *m, int N, int *map) {
    int n = 0;
    for (int i = 0; i < N; i++) if (m[i]) map[n++] = i;
    return n;
}

/* dp_refine_chunk: for gap in {-0.6, 0}: up to max_iter rounds of score
 * matrix under the current (R,t) -> NW -> traceback -> Kabsch on the aligned
 * pairs -> compact TM (no d8) -> detailed search on the aligned pairs (with
 * fragments unless lite); best starts at score 0 / identity (align.h:54-145).
 */
static OraSeed dp_refine(const double *pred, const double *native,
                         const uint8_t *pv, const uint8_t *nv, const double *R0,
                         const double *t0, double d0, double d0s, double sd8,
                         double Lnorm, int N, int max_iter, int lite) {
    static const double gaps[2] = {-0.6, 0.0};
    OraSeed best;
    int *pm = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    int *nm = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    int plen = compact(pv, N, pm), nlen = compact(nv, N, nm), mn;
    double *moved, *smat, *Pa, *Qa;
    int *ap, *an;
    uint8_t *ones;
    double d0dp = dmax(d0, 1.0), d0sq_dp = dmax(d0dp * d0dp, 1e-12);
    double sd8sq = sd8 * sd8, d0sq_s = dmax(d0 * d0, 1e-12);
    seed_ident(&best, 0.0);
    if (plen < 3 || nlen < 3) { free(pm); free(nm); return best; }
    mn = imin(plen, nlen);
    moved = (double *)malloc(sizeof(double) * 3 * (size_t)N);
    smat = (double *)malloc(sizeof(double) * (size_t)plen * (size_t)nlen);
    ap = (int *)malloc(sizeof(int) * (size_t)mn);
    an = (int *)malloc(sizeof(int) * (size_t)mn);
    Pa = (double *)malloc(sizeof(double) * 3 * (size_t)mn);
    Qa = (double *)malloc(sizeof(double) * 3 * (size_t)mn);
    ones = (uint8_t *)malloc((size_t)mn);
    for (int g = 0; g < 2; g++) {
        double cR[9], ct[3];
        memcpy(cR, R0, 72); memcpy(ct, t0, 24);
        for (int it = 0; it < max_iter; it++) {
            double nR[9], nt[3], sc = 0;
            int na;
            OraSeed det;
            for (int i = 0; i < N; i++)
                for (int d = 0; d < 3; d++)
                    moved[i * 3 + d] = pred[i * 3] * cR[d] + pred[i * 3 + 1] * cR[3 + d] +
                                       pred[i * 3 + 2] * cR[6 + d] + ct[d];
            for (int a = 0; a < plen; a++) {
                const double *m = moved + 3 * pm[a];
                for (int b = 0; b < nlen; b++) {
                    const double *n = native + 3 * nm[b];
                    double dx = m[0] - n[0], dy = m[1] - n[1], dz = m[2] - n[2];
                    double d2 = dx * dx + dy * dy + dz * dz;
                    smat[(size_t)a * nlen + b] = d2 <= sd8sq ? 1.0 / (1.0 + d2 / d0sq_dp) : 0.0;
                }
            }
            na = ora_nw_align(smat, plen, nlen, gaps[g], ap, an);
            for (int i = 0; i < na; i++) { ap[i] = pm[ap[i]]; an[i] = nm[an[i]]; }
            if (na < 3) continue;
            for (int i = 0; i < na; i++) {
                memcpy(Pa + 3 * i, pred + 3 * ap[i], 24);
                memcpy(Qa + 3 * i, native + 3 * an[i], 24);
                ones[i] = 1;
            }
            ora_kabsch(Pa, Qa, ones, na, nR, nt);
            for (int i = 0; i < na; i++)
                sc += 1.0 / (1.0 + dist2_at(Pa + 3 * i, Qa + 3 * i, nR, nt) / d0sq_s);
            sc /= dmax(Lnorm, 1.0);
            det = detailed_search(pred, native, ap, an, na, d0, d0s, sd8, Lnorm,
                                  !lite, -1, MAX_FRAG_STARTS);
            if (det.score > sc) {
                memcpy(nR, det.R, 72); memcpy(nt, det.t, 24);
                sc = det.score;
            }
            memcpy(cR, nR, 72); memcpy(ct, nt, 24);
            if (sc > best.score) {
                best.score = sc;
                memcpy(best.R, nR, 72); memcpy(best.t, nt, 24);
            }
        }
    }
    free(pm); free(nm); free(moved); free(smat); free(ap); free(an);
    free(Pa); free(Qa); free(ones);
    return best;
}

void ora_dp_refine(const double *p, const double *q, const uint8_t *pv,
                   const uint8_t *nv, const double *R0, const double *t0,
                   double d0, double d0s, double sd8, double Lnorm, int N,
                   int max_iter, int lite, double *out13) {
    OraSeed r = dp_refine(p, q, pv, nv, R0, t0, d0, d0s, sd8, Lnorm, N, max_iter, lite);
    seed_out(&r, out13);
}

/* ---- secondary structure seeds (indialign_c/ss.h) ---------------------- */

/* assign_rna_ss: greedy first-come base pairs with C1'-C1' in [9,12] A for
 * (i,j) and (i+1,j-1), i ascending, j descending, j > i+3 (ss.h:16-52). */
void ora_assign_ss(const double *x, const uint8_t *v, int N, char *ss) {
    int *bp = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    const double lo = 81.0, hi = 144.0;
    for (int i = 0; i < N; i++) { ss[i] = 'L'; bp[i] = -1; }
    for (int i = 0; i < N - 4; i++) {
        if (!v[i] || !v[i + 1]) continue;
        for (int j = N - 1; j > i + 3; j--) {
            double a, b, dx, dy, dz;
            if (!v[j] || !v[j - 1]) continue;
            dx = x[i * 3] - x[j * 3]; dy = x[i * 3 + 1] - x[j * 3 + 1]; dz = x[i * 3 + 2] - x[j * 3 + 2];
            a = dx * dx + dy * dy + dz * dz;
            dx = x[(i + 1) * 3] - x[(j - 1) * 3]; dy = x[(i + 1) * 3 + 1] - x[(j - 1) * 3 + 1];
            dz = x[(i + 1) * 3 + 2] - x[(j - 1) * 3 + 2];
            b = dx * dx + dy * dy + dz * dz;
            if (a >= lo && a <= hi && b >= lo && b <= hi && bp[i] < 0 && bp[j] < 0) {
                bp[i] = j; bp[j] = i;
            }
        }
    }
    for (int i = 0; i < N; i++)
        if (bp[i] >= 0) ss[i] = i < bp[i] ? '<' : '>';
    free(bp);
}

/* ss_nw_align: identity of SS labels, gap -1 (ss.h:56-83) */
static int ss_nw_align(const char *sp_, const char *sn_, const uint8_t *pv,
                       const uint8_t *nv, int N, int *ap, int *an) {
    int *pm = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    int *nm = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    int plen = compact(pv, N, pm), nlen = compact(nv, N, nm), na = 0;
    if (plen >= 3 && nlen >= 3) {
        double *smat = (double *)malloc(sizeof(double) * (size_t)plen * (size_t)nlen);
        for (int a = 0; a < plen; a++)
            for (int b = 0; b < nlen; b++)
                smat[(size_t)a * nlen + b] = sp_[pm[a]] == sn_[nm[b]] ? 1.0 : 0.0;
        na = ora_nw_align(smat, plen, nlen, -1.0, ap, an);
        for (int i = 0; i < na; i++) { ap[i] = pm[ap[i]]; an[i] = nm[an[i]]; }
        free(smat);
    }
    free(pm); free(nm);
    return na;
}

/* evaluate_ss_seeds: IA2 (SS identity NW) then IA4 (distance + SS bonus NW
 * under the best transform so far), each followed by a detailed search and
 * a dp_refine (ss.h:87-164). */
static OraSeed ss_seeds(const double *pred, const double *native,
                        const uint8_t *pv, const uint8_t *nv, const char *ssp,
                        const char *ssn, const double *R0, const double *t0,
                        double d0, double d0s, double sd8, double Lnorm, int N,
                        int dp_iter) {
    OraSeed best, det, dp;
    int *ap = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    int *an = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    int *pm = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    int *nm = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    int na, plen, nlen;
    seed_ident(&best, -1e30);
    na = ss_nw_align(ssp, ssn, pv, nv, N, ap, an);
    if (na >= 3) {
        det = detailed_search(pred, native, ap, an, na, d0, d0s, sd8, Lnorm, 1, -1, MAX_FRAG_STARTS);
        if (det.score > best.score) best = det;
        if (dp_iter > 0) {
            dp = dp_refine(pred, native, pv, nv, best.R, best.t, d0, d0s, sd8, Lnorm, N, dp_iter, 0);
            if (dp.score > best.score) best = dp;
        }
    }
    plen = compact(pv, N, pm);
    nlen = compact(nv, N, nm);
    if (plen >= 3 && nlen >= 3) {
        const double *rR = best.score > -1e20 ? best.R : R0;
        const double *rt = best.score > -1e20 ? best.t : t0;
        double d01 = dmax(d0 + 1.5, d0s), d01sq = d01 * d01;
        double *moved = (double *)malloc(sizeof(double) * 3 * (size_t)N);
        double *smat = (double *)malloc(sizeof(double) * (size_t)plen * (size_t)nlen);
        for (int i = 0; i < N; i++)
            for (int d = 0; d < 3; d++)
                moved[i * 3 + d] = pred[i * 3] * rR[d] + pred[i * 3 + 1] * rR[3 + d] +
                                   pred[i * 3 + 2] * rR[6 + d] + rt[d];
        for (int a = 0; a < plen; a++) {
            const double *m = moved + 3 * pm[a];
            for (int b = 0; b < nlen; b++) {
                const double *n = native + 3 * nm[b];
                double dx = m[0] - n[0], dy = m[1] - n[1], dz = m[2] - n[2];
                double sc = 1.0 / (1.0 + (dx * dx + dy * dy + dz * dz) / d01sq);
                if (ssp[pm[a]] == ssn[nm[b]]) sc += 0.5;
                smat[(size_t)a * nlen + b] = sc;
            }
        }
        na = ora_nw_align(smat, plen, nlen, -1.0, ap, an);
        for (int i = 0; i < na; i++) { ap[i] = pm[ap[i]]; an[i] = nm[an[i]]; }
        if (na >= 3) {
            det = detailed_search(pred, native, ap, an, na, d0, d0s, sd8, Lnorm, 1, -1, MAX_FRAG_STARTS);
            if (det.score > best.score) best = det;
            if (dp_iter > 0) {
                dp = dp_refine(pred, native, pv, nv, best.R, best.t, d0, d0s, sd8, Lnorm, N, dp_iter, 0);
                if (dp.score > best.score) best = dp;
            }
        }
        free(moved); free(smat);
    }
    free(ap); free(an); free(pm); free(nm);
    return best;
}

/* ---- gapless threading (indialign_c/threading.h) ----------------------- */

/* refine_from_rt (threading.h:15-37) */
static void refine_from_rt(const double *p, const double *q, const uint8_t *v,
                           double d0s, int N, int n_iter, double *R, double *t,
                           uint8_t *sel) {
    double cut = d0s * d0s;
    int prev = -1;
    for (int it = 0; it < n_iter; it++) {
        int c = 0;
        for (int i = 0; i < N; i++) {
            if (!v[i]) { sel[i] = 0; continue; }
            sel[i] = dist2_at(p + 3 * i, q + 3 * i, R, t) <= cut;
            c += sel[i];
        }
        if (c >= 3) ora_kabsch(p, q, sel, N, R, t);
        if (c == prev) break;
        prev = c;
    }
}

/* gapless_threading_search: offsets k = -K..K step ceil(2K/100), k != 0;
 * Kabsch on pred[i] <-> native[i-k] where both valid; skip if fewer than
 * min_ali pairs; 5 same-index refinements; no-d8 score (threading.h:41-80).
 * plen/nlen are byte sums of the masks, as in the reference. */
static OraSeed gapless(const double *p, const double *q, const uint8_t *pv,
                       const uint8_t *nv, const uint8_t *v, double d0,
                       double d0s, double Lnorm, int N) {
    OraSeed best;
    int plen = 0, nlen = 0, min_ali, kr, stride;
    double *Pa, *Qa;
    uint8_t *pm, *sel;
    memset(&best, 0, sizeof best);
    best.score = -1e30;
    for (int i = 0; i < N; i++) { plen += pv[i]; nlen += nv[i]; }
    min_ali = imax(3, imin(plen, nlen) / 2);
    kr = N - min_ali;
    if (kr <= 0) return best;
    stride = imax(1, (2 * kr + 99) / 100);
    Pa = (double *)malloc(sizeof(double) * 3 * (size_t)N);
    Qa = (double *)malloc(sizeof(double) * 3 * (size_t)N);
    pm = (uint8_t *)malloc((size_t)N);
    sel = (uint8_t *)malloc((size_t)N);
    for (int k = -kr; k <= kr; k += stride) {
        int na = 0;
        double R[9], t[3], sc;
        if (k == 0) continue;
        for (int i = 0; i < N; i++) {
            int j = i - k;
            if (j < 0 || j >= N || !pv[i] || !nv[j]) continue;
            memcpy(Pa + 3 * na, p + 3 * i, 24);
            memcpy(Qa + 3 * na, q + 3 * j, 24);
            pm[na++] = 1;
        }
        if (na < min_ali) continue;
        ora_kabsch(Pa, Qa, pm, na, R, t);
        refine_from_rt(p, q, v, d0s, N, 5, R, t, sel);
        sc = ora_tm_score(p, q, v, R, t, d0, Lnorm, 0, N, 0);
        if (sc > best.score) {
            best.score = sc;
            memcpy(best.R, R, 72); memcpy(best.t, t, 24);
        }
    }
    free(Pa); free(Qa); free(pm); free(sel);
    return best;
}

void ora_gapless(const double *p, const double *q, const uint8_t *pv,
                 const uint8_t *nv, const uint8_t *v, double d0, double d0s,
                 double Lnorm, int N, double *out13) {
    OraSeed r = gapless(p, q, pv, nv, v, d0, d0s, Lnorm, N);
    seed_out(&r, out13);
}

/* ---- rescue passes (indialign_c/rescue.h) ------------------------------ */

/* local_frag_lengths (rescue.h:12-28) */
static int local_frag_lengths(int plen, int nlen, int dense, int *out) {
    int ml = imin(plen, nlen), n = 0;
    if (ml < 4) return 0;
    if (dense) {
        int vals[9] = {ml, imin(100, ml / 2), imin(32, ml), imin(24, ml), imin(20, ml / 3), 16, 12, 8, 4};
        for (int a = 0; a < 9; a++) {
            int seen = 0;
            if (vals[a] < 4) continue;
            for (int b = 0; b < n; b++) seen |= out[b] == vals[a];
            if (!seen) out[n++] = vals[a];
        }
    } else {
        int a = imin(20, ml / 3), b = imin(100, ml / 2);
        if (a >= 4) out[n++] = a;
        if (b >= 4 && b != a) out[n++] = b;
    }
    return n;
}

/* local_jump (rescue.h:30-46) */
static int local_jump(int length, int dense) {
    int j;
    if (dense) {
        if (length > 350) j = 50;
        else if (length > 300) j = 30;
        else if (length > 200) j = 10;
        else j = 5;
        return imax(1, imin(j, imax(1, length / 4)));
    }
    if (length > 250) j = 45;
    else if (length > 200) j = 35;
    else if (length > 150) j = 25;
    else j = 15;
    return imax(1, imin(j, imax(1, length / 3)));
}

/* evaluate_local_fragment_dp: windows (flen, ps, ns) over the compact valid
 * lists; Kabsch on the window pair -> dp_refine(2 iterations, lite,
 * sd8 = 100); first max over windows (rescue.h:50-117, serial path). */
static OraSeed local_fragment_dp(const double *p, const double *q,
                                 const uint8_t *pv, const uint8_t *nv,
                                 double d0, double d0s, double Lnorm, int N,
                                 int dense) {
    OraSeed best;
    int *pm = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    int *nm = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    int plen = compact(pv, N, pm), nlen = compact(nv, N, nm), fl[9], nf, jp, jn;
    seed_ident(&best, -1e30);
    nf = local_frag_lengths(plen, nlen, dense, fl);
    jp = local_jump(plen, dense);
    jn = local_jump(nlen, dense);
    if (nf > 0) {
        double *Pf = (double *)malloc(sizeof(double) * 3 * (size_t)(N + 1));
        double *Qf = (double *)malloc(sizeof(double) * 3 * (size_t)(N + 1));
        uint8_t *ones = (uint8_t *)malloc((size_t)N + 1);
        for (int a = 0; a < nf; a++) {
            int flen = fl[a], plim = plen - flen + 1, nlim = nlen - flen + 1;
            if (plim <= 0 || nlim <= 0) continue;
            for (int ps = 0; ps < plim; ps += jp)
                for (int ns = 0; ns < nlim; ns += jn) {
                    double sR[9], st[3];
                    OraSeed dp;
                    for (int i = 0; i < flen; i++) {
                        memcpy(Pf + 3 * i, p + 3 * pm[ps + i], 24);
                        memcpy(Qf + 3 * i, q + 3 * nm[ns + i], 24);
                        ones[i] = 1;
                    }
                    ora_kabsch(Pf, Qf, ones, flen, sR, st);
                    dp = dp_refine(p, q, pv, nv, sR, st, d0, d0s, 100.0, Lnorm, N, 2, 1);
                    if (dp.score > best.score) best = dp;
                }
        }
        free(Pf); free(Qf); free(ones);
    }
    free(pm); free(nm);
    return best;
}

void ora_local_fragment_dp(const double *p, const double *q, const uint8_t *pv,
                           const uint8_t *nv, double d0, double d0s,
                           double Lnorm, int N, int dense, double *out13) {
    OraSeed r = local_fragment_dp(p, q, pv, nv, d0, d0s, Lnorm, N, dense);
    seed_out(&r, out13);
}

/* evaluate_threading_dp: offsets -(nlen-3) .. plen-3 step min/50; detailed
 * search (fragments, 8 iterations, 5 starts, sd8 = 100) on the shifted
 * compact pairs, then dp_refine(1, lite) from it; the better of the two
 * (rescue.h:121-190, serial path). */
static OraSeed threading_dp(const double *p, const double *q, const uint8_t *pv,
                            const uint8_t *nv, double d0, double d0s,
                            double Lnorm, int N) {
    OraSeed best;
    int *pm = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    int *nm = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    int plen = compact(pv, N, pm), nlen = compact(nv, N, nm), step;
    seed_ident(&best, -1e30);
    if (imin(plen, nlen) >= 3) {
        int *ap = (int *)malloc(sizeof(int) * (size_t)(N + 1));
        int *an = (int *)malloc(sizeof(int) * (size_t)(N + 1));
        step = imax(1, imin(plen, nlen) / 50);
        for (int off = -(nlen - 3); off < plen - 2; off += step) {
            int ps = imax(off, 0), ns = imax(-off, 0), ov = imin(plen - ps, nlen - ns);
            OraSeed det, dp, cand;
            if (ov < 3) continue;
            for (int i = 0; i < ov; i++) { ap[i] = pm[ps + i]; an[i] = nm[ns + i]; }
            det = detailed_search(p, q, ap, an, ov, d0, d0s, 100.0, Lnorm, 1, 8, 5);
            dp = dp_refine(p, q, pv, nv, det.R, det.t, d0, d0s, 100.0, Lnorm, N, 1, 1);
            cand = dp.score > det.score ? dp : det;
            cand.score = dmax(det.score, dp.score);
            if (cand.score > best.score) best = cand;
        }
        free(ap); free(an);
    }
    free(pm); free(nm);
    return best;
}

void ora_threading_dp(const double *p, const double *q, const uint8_t *pv,
                      const uint8_t *nv, double d0, double d0s, double Lnorm,
                      int N, double *out13) {
    OraSeed r = threading_dp(p, q, pv, nv, d0, d0s, Lnorm, N);
    seed_out(&r, out13);
}

/* ---- the search (indialign_c/indialign.cpp:29-266) --------------------- */

static void upd(OraSeed *best, const double *R, const double *t, double sc) {
    if (sc > best->score) {
        best->score = sc;
        if (R != best->R) memcpy(best->R, R, 72);
        if (t != best->t) memcpy(best->t, t, 24);
    }
}

static void trace_put(double *st, int s, const OraSeed *b) {
    if (st) seed_out(b, st + 13 * s);
}

static OraSeed search(const double *pred, const double *native,
                      const uint8_t *valid, const uint8_t *pv, const uint8_t *nv,
                      int N, double Lnorm, const OraConfig *cfg, double *st) {
    OraSeed best, r;
    double d0, d0s, sd8, cand[11];
    int C, has_cross = 0, use_frag = cfg->use_fragment_search != 0;
    int max_iter = cfg->max_iter, dp_iter = cfg->dp_iter;
    masklist L = {0, 0, 0, N};
    if (st) for (int s = 0; s < ORA_STAGES; s++) st[13 * s] = -2e30;
    if (Lnorm <= 2.0) { seed_ident(&best, 0); return best; }
    ora_d0(Lnorm, &d0, &d0s, &sd8);
    C = ora_d0_candidates(d0, d0s, cand);
    build_seed_masks(N, valid, use_frag, MAX_FRAG_STARTS, &L);
    anchor_seeds(pred, native, valid, N, d0s, d0, 5, &L);
    if (L.K == 0) { free(L.m); seed_ident(&best, 0); return best; }
    /* 2. seed bank, same-index no-d8 scoring */
    best = seed_bank(pred, native, valid, L.m, L.K, cand, C, d0, sd8, Lnorm, N,
                     max_iter, 0, cfg->early_term_score);
    free(L.m);
    trace_put(st, 0, &best);
    /* 2b. SS seeds, rescored same-index */
    {
        char *ssp = (char *)malloc((size_t)N + 1), *ssn = (char *)malloc((size_t)N + 1);
        ora_assign_ss(pred, pv, N, ssp);
        ora_assign_ss(native, nv, N, ssn);
        r = ss_seeds(pred, native, pv, nv, ssp, ssn, best.R, best.t, d0, d0s,
                     sd8, Lnorm, N, dp_iter);
        r.score = ora_tm_score(pred, native, valid, r.R, r.t, d0, Lnorm, 0, N, 0);
        if (r.score > best.score) best = r;
        free(ssp); free(ssn);
    }
    trace_put(st, 1, &best);
    /* 2c. gapless threading */
    r = gapless(pred, native, pv, nv, valid, d0, d0s, Lnorm, N);
    if (r.score > best.score) best = r;
    trace_put(st, 2, &best);
    /* 3. rescue ladder */
    for (int i = 0; i < N && !has_cross; i++) has_cross = pv[i] != nv[i];
    if (best.score < cfg->rescue_score_1) {
        r = local_fragment_dp(pred, native, pv, nv, d0, d0s, Lnorm, N, 0);
        r.score = ora_tm_score(pred, native, valid, r.R, r.t, d0, Lnorm, 0, N, 0);
        if (r.score > best.score) best = r;
        trace_put(st, 3, &best);
    }
    if (best.score < cfg->rescue_score_1) {
        r = threading_dp(pred, native, pv, nv, d0, d0s, Lnorm, N);
        r.score = ora_tm_score(pred, native, valid, r.R, r.t, d0, Lnorm, 0, N, 0);
        if (r.score > best.score) best = r;
        trace_put(st, 4, &best);
    }
    if (best.score < cfg->rescue_score_2) {
        r = local_fragment_dp(pred, native, pv, nv, d0, d0s, Lnorm, N, 1);
        r.score = ora_tm_score(pred, native, valid, r.R, r.t, d0, Lnorm, 0, N, 0);
        if (r.score > best.score) best = r;
        trace_put(st, 5, &best);
    }
    /* 4. top-50% distance seed */
    {
        double *d2 = (double *)malloc(sizeof(double) * (size_t)N);
        uint8_t *tk = (uint8_t *)malloc((size_t)N);
        int tkc = 0;
        for (int i = 0; i < N; i++)
            d2[i] = valid[i] ? dist2_at(pred + 3 * i, native + 3 * i, best.R, best.t) : 1e12;
        ora_topk_seed(d2, valid, N, 0.5, tk);
        for (int i = 0; i < N; i++) tkc += tk[i];
        if (tkc >= 3) {
            r = seed_bank(pred, native, valid, tk, 1, cand, C, d0, sd8, Lnorm, N,
                          max_iter, 0, cfg->early_term_score);
            if (r.score > best.score) best = r;
        }
        free(d2); free(tk);
    }
    trace_put(st, 6, &best);
    /* 5. DP refinement, every candidate rescored same-index */
    if (dp_iter > 0) {
        double seed_score = best.score, dp_id;
        OraSeed dp = dp_refine(pred, native, pv, nv, best.R, best.t, d0, d0s, sd8,
                               Lnorm, N, dp_iter, 0);
        dp_id = ora_tm_score(pred, native, valid, dp.R, dp.t, d0, Lnorm, 0, N, 0);
        upd(&best, dp.R, dp.t, dp_id);
        upd(&best, best.R, best.t,
            ora_tm_score(pred, native, valid, best.R, best.t, d0, Lnorm, 0, N, 0));
        if (has_cross) {
            OraSeed idp = dp_refine(pred, native, pv, nv, IDENT, (const double[3]){0, 0, 0},
                                    d0, d0s, sd8, Lnorm, N, dp_iter, 1);
            int extra = imax(0, 5 - dp_iter);
            upd(&best, idp.R, idp.t,
                ora_tm_score(pred, native, valid, idp.R, idp.t, d0, Lnorm, 0, N, 0));
            if (extra > 0 && best.score < 0.36) {
                int use_seed = seed_score > dp_id;
                double eR[9], et[3];
                OraSeed ex;
                memcpy(eR, use_seed ? best.R : dp.R, 72);
                memcpy(et, use_seed ? best.t : dp.t, 24);
                ex = dp_refine(pred, native, pv, nv, eR, et, d0, d0s, sd8, Lnorm, N, extra, 1);
                upd(&best, ex.R, ex.t,
                    ora_tm_score(pred, native, valid, ex.R, ex.t, d0, Lnorm, 0, N, 0));
            }
        }
    } else {
        upd(&best, best.R, best.t,
            ora_tm_score(pred, native, valid, best.R, best.t, d0, Lnorm, 0, N, 0));
    }
    trace_put(st, 7, &best);
    /* 5b. DP from same-index-offset Kabsch starts */
    if (dp_iter > 0) {
        double *Pa = (double *)malloc(sizeof(double) * 3 * (size_t)N);
        double *Qa = (double *)malloc(sizeof(double) * 3 * (size_t)N);
        uint8_t *pm = (uint8_t *)malloc((size_t)N);
        int stride = imax(1, N / 10);
        for (int k = -N / 2; k <= N / 2; k += stride) {
            int na = 0;
            double sR[9], stt[3];
            OraSeed tdp;
            if (k == 0) continue;
            for (int i = 0; i < N; i++) {
                int j = i - k;
                if (j < 0 || j >= N || !pv[i] || !nv[j]) continue;
                memcpy(Pa + 3 * na, pred + 3 * i, 24);
                memcpy(Qa + 3 * na, native + 3 * j, 24);
                pm[na++] = 1;
            }
            if (na < 3) continue;
            ora_kabsch(Pa, Qa, pm, na, sR, stt);
            tdp = dp_refine(pred, native, pv, nv, sR, stt, d0, d0s, sd8, Lnorm, N, dp_iter, 1);
            upd(&best, tdp.R, tdp.t,
                ora_tm_score(pred, native, valid, tdp.R, tdp.t, d0, Lnorm, 0, N, 0));
        }
        free(Pa); free(Qa); free(pm);
    }
    trace_put(st, 8, &best);
    /* 6. weighted TM refinement, 4 iterations */
    {
        double wR[9], wt[3], ws;
        memcpy(wR, best.R, 72); memcpy(wt, best.t, 24);
        ora_weighted_refine(pred, native, valid, d0, Lnorm, N, 4, wR, wt, &ws);
        upd(&best, wR, wt, ws);
    }
    trace_put(st, 9, &best);
    return best;
}

void ora_default_config(OraConfig *c) {
    c->backend_mode = 0;
    c->use_fragment_search = 1;
    c->max_iter = 20;
    c->dp_iter = 1;
    c->max_mem_gb = 20.0;
    c->request_cuda = 0;
    c->rescue_score_1 = 0.5;
    c->rescue_score_2 = 0.3;
    c->early_term_score = 0.99;
}

static int run_one(const OraPairInput *in, const OraConfig *cfg,
                   OraPairResult *out, double *st) {
    OraSeed b;
    if (in->length <= 0) return -1;
    b = search(in->pred_xyz, in->native_xyz, in->valid_mask, in->pred_valid_mask,
               in->native_valid_mask, in->length, in->lnorm, cfg, st);
    out->score = b.score;
    memcpy(out->rotation, b.R, 72);
    memcpy(out->translation, b.t, 24);
    return 0;
}

int ora_tmscore_search(const OraPairInput *in, const OraConfig *cfg, OraPairResult *out) {
    return run_one(in, cfg, out, 0);
}

int ora_trace_search(const OraPairInput *in, const OraConfig *cfg,
                     double *stage_best, OraPairResult *out) {
    return run_one(in, cfg, out, stage_best);
}

int ora_tmscore_search_batch(int n, const OraPairInput *in, const OraConfig *cfg,
                     OraPairResult *out) {
#pragma omp parallel for schedule(dynamic)
    for (int p = 0; p < n; p++) run_one(in + p, cfg, out + p, 0);
    return 0;
}
