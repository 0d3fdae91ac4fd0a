// Test-only extern "C" wrappers around the reference's header-only stage
// functions (indialign_c/*.h), compiled against the reference headers where
// they lie (-I$(REF_DIR)); nothing from the reference is copied here.  The
// tests use these to check the C restatement and the CUDA kernels stage by
// stage on identical inputs.
//
// ref_trace_search() replays the stage order of do_tmscore_search
// (indialign_c/indialign.cpp:29-266) through the same reference functions and
// records the running best after every stage, so that a stage-level mismatch
// can be located.  Its final result must equal indialign_tmscore_search()'s.
#include "api.h"
#include "core.h"
#include "seeds.h"
#include "search.h"
#include "align.h"
#include "rescue.h"
#include "threading.h"
#include "ss.h"
#include "nw.h"

#include <cstring>
#include <vector>

extern "C" {

void ref_d0(double L, double *d0, double *d0s, double *sd8) {
    d0_from_length_rna(L, d0, d0s, sd8);
}

void ref_kabsch(const double *P, const double *Q, const uint8_t *mask, int N,
                double *R, double *t) {
    kabsch(P, Q, mask, N, R, t);
}

void ref_cov_to_rotation(const double *H9, double *R) {
    double H[3][3];
    for (int i = 0; i < 9; i++) H[i / 3][i % 3] = H9[i];
    cov_to_rotation(H, R);
}

double ref_tm_score(const double *p, const double *q, const uint8_t *v,
                    const double *R, const double *t, double d0, double Lnorm,
                    double sd8, int N, int use_d8) {
    if (use_d8) return tm_score(p, q, v, R, t, d0, Lnorm, sd8, N);
    return tm_score_no_d8(p, q, v, R, t, d0, Lnorm, N);
}

// H_out: (Np+1)*(Nn+1) doubles, trace_out: same count of int8.
void ref_nw_dp(const double *smat, int Np, int Nn, double gap,
               double *H_out, int8_t *trace_out) {
    std::vector<double> H;
    std::vector<int8_t> tr;
    nw_dp(smat, Np, Nn, H, tr, gap);
    std::memcpy(H_out, H.data(), H.size() * sizeof(double));
    std::memcpy(trace_out, tr.data(), tr.size());
}

int ref_nw_align(const double *smat, int Np, int Nn, double gap,
                 int *ap, int *an) {
    std::vector<double> H;
    std::vector<int8_t> tr;
    nw_dp(smat, Np, Nn, H, tr, gap);
    return nw_traceback(tr, Np, Nn, ap, an, std::min(Np, Nn));
}

void ref_iterative_seed_refine(const double *p, const double *q,
                               const uint8_t *valid, const uint8_t *seed,
                               double d0s, int N, int max_iter,
                               double *R, double *t) {
    std::vector<uint8_t> w(N), s(N);
    iterative_seed_refine(p, q, valid, seed, d0s, N, max_iter, R, t,
                          w.data(), s.data());
}

// masks_out must hold max_K*N bytes; returns K (or -1 if max_K too small).
int ref_seed_masks(int N, const uint8_t *valid, int use_frag, int max_starts,
                   uint8_t *masks_out, int max_K) {
    std::vector<uint8_t> m;
    int K = 0;
    build_seed_masks(N, valid, use_frag != 0, m, K, max_starts);
    if (K > max_K) return -1;
    std::memcpy(masks_out, m.data(), (size_t)K * N);
    return K;
}

// Seeds = fragment masks + anchor contact masks, exactly as
// do_tmscore_search builds them (indialign.cpp:70-75).
int ref_all_seeds(const double *p, const double *q, const uint8_t *valid,
                  int N, double d0s, double d0, int use_frag,
                  uint8_t *masks_out, int max_K) {
    std::vector<uint8_t> m;
    int K = 0;
    build_seed_masks(N, valid, use_frag != 0, m, K);
    build_anchor_contact_seeds(p, q, valid, N, d0s, d0, 5, m, K);
    if (K > max_K) return -1;
    std::memcpy(masks_out, m.data(), (size_t)K * N);
    return K;
}

static void put(const SeedResult &r, double *out13) {
    out13[0] = r.score;
    std::memcpy(out13 + 1, r.R, 72);
    std::memcpy(out13 + 10, r.t, 24);
}

void ref_seed_bank(const double *p, const double *q, const uint8_t *valid,
                   const uint8_t *seeds, int K, const double *cands, int C,
                   double d0, double sd8, double Lnorm, int N, int max_iter,
                   int use_d8, double early_term, double *out13) {
    put(evaluate_seed_bank(p, q, valid, seeds, K, cands, C, d0, sd8, Lnorm, N,
                           max_iter, use_d8 != 0, early_term), out13);
}

void ref_detailed_search(const double *p, const double *q, const int *ap,
                         const int *an, int na, double d0, double d0s,
                         double sd8, double Lnorm, int N, int use_frag,
                         int max_iter_override, int max_starts, double *out13) {
    put(alignment_detailed_search(p, q, ap, an, na, d0, d0s, sd8, Lnorm, N,
                                  use_frag != 0, max_iter_override, max_starts),
        out13);
}

void ref_dp_refine(const double *p, const double *q, const uint8_t *v,
                   const uint8_t *pv, const uint8_t *nv, const double *R0,
                   const double *t0, double d0, double d0s, double sd8,
                   double Lnorm, int N, int max_iter, int lite, double *out13) {
    put(dp_refine(p, q, v, pv, nv, R0, t0, d0, d0s, sd8, Lnorm, N, max_iter,
                  lite != 0), out13);
}

void ref_assign_ss(const double *xyz, const uint8_t *v, int N, char *ss) {
    assign_rna_ss(xyz, v, N, ss);
}

void ref_gapless(const double *p, const double *q, const uint8_t *pv,
                 const uint8_t *nv, const uint8_t *v, double d0, double d0s,
                 double Lnorm, int N, double *out13) {
    put(gapless_threading_search(p, q, pv, nv, v, d0, d0s, Lnorm, N), out13);
}

void ref_local_fragment_dp(const double *p, const double *q, const uint8_t *v,
                           const uint8_t *pv, const uint8_t *nv, double d0,
                           double d0s, double Lnorm, int N, int dense,
                           double *out13) {
    put(evaluate_local_fragment_dp(p, q, v, pv, nv, d0, d0s, Lnorm, N,
                                   dense != 0), out13);
}

void ref_threading_dp(const double *p, const double *q, const uint8_t *v,
                      const uint8_t *pv, const uint8_t *nv, double d0,
                      double d0s, double Lnorm, int N, double *out13) {
    put(evaluate_threading_dp(p, q, v, pv, nv, d0, d0s, Lnorm, N), out13);
}

void ref_topk_seed(const double *d2, const uint8_t *valid, int N, double frac,
                   uint8_t *mask) {
    build_topk_seed(d2, valid, N, frac, mask);
}

void ref_weighted_refine(const double *p, const double *q, const uint8_t *v,
                         double d0, double Lnorm, int N, int n_iters,
                         double *R, double *t, double *score) {
    weighted_tm_refine(p, q, v, d0, Lnorm, N, n_iters, R, t, score);
}

// Candidate schedules (seeds.h:15-37, rescue.h:12-46): each writes at most
// cap entries and returns the count, or -1 when cap is too small.
static int put_list(const std::vector<int> &v, int *out, int cap) {
    if ((int)v.size() > cap) return -1;
    std::copy(v.begin(), v.end(), out);
    return (int)v.size();
}

int ref_fragment_lengths(int max_len, int *out, int cap) {
    return put_list(fragment_lengths(max_len), out, cap);
}

int ref_start_positions(int n, int frag, int ms, int *out, int cap) {
    return put_list(start_positions(n, frag, ms), out, cap);
}

int ref_local_frag_lengths(int plen, int nlen, int dense, int *out, int cap) {
    return put_list(local_frag_lengths(plen, nlen, dense != 0), out, cap);
}

int ref_local_jump(int length, int dense) { return local_jump(length, dense != 0); }

// Stage names in the order the search runs them; stage_best receives one
// {score,R[9],t[3]} record per stage (13 doubles), taken after the stage.
enum { ST_SEED_BANK, ST_SS, ST_GAPLESS, ST_LOCAL, ST_THREAD_DP, ST_DENSE,
       ST_TOPK, ST_DP, ST_OFFSET_DP, ST_WEIGHTED, ST_COUNT };

int ref_trace_stage_count(void) { return ST_COUNT; }

int ref_trace_search(const NativePairInput *inp, const NativeConfig *cfg,
                     double *stage_best, NativePairResult *out) {
    const int N = inp->length;
    if (N <= 0) return -1;
    const double *pred = inp->pred_xyz, *native = inp->native_xyz;
    const uint8_t *valid = inp->valid_mask, *pv = inp->pred_valid_mask,
                  *nv = inp->native_valid_mask;
    const double Lnorm = inp->lnorm;
    const int max_iter = cfg->max_iter, dp_iter = cfg->dp_iter;
    const bool use_frag = cfg->use_fragment_search != 0;
    for (int s = 0; s < ST_COUNT; s++) stage_best[s * 13] = -2e30;

    SeedResult best;
    auto finish = [&](const SeedResult &r) {
        out->score = r.score;
        std::memcpy(out->rotation, r.R, 72);
        std::memcpy(out->translation, r.t, 24);
        return 0;
    };
    auto ident = []() {
        SeedResult r; r.score = 0;
        double I[9] = {1,0,0,0,1,0,0,0,1}; std::memcpy(r.R, I, 72);
        r.t[0] = r.t[1] = r.t[2] = 0; return r;
    };
    if (Lnorm <= 2.0) return finish(ident());
    double d0, d0s, sd8;
    d0_from_length_rna(Lnorm, &d0, &d0s, &sd8);
    double cand[11]; int C = 0;
    for (int c = 0; c < N_D0_MULTS; c++) cand[C++] = d0s * D0_MULTS[c];
    for (int c = 1; c <= 5; c++) {
        double v = d0 + c; bool dup = false;
        for (int e = 0; e < C && !dup; e++) dup = std::abs(cand[e] - v) < 0.01;
        if (!dup) cand[C++] = v;
    }
    std::vector<uint8_t> sm; int K = 0;
    build_seed_masks(N, valid, use_frag, sm, K);
    build_anchor_contact_seeds(pred, native, valid, N, d0s, d0, 5, sm, K);
    if (K == 0) return finish(ident());
    auto rescore = [&](SeedResult &r) {
        r.score = tm_score_no_d8(pred, native, valid, r.R, r.t, d0, Lnorm, N);
    };
    best = evaluate_seed_bank(pred, native, valid, sm.data(), K, cand, C, d0,
                              sd8, Lnorm, N, max_iter, false,
                              cfg->early_term_score);
    put(best, stage_best + ST_SEED_BANK * 13);
    std::vector<char> ssp(N), ssn(N);
    assign_rna_ss(pred, pv, N, ssp.data());
    assign_rna_ss(native, nv, N, ssn.data());
    auto ss = evaluate_ss_seeds(pred, native, valid, pv, nv, ssp.data(),
                                ssn.data(), best.R, best.t, d0, d0s, sd8,
                                Lnorm, N, dp_iter);
    rescore(ss);
    if (ss.score > best.score) best = ss;
    put(best, stage_best + ST_SS * 13);
    auto gt = gapless_threading_search(pred, native, pv, nv, valid, d0, d0s,
                                       Lnorm, N);
    if (gt.score > best.score) best = gt;
    put(best, stage_best + ST_GAPLESS * 13);
    bool has_cross = false;
    for (int i = 0; i < N && !has_cross; i++) has_cross = pv[i] != nv[i];
    if (best.score < cfg->rescue_score_1) {
        auto lf = evaluate_local_fragment_dp(pred, native, valid, pv, nv, d0,
                                             d0s, Lnorm, N, false);
        rescore(lf);
        if (lf.score > best.score) best = lf;
        put(best, stage_best + ST_LOCAL * 13);
    }
    if (best.score < cfg->rescue_score_1) {
        auto th = evaluate_threading_dp(pred, native, valid, pv, nv, d0, d0s,
                                        Lnorm, N);
        rescore(th);
        if (th.score > best.score) best = th;
        put(best, stage_best + ST_THREAD_DP * 13);
    }
    if (best.score < cfg->rescue_score_2) {
        auto dl = evaluate_local_fragment_dp(pred, native, valid, pv, nv, d0,
                                             d0s, Lnorm, N, true);
        rescore(dl);
        if (dl.score > best.score) best = dl;
        put(best, stage_best + ST_DENSE * 13);
    }
    std::vector<double> d2v(N);
    dist2_fused(pred, native, valid, best.R, best.t, d2v.data(), N);
    std::vector<uint8_t> tk(N);
    build_topk_seed(d2v.data(), valid, N, 0.5, tk.data());
    int tkc = 0;
    for (int i = 0; i < N; i++) tkc += tk[i];
    if (tkc >= 3) {
        auto tp = evaluate_seed_bank(pred, native, valid, tk.data(), 1, cand,
                                     C, d0, sd8, Lnorm, N, max_iter, false,
                                     cfg->early_term_score);
        if (tp.score > best.score) best = tp;
    }
    put(best, stage_best + ST_TOPK * 13);
    auto upd = [&](const double *R, const double *t, double sc) {
        if (sc > best.score) {
            best.score = sc;
            if (R != best.R) std::memcpy(best.R, R, 72);
            if (t != best.t) std::memcpy(best.t, t, 24);
        }
    };
    if (dp_iter > 0) {
        double seed_score = best.score;
        auto dp = dp_refine(pred, native, valid, pv, nv, best.R, best.t, d0,
                            d0s, sd8, Lnorm, N, dp_iter, false);
        double dp_id = tm_score_no_d8(pred, native, valid, dp.R, dp.t, d0,
                                      Lnorm, N);
        upd(dp.R, dp.t, dp_id);
        double oid = tm_score_no_d8(pred, native, valid, best.R, best.t, d0,
                                    Lnorm, N);
        upd(best.R, best.t, oid);
        if (has_cross) {
            double I[9] = {1,0,0,0,1,0,0,0,1}, z[3] = {};
            auto idp = dp_refine(pred, native, valid, pv, nv, I, z, d0, d0s,
                                 sd8, Lnorm, N, dp_iter, true);
            upd(idp.R, idp.t, tm_score_no_d8(pred, native, valid, idp.R,
                                             idp.t, d0, Lnorm, N));
            int extra = std::max(0, 5 - dp_iter);
            if (extra > 0 && best.score < 0.36) {
                bool use_seed = seed_score > dp_id;
                const double *eR = use_seed ? best.R : dp.R;
                const double *et = use_seed ? best.t : dp.t;
                auto ex = dp_refine(pred, native, valid, pv, nv, eR, et, d0,
                                    d0s, sd8, Lnorm, N, extra, true);
                upd(ex.R, ex.t, tm_score_no_d8(pred, native, valid, ex.R,
                                               ex.t, d0, Lnorm, N));
            }
        }
    } else {
        upd(best.R, best.t, tm_score_no_d8(pred, native, valid, best.R,
                                           best.t, d0, Lnorm, N));
    }
    put(best, stage_best + ST_DP * 13);
    if (dp_iter > 0) {
        std::vector<double> Pa(N * 3), Qa(N * 3);
        std::vector<uint8_t> pm(N);
        int stride = std::max(1, N / 10);
        for (int k = -N / 2; k <= N / 2; k += stride) {
            if (k == 0) continue;
            int na = 0;
            for (int i = 0; i < N; i++) {
                int j = i - k;
                if (j < 0 || j >= N || !pv[i] || !nv[j]) continue;
                std::memcpy(&Pa[na * 3], &pred[i * 3], 24);
                std::memcpy(&Qa[na * 3], &native[j * 3], 24);
                pm[na++] = 1;
            }
            if (na < 3) continue;
            double sR[9], st[3];
            kabsch(Pa.data(), Qa.data(), pm.data(), na, sR, st);
            auto tdp = dp_refine(pred, native, valid, pv, nv, sR, st, d0, d0s,
                                 sd8, Lnorm, N, dp_iter, true);
            upd(tdp.R, tdp.t, tm_score_no_d8(pred, native, valid, tdp.R,
                                             tdp.t, d0, Lnorm, N));
        }
    }
    put(best, stage_best + ST_OFFSET_DP * 13);
    double wR[9], wt[3], ws;
    std::memcpy(wR, best.R, 72); std::memcpy(wt, best.t, 24);
    weighted_tm_refine(pred, native, valid, d0, Lnorm, N, 4, wR, wt, &ws);
    upd(wR, wt, ws);
    put(best, stage_best + ST_WEIGHTED * 13);
    return finish(best);
}

}  // extern "C"

#include <algorithm>
#include <utility>

extern "C" {

// std::sort with the comparator of build_anchor_contact_seeds
// (indialign_c/seeds.h:237-238): order by count only, descending.
void ref_std_sort_desc(int *keys, int *idx, int n) {
    std::vector<std::pair<int, int>> v(n);
    for (int i = 0; i < n; i++) v[i] = {keys[i], idx[i]};
    std::sort(v.begin(), v.end(), [](auto &x, auto &y) { return x.first > y.first; });
    for (int i = 0; i < n; i++) { keys[i] = v[i].first; idx[i] = v[i].second; }
}

}  // extern "C"
