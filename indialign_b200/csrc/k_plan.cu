// Stage planning, chain reductions and per-pair stage glue.
//
// Plan kernels fill one task descriptor per slot from device state (so a
// gated-off pair gets zero work without a host round trip); chain reducers
// apply the reference's combine rules over a pair's chain results; glue ops
// are the reference's per-pair control flow between stages
// (indialign_c/indialign.cpp:90-264, ss.h:87-164, align.h:54-145).
#include "dmath.cuh"
#include "pipeline.h"
#include "kernels.h"
#include "sched.cuh"

namespace ia {

IA_DEV void rec_copy(double *d, const double *s) {
    for (int a = 0; a < kRec; a++) d[a] = s[a];
}
IA_DEV void rec_ident(double *d, double score) {
    for (int a = 0; a < kRec; a++) d[a] = (a == 1 || a == 5 || a == 9) ? 1.0 : 0.0;
    d[0] = score;
}

// ---- bank plans -------------------------------------------------------------
__global__ void k_plan_bank(DevBatch b, PlanCtx c) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= c.ntasks) return;
    const int p = c.pair ? c.pair[s] : s;
    const int aux = c.aux ? c.aux[s] : 0;
    const PairInfo &I = b.info[p];
    PairState &S = b.state[p];
    BankTask T;
    T.P = b.pred + 3 * (size_t)I.off;
    T.Q = b.nat + 3 * (size_t)I.off;
    T.V = b.v + I.off;
    T.PV = T.NV = nullptr;
    T.table = nullptr;
    T.slist = nullptr;
    T.bits = b.bits + I.bitoff;
    T.words = I.words;
    T.cut = I.cut;
    T.n = I.N;
    T.K = 0;
    T.C = I.C;
    T.mode = SEED_TABLE;
    T.ms = 50;
    T.max_iter = c.max_iter;
    T.use_d8 = 0;
    T.shift_lo = T.shift_stride = 1;
    T.shift_min = 0;
    T.d0 = I.d0;
    T.sd8 = I.sd8;
    T.lnorm = I.lnorm;
    T.early_term = c.early_term;
    T.pair = p;
    T.out_rec = -1;
    T.out = nullptr;
    T.item_base = c.base ? (int)c.base[s] : 0;
    bool on = I.status == 0;
    switch (c.kind) {
    case BK_MAIN:  // seed bank, same-index no-d8 (indialign.cpp:100-103)
        T.table = b.seeds + (size_t)p * kMaxSeeds;
        T.K = I.K;
        T.out_rec = REC_BEST;
        if (c.wcount && c.wcount[p] >= 0) {  // ranked: the selected seeds only
            T.K = c.wcount[p];
            T.slist = c.wlist + (size_t)p * kMaxTopK;
        }
        break;
    case BK_DET_SS:  // detailed search with fragments on an SS alignment
    case BK_DET_DP: {  // ... or on a dp_refine alignment (align.h:115-118)
        const int g = c.kind == BK_DET_SS ? 0 : aux;
        const int na = S.na[g];
        T.P = c.alP + 3 * (2 * (size_t)I.off + (size_t)g * I.N);
        T.Q = c.alQ + 3 * (2 * (size_t)I.off + (size_t)g * I.N);
        T.V = nullptr;
        T.n = na;
        T.mode = SEED_ARITH;
        T.ms = 50;
        T.K = arith_seed_count(na, 50, true);
        T.C = kDetC;
        T.cut = I.dcut;
        T.max_iter = 20;
        T.use_d8 = 1;
        T.early_term = 1.0;
        T.out_rec = REC_DET0 + g;
        on = on && na >= 3 && (c.kind == BK_DET_SS ? S.flag : S.active[g]);
        if (c.wcount) {  // ranked: the selected seeds only (task = pair x slot)
            const int task = kDetSlots * p + g;
            if (c.wcount[task] >= 0) {
                T.K = c.wcount[task];
                T.slist = c.wlist + (size_t)task * kMaxTopK;
            }
        }
        break;
    }
    case BK_GAPLESS: {  // gapless threading (threading.h:41-80)
        int kr, stride, min_ali;
        gapless_params(I.N, I.pvsum, I.nvsum, kr, stride, min_ali);
        T.PV = b.pv + I.off;
        T.NV = b.nv + I.off;
        T.mode = SEED_SHIFT;
        T.shift_lo = -kr;
        T.shift_stride = stride;
        T.shift_min = min_ali;
        T.K = kr > 0 ? offsets_count(-kr, kr, stride) : 0;
        T.C = 1;
        T.cut = &I.dcut[2];  // d0_search x 1.0
        T.max_iter = 5;
        T.early_term = 1e300;
        T.out_rec = REC_STAGE;
        on = on && kr > 0;
        S.flag = on;
        break;
    }
    case BK_THREAD: {  // threading-DP detailed search (rescue.h:146-161)
        int ps, ns, ov;
        thread_at(I.plen, I.nlen, aux, ps, ns, ov);
        T.P = b.predc + 3 * (size_t)(I.off + ps);
        T.Q = b.natc + 3 * (size_t)(I.off + ns);
        T.V = nullptr;
        T.n = ov;
        T.mode = SEED_ARITH;
        T.ms = 5;
        T.K = arith_seed_count(ov, 5, true);
        T.C = kDetC;
        T.cut = I.dcut;
        T.max_iter = 8;
        T.use_d8 = 1;
        T.sd8 = 100.0;
        T.early_term = 1.0;
        T.out = c.recs + (size_t)s * kRec;
        on = on && S.flag && ov >= 3;
        if (on && c.wcount && c.wcount[p] >= 0) {  // ranked: the selected offsets only
            const int *l = c.wlist + (size_t)p * kMaxTopK;
            bool sel = false;
            for (int j = 0; j < c.wcount[p]; j++) sel = sel || l[j] == aux;
            on = sel;
        }
        if (!on) T.out[0] = kNegInf;
        break;
    }
    case BK_TOPK:  // top-50% distance seed bank (indialign.cpp:162-176)
        T.table = b.topk_seed + p;
        T.K = 1;
        T.out_rec = REC_STAGE;
        on = on && S.topk_ok;
        S.flag = on;
        break;
    }
    T.n_items = on ? T.K * T.C : 0;
    const Tune &tn = c.tune.of(I.N);  // the shape of the pair's length bucket
    T.chunk = tn.bank_chunk;
    T.cutoff_major = tn.bank_cutoff_major;
    c.btasks[s] = T;
    c.counts[s] = (T.n_items + T.chunk - 1) / T.chunk;
}

// ---- chain plans ------------------------------------------------------------
__global__ void k_plan_chain(DevBatch b, PlanCtx c) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= c.ntasks) return;
    const int p = c.pair ? c.pair[s] : s;
    const PairInfo &I = b.info[p];
    PairState &S = b.state[p];
    ChainTask T;
    T.pair = p;
    T.start = START_RT;
    T.dense = 0;
    T.n_starts = 1;
    T.gaps = 2;
    T.max_iter = 1;
    T.smode = SMAT_DP;
    T.gap0 = -0.6;
    T.gap1 = 0.0;
    T.sd8 = I.sd8;
    T.rt = S.rec[REC_START];
    T.res = c.base ? c.chain_res + (size_t)c.base[s] * kRec : nullptr;
    T.na_out = nullptr;
    T.live = nullptr;
    T.wlist = nullptr;
    T.alP = T.alQ = nullptr;
    T.al_cap = I.N;
    bool on = I.status == 0;
    switch (c.kind) {
    case CH_SS2:  // ss_nw_align: label identity, gap -1 (ss.h:56-83)
    case CH_SS4:  // distance + label bonus under START, gap -1 (ss.h:108-136)
        T.smode = c.kind == CH_SS2 ? SMAT_SS2 : SMAT_SS4;
        T.gaps = 1;
        T.gap0 = T.gap1 = -1.0;
        T.na_out = S.na;
        T.alP = c.alP + 3 * (2 * (size_t)I.off);
        T.alQ = c.alQ + 3 * (2 * (size_t)I.off);
        T.res = nullptr;
        on = on && I.plen >= 3 && I.nlen >= 3;
        S.flag = on;
        if (!on) S.na[0] = 0;
        break;
    case CH_DP_EMIT:  // one dp_refine iteration's NW for both gaps
        T.n_starts = 2;
        T.gaps = 1;
        T.rt = S.rec[REC_CUR0];
        T.res = S.rec[REC_NEW0];
        T.na_out = S.na;
        T.live = S.active;
        T.alP = c.alP + 3 * (2 * (size_t)I.off);
        T.alQ = c.alQ + 3 * (2 * (size_t)I.off);
        on = on && (S.active[0] || S.active[1]);
        if (!S.active[0]) S.na[0] = 0;
        if (!S.active[1]) S.na[1] = 0;
        break;
    case CH_LOCAL:  // rescue windows, dp_refine(2, lite, sd8=100) (rescue.h:82-96)
        T.start = START_WINDOW;
        T.dense = c.iters;  // 0 normal, 1 dense
        T.n_starts = window_count(I.plen, I.nlen, T.dense);
        if (c.wcount && c.wcount[p] >= 0) {  // ranked: the selected windows only
            T.n_starts = c.wcount[p];
            T.wlist = c.wlist + (size_t)p * kMaxTopK;
        }
        T.max_iter = 2;
        T.sd8 = 100.0;
        on = on && S.flag;
        break;
    case CH_THREAD:  // dp_refine(1, lite, sd8=100) from each offset's det
        T.rt = c.recs + (size_t)c.aux[s] * kRec;
        T.n_starts = thread_count(I.plen, I.nlen);
        T.max_iter = 1;
        T.sd8 = 100.0;
        on = on && S.flag;
        break;
    case CH_SINGLE:  // idp / extra dp_refine from START (indialign.cpp:201-221)
        T.max_iter = c.iters;
        on = on && S.flag;
        break;
    case CH_OFFDP:  // dp_refine(dp_iter, lite) per offset start (:229-256)
        T.rt = c.recs + (size_t)c.aux[s] * kRec;
        T.n_starts = offdp_count(I.N);
        T.max_iter = c.iters;
        on = on && c.iters > 0;
        break;
    }
    T.n_chains = on ? T.n_starts * T.gaps : 0;
    // a gated-on stage with no chains still yields the reference's initial
    // -1e30 / identity result, which the caller then rescores
    if (on && T.n_chains == 0 && (c.kind == CH_LOCAL || c.kind == CH_THREAD || c.kind == CH_SINGLE))
        rec_ident(S.rec[REC_STAGE], kScoreInit);
    T.chunk = c.tune.of(I.N).chain_chunk;  // the shape of the pair's length bucket
    c.ctasks[s] = T;
    c.counts[s] = (T.n_chains + T.chunk - 1) / T.chunk;
}

// ---- chain reductions (warp per pair) ---------------------------------------
// A dp_refine's best over both gap chains: each chain starts from score 0 /
// identity and replaces on strictly greater, gap -0.6 first
// (indialign_c/align.h:131-145), so the later chain wins only if strictly
// better.
IA_DEV const double *combine2(const double *g0, const double *g1) {
    return g1[0] > g0[0] ? g1 : g0;
}

__global__ void k_reduce_chain(DevBatch b, PlanCtx c) {
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (s >= c.ntasks) return;
    const ChainTask &T = c.ctasks[s];
    if (T.n_chains <= 0) return;
    PairState &S = b.state[T.pair];
    double *out = c.kind == CH_OFFDP ? nullptr : S.rec[REC_STAGE];
    if (c.kind == CH_OFFDP) {
        // each offset's dp result into its own record, in offset order
        for (int si = lane; si < T.n_starts; si += 32) {
            double *o = c.recs2 + ((size_t)c.aux[s] + si) * kRec;
            const double *st = T.rt + (size_t)si * kRec;
            if (st[0] <= -1e299) { o[0] = kNegInf; continue; }
            rec_copy(o, combine2(T.res + (size_t)(2 * si) * kRec, T.res + (size_t)(2 * si + 1) * kRec));
        }
        return;
    }
    // first max over starts (initial -1e30 / identity, strict >)
    double bs = kScoreInit;
    int bi = -1, bsrc = 0;  // bsrc: 0 chain result, 1 the offset's det record
    for (int si = lane; si < T.n_starts; si += 32) {
        const double *r = combine2(T.res + (size_t)(2 * si) * kRec, T.res + (size_t)(2 * si + 1) * kRec);
        double sc = r[0];
        int src = 0;
        if (c.kind == CH_THREAD) {
            // cand = dp if dp > det else det, score max (rescue.h:163-168)
            const double *det = T.rt + (size_t)si * kRec;
            if (det[0] <= -1e299) continue;  // offset skipped (overlap < 3)
            if (!(sc > det[0])) { sc = det[0]; src = 1; }
        }
        if (sc > bs) { bs = sc; bi = si; bsrc = src; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double s2 = __shfl_xor_sync(0xffffffffu, bs, o);
        int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        int r2 = __shfl_xor_sync(0xffffffffu, bsrc, o);
        bool take = (s2 > bs) || (s2 == bs && i2 >= 0 && (bi < 0 || i2 < bi));
        if (take) { bs = s2; bi = i2; bsrc = r2; }
    }
    if (lane == 0) {
        if (bi < 0) {
            rec_ident(out, kScoreInit);
        } else if (bsrc == 1) {
            rec_copy(out, T.rt + (size_t)bi * kRec);
        } else {
            rec_copy(out, combine2(T.res + (size_t)(2 * bi) * kRec, T.res + (size_t)(2 * bi + 1) * kRec));
            out[0] = bs;
        }
    }
}

// ---- per-pair glue ------------------------------------------------------------
__global__ void k_glue(DevBatch b, GlueArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= b.n) return;
    const PairInfo &I = b.info[p];
    PairState &S = b.state[p];
    if (I.status != 0) return;
    double *best = S.rec[REC_BEST];
    switch (a.op) {
    case G_GATE:  // rescue trigger on the running best (indialign.cpp:129,137,145)
        S.flag = best[0] < a.thr;
        break;
    case G_STAGE_UPDATE:  // if stage ran and beats best: take it
        if (S.flag && S.rec[REC_STAGE][0] > best[0]) rec_copy(best, S.rec[REC_STAGE]);
        break;
    case G_SS_BEGIN:  // evaluate_ss_seeds: best = -1e30 / identity (ss.h:93-95)
        rec_ident(S.rec[REC_SS], kScoreInit);
        break;
    case G_SS_DET:  // det after an SS alignment, then arm dp_refine (ss.h:96-105)
        S.dp_on = 0;
        if (S.flag && S.na[0] >= 3) {
            if (S.rec[REC_DET0][0] > S.rec[REC_SS][0]) rec_copy(S.rec[REC_SS], S.rec[REC_DET0]);
            if (a.dp_iter > 0) {
                rec_copy(S.rec[REC_CUR0], S.rec[REC_SS]);
                rec_copy(S.rec[REC_CUR1], S.rec[REC_SS]);
                rec_ident(S.rec[REC_DPB0], 0.0);
                rec_ident(S.rec[REC_DPB1], 0.0);
                S.active[0] = S.active[1] = 1;
                S.dp_on = 1;
            }
        }
        break;
    case G_DP_STEP:  // one dp_refine iteration per gap chain (align.h:155-211)
        for (int g = 0; g < 2; g++) {
            if (!S.active[g]) continue;
            if (S.na[g] < 3) { S.active[g] = 0; continue; }
            const double *it = S.rec[REC_DET0 + g][0] > S.rec[REC_NEW0 + g][0] ? S.rec[REC_DET0 + g]
                                                                               : S.rec[REC_NEW0 + g];
            rec_copy(S.rec[REC_CUR0 + g], it);
            if (it[0] > S.rec[REC_DPB0 + g][0]) rec_copy(S.rec[REC_DPB0 + g], it);
        }
        break;
    case G_DP_END:  // dp result = later gap chain only if strictly better
        S.active[0] = S.active[1] = 0;
        if (S.dp_on) rec_copy(S.rec[REC_DP], combine2(S.rec[REC_DPB0], S.rec[REC_DPB1]));
        break;
    case G_SS_DP:  // if (dp.score > best.score) best = dp (ss.h:101-104)
        if (S.dp_on && S.rec[REC_DP][0] > S.rec[REC_SS][0]) rec_copy(S.rec[REC_SS], S.rec[REC_DP]);
        S.dp_on = 0;
        break;
    case G_SS4_START:  // IA4 transform: SS best if any, else the seed-bank best
        rec_copy(S.rec[REC_START], S.rec[REC_SS][0] > -1e20 ? S.rec[REC_SS] : best);
        break;
    case G_SS_FINISH:  // rescored SS result vs best (indialign.cpp:114-115)
        if (S.rec[REC_SS][0] > best[0]) rec_copy(best, S.rec[REC_SS]);
        break;
    case G_DPF_BEGIN:  // final dp_refine from best (indialign.cpp:190-193)
        S.seed_score = best[0];
        S.dp_on = 0;
        if (a.dp_iter > 0) {
            rec_copy(S.rec[REC_CUR0], best);
            rec_copy(S.rec[REC_CUR1], best);
            rec_ident(S.rec[REC_DPB0], 0.0);
            rec_ident(S.rec[REC_DPB1], 0.0);
            S.active[0] = S.active[1] = 1;
            S.dp_on = 1;
        }
        break;
    case G_DPF_UPDATE:  // rescored dp vs best; then best itself rescored (:194-199)
        if (S.dp_on) {
            S.dp_id = S.rec[REC_DP][0];
            if (S.rec[REC_DP][0] > best[0]) rec_copy(best, S.rec[REC_DP]);
        }
        rec_copy(S.rec[REC_TMP], best);
        break;
    case G_TMP_UPDATE:
        if (S.rec[REC_TMP][0] > best[0]) rec_copy(best, S.rec[REC_TMP]);
        break;
    case G_IDP_START:  // identity-start dp_refine when masks differ (:201-208)
        rec_ident(S.rec[REC_START], 0.0);
        S.flag = a.dp_iter > 0 && I.has_cross;
        break;
    case G_EXTRA_START: {  // extra lite dp_refine for weak pairs (:210-221)
        const int extra = a.dp_iter < 5 ? 5 - a.dp_iter : 0;
        S.flag = a.dp_iter > 0 && I.has_cross && extra > 0 && best[0] < 0.36;
        rec_copy(S.rec[REC_START], S.seed_score > S.dp_id ? best : S.rec[REC_DP]);
        break;
    }
    case G_FLAG_ON:
        S.flag = 1;
        break;
    case G_OFFDP_UPDATE: {  // sequential update_best over offsets (:248-253)
        const int n = offdp_count(I.N);
        const double *r = a.recs + (size_t)a.idx[p] * kRec;
        for (int o = 0; o < n; o++)
            if (r[(size_t)o * kRec] > best[0]) rec_copy(best, r + (size_t)o * kRec);
        break;
    }
    }
}

// ---- launch wrappers ------------------------------------------------------
void launch_plan_bank(const DevBatch &b, const PlanCtx &c, cudaStream_t st) {
    if (c.ntasks > 0) k_plan_bank<<<(c.ntasks + 127) / 128, 128, 0, st>>>(b, c);
}
void launch_plan_chain(const DevBatch &b, const PlanCtx &c, cudaStream_t st) {
    if (c.ntasks > 0) k_plan_chain<<<(c.ntasks + 127) / 128, 128, 0, st>>>(b, c);
}
void launch_reduce_chain(const DevBatch &b, const PlanCtx &c, cudaStream_t st) {
    if (c.ntasks > 0) k_reduce_chain<<<(c.ntasks * 32 + 255) / 256, 256, 0, st>>>(b, c);
}
void launch_glue(const DevBatch &b, const GlueArgs &a, cudaStream_t st) {
    if (b.n > 0) k_glue<<<(b.n + 127) / 128, 128, 0, st>>>(b, a);
}

}  // namespace ia
