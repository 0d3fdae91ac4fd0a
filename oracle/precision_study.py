"""Precision study of the search (design evidence; test infrastructure only).

Rebuilds the C oracle (indialign_oracle.c) with its arithmetic lowered to
FP32 in several ways, and once with its eigen-solve replaced; runs each
variant's batch search beside the reference build (_ref/libindialign_ref.so),
rescores every variant's final (R, t) in FP64 with the reference's own
tm_score_no_d8 (_ref/libindialign_ref_stages.so) and prints the per-pair
change of the final TM-score against the reference:

  dist32      FP32 distances and inlier tests, FP64 moments and sums
  kahan32     FP32 distances, TM terms, score-matrix entries and centred
              covariances with Kahan sums; FP64 eigen-solve
  plain32     the same with plain FP32 sums
  raw32       plain FP32 one-pass raw moments about the origin
  raw32c      the same about the mean of each point set
  bank32      only the seed banks (evaluate_seed_bank, the detailed searches'
              banks, gapless threading) lowered, in the GPU seed-bank
              kernel's form: point sets centred on their FP64 mean and
              converted to FP32, FP32 distances / inlier tests / raw moments,
              FP32 item scores with a compensated sum, FP64 eigen-solves, the
              winner rescored in FP64; everything else FP64
  bank32f     bank32 in the seed-bank kernel's explicit FP32 operation
              sequence (fused transform, d2 and moment products; the item
              score's term 1 / fma(d2, 1/d0^2, 1))
  bank32p     bank32f with the cutoff passes' moments summed in two FP32
              partial sets (even / odd residues) combined in FP64: the
              rounding of an accumulate by paired FP32 instructions (an
              estimate for a possible kernel change, not the kernel's form)
  smat32      only the score-matrix entries of dp_refine and of the SS +
              distance NW lowered, in the NW-chain kernel's form: the moved
              pred point rounded to FP32, FP32 difference, d2, cutoff test and
              term 1/(1 + d2 * (1/d0^2)), widened to FP64 for the DP
  dp32        smat32 plus the NW fill's values (H, diagonal and gap moves)
              in FP32
  qcp64       all FP64, every Kabsch eigen-solve by the characteristic
              polynomial of Horn's key matrix (Newton for its top roots,
              eigenvector from an adjugate column) instead of Jacobi sweeps,
              Jacobi kept where the top two eigenvalues lie within 1e-4 of
              the spectrum's scale; prints the fallback rate

Variant sources and libraries go to oracle/_variants/.  The variants are
compiled without -ffast-math (it would fold the Kahan compensation away).

    python oracle/precision_study.py --pairs 400 --seed 21 --hard 160 --hard-seed 22

takes ~30 min on 8 host cores; every textual substitution is checked, so a
changed oracle source fails loudly instead of measuring the wrong thing.
"""
from __future__ import annotations

import argparse
import ctypes
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

from indialign_b200 import abi, workloads as W  # noqa: E402

OUT = os.path.join(HERE, "_variants")
REF_SO = os.path.join(HERE, "_ref", "libindialign_ref.so")
STAGES_SO = os.path.join(HERE, "_ref", "libindialign_ref_stages.so")


def _sub(s: str, old: str, new: str) -> str:
    if s.count(old) != 1:
        raise SystemExit(f"substitution does not apply (found {s.count(old)}x): {old[:60]!r}")
    return s.replace(old, new)


DIST64 = '''static inline double dist2_at(const double *p, const double *q, const double *R,
                              const double *t) {
    double mx = p[0] * R[0] + p[1] * R[3] + p[2] * R[6] + t[0];
    double my = p[0] * R[1] + p[1] * R[4] + p[2] * R[7] + t[1];
    double mz = p[0] * R[2] + p[1] * R[5] + p[2] * R[8] + t[2];
    double dx = mx - q[0], dy = my - q[1], dz = mz - q[2];
    return dx * dx + dy * dy + dz * dz;
}'''
DIST32 = '''static inline double dist2_at(const double *p, const double *q, const double *R,
                              const double *t) {
    float px = (float)p[0], py = (float)p[1], pz = (float)p[2];
    float mx = px * (float)R[0] + py * (float)R[3] + pz * (float)R[6] + (float)t[0];
    float my = px * (float)R[1] + py * (float)R[4] + pz * (float)R[7] + (float)t[1];
    float mz = px * (float)R[2] + py * (float)R[5] + pz * (float)R[8] + (float)t[2];
    float dx = mx - (float)q[0], dy = my - (float)q[1], dz = mz - (float)q[2];
    return (double)(dx * dx + dy * dy + dz * dz);
}
static inline float tmterm(double d2, double d0sq) { return 1.0f / (1.0f + (float)d2 / (float)d0sq); }'''
IMIN = 'static int imin(int a, int b) { return a < b ? a : b; }\n'
KAHAN = '''typedef struct { float s, c; } kahan;
static inline void kadd(kahan *k, float x) { float y = x - k->c; float t = k->s + y; k->c = (t - k->s) - y; k->s = t; }
'''
PLAIN = '''typedef struct { float s, c; } kahan;
static inline void kadd(kahan *k, float x) { k->s += x; }
'''

KABSCH64 = '''    double w = 0, cP[3] = {0, 0, 0}, cQ[3] = {0, 0, 0}, H[3][3];
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
    cov_to_rotation((const double(*)[3])H, R);'''
KABSCH_CENTRED32 = '''    double w = 0, cP[3] = {0, 0, 0}, cQ[3] = {0, 0, 0}, H[3][3];
    kahan kP[3] = {{0, 0}}, kQ[3] = {{0, 0}}, kH[9] = {{0, 0}};
    float fP[3], fQ[3];
    for (int i = 0; i < N; i++) {
        if (!mask[i]) continue;
        for (int d = 0; d < 3; d++) { kadd(&kP[d], (float)P[i * 3 + d]); kadd(&kQ[d], (float)Q[i * 3 + d]); }
        w += 1.0;
    }
    if (w < 3.0) {
        memcpy(R, IDENT, sizeof IDENT);
        t[0] = t[1] = t[2] = 0;
        return;
    }
    for (int d = 0; d < 3; d++) { fP[d] = kP[d].s / (float)w; fQ[d] = kQ[d].s / (float)w; cP[d] = fP[d]; cQ[d] = fQ[d]; }
    for (int i = 0; i < N; i++) {
        float dp[3], dq[3];
        if (!mask[i]) continue;
        for (int d = 0; d < 3; d++) { dp[d] = (float)P[i * 3 + d] - fP[d]; dq[d] = (float)Q[i * 3 + d] - fQ[d]; }
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) kadd(&kH[r * 3 + c], dp[r] * dq[c]);
    }
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) H[r][c] = kH[r * 3 + c].s;
    cov_to_rotation((const double(*)[3])H, R);'''
KABSCH_RAW32 = '''    double oP[3] = {0, 0, 0}, oQ[3] = {0, 0, 0}, cP[3], cQ[3], H[3][3], w = 0;
    kahan sp[3] = {{0, 0}}, sq[3] = {{0, 0}}, h[9] = {{0, 0}};
    if (OFFSET_MEAN && N > 0) {
        for (int i = 0; i < N; i++)
            for (int d = 0; d < 3; d++) { oP[d] += P[i * 3 + d]; oQ[d] += Q[i * 3 + d]; }
        for (int d = 0; d < 3; d++) { oP[d] /= N; oQ[d] /= N; }
    }
    for (int i = 0; i < N; i++) {
        float p[3], q[3];
        if (!mask[i]) continue;
        for (int d = 0; d < 3; d++) { p[d] = (float)(P[i * 3 + d] - oP[d]); q[d] = (float)(Q[i * 3 + d] - oQ[d]); }
        for (int d = 0; d < 3; d++) { kadd(&sp[d], p[d]); kadd(&sq[d], q[d]); }
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) kadd(&h[r * 3 + c], p[r] * q[c]);
        w += 1.0;
    }
    if (w < 3.0) {
        memcpy(R, IDENT, sizeof IDENT);
        t[0] = t[1] = t[2] = 0;
        return;
    }
    for (int d = 0; d < 3; d++) { cP[d] = sp[d].s / w; cQ[d] = sq[d].s / w; }
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) H[r][c] = h[r * 3 + c].s - w * cP[r] * cQ[c];
    cov_to_rotation((const double(*)[3])H, R);
    for (int d = 0; d < 3; d++) { cP[d] += oP[d]; cQ[d] += oQ[d]; }'''


def _fp32_sums(s: str) -> str:
    """TM sums, weights and score-matrix entries in FP32 (needs kahan/kadd)."""
    s = _sub(s, '''    double d0sq = dmax(d0 * d0, 1e-12), sd8sq = sd8 * sd8, sum = 0;
    for (int i = 0; i < N; i++) {
        double d2;
        if (!v[i]) continue;
        d2 = dist2_at(p + 3 * i, q + 3 * i, R, t);
        if (!use_d8 || d2 <= sd8sq) sum += 1.0 / (1.0 + d2 / d0sq);
    }
    return sum / dmax(Lnorm, 1.0);''', '''    double d0sq = dmax(d0 * d0, 1e-12), sd8sq = sd8 * sd8;
    kahan sum = {0, 0};
    for (int i = 0; i < N; i++) {
        double d2;
        if (!v[i]) continue;
        d2 = dist2_at(p + 3 * i, q + 3 * i, R, t);
        if (!use_d8 || d2 <= (double)(float)sd8sq) kadd(&sum, tmterm(d2, d0sq));
    }
    return (double)sum.s / dmax(Lnorm, 1.0);''')
    s = _sub(s, '''            w[i] = v[i] ? 1.0 / (1.0 + dist2_at(p + 3 * i, q + 3 * i, R, t) / d0sq) : 0.0;''',
             '''            w[i] = v[i] ? (double)tmterm(dist2_at(p + 3 * i, q + 3 * i, R, t), d0sq) : 0.0;''')
    s = _sub(s, '''                    double dx = m[0] - n[0], dy = m[1] - n[1], dz = m[2] - n[2];
                    double d2 = dx * dx + dy * dy + dz * dz;
                    smat[(size_t)a * nlen + b] = d2 <= sd8sq ? 1.0 / (1.0 + d2 / d0sq_dp) : 0.0;''',
             '''                    float dx = (float)m[0] - (float)n[0], dy = (float)m[1] - (float)n[1],
                          dz = (float)m[2] - (float)n[2];
                    float d2 = dx * dx + dy * dy + dz * dz;
                    smat[(size_t)a * nlen + b] = d2 <= (float)sd8sq ? (double)tmterm(d2, d0sq_dp) : 0.0;''')
    s = _sub(s, '''            for (int i = 0; i < na; i++)
                sc += 1.0 / (1.0 + dist2_at(Pa + 3 * i, Qa + 3 * i, nR, nt) / d0sq_s);
            sc /= dmax(Lnorm, 1.0);''', '''            {
                kahan ks = {0, 0};
                for (int i = 0; i < na; i++) kadd(&ks, tmterm(dist2_at(Pa + 3 * i, Qa + 3 * i, nR, nt), d0sq_s));
                sc = (double)ks.s / dmax(Lnorm, 1.0);
            }''')
    s = _sub(s, '''                    moved[i * 3 + d] = pred[i * 3] * cR[d] + pred[i * 3 + 1] * cR[3 + d] +
                                       pred[i * 3 + 2] * cR[6 + d] + ct[d];''',
             '''                    moved[i * 3 + d] = (float)pred[i * 3] * (float)cR[d] + (float)pred[i * 3 + 1] * (float)cR[3 + d] +
                                       (float)pred[i * 3 + 2] * (float)cR[6 + d] + (float)ct[d];''')
    s = _sub(s, '''                double dx = m[0] - n[0], dy = m[1] - n[1], dz = m[2] - n[2];
                double sc = 1.0 / (1.0 + (dx * dx + dy * dy + dz * dz) / d01sq);''',
             '''                float dx = (float)m[0] - (float)n[0], dy = (float)m[1] - (float)n[1], dz = (float)m[2] - (float)n[2];
                double sc = (double)tmterm(dx * dx + dy * dy + dz * dz, d01sq);''')
    return s


BANK32_HELPERS = r"""
/* ---- bank32: the GPU seed bank's arithmetic ---- */
static void mean3(const double *X, int N, double *o) {
    o[0] = o[1] = o[2] = 0;
    for (int i = 0; i < N; i++)
        for (int d = 0; d < 3; d++) o[d] += X[3 * i + d];
    for (int d = 0; d < 3; d++) o[d] = N > 0 ? o[d] / N : 0.0;
}
static float *centred32(const double *X, int N, const double *o) {
    float *f = (float *)malloc(sizeof(float) * 3 * (size_t)(N > 0 ? N : 1));
    for (int i = 0; i < N; i++)
        for (int d = 0; d < 3; d++) f[3 * i + d] = (float)(X[3 * i + d] - o[d]);
    return f;
}
typedef struct { float sp[3], sq[3], h[9]; int w; } mom32;
static void m32_add(mom32 *m, const float *p, const float *q) {
    for (int d = 0; d < 3; d++) { m->sp[d] += p[d]; m->sq[d] += q[d]; }
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) m->h[3 * r + c] += p[r] * q[c];
    m->w++;
}
static void m32_kabsch(const mom32 *m, double *R, double *t) {
    double cP[3], cQ[3], H[3][3];
    if (m->w < 3) { memcpy(R, IDENT, sizeof IDENT); t[0] = t[1] = t[2] = 0; return; }
    for (int d = 0; d < 3; d++) { cP[d] = m->sp[d] / (double)m->w; cQ[d] = m->sq[d] / (double)m->w; }
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) H[r][c] = m->h[3 * r + c] - m->sp[r] * cQ[c];
    cov_to_rotation((const double(*)[3])H, R);
    for (int d = 0; d < 3; d++) t[d] = cQ[d] - (cP[0] * R[d] + cP[1] * R[3 + d] + cP[2] * R[6 + d]);
}
static float d2_32(const float *p, const float *q, const float *Rf, const float *tf) {
    float dx = p[0] * Rf[0] + p[1] * Rf[3] + p[2] * Rf[6] + tf[0] - q[0];
    float dy = p[0] * Rf[1] + p[1] * Rf[4] + p[2] * Rf[7] + tf[1] - q[1];
    float dz = p[0] * Rf[2] + p[1] * Rf[5] + p[2] * Rf[8] + tf[2] - q[2];
    return dx * dx + dy * dy + dz * dz;
}
static void rt32(const double *R, const double *t, float *Rf, float *tf) {
    for (int a = 0; a < 9; a++) Rf[a] = (float)R[a];
    for (int a = 0; a < 3; a++) tf[a] = (float)t[a];
}
static void refine32(const float *P, const float *Q, const uint8_t *v, int N, float cut2, int max_iter,
                     double *R, double *t) {
    int prev = -1;
    for (int it = 0; it < max_iter; it++) {
        float Rf[9], tf[3];
        mom32 m;
        int c = 0;
        memset(&m, 0, sizeof m);
        rt32(R, t, Rf, tf);
        for (int i = 0; i < N; i++) {
            if (!v[i]) continue;
            if (d2_32(P + 3 * i, Q + 3 * i, Rf, tf) <= cut2) { m32_add(&m, P + 3 * i, Q + 3 * i); c++; }
        }
        if (c >= 3) m32_kabsch(&m, R, t);
        if (c == prev) break;
        prev = c;
    }
}
static double score32(const float *P, const float *Q, const uint8_t *v, int N, const double *R, const double *t,
                      double d0, double sd8, double Lnorm, int use_d8) {
    float Rf[9], tf[3], d0sq = (float)dmax(d0 * d0, 1e-12), sd8sq = (float)(sd8 * sd8), sum = 0.f, comp = 0.f;
    rt32(R, t, Rf, tf);
    for (int i = 0; i < N; i++) {
        float d2;
        if (!v[i]) continue;
        d2 = d2_32(P + 3 * i, Q + 3 * i, Rf, tf);
        if (!use_d8 || d2 <= sd8sq) {
            float y = 1.0f / (1.0f + d2 / d0sq) - comp, s2 = sum + y;
            comp = (s2 - sum) - y;
            sum = s2;
        }
    }
    return (double)sum / dmax(Lnorm, 1.0);
}
static void to_caller(const double *oP, const double *oQ, const double *R, double *t) {
    for (int d = 0; d < 3; d++) t[d] += oQ[d] - (oP[0] * R[d] + oP[1] * R[3 + d] + oP[2] * R[6 + d]);
}
"""

BANK32_SEED_BANK = r"""static OraSeed seed_bank(const double *p, const double *q, const uint8_t *valid,
                         const uint8_t *seeds, int K, const double *cands,
                         int C, double d0, double sd8, double Lnorm, int N,
                         int max_iter, int use_d8, double early_term) {
    OraSeed best;
    double R[9], t[3], oP[3], oQ[3];
    float *Pf, *Qf;
    memset(&best, 0, sizeof best);
    best.score = -1e30;
    mean3(p, N, oP); mean3(q, N, oQ);
    Pf = centred32(p, N, oP); Qf = centred32(q, N, oQ);
    for (int k = 0; k < K; k++) {
        if (best.score >= early_term) break;
        for (int c = 0; c < C; c++) {
            mom32 m;
            double sc;
            memset(&m, 0, sizeof m);
            for (int i = 0; i < N; i++)
                if (seeds[(size_t)k * N + i] & valid[i]) m32_add(&m, Pf + 3 * i, Qf + 3 * i);
            m32_kabsch(&m, R, t);
            refine32(Pf, Qf, valid, N, (float)(cands[c] * cands[c]), max_iter, R, t);
            sc = score32(Pf, Qf, valid, N, R, t, d0, sd8, Lnorm, use_d8);
            if (sc > best.score) {
                best.score = sc;
                memcpy(best.R, R, 72);
                memcpy(best.t, t, 24);
            }
        }
    }
    if (best.score > -1e30) {
        to_caller(oP, oQ, best.R, best.t);
        best.score = ora_tm_score(p, q, valid, best.R, best.t, d0, Lnorm, sd8, N, use_d8);
    }
    free(Pf); free(Qf);
    return best;
}

"""

BANK32_GAPLESS_OLD = r"""    for (int k = -kr; k <= kr; k += stride) {
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
    }"""
BANK32_GAPLESS_NEW = r"""    {
        double oP[3], oQ[3];
        float *Pf, *Qf;
        mean3(p, N, oP); mean3(q, N, oQ);
        Pf = centred32(p, N, oP); Qf = centred32(q, N, oQ);
        for (int k = -kr; k <= kr; k += stride) {
            mom32 m;
            double R[9], t[3], sc;
            if (k == 0) continue;
            memset(&m, 0, sizeof m);
            for (int i = 0; i < N; i++) {
                int j = i - k;
                if (j < 0 || j >= N || !pv[i] || !nv[j]) continue;
                m32_add(&m, Pf + 3 * i, Qf + 3 * j);
            }
            if (m.w < min_ali) continue;
            m32_kabsch(&m, R, t);
            refine32(Pf, Qf, v, N, (float)(d0s * d0s), 5, R, t);
            sc = score32(Pf, Qf, v, N, R, t, d0, 0.0, Lnorm, 0);
            if (sc > best.score) {
                best.score = sc;
                memcpy(best.R, R, 72); memcpy(best.t, t, 24);
            }
        }
        if (best.score > -1e30) {
            to_caller(oP, oQ, best.R, best.t);
            best.score = ora_tm_score(p, q, v, best.R, best.t, d0, Lnorm, 0, N, 0);
        }
        free(Pf); free(Qf);
    }"""


QCP64 = r"""
/* ---- qcp64: the dominant eigenvector of Horn's key matrix F from its
 * characteristic polynomial (Theobald 2005, "Rapid calculation of RMSDs using
 * a quaternion-based characteristic polynomial"): P(x) = x^4 - tr(F^2)/2 x^2
 * - tr(F^3)/3 x + det F (F is traceless), its largest root by Newton from the
 * upper bound sqrt(tr(F^2)), the second root the same way on P(x)/(x - l1),
 * the eigenvector from the largest column of adj(F - l1 I).  When
 * l1 - l2 < 1e-4 sqrt(tr(F^2)) the reference's Jacobi sequence runs instead. */
long qcp_calls = 0, qcp_fallbacks = 0;
static double qdet3(double a, double b, double c, double d, double e, double f, double g, double h, double i) {
    return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
}
static double qminor(const double A[4][4], int row, int col) {
    double m[9];
    int k = 0;
    for (int i = 0; i < 4; i++) {
        if (i == row) continue;
        for (int j = 0; j < 4; j++)
            if (j != col) m[k++] = A[i][j];
    }
    return qdet3(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]);
}
static double qcp_newton_top(double b3, double b2, double b1, double b0, double x, double scale) {
    /* largest root of x^4 + b3 x^3 + b2 x^2 + b1 x + b0 (b3 = 0) or of the
     * cubic x^3 + b2 x^2 + b1 x + b0 (b3 < 0 marks the cubic), from above */
    for (int it = 0; it < 200; it++) {
        double g, dg, nx;
        if (b3 >= 0) { g = ((x * x + b2) * x + b1) * x + b0; dg = (4 * x * x + 2 * b2) * x + b1; }
        else { g = ((x + b2) * x + b1) * x + b0; dg = (3 * x + 2 * b2) * x + b1; }
        if (!(dg > 0)) break;
        nx = x - g / dg;
        if (!(nx < x)) break;
        if (x - nx <= 1e-16 * scale) return nx;
        x = nx;
    }
    return x;
}
static int qcp_rotation(const double F[4][4], double *R) {
    double F2[4][4], p2 = 0, p3 = 0, dt, c2, c1, scale, l1, l2, A[4][4], q[4] = {1, 0, 0, 0}, best = -1, qn;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            double s = 0;
            for (int k = 0; k < 4; k++) s += F[i][k] * F[k][j];
            F2[i][j] = s;
        }
    for (int i = 0; i < 4; i++) {
        p2 += F2[i][i];
        for (int k = 0; k < 4; k++) p3 += F2[i][k] * F[k][i];
    }
    dt = 0;
    for (int j = 0; j < 4; j++) dt += ((j & 1) ? -1.0 : 1.0) * F[0][j] * qminor(F, 0, j);
    c2 = -0.5 * p2; c1 = -p3 / 3.0; scale = sqrt(p2);
    if (!(scale > 0)) return 1;
    l1 = qcp_newton_top(0.0, c2, c1, dt, scale, scale);
    l2 = qcp_newton_top(-1.0, l1, c2 + l1 * l1, c1 + l1 * c2 + l1 * l1 * l1, l1, scale);
    if (l1 - l2 < 1e-4 * scale) return 1;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) A[i][j] = F[i][j] - (i == j ? l1 : 0.0);
    for (int c = 0; c < 4; c++) {
        double v[4], n;
        for (int r = 0; r < 4; r++) v[r] = (((r + c) & 1) ? -1.0 : 1.0) * qminor(A, c, r);
        n = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3];
        if (n > best) { best = n; memcpy(q, v, sizeof q); }
    }
    if (!(best > 0)) return 1;
    qn = sqrt(best);
    for (int i = 0; i < 4; i++) q[i] /= qn;
    R[0] = q[0] * q[0] + q[1] * q[1] - q[2] * q[2] - q[3] * q[3];
    R[1] = 2 * (q[1] * q[2] + q[0] * q[3]);
    R[2] = 2 * (q[1] * q[3] - q[0] * q[2]);
    R[3] = 2 * (q[1] * q[2] - q[0] * q[3]);
    R[4] = q[0] * q[0] - q[1] * q[1] + q[2] * q[2] - q[3] * q[3];
    R[5] = 2 * (q[2] * q[3] + q[0] * q[1]);
    R[6] = 2 * (q[1] * q[3] + q[0] * q[2]);
    R[7] = 2 * (q[2] * q[3] - q[0] * q[1]);
    R[8] = q[0] * q[0] - q[1] * q[1] - q[2] * q[2] + q[3] * q[3];
    return 0;
}
"""
QCP64_CALL_OLD = """    jacobi4(F, V);"""
QCP64_CALL_NEW = """    {
        int fb;
#pragma omp atomic
        qcp_calls++;
        fb = qcp_rotation((const double(*)[4])F, R);
        if (!fb) return;
#pragma omp atomic
        qcp_fallbacks++;
    }
    jacobi4(F, V);"""


def _qcp64(src: str) -> str:
    """The eigen-solve of every Kabsch by the characteristic polynomial."""
    marker = "/* Horn's quaternion matrix from the 3x3 covariance"
    s = _sub(src, marker, QCP64 + "\n" + marker)
    return _sub(s, QCP64_CALL_OLD, QCP64_CALL_NEW)


BANK32F_OLD_D2 = '''static float d2_32(const float *p, const float *q, const float *Rf, const float *tf) {
    float dx = p[0] * Rf[0] + p[1] * Rf[3] + p[2] * Rf[6] + tf[0] - q[0];
    float dy = p[0] * Rf[1] + p[1] * Rf[4] + p[2] * Rf[7] + tf[1] - q[1];
    float dz = p[0] * Rf[2] + p[1] * Rf[5] + p[2] * Rf[8] + tf[2] - q[2];
    return dx * dx + dy * dy + dz * dz;
}'''
BANK32F_NEW_D2 = '''static float d2_32(const float *p, const float *q, const float *Rf, const float *tf) {
    float dx = fmaf(p[0], Rf[0], fmaf(p[1], Rf[3], fmaf(p[2], Rf[6], tf[0] - q[0])));
    float dy = fmaf(p[0], Rf[1], fmaf(p[1], Rf[4], fmaf(p[2], Rf[7], tf[1] - q[1])));
    float dz = fmaf(p[0], Rf[2], fmaf(p[1], Rf[5], fmaf(p[2], Rf[8], tf[2] - q[2])));
    return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
}'''
BANK32F_OLD_ADD = '''        for (int c = 0; c < 3; c++) m->h[3 * r + c] += p[r] * q[c];'''
BANK32F_NEW_ADD = '''        for (int c = 0; c < 3; c++) m->h[3 * r + c] = fmaf(p[r], q[c], m->h[3 * r + c]);'''
BANK32F_OLD_SCORE = '''    float Rf[9], tf[3], d0sq = (float)dmax(d0 * d0, 1e-12), sd8sq = (float)(sd8 * sd8), sum = 0.f, comp = 0.f;'''
BANK32F_NEW_SCORE = '''    float Rf[9], tf[3], inv = (float)(1.0 / dmax(d0 * d0, 1e-12)), sd8sq = (float)(sd8 * sd8), sum = 0.f,
          comp = 0.f;'''
BANK32F_OLD_TERM = '''            float y = 1.0f / (1.0f + d2 / d0sq) - comp, s2 = sum + y;'''
BANK32F_NEW_TERM = '''            float y = 1.0f / fmaf(d2, inv, 1.0f) - comp, s2 = sum + y;'''


def _bank32f(src: str) -> str:
    """bank32 with the seed-bank kernel's explicit FP32 operation sequence:
    fused transform ((t - q) + p_z R + p_y R + p_x R), fused d2 and moment
    products, and the item score's term 1 / fma(d2, 1/d0^2, 1)."""
    s = _bank32(src)
    s = _sub(s, BANK32F_OLD_D2, BANK32F_NEW_D2)
    s = _sub(s, BANK32F_OLD_ADD, BANK32F_NEW_ADD)
    s = _sub(s, BANK32F_OLD_SCORE, BANK32F_NEW_SCORE)
    return _sub(s, BANK32F_OLD_TERM, BANK32F_NEW_TERM)


BANK32P_OLD_LOOP = '''        mom32 m;
        int c = 0;
        memset(&m, 0, sizeof m);
        rt32(R, t, Rf, tf);
        for (int i = 0; i < N; i++) {
            if (!v[i]) continue;
            if (d2_32(P + 3 * i, Q + 3 * i, Rf, tf) <= cut2) { m32_add(&m, P + 3 * i, Q + 3 * i); c++; }
        }
        if (c >= 3) m32_kabsch(&m, R, t);'''
BANK32P_NEW_LOOP = '''        mom32 m, mo;
        int c = 0;
        memset(&m, 0, sizeof m);
        memset(&mo, 0, sizeof mo);
        rt32(R, t, Rf, tf);
        for (int i = 0; i < N; i++) {
            if (!v[i]) continue;
            if (d2_32(P + 3 * i, Q + 3 * i, Rf, tf) <= cut2) {
                m32_add((i & 1) ? &mo : &m, P + 3 * i, Q + 3 * i);
                c++;
            }
        }
        if (c >= 3) m32_kabsch2(&m, &mo, R, t);'''
BANK32P_MARKER = "static float d2_32(const float *p, const float *q, const float *Rf, const float *tf) {"
BANK32P_KABSCH2 = r"""/* Kabsch from two FP32 partial moment sets (even and odd residues),
   combined in FP64 */
static void m32_kabsch2(const mom32 *a, const mom32 *b, double *R, double *t) {
    double sp[3], sq[3], cP[3], cQ[3], H[3][3], w = (double)(a->w + b->w);
    if (a->w + b->w < 3) { memcpy(R, IDENT, sizeof IDENT); t[0] = t[1] = t[2] = 0; return; }
    for (int d = 0; d < 3; d++) {
        sp[d] = (double)a->sp[d] + (double)b->sp[d];
        sq[d] = (double)a->sq[d] + (double)b->sq[d];
        cP[d] = sp[d] / w;
        cQ[d] = sq[d] / w;
    }
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) H[r][c] = ((double)a->h[3 * r + c] + (double)b->h[3 * r + c]) - sp[r] * cQ[c];
    cov_to_rotation((const double(*)[3])H, R);
    for (int d = 0; d < 3; d++) t[d] = cQ[d] - (cP[0] * R[d] + cP[1] * R[3 + d] + cP[2] * R[6 + d]);
}
"""


def _bank32p(src: str) -> str:
    """bank32f with the cutoff passes' moments accumulated in two FP32
    partial sets, even and odd residue indices, combined in FP64 before the
    eigen-solve: the rounding of a seed-bank accumulate that adds the two
    residues of a staged pair with paired FP32 instructions (an estimate for
    that kernel change; the kernel does not do this)."""
    s = _bank32f(src)
    s = _sub(s, BANK32P_MARKER, BANK32P_KABSCH2 + BANK32P_MARKER)
    return _sub(s, BANK32P_OLD_LOOP, BANK32P_NEW_LOOP)


def _bank32(src: str) -> str:
    """Only the seed banks lowered, in the GPU seed-bank kernel's form."""
    marker = "/* ---- seeds (indialign_c/seeds.h)"
    s = _sub(src, marker, BANK32_HELPERS + "\n" + marker)
    a, b = s.index("static OraSeed seed_bank("), s.index("void ora_seed_bank(")
    s = s[:a] + BANK32_SEED_BANK + s[b:]
    return _sub(s, BANK32_GAPLESS_OLD, BANK32_GAPLESS_NEW)


def _smat32(s: str) -> str:
    """Score-matrix entries (dp_refine and the SS+distance NW) in FP32, in the
    NW-chain kernel's form: the pred point moved in FP64 and rounded to FP32,
    FP32 difference / d2 / cutoff test, the term 1/(1 + d2 * (1/d0^2)) in
    FP32, widened to FP64 for the DP."""
    s = _sub(s, '''                    double dx = m[0] - n[0], dy = m[1] - n[1], dz = m[2] - n[2];
                    double d2 = dx * dx + dy * dy + dz * dz;
                    smat[(size_t)a * nlen + b] = d2 <= sd8sq ? 1.0 / (1.0 + d2 / d0sq_dp) : 0.0;''',
             '''                    float dx = (float)m[0] - (float)n[0], dy = (float)m[1] - (float)n[1],
                          dz = (float)m[2] - (float)n[2];
                    float d2 = dx * dx + dy * dy + dz * dz;
                    smat[(size_t)a * nlen + b] =
                        d2 <= (float)sd8sq ? (double)(1.0f / (1.0f + d2 * (float)(1.0 / d0sq_dp))) : 0.0;''')
    s = _sub(s, '''                double dx = m[0] - n[0], dy = m[1] - n[1], dz = m[2] - n[2];
                double sc = 1.0 / (1.0 + (dx * dx + dy * dy + dz * dz) / d01sq);''',
             '''                float dx = (float)m[0] - (float)n[0], dy = (float)m[1] - (float)n[1], dz = (float)m[2] - (float)n[2];
                double sc = (double)(1.0f / (1.0f + (dx * dx + dy * dy + dz * dz) * (float)(1.0 / d01sq)));''')
    return s


def _dp32(s: str) -> str:
    """The NW fill's values (H, the diagonal, gap moves) in FP32 as well."""
    return _sub(_smat32(s), '''            double diag = H[(i - 1) * Hn + (j - 1)] + smat[(i - 1) * Nn + (j - 1)];
            double up = H[(i - 1) * Hn + j], left = H[i * Hn + (j - 1)];
            if (tr[(i - 1) * Hn + j] == 0) up += gap;
            if (tr[i * Hn + (j - 1)] == 0) left += gap;''', '''            float diag = (float)H[(i - 1) * Hn + (j - 1)] + (float)smat[(i - 1) * Nn + (j - 1)];
            float up = (float)H[(i - 1) * Hn + j], left = (float)H[i * Hn + (j - 1)];
            if (tr[(i - 1) * Hn + j] == 0) up += (float)gap;
            if (tr[i * Hn + (j - 1)] == 0) left += (float)gap;''')


def variant_sources(src: str) -> dict[str, str]:
    base = _sub(src, DIST64, DIST32)
    out = {"dist32": base}
    for name, acc in (("kahan32", KAHAN), ("plain32", PLAIN)):
        s = _sub(base, IMIN, IMIN + acc)
        out[name] = _fp32_sums(_sub(s, KABSCH64, KABSCH_CENTRED32))
    for name, mean in (("raw32", 0), ("raw32c", 1)):
        s = _sub(base, IMIN, IMIN + PLAIN)
        s = _fp32_sums(_sub(s, KABSCH64 + '''
    for (int d = 0; d < 3; d++)
        t[d] = cQ[d] - (cP[0] * R[0 * 3 + d] + cP[1] * R[1 * 3 + d] + cP[2] * R[2 * 3 + d]);''', KABSCH_RAW32 + '''
    for (int d = 0; d < 3; d++)
        t[d] = cQ[d] - (cP[0] * R[0 * 3 + d] + cP[1] * R[1 * 3 + d] + cP[2] * R[2 * 3 + d]);'''))
        out[name] = f"#define OFFSET_MEAN {mean}\n" + s
    out["bank32"] = _bank32(src)
    out["qcp64"] = _qcp64(src)
    out["bank32f"] = _bank32f(src)
    out["bank32p"] = _bank32p(src)
    out["smat32"] = _smat32(src)
    out["dp32"] = _dp32(src)
    return out


def build(names, out_dir: str = OUT):
    os.makedirs(out_dir, exist_ok=True)
    src = open(os.path.join(HERE, "indialign_oracle.c")).read()
    libs = {}
    for name, s in variant_sources(src).items():
        if names and name not in names:
            continue
        c = os.path.join(out_dir, f"{name}.c")
        so = os.path.join(out_dir, f"lib{name}.so")
        with open(c, "w") as f:
            f.write(s)
        subprocess.run(["gcc", "-O3", "-std=c11", "-fPIC", "-fopenmp", "-I", HERE, "-shared", "-o", so, c, "-lm"],
                       check=True)
        libs[name] = so
    return libs


def compare(pairs, libs, label):
    ref = abi.bind_reference_abi(ctypes.CDLL(REF_SO))
    st = ctypes.CDLL(STAGES_SO)
    st.ref_tm_score.restype = ctypes.c_double

    def rescore(p, R, t):
        d0, d0s, sd8 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        st.ref_d0(ctypes.c_double(p.lnorm), ctypes.byref(d0), ctypes.byref(d0s), ctypes.byref(sd8))
        arrs = [np.ascontiguousarray(a) for a in (p.pred.reshape(-1), p.native.reshape(-1), p.valid, R, t)]
        ptr = [ctypes.c_void_p(a.ctypes.data) for a in arrs]
        return st.ref_tm_score(*ptr, d0, ctypes.c_double(p.lnorm), sd8, ctypes.c_int(len(p.valid)),
                               ctypes.c_int(0))

    t0 = time.time()
    _, sref, _, _ = abi.run_batch(ref, pairs)
    print(f"{label}: {len(pairs)} pairs, reference build {time.time() - t0:.0f} s", flush=True)
    for name, so in libs.items():
        lib = abi.bind_reference_abi(ctypes.CDLL(so), prefix="ora_")
        t0 = time.time()
        _, _, R, t = abi.run_batch(lib, pairs, prefix="ora_")
        d = np.array([rescore(p, R[k], t[k]) for k, p in enumerate(pairs)]) - sref
        extra = ""
        if hasattr(lib, "qcp_calls"):
            calls = ctypes.c_long.in_dll(lib, "qcp_calls").value
            fb = ctypes.c_long.in_dll(lib, "qcp_fallbacks").value
            extra = f"  eigen-solves {calls}, Jacobi fallbacks {fb} ({fb / max(calls, 1):.1e})"
        print(f"  {name:8s} {time.time() - t0:4.0f} s  mean {d.mean():+.2e}  worst {d.min():+.2e}  "
              f"best {d.max():+.2e}  below -1e-6: {int((d < -1e-6).sum())}  "
              f"below -1e-4: {int((d < -1e-4).sum())}{extra}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=400, help="pairs of the 4096-pair shape (L 40-300)")
    ap.add_argument("--seed", type=int, default=21)
    ap.add_argument("--hard", type=int, default=160, help="hard pairs with L <= 400 (0: none)")
    ap.add_argument("--hard-seed", type=int, default=22)
    ap.add_argument("--variants", nargs="*", default=[])
    a = ap.parse_args()
    if not (os.path.exists(REF_SO) and os.path.exists(STAGES_SO)):
        raise SystemExit("reference build missing: make -C oracle ref")
    libs = build(a.variants)
    if a.pairs:
        compare(W.batch(a.pairs, 40, 300, seed=a.seed), libs, f"batch L 40-300 seed {a.seed}")
    if a.hard:
        hard = [p for p in W.hard(4 * a.hard, seed=a.hard_seed) if p.pred.shape[0] <= 400][:a.hard]
        compare(hard, libs, f"hard L <= 400 seed {a.hard_seed}")


if __name__ == "__main__":
    main()
