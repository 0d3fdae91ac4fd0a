// Learned candidate ranker for the rescue passes of the search: the
// local-fragment windows (evaluate_local_fragment_dp,
// indialign_c/rescue.h:50-117, normal and dense) and the threading-DP offsets
// (evaluate_threading_dp, rescue.h:121-190).
//
// Each rescue pass refines every candidate start of a weak pair (a window
// (fragment length, pred start, native start), or an offset's overlap) with
// NW dp_refine chains, hundreds to thousands per pair.  The ranker predicts
// each candidate's refined score from 16 cheap features, and the search
// refines only the top-k candidates of a pair, falling back to all of them
// when the predicted top-1 / top-k margin is small and on a random audit of
// pairs.
//
//   k_rank    persistent CTAs over 64-candidate chunks: per candidate the
//             warp computes the features (segment Kabsch + diagonal TM sums,
//             FP64), then the 16 -> 128 -> 128 -> 1 GELU MLP runs on BF16
//             tensor cores (mma.sync m16n8k16, FP32 accumulation) over the
//             warp's 16-candidate tile, with the weights in shared memory.
//   k_select  warp per task: top-k by (predicted score desc, index asc),
//             margin fallback, audit draw, list in ascending order (so the
//             stage's reduction keeps the reference's first-max rule).
//   k_audit   audited pairs: did the top-k contain the best refined score?
//   training  forward with saved activations, MSE + pairwise ranking loss,
//             backward: the three weight / activation products on the
//             tcgen05 tensor cores (k_gemm_tc in k_tcgen05.cu: TMA-staged
//             BF16 operands, TMEM accumulators, split-K with a fixed-order
//             sum), the bias and head gradients here over row blocks summed
//             in block order; Adam on FP32 master weights.
#include <cuda_bf16.h>

#include "dmath.cuh"
#include "pipeline.h"
#include "kernels.h"
#include "sched.cuh"

namespace ia {

static_assert(kMaxTopK == 32, "selection lists are one entry per lane");

namespace {

constexpr unsigned kAllLanes = 0xffffffffu;
constexpr int kW1Words = 12;  // bf16 row of W1T (16) padded to 24 -> conflict-free fragments
constexpr int kW2Words = 68;  // bf16 row of W2T (128) padded to 136

struct MlpSmem {
    uint32_t w1t[kHidden][kW1Words];
    uint32_t w2t[kHidden][kW2Words];
    float b1[kHidden], b2[kHidden], w3[kHidden];
    float mean[kFeatures], inv_std[kFeatures];
    float b3, pad_[3];
};

IA_DEV uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}


// D += A B for one m16n8k16 BF16 tile (row-major A, column-major B).
IA_DEV void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).
constexpr float kGeluC = 0.7978845608028654f;
constexpr float kGeluA = 0.044715f;
IA_DEV float gelu(float x) {
    const float u = kGeluC * (x + kGeluA * x * x * x);
    return 0.5f * x * (1.0f + tanhf(u));
}
IA_DEV float gelu_grad(float x) {
    const float u = kGeluC * (x + kGeluA * x * x * x);
    const float th = tanhf(u);
    return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * kGeluC * (1.0f + 3.0f * kGeluA * x * x);
}

// Copy the packed parameters into the fragment-friendly shared layout (all
// threads of the CTA; caller synchronises).
IA_DEV void load_mlp_smem(const MlpPacked *g, MlpSmem *s) {
    const uint32_t *w1 = reinterpret_cast<const uint32_t *>(g->W1T);
    const uint32_t *w2 = reinterpret_cast<const uint32_t *>(g->W2T);
    for (int i = threadIdx.x; i < kHidden * (kFeatures / 2); i += blockDim.x)
        s->w1t[i / (kFeatures / 2)][i % (kFeatures / 2)] = w1[i];
    for (int i = threadIdx.x; i < kHidden * (kHidden / 2); i += blockDim.x)
        s->w2t[i / (kHidden / 2)][i % (kHidden / 2)] = w2[i];
    for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
        s->b1[i] = g->b1[i];
        s->b2[i] = g->b2[i];
        s->w3[i] = g->w3[i];
    }
    for (int i = threadIdx.x; i < kFeatures; i += blockDim.x) {
        s->mean[i] = g->mean[i];
        s->inv_std[i] = g->inv_std[i];
    }
    if (threadIdx.x == 0) s->b3 = g->b3;
}

// The MLP on one 16-row tile by one warp.  xt: [16][16] standardised inputs
// (FP32, shared).  Lane (g = lane/4, c = lane%4) returns the outputs of rows
// g and g+8 (valid on every lane of the quad).  With `sv`, rows < nvalid of
// the tile's activations are stored at rows row0.. of the save arrays.
IA_DEV void mlp_tile(const MlpSmem &S, const float *xt, float &y_g, float &y_g8, const MlpSave *sv,
                     long long row0, int nvalid) {
    const int lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
    const bool st_g = sv && g < nvalid, st_g8 = sv && g + 8 < nvalid;
    const long long rg = row0 + g, rg8 = row0 + g + 8;
    uint32_t a[4];
    a[0] = pack_bf16(xt[g * 16 + 2 * c], xt[g * 16 + 2 * c + 1]);
    a[1] = pack_bf16(xt[(g + 8) * 16 + 2 * c], xt[(g + 8) * 16 + 2 * c + 1]);
    a[2] = pack_bf16(xt[g * 16 + 2 * c + 8], xt[g * 16 + 2 * c + 9]);
    a[3] = pack_bf16(xt[(g + 8) * 16 + 2 * c + 8], xt[(g + 8) * 16 + 2 * c + 9]);
    if (st_g) {
        uint32_t *x = reinterpret_cast<uint32_t *>(sv->xn + rg * kFeatures);
        x[c] = a[0];
        x[4 + c] = a[2];
    }
    if (st_g8) {
        uint32_t *x = reinterpret_cast<uint32_t *>(sv->xn + rg8 * kFeatures);
        x[c] = a[1];
        x[4 + c] = a[3];
    }
    // layer 1: [16 x 16] x [16 x 128]
    uint32_t h[8][4];
#pragma unroll
    for (int kk = 0; kk < 8; kk++) {
        float d[2][4];
#pragma unroll
        for (int half = 0; half < 2; half++) {
            const int nt = 2 * kk + half, col = 8 * nt + 2 * c;
            d[half][0] = d[half][2] = S.b1[col];
            d[half][1] = d[half][3] = S.b1[col + 1];
            mma_bf16(d[half], a, S.w1t[8 * nt + g][c], S.w1t[8 * nt + g][c + 4]);
            if (st_g) *reinterpret_cast<float2 *>(sv->z1 + rg * kHidden + col) = make_float2(d[half][0], d[half][1]);
            if (st_g8) *reinterpret_cast<float2 *>(sv->z1 + rg8 * kHidden + col) = make_float2(d[half][2], d[half][3]);
        }
        // accumulator tiles 2kk, 2kk+1 are the A fragment of k-chunk kk
        h[kk][0] = pack_bf16(gelu(d[0][0]), gelu(d[0][1]));
        h[kk][1] = pack_bf16(gelu(d[0][2]), gelu(d[0][3]));
        h[kk][2] = pack_bf16(gelu(d[1][0]), gelu(d[1][1]));
        h[kk][3] = pack_bf16(gelu(d[1][2]), gelu(d[1][3]));
        if (st_g) {
            uint32_t *o = reinterpret_cast<uint32_t *>(sv->h1 + rg * kHidden + 16 * kk);
            o[c] = h[kk][0];
            o[4 + c] = h[kk][2];
        }
        if (st_g8) {
            uint32_t *o = reinterpret_cast<uint32_t *>(sv->h1 + rg8 * kHidden + 16 * kk);
            o[c] = h[kk][1];
            o[4 + c] = h[kk][3];
        }
    }
    // layer 2: [16 x 128] x [128 x 128], then the w3 head
    float y0 = 0.f, y8 = 0.f;
#pragma unroll 4
    for (int nt = 0; nt < 16; nt++) {
        const int col = 8 * nt + 2 * c;
        float d[4] = {S.b2[col], S.b2[col + 1], S.b2[col], S.b2[col + 1]};
        const uint32_t *wr = S.w2t[8 * nt + g];
#pragma unroll
        for (int kk = 0; kk < 8; kk++) mma_bf16(d, h[kk], wr[8 * kk + c], wr[8 * kk + c + 4]);
        if (st_g) *reinterpret_cast<float2 *>(sv->z2 + rg * kHidden + col) = make_float2(d[0], d[1]);
        if (st_g8) *reinterpret_cast<float2 *>(sv->z2 + rg8 * kHidden + col) = make_float2(d[2], d[3]);
        y0 += gelu(d[0]) * S.w3[col] + gelu(d[1]) * S.w3[col + 1];
        y8 += gelu(d[2]) * S.w3[col] + gelu(d[3]) * S.w3[col + 1];
    }
    y0 += __shfl_xor_sync(kAllLanes, y0, 1);
    y0 += __shfl_xor_sync(kAllLanes, y0, 2);
    y8 += __shfl_xor_sync(kAllLanes, y8, 1);
    y8 += __shfl_xor_sync(kAllLanes, y8, 2);
    y_g = y0 + S.b3;
    y_g8 = y8 + S.b3;
}

// The 16 features of candidate w of a pair (raw, before standardisation),
// computed by the whole warp; every lane returns all 16.
//   0 segment length / ml         1 pred start / (plen-1)   2 native start / (nlen-1)
//   3 start shift / ml            4 segment RMSD / 10       5 TM along the segment's
//   diagonal under its Kabsch     6, 7 fraction of that diagonal within d0, 2 d0
//   8 segment-local TM            9, 10 stem fraction of the pred / native segment
//   11 log(ml) / 7                12 running best score     13 candidate kind / 2
//   14 min(RMSD / d0, 10) / 10    15 TM along the same-index diagonal
// (ml = min(plen, nlen); indices are compact valid-residue positions.)
// Detailed-search seeds are segments of an aligned set (plen == nlen == the
// aligned count, SS labels absent: stem fractions 0).
IA_DEV void window_features(const Pts &x, const uint8_t *Lp, const uint8_t *Ln, const PairInfo &I,
                            int plen, int nlen, double best, int kind, int w, float (&f)[kFeatures]) {
    const int lane = threadIdx.x & 31;
    const int ml = plen < nlen ? plen : nlen;
    int flen, ps, ns;
    cand_at(kind, plen, nlen, w, flen, ps, ns);
    double R[9], t[3];
    warp_kabsch_window(x, ps, ns, flen, R, t);
    const double d0sq = I.d0 * I.d0, inv = 1.0 / d0sq;
    double sd2 = 0.0, stm = 0.0, sp = 0.0, sn = 0.0;
    // one pass over pred residues i: the segment [ps, ps + flen) and the
    // diagonal [lo, hi) pair i with native i + s (the segment lies on that
    // diagonal), the same-index sum pairs i < ml with native i; each moved
    // pred point is computed once for all three
    const int s = ns - ps;
    const int lo = s < 0 ? -s : 0, hi = plen < nlen - s ? plen : nlen - s;
    double dtm = 0.0, c1 = 0.0, c2 = 0.0, tm0 = 0.0;
    const int i_end = hi > ml ? hi : ml;
    for (int i = lane; i < i_end; i += 32) {
        const double *p = x.P + 3 * i;
        double mx, my, mz;
        xform(R, t, p[0], p[1], p[2], mx, my, mz);
        if (i >= lo && i < hi) {
            const double *q = x.Q + 3 * (i + s);
            const double dx = mx - q[0], dy = my - q[1], dz = mz - q[2];
            const double d2 = dx * dx + dy * dy + dz * dz;
            const double term = 1.0 / (1.0 + d2 * inv);
            dtm += term;
            c1 += d2 < d0sq ? 1.0 : 0.0;
            c2 += d2 < 4.0 * d0sq ? 1.0 : 0.0;
            if (i >= ps && i < ps + flen) {
                sd2 += d2;
                stm += term;
                if (Lp) {
                    sp += Lp[i] != 'L' ? 1.0 : 0.0;
                    sn += Ln[i + s] != 'L' ? 1.0 : 0.0;
                }
            }
        }
        if (i < ml) {
            const double *q = x.Q + 3 * i;
            const double dx = mx - q[0], dy = my - q[1], dz = mz - q[2];
            tm0 += 1.0 / (1.0 + (dx * dx + dy * dy + dz * dz) * inv);
        }
    }
    sd2 = warp_sum(sd2);
    stm = warp_sum(stm);
    sp = warp_sum(sp);
    sn = warp_sum(sn);
    dtm = warp_sum(dtm);
    c1 = warp_sum(c1);
    c2 = warp_sum(c2);
    tm0 = warp_sum(tm0);
    const double mld = (double)ml, rmsd = sqrt(sd2 / flen);
    f[0] = (float)(flen / mld);
    f[1] = (float)(ps / (double)(plen > 1 ? plen - 1 : 1));
    f[2] = (float)(ns / (double)(nlen > 1 ? nlen - 1 : 1));
    f[3] = (float)(s / mld);
    f[4] = (float)(rmsd / 10.0);
    f[5] = (float)(dtm / I.lnorm);
    f[6] = (float)(c1 / mld);
    f[7] = (float)(c2 / mld);
    f[8] = (float)(stm / flen);
    f[9] = (float)(sp / flen);
    f[10] = (float)(sn / flen);
    f[11] = (float)(log(mld) / 7.0);
    f[12] = (float)best;
    f[13] = 0.5f * (float)kind;
    f[14] = (float)(fmin(rmsd / I.d0, 10.0) / 10.0);
    f[15] = (float)(tm0 / I.lnorm);
}

// Features of seed w of a pair's main seed bank (seeds.h:41-283): a window
// [s, s+len) of the full pair or an anchor bitmask, restricted to valid
// residues.  Every lane returns all 16:
//   0 selected / valid residues   1 first selected / N     2 selected span / N
//   3 bitmask seed (0/1)          4 seed Kabsch RMSD / 10  5 same-index TM of the
//   seed's Kabsch over all valid residues                  6, 7, 9 fraction of the
//   valid residues within d0, 2 d0, d0_search              8 TM over the seed
//   10 0                          11 log(N) / 7            12 0
//   13 candidate kind / 2         14 min(RMSD / d0, 10) / 10
//   15 TM over the seed / lnorm
IA_DEV void main_seed_features(const DevBatch &b, const PairInfo &I, int p, int w, float (&f)[kFeatures]) {
    const int lane = threadIdx.x & 31, N = I.N;
    const int2 e = b.seeds[(size_t)p * kMaxSeeds + w];
    const bool bitm = e.x < 0;
    const uint32_t *brow = bitm ? b.bits + I.bitoff + (size_t)(-1 - e.x) * I.words : nullptr;
    const int lo = bitm ? 0 : e.x, hi = bitm ? N : min(N, e.x + e.y);
    const double *P = b.pred + 3 * (size_t)I.off, *Q = b.nat + 3 * (size_t)I.off;
    const uint8_t *V = b.v + I.off;
    auto sel = [&](int i) {
        const uint8_t v = V[i];
        return bitm ? (((brow[i >> 5] >> (i & 31)) & 1u) && (v & 1u)) : (v != 0);
    };
    Moments m;
    m.clear();
    int first = 0x7fffffff, last = -1;
    for (int i = lo + lane; i < hi; i += 32)
        if (sel(i)) {
            m.add(P[3 * i], P[3 * i + 1], P[3 * i + 2], Q[3 * i], Q[3 * i + 1], Q[3 * i + 2]);
            first = min(first, i);
            last = max(last, i);
        }
    m.group_sum(32);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        first = min(first, __shfl_xor_sync(kAllLanes, first, o));
        last = max(last, __shfl_xor_sync(kAllLanes, last, o));
    }
    double R[9], t[3];
    kabsch_from_moments(m, 3.0, R, t);
    const double d0sq = I.d0 * I.d0, inv = 1.0 / d0sq, dssq = I.d0s * I.d0s;
    double tm = 0.0, c1 = 0.0, c2 = 0.0, cs = 0.0, sd2 = 0.0, stm = 0.0;
    for (int i = lane; i < N; i += 32) {
        if (!V[i]) continue;
        const double d2 = dist2(R, t, P[3 * i], P[3 * i + 1], P[3 * i + 2], Q[3 * i], Q[3 * i + 1], Q[3 * i + 2]);
        const double term = 1.0 / (1.0 + d2 * inv);
        tm += term;
        c1 += d2 < d0sq ? 1.0 : 0.0;
        c2 += d2 < 4.0 * d0sq ? 1.0 : 0.0;
        cs += d2 < dssq ? 1.0 : 0.0;
        if (i >= lo && i < hi && sel(i)) {
            sd2 += d2;
            stm += term;
        }
    }
    tm = warp_sum(tm);
    c1 = warp_sum(c1);
    c2 = warp_sum(c2);
    cs = warp_sum(cs);
    sd2 = warp_sum(sd2);
    stm = warp_sum(stm);
    const double cnt = fmax(m.w, 1.0), vc = (double)(I.vcount > 0 ? I.vcount : 1), Nd = (double)(N > 0 ? N : 1);
    const double rmsd = sqrt(sd2 / cnt);
    f[0] = (float)(m.w / vc);
    f[1] = (float)((last >= 0 ? first : 0) / Nd);
    f[2] = (float)((last >= 0 ? last - first + 1 : 0) / Nd);
    f[3] = bitm ? 1.f : 0.f;
    f[4] = (float)(rmsd / 10.0);
    f[5] = (float)(tm / I.lnorm);
    f[6] = (float)(c1 / vc);
    f[7] = (float)(c2 / vc);
    f[8] = (float)(stm / cnt);
    f[9] = (float)(cs / vc);
    f[10] = 0.f;
    f[11] = (float)(log(Nd) / 7.0);
    f[12] = 0.f;
    f[13] = 0.5f * (float)CAND_MAIN;
    f[14] = (float)(fmin(rmsd / I.d0, 10.0) / 10.0);
    f[15] = (float)(stm / I.lnorm);
}

// The candidate set of ranking task t: a pair (windows, offsets, seeds) or a
// (pair, alignment slot) of a detailed search, with its point set.
struct RankTask {
    int p, W, plen, nlen;
    bool on;
    Pts x;
    const uint8_t *Lp, *Ln;
};

IA_DEV RankTask rank_task(const DevBatch &b, const RankArgs &a, int t) {
    RankTask r;
    if (a.kind == CAND_DET) {
        r.p = t / kDetSlots;
        const int g = t % kDetSlots;
        const PairInfo &I = b.info[r.p];
        const PairState &S = b.state[r.p];
        const int na = S.na[g];
        // the detailed searches' own gates (align.h:115-118, ss.h:96-99)
        r.on = I.status == 0 && na >= 3 && (a.det_ss ? (g == 0 && S.flag != 0) : S.active[g] != 0);
        const size_t base = 3 * (kDetSlots * (size_t)I.off + (size_t)g * I.N);
        r.x = {a.alP + base, a.alQ + base};
        r.plen = r.nlen = na;
        r.Lp = r.Ln = nullptr;
        r.W = r.on ? cand_count(CAND_DET, na, na) : 0;
    } else if (a.kind == CAND_MAIN) {
        r.p = t;
        const PairInfo &I = b.info[t];
        r.on = I.status == 0 && I.K > 0;
        r.x = {nullptr, nullptr};
        r.plen = I.plen;
        r.nlen = I.nlen;
        r.Lp = r.Ln = nullptr;
        r.W = r.on ? I.K : 0;
    } else {
        r.p = t;
        const PairInfo &I = b.info[t];
        r.on = I.status == 0 && b.state[t].flag != 0;
        r.x = {b.predc + 3 * (size_t)I.off, b.natc + 3 * (size_t)I.off};
        r.plen = I.plen;
        r.nlen = I.nlen;
        r.Lp = reinterpret_cast<const uint8_t *>(b.sspc + I.off);
        r.Ln = reinterpret_cast<const uint8_t *>(b.ssnc + I.off);
        r.W = r.on ? cand_count(a.kind, I.plen, I.nlen) : 0;
    }
    return r;
}

}  // namespace

// ---- ranking: features + MLP over the candidates of gated tasks -----------------
__global__ void k_plan_rank(DevBatch b, RankArgs a, int *counts) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.ntasks) return;
    const RankTask r = rank_task(b, a, t);
    const PairInfo &I = b.info[r.p];
    const bool small = (I.plen < I.nlen ? I.plen : I.nlen) < a.min_len;
    counts[t] = r.on && !small && r.W > 0 ? (r.W + kRankChunk - 1) / kRankChunk : 0;
}

__global__ void __launch_bounds__(128) k_rank(DevBatch b, RankArgs a, const int *__restrict__ chunk_begin,
                                              const ScanOut *__restrict__ scan, int *counter) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpSmem &S = *reinterpret_cast<MlpSmem *>(smem_raw);
    float *xt = reinterpret_cast<float *>(smem_raw + sizeof(MlpSmem)) + (threadIdx.x >> 5) * 256;
    __shared__ int s_chunk, s_pair;
    if (a.mlp) load_mlp_smem(a.mlp, &S);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = scan->total_chunks;
    for (;;) {
        if (threadIdx.x == 0) {
            const int c = atomicAdd(counter, 1);
            int t = -1;
            if (c < total) {
                int lo = 0, hi = a.ntasks;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (chunk_begin[mid] <= c) lo = mid + 1; else hi = mid;
                }
                t = lo - 1;
            }
            s_chunk = c;
            s_pair = t;
        }
        __syncthreads();
        const int c = s_chunk, ti = s_pair;
        if (c >= total || ti < 0) break;
        const RankTask rt = rank_task(b, a, ti);
        const PairInfo &I = b.info[rt.p];
        const int W = rt.W;
        const int w0 = (c - chunk_begin[ti]) * kRankChunk + warp * 16;
        if (w0 < W) {
            const double best = b.state[rt.p].rec[REC_BEST][0];
            const long long wb = a.wbase[ti];
            for (int r = 0; r < 16; r++) {
                const int w = w0 + r;
                float mine = 0.f;
                if (w < W) {
                    float f[kFeatures];
                    if (a.kind == CAND_MAIN)
                        main_seed_features(b, I, rt.p, w, f);
                    else
                        window_features(rt.x, rt.Lp, rt.Ln, I, rt.plen, rt.nlen, best, a.kind, w, f);
#pragma unroll
                    for (int j = 0; j < kFeatures; j++)
                        if (lane == j) mine = f[j];
                    if (a.feat && lane < kFeatures) a.feat[(wb + w) * kFeatures + lane] = mine;
                }
                if (lane < kFeatures)
                    xt[r * 16 + lane] = (w < W && a.mlp) ? (mine - S.mean[lane]) * S.inv_std[lane] : 0.f;
            }
            __syncwarp();
            if (a.mlp) {
                float y0, y8;
                mlp_tile(S, xt, y0, y8, nullptr, 0, 0);
                const int g = lane >> 2;
                if ((lane & 3) == 0) {
                    if (w0 + g < W) a.score[wb + w0 + g] = y0;
                    if (w0 + g + 8 < W) a.score[wb + w0 + g + 8] = y8;
                }
            }
            __syncwarp();
        }
        __syncthreads();
    }
}

// ---- top-k selection ------------------------------------------------------------
IA_DEV unsigned long long mix64(unsigned long long z) {  // splitmix64 finaliser
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__global__ void k_select(DevBatch b, SelectArgs a) {
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (t >= a.task.ntasks) return;
    const RankTask rt = rank_task(b, a.task, t);
    const int p = rt.p;  // audit draws are per pair
    int *list = a.wlist + (size_t)t * kMaxTopK;
    if (!rt.on) {
        if (lane == 0) a.wcount[t] = -1;
        list[lane] = -1;
        return;
    }
    const int W = rt.W;
    const int k = a.top_k < kMaxTopK ? (a.top_k > 0 ? a.top_k : 1) : kMaxTopK;
    if (lane == 0) {
        atomicAdd(a.stats + RS_GATED, 1ull);
        atomicAdd(a.stats + RS_WINDOWS, (unsigned long long)W);
    }
    const PairInfo &I = b.info[p];
    if (W <= k || (I.plen < I.nlen ? I.plen : I.nlen) < a.task.min_len) {  // short list or short pair
        list[lane] = -1;
        if (lane == 0) {
            a.wcount[t] = -1;
            atomicAdd(a.stats + RS_SMALL, 1ull);
            atomicAdd(a.stats + RS_REFINED, (unsigned long long)W);
        }
        return;
    }
    const float *sc = a.score + a.wbase[t];
    // k rounds of "next in (score desc, window asc) order"
    float prev_s = INFINITY, top1 = 0.f;
    int prev_i = -1;
    for (int r = 0; r < k; r++) {
        float bs = -INFINITY;
        int bi = 0x7fffffff;
        for (int w = lane; w < W; w += 32) {
            float v = sc[w];
            if (!(v == v)) v = -INFINITY;
            const bool after = v < prev_s || (v == prev_s && w > prev_i);
            if (after && (v > bs || (v == bs && w < bi))) {
                bs = v;
                bi = w;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float s2 = __shfl_xor_sync(kAllLanes, bs, o);
            const int i2 = __shfl_xor_sync(kAllLanes, bi, o);
            if (s2 > bs || (s2 == bs && i2 < bi)) {
                bs = s2;
                bi = i2;
            }
        }
        if (r == 0) top1 = bs;
        prev_s = bs;
        prev_i = bi;
        if (lane == 0) list[r] = bi;
    }
    if (lane == 0) {
        for (int i = 1; i < k; i++)  // ascending window order
            for (int j = i; j > 0 && list[j] < list[j - 1]; j--) {
                const int t = list[j]; list[j] = list[j - 1]; list[j - 1] = t;
            }
        // the draw of the pair's index in the caller's batch, so that a
        // length bucket's sub-batch audits the same pairs as the whole batch
        const unsigned long long gp = (unsigned long long)(b.gidx ? b.gidx[p] : p);
        const double u = (double)(mix64(a.seed ^ mix64(gp + 0x9e3779b97f4a7c15ull)) >> 11) *
                         (1.0 / 9007199254740992.0);
        if (u < a.audit_rate) {
            a.wcount[t] = -2;
            atomicAdd(a.stats + RS_AUDIT, 1ull);
            atomicAdd(a.stats + RS_REFINED, (unsigned long long)W);
        } else if (top1 - prev_s < a.margin) {
            a.wcount[t] = -1;
            atomicAdd(a.stats + RS_FALLBACK, 1ull);
            atomicAdd(a.stats + RS_REFINED, (unsigned long long)W);
        } else {
            a.wcount[t] = k;
            atomicAdd(a.stats + RS_PRUNED, 1ull);
            atomicAdd(a.stats + RS_REFINED, (unsigned long long)k);
        }
    }
}

// A candidate's refined score: the dp_refine result over its two gap chains
// (later chain only if strictly better, indialign_c/align.h:131-145); for a
// threading offset the better of that and its detailed search
// (rescue.h:163-165), -inf for an offset that was not searched; for a
// detailed-search seed the best of its cutoff items.
IA_DEV double cand_score(const CandRes &r, int kind, int det_ss, int t, int w) {
    if (kind == CAND_DET || kind == CAND_MAIN) {  // best of the seed's cutoff items
        // the bank launch's task of list t: a DET list is (pair, slot); the
        // SS seeds' detailed search ran one task per pair, dp_refine's (also
        // inside the SS stage) one per slot
        (void)det_ss;
        const BankTask &T = r.btasks[kind == CAND_DET && r.bank_per_pair ? t / kDetSlots : t];
        double s = -INFINITY;
        for (int ci = 0; ci < T.C; ci++)
            s = fmax(s, r.item_res[((size_t)T.item_base + (size_t)w * T.C + ci) * kRec]);
        return s;
    }
    const int p = t;
    const double *res = r.chain_res + (size_t)r.chain_base[p] * kRec;
    const double s0 = res[(size_t)(2 * w) * kRec], s1 = res[(size_t)(2 * w + 1) * kRec];
    double s = s1 > s0 ? s1 : s0;
    if (r.det) {
        const double dt = r.det[((size_t)r.det_base[p] + w) * kRec];
        if (dt <= -1e299) return -INFINITY;
        if (!(s > dt)) s = dt;
    }
    return s;
}

// Audited pairs ran every candidate: count those whose selected candidates
// miss the best refined score.
__global__ void k_audit(DevBatch b, SelectArgs a, CandRes r) {
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (t >= a.task.ntasks || a.wcount[t] != -2) return;
    const RankTask rt = rank_task(b, a.task, t);
    const int W = rt.W, kind = a.task.kind, ds = a.task.det_ss;
    const int k = a.top_k < kMaxTopK ? (a.top_k > 0 ? a.top_k : 1) : kMaxTopK;
    double full = -INFINITY, sel = -INFINITY;
    for (int w = lane; w < W; w += 32) full = fmax(full, cand_score(r, kind, ds, t, w));
    for (int j = lane; j < k; j += 32)
        sel = fmax(sel, cand_score(r, kind, ds, t, a.wlist[(size_t)t * kMaxTopK + j]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        full = fmax(full, __shfl_xor_sync(kAllLanes, full, o));
        sel = fmax(sel, __shfl_xor_sync(kAllLanes, sel, o));
    }
    if (lane == 0 && sel < full) {
        atomicAdd(a.stats + RS_AUDIT_MISS, 1ull);
        if (sel < full - 1e-4) atomicAdd(a.stats + RS_AUDIT_MISS_1E4, 1ull);
        if (sel < full - 1e-3) atomicAdd(a.stats + RS_AUDIT_MISS_1E3, 1ull);
    }
}

// Training labels: every candidate's refined score for pairs that ran the
// stage on all candidates, NaN elsewhere.
// The label array starts as NaN (the host fills it before the search) and
// tasks of a pass that did not run are left alone, so a detailed-search slot
// keeps the (features, labels) of the last search that ran on it.
__global__ void k_collect_labels(DevBatch b, RankArgs a, CandRes r, float *label) {
    const int t = blockIdx.x;
    const RankTask rt = rank_task(b, a, t);
    if (!rt.on) return;
    float *out = label + a.wbase[t];
    for (int w = threadIdx.x; w < rt.W; w += blockDim.x) {
        const double s = cand_score(r, a.kind, a.det_ss, t, w);
        out[w] = s > -1e299 ? (float)s : NAN;
    }
}

// ---- training ---------------------------------------------------------------------
__global__ void k_mlp_pack(const float *__restrict__ blob, MlpPacked *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kHidden * kFeatures) {  // W1T[o][k] = W1[k][o]
        const int o = i / kFeatures, k = i % kFeatures;
        out->W1T[i] = __bfloat16_as_ushort(__float2bfloat16_rn(blob[kBlobW1 + k * kHidden + o]));
    }
    if (i < kHidden * kHidden) {
        const int o = i / kHidden, k = i % kHidden;
        out->W2T[i] = __bfloat16_as_ushort(__float2bfloat16_rn(blob[kBlobW2 + k * kHidden + o]));
        out->W2[i] = __bfloat16_as_ushort(__float2bfloat16_rn(blob[kBlobW2 + i]));
    }
    if (i < kHidden) {
        out->b1[i] = blob[kBlobB1 + i];
        out->b2[i] = blob[kBlobB2 + i];
        out->w3[i] = blob[kBlobW3 + i];
    }
    if (i < kFeatures) {
        out->mean[i] = blob[kBlobMean + i];
        const float sd = blob[kBlobStd + i];
        out->inv_std[i] = sd > 0.f ? 1.0f / sd : 1.0f;
    }
    if (i == 0) out->b3 = blob[kBlobB3];
}

// Forward over n raw feature rows (row-major [n][16]); 4 warps x 16 rows per CTA.
__global__ void __launch_bounds__(128) k_mlp_forward(const MlpPacked *mlp, const float *__restrict__ x, int n,
                                                     float *y, MlpSave sv, int save) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpSmem &S = *reinterpret_cast<MlpSmem *>(smem_raw);
    float *xt = reinterpret_cast<float *>(smem_raw + sizeof(MlpSmem)) + (threadIdx.x >> 5) * 256;
    load_mlp_smem(mlp, &S);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long long row0 = (long long)blockIdx.x * 64 + (threadIdx.x >> 5) * 16;
    if (row0 >= n) return;
    const int nvalid = n - row0 < 16 ? (int)(n - row0) : 16;
    for (int e = lane; e < 256; e += 32) {
        const int r = e >> 4, j = e & 15;
        xt[e] = r < nvalid ? (x[(row0 + r) * kFeatures + j] - S.mean[j]) * S.inv_std[j] : 0.f;
    }
    __syncwarp();
    float y0, y8;
    mlp_tile(S, xt, y0, y8, save ? &sv : nullptr, row0, nvalid);
    const int g = lane >> 2;
    if ((lane & 3) == 0) {
        if (g < nvalid) y[row0 + g] = y0;
        if (g + 8 < nvalid) y[row0 + g + 8] = y8;
    }
}

// Loss over n = 2m predictions: mean squared error plus lambda x a pairwise
// logistic ranking term on the rows (2i, 2i+1), which the caller draws from
// the same pair.  One CTA; fixed-order reduction.
__global__ void __launch_bounds__(1024) k_mlp_loss(const float *__restrict__ y, const float *__restrict__ t,
                                                   int n, float lambda, float *dy, float *loss) {
    __shared__ float red[32];
    const int m = n / 2;
    float acc = 0.f;
    const float inv_n = 1.0f / (float)(n > 0 ? n : 1), inv_m = 1.0f / (float)(m > 0 ? m : 1);
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int ia = 2 * i, ib = 2 * i + 1;
        const float ea = y[ia] - t[ia], eb = y[ib] - t[ib];
        float ga = 2.f * ea * inv_n, gb = 2.f * eb * inv_n;
        acc += (ea * ea + eb * eb) * inv_n;
        const float dt = t[ia] - t[ib];
        if (fabsf(dt) > 1e-6f) {
            const float sgn = dt > 0.f ? 1.f : -1.f;
            const float z = -sgn * (y[ia] - y[ib]);
            const float sp = z > 20.f ? z : log1pf(expf(z));
            const float sig = 1.f / (1.f + expf(-z));
            acc += lambda * sp * inv_m;
            ga += -lambda * sgn * sig * inv_m;
            gb += lambda * sgn * sig * inv_m;
        }
        dy[ia] = ga;
        dy[ib] = gb;
    }
    if ((n & 1) && threadIdx.x == 0) {  // odd tail: MSE only
        const float e = y[n - 1] - t[n - 1];
        acc += e * e * inv_n;
        dy[n - 1] = 2.f * e * inv_n;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kAllLanes, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
        *loss = s;
    }
}

// Head backward over row block blockIdx.y (rows [r0, r1)): dz2 = dy w3
// gelu'(z2) (bf16) and the block's partial sums of dz2 (db2), dy gelu(z2)
// (dw3) and dy (db3) at red[blockIdx.y * kBwdRedStride + {0, 128, 256}].
// Block = 32 columns x 8 row groups; grid (4, row blocks).
__global__ void __launch_bounds__(256) k_mlp_head_bwd(const MlpPacked *mlp, const float *__restrict__ dy,
                                                      const float *__restrict__ z2, int n, int rows_per,
                                                      uint16_t *dz2, float *red) {
    __shared__ float r_b2[8][33], r_w3[8][33];
    const int col = blockIdx.x * 32 + (threadIdx.x & 31), rg = threadIdx.x >> 5;
    const int r0 = blockIdx.y * rows_per, r1 = min(n, r0 + rows_per);
    const float w3 = mlp->w3[col];
    float sb = 0.f, sw = 0.f;
    for (int r = r0 + rg; r < r1; r += 8) {
        const float z = z2[(size_t)r * kHidden + col], d = dy[r];
        const float dz = d * w3 * gelu_grad(z);
        dz2[(size_t)r * kHidden + col] = __bfloat16_as_ushort(__float2bfloat16_rn(dz));
        sb += dz;
        sw += d * gelu(z);
    }
    r_b2[rg][threadIdx.x & 31] = sb;
    r_w3[rg][threadIdx.x & 31] = sw;
    __syncthreads();
    float *out = red + (size_t)blockIdx.y * kBwdRedStride;
    if (rg == 0) {
        float b2 = 0.f, w = 0.f;
        for (int k = 0; k < 8; k++) {
            b2 += r_b2[k][threadIdx.x];
            w += r_w3[k][threadIdx.x];
        }
        out[col] = b2;
        out[kHidden + col] = w;
    }
    if (blockIdx.x == 0 && rg == 1) {
        float t = 0.f;
        for (int r = r0 + (threadIdx.x & 31); r < r1; r += 32) t += dy[r];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(kAllLanes, t, o);
        if ((threadIdx.x & 31) == 0) out[2 * kHidden] = t;
    }
}

// dz = dh gelu'(z) (bf16) over row block blockIdx.y and the block's partial
// column sums at red[blockIdx.y * kBwdRedStride].
__global__ void __launch_bounds__(256) k_mlp_act_bwd(const float *__restrict__ dh, const float *__restrict__ z,
                                                     int n, int rows_per, uint16_t *dz, float *red) {
    __shared__ float r_s[8][33];
    const int col = blockIdx.x * 32 + (threadIdx.x & 31), rg = threadIdx.x >> 5;
    const int r0 = blockIdx.y * rows_per, r1 = min(n, r0 + rows_per);
    float s = 0.f;
    for (int r = r0 + rg; r < r1; r += 8) {
        const size_t i = (size_t)r * kHidden + col;
        const float v = dh[i] * gelu_grad(z[i]);
        dz[i] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
        s += v;
    }
    r_s[rg][threadIdx.x & 31] = s;
    __syncthreads();
    if (rg == 0) {
        float t = 0.f;
        for (int k = 0; k < 8; k++) t += r_s[k][threadIdx.x];
        red[(size_t)blockIdx.y * kBwdRedStride + col] = t;
    }
}

// out[j] = sum over row blocks b (in order) of red[b * kBwdRedStride + j],
// j < width, to dst[j] with dst = d0 (j < 128), d1 (j < 256), d2 (j = 256).
__global__ void k_bwd_reduce(const float *__restrict__ red, int nblocks, int width, float *d0, float *d1,
                             float *d2) {
    const int j = threadIdx.x;
    if (j >= width) return;
    float t = 0.f;
    for (int b = 0; b < nblocks; b++) t += red[(size_t)b * kBwdRedStride + j];
    if (j < kHidden) d0[j] = t;
    else if (j < 2 * kHidden) d1[j - kHidden] = t;
    else d2[0] = t;
}

// Adam with bias correction factors bc1 = 1 - b1^t, bc2 = 1 - b2^t.
__global__ void k_adam(float *w, const float *__restrict__ g, float *m, float *v, int n, int first,
                       float lr, float b1, float b2, float eps, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + first;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// ---- launch wrappers ------------------------------------------------------------
size_t rank_smem_bytes() { return sizeof(MlpSmem) + 4 * 256 * sizeof(float); }

const void *rank_kernel_ptr() { return (const void *)k_rank; }

cudaError_t rank_set_attributes() {
    cudaError_t e = cudaFuncSetAttribute(k_rank, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)rank_smem_bytes());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)rank_smem_bytes());
    return e;
}

void launch_plan_rank(const DevBatch &b, const RankArgs &a, int *counts, cudaStream_t st) {
    if (a.ntasks > 0) k_plan_rank<<<(a.ntasks + 127) / 128, 128, 0, st>>>(b, a, counts);
}

void launch_rank(const DevBatch &b, const RankArgs &a, const int *chunk_begin, const ScanOut *scan,
                 int *counter, int grid, cudaStream_t st) {
    if (b.n > 0) k_rank<<<grid, 128, rank_smem_bytes(), st>>>(b, a, chunk_begin, scan, counter);
}

void launch_select(const DevBatch &b, const SelectArgs &a, cudaStream_t st) {
    const int nt = a.task.ntasks;
    if (nt > 0) k_select<<<(nt * 32 + 127) / 128, 128, 0, st>>>(b, a);
}

void launch_audit(const DevBatch &b, const SelectArgs &a, const CandRes &r, cudaStream_t st) {
    const int nt = a.task.ntasks;
    if (nt > 0) k_audit<<<(nt * 32 + 127) / 128, 128, 0, st>>>(b, a, r);
}

void launch_collect_labels(const DevBatch &b, const RankArgs &a, const CandRes &r, float *label,
                           cudaStream_t st) {
    if (a.ntasks > 0) k_collect_labels<<<a.ntasks, 256, 0, st>>>(b, a, r, label);
}

void launch_mlp_pack(const float *blob, MlpPacked *out, cudaStream_t st) {
    k_mlp_pack<<<(kHidden * kHidden + 255) / 256, 256, 0, st>>>(blob, out);
}

void launch_mlp_forward(const MlpPacked *mlp, const float *x, int n, float *y, const MlpSave *save,
                        cudaStream_t st) {
    if (n <= 0) return;
    MlpSave sv = save ? *save : MlpSave{nullptr, nullptr, nullptr, nullptr};
    k_mlp_forward<<<(n + 63) / 64, 128, rank_smem_bytes(), st>>>(mlp, x, n, y, sv, save ? 1 : 0);
}

void launch_mlp_loss(const float *y, const float *t, int n, float lambda, float *dy, float *loss,
                     cudaStream_t st) {
    k_mlp_loss<<<1, 1024, 0, st>>>(y, t, n, lambda, dy, loss);
}

int bwd_row_blocks(int n) {
    const int b = (n + kBwdRows - 1) / kBwdRows;
    return b < 1 ? 1 : (b > kBwdBlocksMax ? kBwdBlocksMax : b);
}

void launch_mlp_head_bwd(const MlpPacked *mlp, const float *dy, const float *z2, int n, uint16_t *dz2,
                         float *red, float *grad, cudaStream_t st) {
    const int nb = bwd_row_blocks(n), rows_per = (n + nb - 1) / nb;
    k_mlp_head_bwd<<<dim3(kHidden / 32, nb), 256, 0, st>>>(mlp, dy, z2, n, rows_per, dz2, red);
    k_bwd_reduce<<<1, 2 * kHidden + 32, 0, st>>>(red, nb, 2 * kHidden + 1, grad + kBlobB2, grad + kBlobW3,
                                                 grad + kBlobB3);
}

void launch_mlp_act_bwd(const float *dh, const float *z, int n, uint16_t *dz, float *red, float *dbias,
                        cudaStream_t st) {
    const int nb = bwd_row_blocks(n), rows_per = (n + nb - 1) / nb;
    k_mlp_act_bwd<<<dim3(kHidden / 32, nb), 256, 0, st>>>(dh, z, n, rows_per, dz, red);
    k_bwd_reduce<<<1, kHidden, 0, st>>>(red, nb, kHidden, dbias, nullptr, nullptr);
}

void launch_adam(float *w, const float *g, float *m, float *v, int n, int first, float lr, float b1,
                 float b2, float eps, float bc1, float bc2, cudaStream_t st) {
    if (n > first)
        k_adam<<<(n - first + 255) / 256, 256, 0, st>>>(w, g, m, v, n, first, lr, b1, b2, eps, bc1, bc2);
}

}  // namespace ia
