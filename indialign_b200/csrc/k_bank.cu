// Seed-bank kernel: iterative distance-cutoff Kabsch refinement of many
// (seed, cutoff) items over one point set, thread per item.
//
// Restates iterative_seed_refine / evaluate_seed_bank
// (indialign_c/search.h:28-138), refine_from_rt + gapless_threading_search
// (indialign_c/threading.h:15-80) and alignment_detailed_search
// (indialign_c/align.h:15-50).  All 32 lanes of a warp refine items of the
// same point set, so every residue load from shared memory is a broadcast;
// a lane's refinement is a sequential sum over residues in the reference's
// order.  Each item writes {score, R, t}; reduce_bank then applies the
// reference's serial first-max and early-termination rules.
//
// Precision: the residue visits -- transform, distance, inlier test, raw
// moment sums and the item's TM sum -- run in FP32 (the point set is staged
// as FP64, centred on its FP64 mean and converted to FP32 in shared memory;
// the TM sum is compensated; the operation order is fixed with explicit
// fused multiply-adds, as restated by the oracle's FP32 study build); each
// Kabsch eigen-solve runs in FP64 from the FP32 moments, and reduce_bank
// rescores the task's winning item in FP64, so every reported score is an
// FP64 TM-score of the returned (R, t).  The oracle rebuilt with this
// arithmetic in its seed banks stayed within 2e-8 of the reference build's
// final TM-scores on 560 pairs.
#include "dmath.cuh"
#include "stage.cuh"
#include "pipeline.h"
#include "kernels.h"
#include "sched.cuh"

// build-time knob: minimum resident bank CTAs per SM (caps registers)
#ifndef IA_BANK_MINB
#define IA_BANK_MINB 4
#endif


namespace ia {

// ---- the bank kernel -------------------------------------------------------
struct BankSmem {
    int chunk, task;
};

// Raw moments of the selected pairs in FP32 (counts exact).
struct MomentsF {
    float sp[3], sq[3], h[9];
    int w;
    IA_DEV void clear() {
#pragma unroll
        for (int i = 0; i < 3; i++) sp[i] = sq[i] = 0.f;
#pragma unroll
        for (int i = 0; i < 9; i++) h[i] = 0.f;
        w = 0;
    }
    IA_DEV void add(float px, float py, float pz, float qx, float qy, float qz) {
        sp[0] += px; sp[1] += py; sp[2] += pz;
        sq[0] += qx; sq[1] += qy; sq[2] += qz;
        h[0] = fmaf(px, qx, h[0]); h[1] = fmaf(px, qy, h[1]); h[2] = fmaf(px, qz, h[2]);
        h[3] = fmaf(py, qx, h[3]); h[4] = fmaf(py, qy, h[4]); h[5] = fmaf(py, qz, h[5]);
        h[6] = fmaf(pz, qx, h[6]); h[7] = fmaf(pz, qy, h[7]); h[8] = fmaf(pz, qz, h[8]);
        w++;
    }
    // Kabsch in FP64 from these sums (identity below 3 pairs)
    IA_DEV void kabsch(double *R, double *t) const {
        Moments m;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            m.sp[i] = sp[i];
            m.sq[i] = sq[i];
        }
#pragma unroll
        for (int i = 0; i < 9; i++) m.h[i] = h[i];
        m.w = (double)w;
        kabsch_from_moments(m, 3.0, R, t);
    }
};

// The FP32 work runs on coordinates centred on their point set's FP64 mean
// (so the raw moments do not cancel against a large offset); the kernel's
// (R, t) live in that frame until an item is written out.  A point is a
// float4 (x, y, z, w) with w = 1 for a valid residue of the cutoff and score
// passes (V[i] != 0, or no mask) and 0 otherwise.
//
// The shared FP32 copy holds residues in pairs, so one paired FP32
// instruction (f32x2) serves two residues: pair k = residues 2k, 2k+1 is two
// float4 blocks {x_2k, x_2k+1, y_2k, y_2k+1} {z_2k, z_2k+1, w_2k, w_2k+1}; an
// odd set ends with a zero point of w = 0.
//
// Point i of a set in the centred FP32 frame: the converted shared copy, or
// converted on load from the FP64 global array (point sets too large for
// shared memory).  Both give the same floats, so a pair's results do not
// depend on which path its batch takes.
template <bool SMEM>
IA_DEV float4 point(const float4 *f, const double *d, const double *off, const uint8_t *V, int i) {
    if constexpr (SMEM) {
        const float *e = reinterpret_cast<const float *>(f) + (i >> 1) * 8 + (i & 1);
        return make_float4(e[0], e[2], e[4], e[6]);
    }
    else return make_float4((float)(d[3 * i] - off[0]), (float)(d[3 * i + 1] - off[1]),
                            (float)(d[3 * i + 2] - off[2]), (V == nullptr || V[i] != 0) ? 1.f : 0.f);
}

// Squared distance of p moved by (Rf, tf) from q, in a fixed FP32 operation
// order (the order the oracle's FP32 study build restates):
// d = ((t - q) + p_z R + p_y R) + p_x R per axis, d2 = (dx^2 + dy^2) + dz^2.
IA_DEV float dist2_f32(const float4 &p, const float4 &q, const float *Rf, const float *tf) {
    const float dx = fmaf(p.x, Rf[0], fmaf(p.y, Rf[3], fmaf(p.z, Rf[6], tf[0] - q.x)));
    const float dy = fmaf(p.x, Rf[1], fmaf(p.y, Rf[4], fmaf(p.z, Rf[7], tf[1] - q.y)));
    const float dz = fmaf(p.x, Rf[2], fmaf(p.y, Rf[5], fmaf(p.z, Rf[8], tf[2] - q.z)));
    return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
}

// A transform with every entry duplicated, the operand form of paired FP32
// instructions.
struct XformF2 {
    float2 r[9], t[3];
    IA_DEV void set(const double *R, const double *t_) {
#pragma unroll
        for (int a = 0; a < 9; a++) r[a] = make_float2((float)R[a], (float)R[a]);
#pragma unroll
        for (int a = 0; a < 3; a++) t[a] = make_float2((float)t_[a], (float)t_[a]);
    }
};

// dist2_f32 of the two residues of a staged pair (P blocks PA, PB; Q blocks
// QA, QB), element by element the same operations in the same order, two
// residues per paired instruction (t - q is the single rounding of
// q * (-1) + t).
IA_DEV float2 dist2_pair(const float4 &PA, const float4 &PB, const float4 &QA, const float4 &QB,
                         const XformF2 &X) {
    const float2 px = make_float2(PA.x, PA.y), py = make_float2(PA.z, PA.w), pz = make_float2(PB.x, PB.y);
    const float2 m1 = make_float2(-1.f, -1.f);
    float2 ax = __ffma2_rn(make_float2(QA.x, QA.y), m1, X.t[0]);
    float2 ay = __ffma2_rn(make_float2(QA.z, QA.w), m1, X.t[1]);
    float2 az = __ffma2_rn(make_float2(QB.x, QB.y), m1, X.t[2]);
    ax = __ffma2_rn(px, X.r[0], __ffma2_rn(py, X.r[3], __ffma2_rn(pz, X.r[6], ax)));
    ay = __ffma2_rn(px, X.r[1], __ffma2_rn(py, X.r[4], __ffma2_rn(pz, X.r[7], ay)));
    az = __ffma2_rn(px, X.r[2], __ffma2_rn(py, X.r[5], __ffma2_rn(pz, X.r[8], az)));
    return __ffma2_rn(az, az, __ffma2_rn(ay, ay, __fmul2_rn(ax, ax)));
}

// CTA-wide FP64 mean of the finite values of n points, per axis, into
// out[3] (shared); red holds 6 doubles per warp.  The summation order
// depends only on n, so both kernel paths get the same mean.  Non-finite
// coordinates are left out: the mean is only the frame the FP32 work runs
// in, and one Inf must not turn every centred point into NaN (the
// reference's FP64 seeds that avoid such a residue still score finitely).
// With all values finite this is the plain mean.
IA_DEV void points_mean(const double *src, int n, double *out, double *red) {
    double a[3] = {0.0, 0.0, 0.0}, c[3] = {0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += kBankChunk) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double x = src[3 * i + d];
            if (isfinite(x)) {
                a[d] += x;
                c[d] += 1.0;
            }
        }
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        a[d] = warp_sum(a[d]);
        c[d] = warp_sum(c[d]);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            red[6 * w + d] = a[d];
            red[6 * w + 3 + d] = c[d];
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0.0, m = 0.0;
        for (int k = 0; k < kBankChunk / 32; k++) {
            v += red[6 * k + threadIdx.x];
            m += red[6 * k + 3 + threadIdx.x];
        }
        out[threadIdx.x] = m > 0.0 ? v / m : 0.0;
    }
    __syncthreads();
}

// CTA-wide in-place conversion of n staged FP64 points (at src, inside the
// region that starts at dst) to centred FP32 residue pairs at dst (layout
// above), w from the validity bytes V (null: all valid).  Round r reads
// points [128r, 128r+128) before any thread writes them; its writes end at
// byte 16*128(r+1) + 16, below the first byte (24*128(r+1)) that a later
// round reads; the pairs of n points take 32*ceil(n/2) <= 16n + 16 bytes,
// inside the 24n + 32 bytes of the staged region.
IA_DEV void points_to_f32(const double *src, float4 *dst4, int n, const double *off, const uint8_t *V) {
    float *dst = reinterpret_cast<float *>(dst4);
    for (int base = 0; base < n; base += kBankChunk) {
        const int i = base + (int)threadIdx.x;
        double x = 0.0, y = 0.0, z = 0.0;
        float w = 0.f;
        if (i < n) {
            x = src[3 * i] - off[0];
            y = src[3 * i + 1] - off[1];
            z = src[3 * i + 2] - off[2];
            w = (V == nullptr || V[i] != 0) ? 1.f : 0.f;
        }
        __syncthreads();
        if (i < n || (i == n && (n & 1))) {  // residue i, or the zero point after an odd set
            float *e = dst + (i >> 1) * 8 + (i & 1);
            e[0] = (float)x;
            e[2] = (float)y;
            e[4] = (float)z;
            e[6] = w;
        }
    }
    __syncthreads();
}

template <bool SMEM>
__global__ void __launch_bounds__(kBankChunk, IA_BANK_MINB)
k_bank(const BankTask *__restrict__ tasks, const int *__restrict__ chunk_begin,
       int ntasks, const ScanOut *__restrict__ scan, int *counter,
       double *__restrict__ item_res, int *err, int nmax, unsigned long long *ctr) {
    extern __shared__ __align__(16) char smem[];
    __shared__ BankSmem ctl;
    __shared__ uint64_t bar;
    __shared__ double oP[3], oQ[3], red[6 * (kBankChunk / 32)];  // point-set means
    __shared__ int s_next;  // next group of 32 items of the chunk
    // layout: P[nmax*3] Q[nmax*3] (each +16 B lead room), V, PV, NV bytes
    // room for a 15-byte lead and the rounded-up tail of a bulk copy
    const uint32_t coord_bytes = ((uint32_t)nmax * 24u + 47u) & ~15u;
    const uint32_t mask_bytes = ((uint32_t)nmax + 47u) & ~15u;
    char *sP = smem, *sQ = smem + coord_bytes, *sV = sQ + coord_bytes;
    char *sPV = sV + mask_bytes, *sNV = sPV + mask_bytes;
    uint32_t phase = 0;
    if (threadIdx.x == 0) mbar_init(&bar);
    __syncthreads();
    const int total = scan->total_chunks;
    int staged = -1;
    const float4 *Pf = nullptr, *Qf = nullptr;  // shared FP32 copies (SMEM)
    const double *Pd = nullptr, *Qd = nullptr;  // global FP64 arrays (!SMEM)
    const uint8_t *V = nullptr, *PV = nullptr, *NV = nullptr;
    for (;;) {
        if (threadIdx.x == 0) {
            int c = atomicAdd(counter, 1);
            int t = -1;
            if (c < total) {
                int lo = 0, hi = ntasks;  // first begin > c
                while (lo < hi) {
                    int mid = (lo + hi) >> 1;
                    if (chunk_begin[mid] <= c) lo = mid + 1; else hi = mid;
                }
                t = lo - 1;
                s_next = (c - chunk_begin[t]) * tasks[t].chunk;
            }
            ctl.chunk = c;
            ctl.task = t;
        }
        __syncthreads();
        const int c = ctl.chunk, ti = ctl.task;
        if (c >= total || ti < 0) break;
        const BankTask &T = tasks[ti];
        const int n = T.n;
        if (ti != staged) {
            if (SMEM) {
                Copy cp[5];
                char *dst[5];
                int nc = 0;
                cp[nc] = plan_copy(T.P, (uint32_t)n * 24u); dst[nc++] = sP;
                cp[nc] = plan_copy(T.Q, (uint32_t)n * 24u); dst[nc++] = sQ;
                if (T.V) { cp[nc] = plan_copy(T.V, (uint32_t)n); dst[nc++] = sV; }
                if (T.PV) { cp[nc] = plan_copy(T.PV, (uint32_t)n); dst[nc++] = sPV; }
                if (T.NV) { cp[nc] = plan_copy(T.NV, (uint32_t)n); dst[nc++] = sNV; }
                stage_copies(cp, dst, nc, &bar, phase, err);
                const double *dP = reinterpret_cast<const double *>(sP + cp[0].lead);
                const double *dQ = reinterpret_cast<const double *>(sQ + cp[1].lead);
                points_mean(dP, n, oP, red);
                points_mean(dQ, n, oQ, red);
                int k = 2;
                V = T.V ? reinterpret_cast<const uint8_t *>(sV + cp[k++].lead) : nullptr;
                points_to_f32(dP, reinterpret_cast<float4 *>(sP), n, oP, V);
                points_to_f32(dQ, reinterpret_cast<float4 *>(sQ), n, oQ, nullptr);
                Pf = reinterpret_cast<const float4 *>(sP);
                Qf = reinterpret_cast<const float4 *>(sQ);
                PV = T.PV ? reinterpret_cast<const uint8_t *>(sPV + cp[k++].lead) : nullptr;
                NV = T.NV ? reinterpret_cast<const uint8_t *>(sNV + cp[k++].lead) : nullptr;
            } else {
                Pd = T.P; Qd = T.Q; V = T.V; PV = T.PV; NV = T.NV;
                points_mean(Pd, n, oP, red);
                points_mean(Qd, n, oQ, red);
            }
            staged = ti;
        }
        // the chunk's items [cb, ce) go to the warps 32 at a time, so a warp
        // whose items converged early takes the next group instead of
        // waiting at the chunk's barrier for the others
        const int cb = (c - chunk_begin[ti]) * T.chunk;
        const int ce = min(cb + T.chunk, T.n_items);
        const int lane = threadIdx.x & 31;
        for (;;) {
        int gi = 0;
        if (lane == 0) gi = atomicAdd(&s_next, 32);
        gi = __shfl_sync(0xffffffffu, gi, 0);
        if (gi >= ce) break;
        const int pi = gi + lane;  // processing order within the task
        const bool active = pi < ce;
        const int C = T.C > 0 ? T.C : 1;
        // item (seed k, cutoff ci) and its record slot li = k*C + ci: seed
        // major (the slot order), or cutoff major (a warp refines one cutoff
        // over 32 seeds; measured 1.38x faster than seed major on the
        // learned16384 step, because a warp iterates until its slowest item
        // converges and the iteration counts of one cutoff are far more alike
        // than those of one seed's cutoffs)
        int sk = 0, ci = 0;
        if (active) {
            if (T.cutoff_major) {
                const int K = T.n_items / C;
                sk = pi % K;
                ci = pi / K;
            } else {
                sk = pi / C;
                ci = pi % C;
            }
        }
        const int li = sk * C + ci;
        const int k = active ? (T.slist ? T.slist[sk] : sk) : 0;
        const double cut = T.cut[ci];
        const float cut2 = (float)(cut * cut);
        double R[9], t[3];
        MomentsF m;
        m.clear();
        bool skip = false;
        // ---- initial Kabsch on the seed ----
        if (T.mode == SEED_SHIFT) {
            const int o = offset_at(T.shift_lo, T.shift_stride, k);
            for (int i = 0; i < n; i++) {
                int j = i - o;
                bool sel = active && j >= 0 && j < n && PV[i] != 0 && NV[j] != 0;
                if (sel) {
                    const float4 pp = point<SMEM>(Pf, Pd, oP, V, i), qq = point<SMEM>(Qf, Qd, oQ, nullptr, j);
                    m.add(pp.x, pp.y, pp.z, qq.x, qq.y, qq.z);
                }
            }
            skip = m.w < T.shift_min;
        } else {
            int s = 0, len = 0, bitrow = -1;
            if (active) {
                if (T.mode == SEED_TABLE) {
                    int2 e = T.table[k];
                    if (e.x >= 0) { s = e.x; len = e.y; }
                    else { bitrow = -1 - e.x; s = 0; len = n; }
                } else {
                    arith_seed(n, T.ms, k, s, len);
                }
            }
            const uint32_t *brow = bitrow >= 0 ? T.bits + (size_t)bitrow * T.words : nullptr;
            for (int i = 0; i < n; i++) {
                uint8_t v = V ? V[i] : (uint8_t)1;
                bool sel;
                if (brow) sel = ((brow[i >> 5] >> (i & 31)) & 1u) && (v & 1u);  // 1 & valid
                else sel = i >= s && i < s + len && v != 0;                    // valid & valid
                if (active && sel) {
                    const float4 pp = point<SMEM>(Pf, Pd, oP, V, i), qq = point<SMEM>(Qf, Qd, oQ, nullptr, i);
                    m.add(pp.x, pp.y, pp.z, qq.x, qq.y, qq.z);
                }
            }
        }
        if (active && !skip) m.kabsch(R, t);
        else set_identity(R, t);
        // ---- cutoff iterations: select d2 <= cut^2, Kabsch, stop on a
        // repeated count ----
        bool running = active && !skip && T.max_iter > 0;
        int prev = -1, iter = 0;
        while (__any_sync(0xffffffffu, running)) {
            float Rf[9], tf[3];
#pragma unroll
            for (int a = 0; a < 9; a++) Rf[a] = (float)R[a];
#pragma unroll
            for (int a = 0; a < 3; a++) tf[a] = (float)t[a];
            m.clear();
            int cnt = 0;
            if constexpr (SMEM) {
                // two residues per step: distances by paired instructions,
                // the accumulate per residue in residue order
                XformF2 X;
                X.set(R, t);
                for (int k2 = 0; k2 < (n + 1) >> 1; k2++) {
                    const float4 PA = Pf[2 * k2], PB = Pf[2 * k2 + 1], QA = Qf[2 * k2], QB = Qf[2 * k2 + 1];
                    const float2 d2 = dist2_pair(PA, PB, QA, QB, X);
                    if (running && PB.z != 0.f && d2.x <= cut2) {
                        m.add(PA.x, PA.z, PB.x, QA.x, QA.z, QB.x);
                        cnt++;
                    }
                    if (running && PB.w != 0.f && d2.y <= cut2) {
                        m.add(PA.y, PA.w, PB.y, QA.y, QA.w, QB.y);
                        cnt++;
                    }
                }
            } else {
                for (int i = 0; i < n; i++) {
                    const float4 pp = point<SMEM>(Pf, Pd, oP, V, i), qq = point<SMEM>(Qf, Qd, oQ, nullptr, i);
                    if (running && pp.w != 0.f && dist2_f32(pp, qq, Rf, tf) <= cut2) {
                        m.add(pp.x, pp.y, pp.z, qq.x, qq.y, qq.z);
                        cnt++;
                    }
                }
            }
            if (running) {
                if (cnt >= 3) m.kabsch(R, t);
                ++iter;
                if (cnt == prev || iter >= T.max_iter) running = false;
                prev = cnt;
            }
        }
        // ---- score: sum 1/(1+d2/d0^2) over the set (optionally d2 <= sd8^2)
        // divided by max(Lnorm, 1) (indialign_c/core.h:134-166), FP32 terms
        // with a compensated sum; reduce_bank rescores the winner in FP64 ----
        double score = kNegInf;
        if (active && !skip) {
            // term 1 / fma(d2, 1/d0^2, 1): a correctly rounded reciprocal of
            // one fused operation instead of two divisions
            const float inv_d0sq = (float)(1.0 / fmax(T.d0 * T.d0, 1e-12)), sd8sq = (float)(T.sd8 * T.sd8);
            float Rf[9], tf[3];
#pragma unroll
            for (int a = 0; a < 9; a++) Rf[a] = (float)R[a];
#pragma unroll
            for (int a = 0; a < 3; a++) tf[a] = (float)t[a];
            float sum = 0.f, comp = 0.f;
            auto add_term = [&](float d2) {
                if (!T.use_d8 || d2 <= sd8sq) {
                    const float y = __frcp_rn(fmaf(d2, inv_d0sq, 1.0f)) - comp;
                    const float s2 = sum + y;
                    comp = (s2 - sum) - y;
                    sum = s2;
                }
            };
            if constexpr (SMEM) {
                XformF2 X;
                X.set(R, t);
                for (int k2 = 0; k2 < (n + 1) >> 1; k2++) {
                    const float4 PA = Pf[2 * k2], PB = Pf[2 * k2 + 1], QA = Qf[2 * k2], QB = Qf[2 * k2 + 1];
                    const float2 d2 = dist2_pair(PA, PB, QA, QB, X);
                    if (PB.z != 0.f) add_term(d2.x);
                    if (PB.w != 0.f) add_term(d2.y);
                }
            } else {
                for (int i = 0; i < n; i++) {
                    const float4 pp = point<SMEM>(Pf, Pd, oP, V, i);
                    if (pp.w == 0.f) continue;
                    add_term(dist2_f32(pp, point<SMEM>(Qf, Qd, oQ, nullptr, i), Rf, tf));
                }
            }
            score = (double)sum / fmax(T.lnorm, 1.0);
        }
        {
            // residue visits: seed pass + `iter` cutoff passes + score pass
            unsigned long long visits = active && !skip ? (unsigned long long)(iter + 2) * n : 0ull;
            unsigned long long items = active ? 1ull : 0ull;
#pragma unroll
            for (int o2 = 16; o2 > 0; o2 >>= 1) {
                visits += __shfl_xor_sync(0xffffffffu, visits, o2);
                items += __shfl_xor_sync(0xffffffffu, items, o2);
            }
            if ((threadIdx.x & 31) == 0 && items) {
                atomicAdd(ctr + CTR_BANK_RES, visits);
                atomicAdd(ctr + CTR_BANK_ITEMS, items);
            }
        }
        if (active) {
            // back to the caller's frame: t = t_c + oQ - sum_k oP_k R[3k+d]
            double *o = item_res + (size_t)(T.item_base + li) * kRec;
            o[0] = score;
#pragma unroll
            for (int a = 0; a < 9; a++) o[1 + a] = R[a];
#pragma unroll
            for (int a = 0; a < 3; a++) o[10 + a] = t[a] + oQ[a] - (oP[0] * R[a] + oP[1] * R[3 + a] + oP[2] * R[6 + a]);
        }
        }  // next group of 32 items
        __syncthreads();
    }
}

// ---- first-max reduction of a task's items ---------------------------------
// Serial semantics of evaluate_seed_bank (indialign_c/search.h:62-98): seeds
// outer, cutoffs inner, a candidate replaces the best only if strictly
// greater, and before each seed the loop stops once best >= early_term.  The
// last seed processed is therefore k* = the first seed holding an item
// >= early_term; every earlier item is below early_term, so the result is the
// first maximum over the items of seeds 0..k*.
__global__ void k_reduce_bank(const BankTask *__restrict__ tasks, int ntasks,
                              const double *__restrict__ item_res,
                              PairState *__restrict__ state) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= ntasks) return;
    const BankTask &T = tasks[w];
    if (T.n_items <= 0) return;
    const int C = T.C > 0 ? T.C : 1;
    const double *base = item_res + (size_t)T.item_base * kRec;
    int end = T.n_items;
    if (T.early_term < 1e30) {
        int kst = 0x7fffffff;
        for (int i = lane; i < T.n_items; i += 32)
            if (base[(size_t)i * kRec] >= T.early_term) kst = min(kst, i / C);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) kst = min(kst, __shfl_xor_sync(0xffffffffu, kst, o));
        if (kst != 0x7fffffff) end = min(end, (kst + 1) * C);
    }
    double bs = kScoreInit;
    int bi = -1;
    for (int i = lane; i < end; i += 32) {
        double s = base[(size_t)i * kRec];
        if (s > bs) { bs = s; bi = i; }  // lane-local: ascending i, strict >
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double s2 = __shfl_xor_sync(0xffffffffu, bs, o);
        int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        bool take = (s2 > bs) || (s2 == bs && i2 >= 0 && (bi < 0 || i2 < bi));
        if (take) { bs = s2; bi = i2; }
    }
    // the winner's score in FP64 over the task's own point set (the items
    // were scored in FP32): the same formula as k_bank's score pass
    double score = kScoreInit;
    if (bi >= 0) {
        const double *rec = base + (size_t)bi * kRec;
        double R[9], t[3];
#pragma unroll
        for (int a = 0; a < 9; a++) R[a] = rec[1 + a];
#pragma unroll
        for (int a = 0; a < 3; a++) t[a] = rec[10 + a];
        const double d0sq = fmax(T.d0 * T.d0, 1e-12), sd8sq = T.sd8 * T.sd8;
        double sum = 0.0;
        for (int i = lane; i < T.n; i += 32) {
            if (T.V && T.V[i] == 0) continue;
            const double d2 = dist2(R, t, T.P[3 * i], T.P[3 * i + 1], T.P[3 * i + 2], T.Q[3 * i], T.Q[3 * i + 1],
                                    T.Q[3 * i + 2]);
            if (!T.use_d8 || d2 <= sd8sq) sum += 1.0 / (1.0 + d2 / d0sq);
        }
        score = warp_sum(sum) / fmax(T.lnorm, 1.0);
    }
    double *out = T.out_rec >= 0 ? state[T.pair].rec[T.out_rec] : T.out;
    if (lane < kRec) {
        double v;
        if (bi >= 0) v = lane == 0 ? score : base[(size_t)bi * kRec + lane];
        else v = lane == 0 ? kScoreInit : ((lane == 1 || lane == 5 || lane == 9) ? 1.0 : 0.0);
        out[lane] = v;
    }
}

// ---- launch wrappers -------------------------------------------------------
size_t bank_smem_bytes(int nmax) {
    size_t coord = ((size_t)nmax * 24 + 47) & ~size_t(15);
    size_t mask = ((size_t)nmax + 47) & ~size_t(15);
    return 2 * coord + 3 * mask;
}

void launch_bank(const BankTask *tasks, const int *chunk_begin, int ntasks,
                 const ScanOut *scan, int *counter, double *item_res, int *err,
                 int nmax, int grid, unsigned long long *ctr, cudaStream_t st) {
    size_t sm = bank_smem_bytes(nmax);
    if (sm <= kBankSmemMax) {
        k_bank<true><<<grid, kBankChunk, sm, st>>>(tasks, chunk_begin, ntasks, scan, counter,
                                                   item_res, err, nmax, ctr);
    } else {
        k_bank<false><<<grid, kBankChunk, 0, st>>>(tasks, chunk_begin, ntasks, scan, counter,
                                                   item_res, err, nmax, ctr);
    }
}

void launch_reduce_bank(const BankTask *tasks, int ntasks, const double *item_res,
                        PairState *state, cudaStream_t st) {
    if (ntasks <= 0) return;
    int threads = 256, blocks = (ntasks * 32 + threads - 1) / threads;
    k_reduce_bank<<<blocks, threads, 0, st>>>(tasks, ntasks, item_res, state);
}

const void *bank_kernel_ptr(bool smem) {
    return smem ? (const void *)k_bank<true> : (const void *)k_bank<false>;
}

cudaError_t bank_set_attributes() {
    cudaError_t e = cudaFuncSetAttribute(k_bank<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kBankSmemMax);
    return e;
}

}  // namespace ia
