// NW chains: score matrix + Needleman-Wunsch + traceback + Kabsch + the
// detailed seed search on the alignment, one warp per chain.
//
// Restates nw_dp / nw_traceback (indialign_c/nw.h:10-68), dp_refine_chunk
// (indialign_c/align.h:54-145) and the score matrices of ss_nw_align /
// evaluate_ss_seeds (indialign_c/ss.h:56-164).
//
// NW layout: the warp sweeps horizontal stripes of 32 rows; lane l owns row
// s0+l+1 and computes column j at step j+l-1, so each step is one
// anti-diagonal of the stripe.  H[i-1][j] arrives from lane l-1 by a warp
// shuffle (lane 0 reads the stripe's top boundary row from memory, written
// by lane 31 of the previous stripe), H[i][j-1] is the lane's own previous
// value.  The "reached diagonally" bit that gates the gap penalty travels in
// the sign bit of H (H >= 0 always; -0.0 encodes a diagonal zero).  Score
// entries are computed on the fly from the transformed pred row held in
// registers and the native column in shared memory, never stored.  Trace
// directions (2 bits/cell) go to a per-warp global scratch block in a
// stripe-major layout: for every 16 steps the warp's 64 rows store one
// contiguous 256-byte line (one 8-byte store per lane), so the stores are
// full-sector writes; the traceback walks 32-row tiles held in registers
// (coalesced loads, shuffles inside).
#include <type_traits>

#include "dmath.cuh"
#include "stage.cuh"
#include "pipeline.h"
#include "kernels.h"
#include "sched.cuh"

namespace ia {

constexpr unsigned kFull = 0xffffffffu;

// build-time tuning knobs: minimum resident CTAs per SM for k_chain (caps
// registers; 5 -> 96 registers measured best with the NW fill out of line,
// 8% faster than 4 -> 128, while 6 and 8 were slower) and the NW step-loop
// unroll factor (1 measured best: the rare stripe branches make unrolled
// copies larger without shortening the dependency chain; a 16-step unrolled
// block without those branches measured 2x slower)
#ifndef IA_CHAIN_MINB
#define IA_CHAIN_MINB 5
#endif
#ifndef IA_NW_UNROLL
#define IA_NW_UNROLL 1
#endif
constexpr int kNwUnroll = IA_NW_UNROLL;

// Aligned pair k (forward order) from the reversed traceback list.
IA_DEV void al_get(const uint32_t *al, int na, int k, int &pi, int &ni) {
    uint32_t e = al[na - 1 - k];
    pi = (int)(e >> 16);
    ni = (int)(e & 0xffffu);
}

// Value type of the NW fill of the search's score matrices (dp_refine and
// the SS + distance NW): FP32 by default (1), FP64 like the reference (0).
// Measured on the CPU (the oracle rebuilt with FP32 score entries, and with
// FP32 entries and DP values, against the reference build on 240 pairs of
// the 4096-pair shape and 96 hard pairs): every final TM-score within
// 5.6e-16 of the reference's, for either choice.  The SS-identity
// NW (entries 0/1, gap -1) runs in FP32, where its integer-valued DP is
// exact; the explicit-matrix NW entry stays FP64 (bit-exact with the
// reference's nw_dp on the same matrix).
#ifndef IA_CHAIN_DP32
#define IA_CHAIN_DP32 1
#endif
using ChainDP = std::conditional_t<IA_CHAIN_DP32 != 0, float, double>;

struct NWParams {
    int plen, nlen;
    int smode;
    double gap;
    double inv_d0sq;  // 1/d0^2 of the score matrix
    double cut2;      // SMAT_DP: score only if d2 <= cut2
    const uint8_t *Lp, *Ln;  // SS labels (compact order)
    const double *smat;      // SMAT_EXPLICIT: plen x nlen row-major
    const float4 *Qf;        // native column as FP32 (shared memory), or null
};

// One score-matrix entry (indialign_c/align.h:86-98; ss.h:69-72, 118-131)
// in FP32: the moved pred point (FP64 transform, rounded to FP32) minus the
// native point rounded to FP32, FP32 d2 and cutoff test, and the term
// 1/(1 + d2 * (1/d0^2)) with a correctly rounded FP32 reciprocal; the SS
// bonus 0.5 is added in the DP's type.  A NaN distance gives 0 in the DP
// mode (the cutoff test fails) and NaN in the SS4 mode, an infinite one 0,
// as in the reference's FP64 arithmetic.
template <int SMODE, typename T>
IA_DEV T smat_entry(float inv_d0sq, float cut2, float mx, float my, float mz, uint8_t lp, float qx,
                    float qy, float qz, uint8_t ln) {
    if (SMODE == SMAT_SS2) return (lp == ln) ? T(1) : T(0);
    const float dx = mx - qx, dy = my - qy, dz = mz - qz;
    const float d2 = dx * dx + dy * dy + dz * dz;
    const float r = __frcp_rn(1.0f + d2 * inv_d0sq);
    if (SMODE == SMAT_DP) return d2 <= cut2 ? T(r) : T(0);
    return (lp == ln) ? T(r) + T(0.5) : T(r);
}

// One NW cell (indialign_c/nw.h:20-35).  With a gap penalty the "reached
// diagonally" bit of a cell travels in the sign of its H (H >= 0; -0 is a
// diagonal zero) and a gap move out of a diagonal cell pays the penalty;
// without one the bit is irrelevant and H is kept plain.  Ties prefer diag,
// then left, then up.  Selects only, so a step is one basic block.
// MAXF: the matrix holds no NaN and no -0 (the distance-score mode: entries
// are 1/(1 + d2/d0^2) or +0, sums of them start at +0), so the choice can be
// written with two max operations: diag wins iff diag >= max(left, up), and
// H = max(diag, max(left, up)) equals the selected value (equal candidates
// are the same number).
template <bool GAPZ, typename T, bool MAXF = false>
IA_DEV T nw_cell(T diag_src, T sc, T up_enc, T left_enc, T gap, uint32_t &dir) {
    const T diag = diag_src + sc;
    if (GAPZ && MAXF) {
        const T m = fmax(left_enc, up_enc);
        dir = diag >= m ? 0u : (left_enc >= up_enc ? 2u : 1u);
        return fmax(diag, m);
    }
    T up, left;
    if (GAPZ) {
        up = up_enc;
        left = left_enc;
    } else {
        up = fabs(up_enc) + (signbit(up_enc) ? gap : T(0));
        left = fabs(left_enc) + (signbit(left_enc) ? gap : T(0));
    }
    const bool is_diag = diag >= up && diag >= left;
    const bool l_ge_u = left >= up;
    dir = is_diag ? 0u : (l_ge_u ? 2u : 1u);
    const T nh = is_diag ? diag : (l_ge_u ? left : up);
    return (GAPZ || !is_diag) ? nh : -nh;
}

// Plain value of an encoded H.
template <bool GAPZ, typename T>
IA_DEV T hval(T h) { return GAPZ ? h : fabs(h); }

// Native point jc of the score matrix as FP32: the staged shared copy, or the
// FP64 global array rounded on load.
IA_DEV float4 native_f32(const NWParams &pr, const Pts &x, int jc) {
    if (pr.Qf) return pr.Qf[jc];
    const double *q = x.Q + 3 * jc;
    return make_float4((float)q[0], (float)q[1], (float)q[2], 0.f);
}

// Trace layout: cell (i, j) of stripe k = (i-1)/64, row ri = (i-1)%64 of it
// (lane ri/2, row ri%2 of the lane) is computed at step t = base(i) + j - 1
// with base(i) = k*P + ri.  Its 2 direction bits sit at bit 2*(t%16) of the
// word at ((k*G + g) * 64 + ri), g = t/16 - (k*P)/16 the step word within
// the stripe, G = (P + 127) / 16 words per stripe (a lane stays in stripe k
// for steps below (k+1)*P + 64, so g < G).  Every lane fills and stores its
// two rows' words on the same steps, at adjacent addresses.
IA_DEV int trace_base(int i, int P) { return ((i - 1) >> 6) * P + ((i - 1) & 63); }
IA_DEV int trace_G(int P) { return (P + 127) / 16; }
// Word of row i (1-based) whose row-relative index is w (w = t/16 -
// base(i)/16), as an offset from the trace block.
IA_DEV size_t trace_word(int i, int w, int P, int G) {
    const int k = (i - 1) >> 6, ri = (i - 1) & 63;
    const int g = w + ((k * P + ri) >> 4) - ((k * P) >> 4);
    return ((size_t)k * G + g) * 64 + ri;
}

// Fill the trace of the NW DP for (R,t) and return the aligned pair count;
// the pairs are written (reversed) to al.
//
// Each lane owns two consecutive rows of a 64-row stripe; row r of lane l
// computes column j at step k*P + 2l + r + j - 1 for stripe k, with period
// P = max(nlen+1, 64).  Row 1 trails row 0 by one step inside the lane, lane
// l trails lane l-1 by two steps, and a lane moves on to its rows of the
// next stripe as soon as it finishes the current one (the top row of stripe
// k+1 reads the boundary row that lane 31 wrote for stripe k at least one
// step earlier, since P >= 64).  Per step a lane computes two independent
// cells with one shuffle and one shared-memory column load.  Cells outside
// the matrix are computed on clamped indices and never read by a valid one
// (a row's state is reset when it enters a stripe, its neighbours only read
// its in-range cells, and row 1's column-0 cell, which column 1 reads as its
// left neighbour, is replaced by the boundary +0), so the step has no
// per-cell branches.
// Out of line: inside the chain kernel (register-capped) an inlined fill
// shares the register budget with the caller's live state and spilled inside
// its step loop (measured: ~4 local loads per step); as a call it has the
// whole budget and no spills, and the caller's state is saved once per
// alignment.
#define IA_NW_ATTR __device__ __noinline__
template <int SMODE, bool GAPZ, typename T>
IA_NW_ATTR int nw_align_t(const Pts &x, const NWParams &pr, const double *R, const double *t,
                          double *bH_, uint32_t *trace, uint32_t *al, unsigned long long *ctr) {
    const int lane = threadIdx.x & 31;
    const int plen = pr.plen, nlen = pr.nlen;
    if (lane == 0) atomicAdd(ctr + CTR_NW_CELLS, (unsigned long long)plen * (unsigned long long)nlen);
    const long long clk0 = clock64();
    const int P = max(nlen + 1, 64);
    const int G = trace_G(P);
    const int S = (plen + 63) >> 6;  // stripes
    const T gap = (T)pr.gap;
    const float inv_d0sq = (float)pr.inv_d0sq, cut2 = (float)pr.cut2;
    T *bH = reinterpret_cast<T *>(bH_);  // stripe boundary row (nlen + 1 values)
    for (int j = lane; j <= nlen; j += 32) bH[j] = T(0);
    __syncwarp();
    int k = 0, j0 = 1 - 2 * lane;  // stripe and row-0 column of this lane
    int i0 = 2 * lane + 1;         // 1-based row of row 0
    float m0x = 0, m0y = 0, m0z = 0, m1x = 0, m1y = 0, m1z = 0;
    uint8_t l0 = 0, l1 = 0, ln1 = 0;
    T h0 = 0, h1 = 0, h0prev = 0, up0prev = 0;
    float q1x = 0, q1y = 0, q1z = 0;  // column of row 1 (previous step's row-0 column)
    // direction bits enter at the top and move down 2 bits a step, so after
    // the word's 16th step the bits of its step t sit at 2*(t%16); a word
    // stored after m < 16 of its steps is shifted down by 32 - 2m
    uint32_t acc0 = 0, acc1 = 0;
    bool r0ok = false, r1ok = false;
    bool st31 = false;  // lane 31 writes the stripe's boundary row
    bool ld0 = false;   // lane 0 reads the previous stripe's boundary row
    // this lane's two rows in the current stripe's block: word g of them at
    // blk[g * 64 + 2 * lane], blk[g * 64 + 2 * lane + 1]; g0 = (k*P)/16.
    // Only lanes with a row inside the matrix store (a short window leaves
    // most of its stripe's lanes without one)
    uint2 *blk = reinterpret_cast<uint2 *>(trace) + lane;
    int g0 = 0;
    const int last_lane = ((plen - 1) & 63) >> 1;
    const int total_steps = (S - 1) * P + 2 * last_lane + 1 + nlen + 1;
#pragma unroll kNwUnroll
    for (int step = 0; step < total_steps; step++) {
        T up0 = __shfl_up_sync(kFull, h1, 1);
        if (j0 > P) {  // next stripe (rare): flush the finished rows' last words
            const int w = (step - 1) >> 4;
            if (((step - 1) & 15) != 15 && r0ok) {  // else stored (and cleared) last step
                const int sh = 30 - 2 * ((step - 1) & 15);
                blk[(size_t)(w - g0) * 32] = make_uint2(acc0 >> sh, acc1 >> sh);
            }
            j0 -= P;
            k++;
            i0 += 64;
            blk = reinterpret_cast<uint2 *>(trace + (size_t)k * G * 64) + lane;
            g0 = (k * P) >> 4;
        }
        if (j0 == 1) {  // entering a stripe (rare): set up its two rows
            h0 = h1 = h0prev = up0prev = T(0);
            acc0 = acc1 = 0;
            r0ok = k < S && i0 <= plen;
            r1ok = k < S && i0 + 1 <= plen;
            st31 = lane == 31 && k + 1 < S && r1ok;
            ld0 = k > 0 && r0ok;
            const int a0 = min(i0, plen) - 1, a1 = min(i0 + 1, plen) - 1;
            const double *p0 = x.P + 3 * a0, *p1 = x.P + 3 * a1;
            if (SMODE != SMAT_SS2 && SMODE != SMAT_EXPLICIT) {
                double ax, ay, az, bx, by, bz;
                xform(R, t, p0[0], p0[1], p0[2], ax, ay, az);
                xform(R, t, p1[0], p1[1], p1[2], bx, by, bz);
                m0x = (float)ax; m0y = (float)ay; m0z = (float)az;
                m1x = (float)bx; m1y = (float)by; m1z = (float)bz;
            }
            if (SMODE == SMAT_SS2 || SMODE == SMAT_SS4) {
                l0 = pr.Lp[a0];
                l1 = pr.Lp[a1];
            }
        }
        // 0-based column; a cell outside the matrix (j0 < 1 or > nlen) is
        // computed on column nlen-1 and never read by a valid one (row 1's
        // column-0 cell is replaced by the boundary below)
        const int jc = (int)min((unsigned)(j0 - 1), (unsigned)(nlen - 1));
        float q0x = 0, q0y = 0, q0z = 0;
        if (SMODE == SMAT_DP || SMODE == SMAT_SS4) {
            const float4 q = native_f32(pr, x, jc);
            q0x = q.x; q0y = q.y; q0z = q.z;
        }
        const uint8_t ln0 = (SMODE == SMAT_SS2 || SMODE == SMAT_SS4) ? pr.Ln[jc] : (uint8_t)0;
        if (lane == 0) up0 = (ld0 && (unsigned)(j0 - 1) < (unsigned)nlen) ? bH[j0] : T(0);
        uint32_t d0, d1;
        T sc0, sc1;
        if (SMODE == SMAT_EXPLICIT) {
            const int a0 = min(i0, plen) - 1, a1 = min(i0 + 1, plen) - 1;
            const int jc1 = (int)min((unsigned)(j0 - 2), (unsigned)(nlen - 1));
            sc0 = (T)pr.smat[(size_t)a0 * nlen + jc];
            sc1 = (T)pr.smat[(size_t)a1 * nlen + jc1];
        } else {
            sc1 = smat_entry<SMODE, T>(inv_d0sq, cut2, m1x, m1y, m1z, l1, q1x, q1y, q1z, ln1);
            sc0 = smat_entry<SMODE, T>(inv_d0sq, cut2, m0x, m0y, m0z, l0, q0x, q0y, q0z, ln0);
        }
        const T n1 = nw_cell<GAPZ, T, SMODE == SMAT_DP>(h0prev, sc1, h0, h1, gap, d1);
        const T n0 = nw_cell<GAPZ, T, SMODE == SMAT_DP>(up0prev, sc0, up0, h0, gap, d0);
        acc0 = __funnelshift_r(acc0, d0, 2);
        acc1 = __funnelshift_r(acc1, d1, 2);
        if (st31 && (unsigned)(j0 - 2) < (unsigned)nlen) bH[j0 - 1] = n1;
        if ((step & 15) == 15) {  // uniform: the warp stores one 256-byte line
            if (r0ok) blk[(size_t)((step >> 4) - g0) * 32] = make_uint2(acc0, acc1);
            acc0 = acc1 = 0;
        }
        h0prev = hval<GAPZ, T>(h0);
        up0prev = hval<GAPZ, T>(up0);
        // on a stripe's first step row 1 sits on column 0: keep the boundary
        // H(i, 0) = +0 as its left neighbour for column 1
        h1 = j0 == 1 ? T(0) : n1;
        h0 = n0;
        q1x = q0x; q1y = q0y; q1z = q0z;
        ln1 = ln0;
        j0++;
    }
    if (((total_steps - 1) & 15) != 15 && r0ok) {  // flush the last rows' pending words
        const int sh = 30 - 2 * ((total_steps - 1) & 15);
        blk[(size_t)(((total_steps - 1) >> 4) - g0) * 32] = make_uint2(acc0 >> sh, acc1 >> sh);
    }
    __syncwarp();
    const long long clk1 = clock64();
    // traceback from (plen, nlen): diag emits a pair, up steps i, else j.
    // The walk only moves up and left.  A tile is 32 rows; lane l holds the
    // 4 trace words of row rb-l that end at the word of column jl (the
    // column when the tile was loaded), so a path crosses few tiles.
    int i = plen, j = nlen, cnt = 0, rb = -1, jl = 0;
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;
    while (i > 0 && j > 0) {
        const int bi = trace_base(i, P);
        const int wi = ((bi + j - 1) >> 4) - (bi >> 4);  // word of (i, j) in row i
        const int wl = ((bi + jl - 1) >> 4) - (bi >> 4);  // last word held for row i
        if (i > rb || i <= rb - 32 || wi < wl - 3) {
            rb = i;
            jl = j;
            const int r = rb - lane;
            if (r >= 1) {
                const int br = trace_base(r, P);
                const int wr = ((br + j - 1) >> 4) - (br >> 4);
                t3 = trace[trace_word(r, wr, P, G)];
                t2 = wr >= 1 ? trace[trace_word(r, wr - 1, P, G)] : 0u;
                t1 = wr >= 2 ? trace[trace_word(r, wr - 2, P, G)] : 0u;
                t0 = wr >= 3 ? trace[trace_word(r, wr - 3, P, G)] : 0u;
            }
        }
        const int wk = wi - (((bi + jl - 1) >> 4) - (bi >> 4)) + 3;  // 0..3 within the tile
        const uint32_t mine = wk == 3 ? t3 : wk == 2 ? t2 : wk == 1 ? t1 : t0;
        const uint32_t rw = __shfl_sync(kFull, mine, rb - i);
        const uint32_t dir = (rw >> (2 * ((bi + j - 1) & 15))) & 3u;
        if (dir == 0) {
            if (lane == 0) al[cnt] = ((uint32_t)(i - 1) << 16) | (uint32_t)(j - 1);
            cnt++;
            i--;
            j--;
        } else if (dir == 1) {
            i--;
        } else {
            j--;
        }
    }
    __syncwarp();
    if (lane == 0) {
        const long long clk2 = clock64();
        atomicAdd(ctr + CTR_CYC_NW, (unsigned long long)(clk1 - clk0));
        atomicAdd(ctr + CTR_CYC_TRACE, (unsigned long long)(clk2 - clk1));
    }
    return cnt;
}

IA_DEV int nw_align(const Pts &x, const NWParams &pr, const double *R, const double *t,
                    double *bH, uint32_t *trace, uint32_t *al, unsigned long long *ctr) {
    if (pr.smode == SMAT_DP) {
        if (pr.gap == 0.0) return nw_align_t<SMAT_DP, true, ChainDP>(x, pr, R, t, bH, trace, al, ctr);
        return nw_align_t<SMAT_DP, false, ChainDP>(x, pr, R, t, bH, trace, al, ctr);
    }
    if (pr.smode == SMAT_SS4) return nw_align_t<SMAT_SS4, false, ChainDP>(x, pr, R, t, bH, trace, al, ctr);
    return nw_align_t<SMAT_SS2, false, float>(x, pr, R, t, bH, trace, al, ctr);
}

// Kabsch on the aligned pairs + their compact TM (no d8)
// (indialign_c/align.h:106-124).
IA_DEV double aligned_kabsch(const Pts &x, const uint32_t *al, int na, double d0, double lnorm,
                             double *R, double *t, unsigned long long *ctr) {
    const int lane = threadIdx.x & 31;
    if (lane == 0) atomicAdd(ctr + CTR_CHAIN_RES, 2ull * (unsigned long long)na);
    Moments m;
    m.clear();
    for (int k = lane; k < na; k += 32) {
        int pi, ni;
        al_get(al, na, k, pi, ni);
        const double *p = x.P + 3 * pi, *q = x.Q + 3 * ni;
        m.add(p[0], p[1], p[2], q[0], q[1], q[2]);
    }
    m.group_sum(32);
    kabsch_from_moments(m, 3.0, R, t);
    const double d0sq = fmax(d0 * d0, 1e-12);
    double s = 0.0;
    for (int k = lane; k < na; k += 32) {
        int pi, ni;
        al_get(al, na, k, pi, ni);
        const double *p = x.P + 3 * pi, *q = x.Q + 3 * ni;
        s += 1.0 / (1.0 + dist2(R, t, p[0], p[1], p[2], q[0], q[1], q[2]) / d0sq);
    }
    return warp_sum(s) / fmax(lnorm, 1.0);
}

// alignment_detailed_search without fragments (indialign_c/align.h:15-50,
// use_frag = false): one all-pairs seed x 6 cutoffs x <= 8 iterations,
// d8-filtered score.  The all-pairs seed's Kabsch is the (R0,t0) just
// computed by aligned_kabsch.  Lane groups of 4 run the 6 cutoffs side by
// side; the first maximum in cutoff order wins.
IA_NW_ATTR double lite_detailed(const Pts &x, const uint32_t *al, int na, const double *R0,
                            const double *t0, const double *dcut, double d0, double sd8,
                            double lnorm, double *Ro, double *to, unsigned long long *ctr) {
    const int lane = threadIdx.x & 31, g = lane >> 2, sub = lane & 3;
    const bool grp = g < kDetC;
    const double cut = dcut[grp ? g : 0];
    const double cut2 = cut * cut;
    double R[9], t[3];
#pragma unroll
    for (int a = 0; a < 9; a++) R[a] = R0[a];
#pragma unroll
    for (int a = 0; a < 3; a++) t[a] = t0[a];
    bool running = grp;
    int prev = -1, iter = 0;
    while (__any_sync(kFull, running)) {
        Moments m;
        m.clear();
        int cnt = 0;
        if (running) {
            for (int k = sub; k < na; k += 4) {
                int pi, ni;
                al_get(al, na, k, pi, ni);
                const double *p = x.P + 3 * pi, *q = x.Q + 3 * ni;
                if (dist2(R, t, p[0], p[1], p[2], q[0], q[1], q[2]) <= cut2) {
                    m.add(p[0], p[1], p[2], q[0], q[1], q[2]);
                    cnt++;
                }
            }
        }
        m.group_sum(4);
        cnt += __shfl_xor_sync(kFull, cnt, 1);
        cnt += __shfl_xor_sync(kFull, cnt, 2);
        if (running) {
            if (cnt >= 3) kabsch_from_moments(m, 3.0, R, t);
            ++iter;
            if (cnt == prev || iter >= 8) running = false;
            prev = cnt;
        }
    }
    // residue visits: each active group ran `iter` passes + 1 score pass
    if (sub == 0 && grp) atomicAdd(ctr + CTR_CHAIN_RES, (unsigned long long)(iter + 1) * na);
    const double d0sq = fmax(d0 * d0, 1e-12), sd8sq = sd8 * sd8;
    double s = 0.0;
    if (grp) {
        for (int k = sub; k < na; k += 4) {
            int pi, ni;
            al_get(al, na, k, pi, ni);
            const double *p = x.P + 3 * pi, *q = x.Q + 3 * ni;
            double d2 = dist2(R, t, p[0], p[1], p[2], q[0], q[1], q[2]);
            if (d2 <= sd8sq) s += 1.0 / (1.0 + d2 / d0sq);
        }
    }
    s += __shfl_xor_sync(kFull, s, 1);
    s += __shfl_xor_sync(kFull, s, 2);
    const double score = s / fmax(lnorm, 1.0);
    // first max over cutoffs 0..5 (strict >, initial -1e30)
    double bs = kScoreInit;
    int bg = 0;
    for (int c = 0; c < kDetC; c++) {
        double sc = __shfl_sync(kFull, score, 4 * c);
        if (sc > bs) { bs = sc; bg = c; }
    }
#pragma unroll
    for (int a = 0; a < 9; a++) Ro[a] = __shfl_sync(kFull, R[a], 4 * bg);
#pragma unroll
    for (int a = 0; a < 3; a++) to[a] = __shfl_sync(kFull, t[a], 4 * bg);
    return bs;
}

// ---- the chain kernel ----------------------------------------------------
struct ChainCtl {
    int chunk, task, next;
};

// Element `lane` of a result record {score, R[9], t[3]} by unrolled selects
// (a dynamic index into R or t would move them to local memory).
IA_DEV double rec_elem(int lane, double score, const double *R, const double *t) {
    double v = score;
#pragma unroll
    for (int a = 0; a < 9; a++) v = lane == 1 + a ? R[a] : v;
#pragma unroll
    for (int a = 0; a < 3; a++) v = lane == 10 + a ? t[a] : v;
    return v;
}

// dst[0..11] = {R[9], t[3]} written by lanes 0..11 of the warp.
IA_DEV void put_rt(double *dst, const double *R, const double *t, int lane) {
    const double v = rec_elem(lane + 1, 0.0, R, t);
    if (lane < 12) dst[lane] = v;
}

// EMIT = false: LITE dp_refine chains only (the hot rescue kernel, DP score
// mode only); EMIT = true: single NW alignments for SS seeds / full dp_refine.
// Two instantiations keep the hot kernel's code small.
template <bool EMIT>
__global__ void __launch_bounds__(32 * kChainWarps, IA_CHAIN_MINB)
k_chain(DevBatch b, const ChainTask *__restrict__ tasks, const int *__restrict__ chunk_begin,
        int ntasks, const ScanOut *__restrict__ scan, int *counter, uint32_t *gtrace,
        size_t trace_words, double *gbh, uint32_t *gal, int pmax, int nmax, int flags) {
    extern __shared__ __align__(16) char smem[];
    __shared__ ChainCtl ctl;
    __shared__ uint64_t bar;
    // per warp: the LITE chain's current (R, t) and its best (R, t), kept in
    // shared memory so that no transform stays live in registers across the
    // NW fill
    __shared__ double s_rt[kChainWarps][24];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // shared layout: [native points as float4][pred labels][native labels]
    // (flag 1), then per warp the NW boundary row (flag 2), the alignment
    // (flag 4) and the NW trace block (flag 8, short pairs); the FP64 point
    // sets are read from global memory (L1)
    const bool coord_smem = flags & 1, bh_smem = flags & 2, al_smem = flags & 4, tr_smem = flags & 8;
    const uint32_t qfbytes = (uint32_t)nmax * 16u;
    const uint32_t plb = ((uint32_t)pmax + 47u) & ~15u, nlb = ((uint32_t)nmax + 47u) & ~15u;
    char *sQf = smem;
    char *sLp = sQf + (coord_smem ? qfbytes : 0), *sLn = sLp + (coord_smem ? plb : 0);
    char *wbase = sLn + (coord_smem ? nlb : 0);
    const uint32_t bh_bytes = (((uint32_t)nmax + 1u) * 8u + 15u) & ~15u;
    const uint32_t al_bytes = ((uint32_t)min(pmax, nmax) * 4u + 15u) & ~15u;
    const int gw = blockIdx.x * kChainWarps + warp;  // global warp slot
    double *bH = bh_smem ? reinterpret_cast<double *>(wbase + warp * bh_bytes)
                         : gbh + (size_t)gw * (nmax + 1);
    char *albase = wbase + (bh_smem ? kChainWarps * bh_bytes : 0);
    uint32_t *al = al_smem ? reinterpret_cast<uint32_t *>(albase + warp * al_bytes)
                           : gal + (size_t)gw * min(pmax, nmax);
    char *trbase = albase + (al_smem ? kChainWarps * al_bytes : 0);
    uint32_t *trace = tr_smem ? reinterpret_cast<uint32_t *>(trbase) + (size_t)warp * trace_words
                              : gtrace + (size_t)gw * trace_words;
    uint32_t phase = 0;
    if (threadIdx.x == 0) mbar_init(&bar);
    __syncthreads();
    const int total = scan->total_chunks;
    int staged = -1;
    Pts x = {nullptr, nullptr};
    const uint8_t *Lp = nullptr, *Ln = nullptr;
    const float4 *Qf = nullptr;
    for (;;) {
        if (threadIdx.x == 0) {
            int c = atomicAdd(counter, 1);
            int t = -1;
            if (c < total) {
                int lo = 0, hi = ntasks;
                while (lo < hi) {
                    int mid = (lo + hi) >> 1;
                    if (chunk_begin[mid] <= c) lo = mid + 1; else hi = mid;
                }
                t = lo - 1;
            }
            ctl.chunk = c;
            ctl.task = t;
            ctl.next = 0;
        }
        __syncthreads();
        const int c = ctl.chunk, ti = ctl.task;
        if (c >= total || ti < 0) break;
        const ChainTask &T = tasks[ti];
        const PairInfo &I = b.info[T.pair];
        const int off = I.off, plen = I.plen, nlen = I.nlen;
        if (T.pair != staged) {
            const double *gP = b.predc + 3 * (size_t)off, *gQ = b.natc + 3 * (size_t)off;
            const uint8_t *gLp = reinterpret_cast<const uint8_t *>(b.sspc + off);
            const uint8_t *gLn = reinterpret_cast<const uint8_t *>(b.ssnc + off);
            x.P = gP;
            x.Q = gQ;
            if (coord_smem) {
                Copy cp[2];
                char *dst[2] = {sLp, sLn};
                cp[0] = plan_copy(gLp, (uint32_t)plen);
                cp[1] = plan_copy(gLn, (uint32_t)nlen);
                stage_copies(cp, dst, 2, &bar, phase, b.err);
                float4 *qf = reinterpret_cast<float4 *>(sQf);
                for (int i = threadIdx.x; i < nlen; i += blockDim.x)
                    qf[i] = make_float4((float)gQ[3 * i], (float)gQ[3 * i + 1], (float)gQ[3 * i + 2], 0.f);
                __syncthreads();
                Qf = qf;
                Lp = reinterpret_cast<const uint8_t *>(sLp + cp[0].lead);
                Ln = reinterpret_cast<const uint8_t *>(sLn + cp[1].lead);
            } else {
                Qf = nullptr; Lp = gLp; Ln = gLn;
            }
            staged = T.pair;
        }
        // warps of the CTA pull the chunk's chains one at a time, so a long
        // chain does not hold the other warps at a barrier
        for (;;) {
            int idx = 0;
            if (lane == 0) idx = atomicAdd(&ctl.next, 1);
            idx = __shfl_sync(kFull, idx, 0);
            const int chain = (c - chunk_begin[ti]) * T.chunk + idx;
            if (idx >= T.chunk || chain >= T.n_chains) break;
            if (lane == 0) atomicAdd(b.ctr + CTR_CHAINS, 1ull);
            const int gaps = T.gaps;
            const int si = chain / gaps, g = chain % gaps;
            const double gap = (gaps == 2 ? g : si) == 0 ? T.gap0 : T.gap1;
            double R[9], t[3];
            bool live = true;
            if (T.start == START_WINDOW) {
                int flen, ps, ns;
                window_at(plen, nlen, T.dense, T.wlist ? T.wlist[si] : si, flen, ps, ns);
                warp_kabsch_window(x, ps, ns, flen, R, t);
            } else {
                const double *r = T.rt + (size_t)si * kRec;
                live = r[0] > -1e299;  // start flag: kNegInf = no start
#pragma unroll
                for (int a = 0; a < 9; a++) R[a] = r[1 + a];
#pragma unroll
                for (int a = 0; a < 3; a++) t[a] = r[10 + a];
            }
            NWParams pr;
            pr.plen = plen;
            pr.nlen = nlen;
            pr.smode = T.smode;
            pr.gap = gap;
            pr.Lp = Lp;
            pr.Ln = Ln;
            pr.Qf = Qf;
            if (T.smode == SMAT_SS4) {
                double d01 = fmax(I.d0 + 1.5, I.d0s);
                pr.inv_d0sq = 1.0 / (d01 * d01);
                pr.cut2 = 0.0;
            } else {
                double d0dp = fmax(I.d0, 1.0);
                pr.inv_d0sq = 1.0 / fmax(d0dp * d0dp, 1e-12);
                pr.cut2 = T.sd8 * T.sd8;
            }
            if (T.live && !T.live[si]) live = false;
            if (EMIT) {
                // EMIT: one alignment; aligned coordinates, count and (for
                // SMAT_DP) the Kabsch on it with its compact score.
                int na = 0;
                // ss_nw_align / dp_refine_chunk need >= 3 valid on each side
                // (indialign_c/ss.h:58, align.h:141)
                if (live && plen >= 3 && nlen >= 3) na = nw_align(x, pr, R, t, bH, trace, al, b.ctr);
                if (lane == 0) T.na_out[si] = na;
                double *aP = T.alP + (size_t)si * T.al_cap * 3;
                double *aQ = T.alQ + (size_t)si * T.al_cap * 3;
                for (int k = lane; k < na && k < T.al_cap; k += 32) {
                    int pi, ni;
                    al_get(al, na, k, pi, ni);
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        aP[3 * k + d] = x.P[3 * pi + d];
                        aQ[3 * k + d] = x.Q[3 * ni + d];
                    }
                }
                if (T.smode == SMAT_DP && na >= 3) {
                    double nR[9], nt[3];
                    double s = aligned_kabsch(x, al, na, I.d0, I.lnorm, nR, nt, b.ctr);
                    double *o = T.res + (size_t)si * kRec;
                    const double v = rec_elem(lane, s, nR, nt);
                    if (lane < kRec) o[lane] = v;
                }
            } else {
                // LITE dp_refine chain (indialign_c/align.h:54-145,
                // d0_search_lite): best starts at score 0 / identity.
                double *rt = s_rt[warp];  // [current R, t][best R, t]
                double bs = 0.0;
                {
                    double iR[9], it_[3];
                    set_identity(iR, it_);
                    put_rt(rt, R, t, lane);
                    put_rt(rt + 12, iR, it_, lane);
                }
                __syncwarp();
                // dp_refine_chunk returns 0 / identity unless both sides have
                // >= 3 valid residues (indialign_c/align.h:141)
                const bool sized = plen >= 3 && nlen >= 3;
                for (int it = 0; live && sized && it < T.max_iter; it++) {
                    const int na = pr.gap == 0.0
                                       ? nw_align_t<SMAT_DP, true, ChainDP>(x, pr, rt, rt + 9, bH, trace, al, b.ctr)
                                       : nw_align_t<SMAT_DP, false, ChainDP>(x, pr, rt, rt + 9, bH, trace, al, b.ctr);
                    if (na < 3) break;  // same transform -> same alignment next time
                    double nR[9], nt[3], dR[9], dt[3];
                    const long long ck0 = clock64();
                    double s = aligned_kabsch(x, al, na, I.d0, I.lnorm, nR, nt, b.ctr);
                    const long long ck1 = clock64();
                    double ds = lite_detailed(x, al, na, nR, nt, I.dcut, I.d0, T.sd8, I.lnorm, dR, dt, b.ctr);
                    if (lane == 0) {
                        atomicAdd(b.ctr + CTR_CYC_KABSCH, (unsigned long long)(ck1 - ck0));
                        atomicAdd(b.ctr + CTR_CYC_DETAIL, (unsigned long long)(clock64() - ck1));
                    }
                    if (ds > s) {
                        s = ds;
#pragma unroll
                        for (int a = 0; a < 9; a++) nR[a] = dR[a];
#pragma unroll
                        for (int a = 0; a < 3; a++) nt[a] = dt[a];
                    }
                    __syncwarp();  // every lane's NW reads of the current (R, t) are done
                    put_rt(rt, nR, nt, lane);
                    if (s > bs) {
                        bs = s;
                        put_rt(rt + 12, nR, nt, lane);
                    }
                    __syncwarp();
                }
                double *o = T.res + (size_t)chain * kRec;
                if (lane < kRec) o[lane] = lane == 0 ? (live ? bs : kNegInf) : rt[12 + lane - 1];
                __syncwarp();  // the slot is reused by this warp's next chain
            }
        }
        __syncthreads();
    }
}

// ---- NW on an explicit score matrix (one warp per problem) ---------------
// nw_dp + nw_traceback (indialign_c/nw.h:10-68) on a caller-given FP64 score
// matrix: the same fill and traceback as the chains, so that the DP can be
// checked bit for bit against the reference on identical inputs.
__global__ void k_nw_explicit(const double *__restrict__ smat, int np, int nn, double gap,
                              uint32_t *trace, double *bH, uint32_t *al, int *ap, int *an,
                              int *na_out, unsigned long long *ctr) {
    NWParams pr;
    pr.plen = np;
    pr.nlen = nn;
    pr.smode = SMAT_EXPLICIT;
    pr.gap = gap;
    pr.inv_d0sq = 0.0;
    pr.cut2 = 0.0;
    pr.Lp = pr.Ln = nullptr;
    pr.smat = smat;
    pr.Qf = nullptr;
    Pts x = {nullptr, nullptr};
    const double I[12] = {1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0};
    int na = 0;
    if (np >= 1 && nn >= 1) {
        if (gap == 0.0) na = nw_align_t<SMAT_EXPLICIT, true, double>(x, pr, I, I + 9, bH, trace, al, ctr);
        else na = nw_align_t<SMAT_EXPLICIT, false, double>(x, pr, I, I + 9, bH, trace, al, ctr);
    }
    for (int k = threadIdx.x; k < na; k += 32) {
        const uint32_t e = al[na - 1 - k];
        ap[k] = (int)(e >> 16);
        an[k] = (int)(e & 0xffffu);
    }
    if (threadIdx.x == 0) *na_out = na;
}

size_t nw_trace_words(int np, int nn) { return nw_trace_words_for(np, nn); }

void launch_nw_explicit(const double *smat, int np, int nn, double gap, uint32_t *trace,
                        double *bH, uint32_t *al, int *ap, int *an, int *na,
                        unsigned long long *ctr, cudaStream_t st) {
    k_nw_explicit<<<1, 32, 0, st>>>(smat, np, nn, gap, trace, bH, al, ap, an, na, ctr);
}

size_t chain_smem_bytes(int pmax, int nmax, int flags) {
    size_t s = 0;
    if (flags & 1) {
        s += (size_t)nmax * 16;
        s += (((size_t)pmax + 47) & ~size_t(15)) + (((size_t)nmax + 47) & ~size_t(15));
    }
    if (flags & 2) s += kChainWarps * ((((size_t)nmax + 1) * 8 + 15) & ~size_t(15));
    if (flags & 4) s += kChainWarps * (((size_t)min(pmax, nmax) * 4 + 15) & ~size_t(15));
    if (flags & 8) s += kChainWarps * nw_trace_words_for(pmax, nmax) * 4;
    return s;
}

void launch_chain(const DevBatch &b, const ChainTask *tasks, const int *chunk_begin, int ntasks,
                  const ScanOut *scan, int *counter, uint32_t *gtrace, size_t trace_words,
                  double *gbh, uint32_t *gal, int pmax, int nmax, int flags, int grid, bool emit,
                  cudaStream_t st) {
    size_t sm = chain_smem_bytes(pmax, nmax, flags);
    if (emit)
        k_chain<true><<<grid, 32 * kChainWarps, sm, st>>>(b, tasks, chunk_begin, ntasks, scan, counter,
                                                          gtrace, trace_words, gbh, gal, pmax, nmax, flags);
    else
        k_chain<false><<<grid, 32 * kChainWarps, sm, st>>>(b, tasks, chunk_begin, ntasks, scan, counter,
                                                           gtrace, trace_words, gbh, gal, pmax, nmax, flags);
}

const void *chain_kernel_ptr() { return (const void *)k_chain<false>; }

cudaError_t chain_set_attributes() {
    cudaError_t e = cudaFuncSetAttribute(k_chain<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kChainSmemMax);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_chain<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kChainSmemMax);
    return e;
}

}  // namespace ia
