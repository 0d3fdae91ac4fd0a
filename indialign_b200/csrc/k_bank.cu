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
#include "dmath.cuh"
#include "stage.cuh"
#include "pipeline.h"
#include "kernels.h"
#include "sched.cuh"

// build-time knobs: minimum resident bank CTAs per SM (caps registers; 4 -> 128
// registers measured best, 15 % over the uncapped 146), a
// straight-line cutoff pass (weighted accumulate) and its unroll factor
#ifndef IA_BANK_MINB
#define IA_BANK_MINB 4
#endif
#ifndef IA_BANK_FLAT
#define IA_BANK_FLAT 0
#endif
#ifndef IA_BANK_UNROLL
#define IA_BANK_UNROLL 1
#endif

namespace ia {

#if IA_BANK_FLAT
constexpr int kBankUnroll = IA_BANK_UNROLL;
#endif

// ---- the bank kernel -------------------------------------------------------
struct BankSmem {
    int chunk, task;
};

template <bool SMEM>
__global__ void __launch_bounds__(kBankChunk, IA_BANK_MINB)
k_bank(const BankTask *__restrict__ tasks, const int *__restrict__ chunk_begin,
       int ntasks, const ScanOut *__restrict__ scan, int *counter,
       double *__restrict__ item_res, int *err, int nmax, unsigned long long *ctr) {
    extern __shared__ __align__(16) char smem[];
    __shared__ BankSmem ctl;
    __shared__ uint64_t bar;
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
    const double *P = nullptr, *Q = nullptr;
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
                P = reinterpret_cast<const double *>(sP + cp[0].lead);
                Q = reinterpret_cast<const double *>(sQ + cp[1].lead);
                int k = 2;
                V = T.V ? reinterpret_cast<const uint8_t *>(sV + cp[k++].lead) : nullptr;
                PV = T.PV ? reinterpret_cast<const uint8_t *>(sPV + cp[k++].lead) : nullptr;
                NV = T.NV ? reinterpret_cast<const uint8_t *>(sNV + cp[k++].lead) : nullptr;
            } else {
                P = T.P; Q = T.Q; V = T.V; PV = T.PV; NV = T.NV;
            }
            staged = ti;
        }
        const int li = (c - chunk_begin[ti]) * kBankChunk + threadIdx.x;
        const bool active = li < T.n_items;
        const int C = T.C > 0 ? T.C : 1;
        const int k = active ? (T.slist ? T.slist[li / C] : li / C) : 0, ci = active ? li % C : 0;
        const double cut = T.cut[ci];
        const double cut2 = cut * cut;
        double R[9], t[3];
        Moments m;
        m.clear();
        bool skip = false;
        // ---- initial Kabsch on the seed ----
        if (T.mode == SEED_SHIFT) {
            const int o = offset_at(T.shift_lo, T.shift_stride, k);
            for (int i = 0; i < n; i++) {
                int j = i - o;
                bool sel = active && j >= 0 && j < n && PV[i] != 0 && NV[j] != 0;
                if (sel)
                    m.add(P[3 * i], P[3 * i + 1], P[3 * i + 2], Q[3 * j], Q[3 * j + 1], Q[3 * j + 2]);
            }
            skip = m.w < (double)T.shift_min;
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
                if (active && sel)
                    m.add(P[3 * i], P[3 * i + 1], P[3 * i + 2], Q[3 * i], Q[3 * i + 1], Q[3 * i + 2]);
            }
        }
        if (active && !skip) kabsch_from_moments(m, 3.0, R, t);
        else set_identity(R, t);
        // ---- cutoff iterations: select d2 <= cut^2, Kabsch, stop on a
        // repeated count ----
        bool running = active && !skip && T.max_iter > 0;
        int prev = -1, iter = 0;
        while (__any_sync(0xffffffffu, running)) {
            m.clear();
            int cnt = 0;
#if IA_BANK_FLAT
            // straight-line body: a 0/1 weight leaves the moments exactly as
            // a skipped or plain add, so unrolled residues interleave
#pragma unroll kBankUnroll
            for (int i = 0; i < n; i++) {
                const double px = P[3 * i], py = P[3 * i + 1], pz = P[3 * i + 2];
                const double qx = Q[3 * i], qy = Q[3 * i + 1], qz = Q[3 * i + 2];
                const bool v = V ? V[i] != 0 : true;
                const double d2 = dist2(R, t, px, py, pz, qx, qy, qz);
                const bool sel = running && v && d2 <= cut2;
                m.add_w(sel ? 1.0 : 0.0, px, py, pz, qx, qy, qz);
                cnt += sel ? 1 : 0;
            }
#else
            for (int i = 0; i < n; i++) {
                const double px = P[3 * i], py = P[3 * i + 1], pz = P[3 * i + 2];
                const double qx = Q[3 * i], qy = Q[3 * i + 1], qz = Q[3 * i + 2];
                const bool v = V ? V[i] != 0 : true;
                if (running && v) {
                    double d2 = dist2(R, t, px, py, pz, qx, qy, qz);
                    if (d2 <= cut2) {
                        m.add(px, py, pz, qx, qy, qz);
                        cnt++;
                    }
                }
            }
#endif
            if (running) {
                if (cnt >= 3) kabsch_from_moments(m, 3.0, R, t);
                ++iter;
                if (cnt == prev || iter >= T.max_iter) running = false;
                prev = cnt;
            }
        }
        // ---- score: sum 1/(1+d2/d0^2) over the set (optionally d2 <= sd8^2)
        // divided by max(Lnorm, 1) (indialign_c/core.h:134-166) ----
        double score = kNegInf;
        if (active && !skip) {
            const double d0sq = fmax(T.d0 * T.d0, 1e-12), sd8sq = T.sd8 * T.sd8;
            double sum = 0.0;
            for (int i = 0; i < n; i++) {
                const bool v = V ? V[i] != 0 : true;
                if (!v) continue;
                double d2 = dist2(R, t, P[3 * i], P[3 * i + 1], P[3 * i + 2], Q[3 * i], Q[3 * i + 1],
                                  Q[3 * i + 2]);
                if (!T.use_d8 || d2 <= sd8sq) sum += 1.0 / (1.0 + d2 / d0sq);
            }
            score = sum / fmax(T.lnorm, 1.0);
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
            double *o = item_res + (size_t)(T.item_base + li) * kRec;
            o[0] = score;
#pragma unroll
            for (int a = 0; a < 9; a++) o[1 + a] = R[a];
#pragma unroll
            for (int a = 0; a < 3; a++) o[10 + a] = t[a];
        }
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
    double *out = T.out_rec >= 0 ? state[T.pair].rec[T.out_rec] : T.out;
    if (lane < kRec) {
        double v;
        if (bi >= 0) v = base[(size_t)bi * kRec + lane];
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
