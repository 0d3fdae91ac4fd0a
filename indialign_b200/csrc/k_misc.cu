// Per-pair kernels of the search: input compaction and seed tables, anchor
// contact seeds, SS labels, the top-50% distance seed, the weighted polish,
// same-index rescoring, offset starts, stage glue and the device scan.
#include "dmath.cuh"
#include "pipeline.h"
#include "kernels.h"
#include "sched.cuh"

namespace ia {

constexpr unsigned kAll = 0xffffffffu;
constexpr uint64_t kFnvOffset = 14695981039346656037ULL;
constexpr uint64_t kFnvPrime = 1099511628211ULL;

// ---- block helpers (256 threads) ------------------------------------------
template <typename T>
IA_DEV T block_sum(T v, T *red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kAll, v, o);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    T s = 0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += red[i];
        red[0] = s;
    }
    __syncthreads();
    s = red[0];
    __syncthreads();
    return s;
}

// Exclusive scan of 0/1 flags over one tile of blockDim.x entries; returns
// the rank of this thread's flag and writes the tile total to *tot.
IA_DEV int block_rank(bool f, int *wsum, int *tot) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned bal = __ballot_sync(kAll, f);
    int r = __popc(bal & ((1u << lane) - 1u));
    __syncthreads();
    if (lane == 0) wsum[w] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int i = 0; i < nw; i++) { int c = wsum[i]; wsum[i] = s; s += c; }
        *tot = s;
    }
    __syncthreads();
    r += wsum[w];
    return r;
}

// ---- prep: sums, compaction, d0 schedule, fragment seed table -------------
// build_seed_masks over the full pair (indialign_c/seeds.h:41-82): the global
// seed (the valid mask itself) and windows [s, s+flen) of the valid mask for
// flen in fragment_lengths(sum of valid bytes) at start_positions(N, flen,
// 50), each kept only if its valid-byte sum is >= 3.

__global__ void k_prep(DevBatch b, int use_frag) {
    __shared__ int red_i[32];
    __shared__ int wsum[32], tot;
    const int p = blockIdx.x;
    const int N = b.len[p], off = b.off[p];
    PairInfo &I = b.info[p];
    PairState &S = b.state[p];
    const uint8_t *v = b.v + off, *pv = b.pv + off, *nv = b.nv + off;
    int vs = 0, pvs = 0, nvs = 0, vc = 0, pc = 0, nc = 0, cross = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        vs += v[i]; pvs += pv[i]; nvs += nv[i];
        vc += v[i] != 0; pc += pv[i] != 0; nc += nv[i] != 0;
        cross |= pv[i] != nv[i];
    }
    vs = block_sum(vs, red_i); pvs = block_sum(pvs, red_i); nvs = block_sum(nvs, red_i);
    vc = block_sum(vc, red_i); pc = block_sum(pc, red_i); nc = block_sum(nc, red_i);
    cross = block_sum(cross, red_i);
    // order-preserving compaction of pv / nv / v and prefix sums of v bytes
    int rp = 0, rn = 0, rv = 0, pre = 0;
    int *vpre = b.scratch + off + p;  // N+1 entries
    for (int base = 0; base < N; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const bool in = i < N;
        int r = block_rank(in && pv[i] != 0, wsum, &tot);
        if (in && pv[i] != 0) {
            b.pmap[off + rp + r] = i;
#pragma unroll
            for (int d = 0; d < 3; d++) b.predc[3 * (size_t)(off + rp + r) + d] = b.pred[3 * (size_t)(off + i) + d];
        }
        rp += tot;
        __syncthreads();
        r = block_rank(in && nv[i] != 0, wsum, &tot);
        if (in && nv[i] != 0) {
            b.nmap[off + rn + r] = i;
#pragma unroll
            for (int d = 0; d < 3; d++) b.natc[3 * (size_t)(off + rn + r) + d] = b.nat[3 * (size_t)(off + i) + d];
        }
        rn += tot;
        __syncthreads();
        r = block_rank(in && v[i] != 0, wsum, &tot);
        if (in && v[i] != 0) b.vmap[off + rv + r] = i;
        rv += tot;
        __syncthreads();
        // inclusive prefix of valid bytes within the tile, sequential over warps
        int x = in ? v[i] : 0;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(kAll, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            int s = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); k++) { int c = wsum[k]; wsum[k] = s; s += c; }
            tot = s;
        }
        __syncthreads();
        if (in) vpre[i + 1] = pre + wsum[w] + x;
        pre += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        vpre[0] = 0;
        I.N = N; I.off = off;
        I.plen = pc; I.nlen = nc; I.vcount = vc;
        I.vsum = vs; I.pvsum = pvs; I.nvsum = nvs;
        I.has_cross = cross != 0;
        I.lnorm = b.lnorm[p];
        d0_from_length(I.lnorm, I.d0, I.d0s, I.sd8);
        I.C = d0_candidates(I.d0, I.d0s, I.cut);
        for (int c = 0; c < kDetC; c++) I.dcut[c] = I.d0s * kD0Mults[c];
        I.bitoff = b.bitoff[p];
        I.words = (N + 31) >> 5;
        I.nbits = 0;
        I.status = I.lnorm <= 2.0 ? 1 : 0;
        I.K = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0 && I.status == 0) {
        int2 *tab = b.seeds + (size_t)p * kMaxSeeds;
        int K = 0;
        if (vs >= 3) tab[K++] = make_int2(0, N);
        if (use_frag) {
            int fl[9], nf = frag_lengths(vs, fl);
            for (int a = 0; a < nf; a++) {
                int ns = n_starts(N, fl[a], 50);
                for (int k = 0; k < ns; k++) {
                    int s = start_at(N, fl[a], 50, k);
                    int e = min(s + fl[a], N);
                    if (vpre[e] - vpre[s] < 3) continue;
                    if (K < kMaxSeeds - kMaxBitSeeds) tab[K++] = make_int2(s, fl[a]);
                    else atomicOr(b.err, DERR_CAPACITY);
                }
            }
        }
        I.K = K;
    }
    __syncthreads();
    if (threadIdx.x < kRec) {
        // running best: score 0 / identity for degenerate pairs; otherwise
        // overwritten by the seed bank
        double val = (threadIdx.x == 1 || threadIdx.x == 5 || threadIdx.x == 9) ? 1.0 : 0.0;
        if (threadIdx.x == 0) val = I.status ? 0.0 : kScoreInit;
        S.rec[REC_BEST][threadIdx.x] = val;
    }
    if (threadIdx.x == 0) {
        S.na[0] = S.na[1] = 0;
        S.active[0] = S.active[1] = 0;
        S.flag = 0;
        S.dp_on = 0;
        S.topk_ok = 0;
    }
}

// ---- anchor contact seeds (indialign_c/seeds.h:164-283) -------------------
IA_DEV uint64_t fnv_window(const uint8_t *v, int N, int s, int len, const uint64_t *pw) {
    uint64_t h = kFnvOffset * pw[s];
    int e = min(s + len, N);
    for (int i = s; i < e; i++) { h ^= v[i]; h *= kFnvPrime; }
    return h * pw[N - e];
}

IA_DEV uint64_t fnv_bits(const uint32_t *bits, int N, const uint64_t *pw) {
    uint64_t h = kFnvOffset;
    int pos = 0;
    const int words = (N + 31) >> 5;
    for (int w = 0; w < words; w++) {
        uint32_t x = bits[w];
        while (x) {
            int i = w * 32 + __ffs(x) - 1;
            x &= x - 1;
            h *= pw[i - pos];
            h ^= 1ull;
            h *= kFnvPrime;
            pos = i + 1;
        }
    }
    return h * pw[N - pos];
}

// The reference orders anchor candidates with std::sort on the count only;
// equal counts keep the order its introsort leaves them in.  This is the same
// sequence of element moves (libstdc++ introsort: median-of-three to the
// front, unguarded partition, depth 2*floor(log2 n) then heapsort, runs <= 16
// finished by insertion sort), so ties resolve identically.  The move
// sequence follows GCC's libstdc++ (bits/stl_algo.h: __introsort_loop,
// __unguarded_partition_pivot, __final_insertion_sort; bits/stl_heap.h:
// __adjust_heap, __push_heap), which is licensed under GPLv3 with the GCC
// Runtime Library Exception; it is restated here only so that tie order
// matches the reference build's std::sort, and is pinned against that build
// by a golden fixture of sort orders.
struct KV { int key, idx; };
#define KVL(x, y) ((x).key > (y).key)
IA_DEV void kv_swap(KV *a, KV *b) { KV t = *a; *a = *b; *b = t; }
IA_DEV void kv_adjust(KV *f, long hole, long len, KV val) {
    long top = hole, child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (KVL(f[child], f[child - 1])) child--;
        f[hole] = f[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        f[hole] = f[child - 1];
        hole = child - 1;
    }
    long parent = (hole - 1) / 2;
    while (hole > top && KVL(f[parent], val)) {
        f[hole] = f[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    f[hole] = val;
}
IA_DEV void kv_heapsort(KV *f, long len) {
    if (len >= 2) {
        for (long parent = (len - 2) / 2;; parent--) {
            kv_adjust(f, parent, len, f[parent]);
            if (parent == 0) break;
        }
    }
    while (len > 1) {
        len--;
        KV val = f[len];
        f[len] = f[0];
        kv_adjust(f, 0, len, val);
    }
}
IA_DEV void kv_linear_insert(KV *f, long i) {
    KV val = f[i];
    long j = i - 1;
    while (KVL(val, f[j])) { f[i] = f[j]; i = j; j--; }
    f[i] = val;
}
IA_DEV void kv_sort(KV *f, long n) {
    if (n <= 0) return;
    int lg = 0;
    while ((1L << (lg + 1)) <= n) lg++;
    // explicit stack replaces the recursion on the right part
    long stk_lo[64], stk_hi[64];
    int stk_d[64], sp = 0;
    stk_lo[sp] = 0; stk_hi[sp] = n; stk_d[sp] = 2 * lg; sp++;
    while (sp > 0) {
        sp--;
        long lo = stk_lo[sp], hi = stk_hi[sp];
        int depth = stk_d[sp];
        while (hi - lo > 16) {
            if (depth == 0) { kv_heapsort(f + lo, hi - lo); break; }
            depth--;
            long mid = lo + (hi - lo) / 2, a = lo + 1, c = hi - 1;
            if (KVL(f[a], f[mid])) {
                if (KVL(f[mid], f[c])) kv_swap(&f[lo], &f[mid]);
                else if (KVL(f[a], f[c])) kv_swap(&f[lo], &f[c]);
                else kv_swap(&f[lo], &f[a]);
            } else if (KVL(f[a], f[c])) kv_swap(&f[lo], &f[a]);
            else if (KVL(f[mid], f[c])) kv_swap(&f[lo], &f[c]);
            else kv_swap(&f[lo], &f[mid]);
            long x = lo + 1, y = hi;
            for (;;) {
                while (KVL(f[x], f[lo])) x++;
                y--;
                while (KVL(f[lo], f[y])) y--;
                if (!(x < y)) break;
                kv_swap(&f[x], &f[y]);
                x++;
            }
            // the reference recurses on [cut, hi) first, then loops on
            // [lo, cut); the ranges are disjoint, so the order of the two
            // does not change the result
            if (sp < 64) { stk_lo[sp] = x; stk_hi[sp] = hi; stk_d[sp] = depth; sp++; }
            hi = x;
        }
    }
    if (n > 16) {
        for (long i = 1; i < 16; i++) {
            if (KVL(f[i], f[0])) {
                KV val = f[i];
                for (long k = i; k > 0; k--) f[k] = f[k - 1];
                f[0] = val;
            } else {
                kv_linear_insert(f, i);
            }
        }
        for (long i = 16; i < n; i++) kv_linear_insert(f, i);
    } else {
        for (long i = 1; i < n; i++) {
            if (KVL(f[i], f[0])) {
                KV val = f[i];
                for (long k = i; k > 0; k--) f[k] = f[k - 1];
                f[0] = val;
            } else {
                kv_linear_insert(f, i);
            }
        }
    }
}

IA_DEV bool contact_ok(const double *P, const double *Q, int i, int j, double rad_sq, double tol) {
    double dx = P[3 * i] - P[3 * j], dy = P[3 * i + 1] - P[3 * j + 1], dz = P[3 * i + 2] - P[3 * j + 2];
    double pd2 = dx * dx + dy * dy + dz * dz;
    if (pd2 > rad_sq) return false;
    dx = Q[3 * i] - Q[3 * j]; dy = Q[3 * i + 1] - Q[3 * j + 1]; dz = Q[3 * i + 2] - Q[3 * j + 2];
    double nd2 = dx * dx + dy * dy + dz * dz;
    if (nd2 > rad_sq) return false;
    return fabs(sqrt(pd2) - sqrt(nd2)) <= tol;
}

__global__ void k_anchor(DevBatch b) {
    __shared__ int red_i[32];
    __shared__ uint64_t s_hash;
    __shared__ int s_dup;
    const int p = blockIdx.x;
    PairInfo &I = b.info[p];
    PairState &S = b.state[p];
    if (I.status != 0) return;
    const int N = I.N, off = I.off, V = I.vcount, words = I.words;
    const double *P = b.pred + 3 * (size_t)off, *Q = b.nat + 3 * (size_t)off;
    const uint8_t *v = b.v + off;
    const int *vidx = b.vmap + off;
    int2 *tab = b.seeds + (size_t)p * kMaxSeeds;
    uint64_t *hs = b.hashes + (size_t)p * kMaxSeeds;
    uint32_t *bits = b.bits + I.bitoff;
    int *cnt = b.scratch + off + p;     // V counts (prefix sums no longer needed)
    KV *kv = reinterpret_cast<KV *>(b.kv + 2 * (size_t)off);
    int K0 = I.K;
    if (V >= 3) {
        for (int k = threadIdx.x; k < K0; k += blockDim.x)
            hs[k] = fnv_window(v, N, tab[k].x, tab[k].y, b.fnv_pow);
        double radii[6];
        int nrad = 0;
        const double mr[3] = {I.d0s, I.d0s * 1.5, I.d0s * 2.0};
        const double ar[3] = {I.d0 + 1.0, I.d0 + 2.0, I.d0 + 3.0};
        for (int a = 0; a < 3; a++) radii[nrad++] = mr[a];
        for (int a = 0; a < 3; a++) {
            bool dup = false;
            for (int c = 0; c < nrad; c++) dup |= fabs(radii[c] - ar[a]) < 0.01;
            if (!dup) radii[nrad++] = ar[a];
        }
        int K = K0, nseen = K0, nbits = 0;
        __syncthreads();
        for (int ri = 0; ri < nrad; ri++) {
            const double rad = radii[ri];
            if (rad <= 0) continue;
            const double rad_sq = rad * rad, tol = fmax(0.5, rad * 0.25);
            for (int a = threadIdx.x; a < V; a += blockDim.x) {
                const int i = vidx[a];
                int c = 1;
                for (int bb = 0; bb < V; bb++) {
                    const int j = vidx[bb];
                    if (j != i && contact_ok(P, Q, i, j, rad_sq, tol)) c++;
                }
                cnt[a] = c;
            }
            __syncthreads();
            __shared__ int s_nc;
            if (threadIdx.x == 0) {
                int nc = 0;
                for (int a = 0; a < V; a++)
                    if (cnt[a] >= 3) { kv[nc].key = cnt[a]; kv[nc].idx = a; nc++; }
                kv_sort(kv, nc);
                s_nc = nc;
            }
            __syncthreads();
            const int nc = s_nc;
            int added = 0;
            for (int ci = 0; ci < nc && added < 5; ci++) {
                const int i = vidx[kv[ci].idx];
                const int slot = nbits < kMaxBitSeeds - 1 ? nbits : kMaxBitSeeds - 2;
                uint32_t *mb = bits + (size_t)slot * words;
                for (int w = threadIdx.x; w < words; w += blockDim.x) mb[w] = 0u;
                __syncthreads();
                int mc = 0;
                for (int bb = threadIdx.x; bb < V; bb += blockDim.x) {
                    const int j = vidx[bb];
                    if (j == i || contact_ok(P, Q, i, j, rad_sq, tol)) {
                        atomicOr(mb + (j >> 5), 1u << (j & 31));
                        mc++;
                    }
                }
                mc = block_sum(mc, red_i);
                if (mc < 3) continue;
                if (threadIdx.x == 0) s_hash = fnv_bits(mb, N, b.fnv_pow);
                if (threadIdx.x == 0) s_dup = 0;
                __syncthreads();
                const uint64_t h = s_hash;
                for (int k = threadIdx.x; k < nseen; k += blockDim.x)
                    if (hs[k] == h) s_dup = 1;
                __syncthreads();
                if (s_dup) continue;
                if (nbits >= kMaxBitSeeds - 1 || K >= kMaxSeeds) {
                    if (threadIdx.x == 0) atomicOr(b.err, DERR_CAPACITY);
                    continue;
                }
                if (threadIdx.x == 0) {
                    hs[nseen] = h;
                    tab[K] = make_int2(-1 - nbits, mc);
                }
                nseen++;
                K++;
                nbits++;
                added++;
                __syncthreads();
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) { I.K = K; I.nbits = nbits; }
    }
    __syncthreads();
    if (threadIdx.x == 0 && I.K == 0) {
        // no seeds: score 0 / identity (indialign_c/indialign.cpp:77-81)
        I.status = 1;
        double *r = S.rec[REC_BEST];
        for (int a = 0; a < kRec; a++) r[a] = (a == 1 || a == 5 || a == 9) ? 1.0 : 0.0;
    }
}

// ---- SS labels (indialign_c/ss.h:16-52) -------------------------------------
// Greedy pairing: i ascending, partner = the largest j > i+3 (both valid with
// their inner neighbours, both C1'-C1' distances of (i,j) and (i+1,j-1) in
// [9,12] A) that is still unpaired.  One warp per (pair, side).
__global__ void k_ss(DevBatch b) {
    const int p = blockIdx.x >> 1, side = blockIdx.x & 1;
    const int lane = threadIdx.x;
    const PairInfo &I = b.info[p];
    if (I.status != 0) return;
    const int N = I.N, off = I.off;
    const double *X = (side ? b.nat : b.pred) + 3 * (size_t)off;
    const uint8_t *v = (side ? b.nv : b.pv) + off;
    int *bp = b.kv + 2 * (size_t)off + (size_t)side * N;
    for (int i = lane; i < N; i += 32) bp[i] = -1;
    __syncwarp();
    const double lo = 81.0, hi = 144.0;
    for (int i = 0; i < N - 4; i++) {
        if (!v[i] || !v[i + 1]) continue;
        if (bp[i] >= 0) continue;
        const double xi = X[3 * i], yi = X[3 * i + 1], zi = X[3 * i + 2];
        const double xn = X[3 * i + 3], yn = X[3 * i + 4], zn = X[3 * i + 5];
        for (int jb = N - 1; jb > i + 3; jb -= 32) {
            const int j = jb - lane;
            bool ok = false;
            if (j > i + 3 && v[j] && v[j - 1] && bp[j] < 0) {
                double dx = xi - X[3 * j], dy = yi - X[3 * j + 1], dz = zi - X[3 * j + 2];
                double a = dx * dx + dy * dy + dz * dz;
                dx = xn - X[3 * (j - 1)]; dy = yn - X[3 * (j - 1) + 1]; dz = zn - X[3 * (j - 1) + 2];
                double c = dx * dx + dy * dy + dz * dz;
                ok = a >= lo && a <= hi && c >= lo && c <= hi;
            }
            unsigned bal = __ballot_sync(kAll, ok);
            if (bal) {
                const int jsel = jb - (__ffs(bal) - 1);
                if (lane == 0) { bp[i] = jsel; bp[jsel] = i; }
                break;
            }
        }
        __syncwarp();
    }
    __syncwarp();
    const int len = side ? I.nlen : I.plen;
    const int *map = (side ? b.nmap : b.pmap) + off;
    char *out = (side ? b.ssnc : b.sspc) + off;
    for (int r = lane; r < len; r += 32) {
        const int i = map[r];
        out[r] = bp[i] < 0 ? 'L' : (i < bp[i] ? '<' : '>');
    }
}

// ---- top-50% distance seed (indialign_c/seeds.h:85-98) ---------------------
// The max(3, floor(vsum/2)) valid residues with the smallest (d2, index)
// under the running best, as one bitmask seed.
__global__ void k_topk(DevBatch b) {
    __shared__ int red_i[32];
    const int p = blockIdx.x;
    const PairInfo &I = b.info[p];
    PairState &S = b.state[p];
    if (I.status != 0) return;
    const int N = I.N, off = I.off, words = I.words;
    const double *P = b.pred + 3 * (size_t)off, *Q = b.nat + 3 * (size_t)off;
    const uint8_t *v = b.v + off;
    const double *R = S.rec[REC_BEST] + 1, *t = S.rec[REC_BEST] + 10;
    double *d2 = b.dscr + off;
    for (int i = threadIdx.x; i < N; i += blockDim.x)
        d2[i] = v[i] ? dist2(R, t, P[3 * i], P[3 * i + 1], P[3 * i + 2], Q[3 * i], Q[3 * i + 1], Q[3 * i + 2])
                     : 1e12;
    uint32_t *mb = b.bits + I.bitoff + (size_t)(kMaxBitSeeds - 1) * words;
    for (int w = threadIdx.x; w < words; w += blockDim.x) mb[w] = 0u;
    __syncthreads();
    int k = max(3, (int)(I.vsum * 0.5));
    k = min(k, N);
    int c = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        if (!v[i]) continue;
        const double di = d2[i];
        int rank = 0;
        for (int j = 0; j < N; j++)
            if (v[j] && (d2[j] < di || (d2[j] == di && j < i))) rank++;
        if (rank < k) {
            atomicOr(mb + (i >> 5), 1u << (i & 31));
            c++;
        }
    }
    c = block_sum(c, red_i);
    if (threadIdx.x == 0) {
        b.topk_seed[p] = make_int2(-1 - (kMaxBitSeeds - 1), c);
        S.topk_ok = c >= 3;
    }
}

// ---- weighted TM polish (indialign_c/core.h:218-237; update at
// indialign.cpp:258-263) ------------------------------------------------------
__global__ void k_weighted(DevBatch b) {
    const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (p >= b.n) return;
    const PairInfo &I = b.info[p];
    PairState &S = b.state[p];
    if (I.status != 0) return;
    const int N = I.N, off = I.off;
    const double *P = b.pred + 3 * (size_t)off, *Q = b.nat + 3 * (size_t)off;
    const uint8_t *v = b.v + off;
    double R[9], t[3];
    for (int a = 0; a < 9; a++) R[a] = S.rec[REC_BEST][1 + a];
    for (int a = 0; a < 3; a++) t[a] = S.rec[REC_BEST][10 + a];
    const double d0sq = fmax(I.d0 * I.d0, 1e-12);
    for (int it = 0; it < 4; it++) {
        Moments m;
        m.clear();
        for (int i = lane; i < N; i += 32) {
            if (!v[i]) continue;
            const double *pp = P + 3 * i, *qq = Q + 3 * i;
            double w = 1.0 / (1.0 + dist2(R, t, pp[0], pp[1], pp[2], qq[0], qq[1], qq[2]) / d0sq);
            if (w <= 0) continue;
            m.add_w(w, pp[0], pp[1], pp[2], qq[0], qq[1], qq[2]);
        }
        m.group_sum(32);
        kabsch_from_moments(m, 1e-12, R, t);
    }
    double s = 0.0;
    for (int i = lane; i < N; i += 32) {
        if (!v[i]) continue;
        s += 1.0 / (1.0 + dist2(R, t, P[3 * i], P[3 * i + 1], P[3 * i + 2], Q[3 * i], Q[3 * i + 1], Q[3 * i + 2]) / d0sq);
    }
    s = warp_sum(s) / fmax(I.lnorm, 1.0);
    __syncwarp();
    if (s > S.rec[REC_BEST][0]) {
        if (lane < kRec) S.rec[REC_BEST][lane] = lane == 0 ? s : (lane < 10 ? R[lane - 1] : t[lane - 10]);
    }
}

// ---- same-index rescoring: tm_score_no_d8 over the full pair
// (indialign_c/indialign.cpp:86-88) -------------------------------------------
IA_DEV double pair_tm(const DevBatch &b, const PairInfo &I, const double *rec, int lane) {
    const int N = I.N, off = I.off;
    const double *P = b.pred + 3 * (size_t)off, *Q = b.nat + 3 * (size_t)off;
    const uint8_t *v = b.v + off;
    const double *R = rec + 1, *t = rec + 10;
    const double d0sq = fmax(I.d0 * I.d0, 1e-12);
    double s = 0.0;
    for (int i = lane; i < N; i += 32)
        if (v[i]) s += 1.0 / (1.0 + dist2(R, t, P[3 * i], P[3 * i + 1], P[3 * i + 2], Q[3 * i], Q[3 * i + 1], Q[3 * i + 2]) / d0sq);
    return warp_sum(s) / fmax(I.lnorm, 1.0);
}

__global__ void k_rescore(DevBatch b, int slot, int need_flag) {
    const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (p >= b.n) return;
    const PairInfo &I = b.info[p];
    PairState &S = b.state[p];
    if (I.status != 0 || (need_flag && !S.flag)) return;
    double s = pair_tm(b, I, S.rec[slot], lane);
    __syncwarp();
    if (lane == 0) S.rec[slot][0] = s;
}

__global__ void k_rescore_list(DevBatch b, double *recs, const int *rec_pair, int nrec) {
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (r >= nrec) return;
    double *rec = recs + (size_t)r * kRec;
    if (rec[0] <= -1e299) return;
    const PairInfo &I = b.info[rec_pair[r]];
    double s = pair_tm(b, I, rec, lane);
    __syncwarp();
    if (lane == 0) rec[0] = s;
}

// ---- offset-DP starts (indialign_c/indialign.cpp:229-247) -----------------
// k = -N/2 .. N/2 step max(1, N/10), k != 0: Kabsch on pred[i] <-> native[i-k]
// over pv[i] && nv[i-k]; a start exists when >= 3 pairs.
__global__ void k_offset_starts(DevBatch b, double *starts, const int *slot_pair,
                                const int *slot_idx, int nslots) {
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (s >= nslots) return;
    const int p = slot_pair[s], o = slot_idx[s];
    const PairInfo &I = b.info[p];
    double *rec = starts + (size_t)s * kRec;
    const int N = I.N, off = I.off;
    const int stride = max(1, N / 10), lo = -N / 2;
    int k = lo + o * stride;
    if ((-lo) % stride == 0 && k >= 0) k += stride;
    if (I.status != 0 || k > N / 2) {
        if (lane == 0) rec[0] = kNegInf;
        return;
    }
    const double *P = b.pred + 3 * (size_t)off, *Q = b.nat + 3 * (size_t)off;
    const uint8_t *pv = b.pv + off, *nv = b.nv + off;
    Moments m;
    m.clear();
    for (int i = lane; i < N; i += 32) {
        int j = i - k;
        if (j < 0 || j >= N || !pv[i] || !nv[j]) continue;
        m.add(P[3 * i], P[3 * i + 1], P[3 * i + 2], Q[3 * j], Q[3 * j + 1], Q[3 * j + 2]);
    }
    m.group_sum(32);
    double R[9], t[3];
    kabsch_from_moments(m, 3.0, R, t);
    if (lane < kRec) rec[lane] = lane == 0 ? (m.w >= 3.0 ? 0.0 : kNegInf)
                                           : (lane < 10 ? R[lane - 1] : t[lane - 10]);
}

// ---- device scan of per-task chunk counts ---------------------------------
__global__ void k_scan(const int *counts, int *begins, int ntasks, ScanOut *out, int *counter) {
    __shared__ int wsum[32];
    __shared__ int carry, tile_sum;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < ntasks; base += blockDim.x) {
        const int i = base + threadIdx.x;
        int x = i < ntasks ? counts[i] : 0, inc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(kAll, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) wsum[w] = inc;
        __syncthreads();
        if (threadIdx.x == 0) {
            int s = 0;
            for (int k = 0; k < nw; k++) { int c = wsum[k]; wsum[k] = s; s += c; }
            tile_sum = s;
        }
        __syncthreads();
        const int tile_total = tile_sum;
        if (i < ntasks) begins[i] = carry + wsum[w] + inc - x;
        __syncthreads();
        if (threadIdx.x == 0) carry += tile_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out->total_chunks = carry;
        *counter = 0;
    }
}

// ---- launch wrappers ------------------------------------------------------
void launch_prep(const DevBatch &b, int use_frag, cudaStream_t st) {
    if (b.n > 0) k_prep<<<b.n, 256, 0, st>>>(b, use_frag);
}
void launch_anchor(const DevBatch &b, cudaStream_t st) {
    if (b.n > 0) k_anchor<<<b.n, 256, 0, st>>>(b);
}
void launch_ss(const DevBatch &b, cudaStream_t st) {
    if (b.n > 0) k_ss<<<2 * b.n, 32, 0, st>>>(b);
}
void launch_topk(const DevBatch &b, cudaStream_t st) {
    if (b.n > 0) k_topk<<<b.n, 256, 0, st>>>(b);
}
void launch_weighted(const DevBatch &b, cudaStream_t st) {
    if (b.n > 0) k_weighted<<<(b.n * 32 + 255) / 256, 256, 0, st>>>(b);
}
void launch_rescore(const DevBatch &b, int slot, int need_flag, cudaStream_t st) {
    if (b.n > 0) k_rescore<<<(b.n * 32 + 255) / 256, 256, 0, st>>>(b, slot, need_flag);
}
void launch_rescore_list(const DevBatch &b, double *recs, const int *rec_pair, int nrec,
                         cudaStream_t st) {
    if (nrec > 0) k_rescore_list<<<(nrec * 32 + 255) / 256, 256, 0, st>>>(b, recs, rec_pair, nrec);
}
void launch_offset_starts(const DevBatch &b, double *starts, const int *slot_pair,
                          const int *slot_idx, int nslots, cudaStream_t st) {
    if (nslots > 0)
        k_offset_starts<<<(nslots * 32 + 255) / 256, 256, 0, st>>>(b, starts, slot_pair, slot_idx, nslots);
}
void launch_scan(const int *counts, int *begins, int ntasks, ScanOut *out, int *counter,
                 cudaStream_t st) {
    k_scan<<<1, 1024, 0, st>>>(counts, begins, ntasks, out, counter);
}

}  // namespace ia

namespace ia {

// Device-resident inputs -> the packed layout (pair blocks at even offsets).
__global__ void k_repack(DevBatch b, const int *off_in, const double *pred, const double *nat,
                         const uint8_t *v, const uint8_t *pv, const uint8_t *nv) {
    const int p = blockIdx.x;
    const int N = b.len[p], si = off_in[p], so = b.off[p];
    double *dp = const_cast<double *>(b.pred) + 3 * (size_t)so;
    double *dn = const_cast<double *>(b.nat) + 3 * (size_t)so;
    for (int i = threadIdx.x; i < 3 * N; i += blockDim.x) {
        dp[i] = pred[3 * (size_t)si + i];
        dn[i] = nat[3 * (size_t)si + i];
    }
    uint8_t *dv = const_cast<uint8_t *>(b.v) + so, *dpv = const_cast<uint8_t *>(b.pv) + so;
    uint8_t *dnv = const_cast<uint8_t *>(b.nv) + so;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        dv[i] = v[si + i];
        dpv[i] = pv[si + i];
        dnv[i] = nv[si + i];
    }
}

// Running best of every pair -> out[n*13].
__global__ void k_export(DevBatch b, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.n * kRec) return;
    const int p = i / kRec, row = b.out_map ? b.out_map[p] : p;
    out[(size_t)row * kRec + i % kRec] = b.state[p].rec[REC_BEST][i % kRec];
}

void launch_repack(const DevBatch &b, const int *off_in, const double *pred, const double *nat,
                   const uint8_t *v, const uint8_t *pv, const uint8_t *nv, cudaStream_t st) {
    if (b.n > 0) k_repack<<<b.n, 256, 0, st>>>(b, off_in, pred, nat, v, pv, nv);
}

void launch_export(const DevBatch &b, double *out, cudaStream_t st) {
    if (b.n > 0) k_export<<<(b.n * kRec + 255) / 256, 256, 0, st>>>(b, out);
}

}  // namespace ia

namespace ia {

// Copy every pair's running best into snap[(p*stages + stage)*13].
__global__ void k_snapshot(DevBatch b, double *snap, int stage, int stages) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.n * kRec) return;
    const int p = i / kRec, a = i % kRec;
    snap[((size_t)p * stages + stage) * kRec + a] = b.state[p].rec[REC_BEST][a];
}

void launch_snapshot(const DevBatch &b, double *snap, int stage, int stages, cudaStream_t st) {
    if (b.n > 0 && snap) k_snapshot<<<(b.n * kRec + 255) / 256, 256, 0, st>>>(b, snap, stage, stages);
}

}  // namespace ia
