// Work schedules of the search, shared by host planning and device kernels:
// fragment seeds, start positions, local-fragment windows, threading and
// offset lists.  Each function restates the reference loop it counts.
#pragma once

#ifdef __CUDACC__
#define IA_HD __host__ __device__ __forceinline__
#else
#define IA_HD inline
#endif

namespace ia {

IA_HD int imin_(int a, int b) { return a < b ? a : b; }
IA_HD int imax_(int a, int b) { return a > b ? a : b; }

// fragment_lengths: {L, L/2, L/4, L/8, 64, 32, 16, 8, 4} within [4, L],
// distinct, descending (indialign_c/seeds.h:15-22).
IA_HD int frag_lengths(int L, int *out) {
    int vals[9] = {L, L / 2, L / 4, L / 8, 64, 32, 16, 8, 4}, n = 0;
    if (L < 4) return 0;
    for (int a = 0; a < 9; a++) {
        int v = vals[a];
        if (v < 4 || v > L) continue;
        bool seen = false;
        for (int b = 0; b < n; b++) seen = seen || out[b] == v;
        if (!seen) out[n++] = v;
    }
    for (int a = 1; a < n; a++)
        for (int b = a; b > 0 && out[b] > out[b - 1]; b--) {
            int t = out[b]; out[b] = out[b - 1]; out[b - 1] = t;
        }
    return n;
}

// start_positions (indialign_c/seeds.h:24-37): all starts when there are at
// most ms, else every (total/ms)-th plus the last.  Between ms and 2ms starts
// the step is 1, so the count can exceed ms.
IA_HD int n_starts(int n, int frag, int ms) {
    int total = n - frag + 1;
    if (total <= 0) return 0;
    if (total <= ms) return total;
    int step = imax_(1, total / ms);
    int cnt = (total - 1) / step + 1;
    if ((cnt - 1) * step != total - 1) cnt++;
    return cnt;
}
IA_HD int start_at(int n, int frag, int ms, int i) {
    int total = n - frag + 1;
    if (total <= ms) return i;
    int step = imax_(1, total / ms);
    int v = i * step;
    return v > total - 1 ? total - 1 : v;
}

// Seeds of an all-valid set of n points (alignment_detailed_search,
// indialign_c/align.h:33-37): the global seed, then fragment windows; each
// window has >= 4 points, so the >= 3 filter keeps all of them.
IA_HD int arith_seed_count(int n, int ms, bool use_frag) {
    if (n < 3) return 0;
    if (!use_frag) return 1;
    int fl[9], nf = frag_lengths(n, fl), K = 1;
    for (int a = 0; a < nf; a++) K += n_starts(n, fl[a], ms);
    return K;
}
IA_HD void arith_seed(int n, int ms, int k, int &s, int &len) {
    if (k == 0) { s = 0; len = n; return; }
    k -= 1;
    int fl[9], nf = frag_lengths(n, fl);
    for (int a = 0; a < nf; a++) {
        int c = n_starts(n, fl[a], ms);
        if (k < c) { s = start_at(n, fl[a], ms, k); len = fl[a]; return; }
        k -= c;
    }
    s = 0; len = 0;
}

// Offsets lo, lo+stride, ... <= hi with 0 left out (gapless threading,
// indialign_c/threading.h:50-56; offset DP, indialign.cpp:234-236).
IA_HD int offsets_count(int lo, int hi, int stride) {
    if (hi < lo) return 0;
    int c = (hi - lo) / stride + 1;
    if ((-lo) % stride == 0 && lo <= 0 && hi >= 0) c--;
    return c;
}
IA_HD int offset_at(int lo, int stride, int k) {
    int o = lo + k * stride;
    if (lo <= 0 && (-lo) % stride == 0 && o >= 0) o += stride;
    return o;
}

// Gapless threading parameters (indialign_c/threading.h:48-53); plen/nlen
// there are byte sums of the masks.
IA_HD void gapless_params(int N, int pvsum, int nvsum, int &kr, int &stride, int &min_ali) {
    min_ali = imax_(3, imin_(pvsum, nvsum) / 2);
    kr = N - min_ali;
    stride = kr > 0 ? imax_(1, (2 * kr + 99) / 100) : 1;
}

// Local fragment window schedule (indialign_c/rescue.h:12-46, 65-78).
IA_HD int local_frag_lengths(int plen, int nlen, int dense, int *out) {
    int ml = imin_(plen, nlen), n = 0;
    if (ml < 4) return 0;
    if (dense) {
        int vals[9] = {ml, imin_(100, ml / 2), imin_(32, ml), imin_(24, ml), imin_(20, ml / 3), 16, 12, 8, 4};
        for (int a = 0; a < 9; a++) {
            if (vals[a] < 4) continue;
            bool seen = false;
            for (int b = 0; b < n; b++) seen = seen || out[b] == vals[a];
            if (!seen) out[n++] = vals[a];
        }
    } else {
        int a = imin_(20, ml / 3), b = imin_(100, ml / 2);
        if (a >= 4) out[n++] = a;
        if (b >= 4 && b != a) out[n++] = b;
    }
    return n;
}

IA_HD int local_jump(int length, int dense) {
    int j;
    if (dense) {
        if (length > 350) j = 50;
        else if (length > 300) j = 30;
        else if (length > 200) j = 10;
        else j = 5;
        return imax_(1, imin_(j, imax_(1, length / 4)));
    }
    if (length > 250) j = 45;
    else if (length > 200) j = 35;
    else if (length > 150) j = 25;
    else j = 15;
    return imax_(1, imin_(j, imax_(1, length / 3)));
}

IA_HD int window_count(int plen, int nlen, int dense) {
    int fl[9], nf = local_frag_lengths(plen, nlen, dense, fl);
    int jp = local_jump(plen, dense), jn = local_jump(nlen, dense), W = 0;
    for (int a = 0; a < nf; a++) {
        int plim = plen - fl[a] + 1, nlim = nlen - fl[a] + 1;
        if (plim <= 0 || nlim <= 0) continue;
        W += ((plim + jp - 1) / jp) * ((nlim + jn - 1) / jn);
    }
    return W;
}

IA_HD void window_at(int plen, int nlen, int dense, int w, int &flen, int &ps, int &ns) {
    int fl[9], nf = local_frag_lengths(plen, nlen, dense, fl);
    int jp = local_jump(plen, dense), jn = local_jump(nlen, dense);
    flen = 0; ps = ns = 0;
    for (int a = 0; a < nf; a++) {
        int plim = plen - fl[a] + 1, nlim = nlen - fl[a] + 1;
        if (plim <= 0 || nlim <= 0) continue;
        int cp = (plim + jp - 1) / jp, cn = (nlim + jn - 1) / jn;
        if (w < cp * cn) {
            flen = fl[a];
            ps = (w / cn) * jp;
            ns = (w % cn) * jn;
            return;
        }
        w -= cp * cn;
    }
}

// Threading-DP offsets -(nlen-3) .. plen-3 step max(1, min/50)
// (indialign_c/rescue.h:136-142).
IA_HD int thread_count(int plen, int nlen) {
    if (imin_(plen, nlen) < 3) return 0;
    int step = imax_(1, imin_(plen, nlen) / 50);
    int lo = -(nlen - 3), hi = plen - 3;  // offset < plen-2
    if (hi < lo) return 0;
    return (hi - lo) / step + 1;
}
IA_HD void thread_at(int plen, int nlen, int o, int &ps, int &ns, int &ov) {
    int step = imax_(1, imin_(plen, nlen) / 50);
    int off = -(nlen - 3) + o * step;
    ps = imax_(off, 0);
    ns = imax_(-off, 0);
    ov = imin_(plen - ps, nlen - ns);
}

// Ranked candidates of a kind (pipeline.h CandKind): windows, or threading
// offsets as the segment of their overlap.
IA_HD int cand_count(int kind, int plen, int nlen) {
    if (kind == 3) return arith_seed_count(imin_(plen, nlen), 50, true);
    return kind == 1 ? thread_count(plen, nlen) : window_count(plen, nlen, kind == 2 ? 1 : 0);
}
IA_HD void cand_at(int kind, int plen, int nlen, int i, int &flen, int &ps, int &ns) {
    if (kind == 3) {  // detailed-search seed on an aligned set of plen == nlen points
        arith_seed(plen, 50, i, ps, flen);
        ns = ps;
    } else if (kind == 1) {
        thread_at(plen, nlen, i, ps, ns, flen);
    } else {
        window_at(plen, nlen, kind == 2 ? 1 : 0, i, flen, ps, ns);
    }
}

// Offset-DP starts: k = -N/2 .. N/2 step max(1, N/10), k != 0
// (indialign_c/indialign.cpp:234-236).
IA_HD int offdp_count(int N) { return offsets_count(-N / 2, N / 2, imax_(1, N / 10)); }

}  // namespace ia
