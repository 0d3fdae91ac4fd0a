// Splitting one batch over several GPUs of this process.
//
// Pairs are independent, so the split needs no data-path collective: every
// device searches its own shard with its own context and stream, and the
// results go back to the caller's arrays in batch order.  The split balances
// an estimate of each pair's device work:
//
//   cost = NW cells of the always-run passes (SS seeds, dp_refine, offset DP)
//        + seed-bank residue visits (fragment + anchor seeds x cutoffs x a
//          typical 8 passes x L), in NW-cell units (a visit costs ~0.65 of a
//          cell, from the kernels' measured rates)
//        + P(rescue) x NW cells of the local-fragment and threading-DP passes
//        + P(dense)  x NW cells of the dense local-fragment pass
//
// with the rescue window and offset counts from the reference's own
// schedules (rescue.h:12-46, 136-142; the same functions the kernels use) and
// 2 iterations x 2 gaps x plen x nlen cells per window.  The rescue passes
// are gated on the running best (< 0.5, < 0.3; indialign.cpp:129-152), which
// is not known before the search; the prior is the pair's TM-score under one
// Kabsch superposition of all valid residues (FP64, O(L) on the host), an
// estimate of where the seed bank starts: below 0.3 both passes are likely,
// below 0.5 the first is.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/indialign_b200.h"
#include "kernels.h"
#include "sched.cuh"

namespace ia {

namespace {

// Horn's quaternion Kabsch of all valid residues (the key matrix's top
// eigenvector by repeated squaring; only an estimate is needed here), then
// the same-index TM-score without the d8 filter.
double global_kabsch_tm(const NativePairInput &in) {
    const int N = in.length;
    double cp[3] = {0, 0, 0}, cq[3] = {0, 0, 0};
    int n = 0;
    for (int i = 0; i < N; i++) {
        if (!in.valid_mask[i]) continue;
        for (int d = 0; d < 3; d++) {
            cp[d] += in.pred_xyz[3 * i + d];
            cq[d] += in.native_xyz[3 * i + d];
        }
        n++;
    }
    if (n < 3) return 0.0;
    for (int d = 0; d < 3; d++) {
        cp[d] /= n;
        cq[d] /= n;
    }
    double H[3][3] = {{0}};
    for (int i = 0; i < N; i++) {
        if (!in.valid_mask[i]) continue;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                H[a][b] += (in.pred_xyz[3 * i + a] - cp[a]) * (in.native_xyz[3 * i + b] - cq[b]);
    }
    const double F[4][4] = {
        {H[0][0] + H[1][1] + H[2][2], H[1][2] - H[2][1], H[2][0] - H[0][2], H[0][1] - H[1][0]},
        {H[1][2] - H[2][1], H[0][0] - H[1][1] - H[2][2], H[0][1] + H[1][0], H[2][0] + H[0][2]},
        {H[2][0] - H[0][2], H[0][1] + H[1][0], -H[0][0] + H[1][1] - H[2][2], H[1][2] + H[2][1]},
        {H[0][1] - H[1][0], H[2][0] + H[0][2], H[1][2] + H[2][1], -H[0][0] - H[1][1] + H[2][2]}};
    // F + shift I is positive semi-definite with F's top eigenvector; its
    // 2^20-th power (repeated squaring, rescaled) is ~ v v^T
    double shift = 0.0;
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) shift += std::fabs(F[a][b]);
    double M[4][4];
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) M[a][b] = F[a][b] + (a == b ? shift : 0.0);
    for (int it = 0; it < 20; it++) {
        double S[4][4], mx = 0.0;
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                double v = 0.0;
                for (int c = 0; c < 4; c++) v += M[a][c] * M[c][b];
                S[a][b] = v;
                mx = std::max(mx, std::fabs(v));
            }
        if (!(mx > 0.0) || !std::isfinite(mx)) return 0.0;
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) M[a][b] = S[a][b] / mx;
    }
    int col = 0;
    double best = -1.0;
    for (int c = 0; c < 4; c++) {
        double nn = 0.0;
        for (int a = 0; a < 4; a++) nn += M[a][c] * M[a][c];
        if (nn > best) { best = nn; col = c; }
    }
    const double nq = std::sqrt(best);
    if (!(nq > 0.0)) return 0.0;
    const double w = M[0][col] / nq, x = M[1][col] / nq, y = M[2][col] / nq, z = M[3][col] / nq;
    // rotation taking pred onto native (row-major Rm, native ~ Rm p)
    const double Rm[3][3] = {{w * w + x * x - y * y - z * z, 2 * (x * y - w * z), 2 * (x * z + w * y)},
                            {2 * (x * y + w * z), w * w - x * x + y * y - z * z, 2 * (y * z - w * x)},
                            {2 * (x * z - w * y), 2 * (y * z + w * x), w * w - x * x - y * y + z * z}};
    const double L = in.length;
    double d0 = L >= 30 ? 0.6 * std::sqrt(L - 0.5) - 2.5 : 0.3;
    if (d0 < 0.3) d0 = 0.3;
    double s = 0.0;
    for (int i = 0; i < N; i++) {
        if (!in.valid_mask[i]) continue;
        double d2 = 0.0;
        for (int a = 0; a < 3; a++) {
            double m = 0.0;
            for (int b = 0; b < 3; b++) m += Rm[a][b] * (in.pred_xyz[3 * i + b] - cp[b]);
            const double e = m + cq[a] - in.native_xyz[3 * i + a];
            d2 += e * e;
        }
        s += 1.0 / (1.0 + d2 / (d0 * d0));
    }
    const double ln = in.lnorm > 1.0 ? in.lnorm : 1.0;
    return s / ln;
}

double pair_cost(const NativePairInput &in, double *tm0_out) {
    const int N = in.length;
    if (N <= 0) return 0.0;
    int plen = 0, nlen = 0;
    for (int i = 0; i < N; i++) {
        plen += in.pred_valid_mask[i] != 0;
        nlen += in.native_valid_mask[i] != 0;
    }
    const double cells = (double)plen * (double)nlen;
    // fragment windows of the main seed bank (+ up to 30 anchor seeds)
    int fl[9], nf = frag_lengths(N, fl), K = 1 + 30;
    for (int a = 0; a < nf; a++) K += n_starts(N, fl[a], 50);
    const double bank = 0.65 * K * 11.0 * 8.0 * N;
    // SS seeds (2 NWs + 2 dp_refines), final dp_refine, ~10 offset DPs
    const double base = 16.0 * cells;
    const double rescue = 4.0 * window_count(plen, nlen, 0) * cells + 2.0 * thread_count(plen, nlen) * cells;
    const double dense = 4.0 * window_count(plen, nlen, 1) * cells;
    const double tm0 = global_kabsch_tm(in);
    if (tm0_out) *tm0_out = tm0;
    const double p1 = tm0 < 0.5 ? 1.0 : 0.1;
    const double p2 = tm0 < 0.3 ? 1.0 : (tm0 < 0.5 ? 0.3 : 0.02);
    return bank + base + p1 * rescue + p2 * dense;
}

}  // namespace

}  // namespace ia

extern "C" {

int indialign_pair_costs(int n_pairs, const NativePairInput *inputs, double *cost, double *tm0) {
    if (n_pairs < 0 || (n_pairs > 0 && (!inputs || !cost))) return INDIALIGN_E_INPUT;
    for (int p = 0; p < n_pairs; p++) {
        const NativePairInput &in = inputs[p];
        if (in.length > 0 && (!in.pred_xyz || !in.native_xyz || !in.valid_mask || !in.pred_valid_mask ||
                              !in.native_valid_mask))
            return INDIALIGN_E_INPUT;
        double t = 0.0;
        cost[p] = ia::pair_cost(in, &t);
        if (tm0) tm0[p] = t;
    }
    return INDIALIGN_OK;
}

int indialign_shard_pairs(int n_pairs, const NativePairInput *inputs, int n_shards, int *shard_of) {
    if (n_pairs < 0 || n_shards < 1 || (n_pairs > 0 && (!inputs || !shard_of))) return INDIALIGN_E_INPUT;
    std::vector<double> cost(n_pairs);
    if (int rc = indialign_pair_costs(n_pairs, inputs, cost.data(), nullptr)) return rc;
    // longest-processing-time greedy: costliest first (ties: lower index),
    // onto the least-loaded shard (ties: lower shard)
    std::vector<int> order(n_pairs);
    for (int i = 0; i < n_pairs; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        return cost[a] != cost[b] ? cost[a] > cost[b] : a < b;
    });
    std::vector<double> load(n_shards, 0.0);
    for (int i : order) {
        int k = 0;
        for (int j = 1; j < n_shards; j++)
            if (load[j] < load[k]) k = j;
        shard_of[i] = k;
        load[k] += cost[i];
    }
    return INDIALIGN_OK;
}

int indialign_tmscore_search_multi(int n_pairs, const NativePairInput *inputs, const NativeConfig *cfg,
                                   const IndialignBatchOptions *opts, const int *devices, int n_devices,
                                   NativePairResult *outputs) {
    ia::set_last_error_text("");
    if (n_pairs < 0 || n_devices < 1 || !devices || !cfg || (n_pairs > 0 && (!inputs || !outputs))) {
        ia::set_last_error_text("search_multi: null argument or no device");
        return INDIALIGN_E_INPUT;
    }
    if (opts && (opts->stream || opts->stage_best || opts->win_feat || opts->win_label || opts->win_score ||
                 opts->win_select)) {
        ia::set_last_error_text("search_multi: per-pair outputs and a caller stream are per-device options");
        return INDIALIGN_E_INPUT;
    }
    std::vector<int> shard(n_pairs);
    if (int rc = indialign_shard_pairs(n_pairs, inputs, n_devices, shard.data())) {
        ia::set_last_error_text("search_multi: invalid pair input");
        return rc;
    }
    struct Part {
        std::vector<int> idx;
        std::vector<NativePairInput> in;
        std::vector<NativePairResult> out;
        IndialignBatchOptions o;
        double stage_ms[INDIALIGN_STAGES];
        long long counters[INDIALIGN_COUNTERS];
        double kernel_ms[6];
        long long rank_stats[INDIALIGN_RANK_STATS];
        int rc = 0;
        std::string err;
    };
    std::vector<Part> parts(n_devices);
    for (int p = 0; p < n_pairs; p++) {
        parts[shard[p]].idx.push_back(p);
        parts[shard[p]].in.push_back(inputs[p]);
    }
    for (int d = 0; d < n_devices; d++) {
        Part &P = parts[d];
        P.out.resize(P.idx.size());
        std::memset(&P.o, 0, sizeof(P.o));
        if (opts) P.o = *opts;
        P.o.device = devices[d];
        std::memset(P.stage_ms, 0, sizeof(P.stage_ms));
        std::memset(P.counters, 0, sizeof(P.counters));
        std::memset(P.kernel_ms, 0, sizeof(P.kernel_ms));
        std::memset(P.rank_stats, 0, sizeof(P.rank_stats));
        P.o.stage_ms = opts && opts->stage_ms ? P.stage_ms : nullptr;
        P.o.counters = opts && opts->counters ? P.counters : nullptr;
        P.o.kernel_ms = opts && opts->kernel_ms ? P.kernel_ms : nullptr;
        P.o.rank_stats = opts && opts->rank_stats ? P.rank_stats : nullptr;
    }
    std::vector<std::thread> th;
    for (int d = 0; d < n_devices; d++) {
        th.emplace_back([&parts, cfg, d]() {
            Part &P = parts[d];
            if (P.idx.empty()) return;
            P.rc = indialign_tmscore_search_batch_ex((int)P.in.size(), P.in.data(), cfg, &P.o, P.out.data());
            if (P.rc) P.err = indialign_last_error();
        });
    }
    for (auto &t : th) t.join();
    for (int d = 0; d < n_devices; d++) {
        if (parts[d].rc) {
            ia::set_last_error_text(("device " + std::to_string(devices[d]) + ": " + parts[d].err).c_str());
            return parts[d].rc;
        }
    }
    for (int d = 0; d < n_devices; d++) {
        const Part &P = parts[d];
        for (size_t k = 0; k < P.idx.size(); k++)
            if (inputs[P.idx[k]].length > 0) outputs[P.idx[k]] = P.out[k];
        if (opts && opts->stage_ms)  // devices run side by side: the slowest
            for (int s = 0; s < INDIALIGN_STAGES; s++)
                opts->stage_ms[s] = d == 0 ? P.stage_ms[s] : std::max(opts->stage_ms[s], P.stage_ms[s]);
        if (opts && opts->counters)
            for (int s = 0; s < INDIALIGN_COUNTERS; s++)
                opts->counters[s] = (d == 0 ? 0 : opts->counters[s]) + P.counters[s];
        if (opts && opts->kernel_ms)
            for (int s = 0; s < 6; s++) opts->kernel_ms[s] = (d == 0 ? 0.0 : opts->kernel_ms[s]) + P.kernel_ms[s];
        if (opts && opts->rank_stats)
            for (int s = 0; s < INDIALIGN_RANK_STATS; s++)
                opts->rank_stats[s] = (d == 0 ? 0 : opts->rank_stats[s]) + P.rank_stats[s];
    }
    return INDIALIGN_OK;
}

}  // extern "C"
