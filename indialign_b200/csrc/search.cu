// Host side of the search: the C ABI, a pool of per-call contexts (stream +
// grow-only device workspace), packing of host inputs into the device
// layout, static result layouts, and the fixed launch sequence that restates
// do_tmscore_search (indialign_c/indialign.cpp:29-266) stage by stage for a
// whole batch.  All arithmetic runs in the kernels; the host only packs,
// plans capacities once per batch and launches.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/indialign_b200.h"
#include "kernels.h"
#include "sched.cuh"

namespace ia {

static thread_local std::string g_last_error;
static std::atomic<int> g_inject{0};

static void set_error(const char *what, cudaError_t e) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
}

void set_last_error_text(const char *msg) { g_last_error = msg; }

#define CK(x)                                 \
    do {                                      \
        cudaError_t e_ = (x);                 \
        if (e_ != cudaSuccess) {              \
            set_error(#x, e_);                \
            return INDIALIGN_E_CUDA;          \
        }                                     \
    } while (0)

// Grow-only device buffer with 64 bytes of tail padding, zeroed when it
// grows.  The zeroing runs on the legacy default stream, which does not order
// against the library's non-blocking streams, so it is waited for here:
// otherwise it could land after the stream's first upload into the buffer.
template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = n < 16 ? 16 : n + n / 8;
        cudaError_t e = cudaMalloc(&p, want * sizeof(T) + 64);
        if (e != cudaSuccess) return e;
        cap = want;
        e = cudaMemset(p, 0, want * sizeof(T) + 64);
        if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
        return e;
    }
};

// Static per-stage slot layout (uploaded once per batch).
struct Layout {
    int ntasks = 0;
    std::vector<int> pair, aux;
    std::vector<long long> base;
    long long total = 0;  // result records / items
    const int *d_pair = nullptr, *d_aux = nullptr;
    const long long *d_base = nullptr;
};

struct Ctx {
    int device = 0;
    int tag = 0;  // the kind of batch it last served (length bucket + 1, 0: whole batches)
    cudaStream_t stream = nullptr;
    int sms = 148;
    DBuf<int> off, len, bitoff, err;
    DBuf<double> lnorm, pred, nat, dscr, predc, natc;
    DBuf<uint8_t> v, pv, nv;
    DBuf<char> sspc, ssnc;
    DBuf<PairInfo> info;
    DBuf<PairState> state;
    DBuf<int> pmap, nmap, vmap, scratch, kv;
    DBuf<int2> seeds, topk;
    DBuf<uint32_t> bits, gtrace, gal;
    DBuf<uint64_t> hashes, fnv_pow;
    DBuf<BankTask> btasks;
    DBuf<ChainTask> ctasks;
    DBuf<int> counts, begins, counter;
    DBuf<ScanOut> scan;
    DBuf<double> item_res, chain_res, alP, alQ, thread_rec, off_start, off_res, gbh, out, snap;
    DBuf<int> lay_i, gidx, omap;
    DBuf<long long> lay_l;
    DBuf<unsigned long long> ctr;
    // learned window ranker
    DBuf<float> blob, wscore, wfeat, wlabel;
    DBuf<MlpPacked> mlp;
    DBuf<int> wcount, wlist, wsel;
    DBuf<unsigned long long> rstats;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<double> h_pred, h_nat, h_lnorm;
    std::vector<uint8_t> h_v, h_pv, h_nv;
    std::vector<int> h_off, h_len, h_bitoff;
    int fnv_n = 0;
};

static std::mutex g_pool_mu;
static std::vector<Ctx *> g_pool;
static std::once_flag g_attr_once[64];

// Stream priority of a context serving `tag`: a length-bucket sub-batch (tag
// = bucket + 1) gets a priority that grows with the bucket's lengths.  The
// sub-batches of one call run side by side and the longest pairs are their
// critical path, so their pending work is scheduled first whenever SMs free
// up; whole batches (tag 0) get the default.
static int stream_priority(int tag) {
    int least = 0, greatest = 0;
    if (tag <= 0 || cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess || greatest >= least)
        return 0;
    return std::max(greatest, least - (tag - 1) * std::max(1, (least - greatest) / 2));
}

// A pooled context of `device`, preferring one that last served the same
// kind of batch (`tag`), so that its grow-only buffers already fit; a
// context taken over from another tag gets a stream of this tag's priority.
static int acquire(int device, Ctx **out, int tag = 0) {
    if (device < 0) CK(cudaGetDevice(&device));
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        long pick = -1;
        for (size_t i = 0; i < g_pool.size(); i++)
            if (g_pool[i]->device == device && (pick < 0 || g_pool[i]->tag == tag)) {
                pick = (long)i;
                if (g_pool[i]->tag == tag) break;
            }
        if (pick >= 0) {
            Ctx *c = g_pool[pick];
            g_pool.erase(g_pool.begin() + pick);
            CK(cudaSetDevice(device));
            if (c->tag != tag) {  // its stream is idle: the last call synchronized it
                int prio = 0;
                CK(cudaStreamGetPriority(c->stream, &prio));
                if (prio != stream_priority(tag)) {
                    CK(cudaStreamDestroy(c->stream));
                    CK(cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, stream_priority(tag)));
                }
            }
            c->tag = tag;
            *out = c;
            return INDIALIGN_OK;
        }
    }
    CK(cudaSetDevice(device));
    Ctx *c = new Ctx();
    c->device = device;
    c->tag = tag;
    CK(cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, stream_priority(tag)));
    CK(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device));
    cudaError_t attr_err = cudaSuccess;
    std::call_once(g_attr_once[device & 63], [&]() {
        attr_err = bank_set_attributes();
        if (attr_err == cudaSuccess) attr_err = chain_set_attributes();
        if (attr_err == cudaSuccess) attr_err = rank_set_attributes();
    });
    CK(attr_err);
    *out = c;
    return INDIALIGN_OK;
}

static void release(Ctx *c) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    g_pool.push_back(c);
}

// detailed-search items bound: max over n' <= n of seeds(n') x 6
static std::vector<int> g_kdet;
static int kdet_max(int n) {
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)g_kdet.size() <= n) {
        int start = (int)g_kdet.size();
        g_kdet.resize(n + 1);
        for (int m = start; m <= n; m++) {
            int v = arith_seed_count(m, 50, true);
            g_kdet[m] = m > 0 ? (v > g_kdet[m - 1] ? v : g_kdet[m - 1]) : v;
        }
    }
    return g_kdet[n];
}

constexpr int kTrace = INDIALIGN_TRACE_STAGES;

struct Cfg {
    int use_frag, max_iter, dp_iter;
    double r1, r2, early;
    // dense-rescue mode (INDIALIGN_MODE_*) and ranker selection parameters
    int mode = INDIALIGN_MODE_PLAIN, top_k = 8, rank_mask = INDIALIGN_RANK_DEFAULT,
        min_len = INDIALIGN_RANK_MIN_LEN;
    double margin = 0.02, audit = 0.02;
    unsigned long long seed = 0;
    TuneRows tune;              // kernel shapes per length bucket (per task)
    int chain_smem_trace = 1;  // NW traces in shared memory (the longest pair's bucket)
};

// Host view of per-pair facts after k_prep / k_anchor.
struct Plan {
    std::vector<PairInfo> info;
};

class Runner {
  public:
    Runner(Ctx *c, const Cfg &cfg, int n) : c_(c), cfg_(cfg), n_(n) {}
    ~Runner() { recycle(); }  // events go back to the context's pool on every exit path
    Runner(const Runner &) = delete;
    Runner &operator=(const Runner &) = delete;
    long long windows() const { return koff_[kCandKinds]; }
    int *sel_out = nullptr;  // device copy of each pass's selection (LEARNED, win_select)
    long long cand_offset(int kind) const { return koff_[kind]; }
    bool use_mlp = false;

    int build_layouts(const std::vector<PairInfo> &info);
    int run_stages();
    DevBatch b;
    double *snap = nullptr;  // device [n*kTrace*13] or nullptr
    void mark(int stage) {
        launch_snapshot(b, snap, stage, kTrace, c_->stream);
        if (snap) launches_++;
        stage_event(stage + 1);
    }
    // timing: events at stage boundaries and around every chain / bank launch
    bool timing = false;
    std::vector<std::pair<int, cudaEvent_t>> stage_ev;     // (boundary id, event)
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> chain_ev, bank_ev, rank_ev;
    long long launches_ = 0, chain_launches_ = 0, bank_launches_ = 0, rank_launches_ = 0;
    cudaEvent_t new_event() {
        cudaEvent_t e = nullptr;
        if (!c_->ev_pool.empty()) {
            e = c_->ev_pool.back();
            c_->ev_pool.pop_back();
        } else {
            cudaEventCreate(&e);
        }
        return e;
    }
    void stage_event(int id) {
        if (!timing) return;
        cudaEvent_t e = new_event();
        cudaEventRecord(e, c_->stream);
        stage_ev.push_back({id, e});
    }
    void recycle() {
        for (auto &x : stage_ev) c_->ev_pool.push_back(x.second);
        for (auto &x : chain_ev) { c_->ev_pool.push_back(x.first); c_->ev_pool.push_back(x.second); }
        for (auto &x : bank_ev) { c_->ev_pool.push_back(x.first); c_->ev_pool.push_back(x.second); }
        for (auto &x : rank_ev) { c_->ev_pool.push_back(x.first); c_->ev_pool.push_back(x.second); }
        stage_ev.clear(); chain_ev.clear(); bank_ev.clear(); rank_ev.clear();
    }
    int pmax = 0, nmax = 0, Nmax = 0;

  private:
    int bank(int kind, Layout &L, double *recs = nullptr, int set_iter = -1, double early = -1,
             const int *wcount = nullptr, const int *wlist = nullptr);
    int chain(int kind, Layout &L, int iters, double *recs = nullptr, double *recs2 = nullptr,
              bool reduce = true, const int *wcount = nullptr, const int *wlist = nullptr);
    int rank_stage(int kind, int det_ss = 0);
    RankArgs rank_args(int kind, int det_ss);
    SelectArgs select_args(int kind, int det_ss);
    int after_stage(int kind, const CandRes &r, int det_ss = 0);
    int ntasks(int kind) const { return kind == CAND_DET ? kDetSlots * n_ : n_; }
    // first selection row of a kind in the win_select output (kinds back to back)
    long long sel_row(int kind) const {
        return kind == CAND_MAIN ? 5LL * n_ : (kind == CAND_DET ? 3LL * n_ : (long long)kind * n_);
    }
    // ranked candidate lists this call: bit of INDIALIGN_RANK_* per pass
    int rank_bit(int kind, int det_ss) const {
        if (kind == CAND_MAIN) return INDIALIGN_RANK_MAIN;
        return kind == CAND_DET ? (det_ss ? INDIALIGN_RANK_DET_SS : INDIALIGN_RANK_DET_DP) : (1 << kind);
    }
    bool ranked(int kind, int det_ss = 0) const {
        return cfg_.mode != INDIALIGN_MODE_PLAIN && (cfg_.rank_mask & rank_bit(kind, det_ss)) != 0;
    }
    const int *sel_count(int kind, int det_ss = 0) const {
        return cfg_.mode == INDIALIGN_MODE_LEARNED && ranked(kind, det_ss) ? c_->wcount.p : nullptr;
    }
    const int *sel_list(int kind, int det_ss = 0) const {
        return cfg_.mode == INDIALIGN_MODE_LEARNED && ranked(kind, det_ss) ? c_->wlist.p : nullptr;
    }
    int glue(int op, double thr = 0.0, const double *recs = nullptr, const int *idx = nullptr);
    int dp_full(int det_ss);

    Ctx *c_;
    Cfg cfg_;
    int n_;
    Layout L_pair, L_main, L_detss, L_detdp, L_gapless, L_thread, L_topk, L_localn, L_locald,
        L_threadch, L_single, L_offdp, L_offslots, L_cand[kCandKinds];
    long long koff_[kCandKinds + 1] = {0, 0, 0, 0, 0, 0};
    long long max_items_ = 0, max_chain_recs_ = 0, n_thread_ = 0, n_off_ = 0;
    int chain_grid_ = 0, chain_flags_ = 0, rank_grid_ = 1;
    size_t trace_words_ = 0;
};

static void finish_layout(Layout &L) {
    L.ntasks = (int)L.base.size();
    long long acc = 0;
    for (auto &x : L.base) {
        long long cnt = x;
        x = acc;
        acc += cnt;
    }
    L.total = acc;
}

int Runner::build_layouts(const std::vector<PairInfo> &info) {
    const int n = n_;
    auto perpair = [&](Layout &L, auto count) {
        L.base.resize(n);
        for (int p = 0; p < n; p++) L.base[p] = info[p].status ? 0 : count(info[p]);
        finish_layout(L);
    };
    L_pair.base.assign(0, 0);
    L_pair.ntasks = n;
    perpair(L_main, [](const PairInfo &I) { return (long long)I.K * I.C; });
    perpair(L_detss, [](const PairInfo &I) {
        int m = I.plen < I.nlen ? I.plen : I.nlen;
        return (long long)kdet_max(m) * kDetC;
    });
    L_detdp.base.resize(2 * n);
    L_detdp.pair.resize(2 * n);
    L_detdp.aux.resize(2 * n);
    for (int p = 0; p < n; p++)
        for (int g = 0; g < 2; g++) {
            const PairInfo &I = info[p];
            int m = I.plen < I.nlen ? I.plen : I.nlen;
            L_detdp.pair[2 * p + g] = p;
            L_detdp.aux[2 * p + g] = g;
            L_detdp.base[2 * p + g] = I.status ? 0 : (long long)kdet_max(m) * kDetC;
        }
    finish_layout(L_detdp);
    perpair(L_gapless, [](const PairInfo &I) {
        int kr, st, ma;
        gapless_params(I.N, I.pvsum, I.nvsum, kr, st, ma);
        return (long long)(kr > 0 ? offsets_count(-kr, kr, st) : 0);
    });
    perpair(L_topk, [](const PairInfo &I) { return (long long)I.C; });
    // threading-DP: one bank slot per (pair, offset)
    L_thread.pair.clear();
    L_thread.aux.clear();
    L_thread.base.clear();
    L_threadch.base.resize(n);
    L_threadch.aux.resize(n);
    for (int p = 0; p < n; p++) {
        const PairInfo &I = info[p];
        int cnt = I.status ? 0 : thread_count(I.plen, I.nlen);
        L_threadch.aux[p] = (int)L_thread.pair.size();
        L_threadch.base[p] = 2LL * cnt;
        for (int o = 0; o < cnt; o++) {
            int ps, ns, ov;
            thread_at(I.plen, I.nlen, o, ps, ns, ov);
            L_thread.pair.push_back(p);
            L_thread.aux.push_back(o);
            L_thread.base.push_back(ov >= 3 ? (long long)arith_seed_count(ov, 5, true) * kDetC : 0);
        }
    }
    finish_layout(L_thread);
    finish_layout(L_threadch);
    n_thread_ = L_thread.ntasks;
    perpair(L_localn, [](const PairInfo &I) { return 2LL * window_count(I.plen, I.nlen, 0); });
    perpair(L_locald, [](const PairInfo &I) { return 2LL * window_count(I.plen, I.nlen, 1); });
    perpair(L_single, [](const PairInfo &) { return 2LL; });
    // ranked candidates of every pair (degenerate ones included, so that
    // callers can lay out per-candidate outputs from the valid counts alone),
    // kinds back to back
    for (int k = 0; k < kCandKinds; k++) {
        if (k == CAND_DET) {  // kDetSlots alignment slots per pair, each sized for the largest aligned set
            L_cand[k].base.resize((size_t)kDetSlots * n);
            for (int p = 0; p < n; p++) {
                const int m = info[p].plen < info[p].nlen ? info[p].plen : info[p].nlen;
                for (int g = 0; g < kDetSlots; g++) L_cand[k].base[(size_t)kDetSlots * p + g] = kdet_max(m);
            }
        } else if (k == CAND_MAIN) {  // room for the largest seed table
            L_cand[k].base.assign(n, (long long)kMaxSeeds);
        } else {
            L_cand[k].base.resize(n);
            for (int p = 0; p < n; p++) L_cand[k].base[p] = cand_count(k, info[p].plen, info[p].nlen);
        }
        finish_layout(L_cand[k]);
        koff_[k + 1] = koff_[k] + L_cand[k].total;
    }
    // offset DP: start slots per (pair, offset)
    L_offdp.base.resize(n);
    L_offdp.aux.resize(n);
    L_offslots.pair.clear();
    L_offslots.aux.clear();
    for (int p = 0; p < n; p++) {
        const PairInfo &I = info[p];
        int cnt = I.status ? 0 : offdp_count(I.N);
        L_offdp.aux[p] = (int)L_offslots.pair.size();
        L_offdp.base[p] = 2LL * cnt;
        for (int o = 0; o < cnt; o++) {
            L_offslots.pair.push_back(p);
            L_offslots.aux.push_back(o);
        }
    }
    finish_layout(L_offdp);
    L_offslots.ntasks = (int)L_offslots.pair.size();
    n_off_ = L_offslots.ntasks;
    for (Layout *L : {&L_main, &L_detss, &L_detdp, &L_gapless, &L_thread, &L_topk})
        max_items_ = L->total > max_items_ ? L->total : max_items_;
    for (Layout *L : {&L_localn, &L_locald, &L_threadch, &L_single, &L_offdp})
        max_chain_recs_ = L->total > max_chain_recs_ ? L->total : max_chain_recs_;
    // upload all layouts into one int and one long long arena
    size_t ni = 0, nl = 0;
    for (Layout *L : {&L_pair, &L_main, &L_detss, &L_detdp, &L_gapless, &L_thread, &L_topk,
                      &L_localn, &L_locald, &L_threadch, &L_single, &L_offdp, &L_offslots,
                      &L_cand[0], &L_cand[1], &L_cand[2], &L_cand[3], &L_cand[4]}) {
        ni += L->pair.size() + L->aux.size();
        nl += L->base.size();
    }
    CK(c_->lay_i.ensure(ni + 1));
    CK(c_->lay_l.ensure(nl + 1));
    std::vector<int> hi;
    std::vector<long long> hl;
    hi.reserve(ni);
    hl.reserve(nl);
    for (Layout *L : {&L_pair, &L_main, &L_detss, &L_detdp, &L_gapless, &L_thread, &L_topk,
                      &L_localn, &L_locald, &L_threadch, &L_single, &L_offdp, &L_offslots,
                      &L_cand[0], &L_cand[1], &L_cand[2], &L_cand[3], &L_cand[4]}) {
        L->d_pair = L->pair.empty() ? nullptr : c_->lay_i.p + hi.size();
        hi.insert(hi.end(), L->pair.begin(), L->pair.end());
        L->d_aux = L->aux.empty() ? nullptr : c_->lay_i.p + hi.size();
        hi.insert(hi.end(), L->aux.begin(), L->aux.end());
        L->d_base = L->base.empty() ? nullptr : c_->lay_l.p + hl.size();
        hl.insert(hl.end(), L->base.begin(), L->base.end());
        if (L->ntasks == 0 && !L->pair.empty()) L->ntasks = (int)L->pair.size();
    }
    if (!hi.empty())
        CK(cudaMemcpyAsync(c_->lay_i.p, hi.data(), hi.size() * sizeof(int), cudaMemcpyHostToDevice,
                           c_->stream));
    if (!hl.empty())
        CK(cudaMemcpyAsync(c_->lay_l.p, hl.data(), hl.size() * sizeof(long long),
                           cudaMemcpyHostToDevice, c_->stream));
    // stage buffers
    int maxtasks = n > 0 ? 2 * n : 1;
    if (L_thread.ntasks > maxtasks) maxtasks = L_thread.ntasks;
    CK(c_->btasks.ensure(maxtasks));
    CK(c_->ctasks.ensure(maxtasks));
    CK(c_->counts.ensure(maxtasks));
    CK(c_->begins.ensure(maxtasks));
    CK(c_->scan.ensure(1));
    CK(c_->counter.ensure(1));
    CK(c_->item_res.ensure((size_t)(max_items_ > 0 ? max_items_ : 1) * kRec));
    CK(c_->chain_res.ensure((size_t)(max_chain_recs_ > 0 ? max_chain_recs_ : 1) * kRec));
    CK(c_->thread_rec.ensure((size_t)(n_thread_ > 0 ? n_thread_ : 1) * kRec));
    CK(c_->off_start.ensure((size_t)(n_off_ > 0 ? n_off_ : 1) * kRec));
    CK(c_->off_res.ensure((size_t)(n_off_ > 0 ? n_off_ : 1) * kRec));
    // chain kernel scratch: trace blocks per resident warp
    pmax = nmax = 1;
    for (auto &I : info) {
        if (I.plen > pmax) pmax = I.plen;
        if (I.nlen > nmax) nmax = I.nlen;
    }
    chain_flags_ = 0;
    if ((size_t)nmax * 17 + pmax + 256 <= 96 * 1024) chain_flags_ |= 1;
    if (nmax <= 512) chain_flags_ |= 2;
    if ((pmax < nmax ? pmax : nmax) <= 2048) chain_flags_ |= 4;
    size_t smem = chain_smem_bytes(pmax, nmax, chain_flags_);
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chain_kernel_ptr(), 32 * kChainWarps,
                                                     smem));
    if (per_sm < 1) per_sm = 1;
    trace_words_ = nw_trace_words_for(pmax, nmax);  // NW trace block per warp (k_chain.cu)
    // short pairs: the warps' traces in shared memory, when that keeps the
    // number of resident CTAs
    if (cfg_.chain_smem_trace) {
        const size_t with = chain_smem_bytes(pmax, nmax, chain_flags_ | 8);
        int per_sm8 = 0;
        if (with <= kChainSmemMax &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm8, chain_kernel_ptr(), 32 * kChainWarps,
                                                          with) == cudaSuccess &&
            per_sm8 >= per_sm) {
            chain_flags_ |= 8;
            smem = with;
        }
        cudaGetLastError();
    }
    long long warps = (long long)c_->sms * per_sm * kChainWarps;
    const size_t budget = (size_t)4 << 30;  // trace scratch budget
    long long cap = (long long)(budget / (trace_words_ * 4 + 1));
    if (warps > cap) warps = cap < kChainWarps ? kChainWarps : cap;
    chain_grid_ = (int)(warps / kChainWarps);
    if (chain_grid_ < 1) chain_grid_ = 1;
    size_t nw = (size_t)chain_grid_ * kChainWarps;
    CK(c_->gtrace.ensure((chain_flags_ & 8) ? 1 : nw * trace_words_));
    CK(c_->gbh.ensure((chain_flags_ & 2) ? 1 : nw * (nmax + 1)));
    CK(c_->gal.ensure((chain_flags_ & 4) ? 1 : nw * (pmax < nmax ? pmax : nmax)));
    CK(c_->alP.ensure(3 * 2 * (size_t)(c_->h_off.empty() ? 1 : c_->h_off.back() + 2)));
    CK(c_->alQ.ensure(3 * 2 * (size_t)(c_->h_off.empty() ? 1 : c_->h_off.back() + 2)));
    if (cfg_.mode != INDIALIGN_MODE_PLAIN) {
        const size_t nw = (size_t)(windows() > 0 ? windows() : 1);
        CK(c_->wscore.ensure(nw));
        CK(c_->wcount.ensure((size_t)kDetSlots * (n > 0 ? n : 1)));
        CK(c_->wlist.ensure((size_t)kDetSlots * (n > 0 ? n : 1) * kMaxTopK));
        CK(c_->rstats.ensure(kCandKinds * kRankStats));
        if (cfg_.mode == INDIALIGN_MODE_COLLECT) {
            CK(c_->wfeat.ensure(nw * kFeatures));
            CK(c_->wlabel.ensure(nw));
        }
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rank_kernel_ptr(), 128, rank_smem_bytes()));
        rank_grid_ = c_->sms * (per_sm > 0 ? per_sm : 1);
    }
    return INDIALIGN_OK;
}

int Runner::bank(int kind, Layout &L, double *recs, int set_iter, double early, const int *wcount,
                 const int *wlist) {
    if (L.ntasks <= 0) return INDIALIGN_OK;
    PlanCtx pc = {};
    pc.kind = kind;
    pc.ntasks = L.ntasks;
    pc.pair = L.d_pair;
    pc.aux = L.d_aux;
    pc.base = L.d_base;
    pc.btasks = c_->btasks.p;
    pc.counts = c_->counts.p;
    pc.alP = c_->alP.p;
    pc.alQ = c_->alQ.p;
    pc.recs = recs;
    pc.max_iter = set_iter >= 0 ? set_iter : cfg_.max_iter;
    pc.early_term = early >= 0 ? early : cfg_.early;
    pc.wcount = wcount;
    pc.wlist = wlist;
    pc.tune = cfg_.tune;
    launch_plan_bank(b, pc, c_->stream);
    launch_scan(c_->counts.p, c_->begins.p, L.ntasks, c_->scan.p, c_->counter.p, c_->stream);
    launches_ += 4;
    bank_launches_++;
    int nmx = Nmax;
    size_t sm = bank_smem_bytes(nmx);
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bank_kernel_ptr(sm <= kBankSmemMax),
                                                     kBankChunk, sm <= kBankSmemMax ? sm : 0));
    if (per_sm < 1) per_sm = 1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (timing) {
        e0 = new_event();
        e1 = new_event();
        cudaEventRecord(e0, c_->stream);
    }
    launch_bank(c_->btasks.p, c_->begins.p, L.ntasks, c_->scan.p, c_->counter.p, c_->item_res.p,
                c_->err.p, nmx, c_->sms * per_sm, b.ctr, c_->stream);
    if (timing) {
        cudaEventRecord(e1, c_->stream);
        bank_ev.push_back({e0, e1});
    }
    launch_reduce_bank(c_->btasks.p, L.ntasks, c_->item_res.p, b.state, c_->stream);
    CK(cudaGetLastError());
    return INDIALIGN_OK;
}

int Runner::chain(int kind, Layout &L, int iters, double *recs, double *recs2, bool reduce,
                  const int *wcount, const int *wlist) {
    if (L.ntasks <= 0) return INDIALIGN_OK;
    PlanCtx pc = {};
    pc.kind = kind;
    pc.ntasks = L.ntasks;
    pc.pair = L.d_pair;
    pc.aux = L.d_aux;
    pc.base = L.d_base;
    pc.ctasks = c_->ctasks.p;
    pc.counts = c_->counts.p;
    pc.alP = c_->alP.p;
    pc.alQ = c_->alQ.p;
    pc.chain_res = c_->chain_res.p;
    pc.recs = recs;
    pc.recs2 = recs2;
    pc.iters = iters;
    pc.wcount = wcount;
    pc.wlist = wlist;
    pc.tune = cfg_.tune;
    launch_plan_chain(b, pc, c_->stream);
    launch_scan(c_->counts.p, c_->begins.p, L.ntasks, c_->scan.p, c_->counter.p, c_->stream);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (timing) {
        e0 = new_event();
        e1 = new_event();
        cudaEventRecord(e0, c_->stream);
    }
    const bool emit = kind == CH_SS2 || kind == CH_SS4 || kind == CH_DP_EMIT;
    launch_chain(b, c_->ctasks.p, c_->begins.p, L.ntasks, c_->scan.p, c_->counter.p, c_->gtrace.p,
                 trace_words_, c_->gbh.p, c_->gal.p, pmax, nmax, chain_flags_, chain_grid_, emit,
                 c_->stream);
    if (timing) {
        cudaEventRecord(e1, c_->stream);
        chain_ev.push_back({e0, e1});
    }
    if (reduce) launch_reduce_chain(b, pc, c_->stream);
    launches_ += reduce ? 4 : 3;
    chain_launches_++;
    CK(cudaGetLastError());
    return INDIALIGN_OK;
}

int Runner::glue(int op, double thr, const double *recs, const int *idx) {
    GlueArgs a = {};
    a.op = op;
    a.thr = thr;
    a.dp_iter = cfg_.dp_iter;
    a.recs = recs;
    a.idx = idx;
    launch_glue(b, a, c_->stream);
    launches_++;
    CK(cudaGetLastError());
    return INDIALIGN_OK;
}

// Where a detailed search's seed items are: the bank's items and tasks.
// Item records of the bank launch just run; per_pair: its tasks are one per
// pair (the SS seeds' detailed search) rather than one per alignment slot.
static CandRes det_res(Ctx *c, int per_pair = 0) {
    return CandRes{nullptr, nullptr, nullptr, nullptr, c->item_res.p, c->btasks.p, per_pair};
}

// dp_refine with fragment detailed searches (indialign_c/align.h:54-145,
// d0_search_lite = false): per iteration one NW per gap chain, then the
// detailed bank on each alignment, then the per-chain update.
int Runner::dp_full(int det_ss) {
    int rc;
    for (int it = 0; it < cfg_.dp_iter; it++) {
        if ((rc = chain(CH_DP_EMIT, L_pair, 1, nullptr, nullptr, false))) return rc;
        if ((rc = rank_stage(CAND_DET, det_ss))) return rc;
        if ((rc = bank(BK_DET_DP, L_detdp, nullptr, -1, -1, sel_count(CAND_DET, det_ss),
                       sel_list(CAND_DET, det_ss))))
            return rc;
        if ((rc = after_stage(CAND_DET, det_res(c_), det_ss))) return rc;
        if ((rc = glue(G_DP_STEP))) return rc;
    }
    return glue(G_DP_END);
}

// Candidate ranking of one rescue pass (pipeline.h CandKind) for the pairs
// its gate let in.  PLAIN: nothing.  LEARNED: features + MLP scores, then the
// per-pair selection the pass's plan reads (wcount / wlist).  COLLECT: the
// features of every candidate.
RankArgs Runner::rank_args(int kind, int det_ss) {
    RankArgs ra;
    ra.mlp = use_mlp ? c_->mlp.p : nullptr;
    ra.wbase = L_cand[kind].d_base;
    ra.score = c_->wscore.p + koff_[kind];
    ra.feat = cfg_.mode == INDIALIGN_MODE_COLLECT ? c_->wfeat.p + koff_[kind] * kFeatures : nullptr;
    ra.kind = kind;
    ra.ntasks = ntasks(kind);
    ra.det_ss = det_ss;
    ra.alP = c_->alP.p;
    ra.alQ = c_->alQ.p;
    ra.min_len = cfg_.mode == INDIALIGN_MODE_LEARNED ? cfg_.min_len : 0;
    return ra;
}

int Runner::rank_stage(int kind, int det_ss) {
    if (!ranked(kind, det_ss)) return INDIALIGN_OK;
    cudaStream_t st = c_->stream;
    const RankArgs ra = rank_args(kind, det_ss);
    if (kind == CAND_DET || kind == CAND_MAIN) {  // hold this search only (NaN beyond its seeds)
        CK(cudaMemsetAsync(c_->wscore.p + koff_[kind], 0xff, (size_t)L_cand[kind].total * sizeof(float), st));
        if (cfg_.mode == INDIALIGN_MODE_COLLECT)
            CK(cudaMemsetAsync(c_->wlabel.p + koff_[kind], 0xff, (size_t)L_cand[kind].total * sizeof(float), st));
    }
    launch_plan_rank(b, ra, c_->counts.p, st);
    launch_scan(c_->counts.p, c_->begins.p, ra.ntasks, c_->scan.p, c_->counter.p, st);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (timing) {
        e0 = new_event();
        e1 = new_event();
        cudaEventRecord(e0, st);
    }
    launch_rank(b, ra, c_->begins.p, c_->scan.p, c_->counter.p, rank_grid_, st);
    if (timing) {
        cudaEventRecord(e1, st);
        rank_ev.push_back({e0, e1});
    }
    launches_ += 3;
    rank_launches_++;
    if (cfg_.mode == INDIALIGN_MODE_LEARNED) {
        launch_select(b, select_args(kind, det_ss), st);
        launches_++;
    }
    CK(cudaGetLastError());
    return INDIALIGN_OK;
}

SelectArgs Runner::select_args(int kind, int det_ss) {
    SelectArgs sa;
    sa.task = rank_args(kind, det_ss);
    sa.wbase = L_cand[kind].d_base;
    sa.score = c_->wscore.p + koff_[kind];
    sa.wcount = c_->wcount.p;
    sa.wlist = c_->wlist.p;
    sa.top_k = cfg_.top_k;
    sa.margin = (float)cfg_.margin;
    sa.audit_rate = cfg_.audit;
    sa.seed = cfg_.seed;
    sa.kind = kind;
    sa.stats = c_->rstats.p + (size_t)kind * kRankStats;
    return sa;
}

// After a ranked pass: LEARNED checks the audited tasks, COLLECT records
// every candidate's refined score.
int Runner::after_stage(int kind, const CandRes &r, int det_ss) {
    if (!ranked(kind, det_ss)) return INDIALIGN_OK;
    cudaStream_t st = c_->stream;
    if (cfg_.mode == INDIALIGN_MODE_LEARNED) {
        launch_audit(b, select_args(kind, det_ss), r, st);
        if (sel_out) {  // keep this pass's selection for the caller
            const int nt = ntasks(kind);
            CK(cudaMemcpyAsync(sel_out + sel_row(kind), c_->wcount.p, nt * sizeof(int), cudaMemcpyDeviceToDevice,
                               st));
            CK(cudaMemcpyAsync(sel_out + 6LL * n_ + sel_row(kind) * kMaxTopK, c_->wlist.p,
                               (size_t)nt * kMaxTopK * sizeof(int), cudaMemcpyDeviceToDevice, st));
        }
    } else if (cfg_.mode == INDIALIGN_MODE_COLLECT) {
        launch_collect_labels(b, rank_args(kind, det_ss), r, c_->wlabel.p + koff_[kind], st);
    } else {
        return INDIALIGN_OK;
    }
    launches_++;
    CK(cudaGetLastError());
    return INDIALIGN_OK;
}

#define RUN(x)                  \
    do {                        \
        int rc_ = (x);          \
        if (rc_) return rc_;    \
    } while (0)

int Runner::run_stages() {
    cudaStream_t st = c_->stream;
    // 2. seed bank (indialign.cpp:90-104)
    RUN(rank_stage(CAND_MAIN));
    RUN(bank(BK_MAIN, L_main, nullptr, -1, -1, sel_count(CAND_MAIN), sel_list(CAND_MAIN)));
    RUN(after_stage(CAND_MAIN, det_res(c_)));
    mark(0);
    // 2b. SS seeds IA2 + IA4, rescored (indialign.cpp:106-116, ss.h:87-164)
    launch_ss(b, st);
    launches_++;
    RUN(glue(G_SS_BEGIN));
    RUN(chain(CH_SS2, L_pair, 1, nullptr, nullptr, false));
    RUN(rank_stage(CAND_DET, 1));
    RUN(bank(BK_DET_SS, L_detss, nullptr, -1, -1, sel_count(CAND_DET, 1), sel_list(CAND_DET, 1)));
    RUN(after_stage(CAND_DET, det_res(c_, 1), 1));
    RUN(glue(G_SS_DET));
    RUN(dp_full(1));
    RUN(glue(G_SS_DP));
    RUN(glue(G_SS4_START));
    RUN(chain(CH_SS4, L_pair, 1, nullptr, nullptr, false));
    RUN(rank_stage(CAND_DET, 1));
    RUN(bank(BK_DET_SS, L_detss, nullptr, -1, -1, sel_count(CAND_DET, 1), sel_list(CAND_DET, 1)));
    RUN(after_stage(CAND_DET, det_res(c_, 1), 1));
    RUN(glue(G_SS_DET));
    RUN(dp_full(1));
    RUN(glue(G_SS_DP));
    launch_rescore(b, REC_SS, 0, st);
    launches_++;
    RUN(glue(G_SS_FINISH));
    mark(1);
    // 2c. gapless threading (indialign.cpp:118-123)
    RUN(bank(BK_GAPLESS, L_gapless, nullptr, 5, 1e300));
    RUN(glue(G_STAGE_UPDATE));
    mark(2);
    // 3. rescue ladder (indialign.cpp:125-152)
    RUN(glue(G_GATE, cfg_.r1));
    RUN(rank_stage(CAND_LOCAL));
    RUN(chain(CH_LOCAL, L_localn, 0, nullptr, nullptr, true, sel_count(CAND_LOCAL), sel_list(CAND_LOCAL)));
    RUN(after_stage(CAND_LOCAL, CandRes{c_->chain_res.p, L_localn.d_base, nullptr, nullptr, nullptr, nullptr}));
    launch_rescore(b, REC_STAGE, 1, st);
    launches_++;
    RUN(glue(G_STAGE_UPDATE));
    mark(3);
    RUN(glue(G_GATE, cfg_.r1));
    RUN(rank_stage(CAND_THREAD));
    RUN(bank(BK_THREAD, L_thread, c_->thread_rec.p, -1, -1, sel_count(CAND_THREAD), sel_list(CAND_THREAD)));
    RUN(chain(CH_THREAD, L_threadch, 1, c_->thread_rec.p));
    RUN(after_stage(CAND_THREAD,
                    CandRes{c_->chain_res.p, L_threadch.d_base, c_->thread_rec.p, L_threadch.d_aux, nullptr, nullptr}));
    launch_rescore(b, REC_STAGE, 1, st);
    launches_++;
    RUN(glue(G_STAGE_UPDATE));
    mark(4);
    RUN(glue(G_GATE, cfg_.r2));
    RUN(rank_stage(CAND_DENSE));
    RUN(chain(CH_LOCAL, L_locald, 1, nullptr, nullptr, true, sel_count(CAND_DENSE), sel_list(CAND_DENSE)));
    RUN(after_stage(CAND_DENSE, CandRes{c_->chain_res.p, L_locald.d_base, nullptr, nullptr, nullptr, nullptr}));
    launch_rescore(b, REC_STAGE, 1, st);
    launches_++;
    RUN(glue(G_STAGE_UPDATE));
    mark(5);
    // 4. top-50% distance seed (indialign.cpp:154-177)
    launch_topk(b, st);
    launches_++;
    RUN(bank(BK_TOPK, L_topk));
    RUN(glue(G_STAGE_UPDATE));
    mark(6);
    // 5. DP refinement (indialign.cpp:179-228)
    RUN(glue(G_DPF_BEGIN));
    RUN(dp_full(0));
    launch_rescore(b, REC_DP, 0, st);
    launches_++;
    RUN(glue(G_DPF_UPDATE));
    launch_rescore(b, REC_TMP, 0, st);
    launches_++;
    RUN(glue(G_TMP_UPDATE));
    if (cfg_.dp_iter > 0) {
        RUN(glue(G_IDP_START));
        RUN(chain(CH_SINGLE, L_single, cfg_.dp_iter));
        launch_rescore(b, REC_STAGE, 1, st);
        launches_++;
        RUN(glue(G_STAGE_UPDATE));
        int extra = cfg_.dp_iter < 5 ? 5 - cfg_.dp_iter : 0;
        if (extra > 0) {
            RUN(glue(G_EXTRA_START));
            RUN(chain(CH_SINGLE, L_single, extra));
            launch_rescore(b, REC_STAGE, 1, st);
            launches_++;
            RUN(glue(G_STAGE_UPDATE));
        }
    }
    mark(7);
    if (cfg_.dp_iter > 0) {
        // 5b. DP from offset Kabsch starts (indialign.cpp:229-256)
        launch_offset_starts(b, c_->off_start.p, L_offslots.d_pair, L_offslots.d_aux,
                             L_offslots.ntasks, st);
        launches_++;
        RUN(chain(CH_OFFDP, L_offdp, cfg_.dp_iter, c_->off_start.p, c_->off_res.p));
        launch_rescore_list(b, c_->off_res.p, L_offslots.d_pair, L_offslots.ntasks, st);
        launches_++;
        RUN(glue(G_OFFDP_UPDATE, 0.0, c_->off_res.p, L_offdp.d_aux));
    }
    mark(8);
    // 6. weighted TM refinement (indialign.cpp:258-264)
    launch_weighted(b, st);
    launches_++;
    mark(9);
    CK(cudaGetLastError());
    return INDIALIGN_OK;
}

}  // namespace ia

namespace ia {

static uint64_t fnv_pow_host(int z) {
    uint64_t r = 1, b = 1099511628211ULL;
    while (z) {
        if (z & 1) r *= b;
        b *= b;
        z >>= 1;
    }
    return r;
}

static const char *kStageNames[] = {"seed_build", "seed_bank", "ss", "gapless_threading",
                                    "local_fragment", "threading_dp", "dense_local_fragment",
                                    "topk_seed", "dp_refine", "offset_dp", "weighted_refine",
                                    "total"};

// Where a batch's inputs live: host pairs, or device arrays packed back to
// back (off[] on the host).
struct Source {
    std::vector<const NativePairInput *> host;
    int n_dev = 0;
    const int *off = nullptr;
    const double *pred = nullptr, *nat = nullptr, *lnorm = nullptr;
    const uint8_t *v = nullptr, *pv = nullptr, *nv = nullptr;
    const int *lens = nullptr;  // optional lengths (padded rows: off[p] = p * N)
    // a length bucket's sub-batch (host arrays, or null): each pair's index
    // in the caller's batch, and its row in the caller's outputs
    const int *gidx = nullptr, *out_map = nullptr;
    cudaEvent_t wait_ev = nullptr;  // work on the caller's stream to wait for
    int n() const { return host.empty() ? n_dev : (int)host.size(); }
    int len(int p) const {
        return host.empty() ? (lens ? lens[p] : off[p + 1] - off[p]) : host[p]->length;
    }
};

// Inputs -> packed device batch; runs the search; writes {score,R,t} per
// pair to results (host) or d_out (device).
static int run_batch(Ctx *c, const Cfg &cfg, const Source &src, double *results, double *d_out,
                     const IndialignBatchOptions *opts) {
    const int n = src.n();
    cudaStream_t own = c->stream;
    if (opts && opts->stream) c->stream = static_cast<cudaStream_t>(opts->stream);
    struct Restore {
        Ctx *c;
        cudaStream_t s;
        ~Restore() { c->stream = s; }
    } restore{c, own};
    cudaStream_t st = c->stream;
    if (src.wait_ev) CK(cudaStreamWaitEvent(st, src.wait_ev, 0));
    // ---- pack (pair blocks padded to an even residue count) ----
    c->h_off.resize(n + 1);
    c->h_len.resize(n);
    c->h_bitoff.resize(n);
    int total = 0, Nmax = 1;
    long long bits = 0;
    for (int p = 0; p < n; p++) {
        const int N = src.len(p);
        c->h_off[p] = total;
        c->h_len[p] = N;
        c->h_bitoff[p] = (int)bits;
        bits += (long long)kMaxBitSeeds * ((N + 31) / 32);
        total += (N + 1) & ~1;
        if (N > Nmax) Nmax = N;
    }
    c->h_off[n] = total;
    if (bits > 0x7fffffffLL) {
        g_last_error = "batch too large";
        return INDIALIGN_E_INPUT;
    }
    const bool on_host = !src.host.empty();
    c->h_lnorm.resize(n);
    if (on_host) {
        c->h_pred.assign(3 * (size_t)total, 0.0);
        c->h_nat.assign(3 * (size_t)total, 0.0);
        c->h_v.assign(total, 0);
        c->h_pv.assign(total, 0);
        c->h_nv.assign(total, 0);
        for (int p = 0; p < n; p++) {
            const NativePairInput *q = src.host[p];
            const size_t o = c->h_off[p], N = q->length;
            std::memcpy(&c->h_pred[3 * o], q->pred_xyz, 24 * N);
            std::memcpy(&c->h_nat[3 * o], q->native_xyz, 24 * N);
            std::memcpy(&c->h_v[o], q->valid_mask, N);
            std::memcpy(&c->h_pv[o], q->pred_valid_mask, N);
            std::memcpy(&c->h_nv[o], q->native_valid_mask, N);
            c->h_lnorm[p] = q->lnorm;
        }
    } else {
        for (int p = 0; p < n; p++) c->h_lnorm[p] = src.lnorm[p];
    }
    // ---- device buffers ----
    const size_t T = (size_t)total + 2;
    CK(c->off.ensure(n + 1));
    CK(c->len.ensure(n));
    CK(c->bitoff.ensure(n));
    CK(c->err.ensure(1));
    CK(c->lnorm.ensure(n));
    CK(c->pred.ensure(3 * T));
    CK(c->nat.ensure(3 * T));
    CK(c->v.ensure(T));
    CK(c->pv.ensure(T));
    CK(c->nv.ensure(T));
    CK(c->info.ensure(n));
    CK(c->state.ensure(n));
    CK(c->pmap.ensure(T));
    CK(c->nmap.ensure(T));
    CK(c->vmap.ensure(T));
    CK(c->scratch.ensure(T + n + 1));
    CK(c->dscr.ensure(T));
    CK(c->predc.ensure(3 * T));
    CK(c->natc.ensure(3 * T));
    CK(c->sspc.ensure(T));
    CK(c->ssnc.ensure(T));
    CK(c->seeds.ensure((size_t)n * kMaxSeeds));
    CK(c->topk.ensure(n));
    CK(c->bits.ensure((size_t)bits + 1));
    CK(c->hashes.ensure((size_t)n * kMaxSeeds));
    CK(c->kv.ensure(2 * T));
    CK(c->ctr.ensure(kCounters));
    if (c->fnv_n < Nmax + 1) {
        std::vector<uint64_t> pw(Nmax + 1);
        for (int z = 0; z <= Nmax; z++) pw[z] = fnv_pow_host(z);
        CK(c->fnv_pow.ensure(Nmax + 1));
        CK(cudaMemcpy(c->fnv_pow.p, pw.data(), pw.size() * 8, cudaMemcpyHostToDevice));
        c->fnv_n = Nmax + 1;
    }
    CK(cudaMemcpyAsync(c->off.p, c->h_off.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->len.p, c->h_len.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->bitoff.p, c->h_bitoff.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->lnorm.p, c->h_lnorm.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    if (on_host) {
        CK(cudaMemcpyAsync(c->pred.p, c->h_pred.data(), c->h_pred.size() * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(c->nat.p, c->h_nat.data(), c->h_nat.size() * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(c->v.p, c->h_v.data(), total, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(c->pv.p, c->h_pv.data(), total, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(c->nv.p, c->h_nv.data(), total, cudaMemcpyHostToDevice, st));
    }
    CK(cudaMemsetAsync(c->err.p, 0, sizeof(int), st));
    CK(cudaMemsetAsync(c->ctr.p, 0, kCounters * sizeof(unsigned long long), st));
    DevBatch b;
    b.n = n;
    b.off = c->off.p;
    b.len = c->len.p;
    b.lnorm = c->lnorm.p;
    b.pred = c->pred.p;
    b.nat = c->nat.p;
    b.v = c->v.p;
    b.pv = c->pv.p;
    b.nv = c->nv.p;
    b.info = c->info.p;
    b.state = c->state.p;
    b.pmap = c->pmap.p;
    b.nmap = c->nmap.p;
    b.vmap = c->vmap.p;
    b.scratch = c->scratch.p;
    b.dscr = c->dscr.p;
    b.predc = c->predc.p;
    b.natc = c->natc.p;
    b.sspc = c->sspc.p;
    b.ssnc = c->ssnc.p;
    b.seeds = c->seeds.p;
    b.topk_seed = c->topk.p;
    b.bits = c->bits.p;
    b.bitoff = c->bitoff.p;
    b.hashes = c->hashes.p;
    b.kv = c->kv.p;
    b.fnv_pow = c->fnv_pow.p;
    b.err = c->err.p;
    b.ctr = c->ctr.p;
    b.gidx = nullptr;
    b.out_map = nullptr;
    if (src.gidx) {
        CK(c->gidx.ensure(n));
        CK(cudaMemcpyAsync(c->gidx.p, src.gidx, n * sizeof(int), cudaMemcpyHostToDevice, st));
        b.gidx = c->gidx.p;
    }
    if (src.out_map && d_out) {
        CK(c->omap.ensure(n));
        CK(cudaMemcpyAsync(c->omap.p, src.out_map, n * sizeof(int), cudaMemcpyHostToDevice, st));
        b.out_map = c->omap.p;
    }
    if (!on_host) {
        // caller's offsets to the device (scratch doubles as staging), repack
        CK(cudaMemcpyAsync(c->scratch.p, src.off, (n + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
        launch_repack(b, c->scratch.p, src.pred, src.nat, src.v, src.pv, src.nv, st);
        CK(cudaGetLastError());
    }
    const bool prof = (opts && (opts->profile || opts->stage_ms)) || std::getenv("INDIALIGN_PROFILE");
    struct EventPair {  // the call's total-time events, destroyed on every exit path
        cudaEvent_t a = nullptr, b = nullptr;
        ~EventPair() {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
        }
    } call_ev;
    cudaEvent_t &e0 = call_ev.a, &e1 = call_ev.b;
    if (prof) {
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        CK(cudaEventRecord(e0, st));
    }
    const bool use_mlp = cfg.mode == INDIALIGN_MODE_LEARNED ||
                         (cfg.mode == INDIALIGN_MODE_COLLECT && opts->ranker);
    if (use_mlp) {
        CK(c->blob.ensure(kBlobSize));
        CK(c->mlp.ensure(1));
        CK(cudaMemcpyAsync(c->blob.p, opts->ranker, kBlobSize * sizeof(float), cudaMemcpyHostToDevice, st));
        launch_mlp_pack(c->blob.p, c->mlp.p, st);
        CK(cudaGetLastError());
    }
    Runner r(c, cfg, n);
    r.b = b;
    r.use_mlp = use_mlp;
    r.Nmax = Nmax;
    const bool print_profile = (opts && opts->profile) || std::getenv("INDIALIGN_PROFILE");
    r.timing = (opts && (opts->stage_ms || opts->kernel_ms)) || print_profile;
    r.stage_event(0);
    // ---- seeds ----
    launch_prep(b, cfg.use_frag, st);
    launch_anchor(b, st);
    r.launches_ += 2;
    CK(cudaGetLastError());
    std::vector<PairInfo> info(n);
    CK(cudaMemcpyAsync(info.data(), c->info.p, n * sizeof(PairInfo), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    r.stage_event(100);  // seeds done
    if (opts && opts->stage_best) {
        CK(c->snap.ensure((size_t)n * kTrace * kRec));
        CK(cudaMemsetAsync(c->snap.p, 0, (size_t)n * kTrace * kRec * 8, st));
        r.snap = c->snap.p;
    }
    int rc = r.build_layouts(info);
    if (rc) return rc;
    const bool win_out = cfg.mode == INDIALIGN_MODE_COLLECT || (use_mlp && opts->win_score);
    if (win_out && r.windows() > (opts->win_cap > 0 ? opts->win_cap : 0)) {
        g_last_error = "per-window outputs: " + std::to_string(r.windows()) + " windows exceed win_cap";
        return INDIALIGN_E_INPUT;
    }
    if (cfg.mode == INDIALIGN_MODE_COLLECT && r.windows() > 0)
        CK(cudaMemsetAsync(c->wlabel.p, 0xff, (size_t)r.windows() * sizeof(float), st));  // NaN
    if (cfg.mode == INDIALIGN_MODE_LEARNED) {
        CK(cudaMemsetAsync(c->rstats.p, 0, kCandKinds * kRankStats * sizeof(unsigned long long), st));
        if (opts->win_select) {
            CK(c->wsel.ensure((size_t)6 * n * (1 + kMaxTopK)));
            r.sel_out = c->wsel.p;
        }
    }
    rc = r.run_stages();
    if (rc) return rc;
    if (prof) CK(cudaEventRecord(e1, st));
    // ---- results ----
    std::vector<PairState> state(d_out ? 0 : n);
    int err = 0;
    if (!d_out)
        CK(cudaMemcpyAsync(state.data(), c->state.p, n * sizeof(PairState), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&err, c->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (prof) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        const char *tag = std::getenv("INDIALIGN_PROFILE_TAG");
        if ((opts && opts->profile) || std::getenv("INDIALIGN_PROFILE"))
            std::fprintf(stderr, "[indialign]%s pairs=%d stage=%s ms=%.3f\n", tag ? tag : "", n,
                         kStageNames[INDIALIGN_STAGES - 1], ms);
        if (opts && opts->stage_ms) opts->stage_ms[INDIALIGN_STAGES - 1] = ms;
    }
    if (err) {
        g_last_error = "device error flag " + std::to_string(err);
        return INDIALIGN_E_DEVICE;
    }
    static_assert(kCandKinds * kRankStats == INDIALIGN_RANK_STATS, "rank_stats layout: [kinds][kRankStats]");
    if (cfg.mode == INDIALIGN_MODE_LEARNED && opts->rank_stats) {
        unsigned long long h[kCandKinds * kRankStats];
        CK(cudaMemcpy(h, c->rstats.p, sizeof(h), cudaMemcpyDeviceToHost));
        for (int k = 0; k < kCandKinds * kRankStats && k < INDIALIGN_RANK_STATS; k++)
            opts->rank_stats[k] = (long long)h[k];
    }
    if (use_mlp && opts->win_score && r.windows() > 0)
        CK(cudaMemcpy(opts->win_score, c->wscore.p, (size_t)r.windows() * sizeof(float),
                      cudaMemcpyDeviceToHost));
    if (cfg.mode == INDIALIGN_MODE_LEARNED && opts->win_select) {
        // rows: kinds back to back, n rows each, 2n for the detailed-search slots
        const size_t rows = (size_t)6 * n;
        std::vector<int> h(rows * (1 + kMaxTopK));
        CK(cudaMemcpy(h.data(), c->wsel.p, h.size() * sizeof(int), cudaMemcpyDeviceToHost));
        const int *wc = h.data(), *wl = h.data() + rows;
        for (size_t r0 = 0; r0 < rows; r0++) {
            int *o = opts->win_select + r0 * (kMaxTopK + 1);
            const int *l = wl + r0 * kMaxTopK;
            o[0] = wc[r0];
            for (int j = 0; j < kMaxTopK; j++) o[1 + j] = j < cfg.top_k ? l[j] : -1;
        }
    }
    if (cfg.mode == INDIALIGN_MODE_COLLECT && r.windows() > 0) {
        if (opts->win_feat)
            CK(cudaMemcpy(opts->win_feat, c->wfeat.p, (size_t)r.windows() * kFeatures * sizeof(float),
                          cudaMemcpyDeviceToHost));
        if (opts->win_label)
            CK(cudaMemcpy(opts->win_label, c->wlabel.p, (size_t)r.windows() * sizeof(float),
                          cudaMemcpyDeviceToHost));
    }
    if (opts && opts->stage_best && r.snap) {
        if (src.out_map) {  // a sub-batch: rows to the caller's pair order
            std::vector<double> tmp((size_t)n * kTrace * kRec);
            CK(cudaMemcpy(tmp.data(), r.snap, tmp.size() * 8, cudaMemcpyDeviceToHost));
            for (int p = 0; p < n; p++)
                std::memcpy(opts->stage_best + (size_t)src.out_map[p] * kTrace * kRec,
                            tmp.data() + (size_t)p * kTrace * kRec, (size_t)kTrace * kRec * 8);
        } else {
            CK(cudaMemcpy(opts->stage_best, r.snap, (size_t)n * kTrace * kRec * 8, cudaMemcpyDeviceToHost));
        }
    }
    if (opts && opts->counters) {
        unsigned long long h[kCounters];
        CK(cudaMemcpy(h, c->ctr.p, sizeof(h), cudaMemcpyDeviceToHost));
        h[CTR_CHAIN_LAUNCHES] = r.chain_launches_;
        h[CTR_BANK_LAUNCHES] = r.bank_launches_;
        h[CTR_LAUNCHES] = r.launches_;
        for (int k = 0; k < kCounters && k < INDIALIGN_COUNTERS; k++) opts->counters[k] = (long long)h[k];
    }
    if (r.timing) {
        // stage boundaries: 0 start, 100 seeds done, s+1 after trace stage s
        float ms = 0;
        cudaEvent_t prev = nullptr;
        double stage[INDIALIGN_STAGES] = {0};
        for (auto &x : r.stage_ev) {
            if (prev) {
                CK(cudaEventElapsedTime(&ms, prev, x.second));
                int slot = x.first == 100 ? 0 : x.first;  // seeds -> 0, trace stage s -> s+1
                if (slot >= 0 && slot < INDIALIGN_STAGES - 1) stage[slot] += ms;
            }
            prev = x.second;
        }
        if (!r.stage_ev.empty()) {
            CK(cudaEventElapsedTime(&ms, r.stage_ev.front().second, r.stage_ev.back().second));
            stage[INDIALIGN_STAGES - 1] = ms;
        }
        if (opts && opts->stage_ms)
            for (int k = 0; k < INDIALIGN_STAGES; k++) opts->stage_ms[k] = stage[k];
        if (print_profile) {  // per-stage device times, the reference's stage names
            const char *tag = std::getenv("INDIALIGN_PROFILE_TAG");
            for (int k = 0; k < INDIALIGN_STAGES - 1; k++)
                std::fprintf(stderr, "[indialign]%s pairs=%d stage=%s ms=%.3f\n", tag ? tag : "", n,
                             kStageNames[k], stage[k]);
        }
        if (opts && opts->kernel_ms) {
            double ch = 0, bk = 0;
            for (auto &x : r.chain_ev) { CK(cudaEventElapsedTime(&ms, x.first, x.second)); ch += ms; }
            for (auto &x : r.bank_ev) { CK(cudaEventElapsedTime(&ms, x.first, x.second)); bk += ms; }
            opts->kernel_ms[0] = ch;
            opts->kernel_ms[1] = bk;
            opts->kernel_ms[2] = (double)r.chain_ev.size();
            opts->kernel_ms[3] = (double)r.bank_ev.size();
            double rk = 0;
            for (auto &x : r.rank_ev) { CK(cudaEventElapsedTime(&ms, x.first, x.second)); rk += ms; }
            opts->kernel_ms[4] = rk;
            opts->kernel_ms[5] = (double)r.rank_ev.size();
        }
        r.recycle();
    }
    if (d_out) {
        launch_export(b, d_out, st);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
    } else {
        for (int p = 0; p < n; p++)
            std::memcpy(results + 13 * (size_t)(src.out_map ? src.out_map[p] : p), state[p].rec[REC_BEST], 13 * 8);
    }
    return INDIALIGN_OK;
}

// ---- length buckets ---------------------------------------------------------
// The tuning table holds one row of kernel shapes per length bucket (N <=
// 128, <= 512, longer): bank items per CTA chunk and their order, NW chains
// per CTA chunk, NW traces in shared memory.  Inside one launch every task
// takes the row of its own pair's bucket (the plan kernels look it up), so a
// batch of mixed lengths runs each pair with its bucket's shapes in the same
// persistent kernels.  Optionally (split = 1) a batch that spans buckets runs
// as one sub-batch per bucket instead, each on its own context and stream
// with launches sized by its own longest pair, side by side on the device;
// every pair's search is independent of the rest of its batch and keeps its
// index in the caller's batch for the learned mode's audit draw, so results
// equal those of one call.  Measured on 2048-pair calls of the learned16384
// workload the split is slower (its sub-batches' full-size persistent grids
// mostly run one after another, adding per-stage tails), so it is off unless
// the tuner finds it faster.
constexpr int kBuckets = INDIALIGN_TUNE_BUCKETS;
static_assert(kBuckets == kTuneBuckets, "bucket count of the C ABI and the kernels");

struct TuneTable {
    int split = 0;       // split batches that span buckets into concurrent sub-batches
    int min_pairs = 64;  // ... of at least this many pairs
    int max_len[kBuckets] = {128, 512, 65535};
    Tune t[kBuckets];
    TuneRows rows() const {
        TuneRows r;
        for (int b = 0; b < kBuckets; b++) {
            r.max_len[b] = max_len[b];
            r.t[b] = t[b];
        }
        return r;
    }
};

static std::mutex g_tune_mu;
static TuneTable g_tune;
static bool g_tune_loaded = false;

static bool tune_row_ok(const int *r) {
    return r[0] >= 1 && r[0] <= 65535 && r[1] >= 32 && r[1] <= 4096 && r[1] % 32 == 0 && (r[2] == 0 || r[2] == 1) &&
           r[3] >= 1 && r[3] <= 256 && (r[4] == 0 || r[4] == 1);
}

// The table file: INDIALIGN_TUNE_TABLE, else tune_b200.txt beside the
// library.  Lines "split S", "min_pairs M" and "bucket B max_len L
// bank_chunk C bank_cutoff_major O chain_chunk H chain_smem_trace T"; '#'
// starts a comment.  A missing or malformed file leaves the built-in rows.
static TuneTable read_tune_file() {
    TuneTable tt;
    std::string path;
    if (const char *e = std::getenv("INDIALIGN_TUNE_TABLE")) {
        path = e;
    } else {
        Dl_info info;
        if (dladdr(reinterpret_cast<void *>(&read_tune_file), &info) && info.dli_fname) {
            path = info.dli_fname;
            const size_t sl = path.rfind('/');
            path = (sl == std::string::npos ? std::string(".") : path.substr(0, sl)) + "/tune_b200.txt";
        }
    }
    FILE *f = path.empty() ? nullptr : std::fopen(path.c_str(), "r");
    if (!f) return tt;
    TuneTable out = tt;
    char line[512];
    bool ok = true;
    while (ok && std::fgets(line, sizeof line, f)) {
        char *hash = std::strchr(line, '#');
        if (hash) *hash = 0;
        int a = 0, r[5];
        char k0[32], k1[32], k2[32], k3[32], k4[32], k5[32];
        if (std::sscanf(line, " split %d", &a) == 1) {
            out.split = a != 0;
        } else if (std::sscanf(line, " min_pairs %d", &a) == 1) {
            out.min_pairs = a;
        } else if (std::sscanf(line, " bucket %d %31s %d %31s %d %31s %d %31s %d %31s %d", &a, k0, &r[0], k1, &r[1],
                               k2, &r[2], k3, &r[3], k4, &r[4]) == 11) {
            ok = a >= 0 && a < kBuckets && !std::strcmp(k0, "max_len") && !std::strcmp(k1, "bank_chunk") &&
                 !std::strcmp(k2, "bank_cutoff_major") && !std::strcmp(k3, "chain_chunk") &&
                 !std::strcmp(k4, "chain_smem_trace") && tune_row_ok(r);
            if (ok) {
                out.max_len[a] = r[0];
                out.t[a].bank_chunk = r[1];
                out.t[a].bank_cutoff_major = r[2];
                out.t[a].chain_chunk = r[3];
                out.t[a].chain_smem_trace = r[4];
            }
        } else {
            for (const char *q = line; *q; q++)
                if (*q != ' ' && *q != '\t' && *q != '\n' && *q != '\r') ok = false;
        }
    }
    std::fclose(f);
    return ok ? out : tt;
}

static TuneTable tune_table() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (!g_tune_loaded) {
        g_tune = read_tune_file();
        g_tune_loaded = true;
    }
    return g_tune;
}

static int bucket_of(const TuneTable &tt, int N) {
    for (int b = 0; b < kBuckets - 1; b++)
        if (N <= tt.max_len[b]) return b;
    return kBuckets - 1;
}

// The search of a batch from `src`: one run, or one run per length bucket
// side by side (see above).  Results to `results` (host) or `d_out` (device).
static int run_search(int device, const Cfg &cfg0, const Source &src, double *results, double *d_out,
                      const IndialignBatchOptions *opts) {
    const TuneTable tt = tune_table();
    const int n = src.n();
    std::vector<int> idx[kBuckets];
    int Lmax = 0;
    for (int p = 0; p < n; p++) {
        const int N = src.len(p);
        idx[bucket_of(tt, N)].push_back(p);
        if (N > Lmax) Lmax = N;
    }
    int nonempty = 0;
    for (int b = 0; b < kBuckets; b++) nonempty += !idx[b].empty();
    // per-candidate outputs are laid out by the whole batch's pair order
    const bool per_cand = opts && (opts->win_feat || opts->win_label || opts->win_score || opts->win_select);
    if (!tt.split || nonempty <= 1 || per_cand || n < tt.min_pairs) {
        Cfg cfg = cfg0;
        cfg.tune = tt.rows();
        cfg.chain_smem_trace = tt.t[bucket_of(tt, Lmax)].chain_smem_trace;
        Ctx *c = nullptr;
        int rc = acquire(device, &c);
        if (rc) return rc;
        rc = run_batch(c, cfg, src, results, d_out, opts);
        release(c);
        return rc;
    }
    if (device < 0) CK(cudaGetDevice(&device));
    CK(cudaSetDevice(device));
    // the sub-batches wait for the caller's stream, then run on their own
    struct Ev {
        cudaEvent_t e = nullptr;
        ~Ev() {
            if (e) cudaEventDestroy(e);
        }
    } start;
    if (opts && opts->stream) {
        CK(cudaEventCreateWithFlags(&start.e, cudaEventDisableTiming));
        CK(cudaEventRecord(start.e, static_cast<cudaStream_t>(opts->stream)));
    }
    struct Part {
        Source src;
        std::vector<int> off, len;
        std::vector<double> lnorm;
        IndialignBatchOptions o;
        double stage_ms[INDIALIGN_STAGES] = {0}, kernel_ms[6] = {0};
        long long counters[INDIALIGN_COUNTERS] = {0}, rank_stats[INDIALIGN_RANK_STATS] = {0};
        Cfg cfg;
        int rc = 0;
        std::string err;
    };
    std::vector<Part> parts(kBuckets);
    for (int b = 0; b < kBuckets; b++) {
        Part &P = parts[b];
        const std::vector<int> &I = idx[b];
        if (I.empty()) continue;
        P.cfg = cfg0;
        P.cfg.tune = tt.rows();
        P.cfg.chain_smem_trace = tt.t[b].chain_smem_trace;
        if (!src.host.empty()) {
            for (int p : I) P.src.host.push_back(src.host[p]);
        } else {
            P.off.resize(I.size() + 1);
            P.len.resize(I.size());
            P.lnorm.resize(I.size());
            for (size_t k = 0; k < I.size(); k++) {
                P.off[k] = src.off[I[k]];
                P.len[k] = src.len(I[k]);
                P.lnorm[k] = src.lnorm[I[k]];
            }
            P.off[I.size()] = 0;
            P.src.n_dev = (int)I.size();
            P.src.off = P.off.data();
            P.src.lens = P.len.data();
            P.src.pred = src.pred;
            P.src.nat = src.nat;
            P.src.v = src.v;
            P.src.pv = src.pv;
            P.src.nv = src.nv;
            P.src.lnorm = P.lnorm.data();
        }
        P.src.gidx = I.data();
        P.src.out_map = I.data();
        P.src.wait_ev = start.e;
        std::memset(&P.o, 0, sizeof P.o);
        if (opts) P.o = *opts;
        P.o.device = device;
        P.o.stream = nullptr;
        P.o.stage_ms = opts && opts->stage_ms ? P.stage_ms : nullptr;
        P.o.kernel_ms = opts && opts->kernel_ms ? P.kernel_ms : nullptr;
        P.o.counters = opts && opts->counters ? P.counters : nullptr;
        P.o.rank_stats = opts && opts->rank_stats ? P.rank_stats : nullptr;
    }
    std::vector<std::thread> th;
    for (int b = 0; b < kBuckets; b++) {
        if (idx[b].empty()) continue;
        th.emplace_back([&parts, b, device, results, d_out]() {
            Part &P = parts[b];
            Ctx *c = nullptr;
            P.rc = acquire(device, &c, b + 1);
            if (!P.rc) {
                P.rc = run_batch(c, P.cfg, P.src, results, d_out, &P.o);
                release(c);
            }
            if (P.rc) P.err = g_last_error;
        });
    }
    for (auto &t : th) t.join();
    for (int b = 0; b < kBuckets; b++)
        if (parts[b].rc) {
            g_last_error = "length bucket " + std::to_string(b) + ": " + parts[b].err;
            return parts[b].rc;
        }
    bool first = true;
    for (int b = 0; b < kBuckets; b++) {
        if (idx[b].empty()) continue;
        const Part &P = parts[b];
        if (opts && opts->stage_ms)  // the sub-batches run side by side: the slowest
            for (int k = 0; k < INDIALIGN_STAGES; k++)
                opts->stage_ms[k] = first ? P.stage_ms[k] : std::max(opts->stage_ms[k], P.stage_ms[k]);
        if (opts && opts->kernel_ms)
            for (int k = 0; k < 6; k++) opts->kernel_ms[k] = (first ? 0.0 : opts->kernel_ms[k]) + P.kernel_ms[k];
        if (opts && opts->counters)
            for (int k = 0; k < INDIALIGN_COUNTERS; k++)
                opts->counters[k] = (first ? 0 : opts->counters[k]) + P.counters[k];
        if (opts && opts->rank_stats)
            for (int k = 0; k < INDIALIGN_RANK_STATS; k++)
                opts->rank_stats[k] = (first ? 0 : opts->rank_stats[k]) + P.rank_stats[k];
        first = false;
    }
    return INDIALIGN_OK;
}

static Cfg make_cfg(const NativeConfig *cfg, const IndialignBatchOptions *opts) {
    Cfg c;
    c.use_frag = cfg->use_fragment_search != 0;
    c.max_iter = cfg->max_iter;
    c.dp_iter = cfg->dp_iter;
    c.r1 = cfg->rescue_score_1;
    c.r2 = cfg->rescue_score_2;
    c.early = cfg->early_term_score;
    if (opts) {
        c.mode = opts->mode;
        c.top_k = opts->top_k > 0 ? opts->top_k : 8;
        c.margin = opts->margin;
        c.audit = opts->audit_rate;
        c.seed = opts->seed;
        c.rank_mask = opts->rank_mask ? opts->rank_mask : INDIALIGN_RANK_DEFAULT;
        c.min_len = opts->rank_min_len > 0 ? opts->rank_min_len : (opts->rank_min_len < 0 ? 0 : INDIALIGN_RANK_MIN_LEN);
    }
    return c;
}

// Mode-specific option checks (before any device work).
static int check_mode(const IndialignBatchOptions *opts) {
    if (!opts || opts->mode == INDIALIGN_MODE_PLAIN) return INDIALIGN_OK;
    if (opts->mode == INDIALIGN_MODE_LEARNED) {
        if (!opts->ranker) {
            g_last_error = "learned mode: ranker parameters missing";
            return INDIALIGN_E_INPUT;
        }
        if (opts->top_k < 0 || opts->top_k > kMaxTopK) {
            g_last_error = "learned mode: top_k must be in 1.." + std::to_string(kMaxTopK);
            return INDIALIGN_E_INPUT;
        }
        return INDIALIGN_OK;
    }
    if (opts->mode == INDIALIGN_MODE_COLLECT) {
        if (!opts->win_feat && !opts->win_label) {
            g_last_error = "collect mode: no output buffers";
            return INDIALIGN_E_INPUT;
        }
        return INDIALIGN_OK;
    }
    g_last_error = "unknown mode " + std::to_string(opts->mode);
    return INDIALIGN_E_INPUT;
}

static int search_host(int n_pairs, const NativePairInput *inputs, const NativeConfig *cfg,
                       const IndialignBatchOptions *opts, NativePairResult *outputs) {
    g_last_error.clear();
    if (g_inject.load() > 0) {
        g_inject.fetch_sub(1);
        g_last_error = "injected failure";
        return INDIALIGN_E_INJECTED;
    }
    if (!inputs || !cfg || !outputs || n_pairs < 0) {
        g_last_error = "null argument";
        return INDIALIGN_E_INPUT;
    }
    if (int rc = check_mode(opts)) return rc;
    Source src;
    std::vector<const NativePairInput *> &in = src.host;
    std::vector<int> ids;
    for (int p = 0; p < n_pairs; p++) {
        const NativePairInput *q = &inputs[p];
        if (q->length <= 0) continue;  // reference: rc -1, output untouched
        if (q->length > 65535 || !q->pred_xyz || !q->native_xyz || !q->valid_mask ||
            !q->pred_valid_mask || !q->native_valid_mask) {
            g_last_error = "pair " + std::to_string(p) + ": null pointer or length > 65535";
            return INDIALIGN_E_INPUT;
        }
        in.push_back(q);
        ids.push_back(p);
    }
    if (in.empty()) return INDIALIGN_OK;
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
        cudaGetLastError();
        g_last_error = "no CUDA device";
        return INDIALIGN_E_NODEVICE;
    }
    std::vector<double> res(13 * in.size());
    int rc = run_search(opts ? opts->device : -1, make_cfg(cfg, opts), src, res.data(), nullptr, opts);
    if (rc) return rc;
    for (size_t k = 0; k < ids.size(); k++) {
        NativePairResult *o = &outputs[ids[k]];
        o->score = res[13 * k];
        std::memcpy(o->rotation, &res[13 * k + 1], 72);
        std::memcpy(o->translation, &res[13 * k + 10], 24);
    }
    return INDIALIGN_OK;
}

}  // namespace ia

extern "C" {

void indialign_default_config(NativeConfig *cfg) {
    cfg->backend_mode = 0;
    cfg->use_fragment_search = 1;
    cfg->max_iter = 20;
    cfg->dp_iter = 1;
    cfg->max_mem_gb = 20.0;
    cfg->request_cuda = 0;
    cfg->rescue_score_1 = 0.5;
    cfg->rescue_score_2 = 0.3;
    cfg->early_term_score = 0.99;
}

int indialign_tmscore_search(const NativePairInput *inp, const NativeConfig *cfg,
                             NativePairResult *out) {
    if (!inp) return INDIALIGN_E_INPUT;
    if (inp->length <= 0) return INDIALIGN_E_LENGTH;
    return ia::search_host(1, inp, cfg, nullptr, out);
}

int indialign_tmscore_search_batch(int n_pairs, const NativePairInput *inputs,
                                   const NativeConfig *cfg, NativePairResult *outputs) {
    return ia::search_host(n_pairs, inputs, cfg, nullptr, outputs);
}

int indialign_tmscore_search_batch_ex(int n_pairs, const NativePairInput *inputs,
                                      const NativeConfig *cfg, const IndialignBatchOptions *opts,
                                      NativePairResult *outputs) {
    return ia::search_host(n_pairs, inputs, cfg, opts, outputs);
}

int indialign_cuda_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return 0;
    }
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, 0) != cudaSuccess) return 0;
    return major == 10 ? 1 : 0;
}

int indialign_nw_align(const double *d_smat, int np, int nn, double gap, int *d_ap, int *d_an,
                       int *d_na, void *stream) {
    ia::g_last_error.clear();
    if (!d_smat || !d_ap || !d_an || !d_na || np < 1 || nn < 1 || np > 65535 || nn > 65535) {
        ia::g_last_error = "nw_align: null pointer or size outside 1..65535";
        return INDIALIGN_E_INPUT;
    }
    ia::Ctx *c = nullptr;
    int rc = ia::acquire(-1, &c);
    if (rc) return rc;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    rc = INDIALIGN_OK;
    do {
        const size_t words = ia::nw_trace_words(np, nn);
        if (c->gtrace.ensure(words) != cudaSuccess || c->gbh.ensure((size_t)nn + 1) != cudaSuccess ||
            c->gal.ensure((size_t)(np < nn ? np : nn)) != cudaSuccess ||
            c->ctr.ensure(ia::kCounters) != cudaSuccess) {
            ia::g_last_error = "nw_align: workspace allocation failed";
            rc = INDIALIGN_E_CUDA;
            break;
        }
        ia::launch_nw_explicit(d_smat, np, nn, gap, c->gtrace.p, c->gbh.p, c->gal.p, d_ap, d_an, d_na,
                               c->ctr.p, st);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            ia::set_error("nw_align", e);
            rc = INDIALIGN_E_CUDA;
        }
    } while (0);
    ia::release(c);
    return rc;
}

int indialign_tmscore_search_device(int n_pairs, const int *off, const double *d_pred,
                                    const double *d_nat, const uint8_t *d_v,
                                    const uint8_t *d_pv, const uint8_t *d_nv,
                                    const double *lnorm, const NativeConfig *cfg,
                                    const IndialignBatchOptions *opts, double *d_out) {
    ia::g_last_error.clear();
    if (ia::g_inject.load() > 0) {
        ia::g_inject.fetch_sub(1);
        ia::g_last_error = "injected failure";
        return INDIALIGN_E_INJECTED;
    }
    if (n_pairs <= 0) return INDIALIGN_OK;
    if (!off || !d_pred || !d_nat || !d_v || !d_pv || !d_nv || !lnorm || !cfg || !d_out)
        return INDIALIGN_E_INPUT;
    if (int rc = ia::check_mode(opts)) return rc;
    for (int p = 0; p < n_pairs; p++) {
        int L = off[p + 1] - off[p];
        if (L <= 0 || L > 65535) {
            ia::g_last_error = "pair " + std::to_string(p) + ": length must be in 1..65535";
            return INDIALIGN_E_INPUT;
        }
    }
    ia::Source src;
    src.n_dev = n_pairs;
    src.off = off;
    src.pred = d_pred;
    src.nat = d_nat;
    src.v = d_v;
    src.pv = d_pv;
    src.nv = d_nv;
    src.lnorm = lnorm;
    return ia::run_search(opts ? opts->device : -1, ia::make_cfg(cfg, opts), src, nullptr, d_out, opts);
}

int indialign_candidate_count(int plen, int nlen, int kind) {
    if (plen < 0 || nlen < 0 || kind < 0 || kind >= ia::kCandKinds) return 0;
    if (kind == ia::CAND_DET) return ia::kDetSlots * ia::kdet_max(plen < nlen ? plen : nlen);
    if (kind == ia::CAND_MAIN) return ia::kMaxSeeds;
    return ia::cand_count(kind, plen, nlen);
}

int indialign_tmscore_search_padded(int n_pairs, int N, const int *lengths, const double *d_pred,
                                    const double *d_nat, const uint8_t *d_v, const uint8_t *d_pv,
                                    const uint8_t *d_nv, const double *lnorm, const NativeConfig *cfg,
                                    const IndialignBatchOptions *opts, double *d_out) {
    ia::g_last_error.clear();
    if (ia::g_inject.load() > 0) {
        ia::g_inject.fetch_sub(1);
        ia::g_last_error = "injected failure";
        return INDIALIGN_E_INJECTED;
    }
    if (n_pairs <= 0) return INDIALIGN_OK;
    if (!lengths || !d_pred || !d_nat || !d_v || !d_pv || !d_nv || !lnorm || !cfg || !d_out || N < 1 ||
        N > 65535) {
        ia::g_last_error = "padded: null pointer or row length outside 1..65535";
        return INDIALIGN_E_INPUT;
    }
    for (int p = 0; p < n_pairs; p++)
        if (lengths[p] < 1 || lengths[p] > N) {
            ia::g_last_error = "pair " + std::to_string(p) + ": length must be in 1..N";
            return INDIALIGN_E_INPUT;
        }
    if (int rc = ia::check_mode(opts)) return rc;
    std::vector<int> off((size_t)n_pairs + 1);
    for (int p = 0; p <= n_pairs; p++) off[p] = p * N;
    if ((long long)n_pairs * N > 0x7fffffffLL) {
        ia::g_last_error = "padded: batch too large";
        return INDIALIGN_E_INPUT;
    }
    ia::Source src;
    src.n_dev = n_pairs;
    src.off = off.data();
    src.lens = lengths;
    src.pred = d_pred;
    src.nat = d_nat;
    src.v = d_v;
    src.pv = d_pv;
    src.nv = d_nv;
    src.lnorm = lnorm;
    return ia::run_search(opts ? opts->device : -1, ia::make_cfg(cfg, opts), src, nullptr, d_out, opts);
}

int indialign_get_tuning(int *split, int *min_pairs, int *table) {
    const ia::TuneTable tt = ia::tune_table();
    if (split) *split = tt.split;
    if (min_pairs) *min_pairs = tt.min_pairs;
    if (table)
        for (int b = 0; b < ia::kBuckets; b++) {
            int *r = table + b * INDIALIGN_TUNE_FIELDS;
            r[0] = tt.max_len[b];
            r[1] = tt.t[b].bank_chunk;
            r[2] = tt.t[b].bank_cutoff_major;
            r[3] = tt.t[b].chain_chunk;
            r[4] = tt.t[b].chain_smem_trace;
        }
    return INDIALIGN_OK;
}

int indialign_set_tuning(int split, int min_pairs, const int *table) {
    ia::TuneTable tt;
    if (!table) {
        tt = ia::read_tune_file();
    } else {
        tt.split = split != 0;
        tt.min_pairs = min_pairs;
        int prev = 0;
        for (int b = 0; b < ia::kBuckets; b++) {
            const int *r = table + b * INDIALIGN_TUNE_FIELDS;
            if (!ia::tune_row_ok(r) || r[0] <= prev) {
                ia::g_last_error = "set_tuning: invalid row " + std::to_string(b);
                return INDIALIGN_E_INPUT;
            }
            prev = r[0];
            tt.max_len[b] = r[0];
            tt.t[b].bank_chunk = r[1];
            tt.t[b].bank_cutoff_major = r[2];
            tt.t[b].chain_chunk = r[3];
            tt.t[b].chain_smem_trace = r[4];
        }
    }
    std::lock_guard<std::mutex> lk(ia::g_tune_mu);
    ia::g_tune = tt;
    ia::g_tune_loaded = true;
    return INDIALIGN_OK;
}

const char *indialign_last_error(void) { return ia::g_last_error.c_str(); }

void indialign_inject_failure(int count) { ia::g_inject.store(count > 0 ? count : 0); }

}  // extern "C"
