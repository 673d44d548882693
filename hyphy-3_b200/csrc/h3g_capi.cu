// h3g_capi.cu — C ABI (include/h3g.h): problem/model upload, device workspace
// and the per-evaluation launch sequence.  No exception crosses the boundary.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/h3g.h"
#include "h3g_checkpoint.h"
#include "h3g_common.cuh"
#include "h3g_fel.h"
#include "h3g_kernels.h"
#include "h3g_mixed.h"

using namespace h3g;

struct h3g_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int live_problems = 0;
    std::string err;
    void* compress = nullptr;      // alignment-compression scratch (h3g_compress.cu), kept between calls
};

namespace h3g {
void compress_scratch_free(void* p);     // h3g_compress.cu
void nuc_state_free(void* p);            // h3g_nuc.cu
}

namespace {

struct DevArena {
    std::vector<void*> ptrs;
    ~DevArena() { release(); }
    void release() { for (void* p : ptrs) cudaFree(p); ptrs.clear(); }
    template <class T> cudaError_t alloc(T** out, size_t count) {
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) { *out = nullptr; return e; }
        ptrs.push_back(p);
        *out = static_cast<T*>(p);
        return cudaSuccess;
    }
};

}  // namespace

struct h3g_problem {
    h3g_ctx* ctx = nullptr;
    h3g_batch* batch = nullptr;        // the batch this problem evaluates in (its workspace lives there)
    int n = 0, root = -1, T = 0, P = 0, Pp = 0, NI = 0, max_state = -1;
    std::vector<int> ch_off, ch, iidx, taxon, in_off, out_off, in_nodes, out_nodes, parent_h;
    std::vector<uint8_t> leaf;
    std::vector<int> bfs_order, depth_h, height_h;   // BFS order from the root, node depths and heights
    std::vector<int8_t> states_pm;     // [P][T] as uploaded (per-pattern checks on the host)
    DevArena topo_mem, model_mem, work_mem;
    int *d_ch_off = nullptr, *d_ch = nullptr, *d_iidx = nullptr, *d_taxon = nullptr, *d_in_nodes = nullptr, *d_out_nodes = nullptr;
    int* d_parent = nullptr;
    uint8_t* d_leaf = nullptr;
    int2* d_kdesc = nullptr;
    int4* d_in_info = nullptr;
    int4* d_out_info = nullptr;
    int* d_chains = nullptr;           // [in_next | in_heads | out_next | out_heads]
    int n_in_heads = 0, n_out_heads = 0;
    WaitCfg wait;                     // flag-wait limit and grid of the persistent mixed passes
    h3g_tuning tuning{};              // launch shapes asked for (0 fields: the recorded tuning or the heuristic)
    h3g_tuning applied{};             // launch shapes of the current workspace
    size_t off_in_heads = 0, off_out_next = 0, off_out_heads = 0;
    int8_t* d_states = nullptr;
    uint64_t* d_masks = nullptr;
    double* d_w = nullptr;
    // model
    bool has_model = false;
    int S = 0, M = 0, K = 0, nmod = 0, ndirs = 0, time_mode = 0, precision = 0, sentinel = 0, has_bg = 0;
    std::vector<double> h_mu;
    Model md{};
    // workspace (sized for the installed model)
    size_t work_key[4] = {0, 0, 0, 0};
    Work w{};
    MixedWork mw{};
    double* h_pin = nullptr;   // pinned: bl[n] | out[...]
    size_t h_pin_count = 0;
    double* d_bl = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaStream_t s2 = nullptr;                       // side stream: model-only work beside the pruning passes
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    float last_ms = 0.f;
    int last_launches = 0;
    size_t last_h2d = 0, last_d2h = 0;
    size_t off_out = 0, off_dir = 0, off_site = 0;    // offsets into h_pin
    // installed model: device buffers reused while the sizes stay the same
    size_t model_key[5] = {0, 0, 0, 0, 0};
    uint64_t model_hash = 0;
    double *m_pi = nullptr, *m_Q = nullptr, *m_lam = nullptr, *m_U = nullptr, *m_V = nullptr, *m_mu = nullptr;
    double *m_UT = nullptr, *m_QT = nullptr;
    double *m_cw = nullptr, *m_bw = nullptr, *m_rt = nullptr, *m_rw = nullptr, *m_dQ = nullptr;
    std::vector<double> h_bw;   // background weights as uploaded (ones when the caller gives none)
    uint8_t* m_it = nullptr;
    int* m_br = nullptr;               // per-branch class offsets (branch_classes)
    // captured evaluation graphs, keyed by (want, with host copies)
    // the site-fit evaluator of the last h3g_fel_run / h3g_meme_run, kept for the next run
    h3g::FelDevice* fel_dev = nullptr;
    void* nuc = nullptr;               // nucleotide evaluator (h3g_nuc.cu), built on first use
    struct GraphEntry { unsigned key; cudaGraphExec_t exec; int launches; };
    std::vector<GraphEntry> graphs;
    void drop_graphs() {
        for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
        graphs.clear();
    }
    ~h3g_problem() {
        drop_graphs();
        h3g::fel_device_free(fel_dev);
        if (nuc) h3g::nuc_state_free(nuc);
        if (h_pin) cudaFreeHost(h_pin);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (s2) cudaStreamDestroy(s2);
    }
    // subtree checkpointing (h3g_checkpoint.h): budget and forced target asked for, the plan of the
    // installed workspace and its device lists
    uint64_t mem_budget = 0;
    int ck_target_req = 0;
    bool ck = false;
    h3g::CkPlan ck_plan;
    DevArena ck_mem;
    int *d_ck_iidx = nullptr, *d_ck_vidx = nullptr, *d_ck_lists = nullptr;
    int2* d_ck_kdesc = nullptr;
    int4* d_ck_info = nullptr;
    struct CkOffsets { int in, out, acc, in_info, out_info, in_next, in_heads, n_in_heads, out_next, out_heads, n_out_heads; };
    std::vector<CkOffsets> ck_off;
    uint64_t ws_bytes = 0, full_bytes = 0;
    Topo topo() const {
        Topo t{};
        t.n = n; t.root = root; t.NI = NI; t.T = T; t.P = P; t.Pp = Pp; t.S = S;
        t.ch_off = d_ch_off; t.ch = d_ch; t.parent = d_parent; t.iidx = d_iidx; t.leaf = d_leaf; t.taxon = d_taxon;
        t.states = d_states; t.masks = d_masks; t.w = d_w;
        t.kdesc = d_kdesc; t.in_info = d_in_info; t.out_info = d_out_info;
        t.in_next = d_chains; t.in_heads = d_chains + off_in_heads;
        t.out_next = d_chains + off_out_next; t.out_heads = d_chains + off_out_heads;
        t.all_mask = S >= 64 ? ~uint64_t(0) : ((uint64_t(1) << S) - 1);
        t.vidx = nullptr;
        t.ncp = 0;
        return t;
    }
    // the topology an evaluation of this problem's own workspace runs on: checkpoint slots when planned
    Topo topo_eval() const {
        Topo t = topo();
        if (ck && !batch) {
            t.iidx = d_ck_iidx; t.vidx = d_ck_vidx; t.kdesc = d_ck_kdesc; t.ncp = ck_plan.ncp;
        }
        return t;
    }
};

#define H3G_TRY_CUDA(ctx, call)                                                         \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            (ctx)->err = std::string(#call) + ": " + cudaGetErrorString(e_);            \
            return e_ == cudaErrorMemoryAllocation ? H3G_ERR_OOM : H3G_ERR_CUDA;        \
        }                                                                               \
    } while (0)

static h3g_status fail(h3g_ctx* ctx, h3g_status code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

extern "C" const char* h3g_version(void) { return "hyphy3-b200 h3g 0.1"; }

extern "C" const char* h3g_last_error(const h3g_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

extern "C" h3g_status h3g_ctx_create(int device, void* cuda_stream, h3g_ctx** out) {
    if (!out) return H3G_ERR_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return H3G_ERR_CUDA;
    if (device < 0 || device >= count) return H3G_ERR_ARG;
    auto* c = new (std::nothrow) h3g_ctx;
    if (!c) return H3G_ERR_OOM;
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess) { delete c; return H3G_ERR_CUDA; }
    if (cuda_stream) {
        c->stream = static_cast<cudaStream_t>(cuda_stream);
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return H3G_ERR_CUDA; }
        c->own_stream = true;
    }
    fp64_configure();
    eigen_configure();
    mixed_configure();
    *out = c;
    return H3G_OK;
}

extern "C" h3g_status h3g_ctx_destroy(h3g_ctx* ctx) {
    if (!ctx) return H3G_ERR_ARG;
    if (ctx->live_problems > 0) return fail(ctx, H3G_ERR_STATE, "destroy every problem before its context");
    cudaSetDevice(ctx->device);
    if (ctx->compress) h3g::compress_scratch_free(ctx->compress);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return H3G_OK;
}

extern "C" h3g_status h3g_problem_create(h3g_ctx* ctx, int n_nodes, const int32_t* parent, const uint8_t* is_leaf,
                                         const int32_t* leaf_taxon, int n_taxa, int n_patterns, const int8_t* states,
                                         const uint64_t* masks, const double* weights, h3g_problem** out) {
    if (!ctx || !out) return H3G_ERR_ARG;
    *out = nullptr;
    if (n_nodes < 2 || !parent || !is_leaf || !leaf_taxon) return fail(ctx, H3G_ERR_ARG, "tree arrays missing or fewer than 2 nodes");
    if (n_taxa < 0 || n_patterns < 0 || (n_patterns > 0 && (!states || !masks || !weights)))
        return fail(ctx, H3G_ERR_ARG, "pattern arrays missing");
    try {
        cudaSetDevice(ctx->device);
        auto* pr = new h3g_problem;
        std::unique_ptr<h3g_problem> guard(pr);
        pr->ctx = ctx;
        const int n = n_nodes;
        pr->n = n; pr->T = n_taxa; pr->P = n_patterns;
        pr->Pp = std::max(TP, (n_patterns + TP - 1) / TP * TP);
        pr->leaf.assign(is_leaf, is_leaf + n);
        pr->taxon.assign(n, -1);
        std::vector<std::vector<int>> kids(n);
        for (int i = 0; i < n; ++i) {
            const int p = parent[i];
            if (p < 0) {
                if (pr->root >= 0) return fail(ctx, H3G_ERR_ARG, "more than one root");
                pr->root = i;
            } else {
                if (p >= n || p == i) return fail(ctx, H3G_ERR_ARG, "parent id out of range");
                if (is_leaf[p]) return fail(ctx, H3G_ERR_ARG, "a leaf has children");
                kids[p].push_back(i);
            }
            if (is_leaf[i]) {
                const int tx = leaf_taxon[i];
                if (tx >= n_taxa) return fail(ctx, H3G_ERR_ARG, "leaf taxon index out of range");
                pr->taxon[i] = tx < 0 ? -1 : tx;
            }
        }
        if (pr->root < 0) return fail(ctx, H3G_ERR_ARG, "no root");
        if (is_leaf[pr->root]) return fail(ctx, H3G_ERR_ARG, "root is a leaf");
        // heights (inside levels) and depths (outside levels); detects cycles
        std::vector<int> order, depth(n, -1), height(n, 0);
        order.reserve(n);
        order.push_back(pr->root);
        depth[pr->root] = 0;
        for (size_t q = 0; q < order.size(); ++q)
            for (int c : kids[order[q]]) {
                if (depth[c] >= 0) return fail(ctx, H3G_ERR_ARG, "cycle in parent array");
                depth[c] = depth[order[q]] + 1;
                order.push_back(c);
            }
        if (int(order.size()) != n) return fail(ctx, H3G_ERR_ARG, "parent array is not a single tree");
        for (int q = n - 1; q >= 0; --q) {
            const int u = order[q];
            for (int c : kids[u]) height[u] = std::max(height[u], height[c] + 1);
            if (!is_leaf[u] && kids[u].empty()) height[u] = 1;
        }
        pr->iidx.assign(n, -1);
        pr->ch_off.assign(n + 1, 0);
        for (int i = 0; i < n; ++i) {
            if (!is_leaf[i]) pr->iidx[i] = pr->NI++;
            pr->ch_off[i + 1] = pr->ch_off[i] + int(kids[i].size());
            for (int c : kids[i]) pr->ch.push_back(c);
        }
        pr->bfs_order = order;
        pr->depth_h = depth;
        pr->height_h = height;
        int H = 0, Dp = 0;
        for (int i = 0; i < n; ++i) if (!is_leaf[i]) { H = std::max(H, height[i]); Dp = std::max(Dp, depth[i]); }
        pr->in_off.assign(1, 0);
        for (int h = 1; h <= H; ++h) {
            for (int i = 0; i < n; ++i) if (!is_leaf[i] && height[i] == h) pr->in_nodes.push_back(i);
            pr->in_off.push_back(int(pr->in_nodes.size()));
        }
        // outside levels: the children of the internal nodes at each depth
        pr->out_off.assign(1, 0);
        for (int d = 0; d <= Dp; ++d) {
            for (int i = 0; i < n; ++i)
                if (!is_leaf[i] && depth[i] == d) for (int c : kids[i]) pr->out_nodes.push_back(c);
            pr->out_off.push_back(int(pr->out_nodes.size()));
        }
        pr->parent_h.assign(parent, parent + n);
        if (n_patterns > 0) pr->states_pm.assign(states, states + size_t(n_patterns) * n_taxa);
        // patterns, taxon-major with padding (missing data, weight 0)
        const int Pp = pr->Pp, T = n_taxa;
        std::vector<int8_t> st(size_t(std::max(T, 1)) * Pp, int8_t(-1));
        std::vector<uint64_t> mk(size_t(std::max(T, 1)) * Pp, ~uint64_t(0));
        std::vector<double> wt(Pp, 0.0);
        for (int p = 0; p < n_patterns; ++p) {
            if (!(weights[p] >= 0.0) || !std::isfinite(weights[p])) return fail(ctx, H3G_ERR_ARG, "pattern weights must be finite and >= 0");
            wt[p] = weights[p];
            for (int t = 0; t < T; ++t) {
                const int8_t sv = states[size_t(p) * T + t];
                if (sv >= SP) return fail(ctx, H3G_ERR_ARG, "state index >= 64");
                pr->max_state = std::max<int>(pr->max_state, sv);
                st[size_t(t) * Pp + p] = states[size_t(p) * T + t];
                mk[size_t(t) * Pp + p] = masks[size_t(p) * T + t];
            }
        }
        auto& A = pr->topo_mem;
        cudaStream_t s = ctx->stream;
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_ch_off, n + 1));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_ch, std::max<size_t>(pr->ch.size(), 1)));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_iidx, n));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_parent, n));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_taxon, n));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_leaf, n));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_in_nodes, std::max<size_t>(pr->in_nodes.size(), 1)));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_out_nodes, std::max<size_t>(pr->out_nodes.size(), 1)));
        // descriptors for the persistent passes
        std::vector<int2> kdesc(std::max<size_t>(pr->ch.size(), 1));
        for (size_t j = 0; j < pr->ch.size(); ++j) {
            const int c = pr->ch[j];
            kdesc[j] = make_int2(c, is_leaf[c] ? pr->taxon[c] : -(2 + pr->iidx[c]));
        }
        std::vector<int4> in_info(std::max<size_t>(pr->in_nodes.size(), 1));
        for (size_t k = 0; k < pr->in_nodes.size(); ++k) {
            const int u = pr->in_nodes[k];
            in_info[k] = make_int4(u, pr->iidx[u], pr->ch_off[u], pr->ch_off[u + 1]);
        }
        std::vector<int4> out_info(2 * std::max<size_t>(pr->out_nodes.size(), 1));
        for (size_t k = 0; k < pr->out_nodes.size(); ++k) {
            const int c = pr->out_nodes[k], u = parent[c];
            out_info[2 * k] = make_int4(c, u, pr->iidx[u], is_leaf[c] ? -1 : pr->iidx[c]);
            out_info[2 * k + 1] = make_int4(pr->ch_off[u], pr->ch_off[u + 1], 0, 0);
        }
        // chains (see Topo): inside, a node whose parent has no other internal child hands its
        // message to the parent in the same CTA; outside, a node continues with its deepest
        // internal child.  Heads keep the pass order, so every wait is on an earlier claim.
        std::vector<int> in_pos(n, -1), out_pos(n, -1);
        for (size_t k = 0; k < pr->in_nodes.size(); ++k) in_pos[pr->in_nodes[k]] = int(k);
        for (size_t k = 0; k < pr->out_nodes.size(); ++k) out_pos[pr->out_nodes[k]] = int(k);
        std::vector<int> n_int(n, 0);
        for (int i = 0; i < n; ++i)
            for (int c : kids[i]) n_int[i] += is_leaf[c] ? 0 : 1;
        std::vector<int> in_next(pr->in_nodes.size(), -1), in_heads, out_next(pr->out_nodes.size(), -1), out_heads;
        std::vector<char> fused_in(pr->in_nodes.size(), 0), fused_out(pr->out_nodes.size(), 0);
        for (size_t k = 0; k < pr->in_nodes.size(); ++k) {
            const int u = pr->in_nodes[k], par = parent[u];
            if (par >= 0 && n_int[par] == 1) {
                in_next[k] = in_pos[par];
                fused_in[size_t(in_pos[par])] = 1;
            }
        }
        for (size_t k = 0; k < pr->in_nodes.size(); ++k)
            if (!fused_in[k]) in_heads.push_back(int(k));
        for (size_t k = 0; k < pr->out_nodes.size(); ++k) {
            const int c = pr->out_nodes[k];
            if (is_leaf[c]) continue;
            int best = -1;
            for (int d : kids[c])
                if (!is_leaf[d] && (best < 0 || height[d] > height[best])) best = d;
            if (best >= 0) {
                out_next[k] = out_pos[best];
                fused_out[size_t(out_pos[best])] = 1;
            }
        }
        for (size_t k = 0; k < pr->out_nodes.size(); ++k)
            if (!fused_out[k]) out_heads.push_back(int(k));
        pr->n_in_heads = int(in_heads.size());
        pr->n_out_heads = int(out_heads.size());
        std::vector<int> chains(in_next);
        pr->off_in_heads = chains.size();
        chains.insert(chains.end(), in_heads.begin(), in_heads.end());
        pr->off_out_next = chains.size();
        chains.insert(chains.end(), out_next.begin(), out_next.end());
        pr->off_out_heads = chains.size();
        chains.insert(chains.end(), out_heads.begin(), out_heads.end());
        if (chains.empty()) chains.push_back(-1);
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_chains, chains.size()));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_chains, chains.data(), chains.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_kdesc, kdesc.size()));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_in_info, in_info.size()));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_out_info, out_info.size()));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_kdesc, kdesc.data(), kdesc.size() * sizeof(int2), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_in_info, in_info.data(), in_info.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_out_info, out_info.data(), out_info.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_states, st.size()));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_masks, mk.size()));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_w, wt.size()));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_ch_off, pr->ch_off.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
        if (!pr->ch.empty()) H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_ch, pr->ch.data(), pr->ch.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_iidx, pr->iidx.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_parent, pr->parent_h.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_taxon, pr->taxon.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_leaf, pr->leaf.data(), n, cudaMemcpyHostToDevice, s));
        if (!pr->in_nodes.empty())
            H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_in_nodes, pr->in_nodes.data(), pr->in_nodes.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        if (!pr->out_nodes.empty())
            H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_out_nodes, pr->out_nodes.data(), pr->out_nodes.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_states, st.data(), st.size(), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_masks, mk.data(), mk.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_w, wt.data(), wt.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaStreamSynchronize(s));
        H3G_TRY_CUDA(ctx, cudaEventCreate(&pr->ev0));
        H3G_TRY_CUDA(ctx, cudaEventCreate(&pr->ev1));
        H3G_TRY_CUDA(ctx, cudaStreamCreateWithFlags(&pr->s2, cudaStreamNonBlocking));
        H3G_TRY_CUDA(ctx, cudaEventCreateWithFlags(&pr->ev_fork, cudaEventDisableTiming));
        H3G_TRY_CUDA(ctx, cudaEventCreateWithFlags(&pr->ev_join, cudaEventDisableTiming));
        *out = guard.release();
        ctx->live_problems++;
        return H3G_OK;
    } catch (const std::bad_alloc&) {
        return fail(ctx, H3G_ERR_OOM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(ctx, H3G_ERR_ARG, e.what());
    }
}

namespace h3g {

cudaStream_t ctx_stream(h3g_ctx* ctx) { return ctx->stream; }
int ctx_device(h3g_ctx* ctx) { return ctx->device; }
h3g_status ctx_fail(h3g_ctx* ctx, h3g_status st, const std::string& msg) { return fail(ctx, st, msg); }
void*& ctx_compress_scratch(h3g_ctx* ctx) { return ctx->compress; }

Topo problem_topo(h3g_problem* pr, int S) {
    Topo t = pr->topo();
    t.S = S;
    t.all_mask = S >= 64 ? ~uint64_t(0) : ((uint64_t(1) << S) - 1);
    return t;
}

cudaStream_t problem_stream(h3g_problem* pr) { return pr->ctx->stream; }

bool fel_problem_view(h3g_problem* pr, FelProblemView* v) {
    if (!pr || !v) return false;
    v->n = pr->n; v->root = pr->root; v->T = pr->T; v->P = pr->P;
    v->parent = pr->parent_h.data(); v->leaf = pr->leaf.data(); v->taxon = pr->taxon.data();
    v->ch_off = pr->ch_off.data(); v->ch = pr->ch.data();
    v->states = pr->states_pm.data();
    v->device = pr->ctx->device;
    return true;
}

void fel_set_error(h3g_problem* pr, const std::string& msg) {
    if (pr && pr->ctx) pr->ctx->err = msg;
}

FelDevice*& problem_fel_device(h3g_problem* pr) { return pr->fel_dev; }
void*& problem_nuc_state(h3g_problem* pr) { return pr->nuc; }
int problem_max_state(h3g_problem* pr) { return pr->max_state; }

void fel_record_transfer(h3g_problem* pr, size_t h2d, size_t d2h, int launches, double ms) {
    pr->last_h2d = h2d;
    pr->last_d2h = d2h;
    pr->last_launches = launches;
    pr->last_ms = float(ms);
}

}  // namespace h3g

extern "C" h3g_status h3g_problem_destroy(h3g_problem* prob) {
    if (!prob) return H3G_ERR_ARG;
    if (prob->batch) return fail(prob->ctx, H3G_ERR_STATE, "destroy the problem's batch first");
    cudaSetDevice(prob->ctx->device);
    cudaStreamSynchronize(prob->ctx->stream);
    prob->ctx->live_problems--;
    delete prob;
    return H3G_OK;
}

static void pad_matrix(const double* src, int S, double* dst) {
    std::fill(dst, dst + SP2, 0.0);
    for (int i = 0; i < S; ++i) std::copy(src + size_t(i) * S, src + size_t(i) * S + S, dst + size_t(i) * SP);
}

static size_t n_out_of(const h3g_problem* pr) { return 2 + size_t(pr->n) + 2 * size_t(pr->nmod) + pr->M; }

// Tunings recorded by h3g_autotune, per problem shape (process-wide).
struct TuneKey {
    int device, n, NI, Pp, M, K, nmod, ndirs, precision;
    bool operator<(const TuneKey& o) const {
        const int a[] = {device, n, NI, Pp, M, K, nmod, ndirs, precision};
        const int b[] = {o.device, o.n, o.NI, o.Pp, o.M, o.K, o.nmod, o.ndirs, o.precision};
        return std::lexicographical_compare(a, a + 9, b, b + 9);
    }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, h3g_tuning> g_tunings;

static TuneKey tune_key(const h3g_problem* pr, int M, int K, int nmod, int ndirs) {
    return {pr->ctx->device, pr->n, pr->NI, pr->Pp, M, K, nmod, ndirs, pr->precision};
}

// The launch shapes a problem runs with: the fields it set, else the tuning recorded for its shape,
// else 0 (the heuristics).
static h3g_tuning effective_tuning(const h3g_problem* pr, int M, int K, int nmod, int ndirs) {
    h3g_tuning tu = pr->tuning;
    if (tu.a_chunk > 0 && tu.ctas_per_sm > 0 && tu.frechet_groups > 0) return tu;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tunings.find(tune_key(pr, M, K, nmod, ndirs));
    if (it != g_tunings.end()) {
        if (tu.a_chunk <= 0) tu.a_chunk = it->second.a_chunk;
        if (tu.ctas_per_sm <= 0) tu.ctas_per_sm = it->second.ctas_per_sm;
        if (tu.frechet_groups <= 0) tu.frechet_groups = it->second.frechet_groups;
    }
    return tu;
}

// Element counts of every device buffer of one evaluation workspace, for a problem of n nodes, NI
// internal nodes, Pp padded patterns and a model of (M, K, nmod, ndirs); plus the A-accumulation
// chunking and the Frechet branch groups those dimensions get.  A batch slot serves several problems
// with one workspace: its counts are the element-wise maximum over them (offsets inside a buffer come
// from the evaluated problem's own dimensions, so a larger buffer serves a smaller problem).
struct WsLayout {
    size_t n = 0, mats = 0, rsz = 0, pcols = 0, ecols = 0, gt = 0, apart = 0, afull = 0, hpart = 0, gsz = 0, hsz = 0,
           dirpart = 0, gdir = 0, out = 0, part = 0, vf = 0;
    int nchunk = 1, chunk = TP, ngroups = 1;
    void max_with(const WsLayout& o) {
        size_t* a[] = {&n, &mats, &rsz, &pcols, &ecols, &gt, &apart, &afull, &hpart, &gsz, &hsz, &dirpart, &gdir, &out, &part, &vf};
        const size_t* b[] = {&o.n, &o.mats, &o.rsz, &o.pcols, &o.ecols, &o.gt, &o.apart, &o.afull, &o.hpart, &o.gsz, &o.hsz,
                             &o.dirpart, &o.gdir, &o.out, &o.part, &o.vf};
        for (size_t i = 0; i < sizeof(a) / sizeof(a[0]); ++i) *a[i] = std::max(*a[i], *b[i]);
    }
};

// part_nodes / vf_nodes: partial slots of internal nodes and gradient-operand slots (NI and n, or
// fewer under a checkpoint plan).
static WsLayout ws_layout(size_t n, size_t NI, size_t Pp, int M, int K, int nmod, int ndirs, const h3g_tuning& tu,
                          size_t part_nodes = 0, size_t vf_nodes = 0) {
    (void)K;
    if (!part_nodes) part_nodes = NI;
    if (!vf_nodes) vf_nodes = n;
    WsLayout L;
    L.n = n;
    L.mats = size_t(M) * n * SP2;
    L.rsz = size_t(M) * n * SP;
    L.pcols = size_t(M) * Pp;
    L.ecols = part_nodes * M * Pp;
    L.gt = size_t(M) * n;
    // enough A chunks for ~600 CTAs, never below 256 patterns per chunk
    const int want_chunks = std::max<int>(1, int((600 + n * M - 1) / (n * M)));
    const int max_chunks = std::max<int>(1, int(Pp / 256));
    L.nchunk = std::min(want_chunks, max_chunks);
    L.chunk = int((Pp / TP + L.nchunk - 1) / L.nchunk) * TP;
    if (tu.a_chunk > 0) L.chunk = int(std::min<size_t>(Pp, size_t(std::max(2 * TP, tu.a_chunk / TP * TP))));
    L.nchunk = int((Pp + L.chunk - 1) / L.chunk);
    L.apart = n * M * size_t(L.nchunk) * SP2;
    L.afull = n * M * SP2;
    // Frechet branch groups: about two CTAs per SM over (group, rate class, model)
    L.ngroups = int(std::max<size_t>(1, std::min<size_t>(n, (296 + size_t(M) * nmod - 1) / (size_t(M) * nmod))));
    if (tu.frechet_groups > 0) L.ngroups = int(std::min<size_t>(n, size_t(tu.frechet_groups)));
    const size_t G = size_t(L.ngroups);
    L.hpart = size_t(nmod) * M * G * SP2;
    L.gsz = size_t(nmod) * M * G;
    L.hsz = size_t(nmod) * SP2;
    L.dirpart = size_t(std::max(ndirs, 1)) * nmod * 17;
    L.gdir = size_t(std::max(ndirs, 1)) * nmod * SP2;
    L.out = 2 + n + 2 * size_t(nmod) + M;
    L.part = part_nodes * M * SP * Pp;
    L.vf = vf_nodes * M * SP * Pp;
    return L;
}

// Device bytes ws_alloc takes for layout L.
static uint64_t ws_bytes(const WsLayout& L, int precision) {
    const uint64_t f64 = 3 * L.mats + L.rsz + 4 * L.pcols + L.gt + L.apart + L.afull + L.hpart + 2 * L.gsz + L.hsz +
                         L.dirpart + L.gdir + L.out;
    uint64_t b = f64 * 8 + 2 * uint64_t(L.ecols) * 4 + 4;
    if (precision == H3G_PREC_FP64)
        b += (3 * uint64_t(L.part) + L.vf) * 8;
    else   // FP32 partials, three exponent planes, FP32 P^T and row sums, six BF16 split planes, two flag planes
        b += (3 * uint64_t(L.part) + L.vf) * 4 + 3 * uint64_t(L.ecols) * 4 + L.mats * 4 + L.rsz * 4 + 6 * uint64_t(L.mats) * 2 +
             2 * uint64_t(L.ecols / TP) * 4 + 16;
    return b;
}

// Allocate a workspace of layout L (FP64 or mixed partials) into A; w.bl is left to the caller.
static h3g_status ws_alloc(h3g_ctx* ctx, const WsLayout& L, int precision, DevArena& A, Work& w, MixedWork& mw) {
    w = Work{};
    mw = MixedWork{};
    w.nchunk = L.nchunk;
    w.chunk = L.chunk;
    w.ngroups = L.ngroups;
    H3G_TRY_CUDA(ctx, A.alloc(&w.P, L.mats));
    H3G_TRY_CUDA(ctx, A.alloc(&w.PT, L.mats));
    H3G_TRY_CUDA(ctx, A.alloc(&w.dP, L.mats));
    H3G_TRY_CUDA(ctx, A.alloc(&w.rs, L.rsz));
    H3G_TRY_CUDA(ctx, A.alloc(&w.f, L.pcols));
    H3G_TRY_CUDA(ctx, A.alloc(&w.rw, L.pcols));
    H3G_TRY_CUDA(ctx, A.alloc(&w.contrib, L.pcols));
    H3G_TRY_CUDA(ctx, A.alloc(&w.site, L.pcols));
    H3G_TRY_CUDA(ctx, A.alloc(&w.Ecum, L.ecols));
    H3G_TRY_CUDA(ctx, A.alloc(&w.Eown, L.ecols));
    H3G_TRY_CUDA(ctx, A.alloc(&w.gt, L.gt));
    H3G_TRY_CUDA(ctx, A.alloc(&w.Apart, L.apart));
    H3G_TRY_CUDA(ctx, A.alloc(&w.Afull, L.afull));
    H3G_TRY_CUDA(ctx, A.alloc(&w.Hpart, L.hpart));
    H3G_TRY_CUDA(ctx, A.alloc(&w.gc, L.gsz));
    H3G_TRY_CUDA(ctx, A.alloc(&w.stg, L.gsz));
    H3G_TRY_CUDA(ctx, A.alloc(&w.H, L.hsz));
    H3G_TRY_CUDA(ctx, A.alloc(&w.dirpart, L.dirpart));
    H3G_TRY_CUDA(ctx, A.alloc(&w.G, L.gdir));
    H3G_TRY_CUDA(ctx, A.alloc(&w.out, L.out));
    H3G_TRY_CUDA(ctx, A.alloc(&w.err, 1));
    cudaMemsetAsync(w.err, 0, sizeof(int), ctx->stream);
    if (precision == H3G_PREC_FP64) {
        H3G_TRY_CUDA(ctx, A.alloc(&w.D, L.part));
        H3G_TRY_CUDA(ctx, A.alloc(&w.Ms, L.part));
        H3G_TRY_CUDA(ctx, A.alloc(&w.U, L.part));
        H3G_TRY_CUDA(ctx, A.alloc(&w.Vf, L.vf));
    } else {
        MixedSizes z;
        z.part = L.part; z.vf = L.vf; z.cols = L.ecols; z.mats = L.mats; z.rs = L.rsz; z.flags = L.ecols / TP;
        h3g_status st = mixed_alloc(mw, A.ptrs, z, ctx->stream);
        if (st != H3G_OK) return fail(ctx, st, "mixed-precision workspace allocation failed");
    }
    cudaMemsetAsync(w.gc, 0, L.gsz * sizeof(double), ctx->stream);
    cudaMemsetAsync(w.stg, 0, L.gsz * sizeof(double), ctx->stream);
    // batch slots run on streams of their own: the zeroing completes before any of them starts
    H3G_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return H3G_OK;
}

// Pinned host buffer of a problem: bl[n] | out | directional partials | per-pattern lnL.
static h3g_status ensure_host_buffer(h3g_problem* pr, int M, int nmod, int ndirs) {
    const size_t n_out = 2 + size_t(pr->n) + 2 * size_t(nmod) + M;
    const size_t off_out = size_t(pr->n), off_dir = off_out + n_out;
    const size_t off_site = off_dir + size_t(std::max(ndirs, 1)) * nmod * 17;
    const size_t count = off_site + size_t(std::max(pr->P, 1));
    if (pr->h_pin && count <= pr->h_pin_count) {
        pr->off_out = off_out; pr->off_dir = off_dir; pr->off_site = off_site;
        return H3G_OK;
    }
    cudaStreamSynchronize(pr->ctx->stream);
    pr->drop_graphs();
    if (pr->h_pin) { cudaFreeHost(pr->h_pin); pr->h_pin = nullptr; }
    pr->off_out = off_out; pr->off_dir = off_dir; pr->off_site = off_site;
    pr->h_pin_count = count;
    H3G_TRY_CUDA(pr->ctx, cudaMallocHost(reinterpret_cast<void**>(&pr->h_pin), count * sizeof(double)));
    return H3G_OK;
}

static std::vector<std::vector<int>> children_of(const h3g_problem* pr) {
    std::vector<std::vector<int>> kids(pr->n);
    for (int u = 0; u < pr->n; ++u) kids[u].assign(pr->ch.begin() + pr->ch_off[u], pr->ch.begin() + pr->ch_off[u + 1]);
    return kids;
}

// Upload a checkpoint plan's slots and per-block lists: node lists of the FP64 level launches, and
// the item descriptors and chains of the mixed path's persistent passes restricted to each block
// (a chain never enters a block root, so a block's recompute list is its full list without the
// root, which comes last).
static h3g_status upload_checkpoints(h3g_problem* pr) {
    h3g_ctx* ctx = pr->ctx;
    const h3g::CkPlan& pl = pr->ck_plan;
    const int n = pr->n;
    const auto kids = children_of(pr);
    std::vector<int> n_int(n, 0);
    for (int u = 0; u < n; ++u)
        for (int c : kids[u]) n_int[u] += pr->leaf[c] ? 0 : 1;
    std::vector<int2> kdesc(std::max<size_t>(pr->ch.size(), 1));
    for (size_t j = 0; j < pr->ch.size(); ++j) {
        const int c = pr->ch[j];
        kdesc[j] = make_int2(c, pr->leaf[c] ? pr->taxon[c] : -(2 + pl.iidx[c]));
    }
    std::vector<int> lists;
    std::vector<int4> info;
    std::vector<int> pos(n, -1);
    pr->ck_off.clear();
    for (const h3g::CkBlock& B : pl.blocks) {
        h3g_problem::CkOffsets o{};
        o.in = int(lists.size());
        lists.insert(lists.end(), B.in_nodes.begin(), B.in_nodes.end());
        o.out = int(lists.size());
        lists.insert(lists.end(), B.out_kids.begin(), B.out_kids.end());
        o.acc = int(lists.size());
        lists.insert(lists.end(), B.acc.begin(), B.acc.end());
        // inside items
        o.in_info = int(info.size());
        for (size_t k = 0; k < B.in_nodes.size(); ++k) {
            const int u = B.in_nodes[k];
            pos[u] = int(k);
            info.push_back(make_int4(u, pl.iidx[u], pr->ch_off[u], pr->ch_off[u + 1]));
        }
        std::vector<int> nxt(B.in_nodes.size(), -1), heads;
        std::vector<char> fused(B.in_nodes.size(), 0);
        for (size_t k = 0; k < B.in_nodes.size(); ++k) {
            const int u = B.in_nodes[k], par = pr->parent_h[u];
            if (u != B.root && par != B.root && n_int[par] == 1) {
                nxt[k] = pos[par];
                fused[size_t(pos[par])] = 1;
            }
        }
        for (size_t k = 0; k < B.in_nodes.size(); ++k)
            if (!fused[k]) heads.push_back(int(k));
        o.in_next = int(lists.size());
        lists.insert(lists.end(), nxt.begin(), nxt.end());
        o.in_heads = int(lists.size());
        o.n_in_heads = int(heads.size());
        lists.insert(lists.end(), heads.begin(), heads.end());
        for (int u : B.in_nodes) pos[u] = -1;
        // outside items
        o.out_info = int(info.size());
        for (size_t k = 0; k < B.out_kids.size(); ++k) {
            const int c = B.out_kids[k], u = pr->parent_h[c];
            pos[c] = int(k);
            info.push_back(make_int4(c, u, pl.iidx[u], pr->leaf[c] ? -1 : pl.iidx[c]));
            info.push_back(make_int4(pr->ch_off[u], pr->ch_off[u + 1], 0, 0));
        }
        std::vector<int> onxt(B.out_kids.size(), -1), oheads;
        std::vector<char> ofused(B.out_kids.size(), 0);
        for (size_t k = 0; k < B.out_kids.size(); ++k) {
            const int c = B.out_kids[k];
            if (pr->leaf[c] || pl.is_ckpt[c]) continue;
            int best = -1;
            for (int d : kids[c])
                if (!pr->leaf[d] && (best < 0 || pr->height_h[d] > pr->height_h[best])) best = d;
            if (best >= 0) {
                onxt[k] = pos[best];
                ofused[size_t(pos[best])] = 1;
            }
        }
        for (size_t k = 0; k < B.out_kids.size(); ++k)
            if (!ofused[k]) oheads.push_back(int(k));
        o.out_next = int(lists.size());
        lists.insert(lists.end(), onxt.begin(), onxt.end());
        o.out_heads = int(lists.size());
        o.n_out_heads = int(oheads.size());
        lists.insert(lists.end(), oheads.begin(), oheads.end());
        for (int c : B.out_kids) pos[c] = -1;
        pr->ck_off.push_back(o);
    }
    if (lists.empty()) lists.push_back(-1);
    if (info.empty()) info.push_back(make_int4(0, 0, 0, 0));
    auto& A = pr->ck_mem;
    A.release();
    cudaStream_t s = ctx->stream;
    H3G_TRY_CUDA(ctx, A.alloc(&pr->d_ck_iidx, size_t(n)));
    H3G_TRY_CUDA(ctx, A.alloc(&pr->d_ck_vidx, size_t(n)));
    H3G_TRY_CUDA(ctx, A.alloc(&pr->d_ck_kdesc, kdesc.size()));
    H3G_TRY_CUDA(ctx, A.alloc(&pr->d_ck_lists, lists.size()));
    H3G_TRY_CUDA(ctx, A.alloc(&pr->d_ck_info, info.size()));
    H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_ck_iidx, pl.iidx.data(), size_t(n) * sizeof(int), cudaMemcpyHostToDevice, s));
    H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_ck_vidx, pl.vidx.data(), size_t(n) * sizeof(int), cudaMemcpyHostToDevice, s));
    H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_ck_kdesc, kdesc.data(), kdesc.size() * sizeof(int2), cudaMemcpyHostToDevice, s));
    H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_ck_lists, lists.data(), lists.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_ck_info, info.data(), info.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
    H3G_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    return H3G_OK;
}

// The workspace layout of (M, K, nmod, ndirs) and whether it is checkpointed: the full layout when it fits
// the budget (the problem's, else the device's free memory plus the `held` bytes about to be released) and
// no block size is forced; else the plan with the largest block size whose layout fits.
static h3g_status choose_layout(h3g_problem* pr, int M, int K, int nmod, int ndirs, const h3g_tuning& tu, uint64_t held,
                                WsLayout& L) {
    const WsLayout full = ws_layout(size_t(pr->n), size_t(pr->NI), size_t(pr->Pp), M, K, nmod, ndirs, tu);
    pr->full_bytes = ws_bytes(full, pr->precision);
    uint64_t budget = pr->mem_budget;
    if (!budget) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) fr = 0;
        budget = uint64_t(double(fr + held) * 0.92);
    }
    pr->ck = false;
    if (pr->ck_target_req <= 0 && (pr->full_bytes <= budget || (pr->mem_budget == 0 && budget == 0))) {
        L = full;
        return H3G_OK;
    }
    const auto kids = children_of(pr);
    auto make = [&](int target) {
        return h3g::plan_checkpoints(pr->n, pr->root, kids, pr->leaf.data(), pr->bfs_order, pr->depth_h, pr->height_h, target);
    };
    auto layout_of = [&](const h3g::CkPlan& p) {
        return ws_layout(size_t(pr->n), size_t(pr->NI), size_t(pr->Pp), M, K, nmod, ndirs, tu, size_t(p.ncp + p.scratch_int),
                         size_t(p.ncp + p.scratch_all));
    };
    if (pr->ck_target_req > 0) {
        pr->ck_plan = make(pr->ck_target_req);
        L = layout_of(pr->ck_plan);
        pr->ck = true;
        return H3G_OK;
    }
    for (int target = pr->n;; target = std::max(2, target * 4 / 5)) {
        h3g::CkPlan p = make(target);
        const WsLayout Lc = layout_of(p);
        if (ws_bytes(Lc, pr->precision) <= budget) {
            pr->ck_plan = std::move(p);
            L = Lc;
            pr->ck = true;
            return H3G_OK;
        }
        if (target == 2) break;
    }
    return fail(pr->ctx, H3G_ERR_OOM, "the evaluation workspace does not fit the memory budget even with subtree checkpoints");
}

// Allocate the evaluation workspace for (M, K, nmod, ndirs); reuses it when unchanged.
static h3g_status ensure_workspace(h3g_problem* pr, int M, int K, int nmod, int ndirs) {
    h3g_ctx* ctx = pr->ctx;
    if (!pr->d_bl) H3G_TRY_CUDA(ctx, pr->topo_mem.alloc(&pr->d_bl, size_t(pr->n)));
    if (h3g_status st = ensure_host_buffer(pr, M, nmod, ndirs); st != H3G_OK) return st;
    if (pr->batch) return H3G_OK;       // a batch member evaluates in its batch's slot workspaces
    // grow-only: a workspace sized for larger (M, K, models, directions) serves every smaller model (strides and
    // offsets come from the installed model), so optimisers that alternate gradient and value-only evaluations
    // (different direction counts) do not reallocate
    size_t key[4] = {size_t(M), size_t(K), size_t(nmod), size_t(ndirs)};
    const h3g_tuning tu = effective_tuning(pr, M, K, nmod, ndirs);
    pr->wait.ctas_per_sm = tu.ctas_per_sm > 0 ? tu.ctas_per_sm : 2;
    const bool same_tuning = tu.a_chunk == pr->applied.a_chunk && tu.frechet_groups == pr->applied.frechet_groups;
    if (pr->w.P && same_tuning && key[0] <= pr->work_key[0] && key[1] <= pr->work_key[1] && key[2] <= pr->work_key[2] &&
        key[3] <= pr->work_key[3])
        return H3G_OK;
    if (pr->w.P)
        for (int i = 0; i < 4; ++i) key[i] = std::max(key[i], pr->work_key[i]);
    M = int(key[0]); K = int(key[1]); nmod = int(key[2]); ndirs = int(key[3]);
    cudaStreamSynchronize(ctx->stream);
    pr->drop_graphs();
    const uint64_t held = pr->w.P ? pr->ws_bytes : 0;
    pr->work_mem.release();
    pr->w = Work{};
    pr->mw = MixedWork{};
    pr->ws_bytes = 0;
    WsLayout L;
    h3g_status st = choose_layout(pr, M, K, nmod, ndirs, tu, held, L);
    if (st == H3G_OK && pr->ck) st = upload_checkpoints(pr);
    if (st != H3G_OK) { pr->ck = false; return st; }
    std::copy(key, key + 4, pr->work_key);
    pr->applied = tu;
    st = ws_alloc(ctx, L, pr->precision, pr->work_mem, pr->w, pr->mw);
    pr->w.bl = pr->d_bl;
    if (st != H3G_OK) { pr->work_mem.release(); pr->w = Work{}; pr->mw = MixedWork{}; pr->ck = false; return st; }
    pr->ws_bytes = ws_bytes(L, pr->precision);
    return st;
}

static uint64_t hash_bytes(uint64_t h, const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        std::memcpy(&w, c + i, 8);
        h = (h ^ w) * 0x9E3779B97F4A7C15ull;
        h ^= h >> 29;
    }
    for (; i < n; ++i) { h ^= c[i]; h *= 1099511628211ull; }
    return h;
}

extern "C" h3g_status h3g_model_set(h3g_problem* pr, const h3g_model_desc* d) {
    if (!pr || !d) return H3G_ERR_ARG;
    h3g_ctx* ctx = pr->ctx;
    if (d->S < 1 || d->S > SP) return fail(ctx, H3G_ERR_ARG, "S must be in [1, 64]");
    if (d->K < 1 || d->M < 1 || d->M > kMaxRateClasses) return fail(ctx, H3G_ERR_ARG, "need K >= 1 and 1 <= M <= 16");
    if (d->has_bg < 0 || d->n_models != d->K + d->has_bg) return fail(ctx, H3G_ERR_ARG, "n_models must equal K + has_bg");
    if (d->has_bg > 1 && !d->bg_w) return fail(ctx, H3G_ERR_ARG, "several background classes need bg_w");
    if (d->branch_classes) {
        if (d->has_bg != 0 || d->is_test) return fail(ctx, H3G_ERR_ARG, "per-branch classes exclude has_bg and is_test");
        const int32_t* o = d->branch_classes;
        for (int b = 0; b < pr->n; ++b) {
            if (o[b] < 0 || o[b + 1] > d->K || o[b + 1] < o[b]) return fail(ctx, H3G_ERR_ARG, "branch_classes must be non-decreasing in [0, K]");
            if (b != pr->root && o[b + 1] == o[b]) return fail(ctx, H3G_ERR_ARG, "every branch needs at least one class");
        }
    }
    // U, V and lam all NULL: the device diagonalises every Q_k (h3g_eigen.cu)
    const bool dev_eig = !d->U && !d->V && !d->lam;
    if (!d->pi || !d->Q || (!dev_eig && (!d->lam || !d->U || !d->V)) || !d->class_w || !d->rates || !d->rate_w)
        return fail(ctx, H3G_ERR_ARG, "model arrays missing");
    if (d->time_mode == H3G_TIME_NORMALIZED && !d->mu && !dev_eig) return fail(ctx, H3G_ERR_ARG, "normalized time needs mu");
    if (d->n_dirs < 0 || (d->n_dirs > 0 && !d->dQ)) return fail(ctx, H3G_ERR_ARG, "dQ directions missing");
    const int n_model_dirs = d->dQ_model ? d->n_models : 0;     // one extra direction per model
    const int n_dirs_all = d->n_dirs + n_model_dirs;
    if (d->precision != H3G_PREC_FP64 && d->precision != H3G_PREC_MIXED) return fail(ctx, H3G_ERR_ARG, "unknown precision");
    if (d->precision == H3G_PREC_MIXED && !mixed_available()) return fail(ctx, H3G_ERR_CUDA, "mixed-precision path not built");
    const int S = d->S, nm = d->n_models;
    if (pr->max_state >= S) return fail(ctx, H3G_ERR_ARG, "a pattern state index is >= S");
    auto finite = [](const double* a, size_t k) { for (size_t i = 0; i < k; ++i) if (!std::isfinite(a[i])) return false; return true; };
    if (d->bg_w && !finite(d->bg_w, size_t(d->has_bg))) return fail(ctx, H3G_ERR_NUMERIC, "non-finite background weights");
    if (!finite(d->pi, S) || !finite(d->Q, size_t(nm) * S * S) ||
        (!dev_eig && (!finite(d->lam, size_t(nm) * S) || !finite(d->U, size_t(nm) * S * S) || !finite(d->V, size_t(nm) * S * S))) ||
        !finite(d->class_w, d->K) || !finite(d->rates, d->M) || !finite(d->rate_w, d->M))
        return fail(ctx, H3G_ERR_NUMERIC, "non-finite model parameters");
    try {
        cudaSetDevice(ctx->device);
        // identical model already installed: nothing to upload
        uint64_t h = 1469598103934665603ull;
        const int scal[10] = {S, nm, d->K, d->has_bg, d->M, d->time_mode, d->n_dirs, d->precision, d->zero_l_sentinel,
                              n_model_dirs};
        h = hash_bytes(h, scal, sizeof(scal));
        h = hash_bytes(h, d->pi, S * sizeof(double));
        h = hash_bytes(h, d->Q, size_t(nm) * S * S * sizeof(double));
        h = hash_bytes(h, &dev_eig, sizeof(dev_eig));
        if (!dev_eig) {
            h = hash_bytes(h, d->lam, size_t(nm) * S * sizeof(double));
            h = hash_bytes(h, d->U, size_t(nm) * S * S * sizeof(double));
            h = hash_bytes(h, d->V, size_t(nm) * S * S * sizeof(double));
        }
        if (d->mu) h = hash_bytes(h, d->mu, nm * sizeof(double));
        h = hash_bytes(h, d->class_w, d->K * sizeof(double));
        if (d->bg_w) h = hash_bytes(h, d->bg_w, size_t(d->has_bg) * sizeof(double));
        h = hash_bytes(h, d->rates, d->M * sizeof(double));
        h = hash_bytes(h, d->rate_w, d->M * sizeof(double));
        if (d->is_test) h = hash_bytes(h, d->is_test, size_t(pr->n));
        if (d->branch_classes) h = hash_bytes(h, d->branch_classes, size_t(pr->n + 1) * sizeof(int32_t));
        if (d->dQ_model) h = hash_bytes(h, d->dQ_model, size_t(nm) * S * S * sizeof(double));
        if (d->n_dirs > 0) h = hash_bytes(h, d->dQ, size_t(d->n_dirs) * nm * S * S * sizeof(double));
        if (pr->has_model && h == pr->model_hash) return H3G_OK;
        cudaStreamSynchronize(ctx->stream);
        pr->has_model = false;
        pr->S = S; pr->M = d->M; pr->K = d->K; pr->nmod = nm; pr->ndirs = n_dirs_all; pr->has_bg = d->has_bg;
        pr->time_mode = d->time_mode; pr->sentinel = d->zero_l_sentinel;
        if (pr->precision != d->precision) { pr->drop_graphs(); pr->work_mem.release(); pr->w = Work{}; }
        pr->precision = d->precision;
        std::vector<double> pi(SP, 0.0), Q(size_t(nm) * SP2), U(size_t(nm) * SP2), V(size_t(nm) * SP2), lam(size_t(nm) * SP, 0.0);
        std::vector<double> UT(size_t(nm) * SP2), QT(size_t(nm) * SP2);
        std::copy(d->pi, d->pi + S, pi.begin());
        for (int k = 0; k < nm; ++k) {
            pad_matrix(d->Q + size_t(k) * S * S, S, &Q[size_t(k) * SP2]);
            if (!dev_eig) {
                pad_matrix(d->U + size_t(k) * S * S, S, &U[size_t(k) * SP2]);
                pad_matrix(d->V + size_t(k) * S * S, S, &V[size_t(k) * SP2]);
                std::copy(d->lam + size_t(k) * S, d->lam + size_t(k) * S + S, &lam[size_t(k) * SP]);
            }
            for (int i = 0; i < SP; ++i)
                for (int j = 0; j < SP; ++j) {
                    UT[size_t(k) * SP2 + size_t(j) * SP + i] = U[size_t(k) * SP2 + size_t(i) * SP + j];
                    QT[size_t(k) * SP2 + size_t(j) * SP + i] = Q[size_t(k) * SP2 + size_t(i) * SP + j];
                }
        }
        std::vector<double> mu(nm, 1.0);
        if (d->mu) {
            std::copy(d->mu, d->mu + nm, mu.begin());
        } else if (dev_eig) {
            // the reference's scale_factor, stored but not applied (rate_matrix.hpp:228-233)
            for (int k = 0; k < nm; ++k) {
                double m = 0.0;
                for (int i = 0; i < S; ++i) m -= d->pi[i] * d->Q[size_t(k) * S * S + size_t(i) * S + i];
                mu[k] = m;
            }
        }
        pr->h_mu = mu;
        // dense directions [n_dirs][nm], then the per-model ones [nm]
        std::vector<double> dQ((size_t(std::max(d->n_dirs, 1)) * nm + size_t(n_model_dirs)) * SP2, 0.0);
        for (int x = 0; x < d->n_dirs; ++x)
            for (int k = 0; k < nm; ++k) pad_matrix(d->dQ + (size_t(x) * nm + k) * S * S, S, &dQ[(size_t(x) * nm + k) * SP2]);
        for (int k = 0; k < n_model_dirs; ++k)
            pad_matrix(d->dQ_model + size_t(k) * S * S, S, &dQ[(size_t(d->n_dirs) * nm + k) * SP2]);
        std::vector<uint8_t> it(pr->n, 1);
        if (d->is_test) std::copy(d->is_test, d->is_test + pr->n, it.begin());
        // grow-only, like the workspace
        size_t mkey[5] = {size_t(nm), size_t(d->K), size_t(d->M), size_t(std::max(d->n_dirs, 1) + (n_model_dirs ? 1 : 0)),
                          size_t(pr->n)};
        bool fits = pr->m_pi != nullptr;
        for (int i = 0; i < 5 && fits; ++i) fits = mkey[i] <= pr->model_key[i];
        if (!fits && pr->m_pi)
            for (int i = 0; i < 5; ++i) mkey[i] = std::max(mkey[i], pr->model_key[i]);
        if (!fits) {
            pr->drop_graphs();
            auto& A = pr->model_mem;
            A.release();
            const size_t cnm = mkey[0], cK = mkey[1], cM = mkey[2], cdirs = mkey[3];
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_pi, SP));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_Q, cnm * SP2));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_lam, cnm * SP));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_U, cnm * SP2));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_UT, cnm * SP2));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_QT, cnm * SP2));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_V, cnm * SP2));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_mu, cnm));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_cw, cK));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_bw, cnm));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_rt, cM));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_rw, cM));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_dQ, cdirs * cnm * SP2));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_it, it.size()));
            H3G_TRY_CUDA(ctx, A.alloc(&pr->m_br, size_t(pr->n) + 1));
            std::copy(mkey, mkey + 5, pr->model_key);
        }
        cudaStream_t s = ctx->stream;
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_pi, pi.data(), SP * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_Q, Q.data(), Q.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_QT, QT.data(), QT.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        if (dev_eig) {
            launch_model_eig(pr->m_Q, pr->m_pi, S, nm, pr->m_lam, pr->m_U, pr->m_UT, pr->m_V, s);
            H3G_TRY_CUDA(ctx, cudaGetLastError());
        } else {
            H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_lam, lam.data(), lam.size() * sizeof(double), cudaMemcpyHostToDevice, s));
            H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_U, U.data(), U.size() * sizeof(double), cudaMemcpyHostToDevice, s));
            H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_UT, UT.data(), UT.size() * sizeof(double), cudaMemcpyHostToDevice, s));
            H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_V, V.data(), V.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        }
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_mu, mu.data(), mu.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_cw, d->class_w, d->K * sizeof(double), cudaMemcpyHostToDevice, s));
        if (d->has_bg > 0) {
            pr->h_bw.assign(size_t(d->has_bg), 1.0);
            if (d->bg_w) std::copy(d->bg_w, d->bg_w + d->has_bg, pr->h_bw.begin());
            H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_bw, pr->h_bw.data(), pr->h_bw.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        }
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_rt, d->rates, d->M * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_rw, d->rate_w, d->M * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_dQ, dQ.data(), dQ.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_it, it.data(), it.size(), cudaMemcpyHostToDevice, s));
        if (d->branch_classes)
            H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->m_br, d->branch_classes, size_t(pr->n + 1) * sizeof(int32_t),
                                              cudaMemcpyHostToDevice, s));
        Model md{};
        md.M = d->M; md.K = d->K; md.has_bg = d->has_bg; md.nmod = nm; md.time_mode = d->time_mode; md.ndirs = n_dirs_all;
        md.ndirs_dense = d->n_dirs;
        md.sentinel = d->zero_l_sentinel;
        md.pi = pr->m_pi; md.Q = pr->m_Q; md.lam = pr->m_lam; md.U = pr->m_U; md.V = pr->m_V; md.mu = pr->m_mu;
        md.UT = pr->m_UT; md.QT = pr->m_QT;
        md.class_w = pr->m_cw; md.bg_w = pr->m_bw; md.rates = pr->m_rt; md.rate_w = pr->m_rw; md.is_test = d->is_test ? pr->m_it : nullptr;
        md.br_off = d->branch_classes ? pr->m_br : nullptr;
        md.dQ = pr->m_dQ;
        if (std::memcmp(&md, &pr->md, sizeof(Model)) != 0) pr->drop_graphs();
        pr->md = md;
        h3g_status st = ensure_workspace(pr, d->M, d->K, nm, n_dirs_all);
        if (st != H3G_OK) return st;
        H3G_TRY_CUDA(ctx, cudaStreamSynchronize(s));
        pr->model_hash = h;
        pr->has_model = true;
        return H3G_OK;
    } catch (const std::bad_alloc&) {
        return fail(ctx, H3G_ERR_OOM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(ctx, H3G_ERR_ARG, e.what());
    }
}

// Stage boundaries for h3g_profile_stages (same order as H3G_STAGE_NAMES in h3g.h).
enum Stage { ST_BUILD_P, ST_PREP_MIXED, ST_INSIDE, ST_ROOT, ST_OUTSIDE, ST_ACCUM_A, ST_FRECHET, ST_HSUM, ST_SMALL, ST_DIR, ST_COUNT };
struct StageMarks {
    cudaEvent_t ev[ST_COUNT + 1];
    bool seen[ST_COUNT];
    int launches[ST_COUNT];
};

// Enqueue the pruning pipeline (inside, root and optionally outside + gradients) on stream s (the
// context stream, or a batch slot's), in workspace w / mw.
static int enqueue_eval_ck(h3g_problem* pr, unsigned want, bool from_given_P, cudaStream_t s, const Work& w,
                           const MixedWork& mwk, StageMarks* mk);

static int enqueue_eval_on(h3g_problem* pr, unsigned want, bool from_given_P, cudaStream_t s, const Work& w,
                           const MixedWork& mwk, StageMarks* mk = nullptr) {
    if (pr->ck && !pr->batch) return enqueue_eval_ck(pr, want, from_given_P, s, w, mwk, mk);
    const Topo t = pr->topo();
    const Model& md = pr->md;
    const bool mixed = pr->precision == H3G_PREC_MIXED;
    const bool grads = (want & (H3G_WANT_GRAD_T | H3G_WANT_GRAD_GLOBAL)) != 0;
    const bool global = (want & H3G_WANT_GRAD_GLOBAL) != 0;
    int L = 0;
    auto mark = [&](Stage st, int launched) {
        L += launched;
        if (mk && launched) { cudaEventRecord(mk->ev[st + 1], s); mk->seen[st] = true; mk->launches[st] += launched; }
    };
    if (mk) cudaEventRecord(mk->ev[0], s);
    // model-only directional products on the side stream, joined before their contraction
    const bool side = global && md.ndirs > 0;
    if (side) {
        cudaEventRecord(pr->ev_fork, s);
        cudaStreamWaitEvent(pr->s2, pr->ev_fork, 0);
        L += launch_dir(t, md, w, pr->s2);
        cudaEventRecord(pr->ev_join, pr->s2);
    }
    mark(ST_BUILD_P, from_given_P ? launch_prep_given_P(t, w, s)
                                  : (mixed ? launch_build_P_mixed(t, md, w, mwk, s) : launch_build_P(t, md, w, s)));
    if (mixed && from_given_P) mark(ST_PREP_MIXED, mixed_prepare(t, md, w, mwk, s));
    int l = 0;
    if (mixed) {
        // one persistent launch over every level, per-tile dependencies
        l = launch_inside_mixed(t, md, w, mwk, pr->n_in_heads, pr->wait, s);
    } else {
        for (size_t lv = 0; lv + 1 < pr->in_off.size(); ++lv) {
            const int cnt = pr->in_off[lv + 1] - pr->in_off[lv];
            if (!cnt) continue;
            l += launch_inside_fp64(t, md, w, pr->d_in_nodes + pr->in_off[lv], cnt, s);
        }
    }
    mark(ST_INSIDE, l);
    mark(ST_ROOT, mixed ? launch_root_mixed(t, md, w, mwk, s) : launch_root(t, md, w, s));
    if (grads) {
        l = 0;
        if (mixed) {
            l = launch_outside_mixed(t, md, w, mwk, pr->n_out_heads, pr->wait, s);
        } else {
            for (size_t lv = 0; lv + 1 < pr->out_off.size(); ++lv) {
                const int cnt = pr->out_off[lv + 1] - pr->out_off[lv];
                if (!cnt) continue;
                l += launch_outside_fp64(t, md, w, pr->d_out_nodes + pr->out_off[lv], cnt, 1, s);
            }
        }
        mark(ST_OUTSIDE, l);
        mark(ST_ACCUM_A, mixed ? launch_accumA_mixed(t, md, w, mwk, nullptr, 0, s) : launch_accumA_fp64(t, md, w, nullptr, 0, s));
        mark(ST_FRECHET, launch_frechet(t, md, w, global ? 1 : 0, s));
        if (side) cudaStreamWaitEvent(s, pr->ev_join, 0);
        if (global) mark(ST_HSUM, launch_global(t, md, w, s));
    }
    if (side && !grads) cudaStreamWaitEvent(s, pr->ev_join, 0);
    mark(ST_SMALL, launch_small(t, md, w, grads ? 1 : 0, s));
    return L;
}

// The same pipeline over a checkpoint plan (h3g_checkpoint.h): inside block by block in post-order,
// then per block in reverse post-order the recompute of its inside partials below its root, its
// outside walk and its gradient-operand accumulation.  Stage marks: the recompute and the
// accumulation of the blocks count under "outside".
static int enqueue_eval_ck(h3g_problem* pr, unsigned want, bool from_given_P, cudaStream_t s, const Work& w,
                           const MixedWork& mwk, StageMarks* mk) {
    const Topo t = pr->topo_eval();
    const Model& md = pr->md;
    const h3g::CkPlan& pl = pr->ck_plan;
    const bool mixed = pr->precision == H3G_PREC_MIXED;
    const bool grads = (want & (H3G_WANT_GRAD_T | H3G_WANT_GRAD_GLOBAL)) != 0;
    const bool global = (want & H3G_WANT_GRAD_GLOBAL) != 0;
    const int* lists = pr->d_ck_lists;
    const int4* info = pr->d_ck_info;
    int L = 0;
    auto mark = [&](Stage st, int launched) {
        L += launched;
        if (mk && launched) { cudaEventRecord(mk->ev[st + 1], s); mk->seen[st] = true; mk->launches[st] += launched; }
    };
    if (mk) cudaEventRecord(mk->ev[0], s);
    const bool side = global && md.ndirs > 0;
    if (side) {
        cudaEventRecord(pr->ev_fork, s);
        cudaStreamWaitEvent(pr->s2, pr->ev_fork, 0);
        L += launch_dir(t, md, w, pr->s2);
        cudaEventRecord(pr->ev_join, pr->s2);
    }
    mark(ST_BUILD_P, from_given_P ? launch_prep_given_P(t, w, s)
                                  : (mixed ? launch_build_P_mixed(t, md, w, mwk, s) : launch_build_P(t, md, w, s)));
    if (mixed && from_given_P) mark(ST_PREP_MIXED, mixed_prepare(t, md, w, mwk, s));
    // inside partials of block bi: every level, or every level below the block root
    auto inside = [&](size_t bi, bool with_root) {
        const h3g::CkBlock& B = pl.blocks[bi];
        const h3g_problem::CkOffsets& o = pr->ck_off[bi];
        const int levels = int(B.in_lv.size()) - 1 - (with_root ? 0 : 1);
        int l = 0;
        if (levels <= 0) return 0;
        if (mixed) {
            Topo tb = t;
            tb.in_info = info + o.in_info;
            tb.in_next = lists + o.in_next;
            tb.in_heads = lists + o.in_heads;
            l += mixed_new_epoch(mwk, s);
            l += launch_inside_mixed(tb, md, w, mwk, o.n_in_heads - (with_root ? 0 : 1), pr->wait, s);
        } else {
            for (int lv = 0; lv < levels; ++lv)
                l += launch_inside_fp64(t, md, w, lists + o.in + B.in_lv[lv], B.in_lv[lv + 1] - B.in_lv[lv], s);
        }
        return l;
    };
    int l = 0;
    for (size_t bi = 0; bi < pl.blocks.size(); ++bi) l += inside(bi, true);
    mark(ST_INSIDE, l);
    mark(ST_ROOT, mixed ? launch_root_mixed(t, md, w, mwk, s) : launch_root(t, md, w, s));
    if (grads) {
        l = 0;
        for (size_t r = pl.blocks.size(); r-- > 0;) {
            const h3g::CkBlock& B = pl.blocks[r];
            const h3g_problem::CkOffsets& o = pr->ck_off[r];
            if (r + 1 != pl.blocks.size()) l += inside(r, false);      // the root's block is still in scratch
            if (mixed) {
                Topo tb = t;
                tb.out_info = info + o.out_info;
                tb.out_next = lists + o.out_next;
                tb.out_heads = lists + o.out_heads;
                l += mixed_new_epoch(mwk, s);
                l += launch_outside_mixed(tb, md, w, mwk, o.n_out_heads, pr->wait, s);
                if (!B.acc.empty()) l += launch_accumA_mixed(t, md, w, mwk, lists + o.acc, int(B.acc.size()), s);
            } else {
                for (size_t lv = 0; lv + 1 < B.out_lv.size(); ++lv)
                    l += launch_outside_fp64(t, md, w, lists + o.out + B.out_lv[lv], B.out_lv[lv + 1] - B.out_lv[lv], 1, s);
                if (!B.acc.empty()) l += launch_accumA_fp64(t, md, w, lists + o.acc, int(B.acc.size()), s);
            }
        }
        mark(ST_OUTSIDE, l);
        mark(ST_FRECHET, launch_frechet(t, md, w, global ? 1 : 0, s));
        if (side) cudaStreamWaitEvent(s, pr->ev_join, 0);
        if (global) mark(ST_HSUM, launch_global(t, md, w, s));
    }
    if (side && !grads) cudaStreamWaitEvent(s, pr->ev_join, 0);
    mark(ST_SMALL, launch_small(t, md, w, grads ? 1 : 0, s));
    return L;
}

static int enqueue_eval(h3g_problem* pr, unsigned want, bool from_given_P, StageMarks* mk = nullptr) {
    return enqueue_eval_on(pr, want, from_given_P, pr->ctx->stream, pr->w, pr->mw, mk);
}

static unsigned norm_want(unsigned want) {
    unsigned w = want & (H3G_WANT_SITE_LNL | H3G_WANT_GRAD_T | H3G_WANT_GRAD_GLOBAL);
    return w | H3G_WANT_LNL;
}

// Results the host reads back after an evaluation: the small output vector,
// the directional partials and (optionally) the per-pattern lnL.
static size_t enqueue_readback_on(h3g_problem* pr, unsigned want, cudaStream_t s, const Work& w) {
    size_t bytes = n_out_of(pr) * sizeof(double);
    cudaMemcpyAsync(pr->h_pin + pr->off_out, w.out, bytes, cudaMemcpyDeviceToHost, s);
    if ((want & H3G_WANT_GRAD_GLOBAL) && pr->ndirs > 0) {
        const size_t b = size_t(pr->ndirs) * pr->nmod * 17 * sizeof(double);
        cudaMemcpyAsync(pr->h_pin + pr->off_dir, w.dirpart, b, cudaMemcpyDeviceToHost, s);
        bytes += b;
    }
    if ((want & H3G_WANT_SITE_LNL) && pr->P > 0) {
        const size_t b = size_t(pr->P) * sizeof(double);
        cudaMemcpyAsync(pr->h_pin + pr->off_site, w.site, b, cudaMemcpyDeviceToHost, s);
        bytes += b;
    }
    return bytes;
}
static size_t enqueue_readback(h3g_problem* pr, unsigned want) {
    return enqueue_readback_on(pr, want, pr->ctx->stream, pr->w);
}

static bool graphs_enabled() {
    static const bool on = [] { const char* e = std::getenv("H3G_NO_GRAPH"); return !(e && e[0] == '1'); }();
    return on;
}

// Run one evaluation: as a captured CUDA graph (host copies included when
// `copies`), instantiated once per (want, copies) and replayed afterwards.
static h3g_status run_eval(h3g_problem* pr, unsigned want, bool copies) {
    h3g_ctx* ctx = pr->ctx;
    cudaStream_t s = ctx->stream;
    const unsigned key = norm_want(want) | (copies ? 0x100u : 0u);
    cudaGraphExec_t exec = nullptr;
    for (auto& g : pr->graphs) if (g.key == key) { exec = g.exec; pr->last_launches = g.launches; }
    if (!exec && graphs_enabled()) {
        cudaGraph_t graph = nullptr;
        H3G_TRY_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        if (copies) cudaMemcpyAsync(pr->d_bl, pr->h_pin, pr->n * sizeof(double), cudaMemcpyHostToDevice, s);
        pr->last_launches = enqueue_eval(pr, key, false);
        if (copies) enqueue_readback(pr, key);
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (e != cudaSuccess) { ctx->err = std::string("graph capture: ") + cudaGetErrorString(e); return H3G_ERR_CUDA; }
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) { ctx->err = std::string("graph instantiate: ") + cudaGetErrorString(e); return H3G_ERR_CUDA; }
        pr->graphs.push_back({key, exec, pr->last_launches});
    }
    H3G_TRY_CUDA(ctx, cudaEventRecord(pr->ev0, s));
    if (exec) {
        H3G_TRY_CUDA(ctx, cudaGraphLaunch(exec, s));
    } else {
        if (copies) H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_bl, pr->h_pin, pr->n * sizeof(double), cudaMemcpyHostToDevice, s));
        pr->last_launches = enqueue_eval(pr, key, false);
        H3G_TRY_CUDA(ctx, cudaGetLastError());
        if (copies) enqueue_readback(pr, key);
    }
    H3G_TRY_CUDA(ctx, cudaEventRecord(pr->ev1, s));
    pr->last_h2d = copies ? pr->n * sizeof(double) : 0;
    pr->last_d2h = 0;
    if (copies) {
        pr->last_d2h = n_out_of(pr) * sizeof(double);
        if ((key & H3G_WANT_GRAD_GLOBAL) && pr->ndirs > 0) pr->last_d2h += size_t(pr->ndirs) * pr->nmod * 17 * sizeof(double);
        if ((key & H3G_WANT_SITE_LNL) && pr->P > 0) pr->last_d2h += size_t(pr->P) * sizeof(double);
    }
    return H3G_OK;
}

static void unpack_result(h3g_problem* pr, unsigned want, h3g_result* out) {
    const int n = pr->n;
    const double* hout = pr->h_pin + pr->off_out;
    const bool grads = (want & (H3G_WANT_GRAD_T | H3G_WANT_GRAD_GLOBAL)) != 0;
    const bool global = (want & H3G_WANT_GRAD_GLOBAL) != 0;
    out->lnl = hout[0];
    if (out->grad_t) {
        for (int b = 0; b < n; ++b) out->grad_t[b] = grads ? hout[2 + b] : 0.0;
        out->grad_t[pr->root] = 0.0;
    }
    if (out->grad_class_w) for (int k = 0; k < pr->K; ++k) out->grad_class_w[k] = global ? hout[2 + n + k] : 0.0;
    if (out->grad_bg_w)
        for (int j = 0; j < pr->nmod - pr->K; ++j) out->grad_bg_w[j] = global ? hout[2 + n + pr->K + j] : 0.0;
    if (out->grad_rate_w) for (int m = 0; m < pr->M; ++m) out->grad_rate_w[m] = grads ? hout[2 + n + 2 * pr->nmod + m] : 0.0;
    if (out->grad_dir) {
        // sum_k sum (V dQ U) o H_k, minus (normalised time) sum_k dmu_k / mu_k * sum_b tau_b dL/dtau_b
        const double* dir = pr->h_pin + pr->off_dir;
        for (int x = 0; x < pr->ndirs; ++x) {
            double g = 0.0;
            if (global)
                for (int k = 0; k < pr->nmod; ++k) {
                    const double* d = dir + (size_t(x) * pr->nmod + k) * 17;
                    double v = 0.0;
                    for (int b = 0; b < 16; ++b) v += d[b];
                    if (pr->time_mode == H3G_TIME_NORMALIZED)
                        v -= d[16] / std::max(pr->h_mu[size_t(k)], 1e-12) * hout[2 + n + pr->nmod + k];
                    g += v;
                }
            out->grad_dir[x] = g;
        }
    }
    if ((want & H3G_WANT_SITE_LNL) && out->site_lnl && pr->P > 0)
        std::copy(pr->h_pin + pr->off_site, pr->h_pin + pr->off_site + pr->P, out->site_lnl);
}

static h3g_status check_bl(h3g_problem* pr, const double* bl) {
    for (int i = 0; i < pr->n; ++i)
        if (i != pr->root && !std::isfinite(bl[i])) return fail(pr->ctx, H3G_ERR_NUMERIC, "non-finite branch length");
    return H3G_OK;
}

// A bounded device wait expired during the evaluation just read back: clear the device's sticky
// error word (so the next evaluation on this problem starts clean) and report H3G_ERR_TIMEOUT.
static h3g_status timed_out(h3g_problem* pr) {
    h3g_ctx* ctx = pr->ctx;
    if (pr->w.err) {
        cudaMemsetAsync(pr->w.err, 0, sizeof(int), ctx->stream);
        cudaStreamSynchronize(ctx->stream);
    }
    return fail(ctx, H3G_ERR_TIMEOUT, "a bounded device wait expired (results of this evaluation are invalid)");
}

extern "C" h3g_status h3g_eval(h3g_problem* pr, const double* bl, unsigned want, h3g_result* out) {
    if (!pr || !bl || !out) return H3G_ERR_ARG;
    h3g_ctx* ctx = pr->ctx;
    if (pr->batch) return fail(ctx, H3G_ERR_STATE, "the problem belongs to a batch: use h3g_batch_eval");
    if (!pr->has_model) return fail(ctx, H3G_ERR_STATE, "h3g_eval before h3g_model_set");
    if (h3g_status st = check_bl(pr, bl); st != H3G_OK) return st;
    cudaSetDevice(ctx->device);
    std::copy(bl, bl + pr->n, pr->h_pin);
    pr->h_pin[pr->root] = 0.0;
    if (h3g_status st = run_eval(pr, want, true); st != H3G_OK) return st;
    H3G_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    cudaEventElapsedTime(&pr->last_ms, pr->ev0, pr->ev1);
    unpack_result(pr, norm_want(want), out);
    if (pr->h_pin[pr->off_out + 1] != 0.0) return timed_out(pr);
    if (!std::isfinite(out->lnl)) return fail(ctx, H3G_ERR_NUMERIC, "non-finite log-likelihood");
    return H3G_OK;
}

extern "C" h3g_status h3g_model_get_eigensystem(h3g_problem* pr, int k, double* lam, double* U, double* V) {
    if (!pr || !lam || !U || !V) return H3G_ERR_ARG;
    if (!pr->has_model) return fail(pr->ctx, H3G_ERR_STATE, "no model installed");
    if (k < 0 || k >= pr->nmod) return fail(pr->ctx, H3G_ERR_ARG, "model index out of range");
    cudaSetDevice(pr->ctx->device);
    std::vector<double> l(SP), u(SP2), v(SP2);
    cudaStream_t s = pr->ctx->stream;
    H3G_TRY_CUDA(pr->ctx, cudaMemcpyAsync(l.data(), pr->m_lam + size_t(k) * SP, SP * sizeof(double), cudaMemcpyDeviceToHost, s));
    H3G_TRY_CUDA(pr->ctx, cudaMemcpyAsync(u.data(), pr->m_U + size_t(k) * SP2, SP2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    H3G_TRY_CUDA(pr->ctx, cudaMemcpyAsync(v.data(), pr->m_V + size_t(k) * SP2, SP2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    H3G_TRY_CUDA(pr->ctx, cudaStreamSynchronize(s));
    const int S = pr->S;
    for (int i = 0; i < S; ++i) {
        lam[i] = l[i];
        for (int j = 0; j < S; ++j) {
            U[size_t(i) * S + j] = u[size_t(i) * SP + j];
            V[size_t(i) * S + j] = v[size_t(i) * SP + j];
        }
    }
    return H3G_OK;
}

extern "C" h3g_status h3g_problem_set_tuning(h3g_problem* pr, const h3g_tuning* tu) {
    if (!pr || !tu) return H3G_ERR_ARG;
    if (tu->a_chunk < 0 || (tu->a_chunk > 0 && (tu->a_chunk % TP != 0 || tu->a_chunk < 2 * TP)))
        return fail(pr->ctx, H3G_ERR_ARG, "a_chunk must be 0 or a multiple of 128 that is at least 256");
    if (tu->ctas_per_sm < 0 || tu->ctas_per_sm > 2) return fail(pr->ctx, H3G_ERR_ARG, "ctas_per_sm must be 0, 1 or 2");
    if (tu->frechet_groups < 0) return fail(pr->ctx, H3G_ERR_ARG, "frechet_groups must be >= 0");
    pr->tuning = *tu;
    pr->drop_graphs();               // launch shapes are captured in the graphs
    if (pr->has_model) return ensure_workspace(pr, pr->M, pr->K, pr->nmod, pr->ndirs);
    return H3G_OK;
}

extern "C" h3g_status h3g_problem_get_tuning(const h3g_problem* pr, h3g_tuning* tu) {
    if (!pr || !tu) return H3G_ERR_ARG;
    const WsLayout L = ws_layout(size_t(pr->n), size_t(pr->NI), size_t(pr->Pp), std::max(pr->M, 1), pr->K,
                                 std::max(pr->nmod, 1), pr->ndirs, effective_tuning(pr, pr->M, pr->K, pr->nmod, pr->ndirs));
    tu->a_chunk = L.chunk;
    tu->ctas_per_sm = pr->wait.ctas_per_sm;
    tu->frechet_groups = L.ngroups;
    return H3G_OK;
}

extern "C" h3g_status h3g_autotune(h3g_problem* pr, const double* bl, unsigned want, int reps, h3g_tuning* best,
                                   double* best_ms) {
    if (!pr || !bl || reps < 1) return H3G_ERR_ARG;
    h3g_ctx* ctx = pr->ctx;
    if (pr->batch) return fail(ctx, H3G_ERR_STATE, "the problem belongs to a batch");
    if (!pr->has_model) return fail(ctx, H3G_ERR_STATE, "h3g_autotune before h3g_model_set");
    if (h3g_status st = check_bl(pr, bl); st != H3G_OK) return st;
    cudaSetDevice(ctx->device);
    const unsigned key = norm_want(want);
    auto measure = [&](const h3g_tuning& tu, double* ms) -> h3g_status {
        if (h3g_status st = h3g_problem_set_tuning(pr, &tu); st != H3G_OK) return st;
        std::copy(bl, bl + pr->n, pr->h_pin);
        pr->h_pin[pr->root] = 0.0;
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_bl, pr->h_pin, pr->n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        if (h3g_status st = run_eval(pr, key, false); st != H3G_OK) return st;      // warm-up (and graph capture)
        H3G_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        double tot = 0.0;
        for (int r = 0; r < reps; ++r) {
            if (h3g_status st = run_eval(pr, key, false); st != H3G_OK) return st;
            H3G_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            float m = 0.f;
            cudaEventElapsedTime(&m, pr->ev0, pr->ev1);
            tot += m;
        }
        *ms = tot / reps;
        return H3G_OK;
    };
    const WsLayout L0 = ws_layout(size_t(pr->n), size_t(pr->NI), size_t(pr->Pp), pr->M, pr->K, pr->nmod, pr->ndirs, h3g_tuning{});
    h3g_tuning cur{L0.chunk, 2, L0.ngroups};
    double cur_ms = 0.0;
    if (h3g_status st = measure(cur, &cur_ms); st != H3G_OK) return st;
    auto uniq = [](std::vector<int> v) { std::sort(v.begin(), v.end()); v.erase(std::unique(v.begin(), v.end()), v.end()); return v; };
    const int Pp = pr->Pp;
    auto chunk_of = [&](int c) { return std::max(2 * TP, std::min(Pp, c / TP * TP)); };
    std::vector<int> chunks = uniq({chunk_of(L0.chunk), chunk_of(Pp), chunk_of(Pp / 2), chunk_of(Pp / 4), chunk_of(Pp / 8),
                                    chunk_of(1024), chunk_of(512), chunk_of(256)});
    std::vector<int> groups = uniq({L0.ngroups, std::max(1, L0.ngroups / 2), std::min(pr->n, 2 * L0.ngroups),
                                    std::min(pr->n, 4 * L0.ngroups)});
    std::vector<int> ctas = pr->precision == H3G_PREC_MIXED ? std::vector<int>{2, 1} : std::vector<int>{2};
    for (int field = 0; field < 3; ++field) {
        const std::vector<int>& cand = field == 0 ? chunks : (field == 1 ? ctas : groups);
        for (int v : cand) {
            h3g_tuning tu = cur;
            (field == 0 ? tu.a_chunk : (field == 1 ? tu.ctas_per_sm : tu.frechet_groups)) = v;
            if (tu.a_chunk == cur.a_chunk && tu.ctas_per_sm == cur.ctas_per_sm && tu.frechet_groups == cur.frechet_groups)
                continue;
            double ms = 0.0;
            if (h3g_status st = measure(tu, &ms); st != H3G_OK) return st;
            if (ms < cur_ms) { cur = tu; cur_ms = ms; }
        }
    }
    if (h3g_status st = h3g_problem_set_tuning(pr, &cur); st != H3G_OK) return st;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tunings[tune_key(pr, pr->M, pr->K, pr->nmod, pr->ndirs)] = cur;
    }
    if (best) *best = cur;
    if (best_ms) *best_ms = cur_ms;
    return H3G_OK;
}

extern "C" h3g_status h3g_pack_result_device(h3g_problem* pr, unsigned want, double* d_vec) {
    if (!pr || !d_vec) return H3G_ERR_ARG;
    if (!pr->has_model) return fail(pr->ctx, H3G_ERR_STATE, "h3g_pack_result_device before h3g_model_set");
    if (pr->batch || !pr->w.out) return fail(pr->ctx, H3G_ERR_STATE, "no evaluation workspace on this problem");
    cudaSetDevice(pr->ctx->device);
    const unsigned key = norm_want(want);
    const int grads = (key & (H3G_WANT_GRAD_T | H3G_WANT_GRAD_GLOBAL)) != 0, global = (key & H3G_WANT_GRAD_GLOBAL) != 0;
    launch_pack_result(pr->topo(), pr->md, pr->w, grads, global, d_vec, pr->ctx->stream);
    H3G_TRY_CUDA(pr->ctx, cudaGetLastError());
    return H3G_OK;
}

extern "C" h3g_status h3g_ctx_stream(const h3g_ctx* ctx, void** stream) {
    if (!ctx || !stream) return H3G_ERR_ARG;
    *stream = ctx->stream;
    return H3G_OK;
}

extern "C" h3g_status h3g_problem_set_wait_limit(h3g_problem* pr, uint32_t polls, int unmatched) {
    if (!pr) return H3G_ERR_ARG;
    pr->wait.polls = polls ? polls : WaitCfg{}.polls;
    pr->wait.skew = unmatched ? 1 : 0;
    pr->drop_graphs();               // the limit is a launch parameter of the captured passes
    return H3G_OK;
}

extern "C" h3g_status h3g_problem_set_memory_budget(h3g_problem* pr, uint64_t bytes, int target) {
    if (!pr) return H3G_ERR_ARG;
    if (target < 0) return fail(pr->ctx, H3G_ERR_ARG, "target must be >= 0");
    if (pr->batch) return fail(pr->ctx, H3G_ERR_STATE, "the problem belongs to a batch (its workspace lives there)");
    cudaSetDevice(pr->ctx->device);
    cudaStreamSynchronize(pr->ctx->stream);
    pr->mem_budget = bytes;
    pr->ck_target_req = target;
    pr->drop_graphs();
    pr->work_mem.release();
    pr->w = Work{};
    pr->mw = MixedWork{};
    pr->ws_bytes = 0;
    pr->ck = false;
    if (pr->has_model) return ensure_workspace(pr, pr->M, pr->K, pr->nmod, pr->ndirs);
    return H3G_OK;
}

extern "C" h3g_status h3g_problem_checkpoint_info(const h3g_problem* pr, h3g_checkpoint_info* info) {
    if (!pr || !info) return H3G_ERR_ARG;
    *info = h3g_checkpoint_info{};
    info->active = pr->ck ? 1 : 0;
    info->workspace_bytes = pr->ws_bytes;
    info->full_bytes = pr->full_bytes;
    if (pr->ck) {
        const h3g::CkPlan& pl = pr->ck_plan;
        info->n_blocks = int32_t(pl.blocks.size());
        info->target = pl.target;
        info->n_persistent = pl.ncp;
        info->scratch_internal = pl.scratch_int;
        info->scratch_nodes = pl.scratch_all;
    }
    return H3G_OK;
}

extern "C" h3g_status h3g_checkpoint_plan(int n, const int32_t* parent, const uint8_t* is_leaf, int target,
                                          int32_t* is_checkpoint, int32_t* block, int32_t* slot_internal,
                                          int32_t* slot_vf, int32_t* counts) {
    if (n < 2 || !parent || !is_leaf || target < 1) return H3G_ERR_ARG;
    try {
        std::vector<std::vector<int>> kids(n);
        int root = -1;
        for (int i = 0; i < n; ++i) {
            const int p = parent[i];
            if (p < 0) {
                if (root >= 0) return H3G_ERR_ARG;
                root = i;
            } else {
                if (p >= n || p == i || is_leaf[p]) return H3G_ERR_ARG;
                kids[p].push_back(i);
            }
        }
        if (root < 0 || is_leaf[root]) return H3G_ERR_ARG;
        std::vector<int> order(1, root), depth(n, -1), height(n, 0);
        depth[root] = 0;
        for (size_t q = 0; q < order.size(); ++q)
            for (int c : kids[order[q]]) {
                if (depth[c] >= 0) return H3G_ERR_ARG;
                depth[c] = depth[order[q]] + 1;
                order.push_back(c);
            }
        if (int(order.size()) != n) return H3G_ERR_ARG;
        for (int q = n - 1; q >= 0; --q) {
            const int u = order[q];
            for (int c : kids[u]) height[u] = std::max(height[u], height[c] + 1);
            if (!is_leaf[u] && kids[u].empty()) height[u] = 1;
        }
        const h3g::CkPlan pl = h3g::plan_checkpoints(n, root, kids, is_leaf, order, depth, height, target);
        for (int i = 0; i < n; ++i) {
            if (is_checkpoint) is_checkpoint[i] = pl.is_ckpt[i];
            if (block) block[i] = pl.block_of[i];
            if (slot_internal) slot_internal[i] = pl.iidx[i];
            if (slot_vf) slot_vf[i] = pl.vidx[i];
        }
        if (counts) {
            counts[0] = int32_t(pl.blocks.size());
            counts[1] = pl.ncp;
            counts[2] = pl.scratch_int;
            counts[3] = pl.scratch_all;
        }
        return H3G_OK;
    } catch (const std::bad_alloc&) {
        return H3G_ERR_OOM;
    }
}

extern "C" h3g_status h3g_stage_branch_lengths(h3g_problem* pr, const double* bl) {
    if (!pr || !bl) return H3G_ERR_ARG;
    h3g_ctx* ctx = pr->ctx;
    if (!pr->has_model) return fail(ctx, H3G_ERR_STATE, "stage before h3g_model_set");
    if (h3g_status st = check_bl(pr, bl); st != H3G_OK) return st;
    cudaSetDevice(ctx->device);
    std::copy(bl, bl + pr->n, pr->h_pin);
    pr->h_pin[pr->root] = 0.0;
    H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_bl, pr->h_pin, pr->n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    H3G_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return H3G_OK;
}

extern "C" h3g_status h3g_eval_resident(h3g_problem* pr, unsigned want) {
    if (!pr) return H3G_ERR_ARG;
    if (pr->batch) return fail(pr->ctx, H3G_ERR_STATE, "the problem belongs to a batch: use h3g_batch_eval");
    if (!pr->has_model) return fail(pr->ctx, H3G_ERR_STATE, "h3g_eval_resident before h3g_model_set");
    cudaSetDevice(pr->ctx->device);
    return run_eval(pr, want, false);
}

extern "C" h3g_status h3g_read_result(h3g_problem* pr, unsigned want, h3g_result* out) {
    if (!pr || !out) return H3G_ERR_ARG;
    h3g_ctx* ctx = pr->ctx;
    if (!pr->has_model) return fail(ctx, H3G_ERR_STATE, "h3g_read_result before h3g_model_set");
    cudaSetDevice(ctx->device);
    enqueue_readback(pr, norm_want(want));
    H3G_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    unpack_result(pr, norm_want(want), out);
    if (pr->h_pin[pr->off_out + 1] != 0.0) return timed_out(pr);
    return H3G_OK;
}

extern "C" h3g_status h3g_profile_stages(h3g_problem* pr, unsigned want, int reps, double* stage_ms, int* stage_launches) {
    if (!pr || !stage_ms || reps < 1) return H3G_ERR_ARG;
    if (pr->batch) return fail(pr->ctx, H3G_ERR_STATE, "the problem belongs to a batch");
    h3g_ctx* ctx = pr->ctx;
    if (!pr->has_model) return fail(ctx, H3G_ERR_STATE, "profile before h3g_model_set");
    cudaSetDevice(ctx->device);
    StageMarks mk{};
    for (auto& e : mk.ev) H3G_TRY_CUDA(ctx, cudaEventCreate(&e));
    std::fill(stage_ms, stage_ms + ST_COUNT, 0.0);
    if (stage_launches) std::fill(stage_launches, stage_launches + ST_COUNT, 0);
    h3g_status st = H3G_OK;
    for (int r = 0; r < reps && st == H3G_OK; ++r) {
        std::fill(mk.seen, mk.seen + ST_COUNT, false);
        std::fill(mk.launches, mk.launches + ST_COUNT, 0);
        enqueue_eval(pr, norm_want(want), false, &mk);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { st = fail(ctx, H3G_ERR_CUDA, "profile run failed"); break; }
        cudaEvent_t prev = mk.ev[0];
        for (int k = 0; k < ST_COUNT; ++k) {
            if (!mk.seen[k]) continue;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, prev, mk.ev[k + 1]);
            stage_ms[k] += ms / reps;
            if (stage_launches && r == 0) stage_launches[k] = mk.launches[k];
            prev = mk.ev[k + 1];
        }
    }
    for (auto& e : mk.ev) cudaEventDestroy(e);
    return st;
}

extern "C" h3g_status h3g_eval_from_P(h3g_problem* pr, int S, const double* P, const double* pi, double* lnl, double* site_lnl) {
    if (!pr || !P || !pi || !lnl) return H3G_ERR_ARG;
    h3g_ctx* ctx = pr->ctx;
    if (pr->batch) return fail(ctx, H3G_ERR_STATE, "the problem belongs to a batch");
    if (S < 1 || S > SP) return fail(ctx, H3G_ERR_ARG, "S must be in [1, 64]");
    // a single-class FP64 model whose transition matrices are given directly
    std::vector<double> zeroSS(size_t(S) * S, 0.0), lam(S, 0.0), one{1.0};
    h3g_model_desc d{};
    d.S = S; d.pi = pi; d.n_models = 1; d.Q = zeroSS.data(); d.lam = lam.data(); d.U = zeroSS.data(); d.V = zeroSS.data();
    d.K = 1; d.class_w = one.data(); d.M = 1; d.rates = one.data(); d.rate_w = one.data();
    d.time_mode = H3G_TIME_RAW; d.precision = H3G_PREC_FP64; d.zero_l_sentinel = 1;
    h3g_status st = h3g_model_set(pr, &d);
    if (st != H3G_OK) return st;
    const int n = pr->n;
    std::vector<double> padded(size_t(n) * SP2, 0.0);
    for (int b = 0; b < n; ++b) if (b != pr->root) pad_matrix(P + size_t(b) * S * S, S, &padded[size_t(b) * SP2]);
    cudaStream_t s = ctx->stream;
    H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->w.P, padded.data(), padded.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    H3G_TRY_CUDA(ctx, cudaEventRecord(pr->ev0, s));
    pr->last_launches = enqueue_eval(pr, H3G_WANT_LNL, true);
    H3G_TRY_CUDA(ctx, cudaGetLastError());
    H3G_TRY_CUDA(ctx, cudaEventRecord(pr->ev1, s));
    double* hout = pr->h_pin + pr->off_out;
    H3G_TRY_CUDA(ctx, cudaMemcpyAsync(hout, pr->w.out, sizeof(double), cudaMemcpyDeviceToHost, s));
    if (site_lnl && pr->P > 0)
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(site_lnl, pr->w.site, pr->P * sizeof(double), cudaMemcpyDeviceToHost, s));
    H3G_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    cudaEventElapsedTime(&pr->last_ms, pr->ev0, pr->ev1);
    pr->has_model = false;   // the installed model described caller P matrices only
    pr->model_hash = 0;
    *lnl = hout[0];
    return H3G_OK;
}

extern "C" h3g_status h3g_branch_length_gradients(h3g_problem* pr, int S, const double* pi, const double* Q, const double* lam,
                                                  const double* U, const double* V, const double* bl, int precision,
                                                  double* lnl, double* grad) {
    if (!pr || !lnl) return H3G_ERR_ARG;
    const double one = 1.0;
    h3g_model_desc d{};
    d.S = S; d.pi = pi; d.n_models = 1; d.Q = Q; d.lam = lam; d.U = U; d.V = V;
    d.K = 1; d.class_w = &one; d.M = 1; d.rates = &one; d.rate_w = &one;
    d.time_mode = H3G_TIME_RAW; d.precision = precision; d.zero_l_sentinel = 0;
    h3g_status st = h3g_model_set(pr, &d);
    if (st != H3G_OK) return st;
    h3g_result r{};
    r.grad_t = grad;
    st = h3g_eval(pr, bl, H3G_WANT_LNL | H3G_WANT_GRAD_T, &r);
    *lnl = r.lnl;
    return st;
}


// ------------------------------------------------------------------ batches
// Many independent problems (genes) evaluated by one graph launch.  The genes are spread over
// n_slots CUDA streams by longest-processing-time assignment on n x Pp x M; each slot owns one
// workspace sized for the largest gene it serves, so device memory is n_slots workspaces rather
// than one per gene.  A slot runs its genes one after another (H2D branch lengths, the evaluation's
// kernels, D2H results); the slots run concurrently.  The whole batch is captured once per `want`
// into one CUDA graph and replayed.
struct h3g_batch {
    h3g_ctx* ctx = nullptr;
    std::vector<h3g_problem*> probs;
    struct Slot {
        cudaStream_t s = nullptr;
        cudaEvent_t done = nullptr;
        DevArena mem;
        Work w{};
        MixedWork mw{};
        WsLayout L{};
        std::vector<int> genes;
    };
    std::vector<std::unique_ptr<Slot>> slots;
    int precision = -1;
    std::vector<WsLayout> gene_layout;                // per gene, for its chunking and branch groups
    std::vector<Model> captured_md;                   // models the graphs were captured with
    cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
    struct GraphEntry { unsigned key; cudaGraphExec_t exec; int launches; };
    std::vector<GraphEntry> graphs;
    float last_ms = 0.f;
    int last_launches = 0;
    void drop_graphs() {
        for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
        graphs.clear();
    }
    ~h3g_batch() {
        drop_graphs();
        for (auto& sl : slots) {
            if (sl->done) cudaEventDestroy(sl->done);
            if (sl->s) cudaStreamDestroy(sl->s);
        }
        if (fork) cudaEventDestroy(fork);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
};

extern "C" h3g_status h3g_batch_create(h3g_ctx* ctx, int n_problems, h3g_problem* const* problems, int n_slots,
                                       h3g_batch** out) {
    if (!ctx || !out || n_problems < 1 || !problems) return H3G_ERR_ARG;
    *out = nullptr;
    if (n_slots < 1 || n_slots > 64) return fail(ctx, H3G_ERR_ARG, "n_slots must be in [1, 64]");
    for (int i = 0; i < n_problems; ++i) {
        if (!problems[i] || problems[i]->ctx != ctx) return fail(ctx, H3G_ERR_ARG, "every problem must live on this context");
        if (problems[i]->batch) return fail(ctx, H3G_ERR_STATE, "a problem already belongs to a batch");
        for (int j = 0; j < i; ++j)
            if (problems[j] == problems[i]) return fail(ctx, H3G_ERR_ARG, "a problem is listed twice");
    }
    try {
        cudaSetDevice(ctx->device);
        auto b = std::make_unique<h3g_batch>();
        b->ctx = ctx;
        b->probs.assign(problems, problems + n_problems);
        H3G_TRY_CUDA(ctx, cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        H3G_TRY_CUDA(ctx, cudaEventCreate(&b->ev0));
        H3G_TRY_CUDA(ctx, cudaEventCreate(&b->ev1));
        for (int k = 0; k < std::min(n_slots, n_problems); ++k) {
            auto sl = std::make_unique<h3g_batch::Slot>();
            H3G_TRY_CUDA(ctx, cudaStreamCreateWithFlags(&sl->s, cudaStreamNonBlocking));
            H3G_TRY_CUDA(ctx, cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming));
            b->slots.push_back(std::move(sl));
        }
        cudaStreamSynchronize(ctx->stream);
        for (h3g_problem* pr : b->probs) {
            // the problem's own workspace is no longer needed: it evaluates in the batch's slots
            pr->drop_graphs();
            pr->work_mem.release();
            pr->w = Work{};
            pr->mw = MixedWork{};
            std::fill(pr->work_key, pr->work_key + 4, size_t(0));
            pr->batch = b.get();
        }
        *out = b.release();
        return H3G_OK;
    } catch (const std::bad_alloc&) {
        return fail(ctx, H3G_ERR_OOM, "host allocation failed");
    }
}

extern "C" h3g_status h3g_batch_destroy(h3g_batch* b) {
    if (!b) return H3G_ERR_ARG;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    for (auto& sl : b->slots) cudaStreamSynchronize(sl->s);
    for (h3g_problem* pr : b->probs) {
        pr->batch = nullptr;
        pr->has_model = false;        // its workspace went with the batch: install a model again to use it alone
        pr->model_hash = 0;
    }
    delete b;
    return H3G_OK;
}

// Slot assignment and slot workspaces for the installed models (grow-only, like a problem's).
static h3g_status batch_prepare(h3g_batch* b) {
    h3g_ctx* ctx = b->ctx;
    const int G = int(b->probs.size());
    int prec = -1;
    for (h3g_problem* pr : b->probs) {
        if (!pr->has_model) return fail(ctx, H3G_ERR_STATE, "every problem of a batch needs a model (h3g_model_set)");
        if (prec >= 0 && pr->precision != prec) return fail(ctx, H3G_ERR_ARG, "the problems of a batch must share one precision");
        prec = pr->precision;
    }
    std::vector<WsLayout> lay(G);
    for (int g = 0; g < G; ++g) {
        const h3g_problem* pr = b->probs[g];
        lay[g] = ws_layout(size_t(pr->n), size_t(pr->NI), size_t(pr->Pp), pr->M, pr->K, pr->nmod, pr->ndirs,
                           effective_tuning(pr, pr->M, pr->K, pr->nmod, pr->ndirs));
    }
    const bool first = b->slots[0]->genes.empty() && b->slots[0]->w.P == nullptr;
    if (first || prec != b->precision) {
        // longest processing time first: genes by decreasing n x Pp x M, each to the least loaded slot
        std::vector<int> order(G);
        for (int g = 0; g < G; ++g) order[g] = g;
        auto cost = [&](int g) { return double(b->probs[g]->n) * double(b->probs[g]->Pp) * double(b->probs[g]->M); };
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(x) > cost(y); });
        std::vector<double> load(b->slots.size(), 0.0);
        for (auto& sl : b->slots) sl->genes.clear();
        for (int g : order) {
            const size_t k = size_t(std::min_element(load.begin(), load.end()) - load.begin());
            b->slots[k]->genes.push_back(g);
            load[k] += cost(g);
        }
        for (auto& sl : b->slots) std::sort(sl->genes.begin(), sl->genes.end());
    }
    for (auto& sl : b->slots) {
        WsLayout need;
        for (int g : sl->genes) need.max_with(lay[g]);
        WsLayout have = sl->L;
        have.max_with(need);
        const bool fits = sl->w.P && prec == b->precision && std::memcmp(&have, &sl->L, sizeof(WsLayout)) == 0;
        if (fits) continue;
        cudaStreamSynchronize(ctx->stream);
        for (auto& t : b->slots) cudaStreamSynchronize(t->s);
        b->drop_graphs();
        sl->mem.release();
        sl->L = have;
        if (h3g_status st = ws_alloc(ctx, have, prec, sl->mem, sl->w, sl->mw); st != H3G_OK) {
            sl->mem.release();
            sl->w = Work{};
            sl->L = WsLayout{};
            return st;
        }
    }
    b->precision = prec;
    b->gene_layout = lay;
    return H3G_OK;
}

// The workspace view gene g evaluates in: its slot's buffers, its own branch lengths, chunking and groups.
static Work batch_view(const h3g_batch* b, const h3g_batch::Slot& sl, int g) {
    Work w = sl.w;
    w.bl = b->probs[g]->d_bl;
    w.nchunk = b->gene_layout[g].nchunk;
    w.chunk = b->gene_layout[g].chunk;
    w.ngroups = b->gene_layout[g].ngroups;
    return w;
}

extern "C" h3g_status h3g_batch_eval(h3g_batch* b, const double* const* bl, unsigned want, h3g_result* results) {
    if (!b || !bl || !results) return H3G_ERR_ARG;
    h3g_ctx* ctx = b->ctx;
    const int G = int(b->probs.size());
    for (int g = 0; g < G; ++g) {
        if (!bl[g]) return fail(ctx, H3G_ERR_ARG, "branch lengths missing for a problem");
        if (h3g_status st = check_bl(b->probs[g], bl[g]); st != H3G_OK) return st;
    }
    cudaSetDevice(ctx->device);
    if (h3g_status st = batch_prepare(b); st != H3G_OK) return st;
    // models reinstalled with different device buffers invalidate the captured graphs
    bool same = int(b->captured_md.size()) == G;
    for (int g = 0; g < G && same; ++g) same = std::memcmp(&b->captured_md[g], &b->probs[g]->md, sizeof(Model)) == 0;
    if (!same) {
        b->drop_graphs();
        b->captured_md.resize(G);
        for (int g = 0; g < G; ++g) b->captured_md[g] = b->probs[g]->md;
    }
    for (int g = 0; g < G; ++g) {
        h3g_problem* pr = b->probs[g];
        std::copy(bl[g], bl[g] + pr->n, pr->h_pin);
        pr->h_pin[pr->root] = 0.0;
    }
    const unsigned key = norm_want(want);
    cudaStream_t s = ctx->stream;
    cudaGraphExec_t exec = nullptr;
    for (auto& e : b->graphs) if (e.key == key) { exec = e.exec; b->last_launches = e.launches; }
    if (!exec) {
        cudaGraph_t graph = nullptr;
        int launches = 0;
        H3G_TRY_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        cudaEventRecord(b->fork, s);
        for (auto& sl : b->slots) {
            cudaStreamWaitEvent(sl->s, b->fork, 0);
            for (int g : sl->genes) {
                h3g_problem* pr = b->probs[g];
                const Work w = batch_view(b, *sl, g);
                cudaMemcpyAsync(pr->d_bl, pr->h_pin, size_t(pr->n) * sizeof(double), cudaMemcpyHostToDevice, sl->s);
                launches += enqueue_eval_on(pr, key, false, sl->s, w, sl->mw);
                enqueue_readback_on(pr, key, sl->s, w);
            }
            cudaEventRecord(sl->done, sl->s);
            cudaStreamWaitEvent(s, sl->done, 0);
        }
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (e != cudaSuccess) { ctx->err = std::string("batch graph capture: ") + cudaGetErrorString(e); return H3G_ERR_CUDA; }
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) { ctx->err = std::string("batch graph instantiate: ") + cudaGetErrorString(e); return H3G_ERR_CUDA; }
        b->graphs.push_back({key, exec, launches});
        b->last_launches = launches;
    }
    H3G_TRY_CUDA(ctx, cudaEventRecord(b->ev0, s));
    H3G_TRY_CUDA(ctx, cudaGraphLaunch(exec, s));
    H3G_TRY_CUDA(ctx, cudaEventRecord(b->ev1, s));
    H3G_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
    bool expired = false;
    for (int g = 0; g < G; ++g) {
        h3g_problem* pr = b->probs[g];
        unpack_result(pr, key, &results[g]);
        expired = expired || pr->h_pin[pr->off_out + 1] != 0.0;
    }
    if (expired) {
        for (auto& sl : b->slots) if (sl->w.err) cudaMemsetAsync(sl->w.err, 0, sizeof(int), s);
        cudaStreamSynchronize(s);
        return fail(ctx, H3G_ERR_TIMEOUT, "a bounded device wait expired in the batch (results are invalid)");
    }
    for (int g = 0; g < G; ++g)
        if (!std::isfinite(results[g].lnl)) return fail(ctx, H3G_ERR_NUMERIC, "non-finite log-likelihood in the batch");
    return H3G_OK;
}

extern "C" h3g_status h3g_batch_last_stats(const h3g_batch* b, double* device_ms, int* n_launches) {
    if (!b) return H3G_ERR_ARG;
    if (device_ms) *device_ms = b->last_ms;
    if (n_launches) *n_launches = b->last_launches;
    return H3G_OK;
}

extern "C" h3g_status h3g_last_eval_stats(const h3g_problem* pr, double* device_ms, int* n_launches) {
    if (!pr) return H3G_ERR_ARG;
    if (device_ms) *device_ms = pr->last_ms;
    if (n_launches) *n_launches = pr->last_launches;
    return H3G_OK;
}

extern "C" h3g_status h3g_last_eval_transfer(const h3g_problem* pr, size_t* h2d_bytes, size_t* d2h_bytes) {
    if (!pr) return H3G_ERR_ARG;
    if (h2d_bytes) *h2d_bytes = pr->last_h2d;
    if (d2h_bytes) *d2h_bytes = pr->last_d2h;
    return H3G_OK;
}
