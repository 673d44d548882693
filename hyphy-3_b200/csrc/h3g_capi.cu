// h3g_capi.cu — C ABI (include/h3g.h): problem/model upload, device workspace
// and the per-evaluation launch sequence.  No exception crosses the boundary.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/h3g.h"
#include "h3g_common.cuh"
#include "h3g_kernels.h"
#include "h3g_mixed.h"

using namespace h3g;

struct h3g_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
};

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
    int n = 0, root = -1, T = 0, P = 0, Pp = 0, NI = 0;
    std::vector<int> ch_off, ch, iidx, taxon, in_off, out_off, in_nodes, out_nodes;
    std::vector<uint8_t> leaf;
    DevArena topo_mem, model_mem, work_mem;
    int *d_ch_off = nullptr, *d_ch = nullptr, *d_iidx = nullptr, *d_taxon = nullptr, *d_in_nodes = nullptr, *d_out_nodes = nullptr;
    uint8_t* d_leaf = nullptr;
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
    float last_ms = 0.f;
    int last_launches = 0;
    ~h3g_problem() {
        if (h_pin) cudaFreeHost(h_pin);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
    Topo topo() const {
        Topo t;
        t.n = n; t.root = root; t.NI = NI; t.T = T; t.P = P; t.Pp = Pp; t.S = S;
        t.ch_off = d_ch_off; t.ch = d_ch; t.iidx = d_iidx; t.leaf = d_leaf; t.taxon = d_taxon;
        t.states = d_states; t.masks = d_masks; t.w = d_w;
        t.all_mask = S >= 64 ? ~uint64_t(0) : ((uint64_t(1) << S) - 1);
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
    mixed_configure();
    *out = c;
    return H3G_OK;
}

extern "C" h3g_status h3g_ctx_destroy(h3g_ctx* ctx) {
    if (!ctx) return H3G_ERR_ARG;
    cudaSetDevice(ctx->device);
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
        int H = 0, Dp = 0;
        for (int i = 0; i < n; ++i) if (!is_leaf[i]) { H = std::max(H, height[i]); Dp = std::max(Dp, depth[i]); }
        pr->in_off.assign(1, 0);
        for (int h = 1; h <= H; ++h) {
            for (int i = 0; i < n; ++i) if (!is_leaf[i] && height[i] == h) pr->in_nodes.push_back(i);
            pr->in_off.push_back(int(pr->in_nodes.size()));
        }
        pr->out_off.assign(1, 0);
        for (int d = 0; d <= Dp; ++d) {
            for (int i = 0; i < n; ++i) if (!is_leaf[i] && depth[i] == d) pr->out_nodes.push_back(i);
            pr->out_off.push_back(int(pr->out_nodes.size()));
        }
        // patterns, taxon-major with padding (missing data, weight 0)
        const int Pp = pr->Pp, T = n_taxa;
        std::vector<int8_t> st(size_t(std::max(T, 1)) * Pp, int8_t(-1));
        std::vector<uint64_t> mk(size_t(std::max(T, 1)) * Pp, ~uint64_t(0));
        std::vector<double> wt(Pp, 0.0);
        for (int p = 0; p < n_patterns; ++p) {
            if (!(weights[p] >= 0.0) || !std::isfinite(weights[p])) return fail(ctx, H3G_ERR_ARG, "pattern weights must be finite and >= 0");
            wt[p] = weights[p];
            for (int t = 0; t < T; ++t) {
                st[size_t(t) * Pp + p] = states[size_t(p) * T + t];
                mk[size_t(t) * Pp + p] = masks[size_t(p) * T + t];
            }
        }
        auto& A = pr->topo_mem;
        cudaStream_t s = ctx->stream;
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_ch_off, n + 1));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_ch, std::max<size_t>(pr->ch.size(), 1)));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_iidx, n));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_taxon, n));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_leaf, n));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_in_nodes, std::max<size_t>(pr->in_nodes.size(), 1)));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_out_nodes, std::max<size_t>(pr->out_nodes.size(), 1)));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_states, st.size()));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_masks, mk.size()));
        H3G_TRY_CUDA(ctx, A.alloc(&pr->d_w, wt.size()));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_ch_off, pr->ch_off.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
        if (!pr->ch.empty()) H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_ch, pr->ch.data(), pr->ch.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_iidx, pr->iidx.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
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
        *out = guard.release();
        return H3G_OK;
    } catch (const std::bad_alloc&) {
        return fail(ctx, H3G_ERR_OOM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(ctx, H3G_ERR_ARG, e.what());
    }
}

extern "C" h3g_status h3g_problem_destroy(h3g_problem* prob) {
    if (!prob) return H3G_ERR_ARG;
    cudaSetDevice(prob->ctx->device);
    cudaStreamSynchronize(prob->ctx->stream);
    delete prob;
    return H3G_OK;
}

static void pad_matrix(const double* src, int S, double* dst) {
    std::fill(dst, dst + SP2, 0.0);
    for (int i = 0; i < S; ++i) std::copy(src + size_t(i) * S, src + size_t(i) * S + S, dst + size_t(i) * SP);
}

// Allocate the evaluation workspace for (M, K, nmod, ndirs); reuses it when unchanged.
static h3g_status ensure_workspace(h3g_problem* pr, int M, int K, int nmod, int ndirs) {
    h3g_ctx* ctx = pr->ctx;
    const size_t key[4] = {size_t(M), size_t(K), size_t(nmod), size_t(ndirs)};
    if (pr->w.P && std::equal(key, key + 4, pr->work_key)) return H3G_OK;
    cudaStreamSynchronize(ctx->stream);
    pr->work_mem.release();
    if (pr->h_pin) { cudaFreeHost(pr->h_pin); pr->h_pin = nullptr; }
    std::copy(key, key + 4, pr->work_key);
    const size_t n = pr->n, NI = pr->NI, Pp = pr->Pp;
    Work& w = pr->w;
    w = Work{};
    auto& A = pr->work_mem;
    const size_t mats = size_t(M) * n * SP2;
    // enough A chunks for ~600 CTAs, never below 256 patterns per chunk
    const int want_chunks = std::max<int>(1, int((600 + n * M - 1) / (n * M)));
    const int max_chunks = std::max<int>(1, int(Pp / 256));
    w.nchunk = std::min(want_chunks, max_chunks);
    w.chunk = int((Pp / TP + w.nchunk - 1) / w.nchunk) * TP;
    w.nchunk = int((Pp + w.chunk - 1) / w.chunk);
    H3G_TRY_CUDA(ctx, A.alloc(&pr->d_bl, n));
    w.bl = pr->d_bl;
    H3G_TRY_CUDA(ctx, A.alloc(&w.P, mats));
    H3G_TRY_CUDA(ctx, A.alloc(&w.PT, mats));
    H3G_TRY_CUDA(ctx, A.alloc(&w.dP, mats));
    H3G_TRY_CUDA(ctx, A.alloc(&w.rs, size_t(M) * n * SP));
    H3G_TRY_CUDA(ctx, A.alloc(&w.f, size_t(M) * Pp));
    H3G_TRY_CUDA(ctx, A.alloc(&w.rw, size_t(M) * Pp));
    H3G_TRY_CUDA(ctx, A.alloc(&w.contrib, Pp));
    H3G_TRY_CUDA(ctx, A.alloc(&w.site, Pp));
    H3G_TRY_CUDA(ctx, A.alloc(&w.Ecum, NI * M * Pp));
    H3G_TRY_CUDA(ctx, A.alloc(&w.Eown, NI * M * Pp));
    H3G_TRY_CUDA(ctx, A.alloc(&w.gt, size_t(M) * n));
    H3G_TRY_CUDA(ctx, A.alloc(&w.Apart, n * M * size_t(w.nchunk) * SP2));
    H3G_TRY_CUDA(ctx, A.alloc(&w.Hpart, size_t(nmod) * M * n * SP2));
    H3G_TRY_CUDA(ctx, A.alloc(&w.gc, size_t(std::max(K, 1)) * M * n));
    H3G_TRY_CUDA(ctx, A.alloc(&w.stg, size_t(nmod) * M * n));
    H3G_TRY_CUDA(ctx, A.alloc(&w.H, size_t(nmod) * SP2));
    H3G_TRY_CUDA(ctx, A.alloc(&w.dirpart, size_t(std::max(ndirs, 1)) * nmod));
    const size_t n_out = 2 + n + K + nmod + M;
    H3G_TRY_CUDA(ctx, A.alloc(&w.out, n_out));
    if (pr->precision == H3G_PREC_FP64) {
        H3G_TRY_CUDA(ctx, A.alloc(&w.D, NI * M * SP * Pp));
        H3G_TRY_CUDA(ctx, A.alloc(&w.Ms, NI * M * SP * Pp));
        H3G_TRY_CUDA(ctx, A.alloc(&w.U, NI * M * SP * Pp));
        H3G_TRY_CUDA(ctx, A.alloc(&w.Vf, n * M * SP * Pp));
    } else {
        h3g_status st = mixed_alloc(pr->mw, A.ptrs, pr->n, pr->NI, M, pr->Pp);
        if (st != H3G_OK) return fail(ctx, st, "mixed-precision workspace allocation failed");
    }
    cudaMemsetAsync(w.gc, 0, size_t(std::max(K, 1)) * M * n * sizeof(double), ctx->stream);
    cudaMemsetAsync(w.stg, 0, size_t(nmod) * M * n * sizeof(double), ctx->stream);
    cudaMemsetAsync(w.Hpart, 0, size_t(nmod) * M * n * SP2 * sizeof(double), ctx->stream);
    pr->h_pin_count = n + n_out;
    H3G_TRY_CUDA(ctx, cudaMallocHost(reinterpret_cast<void**>(&pr->h_pin), pr->h_pin_count * sizeof(double)));
    return H3G_OK;
}

extern "C" h3g_status h3g_model_set(h3g_problem* pr, const h3g_model_desc* d) {
    if (!pr || !d) return H3G_ERR_ARG;
    h3g_ctx* ctx = pr->ctx;
    if (d->S < 1 || d->S > SP) return fail(ctx, H3G_ERR_ARG, "S must be in [1, 64]");
    if (d->K < 1 || d->M < 1 || d->M > kMaxRateClasses) return fail(ctx, H3G_ERR_ARG, "need K >= 1 and 1 <= M <= 16");
    if (d->n_models != d->K + (d->has_bg ? 1 : 0)) return fail(ctx, H3G_ERR_ARG, "n_models must equal K + has_bg");
    if (!d->pi || !d->Q || !d->lam || !d->U || !d->V || !d->class_w || !d->rates || !d->rate_w)
        return fail(ctx, H3G_ERR_ARG, "model arrays missing");
    if (d->time_mode == H3G_TIME_NORMALIZED && !d->mu) return fail(ctx, H3G_ERR_ARG, "normalized time needs mu");
    if (d->n_dirs < 0 || (d->n_dirs > 0 && !d->dQ)) return fail(ctx, H3G_ERR_ARG, "dQ directions missing");
    if (d->precision != H3G_PREC_FP64 && d->precision != H3G_PREC_MIXED) return fail(ctx, H3G_ERR_ARG, "unknown precision");
    if (d->precision == H3G_PREC_MIXED && !mixed_available()) return fail(ctx, H3G_ERR_CUDA, "mixed-precision path not built");
    const int S = d->S, nm = d->n_models;
    auto finite = [](const double* a, size_t k) { for (size_t i = 0; i < k; ++i) if (!std::isfinite(a[i])) return false; return true; };
    if (!finite(d->pi, S) || !finite(d->Q, size_t(nm) * S * S) || !finite(d->lam, size_t(nm) * S) || !finite(d->U, size_t(nm) * S * S) ||
        !finite(d->V, size_t(nm) * S * S) || !finite(d->class_w, d->K) || !finite(d->rates, d->M) || !finite(d->rate_w, d->M))
        return fail(ctx, H3G_ERR_NUMERIC, "non-finite model parameters");
    try {
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        pr->S = S; pr->M = d->M; pr->K = d->K; pr->nmod = nm; pr->ndirs = d->n_dirs; pr->has_bg = d->has_bg;
        pr->time_mode = d->time_mode; pr->sentinel = d->zero_l_sentinel;
        const bool prec_change = pr->precision != d->precision;
        pr->precision = d->precision;
        if (prec_change) { pr->work_mem.release(); pr->w = Work{}; }
        std::vector<double> pi(SP, 0.0), Q(size_t(nm) * SP2), U(size_t(nm) * SP2), V(size_t(nm) * SP2), lam(size_t(nm) * SP, 0.0);
        std::copy(d->pi, d->pi + S, pi.begin());
        for (int k = 0; k < nm; ++k) {
            pad_matrix(d->Q + size_t(k) * S * S, S, &Q[size_t(k) * SP2]);
            pad_matrix(d->U + size_t(k) * S * S, S, &U[size_t(k) * SP2]);
            pad_matrix(d->V + size_t(k) * S * S, S, &V[size_t(k) * SP2]);
            std::copy(d->lam + size_t(k) * S, d->lam + size_t(k) * S + S, &lam[size_t(k) * SP]);
        }
        std::vector<double> mu(nm, 1.0);
        if (d->mu) std::copy(d->mu, d->mu + nm, mu.begin());
        pr->h_mu = mu;
        std::vector<double> dQ(size_t(std::max(d->n_dirs, 1)) * nm * SP2, 0.0);
        for (int x = 0; x < d->n_dirs; ++x)
            for (int k = 0; k < nm; ++k) pad_matrix(d->dQ + (size_t(x) * nm + k) * S * S, S, &dQ[(size_t(x) * nm + k) * SP2]);
        std::vector<uint8_t> it(pr->n, 1);
        if (d->is_test) std::copy(d->is_test, d->is_test + pr->n, it.begin());
        auto& A = pr->model_mem;
        A.release();
        Model md{};
        double *dpi, *dQd, *dlam, *dU, *dV, *dmu, *dcw, *drt, *drw, *ddQ;
        uint8_t* dit;
        H3G_TRY_CUDA(ctx, A.alloc(&dpi, SP));
        H3G_TRY_CUDA(ctx, A.alloc(&dQd, Q.size()));
        H3G_TRY_CUDA(ctx, A.alloc(&dlam, lam.size()));
        H3G_TRY_CUDA(ctx, A.alloc(&dU, U.size()));
        H3G_TRY_CUDA(ctx, A.alloc(&dV, V.size()));
        H3G_TRY_CUDA(ctx, A.alloc(&dmu, mu.size()));
        H3G_TRY_CUDA(ctx, A.alloc(&dcw, d->K));
        H3G_TRY_CUDA(ctx, A.alloc(&drt, d->M));
        H3G_TRY_CUDA(ctx, A.alloc(&drw, d->M));
        H3G_TRY_CUDA(ctx, A.alloc(&ddQ, dQ.size()));
        H3G_TRY_CUDA(ctx, A.alloc(&dit, it.size()));
        cudaStream_t s = ctx->stream;
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(dpi, pi.data(), SP * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(dQd, Q.data(), Q.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(dlam, lam.data(), lam.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(dU, U.data(), U.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(dV, V.data(), V.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(dmu, mu.data(), mu.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(dcw, d->class_w, d->K * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(drt, d->rates, d->M * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(drw, d->rate_w, d->M * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(ddQ, dQ.data(), dQ.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(dit, it.data(), it.size(), cudaMemcpyHostToDevice, s));
        md.M = d->M; md.K = d->K; md.has_bg = d->has_bg; md.nmod = nm; md.time_mode = d->time_mode; md.ndirs = d->n_dirs;
        md.sentinel = d->zero_l_sentinel;
        md.pi = dpi; md.Q = dQd; md.lam = dlam; md.U = dU; md.V = dV; md.mu = dmu; md.class_w = dcw; md.rates = drt;
        md.rate_w = drw; md.is_test = d->is_test ? dit : nullptr; md.dQ = ddQ;
        pr->md = md;
        h3g_status st = ensure_workspace(pr, d->M, d->K, nm, d->n_dirs);
        if (st != H3G_OK) { pr->has_model = false; return st; }
        H3G_TRY_CUDA(ctx, cudaStreamSynchronize(s));
        pr->has_model = true;
        return H3G_OK;
    } catch (const std::bad_alloc&) {
        return fail(ctx, H3G_ERR_OOM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(ctx, H3G_ERR_ARG, e.what());
    }
}

// Enqueue the pruning pipeline (inside, root and optionally outside + gradients).
static int enqueue_eval(h3g_problem* pr, unsigned want, bool from_given_P) {
    const Topo t = pr->topo();
    const Model& md = pr->md;
    const Work& w = pr->w;
    cudaStream_t s = pr->ctx->stream;
    const bool mixed = pr->precision == H3G_PREC_MIXED;
    const bool grads = (want & (H3G_WANT_GRAD_T | H3G_WANT_GRAD_GLOBAL)) != 0;
    const bool global = (want & H3G_WANT_GRAD_GLOBAL) != 0;
    int L = 0;
    L += from_given_P ? launch_prep_given_P(t, w, s) : launch_build_P(t, md, w, s);
    if (mixed) L += mixed_prepare(t, md, w, pr->mw, s);
    for (size_t lv = 0; lv + 1 < pr->in_off.size(); ++lv) {
        const int cnt = pr->in_off[lv + 1] - pr->in_off[lv];
        if (!cnt) continue;
        const int* nodes = pr->d_in_nodes + pr->in_off[lv];
        L += mixed ? launch_inside_mixed(t, md, w, pr->mw, nodes, cnt, s) : launch_inside_fp64(t, md, w, nodes, cnt, s);
    }
    L += mixed ? launch_root_mixed(t, md, w, pr->mw, s) : launch_root(t, md, w, s);
    if (grads) {
        for (size_t lv = 0; lv + 1 < pr->out_off.size(); ++lv) {
            const int cnt = pr->out_off[lv + 1] - pr->out_off[lv];
            if (!cnt) continue;
            const int* nodes = pr->d_out_nodes + pr->out_off[lv];
            L += mixed ? launch_outside_mixed(t, md, w, pr->mw, nodes, cnt, s) : launch_outside_fp64(t, md, w, nodes, cnt, 1, s);
        }
        L += mixed ? launch_accumA_mixed(t, md, w, pr->mw, s) : launch_accumA_fp64(t, md, w, s);
        L += launch_frechet(t, md, w, global ? 1 : 0, s);
        if (global) L += launch_global(t, md, w, s);
    }
    L += launch_small(t, md, w, grads ? 1 : 0, s);
    if (global) L += launch_dir(t, md, w, s);
    return L;
}

extern "C" h3g_status h3g_eval(h3g_problem* pr, const double* bl, unsigned want, h3g_result* out) {
    if (!pr || !bl || !out) return H3G_ERR_ARG;
    h3g_ctx* ctx = pr->ctx;
    if (!pr->has_model) return fail(ctx, H3G_ERR_STATE, "h3g_eval before h3g_model_set");
    const int n = pr->n;
    for (int i = 0; i < n; ++i)
        if (i != pr->root && !std::isfinite(bl[i])) return fail(ctx, H3G_ERR_NUMERIC, "non-finite branch length");
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    double* hbl = pr->h_pin;
    double* hout = pr->h_pin + n;
    std::copy(bl, bl + n, hbl);
    hbl[pr->root] = 0.0;
    H3G_TRY_CUDA(ctx, cudaMemcpyAsync(pr->d_bl, hbl, n * sizeof(double), cudaMemcpyHostToDevice, s));
    H3G_TRY_CUDA(ctx, cudaEventRecord(pr->ev0, s));
    pr->last_launches = enqueue_eval(pr, want, false);
    H3G_TRY_CUDA(ctx, cudaGetLastError());
    H3G_TRY_CUDA(ctx, cudaEventRecord(pr->ev1, s));
    const size_t n_out = 2 + n + pr->K + pr->nmod + pr->M;
    H3G_TRY_CUDA(ctx, cudaMemcpyAsync(hout, pr->w.out, n_out * sizeof(double), cudaMemcpyDeviceToHost, s));
    std::vector<double> dirpart;
    const bool global = (want & H3G_WANT_GRAD_GLOBAL) != 0;
    if (global && pr->ndirs > 0) {
        dirpart.resize(size_t(pr->ndirs) * pr->nmod);
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(dirpart.data(), pr->w.dirpart, dirpart.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    if ((want & H3G_WANT_SITE_LNL) && out->site_lnl && pr->P > 0)
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(out->site_lnl, pr->w.site, pr->P * sizeof(double), cudaMemcpyDeviceToHost, s));
    H3G_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    cudaEventElapsedTime(&pr->last_ms, pr->ev0, pr->ev1);
    out->lnl = hout[0];
    const bool grads = (want & (H3G_WANT_GRAD_T | H3G_WANT_GRAD_GLOBAL)) != 0;
    if (out->grad_t) {
        for (int b = 0; b < n; ++b) out->grad_t[b] = grads ? hout[2 + b] : 0.0;
        out->grad_t[pr->root] = 0.0;
    }
    if (out->grad_class_w) for (int k = 0; k < pr->K; ++k) out->grad_class_w[k] = global ? hout[2 + n + k] : 0.0;
    if (out->grad_rate_w) for (int m = 0; m < pr->M; ++m) out->grad_rate_w[m] = grads ? hout[2 + n + pr->K + pr->nmod + m] : 0.0;
    if (out->grad_dir)
        for (int x = 0; x < pr->ndirs; ++x) {
            double g = 0.0;
            if (global) for (int k = 0; k < pr->nmod; ++k) g += dirpart[size_t(x) * pr->nmod + k];
            out->grad_dir[x] = g;
        }
    if (!std::isfinite(out->lnl)) return fail(ctx, H3G_ERR_NUMERIC, "non-finite log-likelihood");
    return H3G_OK;
}

extern "C" h3g_status h3g_eval_from_P(h3g_problem* pr, int S, const double* P, const double* pi, double* lnl, double* site_lnl) {
    if (!pr || !P || !pi || !lnl) return H3G_ERR_ARG;
    h3g_ctx* ctx = pr->ctx;
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
    double* hout = pr->h_pin + n;
    H3G_TRY_CUDA(ctx, cudaMemcpyAsync(hout, pr->w.out, sizeof(double), cudaMemcpyDeviceToHost, s));
    if (site_lnl && pr->P > 0)
        H3G_TRY_CUDA(ctx, cudaMemcpyAsync(site_lnl, pr->w.site, pr->P * sizeof(double), cudaMemcpyDeviceToHost, s));
    H3G_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    cudaEventElapsedTime(&pr->last_ms, pr->ev0, pr->ev1);
    pr->has_model = false;   // the installed model described caller P matrices only
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

extern "C" h3g_status h3g_last_eval_stats(const h3g_problem* pr, double* device_ms, int* n_launches) {
    if (!pr) return H3G_ERR_ARG;
    if (device_ms) *device_ms = pr->last_ms;
    if (n_launches) *n_launches = pr->last_launches;
    return H3G_OK;
}
