// h3g_nuc.cu — the nucleotide GTR log-likelihood on the device (h3g_nuc_eval_from_P).
//
// LikelihoodEngine::compute_gtr_log_likelihood (likelihood.hpp:181-254) prunes every
// nucleotide pattern through the tree with 4 x 4 transition matrices.  Here one thread
// owns one pattern and walks the tree depth-first along an event list shared by all
// threads (open an internal node / close a node into its parent), so a warp reads the
// same transition matrix at every step (one broadcast) and there is no inter-thread
// dependency.  The partial of the node being accumulated stays in registers; opening an
// internal node parks its parent's partial in a [depth][pattern] buffer (consecutive
// threads, consecutive addresses), closing it brings the parent back.  Partials are
// rescaled by 2^256 when their maximum falls below 2^-256; L = pi . D_root, the site
// log-likelihood log L - E ln 2, or the reference's -1e20 when L <= 0; the weighted sum
// over patterns is a fixed-order Neumaier sum.  FP64 throughout.
//
// With fewer patterns than it takes to fill the GPU (kLevelBelow), the tree is walked
// level by level instead: one launch per height, one thread per (internal node of the
// level, pattern), partials stored per internal node.
#include <algorithm>
#include <cmath>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "h3g_common.cuh"
#include "h3g_fel.h"

namespace h3g {

Topo problem_topo(h3g_problem* pr, int S);                // h3g_capi.cu
cudaStream_t problem_stream(h3g_problem* pr);
void*& problem_nuc_state(h3g_problem* pr);
int problem_max_state(h3g_problem* pr);

namespace {

constexpr int kNucT = 128;                                 // threads per block (patterns)
constexpr int kLvlT = 256;
constexpr int kSumT = 1024;
constexpr int kLevelBelow = 131072;                        // patterns: below, the level-by-level walk

struct NucState {
    int n_ev = 0, depth = 1, P = 0;
    size_t Pp = 0;
    int* d_ev = nullptr;
    double* d_P = nullptr;                                 // [n][16]
    double* d_pi = nullptr;                                // [4]
    double* d_site = nullptr;                              // [P]
    double4* d_stk = nullptr;                              // [depth][Pp]
    int* d_exp = nullptr;                                  // [depth][Pp]
    bool levels = false;                                   // level-by-level walk
    std::vector<int> lv_off;                               // [H + 1] internal nodes by height
    int* d_lv = nullptr;                                   // [NI]
    double4* d_part = nullptr;                             // [NI][Pp]
    int* d_pexp = nullptr;                                 // [NI][Pp]
    double* d_lnl = nullptr;
    double* h_pin = nullptr;                               // lnl read back
    std::vector<void*> owned;
    ~NucState() {
        for (void* p : owned) cudaFree(p);
        if (h_pin) cudaFreeHost(h_pin);
    }
};

__global__ void __launch_bounds__(kNucT) k_nuc_lnl(Topo t, const int* __restrict__ ev, int n_ev, const double* __restrict__ P,
                                                    const double* __restrict__ pi, double4* __restrict__ stk,
                                                    int* __restrict__ sexp, double* __restrict__ site) {
    pdl_enter();
    const int p = int(blockIdx.x) * kNucT + int(threadIdx.x);
    if (p >= t.P) return;
    const size_t Pp = size_t(t.Pp);
    double d[4] = {1.0, 1.0, 1.0, 1.0};                     // partial of the innermost open node
    int E = 0, sp = -1;                                    // levels 0 .. sp - 1 are parked in stk
    for (int k = 0; k < n_ev; ++k) {
        const int code = __ldg(ev + k), node = code >> 1;
        if (code & 1) {                                    // open an internal node
            if (sp >= 0) {
                stk[size_t(sp) * Pp + p] = make_double4(d[0], d[1], d[2], d[3]);
                sexp[size_t(sp) * Pp + p] = E;
            }
            ++sp;
            d[0] = d[1] = d[2] = d[3] = 1.0;
            E = 0;
            continue;
        }
        double x[4];
        int Ex = 0;
        if (t.leaf[node]) {                                // likelihood.hpp:54-87
            const int tx = t.taxon[node];
            int st = -1;
            uint64_t mk = 0xF;
            if (tx >= 0) {
                st = t.states[size_t(tx) * Pp + p];
                if (!(st >= 0 && st < 4)) mk = t.masks[size_t(tx) * Pp + p];
            }
            if (st >= 0 && st < 4) {
#pragma unroll
                for (int i = 0; i < 4; ++i) x[i] = i == st ? 1.0 : 0.0;
            } else if (mk == 0 || (mk & 0xF) == 0xF) {
#pragma unroll
                for (int i = 0; i < 4; ++i) x[i] = 1.0;
            } else {
#pragma unroll
                for (int i = 0; i < 4; ++i) x[i] = ((mk >> i) & 1) ? 1.0 : 0.0;
            }
        } else {                                           // close an internal node: its partial is d
#pragma unroll
            for (int i = 0; i < 4; ++i) x[i] = d[i];
            Ex = E;
            --sp;
            const double4 v = stk[size_t(sp) * Pp + p];
            d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
            E = sexp[size_t(sp) * Pp + p];
        }
        const double* Pn = P + size_t(node) * 16;          // the same matrix for the whole warp
        double mx = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const double m = __ldg(Pn + 4 * i) * x[0] + __ldg(Pn + 4 * i + 1) * x[1] + __ldg(Pn + 4 * i + 2) * x[2] +
                             __ldg(Pn + 4 * i + 3) * x[3];
            d[i] *= m;
            mx = fmax(mx, d[i]);
        }
        E += Ex;
        if (mx > 0.0 && mx < 0x1p-256) {
#pragma unroll
            for (int i = 0; i < 4; ++i) d[i] *= 0x1p256;
            E += 256;
        }
    }
    const double L = pi[0] * d[0] + pi[1] * d[1] + pi[2] * d[2] + pi[3] * d[3];
    site[p] = L > 0.0 ? log(L) - double(E) * 0.69314718055994530942 : -1e20;
}

// leaf vector of taxon tx at pattern p (likelihood.hpp:54-87)
__device__ __forceinline__ void nuc_leaf(const Topo& t, int tx, int p, double (&x)[4]) {
    int st = -1;
    uint64_t mk = 0xF;
    if (tx >= 0) {
        st = t.states[size_t(tx) * size_t(t.Pp) + p];
        if (!(st >= 0 && st < 4)) mk = t.masks[size_t(tx) * size_t(t.Pp) + p];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
        x[i] = (st >= 0 && st < 4) ? (i == st ? 1.0 : 0.0) : ((mk == 0 || (mk & 0xF) == 0xF || ((mk >> i) & 1)) ? 1.0 : 0.0);
}

// one thread per (internal node of this level, pattern): the product of the children's messages
__global__ void __launch_bounds__(kLvlT) k_nuc_level(Topo t, const int* __restrict__ nodes, int cnt, const double* __restrict__ P,
                                                      const double* __restrict__ pi, double4* __restrict__ part,
                                                      int* __restrict__ pexp, double* __restrict__ site) {
    pdl_enter();                                           // the lower levels' partials are complete
    const int i = int(blockIdx.x) * kLvlT + int(threadIdx.x);
    if (i >= cnt * t.P) return;
    const int u = nodes[i / t.P], p = i - (i / t.P) * t.P;
    const size_t Pp = size_t(t.Pp);
    double d[4] = {1.0, 1.0, 1.0, 1.0};
    int E = 0;
    for (int e = t.ch_off[u]; e < t.ch_off[u + 1]; ++e) {
        const int c = t.ch[e];
        double x[4];
        if (t.leaf[c]) {
            nuc_leaf(t, t.taxon[c], p, x);
        } else {
            const size_t o = size_t(t.iidx[c]) * Pp + p;
            const double4 v = part[o];
            x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
            E += pexp[o];
        }
        const double* Pn = P + size_t(c) * 16;
        double mx = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            d[k] *= __ldg(Pn + 4 * k) * x[0] + __ldg(Pn + 4 * k + 1) * x[1] + __ldg(Pn + 4 * k + 2) * x[2] +
                    __ldg(Pn + 4 * k + 3) * x[3];
            mx = fmax(mx, d[k]);
        }
        if (mx > 0.0 && mx < 0x1p-256) {
#pragma unroll
            for (int k = 0; k < 4; ++k) d[k] *= 0x1p256;
            E += 256;
        }
    }
    if (u == t.root) {
        const double L = pi[0] * d[0] + pi[1] * d[1] + pi[2] * d[2] + pi[3] * d[3];
        site[p] = L > 0.0 ? log(L) - double(E) * 0.69314718055994530942 : -1e20;
    } else {
        const size_t o = size_t(t.iidx[u]) * Pp + p;
        part[o] = make_double4(d[0], d[1], d[2], d[3]);
        pexp[o] = E;
    }
}

// one block: weights x site log-likelihoods, Neumaier over contiguous chunks, then the chunk sums in order
__global__ void __launch_bounds__(kSumT) k_nuc_sum(const double* __restrict__ site, const double* __restrict__ w, int P,
                                                   double* __restrict__ out) {
    pdl_enter();                                           // k_nuc_lnl's site log-likelihoods are complete
    __shared__ double hi[kSumT], lo[kSumT];
    const int tid = threadIdx.x;
    const int chunk = (P + kSumT - 1) / kSumT, b = tid * chunk, e = min(P, b + chunk);
    double s = 0.0, c = 0.0;
    for (int i = b; i < e; ++i) {
        const double x = w[i] * site[i], t = s + x;
        c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
        s = t;
    }
    hi[tid] = s;
    lo[tid] = c;
    __syncthreads();
    if (tid == 0) {
        double S = 0.0, Cc = 0.0;
        for (int k = 0; k < kSumT; ++k)
            for (double x : {hi[k], lo[k]}) {
                const double t = S + x;
                Cc += fabs(S) >= fabs(x) ? (S - t) + x : (x - t) + S;
                S = t;
            }
        *out = S + Cc;
    }
}

// depth-first events (2 node + 1 opens an internal node, 2 node closes a node) and the
// largest number of internal nodes open at once
std::pair<std::vector<int>, int> dfs_events(const FelProblemView& v) {
    std::vector<int> ev;
    ev.reserve(2 * size_t(v.n));
    int open = 1, deepest = 1;
    std::vector<std::pair<int, int>> stk{{v.root, 0}};
    ev.push_back(2 * v.root + 1);
    while (!stk.empty()) {
        auto& [u, k] = stk.back();
        if (k < v.ch_off[u + 1] - v.ch_off[u]) {
            const int c = v.ch[v.ch_off[u] + k++];
            if (v.leaf[c]) {
                ev.push_back(2 * c);
            } else {
                ev.push_back(2 * c + 1);
                deepest = std::max(deepest, ++open);
                stk.push_back({c, 0});
            }
        } else {
            if (u != v.root) {
                ev.push_back(2 * u);
                --open;
            }
            stk.pop_back();
        }
    }
    return {ev, deepest};
}

NucState* nuc_state(h3g_problem* pr, const FelProblemView& v, std::string* err) {
    void*& slot = problem_nuc_state(pr);
    if (slot) return static_cast<NucState*>(slot);
    auto* s = new (std::nothrow) NucState;
    if (!s) { *err = "host allocation failed"; return nullptr; }
    const Topo t = problem_topo(pr, 4);
    auto [ev, deepest] = dfs_events(v);
    s->n_ev = int(ev.size());
    s->depth = deepest;
    s->P = t.P;
    s->Pp = size_t(t.Pp);
    s->levels = t.P < kLevelBelow;
    std::vector<int> lv;
    if (s->levels) {                                       // internal nodes by height, children first
        std::vector<int> h(size_t(v.n), 0);
        for (int e : ev)
            if (!(e & 1)) {                                // a node closes after its descendants
                const int u = e >> 1;
                for (int c = v.ch_off[u]; c < v.ch_off[u + 1]; ++c) h[size_t(u)] = std::max(h[size_t(u)], h[size_t(v.ch[c])] + 1);
            }
        for (int c = v.ch_off[v.root]; c < v.ch_off[v.root + 1]; ++c) h[size_t(v.root)] = std::max(h[size_t(v.root)], h[size_t(v.ch[c])] + 1);
        const int H = h[size_t(v.root)];
        s->lv_off.assign(size_t(H) + 1, 0);
        for (int u = 0; u < v.n; ++u)
            if (!v.leaf[u]) ++s->lv_off[size_t(h[size_t(u)])];
        for (int k = 1; k <= H; ++k) s->lv_off[size_t(k)] += s->lv_off[size_t(k) - 1];
        lv.resize(size_t(s->lv_off[size_t(H)]));
        std::vector<int> fill(s->lv_off.begin(), s->lv_off.end() - 1);
        for (int u = 0; u < v.n; ++u)
            if (!v.leaf[u]) lv[size_t(fill[size_t(h[size_t(u)]) - 1]++)] = u;
    }
    auto take = [&](auto** p, size_t count) {
        void* q = nullptr;
        if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(**p)) != cudaSuccess) return false;
        s->owned.push_back(q);
        *p = static_cast<std::remove_reference_t<decltype(*p)>>(q);
        return true;
    };
    bool ok = take(&s->d_ev, ev.size()) && take(&s->d_P, size_t(v.n) * 16) && take(&s->d_pi, 4) &&
              take(&s->d_site, size_t(std::max(t.P, 1))) && take(&s->d_lnl, 1) &&
              cudaMallocHost(reinterpret_cast<void**>(&s->h_pin), sizeof(double)) == cudaSuccess &&
              cudaMemcpy(s->d_ev, ev.data(), ev.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok && s->levels)
        ok = take(&s->d_lv, lv.size()) && take(&s->d_part, size_t(t.NI) * s->Pp) && take(&s->d_pexp, size_t(t.NI) * s->Pp) &&
             cudaMemcpy(s->d_lv, lv.data(), lv.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
    else if (ok)
        ok = take(&s->d_stk, size_t(deepest) * s->Pp) && take(&s->d_exp, size_t(deepest) * s->Pp);
    // the copies above come from pageable memory on the default stream, which the evaluator's
    // non-blocking stream does not wait for
    ok = ok && cudaStreamSynchronize(cudaStreamLegacy) == cudaSuccess;
    if (!ok) {
        *err = "device allocation failed";
        delete s;
        return nullptr;
    }
    slot = s;
    return s;
}

}  // namespace

void nuc_state_free(void* p) { delete static_cast<NucState*>(p); }

}  // namespace h3g

using namespace h3g;

extern "C" h3g_status h3g_nuc_eval_from_P(h3g_problem* pr, const double* P, const double* pi, double* lnl, double* site_lnl) {
    if (!pr) return H3G_ERR_ARG;
    FelProblemView v;
    if (!P || !pi || !lnl || !fel_problem_view(pr, &v)) { fel_set_error(pr, "h3g_nuc_eval_from_P: null argument"); return H3G_ERR_ARG; }
    if (problem_max_state(pr) >= 4) {
        fel_set_error(pr, "h3g_nuc_eval_from_P: the problem's patterns are not nucleotide patterns (a state is >= 4)");
        return H3G_ERR_ARG;
    }
    for (int i = 0; i < 4; ++i)
        if (!std::isfinite(pi[i]) || pi[i] < 0.0) { fel_set_error(pr, "h3g_nuc_eval_from_P: pi must be finite and >= 0"); return H3G_ERR_NUMERIC; }
    for (int b = 0; b < v.n; ++b)
        for (int e = 0; e < 16 && b != v.root; ++e)
            if (!std::isfinite(P[size_t(b) * 16 + e])) { fel_set_error(pr, "h3g_nuc_eval_from_P: non-finite transition matrix"); return H3G_ERR_NUMERIC; }
    std::string err;
    NucState* s = nuc_state(pr, v, &err);
    if (!s) { fel_set_error(pr, "h3g_nuc_eval_from_P: " + err); return H3G_ERR_OOM; }
    cudaStream_t st = problem_stream(pr);
    const Topo t = problem_topo(pr, 4);
    bool ok = cudaMemcpyAsync(s->d_P, P, size_t(v.n) * 16 * sizeof(double), cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(s->d_pi, pi, 4 * sizeof(double), cudaMemcpyHostToDevice, st) == cudaSuccess;
    if (ok && s->P > 0) {
        if (s->levels) {
            for (size_t k = 0; k + 1 < s->lv_off.size(); ++k) {
                const int cnt = s->lv_off[k + 1] - s->lv_off[k];
                if (cnt == 0) continue;
                launch_k(k_nuc_level, int((size_t(cnt) * size_t(s->P) + kLvlT - 1) / kLvlT), kLvlT, 0, st, t,
                         static_cast<const int*>(s->d_lv + s->lv_off[k]), cnt, static_cast<const double*>(s->d_P),
                         static_cast<const double*>(s->d_pi), s->d_part, s->d_pexp, s->d_site);
            }
        } else {
            launch_k(k_nuc_lnl, (s->P + kNucT - 1) / kNucT, kNucT, 0, st, t, static_cast<const int*>(s->d_ev), s->n_ev,
                     static_cast<const double*>(s->d_P), static_cast<const double*>(s->d_pi), s->d_stk, s->d_exp, s->d_site);
        }
        launch_k(k_nuc_sum, 1, kSumT, 0, st, static_cast<const double*>(s->d_site), t.w, s->P, s->d_lnl);
    }
    ok = ok && cudaGetLastError() == cudaSuccess &&
         cudaMemcpyAsync(s->h_pin, s->d_lnl, sizeof(double), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
         (!site_lnl || s->P == 0 ||
          cudaMemcpyAsync(site_lnl, s->d_site, size_t(s->P) * sizeof(double), cudaMemcpyDeviceToHost, st) == cudaSuccess) &&
         cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) { fel_set_error(pr, std::string("h3g_nuc_eval_from_P: ") + cudaGetErrorString(cudaGetLastError())); return H3G_ERR_CUDA; }
    *lnl = s->P > 0 ? *s->h_pin : 0.0;
    return H3G_OK;
}
