// h3g_sitefit.h — per-pattern optimisers of the site-level analyses (FEL,
// MEME) as C++20 coroutines, advanced in lockstep over device batches.
//
// Each pattern's search is the reference's sequential code, with every
// likelihood evaluation a co_await that parks the pattern and its request(s).
// run_lockstep() gathers the parked requests of all patterns, evaluates them
// in one device batch (h3g_fel.cu) and resumes every pattern.  A search may
// park several independent requests at once (EvalMany: a start grid, the
// vertices of a new simplex); they are evaluated together and the search
// reads the results in order, so its path is the same as one request at a
// time.  Nested searches (one Nelder-Mead inside a site's fit) are Task<T>
// coroutines that resume their caller by symmetric transfer.
//
// Plain host C++20, no device code.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <coroutine>
#include <cstdint>
#include <exception>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "h3g_fel.h"

namespace h3g::sitefit {

// One likelihood request: the pattern's log-likelihood at time scale a with
// omega om1, or, when om2 >= 0, with omegas (om1, om2) mixed at the
// transition-matrix level with weights (w1, 1 - w1).  When om_bg >= 0 the
// run's background branches use omega om_bg alone.  Components: 0 = om1,
// 1 = om2, 2 = om_bg.
struct Req {
    double a = 1.0, om1 = 0.0, om2 = -1.0, w1 = 1.0;
    double lnl = 0.0;
    double om_bg = -1.0;
};
inline double req_omega(const Req& r, int c) { return c == 0 ? r.om1 : c == 1 ? r.om2 : r.om_bg; }
inline bool req_has(const Req& r, int c) { return c == 0 || req_omega(r, c) >= 0.0; }

struct Site {
    int pattern = 0;
    std::vector<Req> one;                   // storage of a single request
    std::vector<Req>* pending = nullptr;    // requests parked at the current co_await
    std::coroutine_handle<> resume;         // innermost coroutine waiting on them
    int slot[3] = {-1, -1, -1};             // eigensystem last used per component (cache, warm starts)
    double cached[3] = {-1.0, -1.0, -1.0};
    int buf[3] = {0, 0, 0};                 // which of the site's two own slots per component is current
    int evaluations = 0;
    bool speculate = false;                 // the last batch was small: a search may evaluate its next
                                            // candidates together (results are unchanged)
};

// Top-level coroutine of one pattern; the driver owns and destroys it.
struct Fit {
    struct promise_type {
        std::exception_ptr error;
        Fit get_return_object() { return Fit{std::coroutine_handle<promise_type>::from_promise(*this)}; }
        std::suspend_always initial_suspend() noexcept { return {}; }
        std::suspend_always final_suspend() noexcept { return {}; }
        void return_void() {}
        void unhandled_exception() { error = std::current_exception(); }
    };
    std::coroutine_handle<promise_type> h;
    explicit Fit(std::coroutine_handle<promise_type> hh) : h(hh) {}
    Fit(Fit&& o) noexcept : h(std::exchange(o.h, {})) {}
    Fit& operator=(Fit&&) = delete;
    ~Fit() { if (h) h.destroy(); }
};

// A nested search returning T; `co_await task` runs it and resumes the caller when it returns.
template <class T>
struct Task {
    struct promise_type {
        T value{};
        std::exception_ptr error;
        std::coroutine_handle<> caller;
        Task get_return_object() { return Task{std::coroutine_handle<promise_type>::from_promise(*this)}; }
        std::suspend_always initial_suspend() noexcept { return {}; }
        struct Final {
            bool await_ready() noexcept { return false; }
            std::coroutine_handle<> await_suspend(std::coroutine_handle<promise_type> h) noexcept {
                return h.promise().caller ? h.promise().caller : std::noop_coroutine();
            }
            void await_resume() noexcept {}
        };
        Final final_suspend() noexcept { return {}; }
        void return_value(T v) { value = std::move(v); }
        void unhandled_exception() { error = std::current_exception(); }
    };
    std::coroutine_handle<promise_type> h;
    explicit Task(std::coroutine_handle<promise_type> hh) : h(hh) {}
    Task(Task&& o) noexcept : h(std::exchange(o.h, {})) {}
    Task& operator=(Task&&) = delete;
    ~Task() { if (h) h.destroy(); }
    bool await_ready() const noexcept { return false; }
    std::coroutine_handle<> await_suspend(std::coroutine_handle<> caller) noexcept {
        h.promise().caller = caller;
        return h;
    }
    T await_resume() {
        if (h.promise().error) std::rethrow_exception(h.promise().error);
        return std::move(h.promise().value);
    }
};

// co_await Eval{site, request}: one log-likelihood
struct Eval {
    Site& s;
    Req r;
    bool await_ready() const noexcept { return false; }
    void await_suspend(std::coroutine_handle<> h) {
        s.one.assign(1, r);
        s.pending = &s.one;
        s.resume = h;
    }
    double await_resume() noexcept { ++s.evaluations; return s.one[0].lnl; }
};

// co_await EvalMany{site, reqs}: independent requests evaluated together, results in reqs[i].lnl
struct EvalMany {
    Site& s;
    std::vector<Req>& reqs;
    bool await_ready() const noexcept { return reqs.empty(); }
    void await_suspend(std::coroutine_handle<> h) noexcept {
        s.pending = &reqs;
        s.resume = h;
    }
    void await_resume() noexcept { s.evaluations += int(reqs.size()); }
};

// Eigensystem slot layout of a run with C components per request: [0,
// kSharedSlots) omegas requested by several patterns in one batch (kept for
// the run), then 2 C slots per site (two buffers per component: a single
// request is solved in place in the current one, the first request of a
// multi-request batch into the other, which then becomes current), then a
// pool for the remaining requests of multi-request sites (reused every
// batch).  Every solve is warm-started from the site's current eigensystem.
constexpr int kSharedSlots = 64;
inline int own_slot(int site, int buf, int c, int comps) { return kSharedSlots + 2 * comps * site + comps * buf + c; }
inline int slots_needed(int n_sites, int temp_slots, int comps) { return kSharedSlots + 2 * comps * n_sites + temp_slots; }

struct LockstepOptions {
    double cache_tol = 0.0;     // a site reuses its eigensystem while |omega - cached| <= cache_tol
    int max_requests = 1;       // per device batch (the device was created with this many)
    int temp_slots = 0;         // pool size for multi-request sites
    int spec_threshold = 0;     // batches of at most this many requests set Site::speculate
    int components = 2;         // components a request may use (2: om1, om2; 3: and om_bg)
};

// What a run's slots hold across its lockstep phases (FEL then MEME on the
// same device and sites): the shared omegas, and which slots were solved in
// which batch.  Sites keep their cached slots from one phase to the next, so
// a shared slot must keep its omega for the whole run.
struct LockstepState {
    std::unordered_map<uint64_t, int> shared;          // omega bits -> shared slot
    std::vector<int> written;                          // batch that last solved each slot
    std::vector<char> solved;
    int batch = 0;
};

// Resume every fit until all have finished.  Returns H3G_OK, or H3G_ERR_CUDA /
// H3G_ERR_NUMERIC / H3G_ERR_STATE with *err set.
h3g_status run_lockstep(FelDevice* dev, std::vector<Site>& sites, std::vector<Fit>& fits, const LockstepOptions& opt,
                        LockstepState& state, std::string* err);

uint64_t bits_of(double x);

// Shared argument checks of h3g_fel_run / h3g_meme_run; fills the problem view
// and the patterns that are fitted (invariant patterns are not, fel.hpp:333-356,
// meme.hpp:190-216).  On failure records the message and returns the status.
h3g_status prepare_site_run(h3g_problem* prob, const h3g_fel_model* m, const double* branch_lengths, const char* who,
                            FelProblemView* v, std::vector<int>* variable_patterns);

// The reference's FEL search of one pattern (fel.hpp:326-446, every branch tested).
Fit fel_search(Site& s, h3g_fel_result& res);
// Its branch-subset search (fel.hpp:462-572): requests carry om_bg (component 2)
// for the background branches, so the run needs LockstepOptions::components = 3.
Fit fel_search_subset(Site& s, h3g_fel_result& res);

template <int D>
using Arr = std::array<double, D>;

template <int D>
struct Pt {
    Arr<D> x{};
    double f = 0.0;
};

// opt/nelder_mead.hpp:209-357, minimising -lnL: the best of the start point and
// the grid seeds a simplex of D perturbed vertices; reflection 1, expansion 2,
// contraction 0.5, shrink 0.5; stops when the f-spread and the coordinate
// spread between the best and worst vertex are both below tol.  Independent
// evaluations (start + grid, the first simplex, a shrink) are parked together.
// make(x) turns a point into its likelihood request.
template <int D, class Make>
Task<Pt<D>> nelder_mead_nd(Site& s, Make make, Arr<D> init, Arr<D> lb, Arr<D> ub, double tol, int max_iter,
                           std::vector<Arr<D>> grid) {
    auto clampx = [&](const Arr<D>& v) {
        Arr<D> c;
        for (int d = 0; d < D; ++d) c[d] = std::clamp(v[d], lb[d], ub[d]);
        return c;
    };
    std::vector<Arr<D>> xs;
    std::vector<Req> rq;
    auto eval_all = [&]() {
        rq.clear();
        for (const auto& x : xs) rq.push_back(make(x));
        return EvalMany{s, rq};
    };
    xs.push_back(clampx(init));
    for (const auto& g : grid) xs.push_back(clampx(g));
    co_await eval_all();
    Pt<D> best{xs[0], -rq[0].lnl};
    for (size_t i = 1; i < xs.size(); ++i)
        if (-rq[i].lnl < best.f) best = Pt<D>{xs[i], -rq[i].lnl};
    std::array<Pt<D>, D + 1> v;
    v[0] = best;
    xs.clear();
    for (int d = 0; d < D; ++d) {
        Arr<D> x = best.x;
        const double step = std::max(0.05, 0.2 * std::fabs(best.x[d]));
        if (best.x[d] + step <= ub[d]) x[d] += step;
        else x[d] -= step;
        xs.push_back(clampx(x));
    }
    co_await eval_all();
    for (int d = 0; d < D; ++d) v[d + 1] = Pt<D>{xs[d], -rq[d].lnl};
    auto by_f = [](const Pt<D>& a, const Pt<D>& b) { return a.f < b.f; };
    auto one = [&](const Arr<D>& x) {
        const Arr<D> c = clampx(x);
        return std::pair<Arr<D>, Req>{c, make(c)};
    };
    for (int iter = 0; iter < max_iter; ++iter) {
        std::sort(v.begin(), v.end(), by_f);
        double dx = 0.0;
        for (int d = 0; d < D; ++d) dx = std::max(dx, std::fabs(v[D].x[d] - v[0].x[d]));
        if (std::fabs(v[D].f - v[0].f) < tol && dx < tol) break;
        Arr<D> c{};
        for (int i = 0; i < D; ++i)
            for (int d = 0; d < D; ++d) c[d] += v[i].x[d];
        for (int d = 0; d < D; ++d) c[d] /= double(D);
        Arr<D> xr;
        for (int d = 0; d < D; ++d) xr[d] = c[d] + 1.0 * (c[d] - v[D].x[d]);
        if (s.speculate) {
            // The step evaluates the reflection r and then at most one of the expansion and the two
            // contractions; all four points are known before r's value, so they are evaluated in one
            // batch and the decisions below are the sequential ones.  Unused values are not counted.
            const Arr<D> xrc = clampx(xr);
            Arr<D> xe, xo, xi;
            for (int d = 0; d < D; ++d) {
                xe[d] = c[d] + 2.0 * (xrc[d] - c[d]);
                xo[d] = c[d] + 0.5 * (xrc[d] - c[d]);
                xi[d] = c[d] + 0.5 * (v[D].x[d] - c[d]);
            }
            xs = {xrc, clampx(xe), clampx(xo), clampx(xi)};
            co_await eval_all();
            const Pt<D> r{xs[0], -rq[0].lnl};
            int used = 1;
            bool shrink = false;
            if (r.f < v[0].f) {
                const Pt<D> e{xs[1], -rq[1].lnl};
                v[D] = (e.f < r.f) ? e : r;
                used = 2;
            } else if (r.f < v[D - 1].f) {
                v[D] = r;
            } else {
                const bool outside = r.f < v[D].f;
                const Pt<D> cc = outside ? Pt<D>{xs[2], -rq[2].lnl} : Pt<D>{xs[3], -rq[3].lnl};
                used = 2;
                if (cc.f < (outside ? r.f : v[D].f)) v[D] = cc;
                else shrink = true;
            }
            s.evaluations -= 4 - used;
            if (shrink) {
                xs.clear();
                for (int i = 1; i <= D; ++i) {
                    Arr<D> x;
                    for (int d = 0; d < D; ++d) x[d] = v[0].x[d] + 0.5 * (v[i].x[d] - v[0].x[d]);
                    xs.push_back(clampx(x));
                }
                co_await eval_all();
                for (int i = 1; i <= D; ++i) v[i] = Pt<D>{xs[i - 1], -rq[i - 1].lnl};
            }
            continue;
        }
        const auto [xrc, rr] = one(xr);
        const Pt<D> r{xrc, -(co_await Eval{s, rr})};
        if (r.f < v[0].f) {
            Arr<D> xe;
            for (int d = 0; d < D; ++d) xe[d] = c[d] + 2.0 * (r.x[d] - c[d]);
            const auto [xec, re] = one(xe);
            const Pt<D> e{xec, -(co_await Eval{s, re})};
            v[D] = (e.f < r.f) ? e : r;
        } else if (r.f < v[D - 1].f) {
            v[D] = r;
        } else {
            const bool outside = r.f < v[D].f;
            Arr<D> xc;
            for (int d = 0; d < D; ++d) xc[d] = c[d] + 0.5 * ((outside ? r.x[d] : v[D].x[d]) - c[d]);
            const auto [xcc, rc] = one(xc);
            const Pt<D> cc{xcc, -(co_await Eval{s, rc})};
            if (cc.f < (outside ? r.f : v[D].f)) {
                v[D] = cc;
            } else {
                xs.clear();
                for (int i = 1; i <= D; ++i) {
                    Arr<D> x;
                    for (int d = 0; d < D; ++d) x[d] = v[0].x[d] + 0.5 * (v[i].x[d] - v[0].x[d]);
                    xs.push_back(clampx(x));
                }
                co_await eval_all();
                for (int i = 1; i <= D; ++i) v[i] = Pt<D>{xs[i - 1], -rq[i - 1].lnl};
            }
        }
    }
    std::sort(v.begin(), v.end(), by_f);
    co_return v[0];
}

}  // namespace h3g::sitefit
