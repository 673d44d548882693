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
// transition-matrix level with weights (w1, 1 - w1).
struct Req {
    double a = 1.0, om1 = 0.0, om2 = -1.0, w1 = 1.0;
    double lnl = 0.0;
};

struct Site {
    int pattern = 0;
    std::vector<Req> one;                   // storage of a single request
    std::vector<Req>* pending = nullptr;    // requests parked at the current co_await
    std::coroutine_handle<> resume;         // innermost coroutine waiting on them
    int slot[2] = {-1, -1};                 // eigensystem last used per component (cache, warm starts)
    double cached[2] = {-1.0, -1.0};
    int buf[2] = {0, 0};                    // which of the site's two own slots per component is current
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

// Eigensystem slot layout of a run: [0, kSharedSlots) omegas requested by
// several patterns in one batch (kept for the run), then four slots per site
// (two buffers per component: a single request is solved in place in the
// current one, the first request of a multi-request batch into the other,
// which then becomes current), then a pool for the remaining requests of
// multi-request sites (reused every batch).  Every solve is warm-started from
// the site's current eigensystem.
constexpr int kSharedSlots = 64;
inline int own_slot(int site, int buf, int c) { return kSharedSlots + 4 * site + 2 * buf + c; }
inline int slots_needed(int n_sites, int temp_slots) { return kSharedSlots + 4 * n_sites + temp_slots; }

struct LockstepOptions {
    double cache_tol = 0.0;     // a site reuses its eigensystem while |omega - cached| <= cache_tol
    int max_requests = 1;       // per device batch (the device was created with this many)
    int temp_slots = 0;         // pool size for multi-request sites
    int spec_threshold = 0;     // batches of at most this many requests set Site::speculate
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

}  // namespace h3g::sitefit
