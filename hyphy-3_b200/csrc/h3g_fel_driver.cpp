// h3g_fel_driver.cpp — h3g_fel_run: FEL per-site fits with every pattern's
// optimiser advanced in lockstep.
//
// Each pattern runs the reference's search (analyses/fel.hpp:326-446 with
// every branch tested; optimisers from opt/nelder_mead.hpp:24-229) written as
// a C++20 coroutine: every likelihood evaluation is a co_await that parks the
// pattern with its requested (alpha, beta).  The driver gathers the parked
// requests of all patterns, evaluates them in one device batch
// (h3g_fel.cu), hands each pattern its log-likelihood and resumes it.  The
// search path of a pattern is therefore exactly the reference's; only the
// likelihood evaluations are batched.
//
// Eigensystems: a pattern keeps its current eigensystem while
// |omega - cached omega| <= 1e-12 (the reference's per-pattern cache,
// fel.hpp:368-376).  An omega requested by several patterns in the same batch
// (the shared start grid, the null model's omega = 1) is diagonalised once
// into a shared slot.
#include <algorithm>
#include <cmath>
#include <coroutine>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "h3g_fel.h"

namespace h3g {
namespace {

constexpr int kSharedSlots = 64;

struct Site {
    int pattern = 0;
    bool pending = false;
    double a = 0.0, b = 0.0, lnl = 0.0;
    double cached_omega = -1.0;
    int slot = -1;
    h3g_fel_result res{};
};

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

// co_await Lnl{site, a, b}: log-likelihood of the site's pattern at (a, b)
struct Lnl {
    Site& s;
    double a, b;
    bool await_ready() const noexcept { return false; }
    void await_suspend(std::coroutine_handle<>) noexcept { s.pending = true; s.a = a; s.b = b; }
    double await_resume() const noexcept { ++s.res.evaluations; return s.lnl; }
};

struct Vertex { double a, b, f; };

// stable order of three simplex vertices by f (std::sort on three elements in libstdc++)
void sort3(Vertex (&v)[3]) {
    for (int i = 1; i < 3; ++i) {
        Vertex x = v[i];
        int j = i;
        while (j > 0 && x.f < v[j - 1].f) { v[j] = v[j - 1]; --j; }
        v[j] = x;
    }
}

// The reference's per-pattern search, one likelihood per co_await.
Fit fit_pattern(Site& s) {
    // 12-point start grid (fel.hpp:385-401)
    static const double grid[12][2] = {{0.01, 0.1}, {1.0, 0.1}, {1.0, 0.5}, {1.0, 1.0}, {1.0, 5.0}, {10.0, 0.1},
                                       {0.01, 0.5}, {0.01, 5.0}, {10.0, 0.5}, {10.0, 1.0}, {10.0, 50.0}, {100.0, 1.0}};
    double best = -1e20, ba = 1.0, bb = 1.0;
    for (const auto& g : grid) {
        const double l = co_await Lnl{s, g[0], g[1]};
        if (l > best) { best = l; ba = g[0]; bb = g[1]; }
    }
    // alternative model: bounded Nelder-Mead on (alpha, beta), minimising -lnL
    // (NelderMead2D::minimize, lb 1e-4, ub 1000, tol 1e-4, 100 iterations)
    {
        const double lb = 1e-4, ub = 1000.0, tol = 1e-4;
        const int max_iter = 100;
        auto cl = [&](double x) { return std::clamp(x, lb, ub); };
#define H3G_NM_EVAL(dst, A_, B_)                                           \
    do {                                                                   \
        const double ca_ = cl(A_), cb_ = cl(B_);                           \
        const double l_ = co_await Lnl{s, ca_, cb_};                       \
        dst = Vertex{ca_, cb_, -l_};                                       \
    } while (0)
        const double step_a = std::max(0.1, 0.2 * ba), step_b = std::max(0.1, 0.2 * bb);
        Vertex v[3];
        H3G_NM_EVAL(v[0], ba, bb);
        H3G_NM_EVAL(v[1], ba + step_a, bb);
        H3G_NM_EVAL(v[2], ba, bb + step_b);
        const double alpha = 1.0, gamma = 2.0, rho = 0.5, sigma = 0.5;
        for (int iter = 0; iter < max_iter; ++iter) {
            sort3(v);
            if (std::fabs(v[2].f - v[0].f) < tol && std::fabs(v[2].a - v[0].a) < tol && std::fabs(v[2].b - v[0].b) < tol) break;
            const double c_a = 0.5 * (v[0].a + v[1].a), c_b = 0.5 * (v[0].b + v[1].b);
            Vertex r;
            H3G_NM_EVAL(r, c_a + alpha * (c_a - v[2].a), c_b + alpha * (c_b - v[2].b));
            if (r.f < v[0].f) {
                Vertex e;
                H3G_NM_EVAL(e, c_a + gamma * (r.a - c_a), c_b + gamma * (r.b - c_b));
                v[2] = (e.f < r.f) ? e : r;
            } else if (r.f < v[1].f) {
                v[2] = r;
            } else {
                const bool outside = r.f < v[2].f;
                Vertex c;
                if (outside) H3G_NM_EVAL(c, c_a + rho * (r.a - c_a), c_b + rho * (r.b - c_b));
                else H3G_NM_EVAL(c, c_a + rho * (v[2].a - c_a), c_b + rho * (v[2].b - c_b));
                const double ref_f = outside ? r.f : v[2].f;
                if (c.f < ref_f) {
                    v[2] = c;
                } else {
                    H3G_NM_EVAL(v[1], v[0].a + sigma * (v[1].a - v[0].a), v[0].b + sigma * (v[1].b - v[0].b));
                    H3G_NM_EVAL(v[2], v[0].a + sigma * (v[2].a - v[0].a), v[0].b + sigma * (v[2].b - v[0].b));
                }
            }
        }
#undef H3G_NM_EVAL
        sort3(v);
        s.res.alpha = v[0].a;
        s.res.beta = v[0].b;
        s.res.log_l_alt = -v[0].f;
    }
    // null model alpha = beta: start grid, then Brent on [1e-4, 50] (fel.hpp:415-434)
    const double init_null = (std::min(s.res.alpha, 100.0) + 3.0 * std::min(s.res.beta, 100.0)) / 4.0;
    double best_null = co_await Lnl{s, init_null, init_null}, best_na = init_null;
    for (double c : {0.01, 0.1, 0.5, 1.0, 2.0, 5.0, 10.0}) {
        const double l = co_await Lnl{s, c, c};
        if (l > best_null) { best_null = l; best_na = c; }
    }
    {
        // Brent1D::minimize_point(f = -lnL(x, x), 1e-4, clamp(best, 0.01, 45), 50, tol 1e-4, 60 iterations)
        const double CGOLD = 0.3819660, ZEPS = 1e-10, tol = 1e-4;
        const int max_iter = 60;
        double a = 1e-4, b = 50.0;
        double x = std::clamp(best_na, 0.01, 45.0), w = x, v = x, e = 0.0;
        double fx = -(co_await Lnl{s, x, x});
        double fv = fx, fw = fx;
        for (int iter = 0; iter < max_iter; ++iter) {
            const double xm = 0.5 * (a + b), tol1 = tol * std::fabs(x) + ZEPS, tol2 = 2.0 * tol1;
            if (std::fabs(x - xm) <= (tol2 - 0.5 * (b - a))) break;
            double d = 0.0;
            if (std::fabs(e) > tol1) {
                double r = (x - w) * (fx - fv), q = (x - v) * (fx - fw), pp = (x - v) * q - (x - w) * r;
                q = 2.0 * (q - r);
                if (q > 0.0) pp = -pp;
                q = std::fabs(q);
                const double etemp = e;
                e = d;
                if (std::fabs(pp) >= std::fabs(0.5 * q * etemp) || pp <= q * (a - x) || pp >= q * (b - x)) {
                    e = (x >= xm) ? a - x : b - x;
                    d = CGOLD * e;
                } else {
                    d = pp / q;
                    const double u = x + d;
                    if (u - a < tol2 || b - u < tol2) d = (xm - x >= 0.0) ? std::fabs(tol1) : -std::fabs(tol1);
                }
            } else {
                e = (x >= xm) ? a - x : b - x;
                d = CGOLD * e;
            }
            const double u = (std::fabs(d) >= tol1) ? x + d : x + ((d >= 0.0) ? std::fabs(tol1) : -std::fabs(tol1));
            const double fu = -(co_await Lnl{s, u, u});
            if (fu <= fx) {
                if (u >= x) a = x; else b = x;
                v = w; fv = fw; w = x; fw = fx; x = u; fx = fu;
            } else {
                if (u < x) a = u; else b = u;
                if (fu <= fw || w == x) { v = w; fv = fw; w = u; fw = fu; }
                else if (fu <= fv || v == x || v == w) { v = u; fv = fu; }
            }
        }
        s.res.alpha_null = x;
        s.res.log_l_null = -fx;
    }
    double lrt = 0.0;
    if (s.res.log_l_alt > -1e10 && s.res.log_l_null > -1e10) lrt = std::max(0.0, 2.0 * (s.res.log_l_alt - s.res.log_l_null));
    s.res.lrt = lrt;
    s.res.p_value = std::erfc(std::sqrt(lrt / 2.0));
}

uint64_t bits_of(double x) {
    uint64_t u;
    std::memcpy(&u, &x, sizeof u);
    return u;
}

}  // namespace
}  // namespace h3g

using namespace h3g;

extern "C" h3g_status h3g_fel_run(h3g_problem* prob, const h3g_fel_model* m, const double* branch_lengths,
                                  h3g_fel_result* out) {
    if (!prob) return H3G_ERR_ARG;
    try {
        FelProblemView v;
        if (!m || !branch_lengths || !out || !fel_problem_view(prob, &v)) {
            fel_set_error(prob, "h3g_fel_run: null argument");
            return H3G_ERR_ARG;
        }
        const int S = m->S;
        if (S < 2 || S > 64 || !m->pi || !m->Qs || !m->Qn) {
            fel_set_error(prob, "h3g_fel_run: model needs 2 <= S <= 64, pi, Qs and Qn");
            return H3G_ERR_ARG;
        }
        for (int i = 0; i < S; ++i)
            if (!std::isfinite(m->pi[i]) || m->pi[i] < 0.0) { fel_set_error(prob, "h3g_fel_run: pi must be finite and >= 0"); return H3G_ERR_NUMERIC; }
        for (int e = 0; e < S * S; ++e)
            if (!std::isfinite(m->Qs[e]) || !std::isfinite(m->Qn[e]) || m->Qs[e] < 0.0 || m->Qn[e] < 0.0) {
                if (e / S == e % S) continue;
                fel_set_error(prob, "h3g_fel_run: rates must be finite and >= 0");
                return H3G_ERR_NUMERIC;
            }
        for (int i = 0; i < v.n; ++i)
            if (i != v.root && (!std::isfinite(branch_lengths[i]) || branch_lengths[i] < 0.0)) {
                fel_set_error(prob, "h3g_fel_run: branch lengths must be finite and >= 0");
                return H3G_ERR_NUMERIC;
            }
        if (v.P > 0 && v.T > 0) {
            int max_state = -1;
            for (size_t e = 0; e < size_t(v.P) * v.T; ++e) max_state = std::max<int>(max_state, v.states[e]);
            if (max_state >= S) { fel_set_error(prob, "h3g_fel_run: a pattern state is >= S"); return H3G_ERR_ARG; }
        }
        // invariant patterns (all resolved states equal) are not fitted (fel.hpp:333-356)
        std::vector<Site> sites;
        sites.reserve(v.P);
        for (int p = 0; p < v.P; ++p) {
            out[p] = h3g_fel_result{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0};
            int first = -1;
            bool invariant = true;
            for (int t = 0; t < v.T; ++t) {
                const int st = v.states[size_t(p) * v.T + t];
                if (st < 0) continue;
                if (first < 0) first = st;
                else if (st != first) { invariant = false; break; }
            }
            if (!invariant) {
                Site s;
                s.pattern = p;
                sites.push_back(s);
            }
        }
        const int N = int(sites.size());
        if (N == 0) return H3G_OK;
        std::string err;
        FelDevice* dev = fel_device_create(prob, S, m->pi, m->Qs, m->Qn, branch_lengths, N, kSharedSlots + N, &err);
        if (!dev) { fel_set_error(prob, "h3g_fel_run: " + err); return H3G_ERR_CUDA; }
        std::vector<Fit> fits;
        fits.reserve(N);
        for (auto& s : sites) fits.push_back(fit_pattern(s));
        for (auto& f : fits) f.h.resume();                 // run to the first evaluation
        std::unordered_map<uint64_t, int> shared;          // omega bits -> shared slot
        std::vector<int> req_site, req_pat, req_slot, eig_slot, eig_prev;
        std::vector<double> req_a, eig_om, lnl;
        std::unordered_map<uint64_t, int> count;
        h3g_status st = H3G_OK;
        while (st == H3G_OK) {
            req_site.clear(); req_pat.clear(); req_slot.clear(); req_a.clear(); eig_slot.clear(); eig_om.clear();
            eig_prev.clear();
            count.clear();
            for (int i = 0; i < N; ++i) {
                if (!sites[i].pending) continue;
                req_site.push_back(i);
                Site& s = sites[i];
                const double om = s.b / std::max(s.a, 1e-12);
                if (!(s.slot >= 0 && std::fabs(om - s.cached_omega) <= 1e-12)) ++count[bits_of(om)];
            }
            if (req_site.empty()) break;
            for (int i : req_site) {
                Site& s = sites[i];
                const double as = std::max(s.a, 1e-12), om = s.b / as;
                if (!(s.slot >= 0 && std::fabs(om - s.cached_omega) <= 1e-12)) {
                    s.cached_omega = om;
                    const uint64_t key = bits_of(om);
                    auto it = shared.find(key);
                    if (it != shared.end()) {
                        s.slot = it->second;
                    } else if (count[key] >= 2 && int(shared.size()) < kSharedSlots) {
                        const int slot = int(shared.size());
                        shared.emplace(key, slot);
                        eig_om.push_back(om);
                        eig_slot.push_back(slot);
                        s.slot = slot;
                    } else {
                        eig_prev.resize(eig_slot.size(), -1);
                        eig_prev.push_back(s.slot);        // warm start from the pattern's last eigensystem
                        s.slot = kSharedSlots + i;
                        eig_om.push_back(om);
                        eig_slot.push_back(s.slot);
                    }
                }
                req_pat.push_back(s.pattern);
                req_a.push_back(as);
                req_slot.push_back(s.slot);
            }
            lnl.assign(req_site.size(), 0.0);
            eig_prev.resize(eig_slot.size(), -1);          // new shared slots start from the identity
            if (!fel_device_eval(dev, int(eig_om.size()), eig_om.data(), eig_slot.data(), eig_prev.data(), int(req_site.size()), req_pat.data(),
                                 req_a.data(), req_slot.data(), lnl.data(), &err)) {
                fel_set_error(prob, "h3g_fel_run: " + err);
                st = H3G_ERR_CUDA;
                break;
            }
            for (size_t r = 0; r < req_site.size(); ++r) {
                Site& s = sites[req_site[r]];
                s.lnl = lnl[r];
                s.pending = false;
                fits[req_site[r]].h.resume();
                if (fits[req_site[r]].h.promise().error) {
                    fel_set_error(prob, "h3g_fel_run: optimiser failed");
                    st = H3G_ERR_NUMERIC;
                    break;
                }
            }
        }
        size_t h2d = 0, d2h = 0;
        fel_device_transfer(dev, &h2d, &d2h);
        fel_device_destroy(dev);
        if (st != H3G_OK) return st;
        // the run's own inputs and outputs: model, branch lengths, per-pattern results
        fel_record_transfer(prob, h2d + (2 * size_t(S) * S + S + v.n) * sizeof(double), d2h);
        for (int i = 0; i < N; ++i) {
            if (!fits[i].h.done()) { fel_set_error(prob, "h3g_fel_run: a pattern did not finish"); return H3G_ERR_STATE; }
            out[sites[i].pattern] = sites[i].res;
        }
        return H3G_OK;
    } catch (const std::bad_alloc&) {
        fel_set_error(prob, "h3g_fel_run: host allocation failed");
        return H3G_ERR_OOM;
    } catch (const std::exception& e) {
        fel_set_error(prob, std::string("h3g_fel_run: ") + e.what());
        return H3G_ERR_ARG;
    }
}
