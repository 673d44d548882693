// h3g_fel_driver.cpp — h3g_fel_run / h3g_fel_run_tested: FEL per-site fits with
// every pattern's optimiser advanced in lockstep.
//
// Each pattern runs the reference's search (analyses/fel.hpp:326-446 with
// every branch tested; optimisers from opt/nelder_mead.hpp:24-229) written as
// a C++20 coroutine (h3g_sitefit.h): every likelihood evaluation is a
// co_await that parks the pattern with its requested (alpha, beta); the
// lockstep loop evaluates the parked requests of all patterns in one device
// batch (h3g_fel.cu) and resumes them.  The search path of a pattern is
// therefore exactly the reference's; only the likelihood evaluations are
// batched.
//
// Eigensystems: a pattern keeps its current eigensystem while
// |omega - cached omega| <= 1e-12 (the reference's per-pattern cache,
// fel.hpp:368-376).  An omega requested by several patterns in the same batch
// (the shared start grid, the null model's omega = 1) is diagonalised once
// into a shared slot.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "h3g_sitefit.h"

namespace h3g::sitefit {
namespace {

// co_await Lnl{site, alpha, beta}: FEL's likelihood at (alpha, beta): time scale
// alpha, omega = beta / alpha
struct Lnl {
    Site& s;
    double a, b;
    Eval ev() const {
        const double as = std::max(a, 1e-12);
        return Eval{s, Req{as, b / as, -1.0, 1.0, 0.0}};
    }
};
inline Eval operator co_await(const Lnl& l) { return l.ev(); }

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

}  // namespace

// The reference's per-pattern search, one likelihood per co_await.
Fit fel_search(Site& s, h3g_fel_result& res) {
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
        res.alpha = v[0].a;
        res.beta = v[0].b;
        res.log_l_alt = -v[0].f;
    }
    // null model alpha = beta: start grid, then Brent on [1e-4, 50] (fel.hpp:415-434)
    const double init_null = (std::min(res.alpha, 100.0) + 3.0 * std::min(res.beta, 100.0)) / 4.0;
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
        res.alpha_null = x;
        res.log_l_null = -fx;
    }
    double lrt = 0.0;
    if (res.log_l_alt > -1e10 && res.log_l_null > -1e10) lrt = std::max(0.0, 2.0 * (res.log_l_alt - res.log_l_null));
    res.lrt = lrt;
    res.p_value = std::erfc(std::sqrt(lrt / 2.0));
    res.evaluations = s.evaluations;
}

namespace {

// (alpha, beta on the tested branches, beta_bg on the background) -> request: time scale alpha,
// omega beta / alpha, and beta_bg / alpha on the background unless |beta - beta_bg| < 1e-9, when
// every branch uses the tested model (fel.hpp:462-500)
Req subset_req(double a, double bt, double bb) {
    Req r{a, bt / a, -1.0, 1.0, 0.0};
    if (std::fabs(bt - bb) >= 1e-9) r.om_bg = bb / a;
    return r;
}

}  // namespace

// The reference's branch-subset search of one pattern (fel.hpp:462-572).  The
// start grids are evaluated together: each grid point is scored independently
// and the best is picked in the reference's order, so the path is unchanged.
Fit fel_search_subset(Site& s, h3g_fel_result& res) {
    using A3 = Arr<3>;
    using A2 = Arr<2>;
    // 12-point start grid of the alternative model (fel.hpp:518-533)
    static const double g3[12][3] = {{0.01, 0.1, 0.1}, {1.0, 0.1, 0.1}, {1.0, 0.5, 0.5},   {1.0, 1.0, 1.0},
                                     {1.0, 5.0, 5.0},  {10.0, 0.1, 0.1}, {0.01, 0.5, 0.5}, {0.01, 5.0, 5.0},
                                     {10.0, 0.5, 0.5}, {10.0, 1.0, 1.0}, {10.0, 50.0, 50.0}, {100.0, 1.0, 1.0}};
    std::vector<Req> rq;
    for (const auto& g : g3) rq.push_back(subset_req(g[0], g[1], g[2]));
    co_await EvalMany{s, rq};
    double best = -1e20;
    A3 init = {1.0, 1.0, 1.0};
    for (int i = 0; i < 12; ++i)
        if (rq[size_t(i)].lnl > best) {
            best = rq[size_t(i)].lnl;
            init = {g3[i][0], g3[i][1], g3[i][2]};
        }
    // alternative model: bounded 3-D Nelder-Mead on (alpha, beta, beta_bg), tol 1e-4, 100 iterations
    auto make3 = [](const A3& x) { return subset_req(x[0], x[1], x[2]); };
    const Pt<3> alt = co_await nelder_mead_nd<3>(s, make3, init, A3{1e-4, 1e-4, 1e-4}, A3{1000.0, 1000.0, 1000.0}, 1e-4,
                                                 100, {});
    res.alpha = alt.x[0];
    res.beta = alt.x[1];
    res.beta_nuisance = alt.x[2];
    res.log_l_alt = -alt.f;
    // null model beta = alpha, beta_bg free: the initial point, then a 7 x 4 grid (fel.hpp:546-563)
    const double ina = (std::min(res.alpha, 100.0) + 3.0 * std::min(res.beta, 100.0)) / 4.0, inb = res.beta_nuisance;
    std::vector<A2> pts = {{ina, inb}};
    for (double ca : {0.01, 0.1, 0.5, 1.0, 2.0, 5.0, 10.0})
        for (double cb : {inb, 0.1, 1.0, 5.0}) pts.push_back({ca, cb});
    rq.clear();
    for (const auto& x : pts) rq.push_back(subset_req(x[0], x[0], x[1]));
    co_await EvalMany{s, rq};
    double best_null = rq[0].lnl;
    A2 initn = pts[0];
    for (size_t i = 1; i < pts.size(); ++i)
        if (rq[i].lnl > best_null) {
            best_null = rq[i].lnl;
            initn = pts[i];
        }
    // bounded 2-D Nelder-Mead on (alpha, beta_bg), tol 1e-4, 80 iterations
    auto make2 = [](const A2& x) { return subset_req(x[0], x[0], x[1]); };
    const Pt<2> nul = co_await nelder_mead_nd<2>(s, make2, initn, A2{1e-4, 1e-4}, A2{1000.0, 1000.0}, 1e-4, 80, {});
    res.alpha_null = nul.x[0];
    res.log_l_null = -nul.f;
    double lrt = 0.0;
    if (res.log_l_alt > -1e10 && res.log_l_null > -1e10) lrt = std::max(0.0, 2.0 * (res.log_l_alt - res.log_l_null));
    res.lrt = lrt;
    res.p_value = std::erfc(std::sqrt(lrt / 2.0));
    res.evaluations = s.evaluations;
}

h3g_status prepare_site_run(h3g_problem* prob, const h3g_fel_model* m, const double* branch_lengths, const char* who,
                            FelProblemView* pv, std::vector<int>* variable) {
    const std::string w(who);
    FelProblemView& v = *pv;
    if (!m || !branch_lengths || !fel_problem_view(prob, &v)) {
        fel_set_error(prob, w + ": null argument");
        return H3G_ERR_ARG;
    }
    const int S = m->S;
    if (S < 2 || S > 64 || !m->pi || !m->Qs || !m->Qn) {
        fel_set_error(prob, w + ": model needs 2 <= S <= 64, pi, Qs and Qn");
        return H3G_ERR_ARG;
    }
    for (int i = 0; i < S; ++i)
        if (!std::isfinite(m->pi[i]) || m->pi[i] < 0.0) { fel_set_error(prob, w + ": pi must be finite and >= 0"); return H3G_ERR_NUMERIC; }
    for (int e = 0; e < S * S; ++e)
        if (!std::isfinite(m->Qs[e]) || !std::isfinite(m->Qn[e]) || m->Qs[e] < 0.0 || m->Qn[e] < 0.0) {
            if (e / S == e % S) continue;
            fel_set_error(prob, w + ": rates must be finite and >= 0");
            return H3G_ERR_NUMERIC;
        }
    for (int i = 0; i < v.n; ++i)
        if (i != v.root && (!std::isfinite(branch_lengths[i]) || branch_lengths[i] < 0.0)) {
            fel_set_error(prob, w + ": branch lengths must be finite and >= 0");
            return H3G_ERR_NUMERIC;
        }
    if (v.P > 0 && v.T > 0) {
        int max_state = -1;
        for (size_t e = 0; e < size_t(v.P) * v.T; ++e) max_state = std::max<int>(max_state, v.states[e]);
        if (max_state >= S) { fel_set_error(prob, w + ": a pattern state is >= S"); return H3G_ERR_ARG; }
    }
    variable->clear();
    for (int p = 0; p < v.P; ++p) {
        int first = -1;
        bool invariant = true;
        for (int t = 0; t < v.T; ++t) {
            const int st = v.states[size_t(p) * v.T + t];
            if (st < 0) continue;
            if (first < 0) first = st;
            else if (st != first) { invariant = false; break; }
        }
        if (!invariant) variable->push_back(p);
    }
    return H3G_OK;
}

}  // namespace h3g::sitefit

using namespace h3g;
using namespace h3g::sitefit;

static h3g_status fel_run_impl(h3g_problem* prob, const h3g_fel_model* m, const double* branch_lengths,
                               const uint8_t* tested, h3g_fel_result* out, const char* who) {
    if (!prob) return H3G_ERR_ARG;
    const auto t_start = std::chrono::steady_clock::now();
    const std::string w(who);
    try {
        FelProblemView v;
        std::vector<int> variable;
        if (!out) { fel_set_error(prob, w + ": null argument"); return H3G_ERR_ARG; }
        const h3g_status pst = prepare_site_run(prob, m, branch_lengths, who, &v, &variable);
        if (pst != H3G_OK) return pst;
        // fel.hpp:215-227: the branches outside the tested set form the background
        std::vector<uint8_t> background(size_t(v.n), 0);
        bool subset = false;
        if (tested)
            for (int b = 0; b < v.n; ++b)
                if (b != v.root && !tested[b]) { background[size_t(b)] = 1; subset = true; }
        const h3g_fel_result zero{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0, 0.0};
        for (int p = 0; p < v.P; ++p) out[p] = zero;
        const int N = int(variable.size());
        if (N == 0) return H3G_OK;
        const int S = m->S;
        std::string err;
        LockstepOptions opt;
        if (!subset) {
            opt.cache_tol = 1e-12;          // fel.hpp:368-376
            opt.max_requests = N;           // one request per pattern at a time
            opt.temp_slots = 0;
        } else {
            // the reference builds both models afresh for every evaluation; a start grid parks
            // up to 29 requests at once, each with up to two eigensystems
            opt.cache_tol = 0.0;
            opt.components = 3;
            opt.max_requests = std::max({64, N, std::min(8 * N, 16384)});
            opt.temp_slots = std::min(2 * opt.max_requests, 32768);
            opt.spec_threshold = 32;
        }
        FelDevice* dev = fel_device_create(prob, S, m->pi, m->Qs, m->Qn, branch_lengths, subset ? background.data() : nullptr,
                                           opt.max_requests, slots_needed(N, opt.temp_slots, opt.components), &err);
        if (!dev) { fel_set_error(prob, w + ": " + err); return H3G_ERR_CUDA; }
        std::vector<Site> sites(N);
        std::vector<h3g_fel_result> res(N, zero);
        std::vector<Fit> fits;
        fits.reserve(N);
        for (int i = 0; i < N; ++i) {
            sites[i].pattern = variable[i];
            fits.push_back(subset ? fel_search_subset(sites[i], res[i]) : fel_search(sites[i], res[i]));
        }
        LockstepState state;
        const h3g_status st = run_lockstep(dev, sites, fits, opt, state, &err);
        size_t h2d = 0, d2h = 0;
        int launches = 0;
        fel_device_transfer(dev, &h2d, &d2h, &launches);
        fel_device_destroy(dev);
        if (st != H3G_OK) { fel_set_error(prob, w + ": " + err); return st; }
        // the run's own inputs and outputs: model, branch lengths, background flags, per-pattern results
        fel_record_transfer(prob, h2d + (2 * size_t(S) * S + S + v.n) * sizeof(double) + size_t(v.n), d2h, launches,
                            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count());
        for (int i = 0; i < N; ++i) out[variable[i]] = res[i];
        return H3G_OK;
    } catch (const std::bad_alloc&) {
        fel_set_error(prob, w + ": host allocation failed");
        return H3G_ERR_OOM;
    } catch (const std::exception& e) {
        fel_set_error(prob, w + ": " + e.what());
        return H3G_ERR_ARG;
    }
}

extern "C" h3g_status h3g_fel_run(h3g_problem* prob, const h3g_fel_model* m, const double* branch_lengths,
                                  h3g_fel_result* out) {
    return fel_run_impl(prob, m, branch_lengths, nullptr, out, "h3g_fel_run");
}

extern "C" h3g_status h3g_fel_run_tested(h3g_problem* prob, const h3g_fel_model* m, const double* branch_lengths,
                                         const uint8_t* tested, h3g_fel_result* out) {
    if (prob && !tested) {
        fel_set_error(prob, "h3g_fel_run_tested: null argument");
        return H3G_ERR_ARG;
    }
    return fel_run_impl(prob, m, branch_lengths, tested, out, "h3g_fel_run_tested");
}
