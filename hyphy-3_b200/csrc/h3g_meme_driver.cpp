// h3g_meme_driver.cpp — h3g_meme_run: MEME per-site fits with every pattern's
// optimisers advanced in lockstep (h3g_sitefit.h).
//
// Per pattern, as analyses/meme.hpp:166-632 with every branch tested:
//   1. the FEL fit of the pattern (the same coroutine as h3g_fel_run);
//   2. the alternative model by the reference's bounded 4-D Nelder-Mead
//      (opt/nelder_mead.hpp:209-357) from its start grid, the null model
//      (beta+ = alpha) by the 3-D one, a warm-started refit, LRT and p-value;
//   3. for the patterns that reach the test, the empirical Bayes factor of
//      every branch from one inside-outside pass on the device (k_meme_ebf).
// A likelihood evaluation needs two eigensystems (omega1 and beta+ / alpha)
// and prunes with their transition matrices mixed (p1, 1 - p1) per branch.
#include <algorithm>
#include <chrono>
#include <array>
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "h3g_sitefit.h"

namespace h3g::sitefit {
namespace {

struct MemeOut {
    h3g_meme_result r{};
    double omega1 = 0.0;      // omega of component 1 at the reported MLE
    bool ebf = false;         // the pattern reached the test: compute its branch EBFs
};

// (alpha, omega1, p1, beta+) -> request: components omega1 and beta+ / alpha, weights (p1, 1 - p1)
Req alt_req(const Arr<4>& x) { return Req{x[0], x[1], x[3] / x[0], x[2], 0.0}; }
// null model: beta+ = alpha
Req null_req(const Arr<3>& x) { return Req{x[0], x[1], x[0] / x[0], x[2], 0.0}; }

// meme.hpp:166-632 with num_background == 0, after the FEL fit
Fit meme_search(Site& s, const h3g_fel_result& fel, MemeOut& out) {
    s.evaluations = 0;
    h3g_meme_result& res = out.r;
    res.fel_alpha = fel.alpha;
    res.fel_beta = fel.beta;
    res.log_l_fel = fel.log_l_alt;
    using A4 = Arr<4>;
    using A3 = Arr<3>;
    // start grid (meme.hpp:282-312)
    const double af = std::clamp(fel.alpha, 1e-4, 10000.0), bf = std::clamp(fel.beta, 1e-4, 100000.0);
    const double w10 = std::clamp(bf / std::max(af, 1e-4), 0.0, 1.0);
    std::vector<A4> grid;
    if (af >= bf) {
        grid = {{af, w10, 0.75, bf}, {af, 0.0, 0.75, bf}, {af, 0.0, 0.95, af * 0.5}, {af, 0.25, 0.85, af * 0.9}};
        const double bp1 = std::max(af * 1.5, bf * 2.0), bp2 = std::max(af * 2.5, bf * 4.0), bp3 = std::max(af * 4.0, bf * 8.0);
        for (double pp : {0.05, 0.10, 0.20}) {
            grid.push_back({af, w10, 1.0 - pp, bp1});
            grid.push_back({af, w10, 1.0 - pp, bp2});
            grid.push_back({af, w10, 1.0 - pp, bp3});
        }
    } else {
        grid = {{af, w10, 0.75, bf}, {af, 0.0, 0.75, bf}, {af, 0.25, 0.50, bf * 2.0}, {af, 0.25, 0.75, bf * 5.0},
                {af, 0.10, 0.90, bf * 15.0}, {af, 0.00, 0.95, bf * 30.0}, {af, 1.00, 0.01, std::max(bf, af * 1.5)}};
    }
    const A4 lb4 = {1e-4, 0.0, 1e-6, 1e-4}, ub4 = {10000.0, 1.0, 1.0 - 1e-6, 100000.0};
    // alternative model (meme.hpp:340-354)
    const Pt<4> alt = co_await nelder_mead_nd<4>(s, alt_req, grid[0], lb4, ub4, 1e-5, 800, grid);
    double omega1 = alt.x[1];
    res.alpha = alt.x[0];
    res.p1 = alt.x[2];
    res.beta_plus = alt.x[3];
    res.beta1 = res.alpha * omega1;
    res.p_plus = 1.0 - res.p1;
    res.log_l_meme = -alt.f;
    if (res.beta_plus > res.alpha && res.p_plus > 1e-6) {
        // null model (meme.hpp:404-435)
        const double an = std::clamp(fel.alpha_null, 1e-4, 50.0);
        std::vector<A3> ng = {{res.alpha, omega1, res.p1}, {an, 1.0, 0.5}, {an, omega1, res.p1},
                              {std::clamp(res.alpha, 1e-4, 50.0), 1.0, 0.5}};
        for (double c : {0.01, 0.1, 0.5, 1.0, 2.0, 5.0, 10.0, 20.0}) {
            ng.push_back({c, 0.5, 0.5});
            ng.push_back({c, 0.0, 0.9});
        }
        const A3 lb3 = {1e-4, 0.0, 1e-6}, ub3 = {10000.0, 1.0, 1.0 - 1e-6};
        const Pt<3> nul = co_await nelder_mead_nd<3>(s, null_req, ng[0], lb3, ub3, 1e-5, 800, ng);
        const double lnl_null = -nul.f, a_null = nul.x[0], w_null = nul.x[1], p_null = nul.x[2];
        if (lnl_null > res.log_l_meme && std::isfinite(lnl_null)) {
            // alternative warm-started from the null MLE (meme.hpp:436-452)
            const std::vector<A4> wg = {{a_null, w_null, p_null, a_null}, {a_null, w_null, 0.99, a_null}};
            const Pt<4> alt2 = co_await nelder_mead_nd<4>(s, alt_req, wg[0], lb4, ub4, 1e-5, 800, wg);
            if (-alt2.f > res.log_l_meme) {
                res.alpha = alt2.x[0];
                omega1 = alt2.x[1];
                res.p1 = alt2.x[2];
                res.beta_plus = alt2.x[3];
                res.beta1 = res.alpha * omega1;
                res.p_plus = 1.0 - res.p1;
                res.log_l_meme = -alt2.f;
            }
        }
        // meme.hpp:456-482
        if (lnl_null <= -1e10 || res.log_l_meme <= -1e10 || !std::isfinite(lnl_null) || !std::isfinite(res.log_l_meme)) {
            res.lrt = 0.0;
            res.p_value = 1.0;
        } else if (lnl_null > res.log_l_meme) {
            res.alpha = a_null;
            res.beta1 = a_null * w_null;
            res.p1 = p_null;
            res.beta_plus = a_null;
            res.p_plus = 1.0 - p_null;
            res.log_l_meme = lnl_null;
            omega1 = w_null;
            res.lrt = 0.0;
            res.p_value = 2.0 / 3.0;
        } else if (std::fabs(res.log_l_meme - lnl_null) <= 1e-12) {
            res.lrt = 0.0;
            res.p_value = 2.0 / 3.0;
        } else {
            res.lrt = 2.0 * (res.log_l_meme - lnl_null);
            res.p_value = (2.0 / 3.0) * (0.45 * std::erfc(std::sqrt(res.lrt / 2.0)) + 0.55 * std::exp(-res.lrt / 2.0));
        }
        out.ebf = true;
    } else {
        res.lrt = 0.0;
        res.p_value = 2.0 / 3.0;
    }
    const double d_fel = 2.0 * (res.log_l_meme - res.log_l_fel);   // meme.hpp:590-597
    res.p_value_meme_vs_fel = d_fel > 0.0 ? std::exp(-d_fel / 2.0) : 1.0;
    out.omega1 = omega1;
    res.evaluations = s.evaluations;
}

}  // namespace
}  // namespace h3g::sitefit

using namespace h3g;
using namespace h3g::sitefit;

extern "C" h3g_status h3g_meme_run(h3g_problem* prob, const h3g_fel_model* m, const double* branch_lengths, h3g_meme_result* out,
                                   double* branch_ebf) {
    if (!prob) return H3G_ERR_ARG;
    const auto t_start = std::chrono::steady_clock::now();
    try {
        FelProblemView v;
        std::vector<int> variable;
        if (!out) { fel_set_error(prob, "h3g_meme_run: null argument"); return H3G_ERR_ARG; }
        const h3g_status pst = prepare_site_run(prob, m, branch_lengths, "h3g_meme_run", &v, &variable);
        if (pst != H3G_OK) return pst;
        const h3g_meme_result zero{0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0};
        for (int p = 0; p < v.P; ++p) out[p] = zero;
        if (branch_ebf) std::fill(branch_ebf, branch_ebf + size_t(v.P) * v.n, 1.0);
        const int N = int(variable.size());
        if (N == 0) return H3G_OK;
        const int S = m->S;
        // mean rate of a site's model is linear in (alpha, beta): alpha mu_s + beta mu_n
        double mu_s = 0.0, mu_n = 0.0, tree_len = 0.0;
        for (int i = 0; i < S; ++i)
            for (int j = 0; j < S; ++j)
                if (j != i) {
                    mu_s += m->pi[i] * m->Qs[i * S + j];
                    mu_n += m->pi[i] * m->Qn[i * S + j];
                }
        for (int b = 0; b < v.n; ++b)
            if (b != v.root) tree_len += branch_lengths[b];
        // a start grid parks up to 21 requests at once; the pool holds two eigensystems per request
        LockstepOptions opt;
        opt.max_requests = std::max({64, N, std::min(8 * N, 16384)});
        opt.temp_slots = std::min(2 * opt.max_requests, 32768);
        opt.spec_threshold = 32;            // four candidates per site still fit one wave of the pruning kernel
        std::string err;
        FelDevice* dev = fel_device_create(prob, S, m->pi, m->Qs, m->Qn, branch_lengths, nullptr, opt.max_requests,
                                           slots_needed(N, opt.temp_slots, opt.components), &err);
        if (!dev) { fel_set_error(prob, "h3g_meme_run: " + err); return H3G_ERR_CUDA; }
        std::vector<Site> sites(N);
        std::vector<h3g_fel_result> fel(N, h3g_fel_result{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0});
        std::vector<MemeOut> mo(N);
        LockstepState state;                // one slot map for both phases: sites keep their slots
        h3g_status st = H3G_OK;
        {
            std::vector<Fit> fits;
            fits.reserve(N);
            for (int i = 0; i < N; ++i) {
                sites[i].pattern = variable[i];
                fits.push_back(fel_search(sites[i], fel[i]));
            }
            opt.cache_tol = 1e-12;          // the FEL baseline keeps FEL's per-pattern cache (fel.hpp:368-376)
            st = run_lockstep(dev, sites, fits, opt, state, &err);
        }
        if (st == H3G_OK) {
            std::vector<Fit> fits;
            fits.reserve(N);
            for (int i = 0; i < N; ++i) fits.push_back(meme_search(sites[i], fel[i], mo[i]));
            opt.cache_tol = 0.0;            // MEME builds its models afresh for every evaluation
            st = run_lockstep(dev, sites, fits, opt, state, &err);
        }
        // empirical Bayes factors at the reported MLE, in chunks
        std::vector<int> todo;
        for (int i = 0; i < N; ++i)
            if (mo[i].ebf) todo.push_back(i);
        const int chunk = fel_device_max_ebf(dev);
        std::vector<double> ebf, eom, ra, rw;
        std::vector<int> eslot, eprev, rpat, rs1, rs2;
        for (size_t k0 = 0; st == H3G_OK && k0 < todo.size(); k0 += size_t(chunk)) {
            const size_t k1 = std::min(todo.size(), k0 + size_t(chunk));
            eom.clear(); eslot.clear(); eprev.clear(); rpat.clear(); ra.clear(); rw.clear(); rs1.clear(); rs2.clear();
            for (size_t k = k0; k < k1; ++k) {
                const int i = todo[k];
                Site& s = sites[i];
                const h3g_meme_result& r = mo[i].r;
                const double om[2] = {mo[i].omega1, r.beta_plus / r.alpha};
                int own[2];
                for (int c = 0; c < 2; ++c) {
                    own[c] = own_slot(i, 1 - s.buf[c], c, opt.components);
                    eom.push_back(om[c]);
                    eslot.push_back(own[c]);
                    eprev.push_back(s.slot[c]);
                }
                rpat.push_back(s.pattern);
                ra.push_back(r.alpha);
                rw.push_back(r.p1);
                rs1.push_back(own[0]);
                rs2.push_back(own[1]);
            }
            ebf.assign((k1 - k0) * size_t(v.n), 1.0);
            if (!fel_device_ebf(dev, int(eom.size()), eom.data(), eslot.data(), eprev.data(), int(rpat.size()), rpat.data(),
                                ra.data(), rs1.data(), rs2.data(), rw.data(), ebf.data(), &err)) {
                st = H3G_ERR_CUDA;
                break;
            }
            for (size_t k = k0; k < k1; ++k) {
                const int i = todo[k];
                const double* e = ebf.data() + (k - k0) * size_t(v.n);
                int bus = 0;
                for (int b = 0; b < v.n; ++b)
                    if (b != v.root && e[b] >= 100.0) ++bus;
                mo[i].r.branches_under_selection = bus;
                if (branch_ebf) {
                    double* dst = branch_ebf + size_t(sites[i].pattern) * v.n;
                    for (int b = 0; b < v.n; ++b) dst[b] = b == v.root ? 1.0 : e[b];
                }
            }
        }
        size_t h2d = 0, d2h = 0;
        int launches = 0;
        fel_device_transfer(dev, &h2d, &d2h, &launches);
        fel_device_destroy(dev);
        if (st != H3G_OK) { fel_set_error(prob, "h3g_meme_run: " + err); return st; }
        fel_record_transfer(prob, h2d + (2 * size_t(S) * S + S + v.n) * sizeof(double), d2h, launches,
                            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count());
        for (int i = 0; i < N; ++i) {
            h3g_meme_result& r = mo[i].r;
            // meme.hpp:599-619: length of the site's mixture model over the tested tree
            const double rate = (r.p1 * (r.alpha * mu_s + r.beta1 * mu_n) + r.p_plus * (r.alpha * mu_s + r.beta_plus * mu_n)) / 3.0;
            r.total_branch_length = tree_len * rate;
            out[variable[i]] = r;
        }
        return H3G_OK;
    } catch (const std::bad_alloc&) {
        fel_set_error(prob, "h3g_meme_run: host allocation failed");
        return H3G_ERR_OOM;
    } catch (const std::exception& e) {
        fel_set_error(prob, std::string("h3g_meme_run: ") + e.what());
        return H3G_ERR_ARG;
    }
}
