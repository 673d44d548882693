// h3g_meme_driver.cpp — h3g_meme_run / h3g_meme_run_tested: MEME per-site fits with every pattern's
// optimisers advanced in lockstep (h3g_sitefit.h).
//
// Per pattern, as analyses/meme.hpp:166-632:
//   1. the FEL fit of the pattern (the same coroutines as h3g_fel_run /
//      h3g_fel_run_tested, on FEL's branch partition);
//   2. the alternative model by the reference's bounded 4-D Nelder-Mead
//      (opt/nelder_mead.hpp:209-357) from its start grid, the null model
//      (beta+ = alpha) by the 3-D one, a warm-started refit, LRT and p-value;
//      with a background branch set, beta_bg joins both (5-D and 4-D);
//   3. for the patterns that reach the test, the empirical Bayes factor of
//      every branch from one inside-outside pass on the device (k_meme_ebf).
// A likelihood evaluation needs two eigensystems (omega1 and beta+ / alpha)
// and prunes with their transition matrices mixed (p1, 1 - p1) per tested
// branch; background branches use a third (beta_bg / alpha) alone.
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

// (alpha, omega1, p1, beta+[, beta_bg]) -> request: components omega1 and beta+ / alpha, weights
// (p1, 1 - p1), and beta_bg / alpha on the background branches (meme.hpp:219-272)
Req alt_req(const Arr<4>& x) { return Req{x[0], x[1], x[3] / x[0], x[2], 0.0}; }
Req alt_req5(const Arr<5>& x) {
    Req r{x[0], x[1], x[3] / x[0], x[2], 0.0};
    r.om_bg = x[4] / x[0];
    return r;
}
// null model: beta+ = alpha
Req null_req(const Arr<3>& x) { return Req{x[0], x[1], x[0] / x[0], x[2], 0.0}; }
Req null_req4(const Arr<4>& x) {
    Req r{x[0], x[1], x[0] / x[0], x[2], 0.0};
    r.om_bg = x[3] / x[0];
    return r;
}

// meme.hpp:166-632 after the FEL fit; has_bg: MEME's tested set leaves a background
Fit meme_search(Site& s, const h3g_fel_result& fel, MemeOut& out, bool has_bg) {
    s.evaluations = 0;
    h3g_meme_result& res = out.r;
    res.fel_alpha = fel.alpha;
    res.fel_beta = fel.beta;
    res.log_l_fel = fel.log_l_alt;
    using A5 = Arr<5>;
    using A4 = Arr<4>;
    using A3 = Arr<3>;
    // start grid (meme.hpp:282-312)
    const double af = std::clamp(fel.alpha, 1e-4, 10000.0), bf = std::clamp(fel.beta, 1e-4, 100000.0);
    const double bg0 = (has_bg && fel.beta_nuisance > 0.0) ? std::clamp(fel.beta_nuisance, 1e-4, 100000.0) : bf;
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
    const A5 lb5 = {1e-4, 0.0, 1e-6, 1e-4, 1e-4}, ub5 = {10000.0, 1.0, 1.0 - 1e-6, 100000.0, 100000.0};
    double omega1 = w10;
    if (has_bg) {
        // alternative model with a free background rate (meme.hpp:318-337)
        std::vector<A5> grid5;
        for (const auto& g : grid) grid5.push_back({g[0], g[1], g[2], g[3], bg0});
        const Pt<5> alt = co_await nelder_mead_nd<5>(s, alt_req5, grid5[0], lb5, ub5, 1e-5, 800, grid5);
        res.alpha = alt.x[0];
        omega1 = alt.x[1];
        res.p1 = alt.x[2];
        res.beta_plus = alt.x[3];
        res.beta_bg = alt.x[4];
        res.log_l_meme = -alt.f;
    } else {
        // alternative model (meme.hpp:338-354)
        const Pt<4> alt = co_await nelder_mead_nd<4>(s, alt_req, grid[0], lb4, ub4, 1e-5, 800, grid);
        res.alpha = alt.x[0];
        omega1 = alt.x[1];
        res.p1 = alt.x[2];
        res.beta_plus = alt.x[3];
        res.beta_bg = 0.0;
        res.log_l_meme = -alt.f;
    }
    res.beta1 = res.alpha * omega1;
    res.p_plus = 1.0 - res.p1;
    if (res.beta_plus > res.alpha && res.p_plus > 1e-6) {
        double lnl_null = -1e20, a_null = res.alpha, w_null = omega1, p_null = res.p1, bg_null = res.beta_bg;
        const double an = std::clamp(fel.alpha_null, 1e-4, 50.0);
        if (has_bg) {
            // null model beta+ = alpha with beta_bg free (meme.hpp:364-405)
            std::vector<A4> ng = {{res.alpha, omega1, res.p1, res.beta_bg}, {an, 1.0, 0.5, bg0}, {an, omega1, res.p1, bg0},
                                  {std::clamp(res.alpha, 1e-4, 50.0), 1.0, 0.5, res.beta_bg}};
            for (double c : {0.01, 0.1, 0.5, 1.0, 2.0, 5.0, 10.0, 20.0}) {
                ng.push_back({c, 0.5, 0.5, res.beta_bg});
                ng.push_back({c, 0.0, 0.9, res.beta_bg});
            }
            const Pt<4> nul = co_await nelder_mead_nd<4>(s, null_req4, ng[0], lb4, ub4, 1e-5, 800, ng);
            lnl_null = -nul.f;
            a_null = nul.x[0];
            w_null = nul.x[1];
            p_null = nul.x[2];
            bg_null = nul.x[3];
            if (lnl_null > res.log_l_meme && std::isfinite(lnl_null)) {
                const std::vector<A5> wg = {{a_null, w_null, p_null, a_null, bg_null}, {a_null, w_null, 0.99, a_null, bg_null}};
                const Pt<5> alt2 = co_await nelder_mead_nd<5>(s, alt_req5, wg[0], lb5, ub5, 1e-5, 800, wg);
                if (-alt2.f > res.log_l_meme) {
                    res.alpha = alt2.x[0];
                    omega1 = alt2.x[1];
                    res.p1 = alt2.x[2];
                    res.beta_plus = alt2.x[3];
                    res.beta_bg = alt2.x[4];
                    res.beta1 = res.alpha * omega1;
                    res.p_plus = 1.0 - res.p1;
                    res.log_l_meme = -alt2.f;
                }
            }
        } else {
            // null model (meme.hpp:406-452)
            std::vector<A3> ng = {{res.alpha, omega1, res.p1}, {an, 1.0, 0.5}, {an, omega1, res.p1},
                                  {std::clamp(res.alpha, 1e-4, 50.0), 1.0, 0.5}};
            for (double c : {0.01, 0.1, 0.5, 1.0, 2.0, 5.0, 10.0, 20.0}) {
                ng.push_back({c, 0.5, 0.5});
                ng.push_back({c, 0.0, 0.9});
            }
            const A3 lb3 = {1e-4, 0.0, 1e-6}, ub3 = {10000.0, 1.0, 1.0 - 1e-6};
            const Pt<3> nul = co_await nelder_mead_nd<3>(s, null_req, ng[0], lb3, ub3, 1e-5, 800, ng);
            lnl_null = -nul.f;
            a_null = nul.x[0];
            w_null = nul.x[1];
            p_null = nul.x[2];
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
            res.beta_bg = bg_null;
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
    const double d_fel = 2.0 * (res.log_l_meme - res.log_l_fel);   // meme.hpp:607-613
    res.p_value_meme_vs_fel = d_fel > 0.0 ? std::exp(-d_fel / 2.0) : 1.0;
    out.omega1 = omega1;
    res.evaluations = s.evaluations;
}

}  // namespace
}  // namespace h3g::sitefit

using namespace h3g;
using namespace h3g::sitefit;

static h3g_status meme_run_impl(h3g_problem* prob, const h3g_fel_model* m, const double* branch_lengths, const uint8_t* tested,
                                const uint8_t* fel_tested, h3g_meme_result* out, double* branch_ebf, const char* who) {
    if (!prob) return H3G_ERR_ARG;
    const auto t_start = std::chrono::steady_clock::now();
    const std::string w(who);
    try {
        FelProblemView v;
        std::vector<int> variable;
        if (!out) { fel_set_error(prob, w + ": null argument"); return H3G_ERR_ARG; }
        const h3g_status pst = prepare_site_run(prob, m, branch_lengths, who, &v, &variable);
        if (pst != H3G_OK) return pst;
        h3g_meme_result zero{0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0, 0.0};
        for (int p = 0; p < v.P; ++p) out[p] = zero;
        if (branch_ebf) std::fill(branch_ebf, branch_ebf + size_t(v.P) * v.n, 1.0);
        // background flags of the MEME test and of the FEL baseline (meme.hpp:84-92)
        std::vector<uint8_t> bg(size_t(v.n), 0), fel_bg(size_t(v.n), 0);
        bool has_bg = false, fel_has_bg = false;
        for (int b = 0; b < v.n; ++b) {
            if (b == v.root) continue;
            if (tested && !tested[b]) { bg[size_t(b)] = 1; has_bg = true; }
            const uint8_t* ft = fel_tested ? fel_tested : tested;
            if (ft && !ft[b]) { fel_bg[size_t(b)] = 1; fel_has_bg = true; }
        }
        const int N = int(variable.size());
        if (N == 0) return H3G_OK;
        const int S = m->S;
        // mean rate of a site's model is linear in (alpha, beta): alpha mu_s + beta mu_n
        double mu_s = 0.0, mu_n = 0.0, len_test = 0.0, len_bg = 0.0;
        for (int i = 0; i < S; ++i)
            for (int j = 0; j < S; ++j)
                if (j != i) {
                    mu_s += m->pi[i] * m->Qs[i * S + j];
                    mu_n += m->pi[i] * m->Qn[i * S + j];
                }
        for (int b = 0; b < v.n; ++b)
            if (b != v.root) (bg[size_t(b)] ? len_bg : len_test) += branch_lengths[b];
        // a start grid parks up to 21 requests at once; the pool holds up to three eigensystems per request
        LockstepOptions opt;
        opt.components = (has_bg || fel_has_bg) ? 3 : 2;
        opt.max_requests = std::max({64, N, std::min(8 * N, 16384)});
        opt.temp_slots = std::min((opt.components == 3 ? 3 : 2) * opt.max_requests, 32768);
        opt.spec_threshold = 32;            // four candidates per site still fit one wave of the pruning kernel
        std::string err;
        // the device's background flags are MEME's; the FEL phase runs on FEL's when they differ
        std::vector<uint8_t> dev_bg = has_bg ? bg : fel_bg;
        FelDevice* dev = fel_device_create(prob, S, m->pi, m->Qs, m->Qn, branch_lengths,
                                           (has_bg || fel_has_bg) ? dev_bg.data() : nullptr, opt.max_requests,
                                           slots_needed(N, opt.temp_slots, opt.components), &err);
        if (!dev) { fel_set_error(prob, w + ": " + err); return H3G_ERR_CUDA; }
        const bool split_phases = fel_has_bg && has_bg && fel_bg != bg;
        std::vector<Site> sites(N);
        std::vector<h3g_fel_result> fel(N, h3g_fel_result{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0, 0.0});
        std::vector<MemeOut> mo(N);
        LockstepState state;                // one slot map for both phases: sites keep their slots
        h3g_status st = H3G_OK;
        if (split_phases) {
            // two different background sets: the FEL phase gets its own evaluator state
            fel_device_destroy(dev);
            dev = fel_device_create(prob, S, m->pi, m->Qs, m->Qn, branch_lengths, fel_bg.data(), opt.max_requests,
                                    slots_needed(N, opt.temp_slots, opt.components), &err);
            if (!dev) { fel_set_error(prob, w + ": " + err); return H3G_ERR_CUDA; }
        }
        {
            std::vector<Fit> fits;
            fits.reserve(N);
            for (int i = 0; i < N; ++i) {
                sites[i].pattern = variable[i];
                fits.push_back(fel_has_bg ? fel_search_subset(sites[i], fel[i]) : fel_search(sites[i], fel[i]));
            }
            // the FEL baseline keeps FEL's caching: per pattern (fel.hpp:368-376) or none (subset path)
            opt.cache_tol = fel_has_bg ? 0.0 : 1e-12;
            st = run_lockstep(dev, sites, fits, opt, state, &err);
        }
        if (st == H3G_OK && split_phases) {
            fel_device_destroy(dev);
            dev = fel_device_create(prob, S, m->pi, m->Qs, m->Qn, branch_lengths, bg.data(), opt.max_requests,
                                    slots_needed(N, opt.temp_slots, opt.components), &err);
            if (!dev) { fel_set_error(prob, w + ": " + err); return H3G_ERR_CUDA; }
        }
        if (st == H3G_OK) {
            std::vector<Fit> fits;
            fits.reserve(N);
            for (int i = 0; i < N; ++i) fits.push_back(meme_search(sites[i], fel[i], mo[i], has_bg));
            opt.cache_tol = 0.0;            // MEME builds its models afresh for every evaluation
            st = run_lockstep(dev, sites, fits, opt, state, &err);
        }
        // empirical Bayes factors at the reported MLE, in chunks
        std::vector<int> todo;
        for (int i = 0; i < N; ++i)
            if (mo[i].ebf) todo.push_back(i);
        const int chunk = fel_device_max_ebf(dev);
        const int nc = has_bg ? 3 : 2;
        std::vector<double> ebf, eom, ra, rw;
        std::vector<int> eslot, eprev, rpat, rs1, rs2, rs3;
        for (size_t k0 = 0; st == H3G_OK && k0 < todo.size(); k0 += size_t(chunk)) {
            const size_t k1 = std::min(todo.size(), k0 + size_t(chunk));
            eom.clear(); eslot.clear(); eprev.clear(); rpat.clear(); ra.clear(); rw.clear(); rs1.clear(); rs2.clear(); rs3.clear();
            for (size_t k = k0; k < k1; ++k) {
                const int i = todo[k];
                Site& s = sites[i];
                const h3g_meme_result& r = mo[i].r;
                // meme.hpp:484-500: the background model at beta_bg, or beta1 when that is not positive
                const double om[3] = {mo[i].omega1, r.beta_plus / r.alpha, (r.beta_bg > 0.0 ? r.beta_bg : r.beta1) / r.alpha};
                int own[3];
                for (int c = 0; c < nc; ++c) {
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
                if (has_bg) rs3.push_back(own[2]);
            }
            ebf.assign((k1 - k0) * size_t(v.n), 1.0);
            if (!fel_device_ebf(dev, int(eom.size()), eom.data(), eslot.data(), eprev.data(), int(rpat.size()), rpat.data(),
                                ra.data(), rs1.data(), rs2.data(), rw.data(), has_bg ? rs3.data() : nullptr, ebf.data(), &err)) {
                st = H3G_ERR_CUDA;
                break;
            }
            for (size_t k = k0; k < k1; ++k) {
                const int i = todo[k];
                const double* e = ebf.data() + (k - k0) * size_t(v.n);
                int bus = 0;
                for (int b = 0; b < v.n; ++b)
                    if (b != v.root && !bg[size_t(b)] && e[b] >= 100.0) ++bus;
                mo[i].r.branches_under_selection = bus;
                if (branch_ebf) {
                    double* dst = branch_ebf + size_t(sites[i].pattern) * v.n;
                    for (int b = 0; b < v.n; ++b) dst[b] = (b == v.root || bg[size_t(b)]) ? 1.0 : e[b];
                }
            }
        }
        size_t h2d = 0, d2h = 0;
        int launches = 0;
        fel_device_transfer(dev, &h2d, &d2h, &launches);
        fel_device_destroy(dev);
        if (st != H3G_OK) { fel_set_error(prob, w + ": " + err); return st; }
        fel_record_transfer(prob, h2d + (2 * size_t(S) * S + S + v.n) * sizeof(double), d2h, launches,
                            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count());
        for (int i = 0; i < N; ++i) {
            h3g_meme_result& r = mo[i].r;
            // meme.hpp:615-634: the site's models over the tree, tested and background branches at their own rates
            const double test_rate = (r.p1 * (r.alpha * mu_s + r.beta1 * mu_n) + r.p_plus * (r.alpha * mu_s + r.beta_plus * mu_n)) / 3.0;
            const double bg_rate = has_bg ? (r.alpha * mu_s + (r.beta_bg > 0.0 ? r.beta_bg : r.beta1) * mu_n) / 3.0 : test_rate;
            r.total_branch_length = len_test * test_rate + len_bg * bg_rate;
            out[variable[i]] = r;
        }
        return H3G_OK;
    } catch (const std::bad_alloc&) {
        fel_set_error(prob, w + ": host allocation failed");
        return H3G_ERR_OOM;
    } catch (const std::exception& e) {
        fel_set_error(prob, w + ": " + e.what());
        return H3G_ERR_ARG;
    }
}

extern "C" h3g_status h3g_meme_run(h3g_problem* prob, const h3g_fel_model* m, const double* branch_lengths, h3g_meme_result* out,
                                   double* branch_ebf) {
    return meme_run_impl(prob, m, branch_lengths, nullptr, nullptr, out, branch_ebf, "h3g_meme_run");
}

extern "C" h3g_status h3g_meme_run_tested(h3g_problem* prob, const h3g_fel_model* m, const double* branch_lengths,
                                          const uint8_t* tested, const uint8_t* fel_tested, h3g_meme_result* out,
                                          double* branch_ebf) {
    if (prob && !tested) {
        fel_set_error(prob, "h3g_meme_run_tested: null argument");
        return H3G_ERR_ARG;
    }
    return meme_run_impl(prob, m, branch_lengths, tested, fel_tested, out, branch_ebf, "h3g_meme_run_tested");
}
