// relax_gpu.hpp — RELAXAnalyzer (include/hyphy/analyses/relax.hpp) on the device.
//
// run() follows the reference's phases (relax.hpp:1625-2185): the nucleotide GTR fit, the MG94 fit with
// separate omegas for the test and reference branch sets, then the RELAX null (k = 1) and alternative
// (k free) fits and the LRT (p = erfc(sqrt(LRT / 2)), chi2_1).  The model is the reference's default:
// three omega classes mixed at the P level on every branch (BranchSite), the reference set with omegas
// omega_R,c, the test set with omega_R,c^k, shared weights, and one time conversion per branch set,
// 3 / sum_c w_c mu(omega_c) ("SharedMixture", relax.hpp:536-570), so a branch length is the
// mixture-expected number of substitutions per nucleotide.
//
// The reference fits with a curated start grid and alternating distribution / branch-length cycles; here
// the branch lengths, the reference omegas, the class weights (stick-breaking) and log k are fitted jointly
// by the bounded L-BFGS of optimizer_gpu.hpp from a few starts.  One device evaluation (test classes and
// background classes mixed on their branches, h3g_model_desc.has_bg = 3) gives lnL and the gradients in
// branch times, every model's omega and both weight vectors; the time conversions depend on the omegas and
// weights through mu(omega) = mu_0 + mu_1 omega (linear in omega), and that dependence is chain-ruled on
// the host exactly.  Test branches are the tagged set ({T} and the other test tags), reference branches the
// rest; an unclassified set, PerClass normalization, site-level mixtures, synonymous-rate variation and the
// JSON writers are not provided.
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../core/likelihood_gpu.hpp"
#include "../opt/optimizer_gpu.hpp"

namespace hyphy::analyses {

struct RELAXSettings {
    Scalar p_value_threshold = 0.05;
    bool refine_branch_lengths = true;
    int max_iterations = 1000;
    Scalar tolerance = 1e-5;
};

struct RELAXRateDistribution {
    std::vector<Scalar> omegas;
    std::vector<Scalar> weights;
};

struct RELAXModelFit {
    Scalar log_likelihood = 0.0;
    Scalar aicc = 0.0;
    size_t parameters = 0;
    Scalar tree_scale = 1.0;
    Scalar k = 1.0;
    int realized_cycles = 0;      // L-BFGS iterations of the final run
    bool converged = false;
    RELAXRateDistribution reference_distribution;
    RELAXRateDistribution test_distribution;
    std::vector<Scalar> branch_lengths;        // per node id, substitutions per nucleotide; root 0
    std::vector<Scalar> site_log_likelihoods;  // per pattern
};

struct RELAXResult {
    RELAXSettings settings;
    Scalar gtr_log_likelihood = 0.0;
    Scalar gtr_aicc = 0.0;
    hyphy::core::GTRParameters gtr_rates;
    std::unordered_map<std::string, Scalar> gtr_branch_lengths;
    Scalar mg94_log_likelihood = 0.0;
    Scalar mg94_aicc = 0.0;
    Scalar mg94_omega_R = 1.0;
    Scalar mg94_omega_T = 1.0;
    std::unordered_map<std::string, Scalar> mg94_branch_lengths;
    RELAXModelFit alternative_fit;
    RELAXModelFit null_fit;
    Scalar lrt = 0.0;
    Scalar p_value = 1.0;
    Scalar k = 1.0;
    bool is_relaxed = false;
    bool is_intensified = false;
    bool is_significant = false;
    bool is_failed = false;
    std::string error_message;
    std::vector<std::string> test_branches;
    std::vector<std::string> reference_branches;
    double runtime_seconds = 0.0;
};

class RELAXAnalyzer {
public:
    Tree tree;
    Alignment aln;
    RELAXSettings settings;
    std::vector<bool> is_test_branch;
    std::vector<std::string> test_branch_names;
    std::vector<std::string> ref_branch_names;

    RELAXAnalyzer(Tree t, Alignment a, RELAXSettings s = RELAXSettings{})
        : tree(std::move(t)), aln(std::move(a)), settings(std::move(s)) {
        partition_branches();
    }

    // relax.hpp:233-240
    static RELAXAnalyzer create(Tree tree, Alignment aln, RELAXSettings settings = RELAXSettings{}) {
        return RELAXAnalyzer(std::move(tree), std::move(aln), std::move(settings));
    }

    // test branches: the tagged set (Tree::select_branches with tag detection); reference: every other branch
    void partition_branches() {
        auto sel = tree.select_branches("All", "", {}, true);
        if (sel.num_selected == 0 || sel.num_unselected == 0)
            throw std::runtime_error("RELAX needs tagged test branches and a non-empty reference set");
        is_test_branch = std::move(sel.is_selected);
        test_branch_names = std::move(sel.selected_names);
        ref_branch_names = std::move(sel.unselected_names);
    }

    // relax.hpp:1625-2185
    RELAXResult run() const {
        const auto t0 = std::chrono::steady_clock::now();
        RELAXResult res;
        res.settings = settings;
        res.test_branches = test_branch_names;
        res.reference_branches = ref_branch_names;
        hyphy::opt::GTRFitter gf(tree, aln);
        const auto gtr = gf.fit();
        res.gtr_log_likelihood = gtr.log_likelihood;
        res.gtr_aicc = gtr.aicc;
        res.gtr_rates = gtr.params;
        for (const auto& nd : gtr.tree.nodes)
            if (nd.id != gtr.tree.root_id) res.gtr_branch_lengths[nd.name] = nd.branch_length;
        MG94Parameters p;
        p.theta_AC = gtr.params.theta_AC; p.theta_AT = gtr.params.theta_AT; p.theta_CG = gtr.params.theta_CG;
        p.theta_CT = gtr.params.theta_CT; p.theta_GT = gtr.params.theta_GT;
        hyphy::opt::MG94Fitter mg(gtr.tree, aln);
        Scalar om_r = -1.0;
        const auto mgfit = mg.fit_full_model(1.0, p, nullptr, 250, 1e-5, &is_test_branch, &om_r);
        res.mg94_log_likelihood = mgfit.log_likelihood;
        res.mg94_omega_T = mgfit.params.beta;
        res.mg94_omega_R = om_r;
        const size_t B = tree.num_nodes() - 1;
        res.mg94_aicc = hyphy::opt::compute_aicc(mgfit.log_likelihood, 5 + 2 + B, aln.num_codons);
        for (const auto& nd : mgfit.tree.nodes)
            if (nd.id != mgfit.tree.root_id) res.mg94_branch_lengths[nd.name] = nd.branch_length;

        res.null_fit = fit_relax(false, mgfit.params, mgfit.tree, om_r, nullptr);
        res.alternative_fit = fit_relax(true, mgfit.params, mgfit.tree, om_r, &res.null_fit);
        const bool failed = !(res.alternative_fit.log_likelihood > -1e19) || !(res.null_fit.log_likelihood > -1e19);
        res.k = res.alternative_fit.k;
        if (failed) {
            res.is_failed = true;
            res.error_message = "Optimization failed: model log-likelihood collapsed to the zero-likelihood sentinel.";
        } else {
            res.lrt = 2.0 * std::max<Scalar>(0.0, res.alternative_fit.log_likelihood - res.null_fit.log_likelihood);
            res.p_value = std::erfc(std::sqrt(res.lrt / 2.0));
            res.is_significant = res.p_value <= settings.p_value_threshold;
            if (res.is_significant) (res.k > 1.0 ? res.is_intensified : res.is_relaxed) = true;
        }
        res.runtime_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return res;
    }

    // One RELAX fit: k = 1 (null) or free (alternative).  start_tree: branch lengths in substitutions per
    // nucleotide (the MG94 fit); base: the MG94 exchangeabilities; warm: an extra start (its distribution,
    // lengths and k).
    RELAXModelFit fit_relax(bool has_k, const MG94Parameters& base, const Tree& start_tree, Scalar mg94_omega_R,
                            const RELAXModelFit* warm) const {
        const size_t n = tree.num_nodes();
        std::vector<int32_t> br;
        for (const auto& nd : tree.nodes) if (nd.id != tree.root_id) br.push_back(nd.id);
        const size_t nb = br.size();
        const bool refine = settings.refine_branch_lengths;
        const size_t n_len = refine ? nb : 1;
        const size_t i_om = n_len, i_w = i_om + 3, i_k = i_w + 2, dim = i_k + (has_k ? 1 : 0);
        std::vector<Scalar> lb(dim), ub(dim);
        for (size_t i = 0; i < n_len; ++i) {
            lb[i] = std::log(refine ? 1e-8 : 1e-3);
            ub[i] = std::log(refine ? 1e3 : 100.0);
        }
        lb[i_om] = lb[i_om + 1] = 0.0;
        ub[i_om] = ub[i_om + 1] = 1.0;
        lb[i_om + 2] = 0.0;
        ub[i_om + 2] = std::log(1e4);
        lb[i_w] = lb[i_w + 1] = 0.0;
        ub[i_w] = ub[i_w + 1] = 1.0;
        if (has_k) { lb[i_k] = std::log(1e-5); ub[i_k] = std::log(50.0); }

        std::vector<Scalar> len0(n, 0.0);
        for (const auto& nd : start_tree.nodes)
            if (nd.id != start_tree.root_id) len0[size_t(nd.id)] = nd.branch_length;
        // mu(omega) = mu0 + mu1 omega: the mean rate of the unnormalised MG94 Q (alpha = 1) is linear in omega
        const auto& code = aln.code ? *aln.code : *hyphy::core::GeneticCode::universal();
        auto mean_rate = [&](Scalar om) {
            MG94Parameters q = base;
            q.alpha = 1.0;
            q.beta = om;
            MG94Matrix mm;
            mm.update(q, aln.pos_nuc_frequencies, aln.codon_frequencies_f3x4, code);
            return mm.scale_factor;
        };
        const Scalar mu0 = mean_rate(0.0), mu1 = mean_rate(1.0) - mu0;
        auto mu = [&](Scalar om) { return mu0 + mu1 * om; };
        std::vector<bool> test(is_test_branch);
        test.resize(n, false);

        struct Point { std::vector<Scalar> t, omR, omT, w; Scalar k = 1.0, scale = 1.0; };
        auto decode = [&](const std::vector<Scalar>& x) {
            Point pt;
            pt.t.assign(n, 0.0);
            if (refine) for (size_t i = 0; i < nb; ++i) pt.t[size_t(br[i])] = std::exp(x[i]);
            else { pt.scale = std::exp(x[0]); for (int32_t id : br) pt.t[size_t(id)] = pt.scale * len0[size_t(id)]; }
            pt.omR = {x[i_om], x[i_om + 1], std::exp(x[i_om + 2])};
            pt.w = {x[i_w], (1.0 - x[i_w]) * x[i_w + 1], (1.0 - x[i_w]) * (1.0 - x[i_w + 1])};
            pt.k = has_k ? std::exp(x[i_k]) : 1.0;
            pt.omT.resize(3);
            for (int c = 0; c < 3; ++c)   // relax.hpp:589-597
                pt.omT[size_t(c)] = pt.omR[size_t(c)] <= 1e-12 ? 0.0 : std::clamp(std::pow(pt.omR[size_t(c)], pt.k), 1e-6, 1e4);
            return pt;
        };
        auto encode = [&](const std::vector<Scalar>& t, Scalar scale, const std::vector<Scalar>& omR, const std::vector<Scalar>& w,
                          Scalar k) {
            std::vector<Scalar> x(dim, 0.0);
            if (refine) for (size_t i = 0; i < nb; ++i) x[i] = std::log(std::max<Scalar>(t[size_t(br[i])], 1e-8));
            else x[0] = std::log(scale);
            x[i_om] = omR[0];
            x[i_om + 1] = omR[1];
            x[i_om + 2] = std::log(std::max<Scalar>(omR[2], 1.0));
            x[i_w] = w[0];
            x[i_w + 1] = w[0] < 1.0 ? w[1] / (1.0 - w[0]) : 0.0;
            if (has_k) x[i_k] = std::log(k);
            for (size_t j = 0; j < dim; ++j) x[j] = std::clamp(x[j], lb[j], ub[j]);
            return x;
        };
        struct Eval { hyphy::core::MixtureGradients r; std::vector<Scalar> tau; Scalar convT = 1, convR = 1, muT = 1, muR = 1; };
        auto evaluate = [&](const Point& pt, bool grads) {
            Eval e;
            e.muR = e.muT = 0.0;
            for (int c = 0; c < 3; ++c) {
                e.muR += pt.w[size_t(c)] * mu(pt.omR[size_t(c)]);
                e.muT += pt.w[size_t(c)] * mu(pt.omT[size_t(c)]);
            }
            e.convR = e.muR > 1e-12 ? 3.0 / e.muR : 1.0;
            e.convT = e.muT > 1e-12 ? 3.0 / e.muT : 1.0;
            e.tau.assign(n, 0.0);
            for (int32_t id : br) e.tau[size_t(id)] = (test[size_t(id)] ? e.convT : e.convR) * pt.t[size_t(id)];
            e.r = hyphy::core::LikelihoodEngine::compute_mixture_gradients(
                tree, aln, base, e.tau, pt.omT, pt.w, {1.0}, {1.0}, &test, -1.0, grads, /*zero_likelihood_sentinel=*/true,
                /*direction_gradients=*/grads, pt.omR, pt.w);
            return e;
        };
        auto fg = [&](const std::vector<Scalar>& x, std::vector<Scalar>& g) -> Scalar {
            const Point pt = decode(x);
            const Eval e = evaluate(pt, true);
            const auto& r = e.r;
            g.assign(dim, 0.0);
            Scalar ET = 0.0, ER = 0.0;   // sum over each set of tau_b dlnL/dtau_b
            for (int32_t id : br) (test[size_t(id)] ? ET : ER) += e.tau[size_t(id)] * r.grad_branches[size_t(id)];
            // conv = 3 / mu_mix, so dlnL/dmu_mix = -E / mu_mix
            const Scalar dT = e.muT > 1e-12 ? -ET / e.muT : 0.0, dR = e.muR > 1e-12 ? -ER / e.muR : 0.0;
            if (refine) {
                for (size_t i = 0; i < nb; ++i) g[i] = -e.tau[size_t(br[i])] * r.grad_branches[size_t(br[i])];
            } else {
                g[0] = -(ET + ER);
            }
            std::vector<Scalar> dOmT(3, 0.0), dOmR(3, 0.0), dW(3, 0.0);
            Scalar dk = 0.0;
            for (size_t c = 0; c < 3; ++c) {
                dOmT[c] = r.grad_omegas[c] + dT * pt.w[c] * mu1;
                dOmR[c] = r.grad_bg_omegas[c] + dR * pt.w[c] * mu1;
                dW[c] = r.grad_weights[c] + r.grad_bg_weights[c] + dT * mu(pt.omT[c]) + dR * mu(pt.omR[c]);
                const Scalar oR = pt.omR[c], oT = pt.omT[c];
                const bool free = oR > 1e-12 && oT > 1e-6 && oT < 1e4;   // omega_T inside its clamp
                if (free) {
                    dOmR[c] += dOmT[c] * pt.k * oT / oR;                 // d(oR^k)/doR = k oR^(k-1)
                    dk += dOmT[c] * oT * std::log(oR);                     // d(oR^k)/dk = oR^k ln oR
                }
            }
            g[i_om] = -dOmR[0];
            g[i_om + 1] = -dOmR[1];
            g[i_om + 2] = -dOmR[2] * pt.omR[2];
            // w0 = p0, w1 = (1-p0) p1, w2 = (1-p0)(1-p1)
            const Scalar p0 = x[i_w], p1 = x[i_w + 1];
            g[i_w] = -(dW[0] - p1 * dW[1] - (1.0 - p1) * dW[2]);
            g[i_w + 1] = -((1.0 - p0) * dW[1] - (1.0 - p0) * dW[2]);
            if (has_k) g[i_k] = -dk * pt.k;
            return -r.log_likelihood;
        };

        std::vector<std::vector<Scalar>> starts;
        const Scalar om_mid = std::clamp(mg94_omega_R, 0.05, 0.9);
        const Scalar so[3][3] = {{0.05, 0.5, 2.0}, {0.0, om_mid, 1.5}, {0.1, 0.8, 5.0}};
        const Scalar sw[3][3] = {{0.6, 0.3, 0.1}, {0.5, 0.4, 0.1}, {0.7, 0.25, 0.05}};
        for (int j = 0; j < 3; ++j)
            starts.push_back(encode(len0, 1.0, {so[j][0], so[j][1], so[j][2]}, {sw[j][0], sw[j][1], sw[j][2]}, 1.0));
        if (warm && warm->branch_lengths.size() == n) {
            starts.push_back(encode(warm->branch_lengths, warm->tree_scale, warm->reference_distribution.omegas,
                                    warm->reference_distribution.weights, has_k ? warm->k : 1.0));
            if (has_k)   // the warm start with the relaxation moved both ways
                for (Scalar kk : {0.5, 2.0})
                    starts.push_back(encode(warm->branch_lengths, warm->tree_scale, warm->reference_distribution.omegas,
                                            warm->reference_distribution.weights, kk));
        }
        // screen every start for 40 iterations, then run the two best to convergence
        std::vector<hyphy::opt::BoxLBFGSResult> screened;
        for (const auto& x0 : starts) {
            auto r = hyphy::opt::box_lbfgs(fg, x0, lb, ub, settings.tolerance, 40);
            if (std::isfinite(r.f)) screened.push_back(std::move(r));
        }
        if (screened.empty()) throw std::runtime_error("RELAX: every start has a zero likelihood");
        std::stable_sort(screened.begin(), screened.end(), [](const auto& a, const auto& b) { return a.f < b.f; });
        hyphy::opt::BoxLBFGSResult best = screened.front();
        for (size_t i = 0; i < std::min<size_t>(2, screened.size()); ++i) {
            auto fin_run = hyphy::opt::box_lbfgs(fg, screened[i].x, lb, ub, settings.tolerance, settings.max_iterations);
            if (std::isfinite(fin_run.f) && fin_run.f < best.f) best = std::move(fin_run);
        }
        // The model sets omega_T,0 = 0 once omega_R,0 <= 1e-12 (relax.hpp:589-597): the likelihood jumps at
        // omega_R,0 -> 0 and a line search can stall just short of it.  Polish once from the optimum with
        // omega_R,0 = 0 exactly and once with fresh curvature memory; keep the best.
        for (int variant = 0; variant < 2; ++variant) {
            std::vector<Scalar> x1 = best.x;
            if (variant == 0) {
                if (x1[i_om] <= lb[i_om]) continue;
                x1[i_om] = lb[i_om];
            }
            auto r = hyphy::opt::box_lbfgs(fg, x1, lb, ub, settings.tolerance, settings.max_iterations);
            if (std::isfinite(r.f) && r.f < best.f) best = std::move(r);
        }

        const Point pt = decode(best.x);
        const Eval e = evaluate(pt, false);
        RELAXModelFit fit;
        fit.log_likelihood = e.r.log_likelihood;
        fit.site_log_likelihoods = e.r.site_log_likelihoods;
        fit.k = pt.k;
        fit.tree_scale = pt.scale;
        fit.branch_lengths = pt.t;
        fit.realized_cycles = best.iterations;
        fit.converged = best.converged || best.pg_inf <= std::max<Scalar>(settings.tolerance, 1e-3);
        fit.reference_distribution = {pt.omR, pt.w};
        fit.test_distribution = {pt.omT, pt.w};
        fit.parameters = n_len + 5 + (has_k ? 1 : 0);
        fit.aicc = hyphy::opt::compute_aicc(fit.log_likelihood, fit.parameters, aln.num_codons);
        return fit;
    }
};

}  // namespace hyphy::analyses
