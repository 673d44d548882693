// busted_gpu.hpp — the likelihood core of BUSTEDAnalyzer (include/hyphy/analyses/busted.hpp)
// on the device: evaluate_log_l (busted.hpp:509-660) and the two EM expectation steps,
// compute_expected_weights (:662-975) and compute_expected_syn_weights (:978-1134).
//
// The reference computes the E-steps with one inside-outside pass per synonymous-rate
// class: for every test branch b and omega class k, the expected share
//   sum_p wt_p sum_m post_m(p) w_k V_b . (P_k,b D_b) / L_m(p),
// normalised by (number of test branches) x sum_p wt_p; and sum_p wt_p post_m(p) / sum_p wt_p
// for the rate classes.  P_mix,b = sum_k w_k P_k,b is linear in the weights, so the first
// sum is w_k dlnL/dw_k and the second rho_m dlnL/drho_m: both come from ONE device mixture
// evaluation (h3g_eval with the class- and rate-weight gradients, no omega/theta
// directions), whose per-branch contraction is the same V . P D.  The posterior cut-off of
// the reference (terms with post_m <= 1e-12 skipped) changes the shares by < 1e-12.
//
// Same members as the reference class for what these methods read (branch_tau,
// is_test_branch, num_test_branches, mg94_omega, mg94_background_omega).
//
// fit_model / run / create_and_fit (busted.hpp:220-258, :1644-2607, :5969-6682) fit the
// same models to the same maxima by a different path.  The reference alternates Brent,
// Nelder-Mead and EM steps with class-rescue heuristics; here every free parameter (branch
// lengths or a tree scale, the omegas, the class weights, the synonymous rates and their
// weights) is fitted jointly by the bounded L-BFGS of optimizer_gpu.hpp from a few starts,
// with the likelihood and the gradients in the branch lengths, omegas and class weights from
// one device mixture evaluation; the synonymous-rate coordinates use central differences of
// the device likelihood.  Not provided: the error sink (eps_sink must be 0), multiple hits,
// bridge resolutions, the full automatic selector, BUSTED-PH / RELAX modes and the branch-site
// diagnostics.  A test set that leaves background branches fits the two-set model (a separate
// K-class background distribution, busted.hpp:4344-5087).
#pragma once

#include <algorithm>
#include <array>
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

using hyphy::core::Alignment;
using hyphy::core::MG94Matrix;
using hyphy::core::MG94Parameters;
using hyphy::core::Scalar;
using hyphy::core::Tree;

// busted_types.hpp: the settings, rate distributions, fits and results of the reference
struct BUSTEDSettings {
    bool full_auto = false;
    size_t num_rate_classes = 3;
    bool srv = false;
    size_t num_syn_rate_classes = 3;
    bool auto_select_k = false;
    size_t max_k = 3;
    bool refine_branch_lengths = true;
    Scalar p_value_threshold = 0.05;
    std::string multiple_hits = "None";
    bool error_sink = false;
    Scalar error_sink_max_weight = 0.01;
    Scalar error_sink_bf_threshold = 100.0;
    std::string test_branches = "All";
    bool phenotype_mode = false;
    bool relax_mode = false;
};

struct BUSTEDRateDistribution {
    std::vector<Scalar> omegas;
    std::vector<Scalar> weights;
    std::vector<Scalar> syn_rates;
    std::vector<Scalar> syn_weights;
    Scalar error_sink_weight = 0.0;
    std::vector<std::string> annotations;   // per class; "" = unannotated
};

struct BUSTEDFit {
    Scalar log_likelihood = 0.0;
    Scalar aicc = 0.0;
    Scalar tree_scale = 1.0;
    size_t num_rate_classes = 3;
    BUSTEDRateDistribution test_distribution;
    bool has_background_distribution = false;
    BUSTEDRateDistribution background_distribution;
    std::vector<Scalar> branch_lengths;        // per node id (raw time), root 0
    std::vector<Scalar> site_log_likelihoods;  // per pattern
    Scalar delta = 0.0;
    Scalar psi = 0.0;
    Scalar error_sink_weight = 0.0;
    bool has_gtr_params = false;
    MG94Parameters gtr_params;                 // the fitted nucleotide exchangeabilities (theta_AC..GT)
    int iterations = 0;
};

struct BUSTEDResult {
    BUSTEDSettings settings;
    size_t optimal_k = 3;
    Scalar lrt = 0.0;
    Scalar p_value = 1.0;
    BUSTEDFit unconstrained;
    BUSTEDFit constrained;
    std::vector<Scalar> evidence_ratios;              // per site: exp(lnL_alt - lnL_null)
    std::vector<Scalar> constrained_evidence_ratios;  // per site: exp(lnL_alt - lnL_alt with omega_K := min(1, omega_K))
    std::vector<BUSTEDFit> k_null_fits;               // auto_select_k: the null fits for K = 1 .. max_k
    bool is_failed = false;
    std::string error_message;
    Scalar runtime_seconds = 0.0;
};

class BUSTEDAnalyzer {
public:
    Tree tree;
    Alignment aln;
    mutable MG94Parameters base_params;
    mutable std::vector<Scalar> branch_tau;       // baseline lengths x 3 / scale factor (busted.hpp:260-281)
    mutable std::vector<bool> is_test_branch;     // per node; the root is never a test branch
    mutable size_t num_test_branches = 0;
    mutable size_t num_background_branches = 0;
    Scalar mg94_omega = 1.0;
    Scalar mg94_background_omega = -1.0;          // < 0: background branches use mg94_omega
    Scalar mg94_tree_length = 0.0;
    Scalar mg94_log_l = 0.0;
    bool has_gtr_fit = false;
    Scalar gtr_log_l = 0.0;
    Scalar gtr_aicc = 0.0;
    hyphy::core::GTRParameters gtr_rates;
    std::unordered_map<std::string, Scalar> gtr_branch_lengths;

    BUSTEDAnalyzer(Tree t, Alignment a, MG94Parameters base_p = MG94Parameters{})
        : tree(std::move(t)), aln(std::move(a)), base_params(base_p) {
        const size_t n = tree.num_nodes();
        branch_tau.assign(n, 0.0);
        is_test_branch.assign(n, true);
        if (tree.root_id >= 0 && size_t(tree.root_id) < n) is_test_branch[size_t(tree.root_id)] = false;
        num_test_branches = n > 0 ? n - 1 : 0;
        prepare_baseline_lengths();
    }

    // busted.hpp:260-281
    void prepare_baseline_lengths() {
        const auto& code = aln.code ? *aln.code : *hyphy::core::GeneticCode::universal();
        MG94Matrix mat;
        mat.update(base_params, aln.pos_nuc_frequencies, aln.codon_frequencies_f3x4, code);
        const Scalar conv = mat.scale_factor > 1e-12 ? 3.0 / mat.scale_factor : 1.0;
        mg94_tree_length = 0.0;
        for (const auto& node : tree.nodes) {
            if (node.id == tree.root_id) continue;
            branch_tau[size_t(node.id)] = node.branch_length * conv;
            mg94_tree_length += branch_tau[size_t(node.id)];
        }
    }

    // busted.hpp:509-660: per-pattern log-sum-exp over rate classes, the -1e20 sentinel for
    // zero-likelihood patterns, Neumaier sum over patterns
    Scalar evaluate_log_l(Scalar s, const std::vector<Scalar>& omegas, const std::vector<Scalar>& weights,
                          const std::vector<Scalar>& syn_rates = {1.0}, const std::vector<Scalar>& syn_weights = {1.0},
                          const std::vector<Scalar>* custom_branch_lengths = nullptr,
                          std::vector<Scalar>* out_pattern_ll = nullptr, Scalar delta = 0.0, Scalar psi = 0.0,
                          Scalar eps_sink = 0.0, const MG94Parameters* custom_base_params = nullptr) const {
        const auto r = mixture(s, omegas, weights, syn_rates, syn_weights, custom_branch_lengths, delta, psi, eps_sink,
                               custom_base_params, false);
        if (out_pattern_ll) *out_pattern_ll = r.site_log_likelihoods;
        return r.log_likelihood;
    }

    // busted.hpp:3146-3378 (no error sinks, no unclassified set): test branches mix (omegas_test, weights_test),
    // every other branch (omegas_bg, weights_bg); lengths s x branch_tau or s x custom_branch_lengths (raw time)
    Scalar evaluate_two_set_log_l(Scalar s, const std::vector<Scalar>& omegas_test, const std::vector<Scalar>& weights_test,
                                  const std::vector<Scalar>& omegas_bg, const std::vector<Scalar>& weights_bg,
                                  const std::vector<Scalar>& syn_rates = {1.0}, const std::vector<Scalar>& syn_weights = {1.0},
                                  const std::vector<Scalar>* custom_branch_lengths = nullptr,
                                  std::vector<Scalar>* out_pattern_ll = nullptr, Scalar delta = 0.0, Scalar psi = 0.0,
                                  Scalar eps_sink_test = 0.0, Scalar eps_sink_bg = 0.0,
                                  const std::vector<Scalar>* omegas_unclass = nullptr,
                                  const std::vector<Scalar>* weights_unclass = nullptr,
                                  const MG94Parameters* custom_base_params = nullptr) const {
        if (eps_sink_test != 0.0 || eps_sink_bg != 0.0 || omegas_unclass || weights_unclass)
            throw std::runtime_error("BUSTEDAnalyzer (device): error sinks and an unclassified set are not supported");
        MG94Parameters base = custom_base_params ? *custom_base_params : base_params;
        base.delta = delta;
        base.psi = psi;
        const size_t n = tree.num_nodes();
        std::vector<Scalar> bl(n, 0.0);
        for (const auto& node : tree.nodes)
            if (node.id != tree.root_id)
                bl[size_t(node.id)] = s * (custom_branch_lengths ? (*custom_branch_lengths)[size_t(node.id)] : branch_tau[size_t(node.id)]);
        std::vector<bool> test(is_test_branch);
        test.resize(n, true);
        if (tree.root_id >= 0) test[size_t(tree.root_id)] = false;
        const auto r = hyphy::core::LikelihoodEngine::compute_mixture_gradients(
            tree, aln, base, bl, omegas_test, weights_test, syn_rates, syn_weights, &test, -1.0, false,
            /*zero_likelihood_sentinel=*/true, false, omegas_bg, weights_bg);
        if (out_pattern_ll) *out_pattern_ll = r.site_log_likelihoods;
        return r.log_likelihood;
    }

    // busted.hpp:662-975 (eps_sink = 0): the E-step for the omega-class weights
    std::vector<Scalar> compute_expected_weights(Scalar s, const std::vector<Scalar>& omegas, const std::vector<Scalar>& weights,
                                                 const std::vector<Scalar>& syn_rates = {1.0},
                                                 const std::vector<Scalar>& syn_weights = {1.0},
                                                 const std::vector<Scalar>* custom_branch_lengths = nullptr, Scalar delta = 0.0,
                                                 Scalar psi = 0.0, Scalar eps_sink = 0.0, Scalar* out_new_eps_sink = nullptr,
                                                 Scalar max_eps_sink = 0.01,
                                                 const MG94Parameters* custom_base_params = nullptr) const {
        (void)max_eps_sink;
        if (out_new_eps_sink) throw std::runtime_error("BUSTEDAnalyzer (device): the error sink is not supported");
        const size_t K = omegas.size();
        if (K <= 1) return {1.0};
        const auto r = mixture(s, omegas, weights, syn_rates, syn_weights, custom_branch_lengths, delta, psi, eps_sink,
                               custom_base_params, true);
        const double total = double(count_test()) * scored_weight(r);
        std::vector<Scalar> acc(K);
        for (size_t k = 0; k < K; ++k) acc[k] = weights[k] * r.grad_weights[k];
        return normalise(acc, total, weights);
    }

    // busted.hpp:978-1134 (eps_sink = 0): the E-step for the synonymous-rate class weights
    std::vector<Scalar> compute_expected_syn_weights(Scalar s, const std::vector<Scalar>& omegas, const std::vector<Scalar>& weights,
                                                     const std::vector<Scalar>& syn_rates, const std::vector<Scalar>& syn_weights,
                                                     const std::vector<Scalar>* custom_branch_lengths = nullptr,
                                                     Scalar delta = 0.0, Scalar psi = 0.0, Scalar eps_sink = 0.0,
                                                     const MG94Parameters* custom_base_params = nullptr) const {
        const size_t M = syn_rates.size();
        if (M <= 1) return {1.0};
        const auto r = mixture(s, omegas, weights, syn_rates, syn_weights, custom_branch_lengths, delta, psi, eps_sink,
                               custom_base_params, true);
        std::vector<Scalar> acc(M);
        for (size_t m = 0; m < M; ++m) acc[m] = syn_weights[m] * r.grad_syn_weights[m];
        return normalise(acc, scored_weight(r), syn_weights);
    }

    // busted.hpp:220-258: nucleotide GTR fit, then the full MG94 fit from its rates (100 iterations,
    // tolerance 1e-4; a separate background omega when a test set is given), then the analyzer on that tree
    static BUSTEDAnalyzer create_and_fit(Tree raw_tree, Alignment aln, const std::vector<bool>* is_test_branch_ptr = nullptr) {
        hyphy::opt::GTRFitter gtr_fitter(raw_tree, aln);
        const auto gtr = gtr_fitter.fit();
        MG94Parameters p;
        p.theta_AC = gtr.params.theta_AC; p.theta_AT = gtr.params.theta_AT; p.theta_CG = gtr.params.theta_CG;
        p.theta_CT = gtr.params.theta_CT; p.theta_GT = gtr.params.theta_GT;
        hyphy::opt::MG94Fitter mg(gtr.tree, aln);
        Scalar bg = -1.0;
        const auto fit = mg.fit_full_model(1.0, p, nullptr, 100, 1e-4, is_test_branch_ptr, is_test_branch_ptr ? &bg : nullptr);
        BUSTEDAnalyzer out(fit.tree, std::move(aln), fit.params);
        out.has_gtr_fit = true;
        out.gtr_log_l = gtr.log_likelihood;
        out.gtr_aicc = gtr.aicc;
        out.gtr_rates = gtr.params;
        for (const auto& nd : gtr.tree.nodes)
            if (nd.id != gtr.tree.root_id) out.gtr_branch_lengths[nd.name] = nd.branch_length;
        out.mg94_log_l = fit.log_likelihood;
        out.mg94_omega = fit.params.beta;
        out.mg94_background_omega = bg;
        return out;
    }

    // busted.hpp:1644-2607: K omega classes on the test branches (the last >= 1, or exactly 1 when
    // constrained; the others in [0, 1]; K = 1: one omega, <= 1 when constrained), optionally M synonymous
    // rate classes of mean 1, every branch length free (refine_branches) or one tree scale, and the five
    // nucleotide exchangeabilities (re-polished by the reference too, busted.hpp:2375-2403).  Starts: a few
    // fixed class layouts around the MG94 omega and, when given, warm_start_fit's distribution and lengths;
    // each is screened by a short joint L-BFGS run and the best one is run to convergence.
    BUSTEDFit fit_model(bool is_constrained, size_t K = 3, bool refine_branches = true, bool srv = false,
                        size_t num_syn_rates = 3, const std::string& multiple_hits = "None",
                        const BUSTEDFit* warm_start_fit = nullptr) const {
        if (!multiple_hits.empty() && multiple_hits != "None")
            throw std::runtime_error("BUSTEDAnalyzer (device): multiple hits are not supported");
        K = std::max<size_t>(1, K);
        const size_t M = srv ? std::max<size_t>(1, num_syn_rates) : 1;
        const size_t n = tree.num_nodes();
        std::vector<bool> test(is_test_branch);
        test.resize(n, true);
        if (tree.root_id >= 0) test[size_t(tree.root_id)] = false;
        std::vector<int32_t> br;
        bool has_bg = false;
        for (const auto& nd : tree.nodes) {
            if (nd.id == tree.root_id) continue;
            if (!test[size_t(nd.id)]) has_bg = true;
            br.push_back(nd.id);
        }
        const size_t nb = br.size();
        // two-set model (busted.hpp:4344-5087): background branches get their own K-class distribution, free in
        // both the unconstrained and the constrained fit; its coordinates follow the exchangeabilities
        const size_t n_bom = has_bg ? K : 0, n_bw = has_bg ? K - 1 : 0;
        // coordinates: lengths (log), omegas, class-weight sticks, log rate ratios, rate-weight sticks
        const size_t n_len = refine_branches ? nb : 1;
        const bool last_free = !is_constrained && K >= 2;
        const size_t n_om = K == 1 ? 1 : (K - 1) + (last_free ? 1 : 0);
        const size_t i_om = n_len, i_w = i_om + n_om, i_r = i_w + (K - 1), i_q = i_r + (M - 1), i_th = i_q + (M - 1),
                     i_bom = i_th + 5, i_bw = i_bom + n_bom, dim = i_bw + n_bw;
        auto bom_is_log = [&](size_t j) { return j == K - 1; };   // K = 1: one free omega on a log scale
        std::vector<Scalar> lb(dim), ub(dim);
        for (size_t i = 0; i < n_len; ++i) {
            lb[i] = std::log(refine_branches ? 1e-8 : 1e-4);
            ub[i] = std::log(refine_branches ? 1e4 : 100.0);
        }
        // K = 1: omega itself (direct in [0, 1] when constrained, log otherwise); K >= 2: lower classes direct in
        // [0, 1], the last on a log scale in [1, 1e4]
        auto om_is_log = [&](size_t j) { return K == 1 ? !is_constrained : j == K - 1; };
        for (size_t j = 0; j < n_om; ++j) {
            if (om_is_log(j)) { lb[i_om + j] = std::log(K == 1 ? 1e-5 : 1.0); ub[i_om + j] = std::log(1e4); }
            else { lb[i_om + j] = 0.0; ub[i_om + j] = 1.0; }
        }
        for (size_t j = i_w; j < i_r; ++j) { lb[j] = 0.0; ub[j] = 1.0; }
        for (size_t j = i_r; j < i_q; ++j) { lb[j] = std::log(1e-4); ub[j] = std::log(1e4); }
        for (size_t j = i_q; j < i_th; ++j) { lb[j] = 0.0; ub[j] = 1.0; }
        for (size_t j = i_th; j < i_bom; ++j) { lb[j] = std::log(1e-4); ub[j] = std::log(1e4); }
        for (size_t j = 0; j < n_bom; ++j) {
            if (bom_is_log(j)) { lb[i_bom + j] = std::log(K == 1 ? 1e-5 : 1.0); ub[i_bom + j] = std::log(1e4); }
            else { lb[i_bom + j] = 0.0; ub[i_bom + j] = 1.0; }
        }
        for (size_t j = i_bw; j < dim; ++j) { lb[j] = 0.0; ub[j] = 1.0; }

        std::vector<Scalar> base_len(n, 0.0);   // the tree-scale mode scales these
        for (int32_t id : br) base_len[size_t(id)] = branch_tau[size_t(id)];
        struct Point { std::vector<Scalar> bl, om, w, r, q, bom, bw; Scalar scale = 1.0; MG94Parameters base; };
        auto sticks = [](const std::vector<Scalar>& x, size_t off, size_t cnt) {
            std::vector<Scalar> w(cnt + 1);
            Scalar rem = 1.0;
            for (size_t k = 0; k < cnt; ++k) { w[k] = rem * x[off + k]; rem -= w[k]; }
            w[cnt] = std::max<Scalar>(rem, 0.0);
            return w;
        };
        auto to_sticks = [](const std::vector<Scalar>& w, std::vector<Scalar>& x, size_t off) {
            Scalar rem = 1.0;
            for (size_t k = 0; k + 1 < w.size(); ++k) {
                x[off + k] = rem > 1e-300 ? std::clamp(w[k] / rem, 0.0, 1.0) : 0.0;
                rem -= w[k];
            }
        };
        auto decode = [&](const std::vector<Scalar>& x) {
            Point pt;
            pt.bl.assign(n, 0.0);
            if (refine_branches) for (size_t i = 0; i < nb; ++i) pt.bl[size_t(br[i])] = std::exp(x[i]);
            else { pt.scale = std::exp(x[0]); for (int32_t id : br) pt.bl[size_t(id)] = pt.scale * base_len[size_t(id)]; }
            pt.om.assign(K, 1.0);
            for (size_t j = 0; j < n_om; ++j) pt.om[j] = om_is_log(j) ? std::exp(x[i_om + j]) : x[i_om + j];
            pt.w = sticks(x, i_w, K - 1);
            pt.q = sticks(x, i_q, M - 1);
            pt.r.assign(M, 1.0);
            for (size_t m = 0; m + 1 < M; ++m) pt.r[m] = std::exp(x[i_r + m]);
            Scalar mean = 0.0;
            for (size_t m = 0; m < M; ++m) mean += pt.q[m] * pt.r[m];
            if (mean > 1e-300) for (auto& v : pt.r) v /= mean;
            pt.base = base_params;
            pt.base.theta_AC = std::exp(x[i_th]); pt.base.theta_AT = std::exp(x[i_th + 1]); pt.base.theta_CG = std::exp(x[i_th + 2]);
            pt.base.theta_CT = std::exp(x[i_th + 3]); pt.base.theta_GT = std::exp(x[i_th + 4]);
            if (has_bg) {
                pt.bom.resize(K);
                for (size_t j = 0; j < K; ++j) pt.bom[j] = bom_is_log(j) ? std::exp(x[i_bom + j]) : x[i_bom + j];
                pt.bw = sticks(x, i_bw, K - 1);
            }
            return pt;
        };
        auto encode = [&](const std::vector<Scalar>& bl, Scalar scale, const std::vector<Scalar>& om, const std::vector<Scalar>& w,
                          const std::vector<Scalar>& r, const std::vector<Scalar>& q, const MG94Parameters& th,
                          const std::vector<Scalar>& bom = {}, const std::vector<Scalar>& bw = {}) {
            std::vector<Scalar> x(dim, 0.0);
            if (refine_branches) for (size_t i = 0; i < nb; ++i) x[i] = std::log(std::max<Scalar>(bl[size_t(br[i])], 1e-8));
            else x[0] = std::log(scale);
            for (size_t j = 0; j < n_om; ++j) x[i_om + j] = om_is_log(j) ? std::log(std::max<Scalar>(om[j], 1e-300)) : om[j];
            to_sticks(w, x, i_w);
            for (size_t m = 0; m + 1 < M; ++m) x[i_r + m] = std::log(r[m] / r[M - 1]);
            to_sticks(q, x, i_q);
            const Scalar t5[5] = {th.theta_AC, th.theta_AT, th.theta_CG, th.theta_CT, th.theta_GT};
            for (size_t j = 0; j < 5; ++j) x[i_th + j] = std::log(std::max<Scalar>(t5[j], 1e-300));
            if (has_bg) {
                for (size_t j = 0; j < K; ++j) {
                    const Scalar v = j < bom.size() ? bom[j] : 1.0;
                    x[i_bom + j] = bom_is_log(j) ? std::log(std::max<Scalar>(v, 1e-300)) : v;
                }
                if (bw.size() == K) to_sticks(bw, x, i_bw);
            }
            for (size_t j = 0; j < dim; ++j) x[j] = std::clamp(x[j], lb[j], ub[j]);
            return x;
        };
        auto evaluate = [&](const Point& pt, bool grads) {
            return hyphy::core::LikelihoodEngine::compute_mixture_gradients(
                tree, aln, pt.base, pt.bl, pt.om, pt.w, pt.r, pt.q, &test, -1.0, grads,
                /*zero_likelihood_sentinel=*/true, /*direction_gradients=*/grads, pt.bom, pt.bw);
        };
        // objective -lnL and its gradient in the coordinates above
        auto fg = [&](const std::vector<Scalar>& x, std::vector<Scalar>& g) -> Scalar {
            const Point pt = decode(x);
            const auto r = evaluate(pt, true);
            g.assign(dim, 0.0);
            if (refine_branches) {
                for (size_t i = 0; i < nb; ++i) g[i] = -pt.bl[size_t(br[i])] * r.grad_branches[size_t(br[i])];
            } else {
                Scalar d = 0.0;
                for (int32_t id : br) d += pt.bl[size_t(id)] * r.grad_branches[size_t(id)];
                g[0] = -d;
            }
            for (size_t j = 0; j < n_om; ++j) g[i_om + j] = -(om_is_log(j) ? pt.om[j] : 1.0) * r.grad_omegas[j];
            // w_k = R_k p_k (k < K-1), w_{K-1} = R_{K-1}, R_k = prod_{i<k} (1 - p_i)
            auto stick_grad = [&](size_t off, const std::vector<Scalar>& gw) {
                for (size_t j = 0; j + 1 < K; ++j) {
                    Scalar d = 0.0;
                    for (size_t k = j; k < K; ++k) {
                        Scalar dw = 1.0;
                        for (size_t i = 0; i < k; ++i) dw *= (i == j) ? -1.0 : (1.0 - x[off + i]);
                        if (k + 1 < K && k != j) dw *= x[off + k];
                        d += gw[k] * dw;
                    }
                    g[off + j] = -d;
                }
            };
            stick_grad(i_w, r.grad_weights);
            if (has_bg) {
                for (size_t j = 0; j < K; ++j) g[i_bom + j] = -(bom_is_log(j) ? pt.bom[j] : 1.0) * r.grad_bg_omegas[j];
                stick_grad(i_bw, r.grad_bg_weights);
            }
            // rate-weight sticks, exactly: r_m = r~_m / sum_k rho_k r~_k, and sum_m r_m dlnL/dr_m (at fixed rho) equals
            // sum_b t_b dlnL/dt_b (every rate scales every branch), so
            // dlnL/dq_j = sum_m G^rho_m drho_m/dq_j - E (sum_k r~_k drho_k/dq_j) / mean
            if (M > 1) {
                Scalar E = 0.0;
                for (int32_t id : br) E += pt.bl[size_t(id)] * r.grad_branches[size_t(id)];
                Scalar mean = 0.0;
                std::vector<Scalar> rt(M, 1.0);
                for (size_t m = 0; m + 1 < M; ++m) rt[m] = std::exp(x[i_r + m]);
                for (size_t m = 0; m < M; ++m) mean += pt.q[m] * rt[m];
                for (size_t j = 0; j + 1 < M; ++j) {
                    Scalar d1 = 0.0, d2 = 0.0;
                    for (size_t k = j; k < M; ++k) {
                        Scalar dq = 1.0;
                        for (size_t i = 0; i < k; ++i) dq *= (i == j) ? -1.0 : (1.0 - x[i_q + i]);
                        if (k + 1 < M && k != j) dq *= x[i_q + k];
                        d1 += r.grad_syn_weights[k] * dq;
                        d2 += rt[k] * dq;
                    }
                    g[i_q + j] = -(d1 - E * d2 / mean);
                }
            }
            const Scalar t5[5] = {pt.base.theta_AC, pt.base.theta_AT, pt.base.theta_CG, pt.base.theta_CT, pt.base.theta_GT};
            for (size_t j = 0; j < 5; ++j) g[i_th + j] = -t5[j] * r.grad_theta[j];
            for (size_t j = i_r; j < i_q; ++j) {        // log rate ratios: central differences of the device likelihood
                std::vector<Scalar> xp = x, xm = x;
                xp[j] = std::min(ub[j], x[j] + 1e-4);
                xm[j] = std::max(lb[j], x[j] - 1e-4);
                if (xp[j] > xm[j])
                    g[j] = -(evaluate(decode(xp), false).log_likelihood - evaluate(decode(xm), false).log_likelihood) / (xp[j] - xm[j]);
            }
            return -r.log_likelihood;
        };

        // starting points
        std::vector<Scalar> r0(M, 1.0), q0(M, 1.0 / Scalar(M));
        if (M == 2) { r0 = {0.35, 1.65}; q0 = {0.5, 0.5}; }
        else if (M == 3) { r0 = {0.3, 1.0, 3.1}; q0 = {0.3, 0.6, 0.1}; }
        else if (M >= 4) for (size_t m = 0; m < M; ++m) r0[m] = 0.15 * std::pow(25.0, Scalar(m) / Scalar(M - 1));
        const Scalar om_mg = std::clamp(mg94_omega, 0.05, 0.9);
        std::vector<Scalar> bom0, bw0;
        if (has_bg) {
            const Scalar obg = std::clamp(mg94_background_omega >= 0.0 ? mg94_background_omega : mg94_omega, 0.01, 0.9);
            if (K == 1) { bom0 = {obg}; bw0 = {1.0}; }
            else {
                for (size_t k = 0; k + 1 < K; ++k) {
                    bom0.push_back(K == 2 ? obg : 0.05 + (obg - 0.05) * Scalar(k) / Scalar(K - 2));
                    bw0.push_back(0.95 / Scalar(K - 1));
                }
                bom0.push_back(1.5);
                bw0.push_back(0.05);
            }
        }
        std::vector<std::vector<Scalar>> starts;
        if (K == 1) {
            starts.push_back(encode(base_len, 1.0, {is_constrained ? std::min<Scalar>(1.0, mg94_omega) : std::max<Scalar>(mg94_omega, 1e-5)},
                                    {1.0}, r0, q0, base_params, bom0, bw0));
        } else {
            const Scalar lo[5] = {0.1, 0.01, 0.0, 0.05, 0.0}, hi[5] = {0.5, om_mg, 0.3, 0.8, 0.1},
                         top[5] = {2.0, 3.0, 1.5, 10.0, 2.0}, wtop[5] = {0.1, 0.1, 0.2, 0.05, 0.5};
            for (int j = 0; j < 5; ++j) {
                std::vector<Scalar> om(K), w(K);
                for (size_t k = 0; k + 1 < K; ++k) {
                    om[k] = K == 2 ? 0.5 * (lo[j] + hi[j]) : lo[j] + (hi[j] - lo[j]) * Scalar(k) / Scalar(K - 2);
                    w[k] = (1.0 - wtop[j]) / Scalar(K - 1);
                }
                om[K - 1] = is_constrained ? 1.0 : top[j];
                w[K - 1] = wtop[j];
                starts.push_back(encode(base_len, 1.0, om, w, r0, q0, base_params, bom0, bw0));
            }
        }
        if (warm_start_fit && warm_start_fit->test_distribution.omegas.size() == K) {
            const auto& d = warm_start_fit->test_distribution;
            std::vector<Scalar> om = d.omegas;
            for (size_t k = 0; k + 1 < K; ++k) om[k] = std::min<Scalar>(om[k], 1.0);
            if (K == 1) om[0] = is_constrained ? std::min<Scalar>(om[0], 1.0) : std::max<Scalar>(om[0], 1e-5);
            else om[K - 1] = is_constrained ? 1.0 : std::max<Scalar>(om[K - 1], 1.0);
            const bool rates_fit = d.syn_rates.size() == M && d.syn_weights.size() == M;
            const auto& bl = warm_start_fit->branch_lengths.size() == n ? warm_start_fit->branch_lengths : base_len;
            starts.push_back(encode(bl, warm_start_fit->tree_scale, om, d.weights, rates_fit ? d.syn_rates : r0,
                                    rates_fit ? d.syn_weights : q0,
                                    warm_start_fit->has_gtr_params ? warm_start_fit->gtr_params : base_params,
                                    warm_start_fit->background_distribution.omegas.size() == K ? warm_start_fit->background_distribution.omegas : bom0,
                                    warm_start_fit->background_distribution.weights.size() == K ? warm_start_fit->background_distribution.weights : bw0));
        }
        hyphy::opt::BoxLBFGSResult best;
        best.f = std::numeric_limits<Scalar>::infinity();
        for (const auto& x0 : starts) {
            auto r = hyphy::opt::box_lbfgs(fg, x0, lb, ub, 1e-5, starts.size() > 1 ? 40 : 1000);
            if (std::isfinite(r.f) && r.f < best.f) best = std::move(r);
        }
        if (!std::isfinite(best.f)) throw std::runtime_error("BUSTEDAnalyzer (device): every start has a zero likelihood");
        int total_it = best.iterations;
        if (starts.size() > 1) {
            auto r = hyphy::opt::box_lbfgs(fg, best.x, lb, ub, 1e-5, 1000);
            total_it += r.iterations;
            if (std::isfinite(r.f) && r.f <= best.f) best = std::move(r);
        }

        const Point pt = decode(best.x);
        const auto fin = evaluate(pt, false);
        BUSTEDFit fit;
        fit.num_rate_classes = K;
        fit.log_likelihood = fin.log_likelihood;
        fit.site_log_likelihoods = fin.site_log_likelihoods;
        fit.branch_lengths = pt.bl;
        fit.tree_scale = pt.scale;
        fit.iterations = total_it;
        fit.has_gtr_params = true;
        fit.gtr_params = pt.base;
        // lower classes in increasing omega (their labels are exchangeable); rate classes likewise
        std::vector<size_t> idx(K);
        for (size_t k = 0; k < K; ++k) idx[k] = k;
        if (K > 2) std::sort(idx.begin(), idx.end() - 1, [&](size_t a, size_t b) { return pt.om[a] < pt.om[b]; });
        for (size_t k : idx) { fit.test_distribution.omegas.push_back(pt.om[k]); fit.test_distribution.weights.push_back(pt.w[k]); }
        if (has_bg) {
            std::vector<size_t> ib(K);
            for (size_t k = 0; k < K; ++k) ib[k] = k;
            if (K > 2) std::sort(ib.begin(), ib.end() - 1, [&](size_t a, size_t b) { return pt.bom[a] < pt.bom[b]; });
            fit.has_background_distribution = true;
            for (size_t k : ib) {
                fit.background_distribution.omegas.push_back(pt.bom[k]);
                fit.background_distribution.weights.push_back(pt.bw[k]);
            }
        }
        if (srv) {
            std::vector<size_t> im(M);
            for (size_t m = 0; m < M; ++m) im[m] = m;
            std::sort(im.begin(), im.end(), [&](size_t a, size_t b) { return pt.r[a] < pt.r[b]; });
            for (size_t m : im) { fit.test_distribution.syn_rates.push_back(pt.r[m]); fit.test_distribution.syn_weights.push_back(pt.q[m]); }
        }
        auto& ann = fit.test_distribution.annotations;
        ann.assign(K, "");
        for (size_t k = 0; k < K; ++k)
            if (fit.test_distribution.weights[k] < 0.005) ann[k] = "Rate class " + std::to_string(k) + " collapsed (weight < 0.5%)";
        for (size_t k = 0; k + 1 < K; ++k)
            if (ann[k].empty() && std::fabs(fit.test_distribution.omegas[k + 1] - fit.test_distribution.omegas[k]) < 0.015)
                ann[k] = "Rate classes " + std::to_string(k) + " and " + std::to_string(k + 1) + " collapsed into identical omega";
        // busted.hpp:2598-2605: 5 exchangeabilities + 9 frequency parameters, lengths (or a scale), mixture and
        // synonymous-rate parameters; N = codons x taxa
        const size_t n_mix = (2 * K - 1) - (is_constrained && K >= 2 ? 1 : 0) + (has_bg ? 2 * K - 1 : 0);
        const size_t k_params = 14 + (refine_branches ? nb : 1) + n_mix + (srv ? 2 * (M - 1) : 0);
        fit.aicc = hyphy::opt::compute_aicc(fit.log_likelihood, k_params, aln.num_codons * aln.num_taxa);
        return fit;
    }

    // busted.hpp:3115-3142: the null model for K = 1 .. max_k; K grows while AICc drops by more than 2
    std::pair<size_t, std::vector<BUSTEDFit>> select_optimal_k(size_t max_k = 3, bool refine_branches = true, bool srv = false,
                                                              size_t num_syn_rates = 3,
                                                              const std::string& multiple_hits = "None") const {
        std::vector<BUSTEDFit> nulls;
        for (size_t k = 1; k <= std::max<size_t>(1, max_k); ++k)
            nulls.push_back(fit_model(true, k, refine_branches, srv, num_syn_rates, multiple_hits));
        size_t best = 1;
        for (size_t k = 2; k <= nulls.size(); ++k)
            if (nulls[k - 1].aicc < nulls[best - 1].aicc - 2.0) best = k;
        return {best, std::move(nulls)};
    }

    // busted.hpp:5969-6682, standard all-branch BUSTED: the unconstrained fit, the constrained fit warm-started from
    // it, the unconstrained refit from the constrained one while that is higher; LRT with the 0.5 chi2_0 +
    // 0.5 chi2_2 null (K >= 2; K = 1: one-sided chi2_1 with omega <= 1 under the null); per-site evidence ratios
    BUSTEDResult run(BUSTEDSettings settings = {}, bool show_progress = false, bool force_progress = false) const {
        (void)show_progress; (void)force_progress;
        const auto t0 = std::chrono::steady_clock::now();
        if (settings.full_auto || settings.error_sink || settings.phenotype_mode || settings.relax_mode)
            throw std::runtime_error("BUSTEDAnalyzer (device): full automatic selection, the error sink, BUSTED-PH and RELAX modes are not supported");
        const auto sel = tree.select_branches(settings.test_branches, "", {}, false);
        is_test_branch = sel.is_selected;
        num_test_branches = sel.num_selected;
        num_background_branches = sel.num_unselected;
        BUSTEDResult res;
        res.settings = settings;
        const size_t K = std::max<size_t>(1, settings.num_rate_classes);
        res.optimal_k = K;
        const bool refine = settings.refine_branch_lengths, srv = settings.srv;
        const size_t M = settings.num_syn_rate_classes;
        if (settings.auto_select_k) {
            // busted.hpp:6339-6412 with select_optimal_k (:3115-3142): null fits for K = 1 .. max_k, a class added
            // only when it lowers AICc by more than 2; the alternative from the chosen null, the null again from it
            auto [opt_k, nulls] = select_optimal_k(settings.max_k, refine, srv, M, settings.multiple_hits);
            res.optimal_k = opt_k;
            res.k_null_fits = std::move(nulls);
            res.constrained = res.k_null_fits[opt_k - 1];
            res.unconstrained = fit_model(false, opt_k, refine, srv, M, settings.multiple_hits, &res.constrained);
            if (opt_k >= 2) {
                BUSTEDFit null2 = fit_model(true, opt_k, refine, srv, M, settings.multiple_hits, &res.unconstrained);
                if (null2.log_likelihood > res.constrained.log_likelihood) res.constrained = std::move(null2);
            }
        } else {
            res.unconstrained = fit_model(false, K, refine, srv, M, settings.multiple_hits);
            res.constrained = fit_model(true, K, refine, srv, M, settings.multiple_hits, &res.unconstrained);
        }
        const size_t Kf = res.optimal_k;
        // the alternative contains the null: refit it from the null with the last omega moved above 1
        for (int retry = 0; retry < 2 && Kf >= 2; ++retry) {
            BUSTEDFit from_null = res.constrained;
            from_null.test_distribution.omegas.back() = 1.5;
            BUSTEDFit alt = fit_model(false, Kf, refine, srv, M, settings.multiple_hits, &from_null);
            const bool better = alt.log_likelihood > res.unconstrained.log_likelihood + 1e-6;
            if (better) res.unconstrained = std::move(alt);
            if (!better || res.constrained.log_likelihood <= res.unconstrained.log_likelihood + 1e-5) break;
        }
        const bool failed = !(res.unconstrained.log_likelihood > -1e19) || !(res.constrained.log_likelihood > -1e19);
        if (failed) {
            res.is_failed = true;
            res.error_message = "Optimization failed: model log-likelihood collapsed to the zero-likelihood sentinel.";
            res.lrt = 0.0;
            res.p_value = 1.0;
        } else if (Kf == 1) {
            if (res.unconstrained.test_distribution.omegas[0] <= 1.0 ||
                res.unconstrained.log_likelihood <= res.constrained.log_likelihood) {
                res.constrained = res.unconstrained;
                res.lrt = 0.0;
                res.p_value = 0.5;
            } else {
                res.lrt = 2.0 * (res.unconstrained.log_likelihood - res.constrained.log_likelihood);
                res.p_value = 0.5 * std::erfc(std::sqrt(0.5 * res.lrt));
            }
        } else if (res.unconstrained.log_likelihood <= res.constrained.log_likelihood) {
            const Scalar penalty = res.unconstrained.aicc + 2.0 * res.unconstrained.log_likelihood;
            res.unconstrained = res.constrained;
            res.unconstrained.aicc = -2.0 * res.unconstrained.log_likelihood + penalty;
            res.lrt = 0.0;
            res.p_value = 0.5;
        } else {
            res.lrt = 2.0 * (res.unconstrained.log_likelihood - res.constrained.log_likelihood);
            res.p_value = 0.5 * std::exp(-0.5 * res.lrt);
        }
        const size_t n_sites = aln.num_codons;
        res.evidence_ratios.assign(n_sites, 1.0);
        res.constrained_evidence_ratios.assign(n_sites, 1.0);
        if (!res.is_failed) {
            const auto& u = res.unconstrained.test_distribution;
            std::vector<Scalar> om = u.omegas;
            om.back() = std::min<Scalar>(1.0, om.back());
            const auto& uf = res.unconstrained;
            std::vector<bool> test(is_test_branch);
            test.resize(tree.num_nodes(), true);
            if (tree.root_id >= 0) test[size_t(tree.root_id)] = false;
            const auto cl = hyphy::core::LikelihoodEngine::compute_mixture_gradients(
                tree, aln, uf.has_gtr_params ? uf.gtr_params : base_params, uf.branch_lengths, om, u.weights,
                u.syn_rates.empty() ? std::vector<Scalar>{1.0} : u.syn_rates,
                u.syn_weights.empty() ? std::vector<Scalar>{1.0} : u.syn_weights, &test, -1.0, false,
                /*zero_likelihood_sentinel=*/true, false, uf.background_distribution.omegas, uf.background_distribution.weights);
            const std::vector<Scalar>& clamped = cl.site_log_likelihoods;
            for (size_t st = 0; st < n_sites; ++st) {
                const size_t p = size_t(aln.site_to_pattern[st]);
                const Scalar alt = res.unconstrained.site_log_likelihoods[p];
                res.evidence_ratios[st] = std::exp(std::clamp(alt - res.constrained.site_log_likelihoods[p], -200.0, 200.0));
                res.constrained_evidence_ratios[st] = std::exp(std::clamp(alt - clamped[p], -200.0, 200.0));
            }
        }
        res.runtime_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return res;
    }

private:
    hyphy::core::MixtureGradients mixture(Scalar s, const std::vector<Scalar>& omegas, const std::vector<Scalar>& weights,
                                          const std::vector<Scalar>& syn_rates, const std::vector<Scalar>& syn_weights,
                                          const std::vector<Scalar>* custom_branch_lengths, Scalar delta, Scalar psi,
                                          Scalar eps_sink, const MG94Parameters* custom_base_params, bool weight_grads) const {
        if (eps_sink != 0.0) throw std::runtime_error("BUSTEDAnalyzer (device): the error sink is not supported");
        MG94Parameters base = custom_base_params ? *custom_base_params : base_params;
        base.delta = delta;
        base.psi = psi;
        const size_t n = tree.num_nodes();
        std::vector<Scalar> bl(n, 0.0);
        for (const auto& node : tree.nodes)
            if (node.id != tree.root_id)
                bl[size_t(node.id)] = s * (custom_branch_lengths ? (*custom_branch_lengths)[size_t(node.id)] : branch_tau[size_t(node.id)]);
        std::vector<bool> test(is_test_branch);
        test.resize(n, true);
        if (tree.root_id >= 0) test[size_t(tree.root_id)] = false;
        bool has_bg = false;
        for (const auto& node : tree.nodes)
            if (node.id != tree.root_id && !test[size_t(node.id)]) has_bg = true;
        const Scalar omega_bg = has_bg ? (mg94_background_omega >= 0.0 ? mg94_background_omega : mg94_omega) : -1.0;
        return hyphy::core::LikelihoodEngine::compute_mixture_gradients(
            tree, aln, base, bl, omegas, weights, syn_rates, syn_weights, &test, omega_bg, weight_grads,
            /*zero_likelihood_sentinel=*/true, /*direction_gradients=*/false);
    }

    size_t count_test() const {
        size_t c = 0;
        for (const auto& node : tree.nodes)
            if (node.id != tree.root_id && size_t(node.id) < is_test_branch.size() && is_test_branch[size_t(node.id)]) ++c;
        return c;
    }

    // total weight of the patterns with a positive likelihood (the reference's pat_wt_accum)
    double scored_weight(const hyphy::core::MixtureGradients& r) const {
        double t = 0.0;
        for (size_t p = 0; p < aln.patterns.size(); ++p)
            if (r.site_log_likelihoods[p] > -1e19) t += double(aln.patterns[p].weight);
        return t;
    }

    static std::vector<Scalar> normalise(std::vector<Scalar> acc, double total, const std::vector<Scalar>& old) {
        if (!(total > 0.0)) return old;
        double sum = 0.0;
        for (auto& x : acc) {
            x = std::clamp(x / total, 1e-6, 1.0 - 1e-6);
            sum += x;
        }
        for (auto& x : acc) x /= sum;
        return acc;
    }
};

}  // namespace hyphy::analyses
