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
// is_test_branch, num_test_branches, mg94_omega, mg94_background_omega).  Not provided: the
// error sink (eps_sink must be 0), bridge resolutions, fit_model / run / create_and_fit
// (the EM driver and model selection around these steps).
#pragma once

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "../core/likelihood_gpu.hpp"

namespace hyphy::analyses {

using hyphy::core::Alignment;
using hyphy::core::MG94Matrix;
using hyphy::core::MG94Parameters;
using hyphy::core::Scalar;
using hyphy::core::Tree;

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
