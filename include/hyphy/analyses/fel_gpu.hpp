// fel_gpu.hpp — drop-in FELAnalyzer (include/hyphy/analyses/fel.hpp) whose
// per-site fits run on the device through h3g_fel_run.
//
// Same constructor and run() as the reference class: the constructor converts
// branch lengths to the FEL time scale (t x 3 / mean rate of the base MG94
// model, fel.hpp:230-273); run() fits every site pattern (fel.hpp:326-446)
// and maps patterns back to sites (fel.hpp:778-833).  The tested branches are
// chosen as in the reference (Tree::select_branches with {T}-tag detection,
// fel.hpp:215-227); with a background set every pattern runs the reference's
// branch-subset search (fel.hpp:462-572) through h3g_fel_run_tested.
// create_and_fit (fel.hpp:145-214) fits the nucleotide GTR model, then the
// global MG94 model from its rates, both on the device, before FEL.
// Ancestral substitution summaries (SiteResult::subs in the reference) and
// bridge resolutions are not produced.
#pragma once

#include <functional>
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

struct FELSettings {
    Scalar p_value_threshold = 0.1;
    bool full_model = true;
    bool srv = true;
    std::string test_branches = "All";
    std::string test_branch_regex = "";
    std::vector<std::string> test_branch_names = {};
};

struct SiteResult {
    size_t site_index = 0;
    Scalar alpha = 0.0;
    Scalar beta = 0.0;
    Scalar beta_nuisance = 0.0;
    Scalar alpha_null = 0.0;
    Scalar lrt = 0.0;
    Scalar p_value = 1.0;
    Scalar total_branch_length = 0.0;
    Scalar log_l_alt = 0.0;
    Scalar log_l_null = 0.0;
    int evaluations = 0;          // likelihood evaluations of the pattern's search (0: invariant)
};

class FELAnalyzer {
public:
    Tree tree;
    Alignment aln;
    MG94Parameters base_params;
    FELSettings settings;
    Scalar p_value_threshold = 0.1;
    Scalar baseline_tree_length = 0.0;
    Scalar baseline_tested_tree_length = 0.0;
    Scalar baseline_bg_tree_length = 0.0;
    Scalar conversion_factor = 1.0;
    Scalar global_log_l = 0.0;
    Scalar global_aicc = 0.0;
    std::vector<SiteResult> site_results;

    // the nucleotide GTR fit create_and_fit starts from
    bool has_gtr_fit = false;
    Scalar gtr_log_l = 0.0;
    Scalar gtr_aicc = 0.0;
    hyphy::core::GTRParameters gtr_rates;
    std::unordered_map<std::string, Scalar> gtr_branch_lengths;
    bool full_model = true;

    // branch partition (fel.hpp:215-227)
    std::vector<bool> is_test_branch;
    std::vector<std::string> test_branch_names;
    std::vector<std::string> bg_branch_names;
    size_t num_tested = 0;
    size_t num_background = 0;
    Scalar background_omega = -1.0;

    FELAnalyzer(Tree t, Alignment a, MG94Parameters params = MG94Parameters{}, FELSettings s = FELSettings{}, Scalar bg_om = -1.0)
        : tree(std::move(t)), aln(std::move(a)), base_params(params), settings(std::move(s)), background_omega(bg_om) {
        p_value_threshold = settings.p_value_threshold;
        full_model = settings.full_model;
        prepare_branch_lengths();
    }

    // fel.hpp:145-201: GTR fit, then the global MG94 fit from its rates (every branch, omega and, with a
    // tested / background split, the background omega; or omega and a tree scale when !full_model), then
    // the analyzer on that tree.  AICc of the MG94 fit: K = 5 + (2 omegas with a split, else 1) + branches,
    // N = codons.
    static FELAnalyzer create_and_fit(Tree input_tree, Alignment aln, FELSettings settings = FELSettings{},
                                      std::function<void(const std::string&, double)> progress_cb = nullptr) {
        if (progress_cb) progress_cb("Phase 1: Fitting Nucleotide GTR Model", 0.1);
        hyphy::opt::GTRFitter gtr_fitter(input_tree, aln);
        const auto gtr = gtr_fitter.fit();
        if (progress_cb) progress_cb("Phase 2: Refining under Global MG94 Model", 0.3);
        MG94Parameters p;
        p.theta_AC = gtr.params.theta_AC; p.theta_AT = gtr.params.theta_AT; p.theta_CG = gtr.params.theta_CG;
        p.theta_CT = gtr.params.theta_CT; p.theta_GT = gtr.params.theta_GT;
        const auto sel = gtr.tree.select_branches(settings.test_branches, settings.test_branch_regex, settings.test_branch_names, true);
        const bool split = sel.num_selected > 0 && sel.num_unselected > 0;
        hyphy::opt::MG94Fitter mg(gtr.tree, aln);
        hyphy::opt::FitResult fit;
        Scalar bg_om = -1.0;
        if (settings.full_model) {
            fit = mg.fit_full_model(1.0, p, progress_cb, 250, 1e-5, split ? &sel.is_selected : nullptr, split ? &bg_om : nullptr);
            p = fit.params;
        } else {
            fit = mg.fit_omega_and_scale(1.0, p);
            p.alpha = 1.0;
            p.beta = fit.x_opt[0];
            bg_om = p.beta;
        }
        FELAnalyzer out(fit.tree, std::move(aln), p, settings, bg_om);
        out.global_log_l = fit.log_likelihood;
        out.global_aicc = hyphy::opt::compute_aicc(fit.log_likelihood, 5 + (split ? 2 : 1) + (fit.tree.num_nodes() - 1),
                                                   out.aln.num_codons);
        out.has_gtr_fit = true;
        out.gtr_log_l = gtr.log_likelihood;
        out.gtr_aicc = gtr.aicc;
        out.gtr_rates = gtr.params;
        for (const auto& nd : gtr.tree.nodes)
            if (nd.id != gtr.tree.root_id) out.gtr_branch_lengths[nd.name] = nd.branch_length;
        return out;
    }

    // fel.hpp:203-214
    static FELAnalyzer create_and_fit(Tree input_tree, Alignment aln, Scalar pvalue_threshold,
                                      std::function<void(const std::string&, double)> progress_cb = nullptr,
                                      bool full_model = true) {
        FELSettings s;
        s.p_value_threshold = pvalue_threshold;
        s.full_model = full_model;
        return create_and_fit(std::move(input_tree), std::move(aln), s, std::move(progress_cb));
    }

    void partition_branches() {
        auto sel = tree.select_branches(settings.test_branches, settings.test_branch_regex, settings.test_branch_names, true);
        is_test_branch = std::move(sel.is_selected);
        test_branch_names = std::move(sel.selected_names);
        bg_branch_names = std::move(sel.unselected_names);
        num_tested = sel.num_selected;
        num_background = sel.num_unselected;
    }

    // fel.hpp:230-273: tested branches t x 3 / mean rate of the base model; background ones
    // by the mean rate at omega = background_omega when that is > 0
    void prepare_branch_lengths() {
        partition_branches();
        const auto& code = aln.code ? *aln.code : *hyphy::core::GeneticCode::universal();
        MG94Matrix base;
        base.update(base_params, aln.pos_nuc_frequencies, aln.codon_frequencies_f3x4, code);
        conversion_factor = base.scale_factor > 1e-12 ? 3.0 / base.scale_factor : 1.0;
        Scalar bg_conv = conversion_factor;
        if (num_background > 0 && background_omega > 0.0) {
            MG94Parameters pbg = base_params;
            pbg.alpha = 1.0;
            pbg.beta = background_omega;
            MG94Matrix mbg;
            mbg.update(pbg, aln.pos_nuc_frequencies, aln.codon_frequencies_f3x4, code);
            if (mbg.scale_factor > 1e-12) bg_conv = 3.0 / mbg.scale_factor;
        }
        baseline_tree_length = baseline_tested_tree_length = baseline_bg_tree_length = 0.0;
        for (auto& node : tree.nodes) {
            if (node.id == tree.root_id) continue;
            baseline_tree_length += node.branch_length;
            if (is_test_branch[size_t(node.id)]) {
                baseline_tested_tree_length += node.branch_length;
                node.branch_length *= conversion_factor;
            } else {
                baseline_bg_tree_length += node.branch_length;
                node.branch_length *= bg_conv;
            }
        }
    }

    std::vector<SiteResult> run(bool show_progress = false, bool force_progress = false) {
        (void)show_progress; (void)force_progress;
        auto& eng = hyphy::core::gpu_detail::Engine::get();
        const auto l2t = hyphy::core::LikelihoodEngine::build_leaf_to_taxon_map(tree, aln);
        h3g_problem* pr = eng.problem(tree, aln, l2t);
        const auto& code = aln.code ? *aln.code : *hyphy::core::GeneticCode::universal();
        const int S = code.num_sense_codons;
        MG94Parameters ps = base_params, pn = base_params;
        ps.alpha = 1.0; ps.beta = 0.0;
        pn.alpha = 0.0; pn.beta = 1.0;
        MG94Matrix ms, mn;
        ms.update(ps, aln.pos_nuc_frequencies, aln.codon_frequencies_f3x4, code);
        mn.update(pn, aln.pos_nuc_frequencies, aln.codon_frequencies_f3x4, code);
        const size_t nS = static_cast<size_t>(S);
        std::vector<double> pi(nS), qs(nS * nS), qn(nS * nS), bl(tree.num_nodes(), 0.0);
        for (int i = 0; i < S; ++i) {
            pi[size_t(i)] = aln.codon_frequencies_f3x4[size_t(i)];
            for (int j = 0; j < S; ++j) {
                qs[size_t(i) * S + j] = i == j ? 0.0 : ms.Q(i, j);
                qn[size_t(i) * S + j] = i == j ? 0.0 : mn.Q(i, j);
            }
        }
        for (const auto& node : tree.nodes)
            if (node.id != tree.root_id) bl[size_t(node.id)] = node.branch_length;
        h3g_fel_model m{S, pi.data(), qs.data(), qn.data()};
        std::vector<h3g_fel_result> res(aln.patterns.size());
        std::vector<uint8_t> tested(tree.num_nodes(), 1);
        for (const auto& node : tree.nodes)
            if (node.id != tree.root_id) tested[size_t(node.id)] = is_test_branch[size_t(node.id)] ? 1 : 0;
        eng.check(h3g_fel_run_tested(pr, &m, bl.data(), tested.data(), res.data()));
        site_results.assign(aln.num_codons, SiteResult{});
        for (size_t s = 0; s < aln.num_codons; ++s) {
            const auto& r = res[aln.site_to_pattern[s]];
            SiteResult& o = site_results[s];
            o.site_index = s;
            o.alpha = r.alpha; o.beta = r.beta; o.beta_nuisance = r.beta_nuisance; o.alpha_null = r.alpha_null;
            o.lrt = r.lrt; o.p_value = r.p_value;
            o.log_l_alt = r.log_l_alt; o.log_l_null = r.log_l_null;
            o.total_branch_length = r.alpha_null * baseline_tested_tree_length;
            o.evaluations = r.evaluations;
        }
        return site_results;
    }
};

}  // namespace hyphy::analyses
