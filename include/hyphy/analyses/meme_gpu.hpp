// meme_gpu.hpp — drop-in MEMEAnalyzer (include/hyphy/analyses/meme.hpp) whose
// per-site fits run on the device through h3g_meme_run.
//
// Same constructor and run() as the reference class: the constructor converts
// branch lengths to the FEL time scale (t x 3 / mean rate of the base MG94
// model, meme.hpp:150-164); run() fits every site pattern (the FEL baseline,
// the 4-D alternative and 3-D null Nelder-Mead searches, LRT, empirical Bayes
// factors; meme.hpp:166-632) and maps patterns back to sites
// (meme.hpp:634-676).  The tested branches follow the reference
// (meme.hpp:84-92): MEME's own set by Tree::select_branches without tag
// detection, its FEL baseline's with detection; with a background set the
// search frees beta_bg (h3g_meme_run_tested).  create_and_fit (meme.hpp:95-148)
// fits the nucleotide GTR model, then the global MG94 model, on the device.
// Bridge resolutions and the ancestral substitution summaries
// (MEMESiteResult::subs) are not provided.
#pragma once

#include <functional>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "fel_gpu.hpp"

namespace hyphy::analyses {

struct MEMESiteResult {
    size_t site_index = 0;
    Scalar alpha = 0.0;
    Scalar beta1 = 0.0;
    Scalar p1 = 1.0;
    Scalar beta_plus = 0.0;
    Scalar p_plus = 0.0;
    Scalar lrt = 0.0;
    Scalar p_value = 1.0;
    int branches_under_selection = 0;
    Scalar total_branch_length = 0.0;
    Scalar log_l_meme = 0.0;
    Scalar log_l_fel = 0.0;
    Scalar p_value_meme_vs_fel = 1.0;
    Scalar fel_alpha = 0.0;
    Scalar fel_beta = 0.0;
    Scalar beta_bg = 0.0;
    std::vector<Scalar> branch_ebf;   // per node id, 1 for the root and where no EBF is computed
    int evaluations = 0;              // likelihood evaluations of the MEME search (0: invariant)
};

class MEMEAnalyzer {
public:
    Tree tree;
    Alignment aln;
    MG94Parameters base_params;
    FELAnalyzer fel_analyzer;
    Scalar p_value_threshold = 0.1;
    Scalar baseline_tree_length = 0.0;
    Scalar conversion_factor = 1.0;
    Scalar global_log_l = 0.0;
    Scalar global_aicc = 0.0;
    std::vector<MEMESiteResult> site_results;
    bool has_gtr_fit = false;
    Scalar gtr_log_l = 0.0;
    Scalar gtr_aicc = 0.0;
    hyphy::core::GTRParameters gtr_rates;
    std::unordered_map<std::string, Scalar> gtr_branch_lengths;
    std::string test_branches = "All";
    size_t num_tested = 0;
    size_t num_background = 0;

    std::vector<bool> is_test_branch;

    MEMEAnalyzer(Tree t, Alignment a, MG94Parameters params = MG94Parameters{}, std::string branches_spec = "All")
        : tree(t), aln(std::move(a)), base_params(params), fel_analyzer(t, aln, params), test_branches(std::move(branches_spec)) {
        prepare_branch_lengths();
        select_test_branches(test_branches);
    }

    // meme.hpp:95-148: the branch set is checked before any fit; GTR fit, then the global MG94 fit from its
    // rates (every branch and omega, with a separate background omega for a split; or omega and a tree scale
    // when !full_model), then the analyzer on that tree
    static MEMEAnalyzer create_and_fit(Tree input_tree, Alignment aln, Scalar pvalue_threshold = 0.1,
                                       std::function<void(const std::string&, double)> progress_cb = nullptr,
                                       bool full_model = true, std::string branches_spec = "All") {
        input_tree.select_branches(branches_spec, "", {}, false);
        if (progress_cb) progress_cb("Phase 1: Fitting Nucleotide GTR Model", 0.1);
        hyphy::opt::GTRFitter gtr_fitter(input_tree, aln);
        const auto gtr = gtr_fitter.fit();
        if (progress_cb) progress_cb("Phase 2: Refining under Global MG94 Model", 0.3);
        MG94Parameters p;
        p.theta_AC = gtr.params.theta_AC; p.theta_AT = gtr.params.theta_AT; p.theta_CG = gtr.params.theta_CG;
        p.theta_CT = gtr.params.theta_CT; p.theta_GT = gtr.params.theta_GT;
        const auto sel = gtr.tree.select_branches(branches_spec, "", {}, true);
        const bool split = sel.num_selected > 0 && sel.num_unselected > 0;
        hyphy::opt::MG94Fitter mg(gtr.tree, aln);
        hyphy::opt::FitResult fit;
        if (full_model) {
            fit = mg.fit_full_model(1.0, p, progress_cb, 250, 1e-5, split ? &sel.is_selected : nullptr);
            p = fit.params;
        } else {
            fit = mg.fit_omega_and_scale(1.0, p);
            p.alpha = 1.0;
            p.beta = fit.x_opt[0];
        }
        MEMEAnalyzer out(fit.tree, std::move(aln), p, std::move(branches_spec));
        out.p_value_threshold = pvalue_threshold;
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

    // meme.hpp:84-92
    void select_test_branches(const std::string& spec) {
        test_branches = spec;
        auto sel = tree.select_branches(spec, "", {}, false);
        is_test_branch = std::move(sel.is_selected);
        num_tested = sel.num_selected;
        num_background = sel.num_unselected;
        fel_analyzer.settings.test_branches = spec;
        fel_analyzer.partition_branches();
    }

    // meme.hpp:150-164
    void prepare_branch_lengths() {
        const auto& code = aln.code ? *aln.code : *hyphy::core::GeneticCode::universal();
        MG94Matrix base;
        base.update(base_params, aln.pos_nuc_frequencies, aln.codon_frequencies_f3x4, code);
        conversion_factor = base.scale_factor > 1e-12 ? 3.0 / base.scale_factor : 1.0;
        baseline_tree_length = 0.0;
        for (auto& node : tree.nodes) {
            if (node.id == tree.root_id) continue;
            baseline_tree_length += node.branch_length;
            node.branch_length *= conversion_factor;
        }
    }

    std::vector<MEMESiteResult> run(bool show_progress = false, bool force_progress = false) {
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
        const size_t nS = static_cast<size_t>(S), n = tree.num_nodes();
        std::vector<double> pi(nS), qs(nS * nS), qn(nS * nS), bl(n, 0.0);
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
        std::vector<h3g_meme_result> res(aln.patterns.size());
        std::vector<double> ebf(aln.patterns.size() * n, 1.0);
        std::vector<uint8_t> tested(n, 1), fel_tested(n, 1);
        for (const auto& node : tree.nodes) {
            if (node.id == tree.root_id) continue;
            tested[size_t(node.id)] = is_test_branch[size_t(node.id)] ? 1 : 0;
            fel_tested[size_t(node.id)] = fel_analyzer.is_test_branch[size_t(node.id)] ? 1 : 0;
        }
        eng.check(h3g_meme_run_tested(pr, &m, bl.data(), tested.data(), fel_tested.data(), res.data(), ebf.data()));
        site_results.assign(aln.num_codons, MEMESiteResult{});
        for (size_t s = 0; s < aln.num_codons; ++s) {
            const size_t p = aln.site_to_pattern[s];
            const auto& r = res[p];
            MEMESiteResult& o = site_results[s];
            o.site_index = s;
            o.alpha = r.alpha; o.beta1 = r.beta1; o.p1 = r.p1; o.beta_plus = r.beta_plus; o.p_plus = r.p_plus;
            o.lrt = r.lrt; o.p_value = r.p_value; o.branches_under_selection = r.branches_under_selection;
            o.total_branch_length = r.total_branch_length;
            o.log_l_meme = r.log_l_meme; o.log_l_fel = r.log_l_fel; o.p_value_meme_vs_fel = r.p_value_meme_vs_fel;
            o.fel_alpha = r.fel_alpha; o.fel_beta = r.fel_beta; o.beta_bg = r.beta_bg;
            o.branch_ebf.assign(ebf.begin() + std::ptrdiff_t(p * n), ebf.begin() + std::ptrdiff_t((p + 1) * n));
            o.evaluations = r.evaluations;
        }
        return site_results;
    }
};

}  // namespace hyphy::analyses
