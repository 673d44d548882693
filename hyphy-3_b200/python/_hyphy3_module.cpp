// _hyphy3 — Python module with the reference binding's names for the likelihood
// core (src/python/bindings.cpp:50-119 core types, :725-732 the gradient call),
// backed by the B200 LikelihoodEngine (include/hyphy/core/likelihood_gpu.hpp).
#include <optional>

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "hyphy/analyses/busted_gpu.hpp"
#include "hyphy/analyses/fel_gpu.hpp"
#include "hyphy/analyses/meme_gpu.hpp"
#include "hyphy/analyses/relax_gpu.hpp"
#include "hyphy/opt/optimizer_gpu.hpp"
#include "hyphy/core/alignment_gpu.hpp"
#include "hyphy/core/likelihood_gpu.hpp"

namespace py = pybind11;
using namespace hyphy::core;
using namespace pybind11::literals;

static py::dict mixture_dict(const MixtureGradients& g) {
    py::dict d;
    d["log_likelihood"] = g.log_likelihood;
    d["grad_branches"] = g.grad_branches;
    d["grad_omegas"] = g.grad_omegas;
    d["grad_omega_bg"] = g.grad_omega_bg;
    d["grad_weights"] = g.grad_weights;
    d["grad_theta"] = std::vector<double>(g.grad_theta, g.grad_theta + 5);
    d["grad_syn_weights"] = g.grad_syn_weights;
    d["grad_bg_omegas"] = g.grad_bg_omegas;
    d["grad_bg_weights"] = g.grad_bg_weights;
    d["site_log_likelihoods"] = g.site_log_likelihoods;
    return d;
}

static const std::vector<bool>* opt_mask(const py::object& o, std::vector<bool>& store) {
    if (o.is_none()) return nullptr;
    store = o.cast<std::vector<bool>>();
    return &store;
}

PYBIND11_MODULE(_hyphy3, m) {
    m.doc() = "HyPhy 3 likelihood core on NVIDIA B200 (libh3g)";

    py::class_<GeneticCode, std::shared_ptr<GeneticCode>>(m, "GeneticCode")
        .def_static("universal", []() { return std::const_pointer_cast<GeneticCode>(GeneticCode::universal()); })
        .def_static("from_name", [](const std::string& nm) { return std::const_pointer_cast<GeneticCode>(GeneticCode::from_name(nm)); })
        .def_readonly("name", &GeneticCode::name)
        .def_readonly("num_sense_codons", &GeneticCode::num_sense_codons)
        .def_readonly("sense_codons", &GeneticCode::sense_codons);

    py::class_<TreeNode>(m, "TreeNode")
        .def_readonly("id", &TreeNode::id)
        .def_readonly("name", &TreeNode::name)
        .def_readonly("parent_id", &TreeNode::parent_id)
        .def_readonly("children", &TreeNode::children)
        .def_readwrite("branch_length", &TreeNode::branch_length)
        .def_readonly("is_leaf", &TreeNode::is_leaf)
        .def_readonly("model_tag", &TreeNode::model_tag);

    py::class_<Tree>(m, "Tree")
        .def(py::init<>())
        .def_static("from_newick", [](const std::string& s, bool keep_rooted) { return Tree::from_newick(s, keep_rooted); },
                    "newick"_a, "keep_rooted"_a = true)
        .def_static("from_newick_file", &Tree::from_newick_file, "filepath"_a, "keep_rooted"_a = true)
        .def("num_nodes", &Tree::num_nodes)
        .def("num_leaves", &Tree::num_leaves)
        .def("select_branches", [](const Tree& t, const std::string& spec, const std::string& regex,
                                   const std::vector<std::string>& names, bool auto_detect, bool throw_on_empty) {
                 const auto sel = t.select_branches(spec, regex, names, auto_detect, throw_on_empty);
                 py::dict d;
                 d["is_selected"] = sel.is_selected;
                 d["selected_names"] = sel.selected_names;
                 d["unselected_names"] = sel.unselected_names;
                 d["num_selected"] = sel.num_selected;
                 d["num_unselected"] = sel.num_unselected;
                 return d;
             }, "spec"_a = "All", "regex"_a = "", "explicit_names"_a = std::vector<std::string>{},
             "auto_detect_test_tags_when_all"_a = false, "throw_on_empty"_a = true)
        .def_readonly("root_id", &Tree::root_id)
        .def_readonly("post_order", &Tree::post_order)
        .def_readonly("nodes", &Tree::nodes)
        .def_readonly("leaf_name_to_id", &Tree::leaf_name_to_id)
        .def("get_branch_lengths", [](const Tree& t) {
            std::vector<Scalar> bl(t.num_nodes(), 0.0);
            for (size_t i = 0; i < t.nodes.size(); ++i) bl[i] = t.nodes[i].branch_length;
            return bl;
        })
        .def("set_branch_lengths", [](Tree& t, const std::vector<Scalar>& bl) {
            for (size_t i = 0; i < t.nodes.size() && i < bl.size(); ++i) t.nodes[i].branch_length = bl[i];
        })
        .def("get_branch_length", [](const Tree& t, int32_t id) { return t.nodes.at(size_t(id)).branch_length; }, "id"_a)
        .def("set_branch_length", [](Tree& t, int32_t id, Scalar v) { t.nodes.at(size_t(id)).branch_length = v; }, "id"_a, "length"_a)
        .def_property_readonly("parents", [](const Tree& t) {
            std::vector<int32_t> p(t.num_nodes());
            for (auto& nd : t.nodes) p[size_t(nd.id)] = nd.parent_id;
            return p;
        });

    py::class_<Alignment>(m, "Alignment")
        .def(py::init<>())
        .def_static("load", [](const std::string& f, bool device, std::optional<std::string> code) {
            const auto gc = code ? GeneticCode::from_name(*code) : nullptr;
            if (!device) return Alignment::load(f, gc);
            Alignment a = Alignment::load_unfinalized(f);
            hyphy::core::finalize_on_device(a, gc);
            return a;
        }, "filepath"_a, "device"_a = false, "genetic_code"_a = std::nullopt)
        .def_static("from_fasta", [](const std::string& f) { return Alignment::load(f); }, "filepath"_a)
        .def_static("from_nexus", [](const std::string& f) { return Alignment::load(f); }, "filepath"_a)
        .def_static("from_text", [](const std::string& s) { return Alignment::from_text(s); }, "text"_a)
        .def_static("from_sequences", [](const std::vector<std::string>& names, const std::vector<std::string>& seqs, const std::string& code,
                                         bool device) {
            if (names.size() != seqs.size()) throw std::runtime_error("names and seqs differ in length");
            Alignment a;
            for (size_t i = 0; i < names.size(); ++i) a.add_sequence(names[i], seqs[i]);
            if (device) hyphy::core::finalize_on_device(a, GeneticCode::from_name(code));
            else a.finalize(GeneticCode::from_name(code));
            return a;
        }, "names"_a, "seqs"_a, "code"_a = "Universal", "device"_a = false)
        .def_property_readonly("site_to_pattern", [](const Alignment& a) { return a.site_to_pattern; })
        .def("to_nucleotide_alignment", &Alignment::to_nucleotide_alignment)
        .def("pattern_weights", [](const Alignment& a) {
            std::vector<size_t> w;
            for (const auto& p : a.patterns) w.push_back(p.weight);
            return w;
        })
        .def("pattern_sites", [](const Alignment& a) {
            std::vector<std::vector<size_t>> s;
            for (const auto& p : a.patterns) s.push_back(p.sites);
            return s;
        })
        .def_readonly("num_taxa", &Alignment::num_taxa)
        .def_property_readonly("num_sequences", [](const Alignment& a) { return a.num_taxa; })
        .def_readonly("num_codons", &Alignment::num_codons)
        .def_readonly("num_nucleotides", &Alignment::num_nucleotides)
        .def_property_readonly("num_sites", [](const Alignment& a) { return a.num_codons; })
        .def_property_readonly("num_patterns", [](const Alignment& a) { return a.patterns.size(); })
        .def_readonly("embedded_tree_newick", &Alignment::embedded_tree_newick)
        .def_readonly("taxon_names", &Alignment::taxon_names)
        .def_readonly("codon_frequencies", &Alignment::codon_frequencies_f3x4)
        .def_property_readonly("nuc_frequencies", [](const Alignment& a) { return std::vector<double>(a.nuc_frequencies, a.nuc_frequencies + 4); })
        .def_property_readonly("pos_nuc_frequencies", [](const Alignment& a) {
            py::array_t<double> r({3, 4});
            std::copy(&a.pos_nuc_frequencies[0][0], &a.pos_nuc_frequencies[0][0] + 12, r.mutable_data());
            return r;
        })
        .def("pattern_arrays", [](const Alignment& a) {
            const size_t P = a.patterns.size(), T = a.num_taxa;
            py::array_t<int8_t> st({P, T});
            py::array_t<uint64_t> mk({P, T});
            py::array_t<double> w(P);
            for (size_t p = 0; p < P; ++p) {
                w.mutable_data()[p] = double(a.patterns[p].weight);
                for (size_t t = 0; t < T; ++t) {
                    st.mutable_data()[p * T + t] = a.patterns[p].states[t];
                    mk.mutable_data()[p * T + t] = a.patterns[p].ambiguous_masks[t];
                }
            }
            return py::make_tuple(st, mk, w);
        }, "(states[P,T] int8, masks[P,T] uint64, weights[P]) of the compressed patterns");

    py::class_<hyphy::core::GTRParameters>(m, "GTRParameters")
        .def(py::init<>())
        .def_readwrite("theta_AC", &hyphy::core::GTRParameters::theta_AC)
        .def_readwrite("theta_AT", &hyphy::core::GTRParameters::theta_AT)
        .def_readwrite("theta_CG", &hyphy::core::GTRParameters::theta_CG)
        .def_readwrite("theta_CT", &hyphy::core::GTRParameters::theta_CT)
        .def_readwrite("theta_GT", &hyphy::core::GTRParameters::theta_GT);
    py::class_<hyphy::core::GTRMatrix>(m, "GTRMatrix")
        .def(py::init<>())
        .def("update", [](hyphy::core::GTRMatrix& g, const hyphy::core::GTRParameters& p, const std::vector<double>& f) {
            if (f.size() != 4) throw std::runtime_error("frequencies need 4 entries");
            g.update(p, f.data());
        }, "params"_a, "frequencies"_a)
        .def("transition_matrix", [](const hyphy::core::GTRMatrix& g, Scalar t) {
            const auto P = g.transition_matrix(t);
            py::array_t<double> r({4, 4});
            std::copy(P.v.begin(), P.v.end(), r.mutable_data());
            return r;
        }, "t"_a)
        .def_readonly("scale_factor", &hyphy::core::GTRMatrix::scale_factor)
        .def_readonly("pi", &hyphy::core::GTRMatrix::pi)
        .def_readonly("eigenvalues", &hyphy::core::GTRMatrix::eigenvalues);
    py::class_<hyphy::opt::GTRFitResult>(m, "GTRFitResult")
        .def_readonly("log_likelihood", &hyphy::opt::GTRFitResult::log_likelihood)
        .def_readonly("aicc", &hyphy::opt::GTRFitResult::aicc)
        .def_readonly("params", &hyphy::opt::GTRFitResult::params)
        .def_readonly("tree", &hyphy::opt::GTRFitResult::tree)
        .def_readonly("iterations", &hyphy::opt::GTRFitResult::iterations)
        .def_readonly("converged", &hyphy::opt::GTRFitResult::converged);
    py::class_<hyphy::opt::GTRFitter>(m, "GTRFitter")
        .def(py::init([](Tree t, const Alignment& a) { return hyphy::opt::GTRFitter(std::move(t), a); }), "tree"_a, "alignment"_a)
        .def("fit", [](hyphy::opt::GTRFitter& f, int max_iters, Scalar tol) {
                 py::gil_scoped_release rel;
                 return f.fit(max_iters, tol);
             }, "max_iters"_a = 500, "tolerance"_a = 1e-5)
        .def_readonly("nuc_aln", &hyphy::opt::GTRFitter::nuc_aln);
    m.def("compute_gtr_gradients", [](const Tree& tree, const Alignment& aln, const hyphy::core::GTRParameters& p,
                                      const std::vector<Scalar>& bl) {
        hyphy::core::LikelihoodEngine::GTRGradients r;
        {
            py::gil_scoped_release rel;
            r = LikelihoodEngine::compute_gtr_gradients(tree, aln, p, bl);
        }
        return py::make_tuple(r.log_likelihood, r.grad_branches,
                              std::vector<Scalar>(r.grad_theta.begin(), r.grad_theta.end()));
    }, "tree"_a, "alignment"_a, "params"_a, "branch_lengths"_a = std::vector<Scalar>{},
       "GTR lnL, d lnL / d t per node and d lnL / d theta (AC AT CG CT GT) on the device");
    m.def("compute_gtr_log_likelihood", [](const Tree& tree, const Alignment& aln, const hyphy::core::GTRMatrix& g) {
        std::vector<Scalar> site;
        Scalar l;
        {
            py::gil_scoped_release rel;
            l = LikelihoodEngine::compute_gtr_log_likelihood(tree, aln, g, nullptr, &site);
        }
        return py::make_tuple(l, site);
    }, "tree"_a, "alignment"_a, "gtr_model"_a,
       "LikelihoodEngine::compute_gtr_log_likelihood on the device: (lnL, per-pattern lnL)");

    py::class_<MG94Parameters>(m, "MG94Parameters")
        .def(py::init<>())
        .def_readwrite("alpha", &MG94Parameters::alpha)
        .def_readwrite("beta", &MG94Parameters::beta)
        .def_readwrite("theta_AC", &MG94Parameters::theta_AC)
        .def_readwrite("theta_AT", &MG94Parameters::theta_AT)
        .def_readwrite("theta_CG", &MG94Parameters::theta_CG)
        .def_readwrite("theta_CT", &MG94Parameters::theta_CT)
        .def_readwrite("theta_GT", &MG94Parameters::theta_GT)
        .def_readwrite("delta", &MG94Parameters::delta)
        .def_readwrite("psi", &MG94Parameters::psi);

    m.def("mg94_eigensystem", [](const Alignment& a, const MG94Parameters& p) {
        MG94Matrix mm;
        mm.update(p, a.pos_nuc_frequencies, a.codon_frequencies_f3x4, a.code ? *a.code : *GeneticCode::universal());
        auto arr = [&](const Matrix& x) {
            py::array_t<double> r({x.rows(), x.cols()});
            std::copy(x.v.begin(), x.v.end(), r.mutable_data());
            return r;
        };
        py::dict d;
        d["Q"] = arr(mm.Q); d["U"] = arr(mm.U_pi); d["V"] = arr(mm.V_pi);
        d["lam"] = mm.eigenvalues; d["mu"] = mm.scale_factor; d["pi"] = mm.pi;
        return d;
    }, "aln"_a, "params"_a);

    m.def("compute_branch_length_gradients", [](const Tree& t, const Alignment& a, const MG94Parameters& p, const std::vector<Scalar>& bl) {
        py::gil_scoped_release rel;
        return LikelihoodEngine::compute_branch_length_gradients(t, a, p, bl);
    }, "tree"_a, "aln"_a, "params"_a, "branch_lengths"_a = std::vector<Scalar>{},
       "Compute log-likelihood and exact analytical branch gradients d ln L / d t_b via Inside-Outside");

    m.def("compute_joint_frechet_gradients", [](const Tree& t, const Alignment& a, const MG94Parameters& p, const std::vector<Scalar>& bl,
                                                py::object is_test, Scalar omega_bg) {
        std::vector<bool> store;
        const std::vector<bool>* mask = opt_mask(is_test, store);
        JointMG94Gradients g;
        {
            py::gil_scoped_release rel;
            g = LikelihoodEngine::compute_joint_frechet_gradients(t, a, p, bl, nullptr, mask, omega_bg);
        }
        py::dict d;
        d["log_likelihood"] = g.log_likelihood;
        d["grad_branches"] = g.grad_branches;
        d["grad_omega"] = g.grad_omega;
        d["grad_omega_bg"] = g.grad_omega_bg;
        d["grad_theta"] = std::vector<double>{g.grad_theta_AC, g.grad_theta_AT, g.grad_theta_CG, g.grad_theta_CT, g.grad_theta_GT};
        return d;
    }, "tree"_a, "aln"_a, "params"_a, "branch_lengths"_a = std::vector<Scalar>{}, "is_test_branch"_a = py::none(), "omega_bg"_a = -1.0);

    m.def("compute_mixture_gradients", [](const Tree& t, const Alignment& a, const MG94Parameters& base, const std::vector<Scalar>& bl,
                                          const std::vector<Scalar>& omegas, const std::vector<Scalar>& weights,
                                          const std::vector<Scalar>& syn_rates, const std::vector<Scalar>& syn_weights,
                                          py::object is_test, Scalar omega_bg, bool want_gradients, bool sentinel,
                                          const std::vector<Scalar>& bg_omegas, const std::vector<Scalar>& bg_weights) {
        std::vector<bool> store;
        const std::vector<bool>* mask = opt_mask(is_test, store);
        MixtureGradients g;
        {
            py::gil_scoped_release rel;
            g = LikelihoodEngine::compute_mixture_gradients(t, a, base, bl, omegas, weights, syn_rates, syn_weights, mask, omega_bg,
                                                            want_gradients, sentinel, true, bg_omegas, bg_weights);
        }
        return mixture_dict(g);
    }, "tree"_a, "aln"_a, "base_params"_a, "branch_lengths"_a, "omegas"_a, "weights"_a,
       "syn_rates"_a = std::vector<Scalar>{1.0}, "syn_weights"_a = std::vector<Scalar>{1.0}, "is_test_branch"_a = py::none(),
       "omega_bg"_a = -1.0, "want_gradients"_a = true, "zero_likelihood_sentinel"_a = false,
       "bg_omegas"_a = std::vector<Scalar>{}, "bg_weights"_a = std::vector<Scalar>{});

    m.def("compute_tree_log_likelihood_from_P", [](const Tree& t, const Alignment& a,
                                                   const std::vector<py::array_t<double, py::array::c_style | py::array::forcecast>>& Ps,
                                                   const std::vector<double>& pi) {
        const int S = int(pi.size());
        std::vector<Matrix> Pb;
        for (auto& x : Ps) {
            if (x.ndim() != 2 || x.shape(0) != S || x.shape(1) != S) throw std::runtime_error("each P must be S x S");
            Matrix mm(S, S);
            std::copy(x.data(), x.data() + size_t(S) * S, mm.v.begin());
            Pb.push_back(std::move(mm));
        }
        std::vector<Scalar> site;
        Scalar l;
        {
            py::gil_scoped_release rel;
            l = LikelihoodEngine::compute_tree_log_likelihood_from_P(t, a, Pb, pi, S, nullptr, &site);
        }
        return py::make_tuple(l, site);
    }, "tree"_a, "aln"_a, "P_branches"_a, "pi"_a);

    m.def("compute_mg94_log_likelihood", [](const Tree& t, const Alignment& a, const MG94Parameters& p, Scalar branch_scale) {
        MG94Matrix mm;
        mm.update(p, a.pos_nuc_frequencies, a.codon_frequencies_f3x4, a.code ? *a.code : *GeneticCode::universal());
        py::gil_scoped_release rel;
        return LikelihoodEngine::compute_mg94_log_likelihood(t, a, mm, nullptr, branch_scale);
    }, "tree"_a, "aln"_a, "params"_a, "branch_scale"_a = 1.0);

    m.def("build_leaf_to_taxon_map", [](const Tree& t, const Alignment& a) {
        auto v = LikelihoodEngine::build_leaf_to_taxon_map(t, a);
        std::vector<long long> out(v.size());
        for (size_t i = 0; i < v.size(); ++i) out[i] = v[i] == size_t(-1) ? -1 : (long long)v[i];
        return out;
    });

    m.def("set_precision", [](const std::string& p) {
        if (p == "fp64") LikelihoodEngine::set_precision(H3G_PREC_FP64);
        else if (p == "mixed") LikelihoodEngine::set_precision(H3G_PREC_MIXED);
        else throw std::runtime_error("precision must be 'fp64' or 'mixed'");
    }, "precision"_a);
    m.def("get_precision", []() { return LikelihoodEngine::get_precision() == H3G_PREC_MIXED ? "mixed" : "fp64"; });
    m.def("set_eigensolver", [](const std::string& w) {
        if (w == "device") LikelihoodEngine::set_device_eigensolver(true);
        else if (w == "host") LikelihoodEngine::set_device_eigensolver(false);
        else throw std::invalid_argument("eigensolver must be 'device' or 'host'");
    }, py::arg("where"));
    m.def("get_eigensolver", []() { return LikelihoodEngine::device_eigensolver() ? "device" : "host"; });
    m.def("set_memory_budget", [](uint64_t bytes) { LikelihoodEngine::set_memory_budget(bytes); }, py::arg("bytes"),
          "Device bytes one evaluation workspace may take (0 = none); above it partials are checkpointed per subtree");
    m.def("get_memory_budget", []() { return LikelihoodEngine::memory_budget(); });
    m.def("library_version", []() { return std::string(h3g_version()); });

    // MG94 global fits (optimizer.hpp:741-1135)
    using hyphy::opt::FitResult;
    using hyphy::opt::MG94Fitter;
    py::class_<FitResult>(m, "FitResult")
        .def_readonly("log_likelihood", &FitResult::log_likelihood)
        .def_readonly("x_opt", &FitResult::x_opt)
        .def_readonly("param_names", &FitResult::param_names)
        .def_readonly("iterations", &FitResult::iterations)
        .def_readonly("converged", &FitResult::converged)
        .def_readonly("tree", &FitResult::tree)
        .def_readonly("params", &FitResult::params);
    py::class_<MG94Fitter>(m, "MG94Fitter")
        .def(py::init([](Tree t, Alignment a) { return MG94Fitter(std::move(t), std::move(a)); }), "tree"_a, "alignment"_a)
        .def("fit_omega_and_scale", [](MG94Fitter& f, Scalar init_omega, const MG94Parameters& base) {
                 py::gil_scoped_release rel;
                 return f.fit_omega_and_scale(init_omega, base);
             }, "init_omega"_a = 1.0, "base_params"_a = MG94Parameters{})
        .def("fit_full_model", [](MG94Fitter& f, Scalar init_omega, const MG94Parameters& base, int max_iters, Scalar tolerance) {
                 py::gil_scoped_release rel;
                 return f.fit_full_model(init_omega, base, nullptr, max_iters, tolerance);
             }, "init_omega"_a = 1.0, "base_params"_a = MG94Parameters{}, "max_iters"_a = 250, "tolerance"_a = 1e-5);

    // FEL (bindings.cpp:121-188 of the reference): settings, per-site results, analyzer
    using hyphy::analyses::FELAnalyzer;
    using hyphy::analyses::FELSettings;
    using hyphy::analyses::SiteResult;
    py::class_<FELSettings>(m, "FELSettings")
        .def(py::init<>())
        .def_readwrite("p_value_threshold", &FELSettings::p_value_threshold)
        .def_readwrite("full_model", &FELSettings::full_model)
        .def_readwrite("srv", &FELSettings::srv)
        .def_readwrite("test_branches", &FELSettings::test_branches)
        .def_readwrite("test_branch_regex", &FELSettings::test_branch_regex)
        .def_readwrite("test_branch_names", &FELSettings::test_branch_names);
    py::class_<SiteResult>(m, "FELSiteResult")
        .def_readonly("site_index", &SiteResult::site_index)
        .def_readonly("alpha", &SiteResult::alpha)
        .def_readonly("beta", &SiteResult::beta)
        .def_readonly("beta_nuisance", &SiteResult::beta_nuisance)
        .def_readonly("beta_background", &SiteResult::beta_nuisance)
        .def_readonly("alpha_null", &SiteResult::alpha_null)
        .def_readonly("lrt", &SiteResult::lrt)
        .def_readonly("p_value", &SiteResult::p_value)
        .def_readonly("total_branch_length", &SiteResult::total_branch_length)
        .def_readonly("log_l_alt", &SiteResult::log_l_alt)
        .def_readonly("log_l_null", &SiteResult::log_l_null)
        .def_readonly("evaluations", &SiteResult::evaluations);
    py::class_<FELAnalyzer>(m, "FELAnalyzer")
        .def(py::init([](Tree tree, Alignment aln, const MG94Parameters& params, const FELSettings& settings, Scalar bg_om) {
                 return FELAnalyzer(std::move(tree), std::move(aln), params, settings, bg_om);
             }),
             "tree"_a, "alignment"_a, "params"_a = MG94Parameters{}, "settings"_a = FELSettings{}, "background_omega"_a = -1.0)
        .def_static("create_and_fit", [](Tree tree, Alignment aln, const FELSettings& settings) {
                        py::gil_scoped_release rel;
                        return FELAnalyzer::create_and_fit(std::move(tree), std::move(aln), settings);
                    }, "tree"_a, "alignment"_a, "settings"_a = FELSettings{})
        .def_static("create_and_fit", [](Tree tree, Alignment aln, Scalar pvalue_threshold, bool full_model) {
                        py::gil_scoped_release rel;
                        return FELAnalyzer::create_and_fit(std::move(tree), std::move(aln), pvalue_threshold, nullptr, full_model);
                    }, "tree"_a, "alignment"_a, "pvalue_threshold"_a = 0.1, "full_model"_a = true)
        .def_readonly("base_params", &FELAnalyzer::base_params)
        .def_readonly("settings", &FELAnalyzer::settings)
        .def_readonly("p_value_threshold", &FELAnalyzer::p_value_threshold)
        .def_readonly("background_omega", &FELAnalyzer::background_omega)
        .def_readonly("global_log_l", &FELAnalyzer::global_log_l)
        .def_readonly("global_aicc", &FELAnalyzer::global_aicc)
        .def_readonly("has_gtr_fit", &FELAnalyzer::has_gtr_fit)
        .def_readonly("gtr_log_l", &FELAnalyzer::gtr_log_l)
        .def_readonly("gtr_aicc", &FELAnalyzer::gtr_aicc)
        .def_readonly("gtr_rates", &FELAnalyzer::gtr_rates)
        .def_readonly("gtr_branch_lengths", &FELAnalyzer::gtr_branch_lengths)
        .def_readonly("full_model", &FELAnalyzer::full_model)
        .def_readonly("is_test_branch", &FELAnalyzer::is_test_branch)
        .def_readonly("test_branch_names", &FELAnalyzer::test_branch_names)
        .def_readonly("bg_branch_names", &FELAnalyzer::bg_branch_names)
        .def_readonly("num_tested", &FELAnalyzer::num_tested)
        .def_readonly("num_background", &FELAnalyzer::num_background)
        .def_readonly("baseline_tested_tree_length", &FELAnalyzer::baseline_tested_tree_length)
        .def_readonly("baseline_bg_tree_length", &FELAnalyzer::baseline_bg_tree_length)
        .def_readonly("tree", &FELAnalyzer::tree)
        .def("run", [](FELAnalyzer& f, bool show_progress, bool force_progress) {
                 py::gil_scoped_release rel;
                 return f.run(show_progress, force_progress);
             }, "show_progress"_a = false, "force_progress"_a = false)
        .def_readonly("conversion_factor", &FELAnalyzer::conversion_factor)
        .def_readonly("baseline_tree_length", &FELAnalyzer::baseline_tree_length)
        .def_readonly("site_results", &FELAnalyzer::site_results);

    // BUSTED likelihood core: evaluate_log_l and the two EM expectation steps
    using hyphy::analyses::BUSTEDAnalyzer;
    using VecS = std::vector<Scalar>;
    using hyphy::analyses::BUSTEDFit;
    using hyphy::analyses::BUSTEDRateDistribution;
    using hyphy::analyses::BUSTEDResult;
    using hyphy::analyses::BUSTEDSettings;
    py::class_<BUSTEDSettings>(m, "BUSTEDSettings")
        .def(py::init<>())
        .def_readwrite("full_auto", &BUSTEDSettings::full_auto)
        .def_readwrite("num_rate_classes", &BUSTEDSettings::num_rate_classes)
        .def_readwrite("srv", &BUSTEDSettings::srv)
        .def_readwrite("num_syn_rate_classes", &BUSTEDSettings::num_syn_rate_classes)
        .def_readwrite("auto_select_k", &BUSTEDSettings::auto_select_k)
        .def_readwrite("max_k", &BUSTEDSettings::max_k)
        .def_readwrite("refine_branch_lengths", &BUSTEDSettings::refine_branch_lengths)
        .def_readwrite("multiple_hits", &BUSTEDSettings::multiple_hits)
        .def_readwrite("error_sink", &BUSTEDSettings::error_sink)
        .def_readwrite("error_sink_max_weight", &BUSTEDSettings::error_sink_max_weight)
        .def_readwrite("error_sink_bf_threshold", &BUSTEDSettings::error_sink_bf_threshold)
        .def_readwrite("test_branches", &BUSTEDSettings::test_branches)
        .def_readwrite("phenotype_mode", &BUSTEDSettings::phenotype_mode)
        .def_readwrite("relax_mode", &BUSTEDSettings::relax_mode)
        .def_readwrite("p_value_threshold", &BUSTEDSettings::p_value_threshold);
    py::class_<BUSTEDRateDistribution>(m, "BUSTEDRateDistribution")
        .def_readonly("omegas", &BUSTEDRateDistribution::omegas)
        .def_readonly("weights", &BUSTEDRateDistribution::weights)
        .def_readonly("syn_rates", &BUSTEDRateDistribution::syn_rates)
        .def_readonly("syn_weights", &BUSTEDRateDistribution::syn_weights)
        .def_readonly("error_sink_weight", &BUSTEDRateDistribution::error_sink_weight)
        .def_readonly("annotations", &BUSTEDRateDistribution::annotations);
    py::class_<BUSTEDFit>(m, "BUSTEDFit")
        .def_readonly("log_likelihood", &BUSTEDFit::log_likelihood)
        .def_readonly("aicc", &BUSTEDFit::aicc)
        .def_readonly("tree_scale", &BUSTEDFit::tree_scale)
        .def_readonly("num_rate_classes", &BUSTEDFit::num_rate_classes)
        .def_readonly("test_distribution", &BUSTEDFit::test_distribution)
        .def_readonly("has_background_distribution", &BUSTEDFit::has_background_distribution)
        .def_readonly("background_distribution", &BUSTEDFit::background_distribution)
        .def_readonly("branch_lengths", &BUSTEDFit::branch_lengths)
        .def_readonly("site_log_likelihoods", &BUSTEDFit::site_log_likelihoods)
        .def_readonly("delta", &BUSTEDFit::delta)
        .def_readonly("psi", &BUSTEDFit::psi)
        .def_readonly("error_sink_weight", &BUSTEDFit::error_sink_weight)
        .def_readonly("has_gtr_params", &BUSTEDFit::has_gtr_params)
        .def_readonly("gtr_params", &BUSTEDFit::gtr_params)
        .def_readonly("iterations", &BUSTEDFit::iterations);
    py::class_<BUSTEDResult>(m, "BUSTEDResult")
        .def_readonly("settings", &BUSTEDResult::settings)
        .def_readonly("optimal_k", &BUSTEDResult::optimal_k)
        .def_readonly("lrt", &BUSTEDResult::lrt)
        .def_readonly("p_value", &BUSTEDResult::p_value)
        .def_readonly("unconstrained", &BUSTEDResult::unconstrained)
        .def_readonly("constrained", &BUSTEDResult::constrained)
        .def_readonly("evidence_ratios", &BUSTEDResult::evidence_ratios)
        .def_readonly("constrained_evidence_ratios", &BUSTEDResult::constrained_evidence_ratios)
        .def_readonly("k_null_fits", &BUSTEDResult::k_null_fits)
        .def_readonly("is_failed", &BUSTEDResult::is_failed)
        .def_readonly("error_message", &BUSTEDResult::error_message)
        .def_readonly("runtime_seconds", &BUSTEDResult::runtime_seconds);
    py::class_<BUSTEDAnalyzer>(m, "BUSTEDAnalyzer")
        .def(py::init([](Tree tree, Alignment aln, const MG94Parameters& params) {
                 return BUSTEDAnalyzer(std::move(tree), std::move(aln), params);
             }),
             "tree"_a, "alignment"_a, "params"_a = MG94Parameters{})
        .def_static("create_and_fit", [](Tree tree, Alignment aln) {
                        py::gil_scoped_release rel;
                        return BUSTEDAnalyzer::create_and_fit(std::move(tree), std::move(aln));
                    }, "tree"_a, "alignment"_a)
        .def("run", [](const BUSTEDAnalyzer& b, const BUSTEDSettings& settings, bool show_progress, bool force_progress) {
                 py::gil_scoped_release rel;
                 return b.run(settings, show_progress, force_progress);
             }, "settings"_a = BUSTEDSettings{}, "show_progress"_a = false, "force_progress"_a = false)
        .def("fit_model", [](const BUSTEDAnalyzer& b, bool is_constrained, size_t K, bool refine, bool srv, size_t M,
                             std::optional<BUSTEDFit> warm) {
                 py::gil_scoped_release rel;
                 return b.fit_model(is_constrained, K, refine, srv, M, "None", warm ? &*warm : nullptr);
             }, "is_constrained"_a, "K"_a = 3, "refine_branches"_a = true, "srv"_a = false, "num_syn_rates"_a = 3,
             "warm_start_fit"_a = std::nullopt)
        .def_readonly("tree", &BUSTEDAnalyzer::tree)
        .def_readonly("base_params", &BUSTEDAnalyzer::base_params)
        .def_readonly("mg94_log_l", &BUSTEDAnalyzer::mg94_log_l)
        .def_readonly("has_gtr_fit", &BUSTEDAnalyzer::has_gtr_fit)
        .def_readonly("gtr_log_l", &BUSTEDAnalyzer::gtr_log_l)
        .def_readonly("gtr_aicc", &BUSTEDAnalyzer::gtr_aicc)
        .def_readonly("gtr_rates", &BUSTEDAnalyzer::gtr_rates)
        .def_readonly("gtr_branch_lengths", &BUSTEDAnalyzer::gtr_branch_lengths)
        .def_readonly("num_background_branches", &BUSTEDAnalyzer::num_background_branches)
        .def("select_test_branches", [](const BUSTEDAnalyzer& b, const std::string& spec) {
                 auto sel = b.tree.select_branches(spec, "", {}, false);
                 b.is_test_branch = sel.is_selected;
                 b.num_test_branches = sel.num_selected;
                 b.num_background_branches = sel.num_unselected;
             }, "spec"_a)
        .def_readwrite("branch_tau", &BUSTEDAnalyzer::branch_tau)
        .def_readwrite("is_test_branch", &BUSTEDAnalyzer::is_test_branch)
        .def_readwrite("num_test_branches", &BUSTEDAnalyzer::num_test_branches)
        .def_readwrite("mg94_omega", &BUSTEDAnalyzer::mg94_omega)
        .def_readwrite("mg94_background_omega", &BUSTEDAnalyzer::mg94_background_omega)
        .def_readonly("mg94_tree_length", &BUSTEDAnalyzer::mg94_tree_length)
        .def("evaluate_log_l", [](const BUSTEDAnalyzer& b, Scalar s, const VecS& omegas, const VecS& weights, const VecS& syn_rates,
                                  const VecS& syn_weights, std::optional<VecS> custom, Scalar delta, Scalar psi) {
                 VecS pll;
                 Scalar l;
                 {
                     py::gil_scoped_release rel;
                     l = b.evaluate_log_l(s, omegas, weights, syn_rates, syn_weights, custom ? &*custom : nullptr, &pll, delta, psi);
                 }
                 return py::make_tuple(l, pll);
             }, "s"_a, "omegas"_a, "weights"_a, "syn_rates"_a = VecS{1.0}, "syn_weights"_a = VecS{1.0},
             "custom_branch_lengths"_a = std::nullopt, "delta"_a = 0.0, "psi"_a = 0.0)
        .def("evaluate_two_set_log_l", [](const BUSTEDAnalyzer& b, Scalar s, const VecS& omegas_test, const VecS& weights_test,
                                          const VecS& omegas_bg, const VecS& weights_bg, const VecS& syn_rates,
                                          const VecS& syn_weights, std::optional<VecS> custom,
                                          std::optional<MG94Parameters> custom_base) {
                 VecS pll;
                 Scalar l;
                 {
                     py::gil_scoped_release rel;
                     l = b.evaluate_two_set_log_l(s, omegas_test, weights_test, omegas_bg, weights_bg, syn_rates, syn_weights,
                                                  custom ? &*custom : nullptr, &pll, 0.0, 0.0, 0.0, 0.0, nullptr, nullptr,
                                                  custom_base ? &*custom_base : nullptr);
                 }
                 return py::make_tuple(l, pll);
             }, "s"_a, "omegas_test"_a, "weights_test"_a, "omegas_bg"_a, "weights_bg"_a, "syn_rates"_a = VecS{1.0},
             "syn_weights"_a = VecS{1.0}, "custom_branch_lengths"_a = std::nullopt, "custom_base_params"_a = std::nullopt)
        .def("compute_expected_weights", [](const BUSTEDAnalyzer& b, Scalar s, const VecS& omegas, const VecS& weights,
                                            const VecS& syn_rates, const VecS& syn_weights, std::optional<VecS> custom,
                                            Scalar delta, Scalar psi) {
                 py::gil_scoped_release rel;
                 return b.compute_expected_weights(s, omegas, weights, syn_rates, syn_weights, custom ? &*custom : nullptr, delta, psi);
             }, "s"_a, "omegas"_a, "weights"_a, "syn_rates"_a = VecS{1.0}, "syn_weights"_a = VecS{1.0},
             "custom_branch_lengths"_a = std::nullopt, "delta"_a = 0.0, "psi"_a = 0.0)
        .def("compute_expected_syn_weights", [](const BUSTEDAnalyzer& b, Scalar s, const VecS& omegas, const VecS& weights,
                                                const VecS& syn_rates, const VecS& syn_weights, std::optional<VecS> custom,
                                                Scalar delta, Scalar psi) {
                 py::gil_scoped_release rel;
                 return b.compute_expected_syn_weights(s, omegas, weights, syn_rates, syn_weights, custom ? &*custom : nullptr, delta,
                                                       psi);
             }, "s"_a, "omegas"_a, "weights"_a, "syn_rates"_a, "syn_weights"_a, "custom_branch_lengths"_a = std::nullopt,
             "delta"_a = 0.0, "psi"_a = 0.0);

    // MEME (bindings.cpp of the reference: MEMESiteResult / MEMEAnalyzer)
    using hyphy::analyses::MEMEAnalyzer;
    using hyphy::analyses::MEMESiteResult;
    py::class_<MEMESiteResult>(m, "MEMESiteResult")
        .def_readonly("site_index", &MEMESiteResult::site_index)
        .def_readonly("alpha", &MEMESiteResult::alpha)
        .def_readonly("beta1", &MEMESiteResult::beta1)
        .def_readonly("p1", &MEMESiteResult::p1)
        .def_readonly("beta_plus", &MEMESiteResult::beta_plus)
        .def_readonly("p_plus", &MEMESiteResult::p_plus)
        .def_readonly("lrt", &MEMESiteResult::lrt)
        .def_readonly("p_value", &MEMESiteResult::p_value)
        .def_readonly("branches_under_selection", &MEMESiteResult::branches_under_selection)
        .def_readonly("total_branch_length", &MEMESiteResult::total_branch_length)
        .def_readonly("log_l_meme", &MEMESiteResult::log_l_meme)
        .def_readonly("log_l_fel", &MEMESiteResult::log_l_fel)
        .def_readonly("p_value_meme_vs_fel", &MEMESiteResult::p_value_meme_vs_fel)
        .def_readonly("fel_alpha", &MEMESiteResult::fel_alpha)
        .def_readonly("fel_beta", &MEMESiteResult::fel_beta)
        .def_readonly("beta_bg", &MEMESiteResult::beta_bg)
        .def_readonly("branch_ebf", &MEMESiteResult::branch_ebf)
        .def_readonly("evaluations", &MEMESiteResult::evaluations);
    py::class_<MEMEAnalyzer>(m, "MEMEAnalyzer")
        .def(py::init([](Tree tree, Alignment aln, const MG94Parameters& params, std::string branches) {
                 return MEMEAnalyzer(std::move(tree), std::move(aln), params, std::move(branches));
             }),
             "tree"_a, "alignment"_a, "params"_a = MG94Parameters{}, "branches"_a = "All")
        .def_static("create_and_fit", [](Tree tree, Alignment aln, Scalar pvalue_threshold, bool full_model, std::string branches) {
                        py::gil_scoped_release rel;
                        return MEMEAnalyzer::create_and_fit(std::move(tree), std::move(aln), pvalue_threshold, nullptr, full_model,
                                                            std::move(branches));
                    }, "tree"_a, "alignment"_a, "pvalue_threshold"_a = 0.1, "full_model"_a = true, "branches"_a = "All")
        .def_readonly("base_params", &MEMEAnalyzer::base_params)
        .def_readonly("tree", &MEMEAnalyzer::tree)
        .def_readonly("global_log_l", &MEMEAnalyzer::global_log_l)
        .def_readonly("global_aicc", &MEMEAnalyzer::global_aicc)
        .def_readonly("has_gtr_fit", &MEMEAnalyzer::has_gtr_fit)
        .def_readonly("gtr_log_l", &MEMEAnalyzer::gtr_log_l)
        .def_readonly("gtr_aicc", &MEMEAnalyzer::gtr_aicc)
        .def_readonly("gtr_rates", &MEMEAnalyzer::gtr_rates)
        .def_readonly("gtr_branch_lengths", &MEMEAnalyzer::gtr_branch_lengths)
        .def("run", [](MEMEAnalyzer& f, bool show_progress, bool force_progress) {
                 py::gil_scoped_release rel;
                 return f.run(show_progress, force_progress);
             }, "show_progress"_a = false, "force_progress"_a = false)
        .def_readwrite("p_value_threshold", &MEMEAnalyzer::p_value_threshold)
        .def_readonly("conversion_factor", &MEMEAnalyzer::conversion_factor)
        .def_readonly("baseline_tree_length", &MEMEAnalyzer::baseline_tree_length)
        .def("select_test_branches", &MEMEAnalyzer::select_test_branches, "spec"_a)
        .def_readonly("test_branches", &MEMEAnalyzer::test_branches)
        .def_readonly("is_test_branch", &MEMEAnalyzer::is_test_branch)
        .def_readonly("num_tested", &MEMEAnalyzer::num_tested)
        .def_readonly("num_background", &MEMEAnalyzer::num_background)
        .def_readonly("site_results", &MEMEAnalyzer::site_results);

    // RELAX (relax.hpp of the reference): settings, fits, result, analyzer
    using hyphy::analyses::RELAXAnalyzer;
    using hyphy::analyses::RELAXModelFit;
    using hyphy::analyses::RELAXRateDistribution;
    using hyphy::analyses::RELAXResult;
    using hyphy::analyses::RELAXSettings;
    py::class_<RELAXSettings>(m, "RELAXSettings")
        .def(py::init<>())
        .def_readwrite("p_value_threshold", &RELAXSettings::p_value_threshold)
        .def_readwrite("refine_branch_lengths", &RELAXSettings::refine_branch_lengths)
        .def_readwrite("max_iterations", &RELAXSettings::max_iterations)
        .def_readwrite("tolerance", &RELAXSettings::tolerance);
    py::class_<RELAXRateDistribution>(m, "RELAXRateDistribution")
        .def_readonly("omegas", &RELAXRateDistribution::omegas)
        .def_readonly("weights", &RELAXRateDistribution::weights);
    py::class_<RELAXModelFit>(m, "RELAXModelFit")
        .def_readonly("log_likelihood", &RELAXModelFit::log_likelihood)
        .def_readonly("aicc", &RELAXModelFit::aicc)
        .def_readonly("parameters", &RELAXModelFit::parameters)
        .def_readonly("tree_scale", &RELAXModelFit::tree_scale)
        .def_readonly("k", &RELAXModelFit::k)
        .def_readonly("realized_cycles", &RELAXModelFit::realized_cycles)
        .def_readonly("converged", &RELAXModelFit::converged)
        .def_readonly("reference_distribution", &RELAXModelFit::reference_distribution)
        .def_readonly("test_distribution", &RELAXModelFit::test_distribution)
        .def_readonly("branch_lengths", &RELAXModelFit::branch_lengths)
        .def_readonly("site_log_likelihoods", &RELAXModelFit::site_log_likelihoods);
    py::class_<RELAXResult>(m, "RELAXResult")
        .def_readonly("gtr_log_likelihood", &RELAXResult::gtr_log_likelihood)
        .def_readonly("gtr_aicc", &RELAXResult::gtr_aicc)
        .def_readonly("gtr_rates", &RELAXResult::gtr_rates)
        .def_readonly("gtr_branch_lengths", &RELAXResult::gtr_branch_lengths)
        .def_readonly("mg94_log_likelihood", &RELAXResult::mg94_log_likelihood)
        .def_readonly("mg94_aicc", &RELAXResult::mg94_aicc)
        .def_readonly("mg94_omega_R", &RELAXResult::mg94_omega_R)
        .def_readonly("mg94_omega_T", &RELAXResult::mg94_omega_T)
        .def_readonly("mg94_branch_lengths", &RELAXResult::mg94_branch_lengths)
        .def_readonly("alternative_fit", &RELAXResult::alternative_fit)
        .def_readonly("null_fit", &RELAXResult::null_fit)
        .def_readonly("lrt", &RELAXResult::lrt)
        .def_readonly("p_value", &RELAXResult::p_value)
        .def_readonly("k", &RELAXResult::k)
        .def_readonly("is_relaxed", &RELAXResult::is_relaxed)
        .def_readonly("is_intensified", &RELAXResult::is_intensified)
        .def_readonly("is_significant", &RELAXResult::is_significant)
        .def_readonly("is_failed", &RELAXResult::is_failed)
        .def_readonly("error_message", &RELAXResult::error_message)
        .def_readonly("test_branches", &RELAXResult::test_branches)
        .def_readonly("reference_branches", &RELAXResult::reference_branches)
        .def_readonly("runtime_seconds", &RELAXResult::runtime_seconds);
    py::class_<RELAXAnalyzer>(m, "RELAXAnalyzer")
        .def(py::init([](Tree t, Alignment a, const RELAXSettings& s) { return RELAXAnalyzer(std::move(t), std::move(a), s); }),
             "tree"_a, "alignment"_a, "settings"_a = RELAXSettings{})
        .def_static("create", [](Tree t, Alignment a, const RELAXSettings& s) { return RELAXAnalyzer::create(std::move(t), std::move(a), s); },
                    "tree"_a, "alignment"_a, "settings"_a = RELAXSettings{})
        .def("run", [](const RELAXAnalyzer& r) {
                 py::gil_scoped_release rel;
                 return r.run();
             })
        .def_readonly("test_branch_names", &RELAXAnalyzer::test_branch_names)
        .def_readonly("ref_branch_names", &RELAXAnalyzer::ref_branch_names)
        .def_readonly("is_test_branch", &RELAXAnalyzer::is_test_branch);
}
