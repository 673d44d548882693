// Python bindings of the CPU oracle (test infrastructure only; see h3_oracle.hpp).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "h3_oracle.hpp"

namespace py = pybind11;
using namespace h3o;

static Params params_from(const py::dict& d) {
    Params p;
    if (d.contains("alpha")) p.alpha = d["alpha"].cast<double>();
    if (d.contains("beta")) p.beta = d["beta"].cast<double>();
    if (d.contains("theta")) {
        auto t = d["theta"].cast<std::vector<double>>();
        if (t.size() != 5) throw std::runtime_error("theta must have 5 entries (AC AT CG CT GT)");
        std::copy(t.begin(), t.end(), p.theta);
    }
    if (d.contains("delta")) p.delta = d["delta"].cast<double>();
    if (d.contains("psi")) p.psi = d["psi"].cast<double>();
    if (d.contains("eig") && !d["eig"].is_none()) {
        // {"U": S x S, "V": S x S, "lam": S} replacing the oracle's own eigensystem
        auto e = d["eig"].cast<py::dict>();
        auto flat = [&](const char* k) {
            auto a = e[k].cast<py::array_t<double, py::array::c_style | py::array::forcecast>>();
            return std::vector<double>(a.data(), a.data() + a.size());
        };
        auto g = std::make_shared<GivenEigen>();
        g->U = flat("U"); g->V = flat("V"); g->lam = flat("lam");
        p.eig = g;
    }
    return p;
}

static py::array_t<double> mat_np(const Mat& m) {
    py::array_t<double> a({m.r, m.c});
    std::copy(m.a.begin(), m.a.end(), a.mutable_data());
    return a;
}
static Mat np_mat(const py::array_t<double, py::array::c_style | py::array::forcecast>& a) {
    if (a.ndim() != 2) throw std::runtime_error("expected a 2-D array");
    Mat m(int(a.shape(0)), int(a.shape(1)));
    std::copy(a.data(), a.data() + m.a.size(), m.a.begin());
    return m;
}

static py::dict mix_dict(const MixResult& r) {
    py::dict d;
    d["lnl"] = r.lnl;
    d["grad_t"] = r.grad_t;
    d["grad_beta"] = r.grad_beta;
    d["grad_beta_bg"] = r.grad_beta_bg;
    d["grad_class_w"] = r.grad_class_w;
    d["grad_theta"] = std::vector<double>(r.grad_theta, r.grad_theta + 5);
    d["grad_rate_w"] = r.grad_rate_w;
    d["site_lnl"] = r.site_lnl;
    return d;
}

PYBIND11_MODULE(h3oracle, m) {
    m.doc() = "FP64 CPU oracle of the MG94xREV likelihood core (test infrastructure only)";

    py::class_<Alignment>(m, "Alignment")
        .def_static("load", &load_alignment, py::arg("path"), py::arg("code") = "Universal")
        .def_static("from_sequences", [](const std::vector<std::string>& names, const std::vector<std::string>& seqs, const std::string& code) {
            Alignment a; a.names = names; a.seqs = seqs; a.finalize(code); return a;
        }, py::arg("names"), py::arg("seqs"), py::arg("code") = "Universal")
        .def("subset_patterns", [](const Alignment& a, int begin, int end) {
            // patterns [begin, end) with the full alignment's frequencies (pattern-sharding tests)
            if (begin < 0 || end > a.P || begin > end) throw std::out_of_range("pattern range");
            Alignment b = a;
            b.P = end - begin;
            b.states.assign(a.states.begin() + size_t(begin) * a.T, a.states.begin() + size_t(end) * a.T);
            b.masks.assign(a.masks.begin() + size_t(begin) * a.T, a.masks.begin() + size_t(end) * a.T);
            b.weights.assign(a.weights.begin() + begin, a.weights.begin() + end);
            return b;
        }, py::arg("begin"), py::arg("end"))
        .def("select_patterns", [](const Alignment& a, const std::vector<int>& idx) {
            // the listed patterns, in the order given, with the full alignment's frequencies
            // (parity checks on a seeded subset of a large alignment)
            Alignment b = a;
            b.P = int(idx.size());
            b.states.clear(); b.masks.clear(); b.weights.clear();
            for (int i : idx) {
                if (i < 0 || i >= a.P) throw std::out_of_range("pattern index");
                b.states.insert(b.states.end(), a.states.begin() + size_t(i) * a.T, a.states.begin() + size_t(i + 1) * a.T);
                b.masks.insert(b.masks.end(), a.masks.begin() + size_t(i) * a.T, a.masks.begin() + size_t(i + 1) * a.T);
                b.weights.push_back(a.weights[size_t(i)]);
            }
            return b;
        }, py::arg("indices"))
        .def_readonly("names", &Alignment::names)
        .def_readonly("embedded_tree", &Alignment::embedded_tree)
        .def_readonly("num_taxa", &Alignment::T)
        .def_readonly("num_patterns", &Alignment::P)
        .def_readonly("num_codons", &Alignment::n_codons)
        .def_readonly("weights", &Alignment::weights)
        .def_readonly("site_pattern", &Alignment::site_pattern)
        .def_readonly("pi", &Alignment::pi)
        .def_property_readonly("nuc_freq", [](const Alignment& a) { return std::vector<double>(a.nuc_freq, a.nuc_freq + 4); })
        .def_property_readonly("pos_freq", [](const Alignment& a) {
            py::array_t<double> r({3, 4}); std::copy(&a.pos_freq[0][0], &a.pos_freq[0][0] + 12, r.mutable_data()); return r; })
        .def_property_readonly("states", [](const Alignment& a) {
            py::array_t<int8_t> r({a.P, a.T}); std::copy(a.states.begin(), a.states.end(), r.mutable_data()); return r; })
        .def_property_readonly("masks", [](const Alignment& a) {
            py::array_t<uint64_t> r({a.P, a.T}); std::copy(a.masks.begin(), a.masks.end(), r.mutable_data()); return r; });

    py::class_<Tree>(m, "Tree")
        .def_static("parse", &Tree::parse, py::arg("newick"), py::arg("keep_rooted") = true)
        .def_readonly("parent", &Tree::parent)
        .def_readonly("children", &Tree::children)
        .def_readonly("names", &Tree::name)
        .def_readonly("branch_lengths", &Tree::bl)
        .def_readonly("post_order", &Tree::post)
        .def_readonly("root", &Tree::root)
        .def_property_readonly("is_leaf", [](const Tree& t) { return std::vector<bool>(t.leaf.begin(), t.leaf.end()); })
        .def("num_nodes", &Tree::n);

    m.def("leaf_map", &leaf_map);
    m.def("genetic_code", [](const std::string& name) {
        Code c = Code::make(name);
        py::dict d; d["S"] = c.S;
        std::vector<std::string> sc; std::string aa;
        const char* N = "ACGT";
        for (int s = 0; s < c.S; ++s) {
            int k = c.codon[s];
            sc.push_back(std::string{N[k >> 4], N[(k >> 2) & 3], N[k & 3]});
            aa += c.aa[k];
        }
        d["sense_codons"] = sc; d["aa"] = aa;
        return d;
    });
    m.def("mg94", [](const Alignment& a, const py::dict& p) {
        MG94 mm; mm.update(params_from(p), a.pos_freq, a.pi, a.code);
        py::dict d; d["Q"] = mat_np(mm.Q); d["U"] = mat_np(mm.U); d["V"] = mat_np(mm.Vp);
        d["lam"] = mm.lam; d["mu"] = mm.mu; d["pi"] = mm.pi;
        return d;
    });
    m.def("transition_matrix", [](const Alignment& a, const py::dict& p, double t) {
        MG94 mm; mm.update(params_from(p), a.pos_freq, a.pi, a.code); return mat_np(mm.P(t));
    });
    m.def("mg94_loglik", [](const Tree& t, const Alignment& a, const py::dict& p, double branch_scale, std::vector<double> bl) {
        MG94 mm; mm.update(params_from(p), a.pos_freq, a.pi, a.code);
        py::gil_scoped_release rel;
        return mg94_loglik(t, a, mm, branch_scale, bl.empty() ? nullptr : &bl);
    }, py::arg("tree"), py::arg("aln"), py::arg("params"), py::arg("branch_scale") = 1.0, py::arg("branch_lengths") = std::vector<double>{});
    m.def("loglik_from_P", [](const Tree& t, const Alignment& a, const std::vector<py::array_t<double, py::array::c_style | py::array::forcecast>>& Ps,
                              const std::vector<double>& pi) {
        std::vector<Mat> Pb; for (auto& x : Ps) Pb.push_back(np_mat(x));
        std::vector<double> site;
        double l;
        { py::gil_scoped_release rel; l = loglik_from_P(t, a, Pb, pi, &site); }
        return py::make_tuple(l, site);
    });
    m.def("branch_length_gradients", [](const Tree& t, const Alignment& a, const py::dict& p, std::vector<double> bl) {
        Params pp = params_from(p);
        py::gil_scoped_release rel;
        return branch_length_gradients(t, a, pp, bl);
    }, py::arg("tree"), py::arg("aln"), py::arg("params"), py::arg("branch_lengths") = std::vector<double>{});
    m.def("joint_frechet_gradients", [](const Tree& t, const Alignment& a, const py::dict& p, std::vector<double> bl,
                                        std::vector<bool> is_test, double omega_bg) {
        Params pp = params_from(p);
        std::vector<char> it(is_test.begin(), is_test.end());
        MixResult r;
        { py::gil_scoped_release rel; r = joint_frechet_gradients(t, a, pp, bl, is_test.empty() ? nullptr : &it, omega_bg); }
        return mix_dict(r);
    }, py::arg("tree"), py::arg("aln"), py::arg("params"), py::arg("branch_lengths") = std::vector<double>{},
       py::arg("is_test") = std::vector<bool>{}, py::arg("omega_bg") = -1.0);
    m.def("mixture_eval", [](const Tree& t, const Alignment& a, const std::vector<py::dict>& classes, const std::vector<double>& class_w,
                             py::object bg, std::vector<bool> is_test, std::vector<double> rates, std::vector<double> rate_w,
                             std::vector<double> bl, bool normalized_time, bool want_global, bool zero_l_sentinel, bool tiled,
                             std::vector<int> branch_classes) {
        MixSpec sp;
        for (auto& c : classes) sp.classes.push_back(params_from(c));
        sp.class_w = class_w;
        if (!bg.is_none()) { sp.has_bg = true; sp.bg = params_from(bg.cast<py::dict>()); }
        sp.is_test.assign(is_test.begin(), is_test.end());
        if (!rates.empty()) { sp.rates = rates; sp.rate_w = rate_w; }
        sp.normalized_time = normalized_time; sp.want_global = want_global; sp.zero_l_sentinel = zero_l_sentinel;
        sp.tiled = tiled;
        if (!branch_classes.empty()) {
            if (int(branch_classes.size()) != t.n() + 1) throw std::runtime_error("branch_classes needs n_nodes + 1 offsets");
            sp.branch_classes = branch_classes;
        }
        if (bl.empty()) bl = t.bl;
        MixResult r;
        { py::gil_scoped_release rel; r = mixture_eval(t, a, sp, bl); }
        return mix_dict(r);
    }, py::arg("tree"), py::arg("aln"), py::arg("classes"), py::arg("class_w"), py::arg("bg") = py::none(),
       py::arg("is_test") = std::vector<bool>{}, py::arg("rates") = std::vector<double>{}, py::arg("rate_w") = std::vector<double>{},
       py::arg("branch_lengths") = std::vector<double>{}, py::arg("normalized_time") = false, py::arg("want_global") = false,
       py::arg("zero_l_sentinel") = false, py::arg("tiled") = false, py::arg("branch_classes") = std::vector<int>{});
    m.def("nucleotide_patterns", &nucleotide_patterns, py::arg("aln"));
    m.def("gtr_matrix", [](const std::vector<double>& theta, const std::vector<double>& freq, double t) {
        if (theta.size() != 5 || freq.size() != 4) throw std::runtime_error("theta needs 5 entries, freq 4");
        GTR g; g.update(theta.data(), freq.data());
        py::dict d; d["Q"] = mat_np(g.Q); d["P"] = mat_np(g.P(t)); d["lam"] = g.lam; d["scale"] = g.scale;
        return d;
    }, py::arg("theta"), py::arg("freq"), py::arg("t") = 0.0);
    m.def("gtr_loglik", [](const Tree& t, const Alignment& nuc, const std::vector<double>& theta, const std::vector<double>& freq,
                           std::vector<double> bl) {
        if (theta.size() != 5 || freq.size() != 4) throw std::runtime_error("theta needs 5 entries, freq 4");
        if (bl.empty()) bl = t.bl;
        GTR g; g.update(theta.data(), freq.data());
        std::vector<double> site;
        double l;
        { py::gil_scoped_release rel; l = gtr_loglik(t, nuc, g, bl, &site); }
        return py::make_tuple(l, site);
    }, py::arg("tree"), py::arg("nuc"), py::arg("theta"), py::arg("freq"), py::arg("branch_lengths") = std::vector<double>{});
    m.def("fel_run", [](const Tree& t, const Alignment& a, const py::dict& p, int max_patterns) {
        const Params pp = params_from(p);
        FelRun r;
        { py::gil_scoped_release rel; r = fel_run(t, a, pp, max_patterns); }
        const size_t P = r.patterns.size();
        py::dict d;
        auto col = [&](auto get) { py::array_t<double> x(P); for (size_t i = 0; i < P; ++i) x.mutable_data()[i] = get(r.patterns[i]); return x; };
        d["alpha"] = col([](const FelSite& s) { return s.alpha; });
        d["beta"] = col([](const FelSite& s) { return s.beta; });
        d["alpha_null"] = col([](const FelSite& s) { return s.alpha_null; });
        d["lrt"] = col([](const FelSite& s) { return s.lrt; });
        d["p_value"] = col([](const FelSite& s) { return s.p_value; });
        d["total_branch_length"] = col([](const FelSite& s) { return s.total_bl; });
        d["log_l_alt"] = col([](const FelSite& s) { return s.lnl_alt; });
        d["log_l_null"] = col([](const FelSite& s) { return s.lnl_null; });
        d["evals"] = col([](const FelSite& s) { return double(s.evals); });
        d["conversion"] = r.conversion;
        d["tested_length"] = r.tested_length;
        d["branch_lengths"] = r.bl;
        return d;
    }, py::arg("tree"), py::arg("aln"), py::arg("params"), py::arg("max_patterns") = -1);
    m.def("fel_run_tested", [](const Tree& t, const Alignment& a, const py::dict& p, const std::vector<bool>& tested,
                               double bg_omega, int max_patterns) {
        const Params pp = params_from(p);
        if (int(tested.size()) != t.n()) throw std::runtime_error("tested needs one entry per node");
        const std::vector<char> tv(tested.begin(), tested.end());
        FelSubsetRun r;
        { py::gil_scoped_release rel; r = fel_run_tested(t, a, pp, tv, bg_omega, max_patterns); }
        const size_t P = r.patterns.size();
        py::dict d;
        auto col = [&](auto get) { py::array_t<double> x(P); for (size_t i = 0; i < P; ++i) x.mutable_data()[i] = get(r.patterns[i]); return x; };
        d["alpha"] = col([](const FelSubsetSite& s) { return s.alpha; });
        d["beta"] = col([](const FelSubsetSite& s) { return s.beta; });
        d["beta_nuisance"] = col([](const FelSubsetSite& s) { return s.beta_nuisance; });
        d["alpha_null"] = col([](const FelSubsetSite& s) { return s.alpha_null; });
        d["lrt"] = col([](const FelSubsetSite& s) { return s.lrt; });
        d["p_value"] = col([](const FelSubsetSite& s) { return s.p_value; });
        d["total_branch_length"] = col([](const FelSubsetSite& s) { return s.total_bl; });
        d["log_l_alt"] = col([](const FelSubsetSite& s) { return s.lnl_alt; });
        d["log_l_null"] = col([](const FelSubsetSite& s) { return s.lnl_null; });
        d["evals"] = col([](const FelSubsetSite& s) { return double(s.evals); });
        d["conversion"] = r.conversion;
        d["bg_conversion"] = r.bg_conversion;
        d["tested_length"] = r.tested_length;
        d["bg_length"] = r.bg_length;
        d["branch_lengths"] = r.bl;
        return d;
    }, py::arg("tree"), py::arg("aln"), py::arg("params"), py::arg("tested"), py::arg("bg_omega") = -1.0,
       py::arg("max_patterns") = -1);
    m.def("fel_subset_lnl", [](const Tree& t, const Alignment& a, const py::dict& p, const std::vector<bool>& tested,
                               double bg_omega, int pattern, double alpha, double beta, double beta_bg) {
        const Params pp = params_from(p);
        if (int(tested.size()) != t.n()) throw std::runtime_error("tested needs one entry per node");
        const std::vector<char> tv(tested.begin(), tested.end());
        const FelSubsetRun r = fel_prepare_tested(t, a, pp, tv, bg_omega);
        return fel_subset_lnl(t, a, pp, r, pattern, alpha, beta, beta_bg);
    }, py::arg("tree"), py::arg("aln"), py::arg("params"), py::arg("tested"), py::arg("bg_omega"), py::arg("pattern"),
       py::arg("alpha"), py::arg("beta"), py::arg("beta_bg"));
    m.def("meme_run", [](const Tree& t, const Alignment& a, const py::dict& p, int max_patterns) {
        const Params pp = params_from(p);
        MemeRun r;
        { py::gil_scoped_release rel; r = meme_run(t, a, pp, max_patterns); }
        const size_t P = r.patterns.size();
        py::dict d;
        auto col = [&](auto get) { py::array_t<double> x(P); for (size_t i = 0; i < P; ++i) x.mutable_data()[i] = get(r.patterns[i]); return x; };
        d["alpha"] = col([](const MemeSite& s) { return s.alpha; });
        d["beta1"] = col([](const MemeSite& s) { return s.beta1; });
        d["p1"] = col([](const MemeSite& s) { return s.p1; });
        d["beta_plus"] = col([](const MemeSite& s) { return s.beta_plus; });
        d["p_plus"] = col([](const MemeSite& s) { return s.p_plus; });
        d["lrt"] = col([](const MemeSite& s) { return s.lrt; });
        d["p_value"] = col([](const MemeSite& s) { return s.p_value; });
        d["branches_under_selection"] = col([](const MemeSite& s) { return double(s.bus); });
        d["total_branch_length"] = col([](const MemeSite& s) { return s.total_bl; });
        d["log_l_meme"] = col([](const MemeSite& s) { return s.lnl_meme; });
        d["log_l_fel"] = col([](const MemeSite& s) { return s.lnl_fel; });
        d["p_value_meme_vs_fel"] = col([](const MemeSite& s) { return s.p_vs_fel; });
        d["fel_alpha"] = col([](const MemeSite& s) { return s.fel_alpha; });
        d["fel_beta"] = col([](const MemeSite& s) { return s.fel_beta; });
        d["beta_bg"] = col([](const MemeSite& s) { return s.beta_bg; });
        d["evals"] = col([](const MemeSite& s) { return double(s.evals); });
        const size_t n = size_t(t.n());
        py::array_t<double> ebf({P, n});
        for (size_t i = 0; i < P; ++i)
            for (size_t b = 0; b < n; ++b) ebf.mutable_data()[i * n + b] = r.patterns[i].ebf[b];
        d["branch_ebf"] = ebf;
        d["conversion"] = r.fel.conversion;
        d["branch_lengths"] = r.fel.bl;
        d["mu_s"] = r.mu_s;
        d["mu_n"] = r.mu_n;
        return d;
    }, py::arg("tree"), py::arg("aln"), py::arg("params"), py::arg("max_patterns") = -1);
    m.def("meme_ebf_at", [](const Tree& t, const Alignment& a, const py::dict& p, const std::vector<double>& bl, int pattern,
                            double alpha, double omega1, double p1, double beta_plus, const std::vector<bool>& tested,
                            double beta_bg) {
        const std::vector<char> tv(tested.begin(), tested.end());
        return meme_ebf_at(t, a, params_from(p), bl, pattern, alpha, omega1, p1, beta_plus, tv, beta_bg);
    }, py::arg("tree"), py::arg("aln"), py::arg("params"), py::arg("branch_lengths"), py::arg("pattern"), py::arg("alpha"),
       py::arg("omega1"), py::arg("p1"), py::arg("beta_plus"), py::arg("tested") = std::vector<bool>{},
       py::arg("beta_bg") = 0.0);
    m.def("meme_lnl_at", [](const Tree& t, const Alignment& a, const py::dict& p, const std::vector<double>& bl, int pattern,
                            double alpha, double omega1, double p1, double beta_plus, const std::vector<bool>& tested,
                            double beta_bg) {
        const std::vector<char> tv(tested.begin(), tested.end());
        return meme_lnl_at(t, a, params_from(p), bl, pattern, alpha, omega1, p1, beta_plus, tv, beta_bg);
    }, py::arg("tree"), py::arg("aln"), py::arg("params"), py::arg("branch_lengths"), py::arg("pattern"), py::arg("alpha"),
       py::arg("omega1"), py::arg("p1"), py::arg("beta_plus"), py::arg("tested") = std::vector<bool>{},
       py::arg("beta_bg") = 0.0);
    m.def("meme_run_tested", [](const Tree& t, const Alignment& a, const py::dict& p, const std::vector<bool>& tested,
                                const std::vector<bool>& fel_tested, int max_patterns) {
        const Params pp = params_from(p);
        if (int(tested.size()) != t.n() || (!fel_tested.empty() && int(fel_tested.size()) != t.n()))
            throw std::runtime_error("tested / fel_tested need one entry per node");
        const std::vector<char> tv(tested.begin(), tested.end());
        const std::vector<char> fv = fel_tested.empty() ? tv : std::vector<char>(fel_tested.begin(), fel_tested.end());
        MemeTestedRun r;
        { py::gil_scoped_release rel; r = meme_run_tested(t, a, pp, tv, fv, max_patterns); }
        const size_t P = r.patterns.size();
        py::dict d;
        auto col = [&](auto get) { py::array_t<double> x(P); for (size_t i = 0; i < P; ++i) x.mutable_data()[i] = get(r.patterns[i]); return x; };
        d["alpha"] = col([](const MemeSite& s) { return s.alpha; });
        d["beta1"] = col([](const MemeSite& s) { return s.beta1; });
        d["p1"] = col([](const MemeSite& s) { return s.p1; });
        d["beta_plus"] = col([](const MemeSite& s) { return s.beta_plus; });
        d["p_plus"] = col([](const MemeSite& s) { return s.p_plus; });
        d["beta_bg"] = col([](const MemeSite& s) { return s.beta_bg; });
        d["lrt"] = col([](const MemeSite& s) { return s.lrt; });
        d["p_value"] = col([](const MemeSite& s) { return s.p_value; });
        d["branches_under_selection"] = col([](const MemeSite& s) { return double(s.bus); });
        d["total_branch_length"] = col([](const MemeSite& s) { return s.total_bl; });
        d["log_l_meme"] = col([](const MemeSite& s) { return s.lnl_meme; });
        d["log_l_fel"] = col([](const MemeSite& s) { return s.lnl_fel; });
        d["p_value_meme_vs_fel"] = col([](const MemeSite& s) { return s.p_vs_fel; });
        d["fel_alpha"] = col([](const MemeSite& s) { return s.fel_alpha; });
        d["fel_beta"] = col([](const MemeSite& s) { return s.fel_beta; });
        d["evals"] = col([](const MemeSite& s) { return double(s.evals); });
        const size_t n = size_t(t.n());
        py::array_t<double> ebf({P, n});
        for (size_t i = 0; i < P; ++i)
            for (size_t b = 0; b < n; ++b) ebf.mutable_data()[i * n + b] = r.patterns[i].ebf[b];
        d["branch_ebf"] = ebf;
        d["branch_lengths"] = r.bl;
        d["mu_s"] = r.mu_s;
        d["mu_n"] = r.mu_n;
        return d;
    }, py::arg("tree"), py::arg("aln"), py::arg("params"), py::arg("tested"), py::arg("fel_tested") = std::vector<bool>{},
       py::arg("max_patterns") = -1);
    m.def("busted_estep", [](const Tree& t, const Alignment& a, const py::dict& p, const std::vector<double>& bl,
                             const std::vector<double>& omegas, const std::vector<double>& weights,
                             const std::vector<double>& syn_rates, const std::vector<double>& syn_weights,
                             const std::vector<int>& is_test, double omega_bg) {
        std::vector<char> it(is_test.begin(), is_test.end());
        const Params base = params_from(p);        // reads Python objects: before the GIL is released
        BustedEStep r;
        { py::gil_scoped_release rel; r = busted_estep(t, a, base, bl, omegas, weights, syn_rates, syn_weights, it, omega_bg); }
        py::dict d;
        d["lnl"] = r.lnl;
        d["weights"] = r.weights;
        d["syn_weights"] = r.syn_weights;
        d["pattern_ll"] = r.pattern_ll;
        return d;
    }, py::arg("tree"), py::arg("aln"), py::arg("params"), py::arg("branch_lengths"), py::arg("omegas"), py::arg("weights"),
       py::arg("syn_rates") = std::vector<double>{1.0}, py::arg("syn_weights") = std::vector<double>{1.0},
       py::arg("is_test") = std::vector<int>{}, py::arg("omega_bg") = -1.0);
    m.def("set_threads", [](int n) {
#ifdef _OPENMP
        omp_set_num_threads(n);
#else
        (void)n;
#endif
    });
    m.def("max_threads", []() {
#ifdef _OPENMP
        return omp_get_max_threads();
#else
        return 1;
#endif
    });
}
