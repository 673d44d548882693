// likelihood_gpu.hpp — drop-in LikelihoodEngine backed by libh3g (B200).
//
// Keeps the reference's entry points (include/hyphy/core/likelihood.hpp):
//   compute_branch_length_gradients   :1102-1211
//   compute_joint_frechet_gradients   :1228-1594  (JointMG94Gradients :1213-1223)
//   compute_tree_log_likelihood_from_P :766-806
//   compute_gtr_log_likelihood         :181-254
//   compute_mg94_log_likelihood        :257-292
//   build_leaf_to_taxon_map            :162-178
// and adds the BUSTED mixture gradient (include/hyphy/analyses/busted.hpp:1138-1429)
// as a free-standing call that also returns omega-class, mixture-weight and
// nucleotide-rate gradients.  Each thread owns one device context; trees and
// alignments are uploaded once and found again by content fingerprint, and
// MG94 eigensystems are cached by parameter value like busted.hpp:301-383.
// Failures throw std::runtime_error carrying the library's message.
#pragma once

#include <cstdlib>
#include <algorithm>
#include <array>
#include <cstring>
#include <unordered_map>
#include <list>
#include <memory>
#include <stdexcept>
#include <utility>
#include <vector>

#include "../../h3g.h"
#include "h3_host.hpp"

namespace hyphy::core {

struct JointMG94Gradients {
    Scalar log_likelihood = 0.0;
    std::vector<Scalar> grad_branches;
    Scalar grad_omega = 0.0;
    Scalar grad_omega_bg = 0.0;
    Scalar grad_theta_AC = 0.0, grad_theta_AT = 0.0, grad_theta_CG = 0.0, grad_theta_CT = 0.0, grad_theta_GT = 0.0;
};

struct MixtureGradients {
    Scalar log_likelihood = 0.0;
    std::vector<Scalar> grad_branches;   // per node, root 0
    std::vector<Scalar> grad_omegas;     // d lnL / d omega_k
    Scalar grad_omega_bg = 0.0;
    std::vector<Scalar> grad_weights;    // d lnL / d w_k (unconstrained partials)
    Scalar grad_theta[5] = {0, 0, 0, 0, 0};   // AC AT CG CT GT
    std::vector<Scalar> grad_syn_weights;     // d lnL / d rho_m (unconstrained partials)
    std::vector<Scalar> grad_bg_omegas;       // background classes: d lnL / d omega_bg_j
    std::vector<Scalar> grad_bg_weights;      // background classes: d lnL / d w_bg_j (unconstrained partials)
    std::vector<Scalar> site_log_likelihoods;
};

namespace gpu_detail {

// Content fingerprint, 8 bytes per step (multiply / xor-shift mixing).
inline uint64_t fnv(uint64_t h, const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        std::memcpy(&w, c + i, 8);
        h = (h ^ w) * 0x9E3779B97F4A7C15ull;
        h ^= h >> 29;
    }
    for (; i < n; ++i) { h ^= c[i]; h *= 1099511628211ull; }
    return h;
}

// Derivative of Q in the direction of one parameter (likelihood.hpp:1522-1576).
inline std::vector<double> dq_beta(const MG94Parameters& p, const double pos[3][4], const GeneticCode& code) {
    const int S = code.num_sense_codons;
    double r[4][4];
    exchangeabilities(p, r);
    std::vector<double> d(size_t(S) * S, 0.0);
    for (int i = 0; i < S; ++i) {
        double row = 0;
        for (int j = 0; j < S; ++j) {
            const auto& df = code.diff_matrix[i][j];
            if (i == j || df.num_diffs != 1 || df.synonymous) continue;
            d[size_t(i) * S + j] = r[df.diff_from[0]][df.diff_to[0]] * pos[df.diff_pos[0]][df.diff_to[0]];
            row += d[size_t(i) * S + j];
        }
        d[size_t(i) * S + i] = -row;
    }
    return d;
}
inline std::vector<double> dq_theta(int u, int v, double alpha, double beta, const double pos[3][4], const GeneticCode& code) {
    const int S = code.num_sense_codons;
    std::vector<double> d(size_t(S) * S, 0.0);
    for (int i = 0; i < S; ++i) {
        double row = 0;
        for (int j = 0; j < S; ++j) {
            const auto& df = code.diff_matrix[i][j];
            if (i == j || df.num_diffs != 1) continue;
            const int f = df.diff_from[0], t = df.diff_to[0];
            if (!((f == u && t == v) || (f == v && t == u))) continue;
            d[size_t(i) * S + j] = (df.synonymous ? alpha : beta) * pos[df.diff_pos[0]][t];
            row += d[size_t(i) * S + j];
        }
        d[size_t(i) * S + i] = -row;
    }
    return d;
}
inline const int kThetaPairs[5][2] = {{0, 1}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

class Engine {
public:
    static Engine& get() {
        thread_local Engine e;
        return e;
    }
    static h3g_precision& precision() {
        static h3g_precision p = [] {
            const char* e = std::getenv("H3G_PRECISION");
            return (e && (e[0] == 'm' || e[0] == 'M')) ? H3G_PREC_MIXED : H3G_PREC_FP64;
        }();
        return p;
    }
    ~Engine() {
        for (auto& e : problems_) h3g_problem_destroy(e.prob);
        if (ctx_) h3g_ctx_destroy(ctx_);
    }
    h3g_ctx* ctx() {
        if (!ctx_) {
            const char* dev = std::getenv("H3G_DEVICE");
            h3g_status st = h3g_ctx_create(dev ? std::atoi(dev) : 0, nullptr, &ctx_);
            if (st != H3G_OK) throw std::runtime_error("libh3g: no usable CUDA device (status " + std::to_string(int(st)) + ")");
        }
        return ctx_;
    }
    void check(h3g_status st) const {
        if (st != H3G_OK) throw std::runtime_error(std::string("libh3g: ") + h3g_last_error(ctx_));
    }
    h3g_problem* problem(const Tree& tree, const Alignment& aln, const std::vector<size_t>& l2t) {
        const int n = int(tree.num_nodes()), T = int(aln.num_taxa), P = int(aln.patterns.size());
        std::vector<int32_t> parent(n), taxon(n, -1);
        std::vector<uint8_t> leaf(n);
        for (const auto& nd : tree.nodes) {
            parent[size_t(nd.id)] = nd.parent_id;
            leaf[size_t(nd.id)] = nd.is_leaf ? 1 : 0;
            if (nd.is_leaf && l2t[size_t(nd.id)] != size_t(-1)) taxon[size_t(nd.id)] = int32_t(l2t[size_t(nd.id)]);
        }
        // content fingerprint straight from the patterns (arrays are only built on a miss);
        // a mask only matters where the state is unresolved, so only those masks are hashed
        uint64_t h = 1469598103934665603ull;
        h = fnv(h, parent.data(), parent.size() * 4);
        h = fnv(h, leaf.data(), leaf.size());
        h = fnv(h, taxon.data(), taxon.size() * 4);
        {
            uint64_t lane[4] = {h, h ^ 0x243F6A8885A308D3ull, h ^ 0x13198A2E03707344ull, h ^ 0xA4093822299F31D0ull};
            for (int p = 0; p < P; ++p) {
                const auto& sp = aln.patterns[size_t(p)];
                uint64_t& l = lane[p & 3];
                l = fnv(l, sp.states.data(), sp.states.size());
                const size_t nt = sp.states.size();
                for (size_t t0 = 0; t0 < nt; t0 += 8) {     // eight states at a time: any unresolved (sign bit)?
                    uint64_t w = 0;
                    const size_t k = std::min<size_t>(8, nt - t0);
                    std::memcpy(&w, sp.states.data() + t0, k);
                    if (!(w & 0x8080808080808080ull)) continue;
                    for (size_t t = t0; t < t0 + k; ++t)
                        if (sp.states[t] < 0) {
                            const uint64_t m = t < sp.ambiguous_masks.size() ? sp.ambiguous_masks[t] : 0;
                            l = fnv(l, &m, 8);
                        }
                }
                const double wt = double(sp.weight);
                l = fnv(l, &wt, 8);
            }
            for (uint64_t l : lane) h = fnv(h, &l, 8);
        }
        for (auto it = problems_.begin(); it != problems_.end(); ++it)
            if (it->key == h && it->n == n && it->P == P) {
                problems_.splice(problems_.begin(), problems_, it);
                return problems_.front().prob;
            }
        std::vector<int8_t> st(size_t(P) * T);
        std::vector<uint64_t> mk(size_t(P) * T);
        std::vector<double> w(P);
        for (int p = 0; p < P; ++p) {
            const auto& sp = aln.patterns[size_t(p)];
            w[size_t(p)] = double(sp.weight);
            for (int t = 0; t < T; ++t) {
                st[size_t(p) * T + t] = sp.states[size_t(t)];
                mk[size_t(p) * T + t] = size_t(t) < sp.ambiguous_masks.size() ? sp.ambiguous_masks[size_t(t)] : 0;
            }
        }
        h3g_problem* pr = nullptr;
        check(h3g_problem_create(ctx(), n, parent.data(), leaf.data(), taxon.data(), T, P, st.data(), mk.data(), w.data(), &pr));
        if (memory_budget()) check(h3g_problem_set_memory_budget(pr, memory_budget(), 0));
        problems_.push_front({h, n, P, pr, 0});
        if (problems_.size() > 4) { h3g_problem_destroy(problems_.back().prob); problems_.pop_back(); }
        return pr;
    }
    // device bytes each problem's evaluation workspace may take (0: none; subtree checkpointing
    // then starts only when a workspace exceeds the device's free memory)
    static uint64_t& memory_budget() { static uint64_t b = 0; return b; }
    void apply_memory_budget() {
        for (auto& e : problems_) check(h3g_problem_set_memory_budget(e.prob, memory_budget(), 0));
    }
    // true (default): models are installed as generators and diagonalised on the device
    // (h3g_model_desc with NULL eigensystems); false: by the host's Householder + QL solver
    static bool& device_eigen() { static bool on = true; return on; }

    const MG94Matrix& model(const MG94Parameters& p, const Alignment& aln) {
        const GeneticCode& code = aln.code ? *aln.code : *GeneticCode::universal();
        const bool dev = device_eigen();
        uint64_t h = 1469598103934665603ull;
        h = fnv(h, &p, sizeof(p));
        h = fnv(h, &dev, sizeof(dev));
        h = fnv(h, aln.pos_nuc_frequencies, sizeof(aln.pos_nuc_frequencies));
        h = fnv(h, aln.codon_frequencies_f3x4.data(), aln.codon_frequencies_f3x4.size() * 8);
        h = fnv(h, code.name.data(), code.name.size());
        for (auto it = models_.begin(); it != models_.end(); ++it)
            if (it->first == h) { models_.splice(models_.begin(), models_, it); return models_.front().second; }
        MG94Matrix m;
        m.update(p, aln.pos_nuc_frequencies, aln.codon_frequencies_f3x4, code, !dev);
        models_.emplace_front(h, std::move(m));
        if (models_.size() > 32) models_.pop_back();
        return models_.front().second;
    }

    // key of the mixture model last installed on a problem by compute_mixture_gradients
    uint64_t installed(h3g_problem* pr) const {
        for (auto& e : problems_) if (e.prob == pr) return e.model_key;
        return 0;
    }
    void set_installed(h3g_problem* pr, uint64_t k) {
        for (auto& e : problems_) if (e.prob == pr) e.model_key = k;
    }

private:
    struct Entry { uint64_t key; int n, P; h3g_problem* prob; uint64_t model_key = 0; };
    h3g_ctx* ctx_ = nullptr;
    std::list<Entry> problems_;
    std::list<std::pair<uint64_t, MG94Matrix>> models_;
};

// Packs eigensystems for h3g_model_desc.
// (models built without an eigensystem leave lam, U, V empty: the device diagonalises Q).
struct ModelPack {
    std::vector<double> Q, lam, U, V, mu, dQ;
    void add(const MG94Matrix& m) {
        Q.insert(Q.end(), m.Q.v.begin(), m.Q.v.end());
        lam.insert(lam.end(), m.eigenvalues.begin(), m.eigenvalues.end());
        U.insert(U.end(), m.U_pi.v.begin(), m.U_pi.v.end());
        V.insert(V.end(), m.V_pi.v.begin(), m.V_pi.v.end());
        mu.push_back(m.scale_factor);
    }
    const double* lam_p() const { return lam.empty() ? nullptr : lam.data(); }
    const double* U_p() const { return U.empty() ? nullptr : U.data(); }
    const double* V_p() const { return V.empty() ? nullptr : V.data(); }
};
inline const double* eig_ptr(const std::vector<double>& v) { return v.empty() ? nullptr : v.data(); }

inline std::vector<double> node_lengths(const Tree& tree, const std::vector<Scalar>& bl) {
    std::vector<double> out(tree.num_nodes(), 0.0);
    for (const auto& nd : tree.nodes)
        if (nd.id != tree.root_id) out[size_t(nd.id)] = size_t(nd.id) < bl.size() ? bl[size_t(nd.id)] : nd.branch_length;
    return out;
}

}  // namespace gpu_detail

class LikelihoodEngine {
public:
    static void set_precision(h3g_precision p) { gpu_detail::Engine::precision() = p; }
    // Where MG94 eigensystems are solved: on the device (default: generators are installed and
    // diagonalised there, h3g_model_desc with NULL eigensystems) or by the host's Householder + QL.
    static void set_device_eigensolver(bool on) { gpu_detail::Engine::device_eigen() = on; }
    static bool device_eigensolver() { return gpu_detail::Engine::device_eigen(); }
    static h3g_precision get_precision() { return gpu_detail::Engine::precision(); }
    // Device bytes one evaluation workspace may take; above it the tree's partials are checkpointed per
    // subtree and recomputed in the outside pass (bit-identical results).  0 = no budget.
    static void set_memory_budget(uint64_t bytes) {
        gpu_detail::Engine::memory_budget() = bytes;
        gpu_detail::Engine::get().apply_memory_budget();
    }
    static uint64_t memory_budget() { return gpu_detail::Engine::memory_budget(); }

    static std::vector<size_t> build_leaf_to_taxon_map(const Tree& tree, const Alignment& aln) {
        std::vector<size_t> m(tree.num_nodes(), size_t(-1));
        size_t leaves = 0, hit = 0;
        // exact names through a hash map (the first taxon of each name, as the linear search finds);
        // the case-insensitive and prefix rules of Alignment::taxon_index for the rest
        std::unordered_map<std::string, size_t> exact;
        exact.reserve(aln.taxon_names.size());
        for (size_t i = 0; i < aln.taxon_names.size(); ++i) exact.emplace(aln.taxon_names[i], i);
        for (const auto& nd : tree.nodes) {
            if (!nd.is_leaf) continue;
            ++leaves;
            std::string nm = nd.name;
            if (nm.size() >= 2 && (nm.front() == '\'' || nm.front() == '"') && nm.back() == nm.front()) nm = nm.substr(1, nm.size() - 2);
            const auto it = exact.find(nm);
            m[size_t(nd.id)] = it != exact.end() ? it->second : aln.taxon_index(nd.name);
            if (m[size_t(nd.id)] != size_t(-1)) ++hit;
        }
        if (leaves > 0 && hit == 0)
            throw std::runtime_error("Phylogenetic tree leaves do not match any sequences in alignment! (0/" + std::to_string(leaves) + " matched)");
        return m;
    }

    static std::pair<Scalar, std::vector<Scalar>> compute_branch_length_gradients(
        const Tree& tree, const Alignment& aln, const MG94Parameters& params,
        const std::vector<Scalar>& branch_lengths = {}, const std::vector<size_t>* custom_leaf_to_taxon = nullptr) {
        auto& eng = gpu_detail::Engine::get();
        std::vector<size_t> local;
        const auto& l2t = custom_leaf_to_taxon ? *custom_leaf_to_taxon : (local = build_leaf_to_taxon_map(tree, aln));
        h3g_problem* pr = eng.problem(tree, aln, l2t);
        const MG94Matrix& mg = eng.model(params, aln);
        auto bl = gpu_detail::node_lengths(tree, branch_lengths);
        std::vector<Scalar> grad(tree.num_nodes(), 0.0);
        double lnl = 0.0;
        eng.set_installed(pr, 0);
        eng.check(h3g_branch_length_gradients(pr, mg.S, aln.codon_frequencies_f3x4.data(), mg.Q.data(),
                                              gpu_detail::eig_ptr(mg.eigenvalues), gpu_detail::eig_ptr(mg.U_pi.v),
                                              gpu_detail::eig_ptr(mg.V_pi.v), bl.data(), int(get_precision()), &lnl, grad.data()));
        return {lnl, grad};
    }

    static JointMG94Gradients compute_joint_frechet_gradients(
        const Tree& tree, const Alignment& aln, const MG94Parameters& params,
        const std::vector<Scalar>& branch_lengths = {}, const std::vector<size_t>* custom_leaf_to_taxon = nullptr,
        const std::vector<bool>* is_test_branch = nullptr, Scalar omega_bg = -1.0) {
        auto& eng = gpu_detail::Engine::get();
        const GeneticCode& code = aln.code ? *aln.code : *GeneticCode::universal();
        std::vector<size_t> local;
        const auto& l2t = custom_leaf_to_taxon ? *custom_leaf_to_taxon : (local = build_leaf_to_taxon_map(tree, aln));
        h3g_problem* pr = eng.problem(tree, aln, l2t);
        const size_t n = tree.num_nodes();
        const bool part = is_test_branch && is_test_branch->size() == n && omega_bg >= 0.0;
        MG94Parameters pbg = params;
        pbg.beta = omega_bg;
        gpu_detail::ModelPack mp;
        mp.add(eng.model(params, aln));
        if (part) mp.add(eng.model(pbg, aln));
        const int nm = part ? 2 : 1, S = code.num_sense_codons;
        // directions: omega [, omega_bg], theta_AC..theta_GT
        std::vector<std::vector<double>> dirs;
        auto zero = std::vector<double>(size_t(S) * S, 0.0);
        auto push_dir = [&](std::vector<double> dt, std::vector<double> db) {
            std::vector<double> d = std::move(dt);
            if (part) d.insert(d.end(), db.begin(), db.end());
            mp.dQ.insert(mp.dQ.end(), d.begin(), d.end());
            dirs.push_back({});
        };
        push_dir(gpu_detail::dq_beta(params, aln.pos_nuc_frequencies, code), zero);
        if (part) push_dir(zero, gpu_detail::dq_beta(pbg, aln.pos_nuc_frequencies, code));
        for (auto& pr2 : gpu_detail::kThetaPairs)
            push_dir(gpu_detail::dq_theta(pr2[0], pr2[1], params.alpha, params.beta, aln.pos_nuc_frequencies, code),
                     gpu_detail::dq_theta(pr2[0], pr2[1], pbg.alpha, pbg.beta, aln.pos_nuc_frequencies, code));
        std::vector<uint8_t> it(n, 1);
        if (part) for (size_t i = 0; i < n; ++i) it[i] = (*is_test_branch)[i] ? 1 : 0;
        const double one = 1.0;
        h3g_model_desc d{};
        d.S = S; d.pi = aln.codon_frequencies_f3x4.data(); d.n_models = nm;
        d.Q = mp.Q.data(); d.lam = mp.lam_p(); d.U = mp.U_p(); d.V = mp.V_p(); d.mu = mp.mu.data();
        d.K = 1; d.class_w = &one; d.has_bg = part ? 1 : 0; d.is_test = part ? it.data() : nullptr;
        d.M = 1; d.rates = &one; d.rate_w = &one; d.time_mode = H3G_TIME_NORMALIZED;
        d.n_dirs = int(dirs.size()); d.dQ = mp.dQ.data(); d.precision = int(get_precision()); d.zero_l_sentinel = 0;
        eng.set_installed(pr, 0);
        eng.check(h3g_model_set(pr, &d));
        auto bl = gpu_detail::node_lengths(tree, branch_lengths);
        JointMG94Gradients res;
        res.grad_branches.assign(n, 0.0);
        std::vector<double> gd(dirs.size(), 0.0);
        h3g_result r{};
        r.grad_t = res.grad_branches.data();
        r.grad_dir = gd.data();
        eng.check(h3g_eval(pr, bl.data(), H3G_WANT_LNL | H3G_WANT_GRAD_T | H3G_WANT_GRAD_GLOBAL, &r));
        res.log_likelihood = r.lnl;
        size_t q = 0;
        res.grad_omega = gd[q++];
        if (part) res.grad_omega_bg = gd[q++];
        res.grad_theta_AC = gd[q++]; res.grad_theta_AT = gd[q++]; res.grad_theta_CG = gd[q++];
        res.grad_theta_CT = gd[q++]; res.grad_theta_GT = gd[q++];
        return res;
    }

    // BUSTED-style mixture (busted.hpp:509-660 and :1138-1429): omega classes mixed at
    // the P level on test branches, one background omega elsewhere, synonymous-rate
    // classes as separate passes; branch lengths are used as given (raw time).
    static MixtureGradients compute_mixture_gradients(
        const Tree& tree, const Alignment& aln, const MG94Parameters& base, const std::vector<Scalar>& branch_lengths,
        const std::vector<Scalar>& omegas, const std::vector<Scalar>& weights,
        const std::vector<Scalar>& syn_rates = {1.0}, const std::vector<Scalar>& syn_weights = {1.0},
        const std::vector<bool>* is_test_branch = nullptr, Scalar omega_bg = -1.0,
        bool want_gradients = true, bool zero_likelihood_sentinel = false, bool direction_gradients = true,
        const std::vector<Scalar>& bg_omegas = {}, const std::vector<Scalar>& bg_weights = {}) {
        // direction_gradients = false: branch, class-weight and rate-weight gradients only (no
        // omega / theta directions, so no directional products are installed or evaluated).
        // bg_omegas / bg_weights (non-empty): background branches mix these classes at the P level (the
        // RELAX and two-set BUSTED models) instead of using the one omega_bg
        auto& eng = gpu_detail::Engine::get();
        const GeneticCode& code = aln.code ? *aln.code : *GeneticCode::universal();
        const int S = code.num_sense_codons, K = int(omegas.size()), M = int(syn_rates.size());
        if (K < 1 || weights.size() != omegas.size() || syn_weights.size() != syn_rates.size())
            throw std::runtime_error("mixture: omegas/weights or syn_rates/syn_weights sizes differ");
        auto l2t = build_leaf_to_taxon_map(tree, aln);
        h3g_problem* pr = eng.problem(tree, aln, l2t);
        const size_t n = tree.num_nodes();
        bool has_bg = false;
        std::vector<uint8_t> it(n, 1);
        if (is_test_branch && is_test_branch->size() == n) {
            for (size_t i = 0; i < n; ++i) {
                it[i] = (*is_test_branch)[i] ? 1 : 0;
                if (!it[i] && int(i) != tree.root_id) has_bg = true;
            }
        }
        const int Kb = has_bg ? (bg_omegas.empty() ? 1 : int(bg_omegas.size())) : 0;
        if (!bg_omegas.empty() && bg_weights.size() != bg_omegas.size())
            throw std::runtime_error("mixture: bg_omegas and bg_weights sizes differ");
        if (has_bg && bg_omegas.empty() && omega_bg < 0) throw std::runtime_error("mixture: background branches need omega_bg >= 0");
        gpu_detail::ModelPack mp;
        std::vector<MG94Parameters> ps;
        for (int k = 0; k < K; ++k) { MG94Parameters p = base; p.alpha = 1.0; p.beta = omegas[size_t(k)]; ps.push_back(p); }
        for (int j = 0; j < Kb; ++j) {
            MG94Parameters p = base;
            p.alpha = 1.0;
            p.beta = bg_omegas.empty() ? omega_bg : bg_omegas[size_t(j)];
            ps.push_back(p);
        }
        const int nm = int(ps.size());
        const size_t SS = size_t(S) * S;
        int ndirs = 0;
        uint64_t key = 0x51ED270B27A4F1C3ull;
        key = gpu_detail::fnv(key, &base, sizeof(base));
        key = gpu_detail::fnv(key, omegas.data(), omegas.size() * 8);
        key = gpu_detail::fnv(key, weights.data(), weights.size() * 8);
        key = gpu_detail::fnv(key, syn_rates.data(), syn_rates.size() * 8);
        key = gpu_detail::fnv(key, syn_weights.data(), syn_weights.size() * 8);
        key = gpu_detail::fnv(key, it.data(), it.size());
        if (!bg_omegas.empty()) {
            key = gpu_detail::fnv(key, bg_omegas.data(), bg_omegas.size() * 8);
            key = gpu_detail::fnv(key, bg_weights.data(), bg_weights.size() * 8);
        }
        const bool dirs = want_gradients && direction_gradients;
        const double flags[5] = {omega_bg, double(want_gradients), double(zero_likelihood_sentinel), double(get_precision()),
                                 double(dirs)};
        key = gpu_detail::fnv(key, flags, sizeof(flags));
        const int n_dirs_expected = dirs ? K + Kb + 5 : 0;
        if (eng.installed(pr) != key) {
        for (auto& p : ps) mp.add(eng.model(p, aln));
        auto add_dir = [&](int only_model, const std::vector<std::vector<double>>& per_model) {
            for (int k = 0; k < nm; ++k) {
                if (only_model >= 0 && k != only_model) mp.dQ.insert(mp.dQ.end(), SS, 0.0);
                else mp.dQ.insert(mp.dQ.end(), per_model[size_t(k)].begin(), per_model[size_t(k)].end());
            }
            ++ndirs;
        };
        if (dirs) {
            std::vector<std::vector<double>> db(nm);
            for (int k = 0; k < nm; ++k) db[size_t(k)] = gpu_detail::dq_beta(ps[size_t(k)], aln.pos_nuc_frequencies, code);
            for (int k = 0; k < K; ++k) add_dir(k, db);
            for (int j = 0; j < Kb; ++j) add_dir(K + j, db);
            for (auto& pr2 : gpu_detail::kThetaPairs) {
                std::vector<std::vector<double>> dt(nm);
                for (int k = 0; k < nm; ++k)
                    dt[size_t(k)] = gpu_detail::dq_theta(pr2[0], pr2[1], ps[size_t(k)].alpha, ps[size_t(k)].beta, aln.pos_nuc_frequencies, code);
                add_dir(-1, dt);
            }
        }
        h3g_model_desc d{};
        d.S = S; d.pi = aln.codon_frequencies_f3x4.data(); d.n_models = nm;
        d.Q = mp.Q.data(); d.lam = mp.lam_p(); d.U = mp.U_p(); d.V = mp.V_p(); d.mu = mp.mu.data();
        d.K = K; d.class_w = weights.data(); d.has_bg = Kb; d.is_test = it.data();
        d.bg_w = bg_omegas.empty() ? nullptr : bg_weights.data();
        d.M = M; d.rates = syn_rates.data(); d.rate_w = syn_weights.data(); d.time_mode = H3G_TIME_RAW;
        d.n_dirs = ndirs; d.dQ = ndirs ? mp.dQ.data() : nullptr; d.precision = int(get_precision());
        d.zero_l_sentinel = zero_likelihood_sentinel ? 1 : 0;
        eng.check(h3g_model_set(pr, &d));
        eng.set_installed(pr, key);
        }
        ndirs = n_dirs_expected;
        auto bl = gpu_detail::node_lengths(tree, branch_lengths);
        MixtureGradients res;
        res.grad_branches.assign(n, 0.0);
        res.grad_weights.assign(size_t(K), 0.0);
        res.grad_syn_weights.assign(size_t(M), 0.0);
        res.grad_bg_weights.assign(size_t(Kb), 0.0);
        res.site_log_likelihoods.assign(aln.patterns.size(), 0.0);
        std::vector<double> gd(size_t(std::max(ndirs, 1)), 0.0);
        h3g_result r{};
        r.site_lnl = res.site_log_likelihoods.data();
        r.grad_t = res.grad_branches.data();
        r.grad_dir = gd.data();
        r.grad_class_w = res.grad_weights.data();
        r.grad_rate_w = res.grad_syn_weights.data();
        r.grad_bg_w = Kb ? res.grad_bg_weights.data() : nullptr;
        unsigned want = H3G_WANT_LNL | H3G_WANT_SITE_LNL;
        if (want_gradients) want |= H3G_WANT_GRAD_T | H3G_WANT_GRAD_GLOBAL;
        eng.check(h3g_eval(pr, bl.data(), want, &r));
        res.log_likelihood = r.lnl;
        if (dirs) {
            res.grad_omegas.assign(gd.begin(), gd.begin() + K);
            size_t q = size_t(K);
            for (int j = 0; j < Kb; ++j) res.grad_bg_omegas.push_back(gd[q++]);
            if (Kb) res.grad_omega_bg = res.grad_bg_omegas[0];
            for (int x = 0; x < 5; ++x) res.grad_theta[x] = gd[q++];
        }
        return res;
    }

    static Scalar compute_tree_log_likelihood_from_P(
        const Tree& tree, const Alignment& aln, const std::vector<Matrix>& P_branches, const Vector& pi, int S,
        const std::vector<size_t>* custom_leaf_to_taxon = nullptr, std::vector<Scalar>* site_log_likelihoods = nullptr) {
        auto& eng = gpu_detail::Engine::get();
        std::vector<size_t> local;
        const auto& l2t = custom_leaf_to_taxon ? *custom_leaf_to_taxon : (local = build_leaf_to_taxon_map(tree, aln));
        h3g_problem* pr = eng.problem(tree, aln, l2t);
        const size_t n = tree.num_nodes();
        std::vector<double> P(n * size_t(S) * S, 0.0);
        for (const auto& nd : tree.nodes) {
            if (nd.id == tree.root_id) continue;
            const Matrix& m = P_branches.at(size_t(nd.id));
            if (m.rows() != S || m.cols() != S) throw std::runtime_error("P_branches entries must be S x S");
            std::copy(m.v.begin(), m.v.end(), P.begin() + ptrdiff_t(size_t(nd.id) * S * S));
        }
        double lnl = 0.0;
        if (site_log_likelihoods) site_log_likelihoods->assign(aln.patterns.size(), 0.0);
        eng.set_installed(pr, 0);
        eng.check(h3g_eval_from_P(pr, S, P.data(), pi.data(), &lnl, site_log_likelihoods ? site_log_likelihoods->data() : nullptr));
        return lnl;
    }

    static Scalar compute_mg94_log_likelihood(const Tree& tree, const Alignment& aln, const MG94Matrix& mg94,
                                              const std::vector<size_t>* custom_leaf_to_taxon = nullptr, Scalar branch_scale = 1.0) {
        const int S = mg94.S;
        std::vector<Matrix> Pb(tree.num_nodes(), Matrix::Identity(S));
        for (const auto& nd : tree.nodes)
            if (nd.id != tree.root_id) Pb[size_t(nd.id)] = mg94.transition_matrix(nd.branch_length * branch_scale);
        return compute_tree_log_likelihood_from_P(tree, aln, Pb, mg94.pi, S, custom_leaf_to_taxon);
    }

    // The GTR log-likelihood with its gradient in every branch length and the five exchangeabilities
    // (theta_AG = 1), for fitting: the device's joint-gradient engine on the 4-state problem, FP64.
    // P = exp(Q_norm t) with Q_norm = Q / mu (rate_matrix.hpp:70-78) is the engine's normalised time
    // exp(Q (t / 3) 3 / mu), so the raw generator, its eigensystem and mu are installed with lengths
    // t / 3; directions dQ / d theta carry the d mu term.  branch_lengths per node (the root's ignored).
    struct GTRGradients {
        Scalar log_likelihood = 0.0;
        std::vector<Scalar> grad_branches;          // d lnL / d t, per node
        std::array<Scalar, 5> grad_theta{};         // AC AT CG CT GT
    };
    static GTRGradients compute_gtr_gradients(const Tree& tree, const Alignment& aln, const GTRParameters& params,
                                              const std::vector<Scalar>& branch_lengths,
                                              const std::vector<size_t>* custom_leaf_to_taxon = nullptr) {
        if (aln.num_codons != 0) {
            const Alignment nuc = aln.to_nucleotide_alignment();
            return compute_gtr_gradients(tree, nuc, params, branch_lengths, custom_leaf_to_taxon);
        }
        auto& eng = gpu_detail::Engine::get();
        std::vector<size_t> local;
        const auto& l2t = custom_leaf_to_taxon ? *custom_leaf_to_taxon : (local = build_leaf_to_taxon_map(tree, aln));
        h3g_problem* pr = eng.problem(tree, aln, l2t);
        const size_t n = tree.num_nodes();
        GTRMatrix g;
        g.update(params, aln.nuc_frequencies);
        const double mu = g.scale_factor;
        std::vector<double> Q(16), lam(4), U(16), V(16), dQ(5 * 16, 0.0);
        for (int i = 0; i < 4; ++i) {
            lam[size_t(i)] = g.eigenvalues[size_t(i)] * mu;
            for (int j = 0; j < 4; ++j) {
                Q[size_t(i) * 4 + j] = g.Q(i, j) * mu;
                U[size_t(i) * 4 + j] = g.U_pi(i, j);
                V[size_t(i) * 4 + j] = g.V_pi(i, j);
            }
        }
        static const int pairs[5][2] = {{0, 1}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
        for (int x = 0; x < 5; ++x) {
            const int a = pairs[x][0], b = pairs[x][1];
            double* d = dQ.data() + size_t(x) * 16;
            d[a * 4 + b] = aln.nuc_frequencies[b];
            d[b * 4 + a] = aln.nuc_frequencies[a];
            d[a * 4 + a] = -aln.nuc_frequencies[b];
            d[b * 4 + b] = -aln.nuc_frequencies[a];
        }
        const double one = 1.0;
        h3g_model_desc d{};
        d.S = 4; d.pi = aln.nuc_frequencies; d.n_models = 1;
        d.Q = Q.data(); d.lam = lam.data(); d.U = U.data(); d.V = V.data(); d.mu = &mu;
        d.K = 1; d.class_w = &one; d.has_bg = 0; d.is_test = nullptr;
        d.M = 1; d.rates = &one; d.rate_w = &one; d.time_mode = H3G_TIME_NORMALIZED;
        d.n_dirs = 5; d.dQ = dQ.data(); d.precision = H3G_PREC_FP64; d.zero_l_sentinel = 1;
        eng.set_installed(pr, 0);
        eng.check(h3g_model_set(pr, &d));
        std::vector<double> bl(n, 0.0);
        for (const auto& nd : tree.nodes)
            if (nd.id != tree.root_id) bl[size_t(nd.id)] = (branch_lengths.empty() ? nd.branch_length : branch_lengths[size_t(nd.id)]) / 3.0;
        GTRGradients res;
        res.grad_branches.assign(n, 0.0);
        std::vector<double> gd(5, 0.0);
        h3g_result r{};
        r.grad_t = res.grad_branches.data();
        r.grad_dir = gd.data();
        eng.check(h3g_eval(pr, bl.data(), H3G_WANT_LNL | H3G_WANT_GRAD_T | H3G_WANT_GRAD_GLOBAL, &r));
        res.log_likelihood = r.lnl;
        for (auto& x : res.grad_branches) x /= 3.0;
        for (int x = 0; x < 5; ++x) res.grad_theta[size_t(x)] = gd[size_t(x)];
        return res;
    }

    // likelihood.hpp:181-254: the GTR log-likelihood of a nucleotide alignment (as from
    // Alignment::to_nucleotide_alignment; a codon alignment is converted first)
    static Scalar compute_gtr_log_likelihood(const Tree& tree, const Alignment& aln, const GTRMatrix& gtr_model,
                                             const std::vector<size_t>* custom_leaf_to_taxon = nullptr,
                                             std::vector<Scalar>* site_log_likelihoods = nullptr) {
        if (aln.num_codons != 0) {
            const Alignment nuc = aln.to_nucleotide_alignment();
            return compute_gtr_log_likelihood(tree, nuc, gtr_model, custom_leaf_to_taxon, site_log_likelihoods);
        }
        auto& eng = gpu_detail::Engine::get();
        std::vector<size_t> local;
        const auto& l2t = custom_leaf_to_taxon ? *custom_leaf_to_taxon : (local = build_leaf_to_taxon_map(tree, aln));
        h3g_problem* pr = eng.problem(tree, aln, l2t);
        std::vector<double> P(tree.num_nodes() * 16, 0.0);
        for (const auto& nd : tree.nodes) {
            if (nd.id == tree.root_id) continue;
            const Matrix m = gtr_model.transition_matrix(nd.branch_length);
            std::copy(m.v.begin(), m.v.end(), P.begin() + ptrdiff_t(size_t(nd.id) * 16));
        }
        double lnl = 0.0;
        if (site_log_likelihoods) site_log_likelihoods->assign(aln.patterns.size(), 0.0);
        eng.check(h3g_nuc_eval_from_P(pr, P.data(), gtr_model.pi.data(), &lnl,
                                      site_log_likelihoods ? site_log_likelihoods->data() : nullptr));
        return lnl;
    }
};

}  // namespace hyphy::core
