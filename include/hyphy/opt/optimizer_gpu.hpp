// optimizer_gpu.hpp — MG94Fitter (include/hyphy/opt/optimizer.hpp:752-1135) on
// the device likelihood core.
//
//   fit_omega_and_scale (optimizer.hpp:857-904): bounded 2-D Nelder-Mead over
//     (omega, global tree scale), the reference's NelderMead2D; every trial is
//     one device evaluation at raw time t * s * 3 / mean rate(omega).
//   fit_full_model (optimizer.hpp:909-1135): all branch lengths, omega (and a
//     background omega for a test/background split) and the five GTR
//     exchangeabilities, in log space with the reference's bounds, from the
//     omega/scale warm start; objective and gradient from the device's joint
//     Frechet gradients (compute_joint_frechet_gradients).
//
// The reference drives fit_full_model with LBFGSpp's L-BFGS-B solver, which is
// not part of the reference tree.  This header uses its own bounded
// quasi-Newton method: L-BFGS (memory 8) two-loop direction on the free
// variables, projection onto the box, backtracking Armijo line search, and the
// same stopping rule on the projected-gradient infinity norm.  It reaches the
// same maximum; the iteration path differs.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <deque>
#include <functional>
#include <limits>
#include <string>
#include <utility>
#include <vector>

#include "../core/likelihood_gpu.hpp"

namespace hyphy::opt {

using hyphy::core::Alignment;
using hyphy::core::LikelihoodEngine;
using hyphy::core::MG94Matrix;
using hyphy::core::MG94Parameters;
using hyphy::core::Scalar;
using hyphy::core::Tree;

struct FitResult {
    Scalar log_likelihood = 0.0;
    std::vector<Scalar> x_opt;
    std::vector<std::string> param_names;
    int iterations = 0;
    bool converged = false;
    Tree tree;
    MG94Parameters params;
};

// opt/nelder_mead.hpp:111-229 (bounded 2-D Nelder-Mead, stable vertex order)
struct NMResult { Scalar a = 0, b = 0, f = 0; int iterations = 0; bool converged = false; };
template <class F>
inline NMResult nelder_mead_2d(F&& f, Scalar init_a, Scalar init_b, Scalar lb, Scalar ub, Scalar tol, int max_iter) {
    struct V { Scalar a, b, f; };
    auto cl = [&](Scalar x) { return std::clamp(x, lb, ub); };
    auto ev = [&](Scalar a, Scalar b) { const Scalar ca = cl(a), cb = cl(b); return V{ca, cb, f(ca, cb)}; };
    auto sort3 = [](V (&v)[3]) {
        for (int i = 1; i < 3; ++i) {
            V x = v[i];
            int j = i;
            while (j > 0 && x.f < v[j - 1].f) { v[j] = v[j - 1]; --j; }
            v[j] = x;
        }
    };
    const Scalar sa = std::max<Scalar>(0.1, 0.2 * init_a), sb = std::max<Scalar>(0.1, 0.2 * init_b);
    V v[3] = {ev(init_a, init_b), ev(init_a + sa, init_b), ev(init_a, init_b + sb)};
    int it = 0;
    bool conv = false;
    for (; it < max_iter; ++it) {
        sort3(v);
        if (std::fabs(v[2].f - v[0].f) < tol && std::fabs(v[2].a - v[0].a) < tol && std::fabs(v[2].b - v[0].b) < tol) { conv = true; break; }
        const Scalar ca = 0.5 * (v[0].a + v[1].a), cb = 0.5 * (v[0].b + v[1].b);
        const V r = ev(ca + (ca - v[2].a), cb + (cb - v[2].b));
        if (r.f < v[0].f) {
            const V e = ev(ca + 2.0 * (r.a - ca), cb + 2.0 * (r.b - cb));
            v[2] = e.f < r.f ? e : r;
        } else if (r.f < v[1].f) {
            v[2] = r;
        } else {
            const bool outside = r.f < v[2].f;
            const V c = outside ? ev(ca + 0.5 * (r.a - ca), cb + 0.5 * (r.b - cb)) : ev(ca + 0.5 * (v[2].a - ca), cb + 0.5 * (v[2].b - cb));
            if (c.f < (outside ? r.f : v[2].f)) {
                v[2] = c;
            } else {
                v[1] = ev(v[0].a + 0.5 * (v[1].a - v[0].a), v[0].b + 0.5 * (v[1].b - v[0].b));
                v[2] = ev(v[0].a + 0.5 * (v[2].a - v[0].a), v[0].b + 0.5 * (v[2].b - v[0].b));
            }
        }
    }
    sort3(v);
    return {v[0].a, v[0].b, v[0].f, it + (conv ? 1 : 0), conv};
}

// Bounded L-BFGS: minimise f(x) over lb <= x <= ub; fg(x, g) returns f and fills g.
struct BoxLBFGSResult { std::vector<Scalar> x; Scalar f = 0; int iterations = 0; bool converged = false; Scalar pg_inf = 0; };
template <class FG>
inline BoxLBFGSResult box_lbfgs(FG&& fg, std::vector<Scalar> x, const std::vector<Scalar>& lb, const std::vector<Scalar>& ub,
                                Scalar eps, int max_iter, int mem = 8) {
    const size_t d = x.size();
    auto project = [&](std::vector<Scalar>& y) { for (size_t i = 0; i < d; ++i) y[i] = std::clamp(y[i], lb[i], ub[i]); };
    auto pg_norm = [&](const std::vector<Scalar>& y, const std::vector<Scalar>& g) {
        Scalar m = 0;
        for (size_t i = 0; i < d; ++i) m = std::max(m, std::fabs(std::clamp(y[i] - g[i], lb[i], ub[i]) - y[i]));
        return m;
    };
    auto norm2 = [](const std::vector<Scalar>& y) { Scalar s = 0; for (Scalar v : y) s += v * v; return std::sqrt(s); };
    project(x);
    std::vector<Scalar> g(d), gn(d), xn(d), dir(d), q(d);
    Scalar f = fg(x, g);
    std::deque<std::pair<std::vector<Scalar>, std::vector<Scalar>>> hist;   // (s, y)
    BoxLBFGSResult res;
    int it = 0;
    for (; it < max_iter; ++it) {
        const Scalar pg = pg_norm(x, g);
        res.pg_inf = pg;
        if (pg <= eps || pg <= eps * norm2(x)) { res.converged = true; break; }
        // free variables: not held at a bound by the gradient
        std::vector<char> freev(d, 1);
        for (size_t i = 0; i < d; ++i)
            if ((x[i] <= lb[i] && g[i] > 0) || (x[i] >= ub[i] && g[i] < 0)) freev[i] = 0;
        // two-loop recursion on the free subspace
        for (size_t i = 0; i < d; ++i) q[i] = freev[i] ? g[i] : 0.0;
        std::vector<Scalar> alpha(hist.size());
        for (size_t k = hist.size(); k-- > 0;) {
            const auto& [s, y] = hist[k];
            Scalar sy = 0, sq = 0;
            for (size_t i = 0; i < d; ++i) if (freev[i]) { sy += s[i] * y[i]; sq += s[i] * q[i]; }
            alpha[k] = sy > 0 ? sq / sy : 0.0;
            for (size_t i = 0; i < d; ++i) if (freev[i]) q[i] -= alpha[k] * y[i];
        }
        Scalar gamma = 1.0;
        if (!hist.empty()) {
            const auto& [s, y] = hist.back();
            Scalar sy = 0, yy = 0;
            for (size_t i = 0; i < d; ++i) if (freev[i]) { sy += s[i] * y[i]; yy += y[i] * y[i]; }
            if (sy > 0 && yy > 0) gamma = sy / yy;
        } else {
            const Scalar gn2 = norm2(q);
            if (gn2 > 0) gamma = std::min<Scalar>(1.0, 1.0 / gn2);
        }
        for (size_t i = 0; i < d; ++i) q[i] *= gamma;
        for (size_t k = 0; k < hist.size(); ++k) {
            const auto& [s, y] = hist[k];
            Scalar sy = 0, yq = 0;
            for (size_t i = 0; i < d; ++i) if (freev[i]) { sy += s[i] * y[i]; yq += y[i] * q[i]; }
            const Scalar beta = sy > 0 ? yq / sy : 0.0;
            for (size_t i = 0; i < d; ++i) if (freev[i]) q[i] += s[i] * (alpha[k] - beta);
        }
        Scalar gd = 0;
        for (size_t i = 0; i < d; ++i) { dir[i] = freev[i] ? -q[i] : 0.0; gd += g[i] * dir[i]; }
        if (!(gd < 0)) {                                   // not a descent direction: steepest descent
            hist.clear();
            gd = 0;
            for (size_t i = 0; i < d; ++i) { dir[i] = freev[i] ? -g[i] : 0.0; gd += g[i] * dir[i]; }
            const Scalar n = norm2(dir);
            if (n > 0) for (auto& v : dir) v /= n;
        }
        // backtracking Armijo along the projected path
        Scalar step = 1.0, fn = f;
        bool ok = false;
        for (int ls = 0; ls < 40; ++ls) {
            for (size_t i = 0; i < d; ++i) xn[i] = x[i] + step * dir[i];
            project(xn);
            Scalar dec = 0;
            for (size_t i = 0; i < d; ++i) dec += g[i] * (xn[i] - x[i]);
            fn = fg(xn, gn);
            if (std::isfinite(fn) && fn <= f + 1e-4 * dec) { ok = true; break; }
            step *= 0.5;
        }
        if (!ok) break;
        std::vector<Scalar> s(d), y(d);
        Scalar sy = 0, ss = 0;
        for (size_t i = 0; i < d; ++i) { s[i] = xn[i] - x[i]; y[i] = gn[i] - g[i]; sy += s[i] * y[i]; ss += s[i] * s[i]; }
        if (sy > 1e-12 * ss) {
            hist.emplace_back(std::move(s), std::move(y));
            if (int(hist.size()) > mem) hist.pop_front();
        }
        const Scalar fprev = f;
        x = xn; g = gn; f = fn;
        if (std::fabs(fprev - f) <= 1e-14 * std::max<Scalar>(1.0, std::fabs(f))) { res.converged = true; ++it; break; }
    }
    res.x = x;
    res.f = f;
    res.iterations = it;
    if (!res.converged) res.pg_inf = pg_norm(x, g);
    return res;
}

class MG94Fitter {
public:
    Tree tree;
    Alignment aln;

    MG94Fitter(Tree t, Alignment a) : tree(std::move(t)), aln(std::move(a)) {}

    // optimizer.hpp:857-904
    FitResult fit_omega_and_scale(Scalar init_omega = 1.0, MG94Parameters base_params = MG94Parameters{}) {
        const auto& code = aln.code ? *aln.code : *hyphy::core::GeneticCode::universal();
        const auto l2t = LikelihoodEngine::build_leaf_to_taxon_map(tree, aln);
        std::vector<Scalar> bl0(tree.num_nodes(), 0.0);
        for (const auto& nd : tree.nodes) if (nd.id != tree.root_id) bl0[size_t(nd.id)] = nd.branch_length;
        auto eval_at = [&](Scalar omega, Scalar s) -> Scalar {
            MG94Parameters p = base_params;
            p.alpha = 1.0;
            p.beta = omega;
            MG94Matrix mg;
            mg.update(p, aln.pos_nuc_frequencies, aln.codon_frequencies_f3x4, code);
            const Scalar conv = mg.scale_factor > 1e-12 ? 3.0 / mg.scale_factor : 1.0;
            std::vector<Scalar> bl(bl0);
            for (auto& x : bl) x *= s * conv;
            return -LikelihoodEngine::compute_branch_length_gradients(tree, aln, p, bl, &l2t).first;
        };
        const NMResult pt = nelder_mead_2d(eval_at, init_omega, 1.0, 1e-4, 50.0, 1e-4, 80);
        FitResult res;
        res.log_likelihood = -pt.f;
        res.x_opt = {pt.a, pt.b};
        res.param_names = {"omega", "tree_scale"};
        res.iterations = pt.iterations;
        res.converged = pt.converged;
        res.params = base_params;
        res.params.alpha = 1.0;
        res.params.beta = pt.a;
        res.tree = tree;
        for (auto& nd : res.tree.nodes) if (nd.id != res.tree.root_id) nd.branch_length *= pt.b;
        return res;
    }

    // optimizer.hpp:909-1135
    FitResult fit_full_model(Scalar init_omega = 1.0, MG94Parameters base_params = MG94Parameters{},
                             std::function<void(const std::string&, double)> progress_cb = nullptr, int max_iters = 250,
                             Scalar tolerance = 1e-5, const std::vector<bool>* is_test_branch = nullptr,
                             Scalar* out_background_omega = nullptr) {
        if (progress_cb) progress_cb("Phase 2: Initializing branch lengths and omega", 0.30);
        const FitResult init = fit_omega_and_scale(init_omega, base_params);
        Tree cur = tree;
        for (auto& nd : cur.nodes) if (nd.id != cur.root_id) nd.branch_length *= init.x_opt[1];
        MG94Parameters p = base_params;
        p.alpha = 1.0;
        p.beta = init.x_opt[0];
        const auto l2t = LikelihoodEngine::build_leaf_to_taxon_map(cur, aln);
        std::vector<int32_t> br;
        for (const auto& nd : cur.nodes) if (nd.id != cur.root_id && nd.parent_id >= 0) br.push_back(nd.id);
        const size_t B = br.size(), n = cur.num_nodes();
        max_iters = std::max<int>(max_iters, std::min<int>(500, 5 * int(B) + 60));
        bool has_bg = false;
        if (is_test_branch && is_test_branch->size() >= n) {
            bool any_t = false, any_b = false;
            for (int32_t id : br) ((*is_test_branch)[size_t(id)] ? any_t : any_b) = true;
            has_bg = any_t && any_b;
        }
        const size_t i_om = B, i_bg = has_bg ? B + 1 : B, i_th = has_bg ? B + 2 : B + 1, dim = i_th + 5;
        std::vector<Scalar> x(dim), lb(dim), ub(dim);
        for (size_t i = 0; i < B; ++i) {
            x[i] = std::log(std::clamp(cur.nodes[size_t(br[i])].branch_length, 1e-7, 100.0));
            lb[i] = -18.420680744;
            ub[i] = 6.91;
        }
        x[i_om] = std::log(std::clamp(p.beta, 1e-4, 100.0)); lb[i_om] = -10.0; ub[i_om] = 6.91;
        if (has_bg) { x[i_bg] = x[i_om]; lb[i_bg] = -10.0; ub[i_bg] = 6.91; }
        const std::array<Scalar, 5> th0 = {p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT};
        for (size_t k = 0; k < 5; ++k) { x[i_th + k] = std::log(std::clamp(th0[k], 1e-4, 100.0)); lb[i_th + k] = -10.0; ub[i_th + k] = 6.91; }

        Scalar best_f = std::numeric_limits<Scalar>::infinity();
        std::vector<Scalar> best_x = x;
        auto fg = [&](const std::vector<Scalar>& y, std::vector<Scalar>& g) -> Scalar {
            std::vector<Scalar> bls(n, 0.0);
            for (size_t i = 0; i < B; ++i) bls[size_t(br[i])] = std::exp(y[i]);
            MG94Parameters q;
            q.alpha = 1.0;
            q.beta = std::exp(y[i_om]);
            const Scalar om_bg = has_bg ? std::exp(y[i_bg]) : q.beta;
            q.theta_AC = std::exp(y[i_th]); q.theta_AT = std::exp(y[i_th + 1]); q.theta_CG = std::exp(y[i_th + 2]);
            q.theta_CT = std::exp(y[i_th + 3]); q.theta_GT = std::exp(y[i_th + 4]);
            const auto r = LikelihoodEngine::compute_joint_frechet_gradients(cur, aln, q, bls, &l2t, has_bg ? is_test_branch : nullptr, om_bg);
            g.assign(y.size(), 0.0);
            for (size_t i = 0; i < B; ++i) g[i] = -bls[size_t(br[i])] * r.grad_branches[size_t(br[i])];
            g[i_om] = -q.beta * r.grad_omega;
            if (has_bg) g[i_bg] = -om_bg * r.grad_omega_bg;
            g[i_th] = -q.theta_AC * r.grad_theta_AC; g[i_th + 1] = -q.theta_AT * r.grad_theta_AT;
            g[i_th + 2] = -q.theta_CG * r.grad_theta_CG; g[i_th + 3] = -q.theta_CT * r.grad_theta_CT;
            g[i_th + 4] = -q.theta_GT * r.grad_theta_GT;
            const Scalar fx = -r.log_likelihood;
            if (std::isfinite(fx) && fx < best_f) { best_f = fx; best_x = y; }
            return fx;
        };
        if (progress_cb) progress_cb("Phase 2: Unified joint Frechet quasi-Newton optimization", 0.45);
        BoxLBFGSResult sol = box_lbfgs(fg, x, lb, ub, tolerance, max_iters);
        Scalar fx = sol.f;
        x = sol.x;
        if (std::isfinite(best_f) && (!std::isfinite(fx) || best_f < fx)) { x = best_x; fx = best_f; }
        for (size_t i = 0; i < B; ++i) cur.nodes[size_t(br[i])].branch_length = std::exp(x[i]);
        p.beta = std::exp(x[i_om]);
        const Scalar om_bg = has_bg ? std::exp(x[i_bg]) : p.beta;
        if (out_background_omega) *out_background_omega = om_bg;
        p.theta_AC = std::exp(x[i_th]); p.theta_AT = std::exp(x[i_th + 1]); p.theta_CG = std::exp(x[i_th + 2]);
        p.theta_CT = std::exp(x[i_th + 3]); p.theta_GT = std::exp(x[i_th + 4]);
        FitResult res;
        res.log_likelihood = -fx;
        res.x_opt = {p.beta, p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT};
        res.param_names = {"omega", "theta_AC", "theta_AT", "theta_CG", "theta_CT", "theta_GT"};
        if (has_bg) { res.x_opt.push_back(om_bg); res.param_names.push_back("omega_background"); }
        res.iterations = sol.iterations;
        res.converged = sol.converged || sol.pg_inf <= std::max<Scalar>(tolerance, 1e-3);
        res.tree = cur;
        res.params = p;
        return res;
    }
};

// opt/nelder_mead.hpp:15-108 (Brent1D::minimize): Brent's parabolic interpolation with golden-section
// steps on [a, c] from x = b, minimising f; returns (x, f(x))
template <class F>
inline std::pair<Scalar, Scalar> brent_minimize(F&& f, Scalar a, Scalar b, Scalar c, Scalar tol, int max_iter) {
    const Scalar CGOLD = 0.3819660, ZEPS = 1e-10;
    Scalar x = b, w = b, v = b, e = 0.0, d = 0.0;
    Scalar fx = f(x), fw = fx, fv = fx;
    Scalar lo = std::min(a, c), hi = std::max(a, c);
    for (int iter = 0; iter < max_iter; ++iter) {
        const Scalar xm = 0.5 * (lo + hi), tol1 = tol * std::fabs(x) + ZEPS, tol2 = 2.0 * tol1;
        if (std::fabs(x - xm) <= tol2 - 0.5 * (hi - lo)) break;
        if (std::fabs(e) > tol1) {
            Scalar r = (x - w) * (fx - fv), q = (x - v) * (fx - fw), pp = (x - v) * q - (x - w) * r;
            q = 2.0 * (q - r);
            if (q > 0.0) pp = -pp;
            q = std::fabs(q);
            const Scalar etemp = e;
            e = d;
            if (std::fabs(pp) >= std::fabs(0.5 * q * etemp) || pp <= q * (lo - x) || pp >= q * (hi - x)) {
                e = x >= xm ? lo - x : hi - x;
                d = CGOLD * e;
            } else {
                d = pp / q;
                const Scalar u = x + d;
                if (u - lo < tol2 || hi - u < tol2) d = xm - x >= 0.0 ? std::fabs(tol1) : -std::fabs(tol1);
            }
        } else {
            e = x >= xm ? lo - x : hi - x;
            d = CGOLD * e;
        }
        const Scalar u = std::fabs(d) >= tol1 ? x + d : x + (d >= 0.0 ? std::fabs(tol1) : -std::fabs(tol1));
        const Scalar fu = f(u);
        if (fu <= fx) {
            if (u >= x) lo = x; else hi = x;
            v = w; fv = fw; w = x; fw = fx; x = u; fx = fu;
        } else {
            if (u < x) lo = u; else hi = u;
            if (fu <= fw || w == x) { v = w; fv = fw; w = u; fw = fu; }
            else if (fu <= fv || v == x || v == w) { v = u; fv = fu; }
        }
    }
    return {x, fx};
}

// stats.hpp:114-121: AICc, falling back to AIC when n <= k + 1
inline Scalar compute_aicc(Scalar log_l, size_t k_params, size_t n_obs) {
    const Scalar k = Scalar(k_params), n = Scalar(n_obs);
    return n > k + 1.0 ? -2.0 * log_l + 2.0 * k * n / (n - k - 1.0) : -2.0 * log_l + 2.0 * k;
}

struct GTRFitResult {
    Scalar log_likelihood = 0.0;
    Scalar aicc = 0.0;
    hyphy::core::GTRParameters params;
    Tree tree;
    int iterations = 0;
    bool converged = false;
};

// GTRFitter (optimizer.hpp:33-200): the nucleotide GTR model (five exchangeabilities, every branch
// length) on the alignment's nucleotide patterns.  Same start as the reference: rates (0.5, 0.3, 0.5,
// 1.0, 0.3), branches shorter than 1e-4 set to 0.05, then the global tree scale by Brent on
// [0.01, 50] (tol 1e-2, 12 iterations).  The reference then alternates coordinate-wise Brent
// searches of the rates with a branch sweep over cavity vectors; here the rates and the branch lengths
// are fitted jointly by the bounded L-BFGS of this header on their log scale, with the objective and
// gradient from the device (compute_gtr_gradients).  Same maximum, different path.  AICc with
// K = 5 + branches and N = nucleotide sites (stats.hpp:114-121).
class GTRFitter {
public:
    Tree tree;
    Alignment aln;
    Alignment nuc_aln;

    GTRFitter(Tree t, const Alignment& a) : tree(std::move(t)), aln(a), nuc_aln(a.to_nucleotide_alignment()) {}

    GTRFitResult fit(int max_iters = 500, Scalar tolerance = 1e-5) {
        std::vector<int32_t> br;
        for (const auto& nd : tree.nodes)
            if (nd.id != tree.root_id && nd.parent_id != hyphy::core::INVALID_INDEX) br.push_back(nd.id);
        const size_t B = br.size(), n = tree.num_nodes();
        hyphy::core::GTRParameters p;
        p.theta_AC = 0.5; p.theta_AT = 0.3; p.theta_CG = 0.5; p.theta_CT = 1.0; p.theta_GT = 0.3;
        Tree cur = tree;
        for (int32_t id : br)
            if (cur.nodes[size_t(id)].branch_length < 1e-4) cur.nodes[size_t(id)].branch_length = 0.05;
        const auto l2t = LikelihoodEngine::build_leaf_to_taxon_map(cur, nuc_aln);
        auto lengths = [&](Scalar scale) {
            std::vector<Scalar> bl(n, 0.0);
            for (int32_t id : br) bl[size_t(id)] = cur.nodes[size_t(id)].branch_length * scale;
            return bl;
        };
        hyphy::core::GTRMatrix g;
        auto lnl_at = [&](const std::vector<Scalar>& bl, const hyphy::core::GTRParameters& q) {
            g.update(q, nuc_aln.nuc_frequencies);
            Tree t = cur;
            for (int32_t id : br) t.nodes[size_t(id)].branch_length = bl[size_t(id)];
            return LikelihoodEngine::compute_gtr_log_likelihood(t, nuc_aln, g, &l2t);
        };
        // stage 1: global tree scale (optimizer.hpp:85-100)
        const auto sc = brent_minimize([&](Scalar s) { return -lnl_at(lengths(s), p); }, 0.01, 1.0, 50.0, 1e-2, 12);
        for (int32_t id : br) cur.nodes[size_t(id)].branch_length *= sc.first;
        // stage 2: rates and branch lengths jointly, log scale, the reference's bounds
        const size_t dim = B + 5;
        std::vector<Scalar> x(dim), lb(dim), ub(dim);
        for (size_t i = 0; i < B; ++i) {
            x[i] = std::log(std::clamp(cur.nodes[size_t(br[i])].branch_length, 1e-6, 50.0));
            lb[i] = std::log(1e-6);
            ub[i] = std::log(50.0);
        }
        const std::array<Scalar, 5> th0 = {p.theta_AC, p.theta_AT, p.theta_CG, p.theta_CT, p.theta_GT};
        for (size_t k = 0; k < 5; ++k) {
            x[B + k] = std::log(th0[k]);
            lb[B + k] = std::log(1e-4);
            ub[B + k] = std::log(100.0);
        }
        auto params_of = [&](const std::vector<Scalar>& y) {
            hyphy::core::GTRParameters q;
            q.theta_AC = std::exp(y[B]); q.theta_AT = std::exp(y[B + 1]); q.theta_CG = std::exp(y[B + 2]);
            q.theta_CT = std::exp(y[B + 3]); q.theta_GT = std::exp(y[B + 4]);
            return q;
        };
        Scalar best_f = std::numeric_limits<Scalar>::infinity();
        std::vector<Scalar> best_x = x;
        auto fg = [&](const std::vector<Scalar>& y, std::vector<Scalar>& gr) -> Scalar {
            std::vector<Scalar> bl(n, 0.0);
            for (size_t i = 0; i < B; ++i) bl[size_t(br[i])] = std::exp(y[i]);
            const auto q = params_of(y);
            const auto r = LikelihoodEngine::compute_gtr_gradients(cur, nuc_aln, q, bl, &l2t);
            gr.assign(y.size(), 0.0);
            for (size_t i = 0; i < B; ++i) gr[i] = -bl[size_t(br[i])] * r.grad_branches[size_t(br[i])];
            const std::array<Scalar, 5> th = {q.theta_AC, q.theta_AT, q.theta_CG, q.theta_CT, q.theta_GT};
            for (size_t k = 0; k < 5; ++k) gr[B + k] = -th[k] * r.grad_theta[k];
            const Scalar fx = -r.log_likelihood;
            if (std::isfinite(fx) && fx < best_f) { best_f = fx; best_x = y; }
            return fx;
        };
        BoxLBFGSResult sol = box_lbfgs(fg, x, lb, ub, tolerance, std::max<int>(max_iters, int(5 * B + 60)));
        Scalar fx = sol.f;
        x = sol.x;
        if (std::isfinite(best_f) && (!std::isfinite(fx) || best_f < fx)) { x = best_x; fx = best_f; }
        for (size_t i = 0; i < B; ++i) cur.nodes[size_t(br[i])].branch_length = std::exp(x[i]);
        GTRFitResult res;
        res.params = params_of(x);
        res.tree = cur;
        res.log_likelihood = lnl_at(lengths(1.0), res.params);
        res.iterations = sol.iterations;
        res.converged = sol.converged || sol.pg_inf <= std::max<Scalar>(tolerance, 1e-3);
        res.aicc = compute_aicc(res.log_likelihood, 5 + B, nuc_aln.num_nucleotides);
        return res;
    }
};

}  // namespace hyphy::opt
