// Host-logic harness for the site-fit drivers (h3g_sitefit.cpp, h3g_fel_driver.cpp with and
// without a background branch set, h3g_meme_driver.cpp likewise): the device evaluator is replaced by a CPU function of the
// solved omegas, so the lockstep loop's batching, eigensystem-slot assignment and
// consistency checks run without a GPU.  The fake likelihood is rugged (a bowl plus
// an oscillation) so the simplex searches take many steps, park several requests at
// once and reach the small-batch (speculative) regime.  Prints one checksum line per
// run; exit status 0 when every run returns H3G_OK.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "h3g.h"
#include "h3g_fel.h"

struct h3g_problem {
    int n = 0, root = 0, T = 0, P = 0;
    std::vector<int> parent, taxon, ch_off, ch;
    std::vector<uint8_t> leaf;
    std::vector<int8_t> states;
    std::string err;
};

namespace h3g {
bool fel_problem_view(h3g_problem* pr, FelProblemView* v) {
    v->n = pr->n; v->root = pr->root; v->T = pr->T; v->P = pr->P;
    v->parent = pr->parent.data(); v->leaf = pr->leaf.data(); v->taxon = pr->taxon.data();
    v->ch_off = pr->ch_off.data(); v->ch = pr->ch.data(); v->states = pr->states.data(); v->device = 0;
    return true;
}
void fel_set_error(h3g_problem* pr, const std::string& msg) { pr->err = msg; }
void fel_record_transfer(h3g_problem*, size_t, size_t, int, double) {}
struct FelDevice { int n_slots, max_req, n; std::vector<double> om; std::vector<int> solved; int batches = 0; };
FelDevice* fel_device_create(h3g_problem* pr, int, const double*, const double*, const double*, const double*, const uint8_t*,
                             int max_requests, int n_slots, std::string*) {
    auto* d = new FelDevice{n_slots, max_requests, pr->n, std::vector<double>(n_slots, -1.0), std::vector<int>(n_slots, 0)};
    return d;
}
static double fake_lnl(int p, double a, double o1, double o2, double w1) {
    // rugged: a smooth bowl plus a small oscillation so simplex searches take many steps
    const double la = std::log(a), u = 0.1 * (p % 7);
    double l = -std::pow(la - u, 2) - std::pow(o1 - 0.05 * (p % 5), 2) - 10.0 + 0.02 * std::sin(13.0 * la + 7.0 * o1 + p);
    if (o2 >= 0) l += -0.1 * std::pow(std::log(o2 + 1e-3) - 0.3 * (p % 3), 2) - std::pow(w1 - 0.7, 2) + 0.01 * std::sin(11.0 * w1 + 5.0 * std::log(o2 + 1e-3));
    return l;
}
bool fel_device_eval(FelDevice* d, int n_eig, const double* eom, const int* es, const int* ep, int n_req, const int* pat,
                     const double* a, const int* s1, const int* s2, const double* w1, const int* sb, double* out,
                     std::string* err) {
    ++d->batches;
    if (n_eig > 3 * d->max_req || n_req > d->max_req) { *err = "too large"; return false; }
    for (int e = 0; e < n_eig; ++e) { d->om[es[e]] = eom[e]; d->solved[es[e]] = 1; (void)ep; }
    for (int r = 0; r < n_req; ++r) {
        const double o1 = d->om[s1[r]], o2 = (s2 && s2[r] >= 0) ? d->om[s2[r]] : -1.0;
        out[r] = fake_lnl(pat[r], a[r], o1, o2, w1 ? w1[r] : 1.0);
        if (sb && sb[r] >= 0) out[r] -= 0.3 * std::pow(std::log(d->om[sb[r]] + 1e-3) + 0.2 * (pat[r] % 4), 2);
    }
    return true;
}
int fel_device_max_ebf(const FelDevice* d) { return std::min(256, d->max_req); }
bool fel_device_ebf(FelDevice* d, int, const double*, const int*, const int*, int n_req, const int*, const double*, const int*,
                    const int*, const double*, const int*, double* ebf, std::string*) {
    for (size_t i = 0; i < size_t(n_req) * d->n; ++i) ebf[i] = 1.0;
    return true;
}
void fel_device_transfer(const FelDevice* d, size_t* h2d, size_t* d2h, int* l) { *h2d = *d2h = 0; *l = d->batches; }
void fel_device_destroy(FelDevice* d) { delete d; }
}  // namespace h3g

static int run(int P) {
    h3g_problem pr;
    // root 0 with four leaves 1..4
    pr.n = 5; pr.root = 0; pr.T = 4; pr.P = P;
    pr.parent = {-1, 0, 0, 0, 0}; pr.leaf = {0, 1, 1, 1, 1}; pr.taxon = {-1, 0, 1, 2, 3};
    pr.ch_off = {0, 4, 4, 4, 4, 4}; pr.ch = {1, 2, 3, 4};
    pr.states.resize(size_t(P) * 4);
    for (int p = 0; p < P; ++p)
        for (int t = 0; t < 4; ++t) pr.states[size_t(p) * 4 + t] = int8_t((p + t * (p % 3 + 1)) % 61);
    const int S = 61;
    std::vector<double> pi(S, 1.0 / S), Q(S * S, 0.1), bl = {0, 0.1, 0.2, 0.3, 0.4};
    h3g_fel_model m{S, pi.data(), Q.data(), Q.data()};
    std::vector<h3g_fel_result> fel(P);
    h3g_status st = h3g_fel_run(&pr, &m, bl.data(), fel.data());
    if (st != H3G_OK) { printf("fel status %d %s\n", int(st), pr.err.c_str()); return 1; }
    // the branch-subset search: leaves 1 and 2 tested, 3 and 4 background
    const uint8_t tested[5] = {0, 1, 1, 0, 0};
    std::vector<h3g_fel_result> sub(P);
    st = h3g_fel_run_tested(&pr, &m, bl.data(), tested, sub.data());
    if (st != H3G_OK) { printf("fel subset status %d %s\n", int(st), pr.err.c_str()); return 1; }
    std::vector<h3g_meme_result> out(P);
    std::vector<double> ebf(size_t(P) * pr.n);
    st = h3g_meme_run(&pr, &m, bl.data(), out.data(), ebf.data());
    if (st != H3G_OK) { printf("meme status %d %s\n", int(st), pr.err.c_str()); return 1; }
    std::vector<h3g_meme_result> msub(P);
    st = h3g_meme_run_tested(&pr, &m, bl.data(), tested, nullptr, msub.data(), ebf.data());
    if (st != H3G_OK) { printf("meme subset status %d %s\n", int(st), pr.err.c_str()); return 1; }
    double sum = 0.0;
    long evals = 0;
    for (int p = 0; p < P; ++p) {
        sum += fel[p].log_l_alt + fel[p].log_l_null + out[p].log_l_meme + out[p].alpha + out[p].beta_plus + out[p].p1;
        sum += sub[p].log_l_alt + sub[p].log_l_null + sub[p].beta_nuisance;
        sum += msub[p].log_l_meme + msub[p].beta_bg + msub[p].alpha;
        evals += fel[p].evaluations + out[p].evaluations + sub[p].evaluations + msub[p].evaluations;
    }
    printf("P %d checksum %.17g evaluations %ld\n", P, sum, evals);
    return 0;
}

int main(int argc, char** argv) {
    int rc = 0;
    for (int a = 1; a < argc; ++a) rc |= run(atoi(argv[a]));
    return rc;
}
