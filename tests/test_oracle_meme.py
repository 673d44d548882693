"""MEME oracle pinned to the reference's HyPhy 2.5 ground truth on CD2 (tests/test_meme.cpp:66-104).

The reference test refits the global model itself (nucleotide GTR, then MG94)
before MEME; here the oracle starts from the global MG94xREV fit that HyPhy
2.5 reports in the same ground-truth file (its branch lengths, omega and GTR
exchangeabilities), so both sides fit the sites on identical models.  The
acceptance is the reference test's: Pearson and Spearman correlations of the
per-site LRT and p-values against HyPhy 2.5 of at least 0.95.
"""
import json

import numpy as np
import pytest


def _ranks(v):
    order = np.argsort(v, kind="stable")
    r = np.empty(len(v))
    i = 0
    while i < len(v):
        j = i + 1
        while j < len(v) and abs(v[order[j]] - v[order[i]]) < 1e-12:
            j += 1
        r[order[i:j]] = 0.5 * (i + j - 1) + 1.0
        i = j
    return r


def _corr(x, y):
    return float(np.corrcoef(x, y)[0, 1])


@pytest.fixture(scope="module")
def cd2_meme(oracle, golden_dir):
    k = json.loads((golden_dir / "known_answers.json").read_text())["cd2_meme"]
    a = oracle.Alignment.load(str(golden_dir / "cd2.fna"))
    t = oracle.Tree.parse(k["newick"])
    return k, a, t, oracle.meme_run(t, a, k["params"])


def test_meme_oracle_matches_hyphy25_cd2(cd2_meme):
    k, a, _, r = cd2_meme
    sp = np.array(a.site_pattern)
    assert len(sp) == len(k["mle"]) == 187
    mle = np.array(k["mle"])
    lrt, pv = np.asarray(r["lrt"])[sp], np.asarray(r["p_value"])[sp]
    assert _corr(lrt, mle[:, 5]) >= k["min_pearson_lrt"]
    assert _corr(_ranks(lrt), _ranks(mle[:, 5])) >= k["min_spearman_lrt"]
    assert _corr(pv, mle[:, 6]) >= k["min_pearson_p"]
    assert _corr(_ranks(pv), _ranks(mle[:, 6])) >= k["min_spearman_p"]
    # the site log-likelihoods under MEME follow HyPhy's closely (column 9)
    assert _corr(np.asarray(r["log_l_meme"])[sp], mle[:, 9]) > 0.999


def test_meme_oracle_structure(cd2_meme):
    _, _, t, r = cd2_meme
    ev = np.asarray(r["evals"])
    inv = ev == 0
    assert inv.any() and (~inv).any()
    # invariant patterns are not fitted (meme.hpp:190-216)
    assert np.all(np.asarray(r["lrt"])[inv] == 0) and np.all(np.asarray(r["p_value"])[inv] == 1.0)
    assert np.all(np.asarray(r["log_l_fel"])[inv] == 0) and np.all(np.asarray(r["branch_ebf"])[inv] == 1.0)
    p1, pp = np.asarray(r["p1"]), np.asarray(r["p_plus"])
    np.testing.assert_allclose(p1 + pp, 1.0, rtol=0, atol=1e-15)
    pv = np.asarray(r["p_value"])
    assert np.all((pv >= 0) & (pv <= 1))
    # a pattern that does not reach the test (beta+ <= alpha or p+ <= 1e-6) reports p = 2/3, LRT 0
    a, bp = np.asarray(r["alpha"]), np.asarray(r["beta_plus"])
    untested = (~inv) & ~((bp > a) & (pp > 1e-6))
    assert untested.any()
    np.testing.assert_allclose(pv[untested], 2.0 / 3.0)
    # branches under selection = branches with EBF >= 100 (the root column stays 1)
    ebf = np.asarray(r["branch_ebf"])
    assert np.all(ebf >= 0) and np.all(ebf[:, t.root] == 1.0)
    np.testing.assert_array_equal((ebf >= 100).sum(axis=1), np.asarray(r["branches_under_selection"]))
    # MEME never reports a worse fit than its own null, and the MEME-vs-FEL p-value is exp(-delta)
    lm, lf = np.asarray(r["log_l_meme"]), np.asarray(r["log_l_fel"])
    d = 2.0 * (lm - lf)
    np.testing.assert_allclose(np.asarray(r["p_value_meme_vs_fel"]), np.where(d > 0, np.exp(-d / 2.0), 1.0))
