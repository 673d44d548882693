"""FEL oracle pinned to the reference's HyPhy 2.5 ground truth on CD2 (tests/test_fel_cd2_parity.cpp:66-118).

Same inputs as the reference test (cd2.fna, the fitted tree cd2_fitted.nwk, the
global MG94 parameters it fixes) and the same acceptance: Pearson and Spearman
correlations of per-site LRT and p-values against HyPhy 2.5.
"""
import json

import numpy as np
import pytest


def _corr(x, y):
    return float(np.corrcoef(x, y)[0, 1])


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


@pytest.fixture(scope="module")
def cd2_fel(oracle, golden_dir):
    k = json.loads((golden_dir / "known_answers.json").read_text())["cd2_fel"]
    a = oracle.Alignment.load(str(golden_dir / "cd2.fna"))
    t = oracle.Tree.parse((golden_dir / "cd2_fitted.nwk").read_text())
    return k, a, t, oracle.fel_run(t, a, k["params"])


def test_fel_oracle_matches_hyphy25_cd2(cd2_fel):
    k, a, _, r = cd2_fel
    sp = np.array(a.site_pattern)
    assert len(sp) == 187
    mle = np.array(k["mle"])
    lrt, pv = np.array(r["lrt"])[sp], np.array(r["p_value"])[sp]
    assert _corr(lrt, mle[:, 3]) > k["min_pearson_lrt"]
    assert _corr(_ranks(lrt), _ranks(mle[:, 3])) > k["min_spearman_lrt"]
    assert _corr(pv, mle[:, 4]) > k["min_pearson_p"]
    assert _corr(_ranks(pv), _ranks(mle[:, 4])) > k["min_spearman_p"]


def test_fel_oracle_invariant_sites_and_ranges(cd2_fel):
    _, a, t, r = cd2_fel
    lrt, pv = np.array(r["lrt"]), np.array(r["p_value"])
    assert np.all(lrt >= 0) and np.all((pv >= 0) & (pv <= 1))
    inv = np.array(r["evals"]) == 0
    assert inv.any() and np.all(pv[inv] == 1.0) and np.all(lrt[inv] == 0.0)
    # alternative fit is never worse than the null (nested models)
    assert np.all(np.array(r["log_l_alt"])[~inv] >= np.array(r["log_l_null"])[~inv] - 1e-6)
