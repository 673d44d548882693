"""FEL and MEME from an alignment and a tree alone (fel.hpp:145-214, meme.hpp:95-148).

Nucleotide GTR fit, global MG94 fit from its rates and the per-site fits, all on the device, held to the
reference's end-to-end acceptance against HyPhy 2.5: LRT (and p-value) correlations of
tests/test_fel_multi_dataset.cpp:66-121 and tests/test_meme.cpp:66-160, the GTR log-likelihood at a
relative 1e-4 (tests/test_fel_multi_dataset.cpp:195-196), the global fits of
python/tests/test_python_autograd.py:46-55 and tests/test_meme.cpp:145-160.
"""
import numpy as np
import pytest

from gpu_helpers import ranks

pytestmark = pytest.mark.gpu


def _inputs(golden_dir, k):
    import _hyphy3 as h3
    aln = h3.Alignment.load(str(golden_dir / k["alignment"]), genetic_code=k["genetic_code"])
    tree = h3.Tree.from_newick_file(str(golden_dir / k["tree"])) if k["tree"] else h3.Tree.from_newick(aln.embedded_tree_newick)
    return tree, aln


def _corr(a, b):
    return float(np.corrcoef(a, b)[0, 1]), float(np.corrcoef(ranks(a), ranks(b))[0, 1])


def _aicc(lnl, k, n):
    return -2 * lnl + 2 * k * n / (n - k - 1)


@pytest.mark.parametrize("case", ["fel_e2e_cd2", "fel_e2e_adh", "fel_e2e_bglobin", "fel_e2e_coxi"])
def test_fel_create_and_fit_matches_hyphy25(golden_dir, known, case):
    import _hyphy3 as h3
    k = known[case]
    tree, aln = _inputs(golden_dir, k)
    fel = h3.FELAnalyzer.create_and_fit(tree, aln, 0.1, full_model=k["full_model"])
    res = fel.run()
    assert len(res) == len(k["lrt"]) == aln.num_codons
    r, rho = _corr(np.array([x.lrt for x in res]), np.array(k["lrt"]))
    assert r >= k["min_pearson_lrt"] and rho >= k["min_spearman_lrt"], (r, rho)
    if k["min_pearson_p"] is not None:
        rp, rhop = _corr(np.array([x.p_value for x in res]), np.array(k["p_value"]))
        assert rp >= k["min_pearson_p"] and rhop >= k["min_spearman_p"], (rp, rhop)
    if k["omega_tol"] is not None:
        assert abs(fel.base_params.beta / fel.base_params.alpha - k["mg94_omega"]) < k["omega_tol"]
    assert fel.has_gtr_fit and fel.full_model == k["full_model"]
    assert fel.gtr_log_l == pytest.approx(k["gtr_log_l"], rel=1e-4)
    # both fits reach HyPhy's maxima (the global one under the same model: full, or omega and a tree scale)
    assert fel.gtr_log_l > k["gtr_log_l"] - 0.05, fel.gtr_log_l
    assert fel.global_log_l > k["mg94_log_l"] - 1.0, fel.global_log_l
    assert len(fel.gtr_branch_lengths) == tree.num_nodes() - 1
    B = tree.num_nodes() - 1
    assert fel.global_aicc == pytest.approx(_aicc(fel.global_log_l, 5 + 1 + B, aln.num_codons), rel=1e-12)
    assert fel.gtr_aicc == pytest.approx(_aicc(fel.gtr_log_l, 5 + B, 3 * aln.num_codons), rel=1e-12)


def test_fel_create_and_fit_adh_full_model(golden_dir, known):
    import _hyphy3 as h3
    k = known["adh_global_fit"]
    aln = h3.Alignment.load(str(golden_dir / "adh.nex"))
    fel = h3.FELAnalyzer.create_and_fit(h3.Tree.from_newick(aln.embedded_tree_newick), aln, 0.1)
    fel.run()
    assert fel.global_log_l == pytest.approx(k["full_model_logl"], abs=k["delta"])
    assert len(fel.site_results) == 254


@pytest.mark.parametrize("case,fname,tree", [("cd2_meme", "cd2.fna", "cd2.nwk"), ("adh_meme", "adh.nex", None)])
def test_meme_create_and_fit_matches_hyphy25(golden_dir, known, case, fname, tree):
    import _hyphy3 as h3
    k = known[case]
    aln = h3.Alignment.load(str(golden_dir / fname))
    t = h3.Tree.from_newick_file(str(golden_dir / tree)) if tree else h3.Tree.from_newick(aln.embedded_tree_newick)
    meme = h3.MEMEAnalyzer.create_and_fit(t, aln, 0.1, full_model=False)
    res = meme.run()
    mle = np.array(k["mle"])
    assert len(res) == len(mle)
    r, rho = _corr(np.array([x.lrt for x in res]), mle[:, 5])
    rp, rhop = _corr(np.array([x.p_value for x in res]), mle[:, 6])
    assert r >= k["min_pearson_lrt"] and rho >= k["min_spearman_lrt"], (r, rho)
    assert rp >= k["min_pearson_p"] and rhop >= k["min_spearman_p"], (rp, rhop)
    assert meme.has_gtr_fit and meme.p_value_threshold == 0.1


def test_meme_create_and_fit_adh_full_model(golden_dir, known):
    import _hyphy3 as h3
    k = known["meme_full_fit_adh"]
    aln = h3.Alignment.load(str(golden_dir / "adh.nex"))
    meme = h3.MEMEAnalyzer.create_and_fit(h3.Tree.from_newick(aln.embedded_tree_newick), aln, 0.1, full_model=True)
    assert meme.global_log_l >= k["min_log_l"]
    assert abs(meme.base_params.beta - k["omega"]) < k["omega_tol"]


def test_meme_create_and_fit_rejects_bad_branch_set(golden_dir):
    import _hyphy3 as h3
    aln = h3.Alignment.load(str(golden_dir / "cd2.fna"))
    with pytest.raises(Exception):
        h3.MEMEAnalyzer.create_and_fit(h3.Tree.from_newick_file(str(golden_dir / "cd2.nwk")), aln, 0.1, False, "NoSuchMode")
