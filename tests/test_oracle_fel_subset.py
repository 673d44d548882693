"""FEL with a tested / background branch split (fel.hpp:215-266, :462-572), on the CPU.

* Branch selection (tree.hpp:893-1075) through the host Tree: the reference test's
  cd2_reduced "Leaves" partition (10 tested, 2 background) and Fig4E's {T}-tag
  detection under "All" (17 / 47, tests/test_fel.cpp:78-170), plus the other specs.
* The oracle's subset likelihood is pinned to the all-branches path: at
  beta_bg = beta the reference builds one model for every branch, so it must equal
  the all-tested FEL likelihood at (alpha, beta) (pinned to HyPhy 2.5 on CD2); with
  beta_bg != beta it must differ.  The optimiser is the N-dimensional Nelder-Mead
  that MEME uses (pinned to HyPhy 2.5 on CD2 and ADH).
* The oracle's subset search on the reference's "Leaves" case: invariant sites
  exactly zero with p = 1, the alternative never below the null.
"""
import json

import numpy as np
import pytest


@pytest.fixture(scope="module")
def leaves_case(golden_dir):
    return json.loads((golden_dir / "known_answers.json").read_text())["cd2_reduced_fel_leaves"]


def _host_tree(newick):
    import _hyphy3 as h3
    return h3.Tree.from_newick(newick)


def test_leaves_partition_matches_reference_counts(leaves_case):
    t = _host_tree(leaves_case["newick"])
    sel = t.select_branches(leaves_case["test_branches"])
    assert sel["num_selected"] == leaves_case["num_tested"]
    assert sel["num_unselected"] == leaves_case["num_background"]
    assert sorted(sel["unselected_names"]) == ["Node12", "Node8"]
    assert not sel["is_selected"][t.root_id]
    for nd in t.nodes:
        if nd.id != t.root_id:
            assert sel["is_selected"][nd.id] == nd.is_leaf


def test_fig4e_tags_select_the_tested_branches(golden_dir, known):
    import _hyphy3 as h3
    k = known["fig4e_tags"]
    aln = h3.Alignment.load(str(golden_dir / "Fig4E.nex"))
    assert aln.embedded_tree_newick
    t = h3.Tree.from_newick(aln.embedded_tree_newick)
    sel = t.select_branches("All", auto_detect_test_tags_when_all=True)
    assert sel["num_selected"] == k["num_tested"] and sel["num_unselected"] == k["num_background"]
    for nd in t.nodes:
        if nd.id != t.root_id:
            assert sel["is_selected"][nd.id] == (nd.model_tag == "T")
    # without detection "All" is every branch; the analyzer detects (fel.hpp:215-227)
    assert t.select_branches("All")["num_unselected"] == 0
    f = h3.FELAnalyzer(t, aln, h3.MG94Parameters())
    assert (f.num_tested, f.num_background) == (k["num_tested"], k["num_background"])


def test_branch_selection_specs(leaves_case):
    t = _host_tree("((a:1,b:1){FG}x:1,(c:1,d:1{bg})y:1,e:1)r;")
    names = lambda sel: sorted(sel["selected_names"])
    assert names(t.select_branches("Internal")) == ["x", "y"]
    assert names(t.select_branches("tips")) == ["a", "b", "c", "d", "e"]
    assert names(t.select_branches("{Foreground}")) == ["x"]           # tag synonyms
    assert names(t.select_branches("background")) == ["d"]
    assert names(t.select_branches("a, C ,internal")) == ["a", "c", "x", "y"]
    assert names(t.select_branches("unlabeled")) == ["a", "b", "c", "e", "y"]
    assert names(t.select_branches("All", auto_detect_test_tags_when_all=True)) == ["x"]
    assert names(t.select_branches("x", regex="^[ab]$")) == ["a", "b"]      # a regex wins
    assert names(t.select_branches("x", explicit_names=["{E}", "y"])) == ["e", "y"]
    assert names(t.select_branches("^[cd]$")) == ["c", "d"]                  # regex fallback
    with pytest.raises(RuntimeError, match="No branches matched"):
        t.select_branches("nothing")
    assert t.select_branches("nothing", throw_on_empty=False)["num_selected"] == 0


def _oracle_inputs(oracle, golden_dir, case):
    a = oracle.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    t = oracle.Tree.parse(case["newick"])
    leaf = t.is_leaf
    tested = [bool(leaf[i]) for i in range(t.num_nodes())]
    return a, t, tested


def test_subset_likelihood_reduces_to_all_tested(oracle, golden_dir, leaves_case):
    a, t, tested = _oracle_inputs(oracle, golden_dir, leaves_case)
    p = leaves_case["params"]
    run = oracle.fel_run(t, a, p, 0)                # FEL time lengths (every branch converted alike)
    for al, be in ((0.7, 1.3), (2.0, 0.4)):
        tot = sum(w * oracle.fel_subset_lnl(t, a, p, tested, -1.0, q, al, be, be) for q, w in enumerate(a.weights))
        ref = oracle.mg94_loglik(t, a, dict(p, alpha=1.0, beta=be / al), al, list(run["branch_lengths"]))
        assert tot == pytest.approx(ref, rel=1e-11, abs=1e-9)
        other = sum(w * oracle.fel_subset_lnl(t, a, p, tested, -1.0, q, al, be, 3.0 * be)
                    for q, w in enumerate(a.weights))
        assert abs(other - tot) > 1e-3


def test_subset_oracle_leaves_run(oracle, golden_dir, leaves_case):
    a, t, tested = _oracle_inputs(oracle, golden_dir, leaves_case)
    r = oracle.fel_run_tested(t, a, leaves_case["params"], tested)
    sp = np.array(a.site_pattern)
    for s in leaves_case["invariant_sites"]:
        p = sp[s]
        assert r["alpha"][p] == 0.0 and r["beta"][p] == 0.0 and r["p_value"][p] == 1.0 and r["evals"][p] == 0
    var = np.array(r["evals"]) > 0
    assert var.any()
    assert np.all(np.array(r["log_l_alt"])[var] >= np.array(r["log_l_null"])[var] - 1e-6)
    assert np.all(np.array(r["lrt"]) >= 0.0)
    bn = np.array(r["beta_nuisance"])[var]
    assert np.all((bn >= 1e-4) & (bn <= 1000.0))
    # the background's lengths carry the base conversion (no background omega given)
    assert r["bg_conversion"] == r["conversion"] and r["bg_length"] > 0.0
