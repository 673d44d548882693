"""aBSREL on the device against the reference's own acceptance test (tests/test_absrel.cpp:17-100).

Beta-globin (17 taxa, 144 codons), max 3 rate classes, p threshold 0.05, every branch tested:
GTR lnL in (-4100, -3800), baseline MG94 above GTR, full adaptive model at least the baseline,
31 tested branches, LRT >= 0 and p-values in [0, 1] everywhere, at least one positive branch.
"""
import time

import pytest

pytestmark = pytest.mark.gpu


def test_absrel_bglobin_meets_reference_acceptance(golden_dir):
    import _hyphy3 as h
    from hyphy3.absrel import ABSRELAnalyzer
    a = h.Alignment.load(str(golden_dir / "bglobin.nex"))
    t = h.Tree.from_newick(a.embedded_tree_newick)
    an = ABSRELAnalyzer(t, a, max_rate_classes=3, p_threshold=0.05)
    t0 = time.perf_counter()
    res = an.run()
    secs = time.perf_counter() - t0
    an.close()
    gtr, base, full = res["gtr_fit"]["log_likelihood"], res["baseline_fit"]["log_likelihood"], \
        res["full_adaptive_fit"]["log_likelihood"]
    print(f"\naBSREL bglobin: GTR {gtr:.3f}  baseline {base:.3f}  full adaptive {full:.3f}  "
          f"positive {res['positive_branches']}  {res['evaluations']} evaluations, {secs:.1f} s")
    assert -4100.0 < gtr < -3800.0
    assert base > gtr
    assert full >= base
    assert len(res["tested_branches"]) == 31
    for name in res["tested_branches"]:
        b = res["branches"][name]
        assert b["lrt"] >= 0.0
        assert 0.0 <= b["uncorrected_p_value"] <= 1.0
        assert 0.0 <= b["corrected_p_value"] <= 1.0
        assert abs(sum(b["weights"]) - 1.0) < 1e-9
    assert len(res["positive_branches"]) > 0
    assert any(res["branches"][n]["rate_classes"] > 1 for n in res["tested_branches"])
