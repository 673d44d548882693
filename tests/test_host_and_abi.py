"""Host-side data model and the C ABI library (CPU only: no kernel is launched)."""
import re
import pathlib

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def h3():
    import _hyphy3
    return _hyphy3


@pytest.mark.parametrize("fname", ["cd2_reduced.fna", "adh.nex", "CD2.nex"])
def test_alignment_matches_oracle(h3, oracle, golden_dir, fname):
    a = h3.Alignment.load(str(golden_dir / fname))
    b = oracle.Alignment.load(str(golden_dir / fname))
    st, mk, w = a.pattern_arrays()
    assert a.num_taxa == b.num_taxa and a.num_codons == b.num_codons and a.num_patterns == b.num_patterns
    np.testing.assert_array_equal(st, b.states)
    np.testing.assert_array_equal(mk, b.masks)
    np.testing.assert_array_equal(w, b.weights)
    np.testing.assert_allclose(a.codon_frequencies, b.pi, rtol=0, atol=1e-15)
    np.testing.assert_allclose(a.pos_nuc_frequencies, b.pos_freq, rtol=0, atol=1e-15)
    if a.embedded_tree_newick:
        t = h3.Tree.from_newick(a.embedded_tree_newick)
        u = oracle.Tree.parse(b.embedded_tree)
        assert t.parents == u.parent and t.post_order == u.post_order


def test_tree_parsing_and_unrooting(h3, oracle, golden_dir):
    nwk = (golden_dir / "cd2_reduced.nwk").read_text()
    t = h3.Tree.from_newick(nwk)
    u = oracle.Tree.parse(nwk)
    assert t.parents == u.parent and t.get_branch_lengths() == u.branch_lengths
    for s in ["((a:1,b:2):0.5,(c:1,d:1):0.25);", "(((x:1,y:1)'q r':2,z:3):0.1,w:0.2);", "((a,b),c,(d,(e,f)));"]:
        for rooted in (True, False):
            t = h3.Tree.from_newick(s, keep_rooted=rooted)
            u = oracle.Tree.parse(s, keep_rooted=rooted)
            assert t.parents == u.parent and t.get_branch_lengths() == u.branch_lengths


def test_unbalanced_newick_raises(h3):
    with pytest.raises(Exception):
        h3.Tree.from_newick("((a,b);")


def test_eigensystem_reproduces_expm(h3, golden_dir):
    import scipy.linalg as sl
    a = h3.Alignment.load(str(golden_dir / "adh.nex"))
    p = h3.MG94Parameters()
    p.beta, p.theta_CT = 0.4, 2.0
    e = h3.mg94_eigensystem(a, p)
    for t in (0.01, 0.1, 1.0):
        P = e["U"] @ np.diag(np.exp(np.asarray(e["lam"]) * t)) @ e["V"]
        np.testing.assert_allclose(P, sl.expm(e["Q"] * t), atol=1e-11)
    np.testing.assert_allclose(e["Q"].sum(1), 0.0, atol=1e-12)


def test_simulator_is_seeded():
    from hyphy3.simulate import make_workload
    a = make_workload(1, n_sites=40, n_taxa=12)
    b = make_workload(1, n_sites=40, n_taxa=12)
    assert a.seqs == b.seqs and a.newick == b.newick
    gaps = sum(s.count("---") for s in make_workload(1, n_sites=400, n_taxa=16).seqs)
    assert 0.01 < gaps / (400 * 16) < 0.06


def _declared_symbols():
    text = (ROOT / "include" / "h3g.h").read_text()
    return sorted(set(re.findall(r"\b(h3g_[A-Za-z_]+)\s*\(", text)))


def test_capi_library_exports_every_declared_symbol():
    import ctypes
    from hyphy3 import _capi
    lib = _capi.load()
    declared = _declared_symbols()
    assert len(declared) >= 10
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_capi.EXPORTED)
    assert lib.h3g_version().decode().startswith("hyphy3-b200")
    # without a device the context cannot be created and nothing is launched
    h = ctypes.c_void_p()
    st = lib.h3g_ctx_create(0, None, ctypes.byref(h))
    import torch
    if not torch.cuda.is_available():
        assert st == _capi.H3G_ERR_CUDA


def test_gpu_entry_points_fail_loudly_without_device(h3, golden_dir):
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    a = h3.Alignment.load(str(golden_dir / "cd2_reduced.fna"))
    t = h3.Tree.from_newick((golden_dir / "cd2_reduced.nwk").read_text())
    with pytest.raises(RuntimeError, match="libh3g"):
        h3.compute_branch_length_gradients(t, a, h3.MG94Parameters())


def test_package_exports_the_device_drivers():
    """hyphy3 re-exports the reference package's names for everything that runs on the device
    (python/hyphy3/__init__.py of the reference), and every name in __all__ resolves."""
    import hyphy3
    for name in hyphy3.__all__:
        assert hasattr(hyphy3, name), name
    for name in ("FELAnalyzer", "MEMEAnalyzer", "BUSTEDAnalyzer", "BUSTEDSettings", "BUSTEDResult", "RELAXAnalyzer",
                 "RELAXSettings", "GTRFitter", "MG94Fitter", "compute_gtr_log_likelihood"):
        assert name in hyphy3.__all__, name
