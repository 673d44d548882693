"""Alignment::finalize on the device (h3g_alignment_compress; alignment.hpp:665-722, :893-911, :1021-1078).

Bit-exact parity with the oracle's restatement of the reference (codon translation with
IUPAC / '!' / stop / gap rules, patterns in first-site order, weights, site-to-pattern)
and with the host finalize for every derived field, on the reference's datasets, on
synthetic alignments with every character class and at tile boundaries, and with the
column hash cut to a few bits so that hash collisions must be resolved by comparison.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from hyphy3 import _capi
    c = _capi.Context(0)
    yield c
    c.close()


def _table(oracle, name="Universal"):
    g = oracle.genetic_code(name)
    t = np.full(64, -1, np.int8)
    idx = {"A": 0, "C": 1, "G": 2, "T": 3}
    for s, cod in enumerate(g["sense_codons"]):
        t[16 * idx[cod[0]] + 4 * idx[cod[1]] + idx[cod[2]]] = s
    return t


def _pos_counts(seqs):
    pc = np.zeros((3, 4), np.int64)
    idx = {c: i for i, c in enumerate("ACGT")}
    idx.update({c.lower(): i for c, i in list(idx.items())})
    idx["U"] = idx["u"] = 3
    for s in seqs:
        for i, ch in enumerate(s):
            if ch in idx:
                pc[i % 3, idx[ch]] += 1
    return pc


def _check_against_oracle(dev, ref, seqs=None):
    np.testing.assert_array_equal(dev["site_to_pattern"], np.asarray(ref.site_pattern))
    np.testing.assert_array_equal(dev["weight"], np.asarray(ref.weights, dtype=np.int64))
    np.testing.assert_array_equal(dev["states"], ref.states)
    np.testing.assert_array_equal(dev["masks"], ref.masks)
    # first sites are the first occurrences, in increasing order
    first = np.array([np.flatnonzero(dev["site_to_pattern"] == p)[0] for p in range(len(dev["weight"]))])
    np.testing.assert_array_equal(dev["first_site"], first)
    assert np.all(np.diff(first) > 0)
    if seqs is not None:
        np.testing.assert_array_equal(dev["pos_counts"], _pos_counts(seqs))


@pytest.mark.parametrize("fname", ["cd2.fna", "adh.nex", "CD2.nex", "Fig4E.nex", "cd2_reduced.fna"])
def test_datasets_match_oracle_and_host(oracle, golden_dir, fname):
    import _hyphy3 as h3
    host = h3.Alignment.load(str(golden_dir / fname))
    dev = h3.Alignment.load(str(golden_dir / fname), device=True)
    ref = oracle.Alignment.load(str(golden_dir / fname))
    hs, hm, hw = host.pattern_arrays()
    ds, dm, dw = dev.pattern_arrays()
    np.testing.assert_array_equal(ds, hs)
    np.testing.assert_array_equal(dm, hm)
    np.testing.assert_array_equal(dw, hw)
    np.testing.assert_array_equal(ds, ref.states)
    np.testing.assert_array_equal(dm, ref.masks)
    np.testing.assert_array_equal(dev.site_to_pattern, host.site_to_pattern)
    np.testing.assert_array_equal(dev.site_to_pattern, ref.site_pattern)
    assert dev.pattern_sites() == host.pattern_sites()
    # frequencies from the device's counts through the same CF3x4 code: identical
    np.testing.assert_array_equal(dev.pos_nuc_frequencies, host.pos_nuc_frequencies)
    np.testing.assert_array_equal(dev.codon_frequencies, host.codon_frequencies)
    np.testing.assert_array_equal(dev.nuc_frequencies, host.nuc_frequencies)
    assert (dev.num_taxa, dev.num_codons, dev.num_nucleotides) == (host.num_taxa, host.num_codons, host.num_nucleotides)


ALPHABET = list("ACGTacgtUuRYSWKMBDHVNnrykm-?.!X*0 ") + ["T", "A", "G", "C"] * 6


def _random_alignment(rng, T, C, dup=0.5, stops=True):
    """Columns drawn from a small pool (duplicates) or fresh, every character class present."""
    pool = [[rng.choice(ALPHABET) + rng.choice(ALPHABET) + rng.choice(ALPHABET) for _ in range(T)] for _ in range(max(1, C // 8))]
    cols = []
    for _ in range(C):
        if rng.random() < dup:
            cols.append(list(pool[rng.integers(len(pool))]))
        else:
            cols.append([rng.choice(ALPHABET) + rng.choice(ALPHABET) + rng.choice(ALPHABET) for _ in range(T)])
    if stops and C > 2 and T > 1:
        cols[1][0] = "TAA"
        cols[2][T - 1] = "tga"
    return ["".join(cols[c][t] for c in range(C)) for t in range(T)]


@pytest.mark.parametrize("T,C,seed", [(1, 1, 0), (1, 40, 1), (33, 1, 2), (31, 33, 3), (32, 32, 4), (33, 65, 5), (70, 300, 6),
                                      (200, 97, 7)])
def test_synthetic_edge_cases(ctx, oracle, T, C, seed):
    rng = np.random.default_rng(seed)
    seqs = _random_alignment(rng, T, C)
    ref = oracle.Alignment.from_sequences([f"t{i}" for i in range(T)], seqs, "Universal")
    dev = ctx.alignment_compress(seqs, _table(oracle))
    _check_against_oracle(dev, ref, seqs)
    assert dev["rounds"] == 1


def test_all_identical_and_all_distinct_columns(ctx, oracle):
    T = 40
    same = ["ACGTTA" * 50] * T
    dev = ctx.alignment_compress(same, _table(oracle))
    assert len(dev["weight"]) == 2 and list(dev["weight"]) == [50, 50]
    rng = np.random.default_rng(11)
    nuc = np.array(list("ACGT"))
    distinct = ["".join(rng.choice(nuc, 3 * 400)) for _ in range(T)]
    ref = oracle.Alignment.from_sequences([f"t{i}" for i in range(T)], distinct, "Universal")
    dev = ctx.alignment_compress(distinct, _table(oracle))
    _check_against_oracle(dev, ref, distinct)
    assert len(dev["weight"]) == 400


def test_vertebrate_mitochondrial_code(ctx, oracle):
    rng = np.random.default_rng(3)
    seqs = _random_alignment(rng, 45, 120)
    seqs[0] = "AGA" + seqs[0][3:]              # a stop in the vertebrate mitochondrial code
    seqs[1] = "TGA" + seqs[1][3:]              # tryptophan there
    ref = oracle.Alignment.from_sequences([f"t{i}" for i in range(45)], seqs, "Vertebrate-mtDNA")
    dev = ctx.alignment_compress(seqs, _table(oracle, "Vertebrate-mtDNA"))
    _check_against_oracle(dev, ref, seqs)


@pytest.mark.parametrize("bits", [1, 3, 8])
def test_hash_collisions_are_resolved_by_comparison(ctx, oracle, bits):
    """With the column hash cut to a few bits, different columns collide; they are told apart by full
    comparison over several rounds and the result is unchanged."""
    rng = np.random.default_rng(bits)
    seqs = _random_alignment(rng, 37, 500, dup=0.6)
    ref = oracle.Alignment.from_sequences([f"t{i}" for i in range(37)], seqs, "Universal")
    dev = ctx.alignment_compress(seqs, _table(oracle), hash_bits=bits)
    _check_against_oracle(dev, ref, seqs)
    assert dev["rounds"] > 1


def test_large_alignment_matches_host(ctx, oracle):
    """1024 taxa x 8000 codons (gaps, ambiguity) through the device and the host finalize."""
    import _hyphy3 as h3
    from hyphy3.simulate import make_workload
    wl = make_workload(1, n_sites=8000, n_taxa=1024)
    host = h3.Alignment.from_sequences(wl.names, wl.seqs)
    dev = h3.Alignment.from_sequences(wl.names, wl.seqs, device=True)
    hs, hm, hw = host.pattern_arrays()
    ds, dm, dw = dev.pattern_arrays()
    np.testing.assert_array_equal(ds, hs)
    np.testing.assert_array_equal(dm, hm)
    np.testing.assert_array_equal(dw, hw)
    np.testing.assert_array_equal(dev.site_to_pattern, host.site_to_pattern)
    np.testing.assert_array_equal(dev.codon_frequencies, host.codon_frequencies)


def test_rejects_bad_arguments(ctx, oracle):
    from hyphy3 import _capi
    with pytest.raises(_capi.H3GError):
        ctx.alignment_compress(["ACGTA", "ACGTT"], _table(oracle))          # not in frame
    bad = _table(oracle)
    bad[0] = 70
    with pytest.raises(_capi.H3GError):
        ctx.alignment_compress(["ACGTAA"], bad)
    out = ctx.alignment_compress(["ACGTAA"], _table(oracle))                # still usable after errors
    assert list(out["weight"]) == [1, 1]
