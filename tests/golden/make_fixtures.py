"""Copy the reference's own parity fixtures for the likelihood path into tests/golden/.

The reference pins its likelihood core with a handful of bundled datasets and a
HyPhy 2.5 ground-truth JSON; the GPU box has no copy of the reference, so the
files its tests read are copied here verbatim (data, not code) and the known
answers its tests assert are recorded in known_answers.json with their source.

Run from the repository root with the reference checked out read-only:
    python tests/golden/make_fixtures.py /path/to/reference
(or set HYPHY3_REFERENCE to that path); there is no default location.
"""
import json
import pathlib
import re
import shutil
import sys

FILES = {
    # benchmarks/data/cd2_reduced.fna: read by tests/test_core.cpp:12-37, :95-124, :149-223
    "cd2_reduced.fna": "benchmarks/data/cd2_reduced.fna",
    "cd2_reduced.nwk": "benchmarks/data/cd2_reduced.nwk",
    # adh.nex: tests/test_cpp_autograd.cpp:47-104, python/tests/test_python_autograd.py:114-153
    "adh.nex": "benchmarks/data/adh.nex",
    # CD2 full alignment with embedded tree (tests/test_fel_cd2_parity.cpp)
    "CD2.nex": "benchmarks/data/CD2.nex",
    "cd2_reduced_point_truth.json": "benchmarks/ground_truth/cd2_reduced_point_truth.json",
    # FEL parity on CD2 with matched branch lengths: tests/test_fel_cd2_parity.cpp:66-118
    "cd2.fna": "benchmarks/data/cd2.fna",
    "cd2_fitted.nwk": "benchmarks/data/cd2_fitted.nwk",
    # BGLOBIN and COXI (Vertebrate-mtDNA code) with embedded trees: tests/test_fel_multi_dataset.cpp:123-197
    "bglobin.nex": "benchmarks/data/bglobin.nex",
    "COXI.nex": "benchmarks/data/COXI.nex",
    # CD2 topology without lengths ({Group} tags) that FEL/MEME create_and_fit start from:
    # tests/test_fel_multi_dataset.cpp:66-69, tests/test_meme.cpp:66-69
    "cd2.nwk": "benchmarks/data/cd2.nwk",
    # FEL branch-subset selection by {T} tags in the embedded tree: tests/test_fel.cpp:128-170
    "Fig4E.nex": "tests/data/Fig4E.nex",
}


def main(ref: str) -> None:
    ref_root = pathlib.Path(ref)
    out = pathlib.Path(__file__).resolve().parent
    for dst, src in FILES.items():
        shutil.copyfile(ref_root / src, out / dst)
    truth = json.loads((ref_root / FILES["cd2_reduced_point_truth.json"]).read_text())
    known = {
        "cd2_reduced": {
            "source": "benchmarks/ground_truth/cd2_reduced_point_truth.json; asserted in tests/test_core.cpp:95-124",
            "newick": "((((Pig:0.147969,Cow:0.213430):0.085099,Horse:0.165787,Cat:0.264806):0.058611,"
                      "((RhMonkey:0.002015,Baboon:0.003108):0.022733,(Human:0.004349,Chimp:0.000799):0.011873)"
                      ":0.101856):0.340802,Rat:0.050958,Mouse:0.097950);",
            "params": {"alpha": 1.0, "beta": 0.5, "theta": [1.0, 1.0, 1.0, 2.0, 1.0]},
            "point_mg94_logl": truth["point_mg94_logl"],
            "sense_codons": truth["sense_codons"][0],
            "taxa": truth["taxa"],
            "sites_codon": truth["sites_codon"],
            # tests/test_core.cpp:21-24 (empirical nucleotide frequencies, epsilon 1e-4)
            "nuc_freqs_test_core": [0.456140, 0.114035, 0.254386, 0.175439],
        },
        "cd2_reduced_frechet": {
            "source": "tests/test_core.cpp:149-223 (analytic vs central FD, h=1e-6, |d|/(|g|+1) < 1e-4)",
            "params": {"alpha": 1.0, "beta": 0.45, "theta": [0.8, 1.2, 0.6, 1.8, 0.9]},
            "min_branch_length": 1e-4,
        },
        "adh_autograd": {
            "source": "tests/test_cpp_autograd.cpp:47-104; python/tests/test_python_autograd.py:114-153",
            "params": {"alpha": 1.0, "beta": 0.4, "theta": [1, 1, 1, 1, 1]},
            "branch_length": 0.05, "fd_eps": 1e-6, "rel_err": 1e-5,
            "num_taxa": 23, "num_codons": 254, "num_nodes": 44,
        },
    }
    # global MG94 fit of adh (full model: every branch, omega, GTR rates): python/tests/test_python_autograd.py:46-55
    known["adh_global_fit"] = {
        "source": "python/tests/test_python_autograd.py:46-55 (FELAnalyzer.create_and_fit global_log_l, delta 5)",
        "full_model_logl": -4686.73, "delta": 5.0,
    }
    # HyPhy 2.5 FEL per-site table for CD2 (columns alpha, beta, alpha=beta, LRT, p-value, total branch
    # length); only the MLE content of benchmarks/ground_truth/cd2_fel.json is kept
    fel = json.loads((ref_root / "benchmarks/ground_truth/cd2_fel.json").read_text())
    known["cd2_fel"] = {
        "source": "benchmarks/ground_truth/cd2_fel.json (HyPhy 2.5); compared in tests/test_fel_cd2_parity.cpp:66-118",
        "headers": [h[0] for h in fel["MLE"]["headers"]],
        "mle": fel["MLE"]["content"]["0"],
        # tests/test_fel_cd2_parity.cpp:71-77
        "params": {"alpha": 1.0, "beta": 1.012387352492807,
                   "theta": [0.5521777318173139, 0.2653120245806623, 0.4932059218537349, 1.03133955537726,
                             0.3054313963126315]},
        # tests/test_fel_cd2_parity.cpp:113-116
        "min_pearson_lrt": 0.998, "min_spearman_lrt": 0.995, "min_pearson_p": 0.993, "min_spearman_p": 0.995,
    }
    # HyPhy 2.5 MEME per-site tables (CD2, ADH) with the global MG94xREV fit they were computed on: the tree with
    # that fit's branch lengths, omega and the GTR exchangeabilities.  Thresholds: tests/test_meme.cpp:66-150.
    known["cd2_meme"] = meme_case(ref_root, "cd2_meme_rel.json", "tests/test_meme.cpp:66-104", 0.95, 0.95, 0.95, 0.95)
    known["adh_meme"] = meme_case(ref_root, "adh_meme_rel.json", "tests/test_meme.cpp:106-144", 0.95, 0.92, 0.95, 0.95)
    known.update(fel_subset_cases(ref_root))
    # HyPhy 2.5's nucleotide GTR fits (rates, frequencies, branch lengths, log-likelihood) recorded in the
    # FEL ground truth of the reference's parity tests (tests/test_fel_multi_dataset.cpp:195-196)
    known["cd2_gtr"] = gtr_case(ref_root, "cd2_fel.json", "cd2.fna")
    known["adh_gtr"] = gtr_case(ref_root, "adh_fel.json", "adh.nex")
    # FEL from an alignment and a tree alone (GTR fit, global MG94 fit, FEL) against HyPhy 2.5:
    # tests/test_fel_multi_dataset.cpp:66-121
    known["fel_e2e_cd2"] = fel_e2e_case(ref_root, "cd2_fel.json", "tests/test_fel_multi_dataset.cpp:66-92",
                                        "cd2.fna", "cd2.nwk", True, 0.998, 0.995)
    known["fel_e2e_adh"] = fel_e2e_case(ref_root, "adh_fel_rel.json", "tests/test_fel_multi_dataset.cpp:94-121",
                                        "adh.nex", None, False, 0.998, 0.998)
    known["fel_e2e_bglobin"] = fel_e2e_case(ref_root, "bglobin_fel_rel.json", "tests/test_fel_multi_dataset.cpp:123-150",
                                            "bglobin.nex", None, False, 0.998, 0.998)
    # p-value correlations, the GTR log-likelihood (relative 1e-4) and omega (0.005): :152-197
    known["fel_e2e_coxi"] = fel_e2e_case(ref_root, "coxi_fel_rel.json", "tests/test_fel_multi_dataset.cpp:152-197",
                                         "COXI.nex", None, False, 0.995, 0.995, code="Vertebrate-mtDNA",
                                         min_p=(0.995, 0.995), omega_tol=0.005)
    # BUSTED on CD2 from cd2.nwk against HyPhy 2.5 (srv on): tests/test_busted.cpp:17-86
    b = json.loads((ref_root / "benchmarks/ground_truth/cd2_busted.json").read_text())
    known["cd2_busted"] = {
        "source": "benchmarks/ground_truth/cd2_busted.json (HyPhy 2.5, srv on); compared in tests/test_busted.cpp:17-86",
        "gtr_log_l": b["fits"]["Nucleotide GTR"]["Log Likelihood"],
        "mg94_log_l": b["fits"]["MG94xREV with separate rates for branch sets"]["Log Likelihood"],
        "unconstrained_log_l": b["fits"]["Unconstrained model"]["Log Likelihood"],
        "constrained_log_l": b["fits"]["Constrained model"]["Log Likelihood"],
        "lrt": b["test results"]["LRT"], "p_value": b["test results"]["p-value"],
        # tolerances of the reference test
        "tol_gtr": 1.0, "tol_mg94": 0.05, "tol_fit": 2.5, "tol_lrt": 1.5, "max_p": 0.01,
    }
    # RELAX on Fig4E (tagged test / reference sets) against HyPhy 2.5.101: tests/test_relax.cpp:17-100
    known["fig4e_relax"] = {
        "source": "tests/test_relax.cpp:17-100 (Fig4E.nex, embedded tree, {T}/{R} tags; HyPhy 2.5.101 relax, 3 rates)",
        "num_test": 17, "num_reference": 47,
        "gtr_log_l": -5317.276, "tol_gtr": 0.5,
        "max_omega_R": 0.25, "min_omega_T": 0.40,
        "alt_minus_mg94": 2.18, "tol_alt_minus_mg94": 1.5, "min_alt": -4983.5,
        "min_null": -5045.16, "max_null": -5000.0,
        "max_k": 0.01, "lrt": 123.27, "tol_lrt": 8.0, "max_p": 1e-15,
    }
    # MEME create_and_fit with the full MG94 fit on ADH: tests/test_meme.cpp:145-160 (HyPhy 2.5: -4686.18, 0.0941)
    known["meme_full_fit_adh"] = {
        "source": "tests/test_meme.cpp:145-160 (global_log_l >= -4687.5, |omega - 0.0941| < 0.01)",
        "min_log_l": -4687.5, "omega": 0.0941, "omega_tol": 0.01,
    }
    (out / "known_answers.json").write_text(json.dumps(known, indent=1) + "\n")


def fel_e2e_case(ref_root: pathlib.Path, name: str, test_ref: str, alignment: str, tree, full_model: bool,
                 r_lrt: float, rho_lrt: float, code=None, min_p=None, omega_tol=None) -> dict:
    """HyPhy's per-site LRT / p-value columns, its nucleotide GTR and global MG94xREV fits for a create_and_fit
    run; tree None means the alignment's embedded tree.  min_p / omega_tol: the p-value correlations and the
    omega tolerance where the reference test checks them."""
    g = json.loads((ref_root / "benchmarks/ground_truth" / name).read_text())
    fit = g["fits"]["Global MG94xREV"]
    mle = g["MLE"]["content"]["0"]
    return {
        "source": f"benchmarks/ground_truth/{name} (HyPhy 2.5); compared in {test_ref}",
        "alignment": alignment, "tree": tree, "full_model": full_model, "genetic_code": code,
        "lrt": [row[3] for row in mle], "p_value": [row[4] for row in mle],
        "mg94_omega": fit["Rate Distributions"]["non-synonymous/synonymous rate ratio for *test*"][0][0],
        "mg94_log_l": fit["Log Likelihood"],
        "gtr_log_l": g["fits"]["Nucleotide GTR"]["Log Likelihood"],
        "min_pearson_lrt": r_lrt, "min_spearman_lrt": rho_lrt,
        "min_pearson_p": min_p[0] if min_p else None, "min_spearman_p": min_p[1] if min_p else None,
        "omega_tol": omega_tol,
    }


def fel_subset_cases(ref_root: pathlib.Path) -> dict:
    """The branch-subset FEL cases of tests/test_fel.cpp: the cd2_reduced "Leaves" run (its fitted
    tree, base parameters, tested / background counts and invariant sites) and the Fig4E {T}-tag
    counts, read from the test source."""
    src = (ref_root / "tests" / "test_fel.cpp").read_text()
    lines = src.splitlines()

    def case(title):
        start = next(i for i, ln in enumerate(lines) if "TEST_CASE" in ln and title in ln)
        end = next((i for i in range(start + 1, len(lines)) if "TEST_CASE" in lines[i]), len(lines))
        return start, "\n".join(lines[start:end])

    s0, leaves = case("Leaves mode")
    nwk = re.search(r'nwk_fitted\s*=\s*"([^"]+)"', leaves).group(1)
    val = {k: float(v) for k, v in re.findall(r"base_p\.(\w+)\s*=\s*([-0-9.eE]+);", leaves)}
    theta = [val[k] for k in ("theta_AC", "theta_AT", "theta_CG", "theta_CT", "theta_GT")]
    n_t = int(re.search(r"num_tested\s*==\s*(\d+)", leaves).group(1))
    n_b = int(re.search(r"num_background\s*==\s*(\d+)", leaves).group(1))
    inv = sorted({int(i) for i in re.findall(r"results\[(\d+)\]\.p_value\s*==\s*1\.0", leaves)})
    s1, tags = case("Fig4E")
    t_t = int(re.search(r"num_tested\s*==\s*(\d+)", tags).group(1))
    t_b = int(re.search(r"num_background\s*==\s*(\d+)", tags).group(1))
    return {
        "cd2_reduced_fel_leaves": {
            "source": f"tests/test_fel.cpp:{s0 + 1} (cd2_reduced.fna, test_branches = Leaves)",
            "newick": nwk, "test_branches": "Leaves",
            "params": {"alpha": val["alpha"], "beta": val["beta"], "theta": theta},
            "num_tested": n_t, "num_background": n_b, "invariant_sites": inv,
        },
        "fig4e_tags": {
            "source": f"tests/test_fel.cpp:{s1 + 1} (Fig4E.nex embedded tree, test_branches = All, {{T}} tags)",
            "num_tested": t_t, "num_background": t_b,
        },
    }


def labelled_newick(topology: str, lengths: dict) -> str:
    """Attach ':length' to every named node of a HyPhy tree string (names only, no lengths)."""
    return re.sub(r"([A-Za-z_][A-Za-z0-9_]*)", lambda m: f"{m.group(1)}:{lengths[m.group(1)]!r}", topology) + ";"


def gtr_case(ref_root: pathlib.Path, name: str, alignment: str) -> dict:
    d = json.loads((ref_root / "benchmarks" / "ground_truth" / name).read_text())
    g = d["fits"]["Nucleotide GTR"]
    lengths = {k: v["Nucleotide GTR"] for k, v in d["branch attributes"]["0"].items()}
    r = g["Rate Distributions"]
    pairs = ["A to nucleotide C", "A to nucleotide T", "C to nucleotide G", "C to nucleotide T", "G to nucleotide T"]
    return {
        "source": f"benchmarks/ground_truth/{name} (HyPhy 2.5): fits / Nucleotide GTR and its branch lengths",
        "alignment": alignment, "newick": labelled_newick(d["input"]["trees"]["0"], lengths),
        "theta": [r[f"Substitution rate from nucleotide {x}"] for x in pairs],
        "freqs": [x[0] for x in g["Equilibrium frequencies"]], "log_l": g["Log Likelihood"],
    }


def meme_case(ref_root: pathlib.Path, name: str, test_ref: str, r_lrt, rho_lrt, r_p, rho_p) -> dict:
    g = json.loads((ref_root / "benchmarks/ground_truth" / name).read_text())
    fit = g["fits"]["Global MG94xREV"]
    gtr = g["fits"]["Nucleotide GTR"]["Rate Distributions"]
    rate = lambda a, b: gtr[f"Substitution rate from nucleotide {a} to nucleotide {b}"]
    lengths = {k: v["Global MG94xREV"] for k, v in g["branch attributes"]["0"].items()}
    return {
        "source": f"benchmarks/ground_truth/{name} (HyPhy 2.5); compared in {test_ref}",
        "headers": [h[0] for h in g["MLE"]["headers"]],
        "mle": g["MLE"]["content"]["0"],
        "newick": labelled_newick(g["input"]["trees"]["0"], lengths),
        "params": {"alpha": 1.0, "beta": fit["Rate Distributions"]["non-synonymous/synonymous rate ratio for *test*"][0][0],
                   "theta": [rate("A", "C"), rate("A", "T"), rate("C", "G"), rate("C", "T"), rate("G", "T")]},
        "global_log_l": fit["Log Likelihood"],
        "min_pearson_lrt": r_lrt, "min_spearman_lrt": rho_lrt, "min_pearson_p": r_p, "min_spearman_p": rho_p,
    }


if __name__ == "__main__":
    import os
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HYPHY3_REFERENCE")
    if not src:
        sys.exit("usage: python tests/golden/make_fixtures.py <reference checkout>  (or set HYPHY3_REFERENCE)")
    main(src)
