"""HyPhy 3 likelihood core on NVIDIA B200.

Re-exports the core types and likelihood entry points of the reference
package (python/hyphy3/__init__.py) from the device-backed _hyphy3 module.
Of the analysis drivers, FELAnalyzer and MEMEAnalyzer (every branch tested),
MG94Fitter and the likelihood core of BUSTEDAnalyzer (evaluate_log_l and the
EM expectation steps) run on the device; the others (BUSTED's fit driver,
aBSREL, RELAX, ...) are not part of this package.
"""
import os
import sys

_here = os.path.dirname(os.path.abspath(__file__))
_pydir = os.path.dirname(_here)
if _pydir not in sys.path:
    sys.path.insert(0, _pydir)

from _hyphy3 import (  # noqa: E402
    Alignment,
    BUSTEDAnalyzer,
    FELAnalyzer,
    FELSettings,
    FELSiteResult,
    FitResult,
    MEMEAnalyzer,
    MEMESiteResult,
    MG94Fitter,
    GeneticCode,
    MG94Parameters,
    Tree,
    TreeNode,
    build_leaf_to_taxon_map,
    compute_branch_length_gradients,
    compute_joint_frechet_gradients,
    compute_mg94_log_likelihood,
    compute_mixture_gradients,
    compute_tree_log_likelihood_from_P,
    get_precision,
    library_version,
    mg94_eigensystem,
    set_precision,
)

from . import autograd  # noqa: E402

__version__ = "3.0.0"
__all__ = [
    "Alignment", "FELAnalyzer", "FELSettings", "FELSiteResult", "FitResult", "MG94Fitter", "GeneticCode", "MG94Parameters", "Tree", "TreeNode", "build_leaf_to_taxon_map",
    "compute_branch_length_gradients", "compute_joint_frechet_gradients", "compute_mg94_log_likelihood",
    "compute_mixture_gradients", "compute_tree_log_likelihood_from_P", "get_precision", "library_version",
    "mg94_eigensystem", "set_precision", "autograd",
]
