"""HyPhy 3 likelihood core on NVIDIA B200.

Re-exports the core types, the likelihood entry points and the analysis drivers of the
reference package (python/hyphy3/__init__.py) that run on the device from the _hyphy3 module:
FELAnalyzer, MEMEAnalyzer, BUSTEDAnalyzer (fits, two-set model, auto K), RELAXAnalyzer,
MG94Fitter, GTRFitter and the GTR likelihood; ABSRELAnalyzer (hyphy3.absrel) and joint fits over
batches of genes (hyphy3.batch).  FUBAR and the other drivers are not part of this package.
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
    BUSTEDFit,
    BUSTEDRateDistribution,
    BUSTEDResult,
    BUSTEDSettings,
    GTRFitResult,
    GTRFitter,
    GTRMatrix,
    GTRParameters,
    RELAXAnalyzer,
    RELAXModelFit,
    RELAXRateDistribution,
    RELAXResult,
    RELAXSettings,
    compute_gtr_gradients,
    compute_gtr_log_likelihood,
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
    set_eigensolver,
    get_eigensolver,
    set_memory_budget,
    get_memory_budget,
    set_precision,
)

from . import autograd  # noqa: E402
from .absrel import ABSRELAnalyzer  # noqa: E402
from .batch import fit_branch_lengths  # noqa: E402

__version__ = "3.0.0"
__all__ = [
    "Alignment", "FELAnalyzer", "FELSettings", "FELSiteResult", "FitResult", "MG94Fitter", "GeneticCode", "MG94Parameters", "Tree", "TreeNode", "build_leaf_to_taxon_map",
    "compute_branch_length_gradients", "compute_joint_frechet_gradients", "compute_mg94_log_likelihood",
    "compute_mixture_gradients", "compute_tree_log_likelihood_from_P", "get_precision", "library_version",
    "mg94_eigensystem", "set_precision", "autograd", "MEMEAnalyzer", "MEMESiteResult", "BUSTEDAnalyzer", "BUSTEDFit",
    "BUSTEDRateDistribution", "BUSTEDResult", "BUSTEDSettings", "GTRFitResult", "GTRFitter", "GTRMatrix", "GTRParameters",
    "RELAXAnalyzer", "RELAXModelFit", "RELAXRateDistribution", "RELAXResult", "RELAXSettings", "compute_gtr_gradients",
    "compute_gtr_log_likelihood", "ABSRELAnalyzer", "fit_branch_lengths", "set_eigensolver", "get_eigensolver",
    "set_memory_budget", "get_memory_budget",
]
