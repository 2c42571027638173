"""B200-native (sm_100a) one-sided Jacobi SVD: a drop-in for the 'jacobi'
solver of uncle-Slava/Pavel-s_SVD (svdbench.standalone.svd).

The directory name is not a Python identifier; import it with
``importlib.import_module('pavel-s_svd_b200')``.  Importing registers the
alias ``pavel_s_svd_b200`` so that ``pavel_s_svd_b200:factory`` also works as a
harness plug-in name (svdbench/algorithms.py:90-93).
"""
import sys as _sys

from .solvers import ALGORITHMS, COMPLEX_ALGORITHMS, REFERENCE_ALGORITHMS, Unsupported, svd, factory
from .batch import UnevenBatch, svd_uneven
from . import native

_sys.modules.setdefault("pavel_s_svd_b200", _sys.modules[__name__])

__all__ = ["ALGORITHMS", "COMPLEX_ALGORITHMS", "REFERENCE_ALGORITHMS", "Unsupported", "svd", "factory", "UnevenBatch",
           "svd_uneven", "native"]
