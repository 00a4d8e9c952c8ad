"""sovereign_b200 -- B200-native Mehrotra predictor-corrector interior-point engine.

A drop-in for the LP / convex-QP interior-point path of Abhishekmishra2808/sovereign
(sovereign::InteriorPointSolver, sovereign::QpInteriorPointSolver): hand-written sm_100a CUDA
kernels behind the C ABI of include/sov_ipm.h (libsovipm.so), with this package as the Python
face of that ABI.
"""
from . import abi, problems  # noqa: F401
from .model import Model, Result  # noqa: F401

__all__ = ["abi", "problems", "Model", "Result"]
