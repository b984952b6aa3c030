"""nelson_b200: a B200-native Schur-complement Levenberg-Marquardt / Gauss-Newton
engine with the interface of nelson's DoubleSection / SolverCholeskySchur /
LevenbergMarquardt (see include/nelson_b200.h for the C ABI)."""
from .native import (PREC_FP64, PREC_MIXED, BAProblemGPU, GNSettings, LMSettings, NelsonError,  # noqa: F401
                     load)
from .problems import BAProblem, make_config  # noqa: F401

__all__ = ["BAProblemGPU", "LMSettings", "GNSettings", "PREC_FP64", "PREC_MIXED", "NelsonError", "load",
           "BAProblem", "make_config"]
