"""Helpers shared by the GPU tests: the package under test and the oracle."""
import importlib

import numpy as np

wos = importlib.import_module("tetsuhiro-wos_b200")

# Tolerances (relative L2 against the FP64 oracle).
TOL_FP64 = 1e-12   # FP64 kernels
TOL_FP32 = 1e-5    # FP32 kernels (FP64 phase arguments)


def rel_l2(a, b) -> float:
    den = np.sum(np.abs(b) ** 2)
    if den <= 0:
        return float(np.sqrt(np.sum(np.abs(a) ** 2)))
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) / den))


def tol(precision) -> float:
    return TOL_FP64 if precision == wos.FP64 else TOL_FP32
