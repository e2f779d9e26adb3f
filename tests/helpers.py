"""Shared helpers of the parity tests: running one Problem through an
instance (this library, the compiled reference, or the numpy oracle) and the
tolerances the comparisons use."""
import numpy as np

# Flag bits of beagle.h.
SINGLE, DOUBLE = 1 << 0, 1 << 1
SCALERS_RAW, SCALERS_LOG = 1 << 9, 1 << 10
PROCESSOR_CPU, PROCESSOR_GPU = 1 << 15, 1 << 16
FRAMEWORK_CUDA = 1 << 22
PRE_MANUAL, PRE_AUTO = 1 << 30, 1 << 31

# Tolerances: relative lnL error, and max |g - g_ref| / max |g_ref| for the
# branch gradient.  FP64 plain path 1e-10; mixed FP32 path 1e-6 (lnL) and
# 1e-4 (gradient).
TOL = {
    "double": dict(lnl=1e-10, grad=1e-8),
    "single": dict(lnl=1e-6, grad=1e-4),
}


def gpu_flags(precision, log_scalers=True, auto_transpose=False):
    pref = (DOUBLE if precision == "double" else SINGLE) | PROCESSOR_GPU
    pref |= SCALERS_LOG if log_scalers else SCALERS_RAW
    pref |= PRE_AUTO if auto_transpose else PRE_MANUAL
    req = (DOUBLE if precision == "double" else SINGLE) | FRAMEWORK_CUDA
    return pref, req


def run_b200(lib, problem, precision, gradient=True, log_scalers=True, auto_transpose=False):
    pref, req = gpu_flags(precision, log_scalers, auto_transpose)
    inst = lib.create(*problem.create_args(), preferenceFlags=pref, requirementFlags=req)
    problem.load(inst)
    transposed = problem.S > 4 and not auto_transpose
    lnl, grad = problem.evaluate(inst, gradient=gradient, transposed_pre=transposed)
    return inst, lnl, grad


def run_oracle(oracle, problem, gradient=True, log_scalers=True):
    flags = SCALERS_LOG if log_scalers else SCALERS_RAW
    inst = oracle.OracleInstance(*problem.create_args(), flags=flags)
    problem.load(inst)
    lnl, grad = problem.evaluate(inst, gradient=gradient)
    return inst, lnl, grad


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def grad_err(g, gref):
    g, gref = np.asarray(g), np.asarray(gref)
    return float(np.max(np.abs(g - gref)) / max(np.max(np.abs(gref)), 1e-300))
