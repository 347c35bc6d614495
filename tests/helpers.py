"""Shared helpers for the parity tests (oracle = CPU restatement)."""
import numpy as np

# tolerances: max |gpu - oracle| / max |oracle|
TOL = {np.dtype(np.float64): 1e-12, np.dtype(np.complex128): 1e-12,
       np.dtype(np.float32): 2e-6, np.dtype(np.complex64): 2e-6}


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.abs(b).max()
    if den == 0:
        return np.abs(a).max()
    return np.abs(a - b).max() / den


def rand(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(shape)
    if np.dtype(dtype).kind == 'c':
        a = a + 1j * rng.standard_normal(shape)
    return a.astype(dtype)


def oracle_dtype(dtype):
    """The oracle computes in float64 / complex128."""
    return complex if np.dtype(dtype).kind == 'c' else float
