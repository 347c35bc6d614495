"""The oracle's NumPy restatement against golden fixtures of the reference C.

tests/golden/golden.npz was produced by tests/golden/make_golden.py from the
reference's own compiled c/bmgs + c/bc.c + c/operators.c + c/transformers.c
(oracle/_ref).  Replaying the same inputs through the NumPy restatement must
give bit-identical outputs; this pins the oracle that the GPU tests use.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, 'golden'))

from make_golden import cases, run_case  # noqa: E402

GOLD = np.load(os.path.join(HERE, 'golden', 'golden.npz'))
CASES = cases()


def inputs_of(name):
    out = {}
    for k in GOLD.files:
        n, key = k.split('/')
        if n == name and key in ('a', 'f', 's', 'rho'):
            out[key] = GOLD[k]
    return out


@pytest.mark.parametrize('name,kind,p', CASES, ids=[c[0] for c in CASES])
def test_numpy_restatement_matches_reference_c(name, kind, p):
    res = run_case(kind, p, 'numpy', 0, arrays=inputs_of(name))
    assert np.array_equal(res['out'], GOLD[name + '/out'])
    if kind == 'poisson':
        assert int(res['niter']) == int(GOLD[name + '/niter'])
