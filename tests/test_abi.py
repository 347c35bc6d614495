"""The C ABI library loads, exports every symbol include/gpwgrid.h declares,
and its host-side argument validation works without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from gpawdft_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, 'include', 'gpwgrid.h')).read()
    txt = re.sub(r'/\*.*?\*/', '', txt, flags=re.S)
    return sorted(set(re.findall(r'\b(gpw_[a-z0-9_]+)\s*\(', txt)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(_lib.EXPORTS) == syms


def test_only_the_c_abi_is_exported():
    import subprocess
    out = subprocess.run(['nm', '-D', '--defined-only', _lib.LIB_PATH],
                         capture_output=True, text=True).stdout
    names = [ln.split()[-1] for ln in out.splitlines() if ' T ' in ln]
    assert names and all(n.startswith('gpw_') for n in names), names


def _op(coefs, offsets, n, mp, nb, cfd=1):
    lib = _lib.load()
    c = np.ascontiguousarray(coefs, float)
    o = np.ascontiguousarray(offsets, np.int64)
    s = np.ascontiguousarray(n, np.int64)
    b = np.ascontiguousarray(nb, np.int64)
    h = ctypes.c_void_p()
    rc = lib.gpw_operator_new(c.ctypes.data, o.ctypes.data, len(c),
                              s.ctypes.data, mp, b.ctypes.data, 1, cfd,
                              ctypes.byref(h))
    return rc, h


def test_operator_validation_and_diagonal():
    lib = _lib.load()
    # 7-point Laplacian on a 4^3 zero-boundary grid padded by 1
    M = 6
    offs = [0, 1, -1, M, -M, M * M, -M * M]
    rc, h = _op([-6.0, 1, 1, 1, 1, 1, 1], offs, (4, 4, 4), 1, [-1] * 6)
    assert rc == _lib.GPW_OK
    d = ctypes.c_double()
    assert lib.gpw_operator_get_diagonal_element(h, ctypes.byref(d)) == 0
    assert d.value == -6.0
    lib.gpw_operator_free(h)
    # mixed neighbour table (an MPI neighbour) is rejected
    rc, _ = _op([1.0], [0], (4, 4, 4), 1, [0, -1, 0, 0, 0, 0])
    assert rc == _lib.GPW_EINVAL
    assert b'neighbors' in lib.gpw_last_error()
    # an offset beyond the padding is rejected
    rc, _ = _op([1.0, 1.0], [0, 3], (4, 4, 4), 1, [-1] * 6)
    assert rc == _lib.GPW_EINVAL
    # a periodic axis shorter than the stencil range is rejected
    rc, _ = _op([1.0, 1.0], [0, 3], (2, 8, 8), 3, [0] * 6)
    assert rc == _lib.GPW_EINVAL


def test_transformer_validation():
    lib = _lib.load()

    def tr(si, so, k, pad, npad, skip, nb, interp):
        h = ctypes.c_void_p()
        arrs = [np.ascontiguousarray(x, np.int64) for x in
                (si, so, pad, npad, skip, nb)]
        return lib.gpw_transformer_new(arrs[0].ctypes.data, arrs[1].ctypes.data,
                                       k, arrs[2].ctypes.data,
                                       arrs[3].ctypes.data, arrs[4].ctypes.data,
                                       arrs[5].ctypes.data, 1, interp,
                                       ctypes.byref(h)), h
    # non-periodic restriction 15^3 -> 7^3, K=2, no padding
    rc, h = tr((15,) * 3, (7,) * 3, 2, [0] * 6, [0] * 6, [0] * 6, [-1] * 6, 0)
    assert rc == _lib.GPW_OK
    lib.gpw_transformer_free(h)
    rc, _ = tr((15,) * 3, (8,) * 3, 2, [0] * 6, [0] * 6, [0] * 6, [-1] * 6, 0)
    assert rc == _lib.GPW_EINVAL
    rc, _ = tr((15,) * 3, (7,) * 3, 3, [0] * 6, [0] * 6, [0] * 6, [-1] * 6, 0)
    assert rc == _lib.GPW_EINVAL


def test_null_and_dtype_checks():
    lib = _lib.load()
    assert lib.gpw_axpy(7, 10, 1.0, 0.0, None, None, None) == _lib.GPW_EINVAL
    assert lib.gpw_operator_apply(None, 0, None, None, 1, None, None) == \
        _lib.GPW_EINVAL
    assert lib.gpw_poisson_solve(None, None, None, 1, None, 10, 0, None, None,
                                 None) == _lib.GPW_EINVAL


def test_launch_plan_switches_validate():
    """The tuning / launch-plan switches check their arguments on the host:
    TMA variant range, Bloch and restriction layout indices, and a null
    engine."""
    lib = _lib.load()
    assert lib.gpw_set_tma_variant(-2, 0) == _lib.GPW_EINVAL
    assert lib.gpw_set_tma_variant(11, 0) == _lib.GPW_EINVAL
    assert lib.gpw_set_tma_variant(-1, 0) == _lib.GPW_OK   # back to the tuned choice
    assert lib.gpw_set_bloch_layout(-1) == _lib.GPW_EINVAL
    assert lib.gpw_set_bloch_layout(17) == _lib.GPW_EINVAL
    assert lib.gpw_set_bloch_layout(0) == _lib.GPW_OK
    assert lib.gpw_set_pdl(1) == _lib.GPW_OK
    for f in (lib.gpw_poisson_set_device_loop, lib.gpw_poisson_set_cluster,
              lib.gpw_poisson_set_fusion):
        assert f(None, 1) == _lib.GPW_EINVAL
    assert lib.gpw_bloch_launch_count() >= 0
    assert lib.gpw_set_restrict_layout(-1) == _lib.GPW_EINVAL
    assert lib.gpw_set_restrict_layout(4) == _lib.GPW_EINVAL
    assert lib.gpw_set_restrict_layout(0) == _lib.GPW_OK
    assert lib.gpw_restrict_rows_launch_count() >= 0


def test_product_fails_loudly_without_cuda():
    torch = pytest.importorskip('torch')
    if torch.cuda.is_available():
        pytest.skip('a CUDA device is present')
    from gpawdft_b200 import arrays
    with pytest.raises(RuntimeError):
        arrays.to_device(np.zeros((2, 2, 2)))
