"""GPU parity of the eigensolver preconditioner (gpaw/preconditioner.py:10-60).

The device Preconditioner runs the three-grid smoothing sequence of
gpaw/preconditioner.py:34-60 (restrictions and interpolations with the
k-point's Bloch phases, the caller's kinetic operator ``kin0`` on the fine grid,
nn=1 Laplacians on the two coarse grids, axpy / scal glue).  The oracle is the
restated Preconditioner (oracle/layer.py) over the compiled reference C
(``backend='ref'``) where it is built, else over the NumPy restatement of the
same C kernels (bit-identical to it, tests/test_oracle_golden.py).  The star
stencils fuse multiply-adds, so the bar is 1e-12 relative.
"""
import numpy as np
import pytest

from helpers import relerr, rand
from oracle import layer as ol
from oracle import ref as oref
from oracle.geometry import GridDescriptor as OGD, phase_cd_for_k

pytestmark = pytest.mark.gpu

BACKEND = 'ref' if oref.available() else 'numpy'


class _Kpt:
    def __init__(self, phase_cd):
        self.phase_cd = phase_cd


def _pair(N, cell, pbc, dtype, block, nn_kin=3):
    from gpawdft_b200.fd_operators import Laplace
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.preconditioner import Preconditioner
    gd = GridDescriptor(N, cell, pbc)
    ogd = OGD(N, cell, pbc)
    pc = Preconditioner(gd, Laplace(gd, -0.5, nn_kin, dtype), dtype, block)
    opc = ol.Preconditioner(ogd, ol.Laplace(ogd, -0.5, nn_kin, dtype,
                                            BACKEND), dtype, block, BACKEND)
    return gd, ogd, pc, opc


@pytest.mark.parametrize('nb', [8, 3])
def test_bloch_complex128_bands(cuda, nb):
    """A block of complex128 Bloch bands, 48^3 periodic, nn=3 kinetic, random k."""
    N = (48, 48, 48)
    gd, ogd, pc, opc = _pair(N, (48 * 0.34,) * 3, 1, complex, 8)
    rng = np.random.default_rng(11)
    ph = phase_cd_for_k(ogd, rng.uniform(-0.5, 0.5, 3))
    res = rand((nb,) + tuple(gd.n_c), complex, 12)
    out = pc(res, _Kpt(ph))
    ref = opc(res.copy(), ph)
    assert out.shape == ref.shape
    assert relerr(out, ref) < 1e-12


def test_bloch_noncubic_cell(cuda):
    """Unequal axes and spacings: each axis keeps its own phase and h."""
    N = (32, 40, 24)
    gd, ogd, pc, opc = _pair(N, (6.0, 8.4, 5.1), 1, complex, 4)
    ph = phase_cd_for_k(ogd, (0.31, -0.17, 0.42))
    res = rand((4,) + tuple(gd.n_c), complex, 13)
    out = pc(res, _Kpt(ph))
    ref = opc(res.copy(), ph)
    assert relerr(out, ref) < 1e-12


def test_float64_zero_boundary(cuda):
    """Real residuals on a zero-boundary grid (no phases)."""
    N = (40, 40, 40)
    gd, ogd, pc, opc = _pair(N, (40 * 0.2,) * 3, 0, float, 5)
    res = rand((5,) + tuple(gd.n_c), float, 14)
    out = pc(res, _Kpt(None))
    ref = opc(res.copy(), None)
    assert relerr(out, ref) < 1e-12


def test_float64_periodic_gamma(cuda):
    """Real residuals on a periodic grid at the Gamma point."""
    N = (32, 32, 32)
    gd, ogd, pc, opc = _pair(N, (32 * 0.2,) * 3, 1, float, 2, nn_kin=2)
    res = rand((2,) + tuple(gd.n_c), float, 15)
    out = pc(res, _Kpt(None))
    ref = opc(res.copy(), None)
    assert relerr(out, ref) < 1e-12


def test_device_tensors_and_block_reuse(cuda):
    """Device residuals in, a device view of scratch out; repeated calls
    reuse the scratch (the reference's contract) and give the same result."""
    import torch
    N = (32, 32, 32)
    gd, ogd, pc, opc = _pair(N, (32 * 0.3,) * 3, 1, complex, 4)
    ph = phase_cd_for_k(ogd, (0.1, 0.2, -0.3))
    res = rand((4,) + tuple(gd.n_c), complex, 16)
    res_d = torch.from_numpy(res).to('cuda')
    out1 = pc(res_d, _Kpt(ph)).cpu().numpy()
    res2 = rand((4,) + tuple(gd.n_c), complex, 17)
    out2 = pc(torch.from_numpy(res2).to('cuda'), _Kpt(ph)).cpu().numpy()
    assert relerr(out1, opc(res.copy(), ph)) < 1e-12
    assert relerr(out2, opc(res2.copy(), ph)) < 1e-12
    with pytest.raises(ValueError):
        pc(rand((5,) + tuple(gd.n_c), complex, 18), _Kpt(ph))
