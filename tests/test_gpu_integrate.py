"""GPU parity of GridDescriptor.integrate (gpaw/grid_descriptor.py:263-319).

``integrate(a)`` is ``sum(a) dv`` per leading index and ``integrate(a, b)`` the
matrix ``sum(conj(a_x) b_y) dv`` (the gemm with transa 'c' of :306), reduced
on the device in a fixed order.  The oracle is the NumPy restatement in
oracle/geometry.py.  Sums of N(0,1) values in a different order than NumPy's
agree to a few ulps of the sum of magnitudes, so the bar is 1e-12 of that.
"""
import numpy as np
import pytest

from helpers import rand
from oracle.geometry import GridDescriptor as OGD

pytestmark = pytest.mark.gpu


def _gds(N, pbc=0):
    from gpawdft_b200.grid_descriptor import GridDescriptor
    cell = tuple(0.2 * n for n in N)
    return GridDescriptor(N, cell, pbc), OGD(N, cell, pbc)


def _close(x, y, scale):
    x = np.asarray(x)
    y = np.asarray(y)
    assert x.shape == y.shape
    assert np.iscomplexobj(x) == np.iscomplexobj(y)
    assert np.abs(x - y).max() <= 1e-12 * scale


@pytest.mark.parametrize('dtype', [float, complex, np.float32])
def test_integrate_one_array(cuda, dtype):
    gd, ogd = _gds((24, 20, 28))
    a = rand((3, 2) + tuple(gd.n_c), dtype, 1)
    got = gd.integrate(a)
    ref = ogd.integrate(a.astype(complex if np.dtype(dtype).kind == 'c'
                                 else float))
    _close(got, ref, np.abs(a).sum() * gd.dv)
    one = gd.integrate(a[1, 0])
    assert np.isscalar(one)
    _close(one, ogd.integrate(a[1, 0].astype(np.asarray(ref).dtype)),
           np.abs(a[1, 0]).sum() * gd.dv)


@pytest.mark.parametrize('dtype', [float, complex])
def test_integrate_two_grids_is_scalar(cuda, dtype):
    """The Hartree-energy form 1/2 integrate(vHt, rhot) (gpaw/hamiltonian.py:618)."""
    gd, ogd = _gds((33, 33, 33), 1)
    a = rand(tuple(gd.n_c), dtype, 2)
    b = rand(tuple(gd.n_c), dtype, 3)
    got = gd.integrate(a, b)
    ref = ogd.integrate(a, b)
    assert np.isscalar(got)
    _close(got, ref, np.abs(a * b).sum() * gd.dv)


@pytest.mark.parametrize('dtype', [float, complex])
def test_integrate_matrix(cuda, dtype):
    """Every (x, y) pair of leading indices; complex results keep the imaginary part."""
    gd, ogd = _gds((16, 18, 20), 1)
    a = rand((2, 3) + tuple(gd.n_c), dtype, 4)
    b = rand((4,) + tuple(gd.n_c), dtype, 5)
    got = gd.integrate(a, b)
    ref = ogd.integrate(a, b)
    assert got.shape == (2, 3, 4)
    _close(got, ref, np.abs(a).max() * np.abs(b).max() * a[0, 0].size * gd.dv)


def test_integrate_same_array(cuda):
    """``a is b``: the reference's rank-k update fills one triangle; the full
    Hermitian matrix here agrees with it there."""
    gd, ogd = _gds((16, 16, 16), 1)
    a = rand((5,) + tuple(gd.n_c), complex, 6)
    got = gd.integrate(a, a)
    ref = ogd.integrate(a, a)
    _close(got, ref, np.abs(a).max() ** 2 * a[0].size * gd.dv)
    assert np.allclose(got, got.conj().T, rtol=0, atol=1e-12 * np.abs(got).max())


def test_integrate_device_tensor_hartree(cuda):
    """Device tensors stay on the device; E_H of a solved potential."""
    import torch
    from gpawdft_b200.poisson import PoissonSolver
    from gpawdft_b200.workloads import gaussian_density
    rho, L = gaussian_density(48, 0.2, 8, 1)
    from gpawdft_b200.grid_descriptor import GridDescriptor
    gd = GridDescriptor((48,) * 3, (L,) * 3, 0)
    ogd = OGD((48,) * 3, (L,) * 3, 0)
    ps = PoissonSolver(nn=3)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    phi = gd.zeros()
    ps.solve(phi, rho)
    e_dev = 0.5 * gd.integrate(torch.from_numpy(phi).cuda(),
                               torch.from_numpy(rho).cuda())
    e_ref = 0.5 * ogd.integrate(phi, rho)
    assert abs(e_dev - e_ref) < 1e-12 * abs(e_ref) + 1e-14


def test_integrate_rejects_mismatch(cuda):
    gd, _ = _gds((16, 16, 16))
    a = rand(tuple(gd.n_c), float, 7)
    with pytest.raises(TypeError):
        gd.integrate(a, a.astype(complex))
