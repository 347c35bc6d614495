"""Known-answer checks of the reference's own hot-path tests.

Restated from gpaw/test/fd_ops/laplace.py, fd_ops/gradient.py,
fd_ops/transformations.py, fd_ops/non_periodic.py, poisson/poisson.py and
poisson/poisson_asym.py with their tolerances, and run twice: on the oracle
(CPU, NumPy restatement) and on the GPU product (marked gpu).
"""
from math import cos, pi, sin

import numpy as np
import pytest


class OracleAPI:
    def __init__(self):
        from oracle import layer
        from oracle.geometry import GridDescriptor
        self.GD = GridDescriptor
        self.Laplace = lambda gd, scale=1.0, n=1, dtype=float: layer.Laplace(
            gd, scale, n, dtype)
        self.Gradient = lambda gd, v, scale=1.0, n=1, dtype=float: \
            layer.Gradient(gd, v, scale, n, dtype)
        self.Transformer = lambda gi, go, nn=1, dtype=float: \
            layer.Transformer(gi, go, nn, dtype)
        self.PoissonSolver = layer.PoissonSolver
        from oracle.gauss import Gaussian
        self.Gaussian = Gaussian

    def integrate(self, gd, a):
        return float(np.real(gd.integrate(a)))


class GpuAPI:
    def __init__(self):
        from gpawdft_b200 import fd_operators, poisson, transformers
        from gpawdft_b200.gauss import Gaussian
        from gpawdft_b200.grid_descriptor import GridDescriptor
        self.GD = GridDescriptor
        self.Laplace = fd_operators.Laplace
        self.Gradient = fd_operators.Gradient
        self.Transformer = transformers.Transformer
        self.PoissonSolver = poisson.PoissonSolver
        self.Gaussian = Gaussian

    def integrate(self, gd, a):
        # integrate on the host copy: the check is about the transformer
        x = a.reshape(a.shape[:-3] + (-1,)).sum(axis=-1) * gd.dv
        return complex(x).real if np.iscomplexobj(x) else float(x)


API = [pytest.param('oracle', id='oracle'),
       pytest.param('gpu', id='gpu', marks=pytest.mark.gpu)]


def api(kind):
    return OracleAPI() if kind == 'oracle' else GpuAPI()


CELLS = [
    ('distorted hexagonal', 4,
     [(1, 0, 0), (1.02 * cos(pi / 3 - 0.02), 1.02 * sin(pi / 3 - 0.02), 0),
      (0, 0, 1.0)]),
    ('hexagonal', 4, [(1, 0, 0), (0.5, 3 ** 0.5 / 2, 0), (0, 0, 1.1)]),
    ('fcc', 6, [(0, 1, 1), (1, 0, 1), (1, 1, 0)]),
    ('fcc-alternative', 6, [(1, 0, 0), (0.5, 3 ** 0.5 / 2, 0),
                            (0.5, 3 ** 0.5 / 6, (2 / 3) ** 0.5)]),
    ('bcc', 4, [(-1, 1, 1), (1, -1, 1), (1, 1, -1)]),
    ('sc', 3, [1.1, 1.02, 1.03]),
    ('distorted sc', 6, [(1, 0, 0), (0.01, 1, 0), (0, 0.02, 1)]),
    ('rocksalt', 6, [(2 * np.sqrt(1 / 3), np.sqrt(1 / 8), -np.sqrt(1 / 24)),
                     (2 * np.sqrt(1 / 3), -np.sqrt(1 / 8), -np.sqrt(1 / 24)),
                     (2 * np.sqrt(1 / 3), 0, np.sqrt(1 / 6))]),
    ('nasty', 6, [(1, 0, 0), (0.0001, 1.03, 0), (0.0001, 0.0001, 1.0)]),
    ('Mike', 6, 5 * np.array([(5.565 / 28, 0, 0), (0.0001 / 28, 5.565 / 28, 0),
                              (0.0001 / 24, 0.0001 / 24, 4.684 / 24)])),
    ('MnO', 6, [(1, 0.5, 0.5), (0.5, 1, 0.5), (0.5, 0.5, 1)]),
]


@pytest.mark.parametrize('kind', API)
@pytest.mark.parametrize('name,D,cell', CELLS, ids=[c[0] for c in CELLS])
def test_laplace_gradient_polynomials(kind, name, D, cell):
    """fd_ops/laplace.py: exact on polynomials of degree <= 2n at the centre
    point (2e-12 Laplacian, 4e-12 gradient); D directions chosen."""
    A = api(kind)
    for n in range(1, 6):
        N = 2 * n + 2
        gd = A.GD((N, N, N), cell)
        b_g = gd.zeros()
        r_gv = gd.get_grid_point_coordinates().transpose((1, 2, 3, 0))
        c_v = gd.cell_cv.sum(0) / 2
        r_gv -= c_v
        lap = A.Laplace(gd, n=n)
        grad_v = [A.Gradient(gd, v, n=n) for v in range(3)]
        assert lap.npoints == D * 2 * n + 1
        for m in range(0, 2 * n + 1):
            for ix in range(m + 1):
                for iy in range(m - ix + 1):
                    iz = m - ix - iy
                    a_g = (r_gv ** (ix, iy, iz)).prod(3)
                    r = 2.0 if (m == 2 and max(ix, iy, iz) == 2) else 0.0
                    lap.apply(a_g, b_g)
                    assert abs(b_g[n + 1, n + 1, n + 1] - r) < 2e-12
                    for v in range(3):
                        grad_v[v].apply(a_g, b_g)
                        r = 1 if (m == 1 and [ix, iy, iz][v] == 1) else 0
                        assert abs(b_g[n + 1, n + 1, n + 1] - r) < 4e-12


@pytest.mark.parametrize('kind', API)
def test_gradient_exact_values(kind):
    """fd_ops/gradient.py."""
    A = api(kind)
    gd = A.GD((8, 1, 1), (8.0, 1.0, 1.0))
    a = gd.zeros()
    dadx = gd.zeros()
    a[:, 0, 0] = np.arange(gd.beg_c[0], gd.end_c[0])
    A.Gradient(gd, v=0).apply(a, dadx)
    assert dadx[3, 0, 0] == 1.0 and np.sum(dadx[:, 0, 0]) == 0.0
    gd = A.GD((1, 8, 1), (1.0, 8.0, 1.0), (1, 0, 1))
    dady = gd.zeros()
    a = gd.zeros()
    a[0, :, 0] = np.arange(gd.beg_c[1], gd.end_c[1]) - 1
    A.Gradient(gd, v=1).apply(a, dady)
    assert dady[0, 0, 0] == 0.5 and np.sum(dady[0, :, 0]) == 3.0
    gd = A.GD((1, 7, 1), ((1.0, 0.0, 0.0), (5.0, 5.0, 0.0), (0.0, 0.0, 0.7)))
    dady = gd.zeros()
    a = gd.zeros()
    a[0, :, 0] = np.arange(gd.beg_c[1], gd.end_c[1]) - 1
    A.Gradient(gd, v=1).apply(a, dady)
    assert dady[0, 0, 0] == -3.5 and abs(np.sum(dady[0, :, 0])) < 1e-12


@pytest.mark.parametrize('kind', API)
def test_transformations_conserve_integral(kind):
    """fd_ops/transformations.py: K=2,4,6,8 conserve the integral (1e-14)."""
    A = api(kind)
    n = 20
    gd = A.GD((n, n, n))
    rng = np.random.RandomState(8)
    a = gd.empty()
    a[:] = rng.random_sample(a.shape)
    ac = gd.empty(dtype=complex)
    ac.real = rng.random_sample(a.shape)
    ac.imag = rng.random_sample(a.shape)
    phase = np.ones((3, 2), complex)
    for gd2 in (gd.refine(), gd.coarsen()):
        for k in [2, 4, 6, 8]:
            b = gd2.zeros()
            A.Transformer(gd, gd2, k // 2).apply(a, b)
            assert abs(A.integrate(gd, a) - A.integrate(gd2, b)) < 1e-14
            bc = gd2.zeros(dtype=complex)
            A.Transformer(gd, gd2, k // 2, complex).apply(ac, bc, phase)
            ia = ac.reshape(-1).sum() * gd.dv
            ib = bc.reshape(-1).sum() * gd2.dv
            assert abs(ia - ib) < 1e-14


@pytest.mark.parametrize('kind', API)
def test_non_periodic_transformations(kind):
    """fd_ops/non_periodic.py (1e-10)."""
    A = api(kind)
    n = 20
    gd1 = A.GD((n, n, n), (8.0, 8.0, 8.0), pbc_c=0)
    a1 = gd1.zeros()
    rng = np.random.RandomState(8)
    a1[:] = rng.random_sample(a1.shape)
    gd2 = gd1.refine()
    a2 = gd2.zeros()
    A.Transformer(gd1, gd2).apply(a1, a2)
    assert abs(A.integrate(gd1, a1) - A.integrate(gd2, a2)) < 1e-10
    a2[0] = 0.0
    a2[:, 0] = 0.0
    a2[:, :, 0] = 0.0
    a2[-1] = 0.0
    a2[:, -1] = 0.0
    a2[:, :, -1] = 0.0
    A.Transformer(gd2, gd1).apply(a2, a1)
    assert abs(A.integrate(gd1, a1) - A.integrate(gd2, a2)) < 1e-10


@pytest.mark.parametrize('kind', API)
def test_poisson_symmetry(kind):
    """poisson/poisson.py: two equal charges at (0,0,0) and (1/2,1/2,1/2) of a
    periodic 16^3 cell give equal potentials there (Jacobi nn=1: 6e-16).  The
    reference's spline charge (LFC + Spline, not on this path) is replaced by
    a smooth radial bump of the same support."""
    A = api(kind)
    L = 2.87 / 0.529177
    N = 16
    gd = A.GD((N, N, N), (L, L, L))
    cut = N / 2.0 * 0.9 * L / N
    r_vg = gd.get_grid_point_coordinates()
    a = gd.zeros()
    for c in (np.zeros(3), np.ones(3) * L / 2):
        d = r_vg - c[:, None, None, None]
        d -= L * np.round(d / L)
        r = np.sqrt((d ** 2).sum(0))
        a += np.where(r < cut, (1 - (r / cut) ** 2) ** 2, 0.0)
    a -= a.sum() * gd.dv / L ** 3
    p = A.PoissonSolver(nn=1, relax='J')
    p.set_grid_descriptor(gd)
    p.initialize()
    b = gd.zeros()
    p.solve(b, a, charge=0)
    # the reference's 6e-16 is absolute for its charge; here relative to |phi|
    assert abs(b[0, 0, 0] - b[8, 8, 8]) < 6e-16 * max(1.0, abs(b[0, 0, 0]))


@pytest.mark.parametrize('kind', API)
def test_poisson_asym(kind):
    """poisson/poisson_asym.py: charged off-centre Gaussian, non-periodic 48^3,
    use_charge_center: |phi - analytic| < 1e-5."""
    A = api(kind)
    a = 20.0
    N = 48
    center = (a / 2, a / 2, 3 * a / 4)
    gd = A.GD((N, N, N), (a, a, a), 0)
    solver = A.PoissonSolver(nn=3, use_charge_center=True)
    solver.set_grid_descriptor(gd)
    solver.initialize()
    gauss = A.Gaussian(gd, a=19, center=center)
    pot = gd.zeros()
    ng = gauss.get_gauss(0)
    vg = gauss.get_gauss_pot(0)
    solver.solve(pot, ng, charge=1.0, zero_initial_phi=False)
    residual = (((pot - vg) ** 2).sum() * gd.dv) ** 0.5
    assert residual < 1e-5
