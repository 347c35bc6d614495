"""GPU parity of the Poisson solver variants.

* The weighted operator of the dielectric solver (gpaw/wfd_operators.py,
  c/woperators.c, c/bmgs/wfd.c, wrelax.c): apply, Jacobi and Gauss-Seidel
  bit-identical to the reference's own WOperator (oracle/_ref; the NumPy
  restatement, itself pinned bit-identically to it in
  tests/test_oracle_variants.py, where that is not built).
* WeightedFDPoissonSolver (gpaw/solvation/poisson.py:62-150): the known
  answers of the reference's gpaw/test/solvation/poisson.py (Gaussian
  charges in a constant or Gaussian-shaped permittivity, neutral and
  charged: potential within 1e-3 of the analytic one) and the oracle solve
  (same V-cycle count, potential within 1e-9).
* HelmholtzSolver (gpaw/helmholtz.py): the known answer of
  gpaw/test/poisson/screened_poisson.py (residual against the analytic
  screened potential below 0.003) and the oracle solve.
* DipoleCorrection (gpaw/dipole_correction.py): a slab with a dipole, against
  the oracle's correction and potential.
"""
from types import SimpleNamespace

import numpy as np
import pytest

from helpers import rand
from oracle import layer as ol
from oracle import ref as oref
from oracle import variants as ov
from oracle.geometry import GridDescriptor as OGD, phase_cd_for_k

pytestmark = pytest.mark.gpu

BACKEND = 'ref' if oref.available() else 'numpy'
BOHR = 0.52917721


# ------------------------------------------------------------ weighted op
def _wops(N, cell, pbc, nn, seed, dtype=float):
    from gpawdft_b200.fd_operators import Gradient, Laplace
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.wfd_operators import WeightedFDOperator
    gd = GridDescriptor(N, cell, pbc)
    ogd = OGD(N, cell, pbc)
    rng = np.random.default_rng(seed)
    W = [1.0 + rng.random(tuple(gd.n_c))] + \
        [rng.standard_normal(tuple(gd.n_c)) for _ in range(3)]
    s = -0.25 / np.pi
    op = WeightedFDOperator(W, [Laplace(gd, s, nn, dtype)] +
                            [Gradient(gd, j, s, nn, dtype) for j in range(3)])
    oop = ov.WeightedFDOperator(
        W, [ol.Laplace(ogd, s, nn, dtype, backend=BACKEND)] +
        [ol.Gradient(ogd, j, s, nn, dtype, backend=BACKEND)
         for j in range(3)], BACKEND)
    return gd, ogd, op, oop


@pytest.mark.parametrize('pbc', [0, 1])
@pytest.mark.parametrize('nn', [1, 2, 3])
def test_weighted_apply_and_jacobi_bit_identical(cuda, pbc, nn):
    gd, ogd, op, oop = _wops((20, 18, 22), (4.0, 3.6, 4.4), pbc, nn, nn)
    a = rand(tuple(gd.n_c), float, 1)
    out, oout = np.empty_like(a), np.empty_like(a)
    op.apply(a, out)
    oop.apply(a, oout)
    assert np.array_equal(out, oout)
    s = rand(tuple(gd.n_c), float, 2)
    f, of = a.copy(), a.copy()
    op.relax(2, f, s, 3, 2.0 / 3.0)
    oop.relax(2, of, s, 3, 2.0 / 3.0)
    assert np.array_equal(f, of)
    assert op.get_diagonal_element() == oop.get_diagonal_element()


@pytest.mark.skipif(not oref.available(), reason='needs oracle/_ref')
@pytest.mark.parametrize('pbc', [0, 1])
def test_weighted_gauss_seidel_bit_identical(cuda, pbc):
    gd, ogd, op, oop = _wops((12, 10, 14), (2.4, 2.0, 2.8), pbc, 2, 5)
    a = rand(tuple(gd.n_c), float, 3)
    s = rand(tuple(gd.n_c), float, 4)
    f, of = a.copy(), a.copy()
    op.relax(1, f, s, 2)
    oop.relax(1, of, s, 2)
    assert np.array_equal(f, of)


@pytest.mark.skipif(not oref.available(), reason='needs oracle/_ref')
def test_weighted_complex_bloch_apply(cuda):
    gd, ogd, op, oop = _wops((16, 16, 16), (3.2,) * 3, 1, 2, 6, complex)
    a = rand((2,) + tuple(gd.n_c), complex, 7)
    ph = phase_cd_for_k(ogd, (0.2, -0.1, 0.3))
    out = np.empty_like(a)
    op.apply(a, out, ph)
    for i in range(2):
        o1 = np.empty_like(a[i])
        oop.apply(a[i].copy(), o1, ph)
        assert np.array_equal(out[i], o1)


# ------------------------------------------------------------ dielectric
BOX = 12.0


def _dielectric_case(kind):
    """gpaw/test/solvation/poisson.py: grid h = 0.4 A in a 12 A box (60^3,
    zero boundary), nn=3."""
    from oracle.gauss import Gaussian as OGauss
    N = int(BOX / 0.4 * 2)
    cell = np.diag([BOX / BOHR] * 3)
    ogd = OGD((N,) * 3, cell, 0)
    epsinf = 80.
    centre = lambda s: (BOX / 2. + s) * np.ones(3) / BOHR  # noqa: E731
    rho = ogd.zeros()
    phi_expected = ogd.zeros()
    if kind in ('neutral-const', 'charged-const'):
        eps = ogd.zeros() + epsinf
        qs, shifts = ((-1., 1.), (-1., 1.)) if kind == 'neutral-const' \
            else ((-2.,), (1.,))
        for q, shift in zip(qs, shifts):
            g = OGauss(ogd, center=centre(shift))
            rho += q / np.sqrt(4 * np.pi) * g.get_gauss(0)
            phi_expected += q / np.sqrt(4 * np.pi) * g.get_gauss_pot(0) \
                / epsinf
        grad = [ogd.zeros() for _ in range(3)]
    else:
        qs, shifts, epsshift = ((-1., 1.), (-.4, .4), 0.) \
            if kind == 'neutral-var' else ((2.,), (-1.,), -1.)
        g = OGauss(ogd, center=centre(epsshift))
        e = g.get_gauss(0)
        eps = epsinf - e / e.max() * (epsinf - 1.)
        grad = []
        for i in range(3):
            out = ogd.empty()
            ol.Gradient(ogd, i, 1.0, 3, backend=BACKEND).apply(
                eps - epsinf, out)
            grad.append(out)
        for q, shift in zip(qs, shifts):
            g = OGauss(ogd, center=centre(shift))
            phi_tmp = g.get_gauss_pot(0)
            fac = 2. * np.sqrt(g.a) * np.exp(-g.a * g.r2)
            fac /= np.sqrt(np.pi) * g.r2
            from scipy.special import erf
            fac -= erf(np.sqrt(g.a) * g.r) / (g.r2 * g.r)
            fac *= 2.0 * 1.7724538509055159
            grad_phi = fac * g.xyz
            laplace_phi = -4. * np.pi * g.get_gauss(0)
            rho_tmp = -1. / (4. * np.pi) * (
                (np.array(grad) * grad_phi).sum(0) + eps * laplace_phi)
            norm = ogd.integrate(rho_tmp)
            rho_tmp /= norm * q
            phi_tmp /= norm * q
            rho += rho_tmp
            phi_expected += phi_tmp
    return N, cell, ogd, [eps] + grad, rho, phi_expected


@pytest.mark.parametrize('kind', ['neutral-const', 'charged-const',
                                  'neutral-var', 'charged-var'])
def test_weighted_poisson_known_answers(cuda, kind):
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.solvation import WeightedFDPoissonSolver
    N, cell, ogd, eg, rho, phi_expected = _dielectric_case(kind)
    gd = GridDescriptor((N,) * 3, cell, 0)
    ps = WeightedFDPoissonSolver(nn=3, relax='J', eps=2e-10)
    ps.set_dielectric(SimpleNamespace(eps_gradeps=[a.copy() for a in eg]))
    ps.set_grid_descriptor(gd)
    ps.initialize()
    phi = gd.zeros()
    n = ps.solve(phi, rho)
    err = np.abs(phi - phi_expected).max()
    print('%s: %d V-cycles, max |phi - analytic| %.2e' % (kind, n, err))
    assert err < 1e-3
    if kind in ('neutral-const', 'charged-var'):
        ops = ov.WeightedFDPoissonSolver(nn=3, relax='J', eps=2e-10,
                                         backend=BACKEND)
        ops.set_dielectric(SimpleNamespace(eps_gradeps=[a.copy()
                                                        for a in eg]))
        ops.set_grid_descriptor(ogd)
        ops.initialize()
        ophi = ogd.zeros()
        on = ops.solve(ophi, rho)
        assert n == on
        assert np.abs(phi - ophi).max() < 1e-9 * np.abs(ophi).max()


# ------------------------------------------------------------ Helmholtz
def test_screened_poisson_known_answer(cuda):
    """gpaw/test/poisson/screened_poisson.py: a Gaussian's screened potential
    (k2 = -0.4, 48^3 in a 20 Bohr box, nn=3, Gauss-Seidel)."""
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.helmholtz import HelmholtzSolver
    from oracle.gauss import Gaussian as OGauss
    a, N, k2 = 20, 48, -0.4
    gd = GridDescriptor((N,) * 3, (a,) * 3, 0)
    ogd = OGD((N,) * 3, (a,) * 3, 0)
    ps = HelmholtzSolver(k2=k2, nn=3)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    ng = OGauss(ogd, a=31).get_gauss(0)
    vg = ov.ScreenedPoissonGaussian(ogd, a=31).get_phi(-k2)
    pot = gd.zeros()
    n = ps.solve(pot, ng, charge=None, zero_initial_phi=True)
    residual = np.sqrt(((pot - vg) ** 2).sum() * ogd.dv)
    assert residual < 0.003, residual
    ops = ov.HelmholtzSolver(k2=k2, nn=3, backend=BACKEND)
    ops.set_grid_descriptor(ogd)
    ops.initialize()
    opot = ogd.zeros()
    on = ops.solve(opot, ng, charge=None, zero_initial_phi=True)
    assert n == on
    assert np.abs(pot - opot).max() < 1e-9 * np.abs(opot).max()


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_helmholtz_jacobi_neutral(cuda, precision):
    """Jacobi smoothing through the device-loop engine (and its float32
    defect-correction form) against the oracle's solve."""
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.helmholtz import HelmholtzSolver
    from gpawdft_b200.workloads import gaussian_density
    rho, L = gaussian_density(40, 0.25, 6, 31)
    gd = GridDescriptor((40,) * 3, (L,) * 3, 0)
    ogd = OGD((40,) * 3, (L,) * 3, 0)
    ps = HelmholtzSolver(k2=-0.3, nn=3, relax='J', eps=1e-14,
                         precision=precision)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    phi = gd.zeros()
    n = ps.solve(phi, rho)
    ops = ov.HelmholtzSolver(k2=-0.3, nn=3, relax='J', eps=1e-14,
                             backend=BACKEND)
    ops.set_grid_descriptor(ogd)
    ops.initialize()
    ophi = ogd.zeros()
    on = ops.solve(ophi, rho)
    assert ps.last_errors[0] <= 1e-14
    if precision == 'fp64':
        assert n == on
        assert np.abs(phi - ophi).max() < 1e-7 * np.abs(ophi).max()
    else:   # another iterate at the same residual
        assert np.abs(phi - ophi).max() < 1e-6 * np.abs(ophi).max()


# ------------------------------------------------------------ dipole layer
def test_dipole_correction_slab(cuda):
    """A neutral slab with a dipole along z, periodic in x and y: the
    corrected potential and the correction follow the oracle's."""
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import FDPoissonSolver, PoissonSolver
    from oracle.gauss import Gaussian as OGauss
    N = (24, 24, 64)
    cell = (6.0, 6.0, 16.0)
    pbc = (1, 1, 0)
    gd = GridDescriptor(N, cell, pbc)
    ogd = OGD(N, cell, pbc)
    rho = ogd.zeros()
    for q, z in ((1.0, 7.0), (-1.0, 9.5)):
        rho += q * OGauss(ogd, a=8.0, center=np.array([3.0, 3.0, z])
                          ).get_gauss(0)
    rho -= rho.mean()
    ps = PoissonSolver(dipolelayer='xy', nn=3, relax='J', eps=1e-14)
    assert not isinstance(ps, FDPoissonSolver)
    ps.set_grid_descriptor(gd)
    assert ps.c == 2
    ps.initialize()
    phi = gd.zeros()
    n = ps.solve(phi, rho)
    ops = ov.DipoleCorrection(ol.PoissonSolver(nn=3, relax='J', eps=1e-14,
                                               backend=BACKEND), 2)
    ops.set_grid_descriptor(ogd)
    ops.initialize()
    ophi = ogd.zeros()
    on = ops.solve(ophi, rho)
    assert abs(n - on) <= 1
    assert abs(ps.correction - ops.correction) < 1e-10 * abs(ops.correction)
    assert np.abs(phi - ophi).max() < 1e-7 * np.abs(ophi).max()
    # the correction flattens the potential far from the slab on both sides
    assert abs(ps.correction) > 1e-3


# ------------------------------------------------------------ extended grid
def test_extended_solver_golden_values(cuda):
    """gpaw/test/poisson/poisson_extended.py on the GPU: every option's
    max |phi - phi_default| equals the reference's own value to 1e-10, and
    each potential follows the oracle's; useprev restarts from the last
    extended potential."""
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    from gpawdft_b200.poisson_extended import ExtendedPoissonSolver
    from test_oracle_variants import EXT_GOLDEN, extended_case
    ogd, rho = extended_case()
    gd = GridDescriptor((16, 16, 48), (1, 1, 3), False)

    def run(ps, g):
        ps.set_grid_descriptor(g)
        ps.initialize()
        phi = g.zeros()
        n = ps.solve(phi, rho)
        return phi, n, ps

    ref, _, _ = run(PoissonSolver(eps=1e-20), gd)
    oref_phi, _, _ = run(ol.PoissonSolver(eps=1e-20, backend=BACKEND), ogd)
    assert np.abs(ref - oref_phi).max() < 1e-9 * np.abs(oref_phi).max()
    for kw, val in EXT_GOLDEN:
        phi, n, ps = run(ExtendedPoissonSolver(eps=1e-20, **kw), gd)
        assert abs(np.abs(phi - ref).max() - val) < 1e-10, kw
        ophi, on, _ = run(ov.ExtendedPoissonSolver(eps=1e-20, backend=BACKEND,
                                                   **kw), ogd)
        assert n == on, kw
        assert np.abs(phi - ophi).max() < 1e-9 * np.abs(ophi).max(), kw
    # useprev: the second solve starts from the first's extended potential
    kw = dict(extended={'gpts': (24, 24, 72), 'useprev': True},
              moment_corrections=[{'moms': range(4), 'center': [.5, .5, 1]},
                                  {'moms': range(4), 'center': [.5, .5, 2]}])
    phi1, n1, ps = run(ExtendedPoissonSolver(eps=1e-20, **kw), gd)
    phi2 = gd.zeros()
    n2 = ps.solve(phi2, rho)
    assert n2 < n1
    assert np.abs(phi2 - phi1).max() < 1e-8 * np.abs(phi1).max()
