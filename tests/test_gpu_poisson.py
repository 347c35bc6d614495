"""GPU parity of the multigrid Poisson solver (gpaw/poisson.py path).

The plain float64 method must reproduce the oracle's V-cycle count, its
potential to the solver tolerance and the Hartree energy E_H = 1/2 dv
sum(phi rho) to 1e-8 Ha.  Also: charged periodic / zero-boundary branches,
Gauss-Seidel, batched solves (each equal to its single solve) and the
float32 defect-correction form (its error vs the float64 result stated).
"""
import numpy as np
import pytest

from gpawdft_b200.workloads import gaussian_density
from oracle import layer as ol
from oracle.geometry import GridDescriptor as OGD

pytestmark = pytest.mark.gpu


def solvers(N, L, pbc, **kw):
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    gd = GridDescriptor((N,) * 3, (L,) * 3, pbc)
    ogd = OGD((N,) * 3, (L,) * 3, pbc)
    ps = PoissonSolver(**kw)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    ops = ol.PoissonSolver(**{k: v for k, v in kw.items() if k != 'batch'})
    ops.set_grid_descriptor(ogd)
    ops.initialize()
    return gd, ogd, ps, ops


def hartree(gd, phi, rho):
    return 0.5 * gd.dv * float(np.dot(phi.ravel(), rho.ravel()))


@pytest.mark.parametrize('N', [32, 64])
def test_neutral_zero_boundary(cuda, N):
    """Benchmark config (b) recipe: 8 neutral Gaussians, nn=3, Jacobi."""
    rho, L = gaussian_density(N, 0.2, 8, 1)
    gd, ogd, ps, ops = solvers(N, L, 0, nn=3, relax='J', eps=2e-10)
    phi = gd.zeros()
    n = ps.solve(phi, rho)
    ophi = ogd.zeros()
    on = ops.solve(ophi, rho)
    assert n == on
    # both stop at sum(r^2) dv <= eps: compare potentials at that accuracy
    assert np.abs(phi - ophi).max() < 1e-6 * np.abs(ophi).max()
    assert abs(hartree(ogd, phi, rho) - hartree(ogd, ophi, rho)) < 1e-8
    assert np.allclose(ps.last_errors, ops.errors[-1], rtol=1e-6)


def test_tight_tolerance_trajectory(cuda):
    """To relative residual 1e-10: every V-cycle's error follows the oracle."""
    N = 32
    rho, L = gaussian_density(N, 0.2, 8, 3)
    gd, ogd, ps, ops = solvers(N, L, 0, nn=3, relax='J', maxiter=200)
    eps = 1e-20 * float(np.dot(rho.ravel(), rho.ravel())) * gd.dv
    phi = gd.zeros()
    n = ps.solve(phi, rho, eps=eps)
    ophi = ogd.zeros()
    on = ops.solve(ophi, rho, eps=eps)
    assert n == on
    assert np.abs(phi - ophi).max() < 1e-12 * np.abs(ophi).max() + 1e-14
    assert abs(hartree(ogd, phi, rho) - hartree(ogd, ophi, rho)) < 1e-8


def test_charged_periodic(cuda):
    N = 32
    rho, L = gaussian_density(N, 0.25, 4, 7, pbc=True)
    rho += 0.01  # net charge -> homogeneous background branch
    gd, ogd, ps, ops = solvers(N, L, 1, nn=2, relax='J', eps=1e-14)
    phi = gd.zeros()
    n = ps.solve(phi, rho)
    ophi = ogd.zeros()
    on = ops.solve(ophi, rho)
    assert abs(n - on) <= 1
    assert np.abs(phi - ophi).max() < 1e-7 * np.abs(ophi).max()
    assert abs(phi.mean()) < 1e-12


@pytest.mark.parametrize('center', [False, True])
def test_charged_zero_boundary(cuda, center):
    """Gaussian-compensation branch (gpaw/poisson.py:249-299)."""
    N = 48
    a = 20.0
    from oracle.gauss import Gaussian as OGauss
    ogd0 = OGD((N,) * 3, (a,) * 3, 0)
    rho = OGauss(ogd0, a=19, center=(a / 2, a / 2, 3 * a / 4)).get_gauss(0)
    gd, ogd, ps, ops = solvers(N, a, 0, nn=3, use_charge_center=center)
    for charge in (1.0, None):
        phi = gd.zeros()
        n = ps.solve(phi, rho, charge=charge)
        ophi = ogd.zeros()
        on = ops.solve(ophi, rho, charge=charge)
        assert n == on
        assert np.abs(phi - ophi).max() < 1e-6 * np.abs(ophi).max()


def test_gauss_seidel_solver(cuda):
    N = 16
    rho, L = gaussian_density(N, 0.3, 4, 9)
    gd, ogd, ps, ops = solvers(N, L, 0, nn=1, relax='GS', eps=1e-12)
    phi = gd.zeros()
    n = ps.solve(phi, rho)
    ophi = ogd.zeros()
    on = ops.solve(ophi, rho)
    assert n == on
    assert np.abs(phi - ophi).max() <= 1e-13 * np.abs(ophi).max()


def test_batch_equals_single(cuda):
    N = 32
    rhos = []
    for s in range(3):
        rho, L = gaussian_density(N, 0.2, 4 + 4 * s, 30 + s)
        rhos.append(rho)
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
    ps = PoissonSolver(nn=3, batch=3)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    phib = np.zeros((3,) + tuple(gd.n_c))
    nb = ps.solve_batch(phib, np.array(rhos), eps=2e-10)
    for s in range(3):
        phi = gd.zeros()
        n = ps.solve(phi, rhos[s], eps=2e-10)
        assert n == nb[s]
        assert np.array_equal(phi, phib[s])


@pytest.mark.parametrize('pbc', [0, 1])
def test_batch_charge_branches(cuda, pbc):
    """solve_batch runs solve()'s charge branches per member on the device
    (gpaw/poisson.py:209-299): a neutral member (background shift), charged
    members (Gaussian compensation on a zero-boundary grid, homogeneous
    background on a periodic one).  Each member equals solve() of it alone,
    and both follow the oracle."""
    N = 32
    rhos = []
    for s in range(3):
        rho, L = gaussian_density(N, 0.25, 4 + 2 * s, 70 + s, pbc=bool(pbc))
        rhos.append(rho)
    gd, ogd, ps, ops = solvers(N, L, pbc, nn=3, relax='J', eps=1e-14,
                               batch=3)
    rhos[1] = rhos[1] + 0.02 * (1 if pbc else np.exp(
        -((np.indices(rhos[1].shape) - 15.0) ** 2).sum(0) / 20.0))
    rhos[2] = rhos[2] - 0.01
    assert abs(gd.integrate(rhos[0])) <= 1e-6
    assert abs(gd.integrate(rhos[1])) > 1e-6
    phib = np.zeros((3,) + tuple(gd.n_c))
    nb = ps.solve_batch(phib, np.array(rhos))
    for s in range(3):
        phi = gd.zeros()
        n = ps.solve(phi, rhos[s])
        assert n == nb[s]
        assert np.array_equal(phi, phib[s])
        ophi = ogd.zeros()
        on = ops.solve(ophi, rhos[s])
        assert abs(n - on) <= 1
        assert np.abs(phi - ophi).max() < 1e-7 * np.abs(ophi).max()


def test_fp32_defect_correction(cuda):
    """FP32 V-cycles inside FP64 defect correction reach the same residual."""
    N = 64
    rho, L = gaussian_density(N, 0.2, 8, 1)
    gd, ogd, ps, ops = solvers(N, L, 0, nn=3, maxiter=200)
    eps = 1e-20 * float(np.dot(rho.ravel(), rho.ravel())) * gd.dv
    phi64 = gd.zeros()
    ps.solve(phi64, rho, eps=eps)
    ps32 = type(ps)(nn=3, maxiter=200, precision='fp32')
    ps32.set_grid_descriptor(gd)
    ps32.initialize()
    phi32 = gd.zeros()
    n32 = ps32.solve(phi32, rho, eps=eps)
    assert ps32.last_errors[0] <= eps
    e64 = hartree(ogd, phi64, rho)
    e32 = hartree(ogd, phi32, rho)
    assert abs(e64 - e32) < 1e-8
    assert n32 < 200


def test_fp32_inner_schedules(cuda):
    """Chebyshev-weighted inner cycles vs the reference schedule (float32
    inner, float64 outer): both reach relative residual 1e-10 with E_H
    within 1e-8 Ha of the float64 method; the Chebyshev schedule needs at
    most about half the outer iterations."""
    N = 64
    rho, L = gaussian_density(N, 0.2, 8, 1)
    gd, ogd, ps, ops = solvers(N, L, 0, nn=3, maxiter=200)
    eps = 1e-20 * float(np.dot(rho.ravel(), rho.ravel())) * gd.dv
    phi64 = gd.zeros()
    n64 = ps.solve(phi64, rho, eps=eps)
    e64 = hartree(ogd, phi64, rho)
    counts = {}
    for inner in ('chebyshev', 'reference'):
        p = type(ps)(nn=3, maxiter=200, precision='fp32', inner=inner)
        p.set_grid_descriptor(gd)
        p.initialize()
        phi = gd.zeros()
        counts[inner] = p.solve(phi, rho, eps=eps)
        assert p.last_errors[0] <= eps
        assert abs(hartree(ogd, phi, rho) - e64) < 1e-8
    assert abs(counts['reference'] - n64) <= 1
    assert counts['chebyshev'] <= (n64 + 1) // 2 + 1, (counts, n64)


def test_fp32_batch_equals_single(cuda):
    N = 32
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    rhos = []
    for s in range(3):
        rho, L = gaussian_density(N, 0.2, 4 + 4 * s, 40 + s)
        rhos.append(rho)
    gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
    ps = PoissonSolver(nn=3, batch=3, precision='fp32', maxiter=100)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    eps = [1e-20 * float(np.dot(r.ravel(), r.ravel())) * gd.dv for r in rhos]
    phib = np.zeros((3,) + tuple(gd.n_c))
    nb = ps.solve_batch(phib, np.array(rhos), eps=eps)
    for s in range(3):
        phi = gd.zeros()
        n = ps.solve(phi, rhos[s], eps=eps[s])
        assert n == nb[s]
        assert np.array_equal(phi, phib[s])


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_solve_stream_equals_batch(cuda, precision):
    """Host batches solved with overlapped transfers (two device slots, copy
    streams): every batch's potentials and iteration counts equal those of
    solve_batch, for pinned and pageable inputs and given initial guesses."""
    import torch
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    N, nb, nbatches = 32, 2, 5
    rhos = []
    for k in range(nbatches):
        batch = []
        for s in range(nb):
            rho, L = gaussian_density(N, 0.2, 3 + 2 * s + k, 60 + 7 * k + s)
            batch.append(rho)
        rhos.append(np.array(batch))
    gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
    ps = PoissonSolver(nn=3, batch=nb, precision=precision, maxiter=200)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    eps = 1e-20 * max(float(np.dot(r.ravel(), r.ravel())) for r in rhos[0])
    want, want_n = [], []
    for k in range(nbatches):
        phi = np.zeros_like(rhos[k])
        want_n.append(ps.solve_batch(phi, rhos[k], eps=eps))
        want.append(phi)
    pinned = [torch.from_numpy(r).pin_memory() for r in rhos]
    for inputs in (pinned, rhos):
        out, niters = ps.solve_stream(inputs, eps=eps)
        for k in range(nbatches):
            assert np.array_equal(niters[k], want_n[k])
            assert np.array_equal(out[k].numpy(), want[k])
    # initial guesses travel too: restarting from the answers converges at
    # once and keeps them within the tolerance
    out, niters = ps.solve_stream(pinned, phis=want, eps=eps)
    for k in range(nbatches):
        assert (np.asarray(niters[k]) <= 2).all()
        assert np.abs(out[k].numpy() - want[k]).max() < 1e-6 * np.abs(
            want[k]).max()


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_pdl_off_equals_on(cuda, precision):
    """Programmatic dependent launch changes when kernels are dispatched,
    not what they compute: solves with it off equal those with it on."""
    from gpawdft_b200 import _lib
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    lib = _lib.load()
    N = 48
    rhos = []
    for s in range(2):
        rho, L = gaussian_density(N, 0.2, 6 + s, 90 + s)
        rhos.append(rho)
    rhos = np.array(rhos)
    gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
    eps = 1e-20 * max(float(np.dot(r.ravel(), r.ravel())) for r in rhos)
    out = []
    try:
        for on in (1, 0):
            _lib.check(lib.gpw_set_pdl(on))
            ps = PoissonSolver(nn=3, batch=2, precision=precision, maxiter=200)
            ps.set_grid_descriptor(gd)
            ps.initialize()
            phi = np.zeros_like(rhos)
            n = ps.solve_batch(phi, rhos, eps=eps)
            out.append((phi, n))
    finally:
        _lib.check(lib.gpw_set_pdl(1))
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][0], out[1][0])


@pytest.mark.parametrize('N', [64, 128, 192])
def test_fused_residual_restriction(cuda, N):
    """The float32 form's fused level-0 plan (the second pre-sweep reads the
    defect alone and scales its stencil once; the residual is restricted in
    the same launch and never stored) against the plan that stores the
    first iterate and the residual: the inner corrections differ only by
    float32 rounding, so both reach the tolerance in the same number of
    outer iterations (one more at most) with potentials that agree to the
    solver's accuracy."""
    from gpawdft_b200 import _lib
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    lib = _lib.load()
    rhos = []
    for s in range(2):
        rho, L = gaussian_density(N, 0.2, 8, 140 + s)
        rhos.append(rho)
    rhos = np.array(rhos)
    gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
    eps = [1e-20 * float(np.dot(r.ravel(), r.ravel())) * gd.dv for r in rhos]
    out = []
    for on in (1, 0):
        ps = PoissonSolver(nn=3, batch=2, precision='fp32', maxiter=100)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        _lib.check(lib.gpw_poisson_set_fusion(ps._engine[0], on))
        phi = np.zeros_like(rhos)
        n = ps.solve_batch(phi, rhos, eps=eps)
        assert (ps.last_errors <= eps).all()
        out.append((phi, n))
    assert (np.abs(out[0][1] - out[1][1]) <= 1).all()
    assert np.abs(out[0][0] - out[1][0]).max() < 1e-9 * np.abs(out[1][0]).max()


@pytest.mark.parametrize('cluster', [1, 0])
@pytest.mark.parametrize('N', [128, 192])
def test_coarse_residual_restriction(cuda, N, cluster):
    """The float32 residual of the coarser levels (63^3 at N_c = 128; 95^3
    and 47^3 at 192, and with the cluster launch off every level above the
    one-CTA kernel's) restricted into the next level's rho and first sweep in
    one launch, against the residual, restriction and sweep launched apart:
    the same operations in the same order, so bit-identical potentials and
    iteration counts."""
    from gpawdft_b200 import _lib
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    lib = _lib.load()
    rhos = np.array([gaussian_density(N, 0.2, 8, 150 + s)[0] for s in range(2)])
    L = gaussian_density(N, 0.2, 8, 150)[1]
    gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
    eps = [1e-20 * float(np.dot(r.ravel(), r.ravel())) * gd.dv for r in rhos]
    out = []
    for on in (1, 2):
        ps = PoissonSolver(nn=3, batch=2, precision='fp32', maxiter=100)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        _lib.check(lib.gpw_poisson_set_fusion(ps._engine[0], on))
        _lib.check(lib.gpw_poisson_set_cluster(ps._engine[0], cluster))
        phi = np.zeros_like(rhos)
        n = ps.solve_batch(phi, rhos, eps=eps)
        assert (ps.last_errors <= eps).all()
        labels = [lab for lab, _ in ps.profile_iteration(2, reps=1)]
        out.append((phi, n, labels))
    # the fused plan launches no coarse residual of its own
    assert any(lab.startswith('L1 f32 residual + restriction')
               for lab in out[0][2]), out[0][2]
    assert 'L1 f32 residual' in out[1][2]
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][0], out[1][0])


@pytest.mark.parametrize('N', [64, 128, 192])
def test_cluster_level_plan(cuda, N):
    """The float32 form with the two levels above the one-CTA coarse levels
    in one cluster launch (31^3 and 15^3 at N_c = 64 and 128, 23^3 and 11^3
    at 192) and as separate launches: outer iteration counts within one of
    each other, both to the tolerance, potentials within the float32 inner
    cycles' rounding."""
    from gpawdft_b200 import _lib
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    lib = _lib.load()
    rhos = []
    for s in range(2):
        rho, L = gaussian_density(N, 0.2, 8, 120 + s)
        rhos.append(rho)
    rhos = np.array(rhos)
    gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
    eps = [1e-20 * float(np.dot(r.ravel(), r.ravel())) * gd.dv for r in rhos]
    out = []
    for on in (1, 0):
        ps = PoissonSolver(nn=3, batch=2, precision='fp32', maxiter=100)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        _lib.check(lib.gpw_poisson_set_cluster(ps._engine[0], on))
        phi = np.zeros_like(rhos)
        n = ps.solve_batch(phi, rhos, eps=eps)
        assert (ps.last_errors <= eps).all()
        out.append((phi, n))
    assert np.abs(np.asarray(out[0][1]) - np.asarray(out[1][1])).max() <= 1
    assert np.abs(out[0][0] - out[1][0]).max() < 1e-7 * np.abs(out[1][0]).max()


def test_full_size_127_trajectory(cuda):
    """127^3 (the benchmark grid): the engine's vector transfers, TMA
    stencil variants and one-CTA coarse levels reproduce the reference's
    V-cycle count and potential (oracle: the compiled reference C when it is
    built, else the NumPy restatement)."""
    from oracle import ref
    N = 128
    rho, L = gaussian_density(N, 0.2, 8, 11)
    backend = 'ref' if ref.available() else 'numpy'
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
    ogd = OGD((N,) * 3, (L,) * 3, 0)
    ps = PoissonSolver(nn=3, relax='J', eps=2e-10)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    ops = ol.PoissonSolver(nn=3, relax='J', eps=2e-10, backend=backend)
    ops.set_grid_descriptor(ogd)
    ops.initialize()
    phi = gd.zeros()
    n = ps.solve(phi, rho)
    ophi = ogd.zeros()
    on = ops.solve(ophi, rho)
    assert n == on
    assert np.abs(phi - ophi).max() < 1e-11 * np.abs(ophi).max()
    assert abs(hartree(ogd, phi, rho) - hartree(ogd, ophi, rho)) < 1e-8


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_solve_many_equals_single(cuda, precision):
    """Three grid sizes in one graph launch (device-side loops): every solve
    equals its own single solve (same V-cycles, identical potential), and the
    per-solve latencies are positive and ordered within the launch."""
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver, solve_many
    sizes = [(32, 2), (40, 1), (48, 3)]
    solvers, phis, rhos, epss = [], [], [], []
    for k, (N, nb) in enumerate(sizes):
        rl = []
        for j in range(nb):
            r, L = gaussian_density(N, 0.2, 4 + 2 * j, 100 * k + j)
            rl.append(r)
        gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
        ps = PoissonSolver(nn=3, batch=nb, precision=precision, maxiter=200)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        solvers.append(ps)
        rhos.append(np.array(rl))
        phis.append(np.zeros((nb,) + tuple(gd.n_c)))
        epss.append([1e-20 * float(np.dot(r.ravel(), r.ravel())) * gd.dv
                     for r in rl])
    nits = solve_many(solvers, phis, rhos, epss)
    for ps, phib, rhob, e, nit in zip(solvers, phis, rhos, epss, nits):
        lat = ps.last_latency(len(nit))
        assert (lat > 0).all()
        for b in range(len(nit)):
            phi = ps.gd.zeros()
            n = ps.solve_neutral(phi, rhob[b], eps=e[b])
            assert n == nit[b]
            assert np.array_equal(phi, phib[b])


def test_device_loop_latencies(cuda):
    """One batched solve: per-solve latencies grow with the iteration count."""
    from gpawdft_b200.grid_descriptor import GridDescriptor
    from gpawdft_b200.poisson import PoissonSolver
    N = 32
    rhos = []
    for s in range(3):
        rho, L = gaussian_density(N, 0.2, 8, 60 + s)
        rhos.append(rho)
    gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
    ps = PoissonSolver(nn=3, batch=3, maxiter=200)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    eps = [1e-12, 1e-16, 1e-20]
    eps = [e * float(np.dot(r.ravel(), r.ravel())) * gd.dv
           for e, r in zip(eps, rhos)]
    n = ps.solve_batch(np.zeros((3,) + tuple(gd.n_c)), np.array(rhos),
                       eps=eps)
    lat = ps.last_latency(3)
    assert n[0] < n[1] < n[2]
    assert 0 < lat[0] < lat[1] < lat[2]
