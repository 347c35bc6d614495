"""Multigrid Poisson solver on the GPU (drop-in for gpaw.poisson.PoissonSolver).

``PoissonSolver(nn=3, relax='J', eps=2e-10, maxiter=1000,
remove_moment=None, use_charge_center=False)`` with ``set_grid_descriptor``,
``initialize``, ``solve(phi, rho, charge=None, eps=None, maxcharge=1e-6,
zero_initial_phi=False) -> niter`` and ``PoissonConvergenceError`` as in
gpaw/poisson.py:55-366.  The level hierarchy, smoothing schedule and the three
charge branches follow the reference line by line; the V-cycles and their
convergence loop run on the device in libgpwgrid.so (``gpw_poisson_*``).

Two options go beyond the reference:
  precision='fp32'  float32 V-cycles inside a float64 defect-correction loop
                    (float64 residual, update, charge integral and norms);
                    the inner cycles use Chebyshev-weighted Jacobi smoothing
                    (``inner='chebyshev'``, see ``inner_schedule``), the
                    reference's schedule (``inner='reference'``) or plain
                    weighted Jacobi, 2 pre- and 2 post-sweeps with w = 2/3
                    and 8 on the coarsest level (``inner='jacobi22'``);
  max_levels=k      at most k multigrid levels (the reference coarsens while
                    the grid allows, up to 9 levels);
  solve_batch()     many independent same-grid solves in one batched launch
                    sequence, each with its own convergence test.
"""
import ctypes
import warnings
from math import pi

import numpy as np

from . import _lib, arrays, blas
from .fd_operators import Laplace, LaplaceA, LaplaceB
from .gauss import Gaussian
from .transformers import Transformer


class PoissonConvergenceError(ArithmeticError):
    """Raised when the V-cycles reach ``maxiter`` (gpaw/__init__.py:37)."""


POISSON_GRID_WARNING = ('Grid unsuitable for Poisson solver!  The coarsest '
                        'multigrid level has more than 36 points per axis.')


def create_poisson_solver(name='fd', **kwargs):
    if name == 'fd':
        return PoissonSolver(**kwargs)
    raise NotImplementedError('only the finite-difference solver is built')


def PoissonSolver(dipolelayer=None, **kwargs):
    """gpaw/poisson.py:51-54: the finite-difference solver, wrapped in the
    dipole-layer correction when ``dipolelayer`` names an axis or plane."""
    if dipolelayer is not None:
        from .dipole_correction import DipoleCorrection
        return DipoleCorrection(PoissonSolver(**kwargs), dipolelayer)
    return FDPoissonSolver(**kwargs)


_PREC = {'fp64': 0, 'fp32': 1}


def jacobi_spectrum(op, lowest=False):
    """Extreme eigenvalue of D^-1 A for a constant-coefficient stencil.

    The symbol of the stencil, sum_p c_p cos(o_p . theta), divided by the
    centre coefficient, sampled on the grid's own Fourier modes (zero
    boundary: theta = pi k / (n + 1), k = 1..n; periodic: 2 pi k / n).
    Returns the largest value, or with ``lowest`` the smallest non-zero one.
    """
    n_c = op.gd.n_c
    axes = []
    for c in range(3):
        n = int(n_c[c])
        if op.gd.pbc_c[c]:
            axes.append(2 * np.pi * np.arange(n) / n)
        else:
            axes.append(np.pi * np.arange(1, n + 1) / (n + 1))
    # the symbol is a sum of per-axis terms for star stencils; sample at
    # most 64 modes per axis (it is smooth in theta)
    axes = [a if len(a) <= 64 else
            np.unique(np.concatenate([a[::max(1, len(a) // 64)], a[-1:],
                                      a[:1]])) for a in axes]
    t0, t1, t2 = np.meshgrid(*axes, indexing='ij')
    c0 = None
    sym = 0.0
    for coef, o in zip(op.coef_p, op.offset_pc):
        if not o.any():
            c0 = coef if c0 is None else c0 + coef
        sym = sym + coef * np.cos(o[0] * t0 + o[1] * t1 + o[2] * t2)
    lam = sym / c0
    if lowest:
        nz = lam[lam > 1e-12 * lam.max()]
        return float(nz.min())
    return float(lam.max())


def chebyshev_weights(k, lo, hi):
    """Jacobi weights whose product of (1 - w_i lambda) is the degree-k
    Chebyshev polynomial of [lo, hi], smallest weight first."""
    return [2.0 / ((hi + lo) + (hi - lo) * np.cos((2 * i - 1) * np.pi /
                                                   (2 * k)))
            for i in range(1, k + 1)]


def inner_schedule(operators, fine=(2, 6.0), coarse=(3, 4.0), coarsest=8):
    """Float32 inner V-cycle schedule of the defect-correction form.

    Level 0: ``fine[0]`` pre- and post-sweeps with Chebyshev weights damping
    the modes with lambda(D^-1 A) in [lambda_max / fine[1], lambda_max];
    coarse levels likewise with ``coarse``; the coarsest level ``coarsest``
    post-sweeps over its whole non-zero spectrum.  Returns (npre, npost,
    weights) in the layout of gpw_poisson_set_inner_schedule.
    """
    npre, npost, weights = [], [], []
    L = len(operators)
    for l, op in enumerate(operators):
        hi = jacobi_spectrum(op)
        if l == L - 1:
            lo = min(jacobi_spectrum(op, lowest=True), hi)
            w = chebyshev_weights(coarsest, lo, hi)
            npre.append(0)
            npost.append(coarsest)
            weights.extend(w)
            continue
        k, ratio = fine if l == 0 else coarse
        w = chebyshev_weights(k, hi / ratio, hi)
        npre.append(k)
        npost.append(k)
        weights.extend(w + w[::-1])
    return npre, npost, weights


def jacobi22_schedule(L, w=2.0 / 3.0, coarsest=8):
    """Plain weighted-Jacobi inner schedule: 2 pre- and 2 post-sweeps of
    weight w on every level but the coarsest, which gets ``coarsest``
    post-sweeps of the same weight (layout of ``inner_schedule``)."""
    npre = [2] * (L - 1) + [0]
    npost = [2] * (L - 1) + [coarsest]
    weights = []
    for a, b in zip(npre, npost):
        weights.extend([w] * (a + b))
    return npre, npost, weights


class FDPoissonSolver:
    def __init__(self, nn=3, relax='J', eps=2e-10, maxiter=1000,
                 remove_moment=None, use_charge_center=False,
                 precision='fp64', batch=1, inner='chebyshev',
                 max_levels=None):
        self.relax = relax
        self.nn = nn
        self.eps = eps
        self.charged_periodic_correction = None
        self.maxiter = maxiter
        self.remove_moment = remove_moment
        self.use_charge_center = use_charge_center
        if relax == 'GS':
            self.relax_method = 1
        elif relax == 'J':
            self.relax_method = 2
        else:
            raise NotImplementedError('Relaxation method %s' % relax)
        if precision not in _PREC:
            raise ValueError("precision must be 'fp64' or 'fp32'")
        self.precision = precision
        if inner not in ('chebyshev', 'reference', 'jacobi22'):
            raise ValueError("inner must be 'chebyshev', 'reference' or "
                             "'jacobi22'")
        self.inner = inner
        if max_levels is not None and int(max_levels) < 1:
            raise ValueError('max_levels must be at least 1')
        self.max_levels = None if max_levels is None else int(max_levels)
        self.batch = int(batch)
        self.description = None
        self._engine = None
        self.last_errors = None

    def todict(self):
        return {'name': 'fd', 'nn': self.nn, 'relax': self.relax,
                'eps': self.eps, 'remove_moment': self.remove_moment}

    def get_stencil(self):
        return self.nn

    def set_grid_descriptor(self, gd):
        """gpaw/poisson.py:91-149."""
        self.gd = gd
        scale = -0.25 / pi
        if self.nn == 'M':
            if not gd.orthogonal:
                raise RuntimeError('Cannot use Mehrstellen stencil with '
                                   'non orthogonal cell.')
            self.operators = [LaplaceA(gd, -scale)]
            self.B = LaplaceB(gd)
        else:
            self.operators = [Laplace(gd, scale, self.nn)]
            self.B = None
        self.interpolators = []
        self.restrictors = []
        level = 0
        self.presmooths = [2]
        self.postsmooths = [1]
        self.weights = [2.0 / 3.0]
        while level < 8 and (self.max_levels is None or
                             level + 1 < self.max_levels):
            try:
                gd2 = gd.coarsen()
            except ValueError:
                break
            self.operators.append(Laplace(gd2, scale, 1))
            self.interpolators.append(Transformer(gd2, gd))
            self.restrictors.append(Transformer(gd, gd2))
            self.presmooths.append(4)
            self.postsmooths.append(4)
            self.weights.append(1.0)
            level += 1
            gd = gd2
        self.levels = level
        self._engine = None
        if self.operators[-1].gd.N_c.max() > 36:
            warnings.warn(POISSON_GRID_WARNING + '\n' + self.get_description(),
                          stacklevel=2)

    def get_description(self):
        name = {1: 'Gauss-Seidel', 2: 'Jacobi'}[self.relax_method]
        coarsest_grid = self.operators[-1].gd.N_c
        lines = ['%s solver with %d multi-grid levels'
                 % (name, self.levels + 1),
                 '    Coarsest grid: %s points' %
                 ' x '.join([str(N) for N in coarsest_grid])]
        if coarsest_grid.max() > 24:
            lines.extend(['    Warning: Coarse grid has more than 24 points.',
                          '             More multi-grid levels recommended.'])
        lines.extend(['    Stencil: %s' % self.operators[0].description,
                      '    Tolerance: %e' % self.eps,
                      '    Max iterations: %d' % self.maxiter])
        if self.remove_moment is not None:
            lines.append('    Remove moments up to L=%d' % self.remove_moment)
        if self.use_charge_center:
            lines.append('    Compensate for charged system using center of '
                         'majority charge')
        return '\n'.join(lines)

    def initialize(self, load_gauss=False):
        """gpaw/poisson.py:174-195 (+ the device engine)."""
        level = self.levels
        self.step = 0.66666666 / self.operators[0].get_diagonal_element()
        self.presmooths[level] = 8
        self.postsmooths[level] = 8
        self._make_engine(self.batch)
        if load_gauss:
            self.load_gauss()

    def _make_engine(self, nbatch):
        lib = _lib.load()
        if self._engine is not None and self._engine[1] >= nbatch:
            return
        self._free_engine()
        L = self.levels + 1
        VP = ctypes.c_void_p
        ops = (VP * L)(*[op.handle for op in self.operators])
        rs = (VP * max(L - 1, 1))(*([t.handle for t in self.restrictors] or
                                    [None]))
        ips = (VP * max(L - 1, 1))(*([t.handle for t in self.interpolators] or
                                     [None]))
        pre = (ctypes.c_int * L)(*self.presmooths)
        post = (ctypes.c_int * L)(*self.postsmooths)
        w = (ctypes.c_double * L)(*self.weights)
        h = VP()
        _lib.check(lib.gpw_poisson_new(L, ops, rs, ips, pre, post, w,
                                       self.relax_method, float(self.gd.dv),
                                       int(nbatch), ctypes.byref(h)))
        self._engine = (h, int(nbatch))
        self._lib = lib
        if not getattr(self, '_device_loop', True):
            _lib.check(lib.gpw_poisson_set_device_loop(h, 0))
        if (self.precision == 'fp32' and self.inner != 'reference' and
                self.relax_method == 2 and L > 1):
            if self.inner == 'chebyshev':
                npre, npost, ws = inner_schedule(self.operators)
            else:
                npre, npost, ws = jacobi22_schedule(L)
            a_pre = (ctypes.c_int * L)(*npre)
            a_post = (ctypes.c_int * L)(*npost)
            a_w = (ctypes.c_double * len(ws))(*ws)
            _lib.check(lib.gpw_poisson_set_inner_schedule(h, a_pre, a_post,
                                                          a_w, len(ws)))

    def set_device_loop(self, on=True):
        """Run the convergence loop on the device (default) or replay one
        iteration graph per outer iteration from the host (same kernels and
        results; for profilers that cannot look inside conditional graph
        nodes)."""
        if self._engine is None:
            self.initialize()
        _lib.check(self._lib.gpw_poisson_set_device_loop(self._engine[0],
                                                         int(bool(on))))
        self._device_loop = bool(on)

    def _free_engine(self):
        if self._engine is not None:
            self._lib.gpw_poisson_free(self._engine[0])
            self._engine = None

    def __del__(self):
        try:
            self._free_engine()
        except Exception:
            pass

    def load_gauss(self, center=None):
        if not hasattr(self, 'rho_gauss') or center is not None:
            gauss = Gaussian(self.gd, center=center)
            self.rho_gauss = arrays.to_device(gauss.get_gauss(0))
            self.phi_gauss = arrays.to_device(gauss.get_gauss_pot(0))

    # ------------------------------------------------------------ solving
    def solve(self, phi, rho, charge=None, eps=None, maxcharge=1e-6,
              zero_initial_phi=False):
        """gpaw/poisson.py:203-304; returns the number of V-cycles."""
        assert np.all(tuple(phi.shape) == tuple(self.gd.n_c))
        assert np.all(tuple(rho.shape) == tuple(self.gd.n_c))
        if self._engine is None:
            self.initialize()
        if eps is None:
            eps = self.eps
        phi_d = arrays.to_device(phi)
        rho_d = arrays.to_device(rho)
        if self.remove_moment:
            raise NotImplementedError('remove_moment is not part of this '
                                      'build')
        if charge is None and not (self.use_charge_center and
                                   not self.gd.pbc_c.any()):
            # the charge integral and the branch run on the device: no host
            # round trip before the solve
            phi_b, rho_b = phi_d.unsqueeze(0), rho_d.unsqueeze(0)
            rho_n, q = self._charge_prepare(phi_b, rho_b, 1, maxcharge,
                                            zero_initial_phi, 0)
            niter = int(self._run(phi_b, rho_n, 1, [eps])[0])
            self._charge_finish(phi_b, 1, q)
            if not arrays.is_device(phi):
                arrays.writeback(phi, phi_d)
            return niter
        actual_charge = self.gd.integrate(rho_d)
        background = (actual_charge / self.gd.dv /
                      self.gd.get_size_of_global_array().prod())
        if charge is None:
            charge = actual_charge
        if abs(charge) <= maxcharge:
            niter = self.solve_neutral(phi_d, self._shifted(rho_d, background),
                                       eps=eps)
        elif abs(charge) > maxcharge and self.gd.pbc_c.all():
            if zero_initial_phi:
                phi_d.zero_()
            niter = self.solve_neutral(phi_d, self._shifted(rho_d, background),
                                       eps=eps)
        elif abs(charge) > maxcharge and not self.gd.pbc_c.any():
            if self.use_charge_center:
                rho_h = rho if not arrays.is_device(rho) else \
                    rho.cpu().numpy()
                charge_sign = actual_charge / abs(actual_charge)
                rho_sign = rho_h * charge_sign
                rho_sign[np.where(rho_sign < 0)] = 0
                absolute_charge = self.gd.integrate(rho_sign)
                center = - self.gd.calculate_dipole_moment(rho_sign) \
                    / absolute_charge
                border_offset = np.inner(self.gd.h_cv, np.array((7, 7, 7)))
                borders = np.inner(self.gd.h_cv, self.gd.N_c)
                borders -= border_offset
                if np.any(center > borders) or np.any(center < border_offset):
                    raise RuntimeError('Poisson solver: center of charge '
                                       'outside borders - please increase box')
                self.load_gauss(center=center)
            else:
                self.load_gauss()
            q = actual_charge / np.sqrt(4 * pi)
            rho_neutral = rho_d.clone()
            blas.axpy(-q, self.rho_gauss, rho_neutral)
            if zero_initial_phi:
                phi_d.zero_()
            else:
                blas.axpy(-q, self.phi_gauss, phi_d)
            niter = self.solve_neutral(phi_d, rho_neutral, eps=eps)
            blas.axpy(q, self.phi_gauss, phi_d)
        else:
            raise NotImplementedError('Charged systems with mixed periodic/'
                                      'zero boundary conditions')
        if not arrays.is_device(phi):
            arrays.writeback(phi, phi_d)
        return niter

    def _shifted(self, rho_d, background):
        out = rho_d.clone()
        blas.add_scalar(rho_d, -background, out)
        return out

    def solve_neutral(self, phi, rho, eps=2e-10):
        """gpaw/poisson.py:306-329 (one grid)."""
        phi_d = arrays.to_device(phi)
        niters = self._run(phi_d, arrays.to_device(rho), 1, [eps])
        if not arrays.is_device(phi):
            arrays.writeback(phi, phi_d)
        return int(niters[0])

    def iterate_batch(self, phi_b, rho_b, k):
        """Exactly k outer iterations (V-cycles, or defect-correction steps)
        on a batch of device tensors, whatever the residual; returns the
        per-member error sum(r^2) dv after them."""
        nb = int(phi_b.shape[0])
        self._run(arrays.to_device(phi_b), arrays.to_device(rho_b), nb,
                  [0.0] * nb, maxiter=int(k), exact=True)
        return np.array(self.last_errors)

    def _run(self, phi_d, rho_d, nb, eps_list, maxiter=None, exact=False):
        if self.B is not None:
            rho2 = arrays.empty_like_device(rho_d.shape,
                                            arrays.np_dtype_of(rho_d))
            self.B.apply(rho_d, rho2)
            rho_d = rho2
        self._make_engine(nb)
        eps_a = np.ascontiguousarray(eps_list, float)
        niter = np.zeros(nb, np.int32)
        err = np.zeros(nb, float)
        rc = self._lib.gpw_poisson_solve(
            self._engine[0], arrays.ptr(phi_d), arrays.ptr(rho_d), nb,
            eps_a.ctypes.data, int(maxiter or self.maxiter),
            _PREC[self.precision], niter.ctypes.data, err.ctypes.data,
            arrays.stream())
        self.last_errors = err
        if exact and rc == _lib.GPW_ECONV:
            rc = _lib.GPW_OK  # the requested iteration count, not a failure
        if rc == _lib.GPW_ECONV:
            raise PoissonConvergenceError(
                'Poisson solver did not converge in %d iterations!' %
                self.maxiter)
        _lib.check(rc)
        if self.gd.pbc_c.all():
            # set the average potential to zero in periodic systems
            npts = int(np.prod(self.gd.get_size_of_global_array()))
            sums = blas.vector_sums(phi_d, nb)
            for b in range(nb):
                blas.add_scalar(phi_d[b] if nb > 1 else phi_d,
                                -sums[b] / npts)
        return niter

    def profile_iteration(self, nbatch=None, reps=5):
        """Live per-launch times (ms) of one outer iteration on the engine's
        buffers: a list of (label, ms).  Call after a solve of this batch
        size (it overwrites the engine's buffers)."""
        nb = self._engine[1] if nbatch is None else int(nbatch)
        cap = 256
        labels = ctypes.create_string_buffer(cap * 64)
        ms = np.zeros(cap)
        count = ctypes.c_int()
        _lib.check(self._lib.gpw_poisson_profile_iteration(
            self._engine[0], nb, _PREC[self.precision], int(reps), labels,
            cap * 64, ms.ctypes.data, cap, ctypes.byref(count),
            arrays.stream()))
        names = labels.raw.split(b'\0')[:count.value]
        return [(n.decode(), float(t)) for n, t in zip(names, ms)]

    def residual_norms(self, phi_b, rho_b):
        """||A phi - rho||_2 of each member of a batch (level-0 operator,
        device tensors (nb, *n_c))."""
        out = np.zeros(phi_b.shape[0])
        for b in range(phi_b.shape[0]):
            out[b] = np.sqrt(float(
                self.operators[0].residual(phi_b[b], rho_b[b])[0].item()))
        return out

    def last_latency(self, nbatch=None):
        """Per-solve device latency (ms) of the last solve: from the start of
        the iterations to the end of the iteration in which each solve
        converged."""
        nb = self._engine[1] if nbatch is None else int(nbatch)
        ms = np.zeros(nb)
        _lib.check(self._lib.gpw_poisson_last_latency(
            self._engine[0], nb, ms.ctypes.data, arrays.stream()))
        return ms

    def solve_batch(self, phi_b, rho_b, eps=None, maxcharge=1e-6,
                    zero_initial_phi=False):
        """``solve(phi, rho)`` of every member of a batch (nb, *n_c) on one grid.

        Each member goes through the charge branches of ``solve``
        (gpaw/poisson.py:209-299: the charge integral, then the background
        shift or the Gaussian compensation), on the device with no host
        round trip, and stops at its own ``error <= eps``; results and
        V-cycle counts equal those of solving each grid alone.  Returns the
        per-solve iteration counts.
        """
        if self._engine is None:
            self.initialize()
        nb = int(phi_b.shape[0])
        if eps is None:
            eps = self.eps
        if self.use_charge_center and not self.gd.pbc_c.any():
            # the Gaussian's centre depends on each member's charge
            return np.array([self.solve(phi_b[b], rho_b[b], eps=np.broadcast_to(
                np.asarray(eps, float), (nb,))[b], maxcharge=maxcharge,
                zero_initial_phi=zero_initial_phi) for b in range(nb)])
        eps_list = np.broadcast_to(np.asarray(eps, float), (nb,))
        phi_d = arrays.to_device(phi_b)
        rho_d = arrays.to_device(rho_b)
        rho_n, q = self._charge_prepare(phi_d, rho_d, nb, maxcharge,
                                        zero_initial_phi, 0)
        niter = self._run(phi_d, rho_n, nb, eps_list)
        self._charge_finish(phi_d, nb, q)
        if not arrays.is_device(phi_b):
            arrays.writeback(phi_b, phi_d)
        return niter

    def _charge_prepare(self, phi_d, rho_d, nb, maxcharge, zero_initial_phi,
                        slot):
        """Device charge branches of ``solve`` for a batch: returns the
        density the neutral solve uses and the per-member Gaussian moments."""
        import torch
        if not self.gd.pbc_c.any():
            self.load_gauss()
            rg, pg = arrays.ptr(self.rho_gauss), arrays.ptr(self.phi_gauss)
        else:
            rg = pg = None
        shape = (nb,) + tuple(int(x) for x in self.gd.n_c)
        bufs = getattr(self, '_charge_bufs', None)
        if bufs is None or bufs[0].shape[0] < nb:
            rows = max(nb, self._engine[1] if self._engine else 1)
            bufs = (torch.empty((rows,) + shape[1:], dtype=torch.float64,
                                device=rho_d.device),
                    torch.empty((2, rows), dtype=torch.float64,
                                device=rho_d.device))
            self._charge_bufs = bufs
        rho_n = bufs[0][:nb]
        q = bufs[1][slot, :nb]
        pbc = sum(1 << c for c in range(3) if self.gd.pbc_c[c])
        npts = float(np.prod(self.gd.get_size_of_global_array()))
        _lib.check(self._lib.gpw_poisson_charge_prepare(
            nb, int(np.prod(shape[1:])), arrays.ptr(rho_d), arrays.ptr(rho_n),
            arrays.ptr(phi_d), rg, pg, float(self.gd.dv), npts,
            float(maxcharge), pbc, int(bool(zero_initial_phi)), arrays.ptr(q),
            arrays.stream()))
        if self.gd.pbc_c.any() and not self.gd.pbc_c.all():
            # only a mixed-boundary grid can meet the unsupported branch
            if torch.isnan(q).any().item():
                raise NotImplementedError('Charged systems with mixed '
                                          'periodic/zero boundary conditions')
        return rho_n, q

    def _charge_finish(self, phi_d, nb, q):
        if self.gd.pbc_c.any():
            return
        _lib.check(self._lib.gpw_poisson_charge_finish(
            nb, int(np.prod(self.gd.n_c)), arrays.ptr(phi_d),
            arrays.ptr(self.phi_gauss), arrays.ptr(q), arrays.stream()))

    def solve_stream(self, rhos, phis=None, eps=None, out=None):
        """``solve_batch`` of a sequence of host batches, each (nb, *n_c)
        float64 (charge branches included), with the host<->device transfers
        overlapped with
        the solves: while batch k is solved, batch k+1's densities travel to
        the device and batch k-1's potentials back (two device slots, one
        copy stream per direction).

        Host tensors should be pinned (``torch.Tensor.pin_memory()``);
        pageable arrays are accepted but their copies do not overlap.
        ``phis``: initial guesses (None: zero, nothing transferred).
        ``out``: host tensors receiving the potentials (None: allocated
        pinned).  Each solve stops at its own ``error <= eps`` exactly as in
        ``solve_batch``.  Returns (out, per-batch iteration counts).
        """
        import torch
        arrays.require_cuda()
        if self._engine is None:
            self.initialize()
        n = len(rhos)
        if n == 0:
            return [], []
        if eps is None:
            eps = self.eps
        shape = tuple(rhos[0].shape)
        nb = int(shape[0])
        dev = torch.device('cuda', torch.cuda.current_device())

        def host(a):
            return a if isinstance(a, torch.Tensor) else torch.from_numpy(
                np.ascontiguousarray(a, float))

        rhos = [host(r) for r in rhos]
        if any(tuple(r.shape) != shape or r.dtype != torch.float64
               for r in rhos):
            raise ValueError('solve_stream: batches must share one float64 '
                             'shape')
        if phis is not None:
            phis = [host(p) for p in phis]
        if out is None:
            out = [torch.empty(shape, dtype=torch.float64).pin_memory()
                   for _ in range(n)]
        compute = torch.cuda.current_stream()
        up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        rho_d = [torch.empty(shape, dtype=torch.float64, device=dev)
                 for _ in range(2)]
        phi_d = [torch.empty_like(rho_d[0]) for _ in range(2)]
        rho_free = [None, None]   # the slot's last solve has read its rho
        phi_free = [None, None]   # the slot's last result has left
        arrived = [None] * n

        def upload(k):
            s = k % 2
            with torch.cuda.stream(up):
                if rho_free[s] is not None:
                    up.wait_event(rho_free[s])
                if phi_free[s] is not None:
                    up.wait_event(phi_free[s])
                rho_d[s].copy_(rhos[k], non_blocking=True)
                if phis is not None:
                    phi_d[s].copy_(phis[k], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(up)
            arrived[k] = ev

        niters = [None] * n
        eps_a = np.ascontiguousarray(np.broadcast_to(np.asarray(eps, float),
                                                     (nb,)))
        # solves are enqueued without waiting (results collected two batches
        # later, before their mailbox slot is reused) where the solve needs no
        # host step after its loop
        use_async = self.B is None and not self.gd.pbc_c.all()
        pending = {}

        def collect(k):
            ev, slot = pending.pop(k)
            ev.synchronize()
            niters[k] = self._collect(nb, slot)

        upload(0)
        if n > 1:
            upload(1)
        for k in range(n):
            s = k % 2
            compute.wait_event(arrived[k])
            if phis is None:
                if phi_free[s] is not None:
                    compute.wait_event(phi_free[s])
                phi_d[s].zero_()
            if k - 2 in pending:
                collect(k - 2)
            if use_async:
                rho_n, q = self._charge_prepare(phi_d[s], rho_d[s], nb, 1e-6,
                                                False, s)
                if not self._solve_async(phi_d[s], rho_n, nb, eps_a, s):
                    # no device-side loop here: this batch and the rest are
                    # solved in turn
                    use_async = False
                    niters[k] = self._run(phi_d[s], rho_n, nb, eps_a)
                self._charge_finish(phi_d[s], nb, q)
            elif niters[k] is None:
                niters[k] = self.solve_batch(phi_d[s], rho_d[s], eps=eps)
            done = torch.cuda.Event()
            done.record(compute)
            rho_free[s] = done
            if use_async and niters[k] is None:
                pending[k] = (done, s)
            with torch.cuda.stream(down):
                down.wait_event(done)
                out[k].copy_(phi_d[s], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(down)
            phi_free[s] = ev
            if k + 2 < n:
                upload(k + 2)
        for k in sorted(pending):
            collect(k)
        down.synchronize()   # every copy and solve has finished
        return out, niters

    def _solve_async(self, phi_d, rho_d, nb, eps_a, slot):
        """Enqueue a solve on the current stream (results to mailbox `slot`);
        False where asynchronous solves are unavailable."""
        self._make_engine(nb)
        rc = self._lib.gpw_poisson_solve_async(
            self._engine[0], arrays.ptr(phi_d), arrays.ptr(rho_d), nb,
            eps_a.ctypes.data, int(self.maxiter), _PREC[self.precision],
            int(slot), arrays.stream())
        if rc == _lib.GPW_ENOTSUP:
            return False
        _lib.check(rc)
        return True

    def _collect(self, nb, slot):
        niter = np.zeros(nb, np.int32)
        err = np.zeros(nb, float)
        rc = self._lib.gpw_poisson_collect(
            self._engine[0], nb, int(self.maxiter), _PREC[self.precision],
            int(slot), niter.ctypes.data, err.ctypes.data)
        self.last_errors = err
        if rc == _lib.GPW_ECONV:
            raise PoissonConvergenceError(
                'Poisson solver did not converge in %d iterations!' %
                self.maxiter)
        _lib.check(rc)
        return niter

    def estimate_memory(self, mem=None):
        gdbytes = int(np.prod(self.gd.n_c)) * 8
        nbytes = 0
        for level in range(self.levels + 1):
            nbytes += 4 * gdbytes
            gdbytes //= 8
        return nbytes

    def __repr__(self):
        return 'PoissonSolver(relax=\'%s\', nn=%s, eps=%e)' % (
            self.relax, repr(self.nn), self.eps)


def solve_many(solvers, phis, rhos, eps):
    """Independent neutral solves on several grids in ONE graph launch.

    ``solvers[i]`` is an initialised FDPoissonSolver (its own grid, same
    ``precision`` for all), ``phis[i]`` / ``rhos[i]`` device or host arrays of
    shape (nb_i, *n_c), ``eps[i]`` the per-solve tolerances (scalar or nb_i
    values).  Every solver's convergence loop runs on the device as one
    branch of a single CUDA graph (gpw_poisson_solve_many).  Returns the
    per-solve iteration counts.
    """
    n = len(solvers)
    if not (len(phis) == len(rhos) == len(eps) == n) or n == 0:
        raise ValueError('solvers, phis, rhos and eps must have one entry per '
                         'solver')
    prec = {s.precision for s in solvers}
    if len(prec) != 1:
        raise ValueError('all solvers must use the same precision')
    lib = _lib.load()
    handles, phid, rhod, nbs, epsa, nits, errs, hosts = [], [], [], [], [], \
        [], [], []
    for s, phi, rho, e in zip(solvers, phis, rhos, eps):
        if s.B is not None or s.gd.pbc_c.any():
            raise NotImplementedError('solve_many: zero-boundary grids with '
                                      'the nn=1..6 stencils only')
        nb = int(phi.shape[0])
        s._make_engine(nb)
        p = arrays.to_device(phi)
        r = arrays.to_device(rho)
        handles.append(s._engine[0])
        phid.append(p)
        rhod.append(r)
        hosts.append(phi)
        nbs.append(nb)
        epsa.append(np.ascontiguousarray(np.broadcast_to(
            np.asarray(e, float), (nb,))))
        nits.append(np.zeros(nb, np.int32))
        errs.append(np.zeros(nb))
    VP = ctypes.c_void_p
    rc = lib.gpw_poisson_solve_many(
        n, (VP * n)(*[h.value for h in handles]),
        (VP * n)(*[arrays.ptr(p) for p in phid]),
        (VP * n)(*[arrays.ptr(r) for r in rhod]),
        np.ascontiguousarray(nbs, np.int64).ctypes.data,
        (VP * n)(*[a.ctypes.data for a in epsa]), int(solvers[0].maxiter),
        _PREC[solvers[0].precision], (VP * n)(*[a.ctypes.data for a in nits]),
        (VP * n)(*[a.ctypes.data for a in errs]), arrays.stream())
    for s, e in zip(solvers, errs):
        s.last_errors = e
    if rc == _lib.GPW_ECONV:
        raise PoissonConvergenceError('Poisson solver did not converge in %d '
                                      'iterations!' % solvers[0].maxiter)
    _lib.check(rc)
    for h, p in zip(hosts, phid):
        if not arrays.is_device(h):
            arrays.writeback(h, p)
    return nits
