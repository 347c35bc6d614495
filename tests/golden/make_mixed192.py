"""Generate tests/golden/mixed192.npz: the mixed-precision Poisson workload
(N_c = 192 zero boundary, 191^3 unknowns, h = 0.15 Angstrom, 64 Gaussians with
log-uniform widths 0.3-2.0 Angstrom and N(0, 1) charges re-centred to
neutral, seed 4) solved by the reference's own C (oracle/_ref, through the
restated FDPoissonSolver of oracle/layer.py) to relative residual 1e-10.

Run where the reference is mounted and oracle/_ref is built:
    python tests/golden/make_mixed192.py

The potential itself (56 MB) is not stored: the fixture keeps the Hartree
energy, the V-cycle count, the potential at 4096 seeded grid points, its
per-plane sums along axis 0 and its largest magnitude, plus checksums of the
density so the GPU test can confirm it regenerated the same input.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gpawdft_b200.workloads import gaussian_density  # noqa: E402
from oracle import layer, ref  # noqa: E402
from oracle.geometry import GridDescriptor  # noqa: E402

N = 192


def density():
    return gaussian_density(N, 0.15, 64, 4, sigma_range=(0.3, 2.0),
                            log_sigma=True, charges='normal')


def main():
    assert ref.available(), 'build oracle/_ref first (make -C oracle)'
    rho, L = density()
    gd = GridDescriptor((N,) * 3, (L,) * 3, 0)
    rho_sq = float(np.dot(rho.ravel(), rho.ravel())) * gd.dv
    eps = 1e-20 * rho_sq
    ps = layer.PoissonSolver(nn=3, relax='J', eps=eps, maxiter=1000,
                             backend='ref')
    ps.set_grid_descriptor(gd)
    ps.initialize()
    phi = gd.zeros()
    t = time.time()
    niter = ps.solve(phi, rho)
    print('reference solve: %d V-cycles in %.1f s' % (niter, time.time() - t))
    idx = np.random.default_rng(192).choice(phi.size, 4096, replace=False)
    np.savez_compressed(
        os.path.join(HERE, 'mixed192.npz'),
        L=L, eps=eps, rho_sq=rho_sq, rho_sum=float(rho.sum()),
        rho_abs_sum=float(np.abs(rho).sum()), niter=niter,
        final_error=float(ps.errors[-1]),
        eh=0.5 * gd.dv * float(np.dot(phi.ravel(), rho.ravel())),
        idx=idx, phi_samples=phi.ravel()[idx],
        phi_plane_sums=phi.sum(axis=(1, 2)), phi_absmax=np.abs(phi).max())


if __name__ == '__main__':
    main()
