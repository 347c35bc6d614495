"""Generate the golden fixtures in tests/golden/ from the reference's own C.

Run in a container where the reference is mounted and oracle/_ref is built
(``make -C oracle``):  python tests/golden/make_golden.py

Every case drives the compiled reference (c/bmgs, c/bc.c, c/operators.c,
c/transformers.c via oracle/_ref) through the restated Python layer of
oracle/layer.py on seeded small inputs and stores inputs + outputs in
golden.npz.  The GPU tests replay these cases through the product; the CPU
tests replay them through the NumPy restatement.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import layer, ref  # noqa: E402
from oracle.geometry import GridDescriptor, phase_cd_for_k  # noqa: E402


def rnd(rng, shape, dtype):
    a = rng.standard_normal(shape)
    if dtype == complex:
        a = a + 1j * rng.standard_normal(shape)
    return a


def cases():
    """(name, kind, params) of every fixture."""
    out = []
    for pbc in (0, 1):
        for dtype in ('float', 'complex'):
            for nn in (1, 2, 3):
                out.append(('laplace_p%d_%s_nn%d' % (pbc, dtype, nn), 'laplace',
                            dict(N=(8, 6, 10), cell=(2.0, 1.5, 2.5), pbc=pbc,
                                 dtype=dtype, nn=nn, scale=-0.5)))
            out.append(('gradient_p%d_%s' % (pbc, dtype), 'gradient',
                        dict(N=(8, 6, 10), cell=(2.0, 1.5, 2.5), pbc=pbc,
                             dtype=dtype, nn=3, v=1)))
            for nn in (1, 3):
                for direction in ('restrict', 'interpolate'):
                    out.append(('%s_p%d_%s_nn%d' % (direction, pbc, dtype, nn),
                                direction,
                                dict(N=(16, 12, 12), cell=(4.0, 3.0, 3.0),
                                     pbc=pbc, dtype=dtype, nn=nn)))
        out.append(('jacobi_p%d' % pbc, 'jacobi',
                    dict(N=(10, 8, 12), cell=(2.5, 2.0, 3.0), pbc=pbc, nn=3,
                         nrelax=3, w=2.0 / 3.0)))
        out.append(('gs_p%d' % pbc, 'gs',
                    dict(N=(8, 6, 10), cell=(2.0, 1.5, 2.5), pbc=pbc, nn=1,
                         nrelax=2)))
    out.append(('guc_fcc', 'guc', dict(N=(8, 8, 8), pbc=1, nn=2,
                                       cell=[(0, 1.7, 1.7), (1.7, 0, 1.7),
                                             (1.7, 1.7, 0)])))
    out.append(('poisson_16', 'poisson', dict(N=16, L=5.0, nn=3)))
    return out


def run_case(kind, p, backend, rng_seed, arrays=None):
    """Evaluate one case; with ``arrays`` given, reuse those inputs."""
    rng = np.random.default_rng(rng_seed)
    dtype = complex if p.get('dtype') == 'complex' else float
    gd = GridDescriptor(p['N'] if kind != 'poisson' else (p['N'],) * 3,
                        p['cell'] if kind != 'poisson' else (p['L'],) * 3,
                        p['pbc'] if kind != 'poisson' else 0)
    inp = dict(arrays or {})
    ph = phase_cd_for_k(gd, [0.21, -0.37, 0.13]) if dtype == complex else None
    if kind in ('laplace', 'gradient', 'guc'):
        a = inp.get('a', rnd(rng, (1,) + tuple(gd.n_c), dtype))
        if kind == 'gradient':
            op = layer.Gradient(gd, p['v'], 1.0, p['nn'], dtype, backend)
        elif kind == 'guc':
            op = layer.Laplace(gd, 1.0, p['nn'], dtype, backend)
        else:
            op = layer.Laplace(gd, p['scale'], p['nn'], dtype, backend)
        o = np.zeros_like(a)
        op.apply(a, o, ph)
        return {'a': a, 'out': o, 'phase': ph if ph is not None else np.ones((3, 2), complex)}
    if kind in ('restrict', 'interpolate'):
        gdc = gd.coarsen()
        gi, go = (gd, gdc) if kind == 'restrict' else (gdc, gd)
        a = inp.get('a', rnd(rng, (1,) + tuple(gi.n_c), dtype))
        t = layer.Transformer(gi, go, p['nn'], dtype, backend)
        o = t.apply(a, None, ph)
        return {'a': a, 'out': o, 'phase': ph if ph is not None else np.ones((3, 2), complex)}
    if kind in ('jacobi', 'gs'):
        f = inp.get('f', rnd(rng, tuple(gd.n_c), float))
        s = inp.get('s', rnd(rng, tuple(gd.n_c), float))
        op = layer.Laplace(gd, -0.25 / np.pi, p['nn'], float, backend)
        g = f.copy()
        op.relax(2 if kind == 'jacobi' else 1, g, s, p['nrelax'],
                 p.get('w', 1.0))
        return {'f': f, 's': s, 'out': g}
    if kind == 'poisson':
        rho = inp.get('rho')
        if rho is None:
            from gpawdft_b200.workloads import gaussian_density
            rho, _ = gaussian_density(p['N'], p['L'] / p['N'] * 0.52917721, 4,
                                      rng_seed)
        ps = layer.PoissonSolver(nn=p['nn'], eps=1e-18, backend=backend)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        phi = gd.zeros()
        n = ps.solve(phi, rho)
        return {'rho': rho, 'out': phi, 'niter': np.array(n)}
    raise ValueError(kind)


def main():
    if not ref.available():
        ref.build()
    data = {}
    for i, (name, kind, p) in enumerate(cases()):
        res = run_case(kind, p, 'ref', 100 + i)
        for k, v in res.items():
            data['%s/%s' % (name, k)] = v
    np.savez_compressed(os.path.join(HERE, 'golden.npz'), **data)
    print('wrote %d arrays' % len(data))


if __name__ == '__main__':
    main()
