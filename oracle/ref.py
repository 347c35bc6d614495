"""Loader for the reference's compiled C kernels (oracle/_ref, test only).

``oracle/Makefile`` builds c/bmgs/bmgs.c, c/bc.c, c/operators.c and
c/transformers.c from the reference tree with a project-written module init
(oracle/ref_module.c).  The resulting ``_gpaw_ref`` module exposes the same two
constructors as the reference's ``_gpaw`` (c/_gpaw.c:154, :157).
"""
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, '_ref')
# the reference source tree (only where it is mounted; never on GPU boxes)
REF_TREE = os.environ.get('GPAW_REFERENCE_TREE', '/root/reference')


def available(omp=False):
    d = os.path.join(REF_DIR, 'omp') if omp else REF_DIR
    if not os.path.isdir(d):
        return False
    return any(f.startswith('_gpaw_ref') and f.endswith('.so')
               for f in os.listdir(d))


def build():
    """Compile the reference's C when its sources are mounted (not on GPU boxes)."""
    if not os.path.isdir(os.path.join(REF_TREE, 'c', 'bmgs')):
        return False
    import subprocess
    subprocess.run(['make', '-s', '-C', HERE, 'REF=' + REF_TREE,
                    'PY=' + sys.executable], check=True)
    return True


_cache = {}


def load(omp=False):
    """Import the compiled reference module (serial or GPAW_OMP build)."""
    key = bool(omp)
    if key in _cache:
        return _cache[key]
    d = os.path.join(REF_DIR, 'omp') if omp else REF_DIR
    fn = [f for f in os.listdir(d)
          if f.startswith('_gpaw_ref') and f.endswith('.so')][0]
    spec = importlib.util.spec_from_file_location('_gpaw_ref',
                                                  os.path.join(d, fn))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    _cache[key] = mod
    return mod
