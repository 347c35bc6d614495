"""Build the in-tree CUDA library ``libgpwgrid.so`` for B200 (sm_100a).

``python -m gpawdft_b200.build`` (or ``build()``) compiles every ``.cu`` file
under ``csrc/`` with nvcc into ``gpawdft_b200/libgpwgrid.so``.  The CUDA
runtime is linked statically so the library does not depend on which
libcudart the host process (e.g. PyTorch) loaded; device pointers and streams
are shared through the driver's primary context.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'libgpwgrid.so')
SOURCES = ['gpw_api.cu', 'gpw_launch.cu', 'gpw_poisson.cu', 'gpw_noalloc.cu',
           'gpw_tma_f64.cu', 'gpw_tma_f32.cu', 'gpw_nn.cu',
           'gpw_bloch.cu', 'gpw_woperator.cu']


def nvcc_path():
    for cand in (shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError('nvcc not found')


STAMP = os.path.join(HERE, '_build', 'sources.mtime')


def sources_mtime():
    """Newest modification time of the library's sources and header."""
    t = 0.0
    for root, _, files in os.walk(CSRC):
        for f in files:
            t = max(t, os.path.getmtime(os.path.join(root, f)))
    hdr = os.path.join(os.path.dirname(HERE), 'include', 'gpwgrid.h')
    if os.path.exists(hdr):
        t = max(t, os.path.getmtime(hdr))
    return t


def needs_build():
    """The library is missing, or a source changed after the sources the
    last build compiled (their newest time is stamped when a build starts,
    so an edit made while nvcc runs is not missed)."""
    if not os.path.exists(LIB):
        return True
    try:
        with open(STAMP) as f:
            built = float(f.read())
    except (OSError, ValueError):
        return sources_mtime() > os.path.getmtime(LIB)
    return sources_mtime() > built


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    objs = []
    builddir = os.path.join(HERE, '_build')
    os.makedirs(builddir, exist_ok=True)
    started = sources_mtime()
    flags = ['-O3', '-std=c++17', '-gencode', 'arch=compute_100a,code=sm_100a',
             '-lineinfo', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr',
             '-I', os.path.dirname(HERE)] + list(extra)
    procs = []
    for src in SOURCES:
        obj = os.path.join(builddir, src.replace('.cu', '.o'))
        objs.append(obj)
        cmd = [nvcc_path(), '-c', os.path.join(CSRC, src), '-o', obj] + flags
        if verbose:
            print(' '.join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError('nvcc failed:\n%s\n%s' % (' '.join(cmd),
                                                         out.decode()))
        if verbose and out:
            print(out.decode())
    tmp = LIB + '.tmp'
    # export only the C ABI; everything else (incl. the static CUDA runtime)
    # binds locally so it cannot interpose with the host process's libcudart
    cmd = [nvcc_path(), '-shared', '-cudart', 'static', '-gencode',
           'arch=compute_100a,code=sm_100a', '-Xlinker',
           '--version-script=' + os.path.join(CSRC, 'exports.map'),
           '-Xlinker', '-Bsymbolic', '-o', tmp] + objs
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    with open(STAMP, 'w') as f:
        f.write(repr(started))
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True,
          extra=['-Xptxas', '-v'] if '--ptxas' in sys.argv else [])
