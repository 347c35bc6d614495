"""NumPy restatement of the reference's C grid kernels (oracle).

Each function follows the C code it cites operation by operation, in the same
order and without fused multiply-adds, so its results are bit-identical to
the compiled reference (pinned by tests/test_oracle_pins.py).

The two classes mirror the reference's extension types exactly -- same
constructor arguments as ``_gpaw.Operator`` (c/operators.c:462-495) and
``_gpaw.Transformer`` (c/transformers.c:219-262) -- so the restated Python layer
can drive either this module or the compiled reference.

Test infrastructure only.
"""
import numpy as np

# ---------------------------------------------------------------- halo fill


def decode_offsets(offset_p, n_c, mp):
    """Linear offsets in the mp-padded array -> (P, 3) offsets.

    Inverse of gpaw/fd_operators.py:50-52 (``offset_p = offset_pc . stride``
    with stride of the array padded by ``mp`` on each face).
    """
    M = np.asarray(n_c, np.int64) + 2 * mp
    out = np.empty((len(offset_p), 3), np.int64)
    for p, o in enumerate(np.asarray(offset_p, np.int64)):
        o2 = (o + mp) % M[2] - mp
        r = (o - o2) // M[2]
        o1 = (r + mp) % M[1] - mp
        o0 = (r - o1) // M[1]
        out[p] = (o0, o1, o2)
    return out


def halo_fill(a, pad_cd, npad_cd, neighbor_cd, phases, cfd):
    """Padded copy with halos, c/bc.c:17-135 (bc_init) + :138-250 (unpack1).

    ``a``: one grid (n0, n1, n2).  Zero-fill everything, paste the interior,
    then per axis i and side d, when the neighbour is this rank (serial
    periodic axis), copy the ``npad[i][d]`` interior planes next to side d into
    the halo on the opposite side, multiplied by ``phases[i][d]`` for complex
    data (bmgs_translate / bmgs_translatemz, c/bmgs/translate.c).  With
    ``cfd == 0`` the later axes copy the full padded extent of the earlier
    axes, which fills edges and corners (c/bc.c:108-112).
    """
    n = np.array(a.shape, np.int64)
    pad = np.asarray(pad_cd, np.int64)
    npad = np.asarray(npad_cd, np.int64)
    size2 = n + pad[:, 0] + pad[:, 1]
    b = np.zeros(tuple(size2), a.dtype)
    sl = tuple(slice(pad[c, 0], pad[c, 0] + n[c]) for c in range(3))
    b[sl] = a
    real = not np.iscomplexobj(a)
    start = pad[:, 0].copy()
    size = n.copy()
    for i in range(3):
        for d in range(2):
            ds = npad[i, d]
            if neighbor_cd[i][d] != 0 or ds <= 0:
                continue            # zero boundary (neighbour -1): halo stays 0
            s0 = start.copy()
            sz = size.copy()
            s0[i] = pad[i, 0] if d == 0 else pad[i, 0] + n[i] - ds
            sz[i] = ds
            r0 = start.copy()
            r0[i] = pad[i, 0] + n[i] if d == 0 else 0
            src = tuple(slice(s0[c], s0[c] + sz[c]) for c in range(3))
            dst = tuple(slice(r0[c], r0[c] + sz[c]) for c in range(3))
            if real:
                b[dst] = b[src]
            else:
                # C99 complex product p*s = (pr sr - pi si) + i (pr si + pi sr),
                # spelled out: NumPy's own complex multiply may fuse (FMA).
                p = complex(phases[i][d])
                s = b[src]
                t = np.empty_like(s)
                t.real = p.real * s.real - p.imag * s.imag
                t.imag = p.real * s.imag + p.imag * s.real
                b[dst] = t
        if not cfd:
            start[i] = 0
            size[i] = size2[i]
    return b


# ---------------------------------------------------------------- stencils


def fd_apply_padded(coef_p, offset_pc, mp, b, n):
    """c/bmgs/fd.c:32-49: x = 0; x += a[offset_c] * coef_c, in order."""
    x = np.zeros(tuple(n), b.dtype)
    for c in range(len(coef_p)):
        o = offset_pc[c]
        sl = tuple(slice(mp + o[k], mp + o[k] + n[k]) for k in range(3))
        x += b[sl] * coef_p[c]
    return x


def relax_padded(method, coef_p, offset_pc, mp, b, f, src, w):
    """c/bmgs/relax.c:7-73 on one padded copy ``b`` of ``f`` (updated in place).

    method 2 (weighted Jacobi, :46-71): f = (1-w) f + w (src - sum')/c0.
    method 1 (lexicographic Gauss-Seidel, :11-45): in-place sweep using the
    freshly written values; pure-Python loops, small grids only.
    """
    n = f.shape
    if method == 1:
        coef = 1.0 / coef_p[0]
        for i0 in range(n[0]):
            for i1 in range(n[1]):
                for i2 in range(n[2]):
                    g = (i0 + mp, i1 + mp, i2 + mp)
                    x = 0.0
                    for c in range(1, len(coef_p)):
                        o = offset_pc[c]
                        x += b[g[0] + o[0], g[1] + o[1], g[2] + o[2]] * \
                            coef_p[c]
                    x = (src[i0, i1, i2] - x) * coef
                    f[i0, i1, i2] = x
                    b[g] = x
        return
    x = np.zeros(n, float)
    for c in range(1, len(coef_p)):
        o = offset_pc[c]
        sl = tuple(slice(mp + o[k], mp + o[k] + n[k]) for k in range(3))
        x += b[sl] * coef_p[c]
    f[:] = (1.0 - w) * f + w * (src - x) / coef_p[0]


class Operator:
    """Same construction and methods as ``_gpaw.Operator``.

    c/operators.c:462-495 (ctor "OOOiOiOi"), :316-405 (apply),
    :49-91 (relax), :408-421 (get_diagonal_element).
    """

    def __init__(self, coef_p, offset_p, n_c, mp, neighbor_cd, real, comm,
                 cfd):
        assert comm is None
        self.coef_p = np.array(coef_p, float)
        self.n_c = np.array(n_c, np.int64)
        self.mp = int(mp)
        self.offset_pc = decode_offsets(offset_p, self.n_c, self.mp)
        self.neighbor_cd = np.array(neighbor_cd).reshape(3, 2)
        self.real = bool(real)
        self.cfd = bool(cfd)
        self.pad_cd = np.full((3, 2), self.mp, np.int64)

    def _pad(self, a, phases):
        return halo_fill(a, self.pad_cd, self.pad_cd, self.neighbor_cd,
                         phases, self.cfd)

    def apply(self, input, output, phases=None):
        a = input.reshape((-1,) + tuple(self.n_c))
        o = output.reshape((-1,) + tuple(self.n_c))
        for m in range(a.shape[0]):
            b = self._pad(a[m], phases)
            o[m] = fd_apply_padded(self.coef_p, self.offset_pc, self.mp, b,
                                   self.n_c)

    def relax(self, relax_method, func, source, nrelax, w=1.0):
        for _ in range(nrelax):
            b = self._pad(func, None)
            relax_padded(relax_method, self.coef_p, self.offset_pc, self.mp,
                         b, func, source, w)

    def get_diagonal_element(self):
        d = 0.0
        for c in range(len(self.coef_p)):
            if (self.offset_pc[c] == 0).all():
                d = self.coef_p[c]
        return d


# ---------------------------------------------------------------- transformers

_RW = {2: (0.5,),
       4: (0.5625, -0.0625),
       6: (0.58593750, -0.09765625, 0.01171875),
       8: (0.59814453125, -0.11962890625, 0.02392578125, -0.00244140625)}


def restrict_1d(a, K):
    """c/bmgs/restrict.c:18-63 along the last axis of ``a``.

    Output i = 0.5 * (a[c] + w1 (a[c+1] + a[c-1]) + w3 (a[c+3] + a[c-3]) ...)
    with c = K - 1 + 2 i, summed left to right.
    """
    L = a.shape[-1]
    n = (L - (2 * K - 3)) // 2
    c = K - 1 + 2 * np.arange(n)
    w = _RW[K]
    s = a[..., c]
    if K == 2:
        return 0.5 * (s + 0.5 * (a[..., c + 1] + a[..., c - 1]))
    for j, wj in enumerate(w):
        t = wj * (a[..., c + 2 * j + 1] + a[..., c - 2 * j - 1])
        s = s + t
    return 0.5 * s


def interpolate_1d(a, K, skip):
    """c/bmgs/interpolate.c:19-64 along the last axis of ``a``.

    For i < n: even output 2i - skip0 copies a[b+i]; odd output 2i+1 - skip0
    is the K-tap midpoint value; skip[0] drops the first even output and
    skip[1] the last odd one.  b = K/2 - 1, n = L - (K-1) + skip[1].
    """
    L = a.shape[-1]
    n = L - (K - 1) + skip[1]
    base = K // 2 - 1
    nout = 2 * n - skip[0] - skip[1]
    out = np.empty(a.shape[:-1] + (nout,), a.dtype)
    i = np.arange(n)
    ev = i[1:] if skip[0] else i
    out[..., 2 * ev - skip[0]] = a[..., base + ev]
    od = i[:-1] if skip[1] else i
    p = base + od
    w = _RW[K]
    if K == 2:
        val = 0.5 * (a[..., p] + a[..., p + 1])
    else:
        val = w[0] * (a[..., p] + a[..., p + 1])
        for j in range(1, len(w)):
            val = val + w[j] * (a[..., p - j] + a[..., p + 1 + j])
    out[..., 2 * od + 1 - skip[0]] = val
    return out


def _along(fn, a, axis, *args):
    return np.moveaxis(fn(np.moveaxis(a, axis, -1), *args), -1, axis)


class Transformer:
    """Same construction and apply as ``_gpaw.Transformer``.

    c/transformers.c:219-262 (ctor "OOiOOOOiOi"), :54-123 (apply worker):
    halo fill with (pad, npad) and cfd = 0, then restriction
    (c/bmgs/restrict.c:137-154: passes over axis 2, 1, 0) or interpolation
    (c/bmgs/interpolate.c:141-168: same pass order).
    """

    def __init__(self, size_in, size_out, k, pad_cd, npad_cd, skip_cd,
                 neighbor_cd, real, comm, interpolate):
        assert comm is None
        self.size_in = np.array(size_in, np.int64)
        self.size_out = np.array(size_out, np.int64)
        self.k = int(k)
        self.pad_cd = np.array(pad_cd, np.int64).reshape(3, 2)
        self.npad_cd = np.array(npad_cd, np.int64).reshape(3, 2)
        self.skip_cd = np.array(skip_cd, np.int64).reshape(3, 2)
        self.neighbor_cd = np.array(neighbor_cd).reshape(3, 2)
        self.real = bool(real)
        self.interpolate = bool(interpolate)

    def apply(self, input, output, phases=None):
        a = input.reshape((-1,) + tuple(self.size_in))
        o = output.reshape((-1,) + tuple(self.size_out))
        for m in range(a.shape[0]):
            b = halo_fill(a[m], self.pad_cd, self.npad_cd, self.neighbor_cd,
                          phases, False)
            for axis in (2, 1, 0):
                if self.interpolate:
                    b = _along(interpolate_1d, b, axis, self.k,
                               tuple(self.skip_cd[axis]))
                else:
                    b = _along(restrict_1d, b, axis, self.k)
            o[m] = b
