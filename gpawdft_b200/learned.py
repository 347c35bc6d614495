"""Learned warm start for the multigrid Poisson solver (no reference
counterpart).

A small 3D convolutional U-Net maps a density rho (one grid of the
zero-boundary N_c = 128 problem, 127^3 points, zero-padded to 128^3) to an
initial potential for the float32 defect-correction solve; the plain
multigrid always finishes the solve to the requested residual and judges
the guess (a member whose residual after the first multigrid iteration is
larger than the zero start's initial residual falls back to phi = 0).

Architecture (channels 16 / 32 / 64 / 64 on the 128^3 / 64^3 / 32^3 / 16^3
levels; every convolution 3x3x3 with bias, GELU unless marked linear; pool =
2x2x2 average; up = nearest 2x upsampling):

    x   = [rho * s, 0 x 15]                  s = 1 / rms(rho)
    a00 = c00(x)      a01 = c01(a00)                       128^3 x 16
    a10 = c10(pool a01)   a11 = c11(a10)                    64^3 x 32
    a20 = c20(pool a11)                                      32^3 x 64
    a30 = c30(pool a20)   a31 = c31(a30)                     16^3 x 64
    a21 = c21(up a31 + a20)   c2 = c22(a21) (linear)         32^3
    a12 = c12(up c2 + a11)    c1 = c13(a12) (linear)         64^3
    a02 = c02(up c1 + a01)                                  128^3
    pred = head_f(a02) + up8(head_c(a31))

head_c on the 16^3 bottleneck is the level-3 coarse correction (the
multigrid's level 3 is the 15^3 grid); it is upsampled and added to the fine
head.  The network predicts phi * s / K (K: the training set's mean
rms(phi) / rms(rho)); the potential is pred * K / s.

Every kernel (bf16 tensor-core convolutions with fp32 accumulation, their
data / weight gradients, GELU, pooling, upsampling, heads, loss, Adam, the
training densities) is in libgpwgrid.so (gpw_nn_*); PyTorch holds the device
buffers.  Training data: densities generated on the device (sums of neutral
Gaussians), potentials from this package's float32 multigrid solver.
"""
import ctypes
import time

import numpy as np

from . import _lib, arrays, blas

CONVS = [('c00', 16, 16), ('c01', 16, 16), ('c10', 16, 32), ('c11', 32, 32),
         ('c20', 32, 64), ('c30', 64, 64), ('c31', 64, 64), ('c21', 64, 64),
         ('c22', 64, 32), ('c12', 32, 32), ('c13', 32, 16), ('c02', 16, 16)]
LINEAR = ('c22', 'c13')
HEADS = [('hf', 16), ('hc', 64)]
BOHR_PER_ANGSTROM = 1.0 / 0.52917721


def _chk(rc):
    _lib.check(rc)


class PoissonUNet:
    """The U-Net's parameters (fp32 master, bf16 copies), Adam state and
    per-shape activation buffers on the current CUDA device."""

    def __init__(self, seed=0):
        import torch
        arrays.require_cuda()
        self.lib = _lib.load()
        self.torch = torch
        # flat parameter layout
        self.layout = {}
        off = 0
        for name, cin, cout in CONVS:
            self.layout[name + '.w'] = (off, (27, cout, cin))
            off += 27 * cout * cin
            self.layout[name + '.b'] = (off, (cout,))
            off += cout
        for name, c in HEADS:
            self.layout[name + '.w'] = (off, (c,))
            off += c
            self.layout[name + '.b'] = (off, (1,))
            off += 1
        # keep every tensor 16-byte aligned in the bf16 copy
        self.nparam = off
        self.p32 = torch.zeros(off, dtype=torch.float32, device='cuda')
        self.g32 = torch.zeros_like(self.p32)
        self.m = torch.zeros_like(self.p32)
        self.v = torch.zeros_like(self.p32)
        self.p16 = torch.zeros(off, dtype=torch.bfloat16, device='cuda')
        self.K = 1.0
        self.step_count = 0
        self.init_params(seed)
        self._bufs = {}
        self._wt = {}

    # ------------------------------------------------------------ parameters
    def init_params(self, seed):
        """He-style initialisation (fan-in 27 cin); the input conv sees only
        channel 0, its other input channels start (and stay) at zero."""
        rng = np.random.default_rng(seed)
        p = np.zeros(self.nparam, np.float32)
        for name, cin, cout in CONVS:
            off, shape = self.layout[name + '.w']
            std = np.sqrt(2.0 / (27 * (1 if name == 'c00' else cin)))
            if name in LINEAR:
                std = np.sqrt(1.0 / (27 * cin))
            w = rng.standard_normal(shape).astype(np.float32) * std
            if name == 'c00':
                w[:, :, 1:] = 0.0
            p[off:off + w.size] = w.ravel()
        for name, c in HEADS:
            off, shape = self.layout[name + '.w']
            p[off:off + c] = rng.standard_normal(c) * np.sqrt(1.0 / c) * 0.1
        self.set_flat(p)

    def set_flat(self, p):
        self.p32.copy_(self.torch.from_numpy(np.asarray(p, np.float32)))
        self.p16.copy_(self.p32.to(self.torch.bfloat16))
        self._wt = {}

    def get_flat(self):
        return self.p32.cpu().numpy()

    def params(self):
        """Dict of fp32 parameter arrays (host copies)."""
        flat = self.get_flat()
        return {k: flat[o:o + int(np.prod(s))].reshape(s)
                for k, (o, s) in self.layout.items()}

    def save(self, path):
        np.savez(path, flat=self.get_flat(), K=self.K, step=self.step_count)

    def load(self, path):
        z = np.load(path)
        self.set_flat(z['flat'])
        self.K = float(z['K'])
        self.step_count = int(z['step'])

    def _ptr(self, t, key):
        off, _ = self.layout[key]
        return t.data_ptr() + off * t.element_size()

    def _flipped(self, name, cin, cout):
        """bf16 weights of the data gradient (taps flipped, cin / cout
        swapped), recomputed after each optimiser step."""
        t = self._wt.get(name)
        if t is None:
            t = self.torch.empty(27 * cin * cout, dtype=self.torch.bfloat16,
                                 device='cuda')
            _chk(self.lib.gpw_nn_flip_weights(cin, cout,
                                              self._ptr(self.p16, name + '.w'),
                                              t.data_ptr(), arrays.stream()))
            self._wt[name] = t
        return t

    # ------------------------------------------------------------ buffers
    def _buffers(self, B, N, training):
        key = (B, N, training)
        if key in self._bufs:
            return self._bufs[key]
        torch = self.torch
        bf = torch.bfloat16
        n1, n2, n3 = N // 2, N // 4, N // 8

        def t(n, c):
            return torch.empty((B, n, n, n, c), dtype=bf, device='cuda')
        b = {'x': t(N, 16), 'a00': t(N, 16), 'a01': t(N, 16),
             'p1': t(n1, 16), 'a10': t(n1, 32), 'a11': t(n1, 32),
             'p2': t(n2, 32), 'a20': t(n2, 64), 'p3': t(n3, 64),
             'a30': t(n3, 64), 'a31': t(n3, 64), 'u2': t(n2, 64),
             'a21': t(n2, 64), 'c2': t(n2, 32), 'u1': t(n1, 32),
             'a12': t(n1, 32), 'c1': t(n1, 16), 'u0': t(N, 16),
             'a02': t(N, 16),
             'pred': torch.empty((B, N, N, N), dtype=torch.float32,
                                 device='cuda'),
             'pc': torch.empty((B, n3, n3, n3), dtype=torch.float32,
                               device='cuda'),
             'scale': torch.empty(B, dtype=torch.float64, device='cuda')}
        if training:
            for k in ('00', '01', '10', '11', '20', '30', '31', '21', '12',
                      '02'):
                b['z' + k] = torch.empty_like(b['a' + k])
            # gradients
            b.update({'da02': t(N, 16), 'dz02': t(N, 16), 'du0': t(N, 16),
                      'dc1': t(n1, 16), 'da12': t(n1, 32), 'dz12': t(n1, 32),
                      'du1': t(n1, 32), 'dc2': t(n2, 32), 'da21': t(n2, 64),
                      'dz21': t(n2, 64), 'du2': t(n2, 64), 'da31': t(n3, 64),
                      'dz31': t(n3, 64), 'da30': t(n3, 64), 'dz30': t(n3, 64),
                      'dp3': t(n3, 64), 'dz20': t(n2, 64), 'dp2': t(n2, 32),
                      'dz11': t(n1, 32), 'da10': t(n1, 32), 'dz10': t(n1, 32),
                      'dp1': t(n1, 16), 'dz01': t(N, 16), 'da00': t(N, 16),
                      'dz00': t(N, 16),
                      'dpred': torch.empty((B, N, N, N), dtype=torch.float32,
                                           device='cuda'),
                      'dpc': torch.empty((B, n3, n3, n3), dtype=torch.float32,
                                         device='cuda'),
                      'tscale': torch.empty(B, dtype=torch.float64,
                                            device='cuda')})
            ws = max(self.lib.gpw_nn_wgrad_scratch(ci, co)
                     for _, ci, co in CONVS)
            b['wscratch'] = torch.empty(ws, dtype=torch.float32, device='cuda')
            npart = self.lib.gpw_nn_partials()
            b['pscratch'] = torch.empty(npart * 65, dtype=torch.float32,
                                        device='cuda')
            b['loss'] = torch.empty(npart, dtype=torch.float64, device='cuda')
        self._bufs[key] = b
        return b

    # ------------------------------------------------------------ layers
    def _conv(self, name, x, out, B, n, z=None, add=None):
        cin, cout = [(ci, co) for nm, ci, co in CONVS if nm == name][0]
        epi = 0 if name in LINEAR else 1
        _chk(self.lib.gpw_nn_conv3(
            cin, cout, epi, x.data_ptr(), self._ptr(self.p16, name + '.w'),
            self._ptr(self.p32, name + '.b'),
            add.data_ptr() if add is not None else None,
            z.data_ptr() if z is not None else None, out.data_ptr(), B, n, n,
            n, arrays.stream()))

    def _dgrad(self, name, dz, dx, B, n):
        cin, cout = [(ci, co) for nm, ci, co in CONVS if nm == name][0]
        wt = self._flipped(name, cin, cout)
        _chk(self.lib.gpw_nn_conv3(cout, cin, 0, dz.data_ptr(), wt.data_ptr(),
                                   None, None, None, dx.data_ptr(), B, n, n, n,
                                   arrays.stream()))

    def _wgrad(self, name, x, dz, B, n, bufs):
        cin, cout = [(ci, co) for nm, ci, co in CONVS if nm == name][0]
        ws = bufs['wscratch']
        _chk(self.lib.gpw_nn_conv3_wgrad(
            cin, cout, x.data_ptr(), dz.data_ptr(),
            self._ptr(self.g32, name + '.w'), ws.data_ptr(), ws.numel(), B, n,
            n, n, arrays.stream()))
        ps = bufs['pscratch']
        _chk(self.lib.gpw_nn_channel_sum(
            cout, B * n ** 3, dz.data_ptr(), self._ptr(self.g32, name + '.b'),
            ps.data_ptr(), ps.numel(), arrays.stream()))

    def _gelu_b(self, z, da, dz):
        _chk(self.lib.gpw_nn_gelu_backward(z.numel(), z.data_ptr(),
                                           da.data_ptr(), dz.data_ptr(),
                                           arrays.stream()))

    def _pool(self, c, x, y, B, n):
        _chk(self.lib.gpw_nn_pool2(c, x.data_ptr(), y.data_ptr(), B, n, n, n,
                                   arrays.stream()))

    def _pool_b(self, c, dy, dx, B, n, acc):
        _chk(self.lib.gpw_nn_pool2_backward(c, dy.data_ptr(), dx.data_ptr(), B,
                                            n, n, n, int(acc),
                                            arrays.stream()))

    def _up(self, c, x, skip, y, B, n):
        _chk(self.lib.gpw_nn_upsample2_add(c, x.data_ptr(), skip.data_ptr(),
                                           y.data_ptr(), B, n, n, n,
                                           arrays.stream()))

    def _up_b(self, c, dy, dx, B, n, acc):
        _chk(self.lib.gpw_nn_upsample2_backward(c, dy.data_ptr(),
                                                dx.data_ptr(), B, n, n, n,
                                                int(acc), arrays.stream()))

    # ------------------------------------------------------------ passes
    def forward_input(self, x, training=False):
        """Run the network on packed inputs x (B, N, N, N, 16) bf16 already
        in the buffer set; returns the buffer dict (pred = the output)."""
        B, N = x.shape[0], x.shape[1]
        b = self._buffers(B, N, training)
        if x.data_ptr() != b['x'].data_ptr():
            b['x'].copy_(x)
        self._forward(b, B, N, training)
        return b

    def _forward(self, b, B, N, training):
        n1, n2, n3 = N // 2, N // 4, N // 8
        z = (lambda k: b['z' + k]) if training else (lambda k: None)
        self._conv('c00', b['x'], b['a00'], B, N, z('00'))
        self._conv('c01', b['a00'], b['a01'], B, N, z('01'))
        self._pool(16, b['a01'], b['p1'], B, N)
        self._conv('c10', b['p1'], b['a10'], B, n1, z('10'))
        self._conv('c11', b['a10'], b['a11'], B, n1, z('11'))
        self._pool(32, b['a11'], b['p2'], B, n1)
        self._conv('c20', b['p2'], b['a20'], B, n2, z('20'))
        self._pool(64, b['a20'], b['p3'], B, n2)
        self._conv('c30', b['p3'], b['a30'], B, n3, z('30'))
        self._conv('c31', b['a30'], b['a31'], B, n3, z('31'))
        self._up(64, b['a31'], b['a20'], b['u2'], B, n2)
        self._conv('c21', b['u2'], b['a21'], B, n2, z('21'))
        self._conv('c22', b['a21'], b['c2'], B, n2)
        self._up(32, b['c2'], b['a11'], b['u1'], B, n1)
        self._conv('c12', b['u1'], b['a12'], B, n1, z('12'))
        self._conv('c13', b['a12'], b['c1'], B, n1)
        self._up(16, b['c1'], b['a01'], b['u0'], B, N)
        self._conv('c02', b['u0'], b['a02'], B, N, z('02'))
        lib, st = self.lib, arrays.stream()
        _chk(lib.gpw_nn_head(16, B * N ** 3, b['a02'].data_ptr(),
                             self._ptr(self.p32, 'hf.w'),
                             self._ptr(self.p32, 'hf.b'), b['pred'].data_ptr(),
                             st))
        _chk(lib.gpw_nn_head(64, B * n3 ** 3, b['a31'].data_ptr(),
                             self._ptr(self.p32, 'hc.w'),
                             self._ptr(self.p32, 'hc.b'), b['pc'].data_ptr(),
                             st))
        _chk(lib.gpw_nn_upsample_add_f32(8, b['pc'].data_ptr(),
                                         b['pred'].data_ptr(), B, N, st))

    def _backward(self, b, B, N):
        """Gradients of the loss (dpred in b) into self.g32."""
        n1, n2, n3 = N // 2, N // 4, N // 8
        lib, st = self.lib, arrays.stream()
        ps = b['pscratch']
        _chk(lib.gpw_nn_downsum_f32(8, b['dpred'].data_ptr(),
                                    b['dpc'].data_ptr(), B, N, st))
        _chk(lib.gpw_nn_head_backward(
            64, B * n3 ** 3, b['a31'].data_ptr(), self._ptr(self.p32, 'hc.w'),
            b['dpc'].data_ptr(), b['da31'].data_ptr(), 0,
            self._ptr(self.g32, 'hc.w'), ps.data_ptr(), ps.numel(), st))
        _chk(lib.gpw_nn_head_backward(
            16, B * N ** 3, b['a02'].data_ptr(), self._ptr(self.p32, 'hf.w'),
            b['dpred'].data_ptr(), b['da02'].data_ptr(), 0,
            self._ptr(self.g32, 'hf.w'), ps.data_ptr(), ps.numel(), st))
        # (hf.w then hf.b are adjacent in the layout: dwb = (dw, dbias))
        self._gelu_b(b['z02'], b['da02'], b['dz02'])
        self._wgrad('c02', b['u0'], b['dz02'], B, N, b)
        self._dgrad('c02', b['dz02'], b['du0'], B, N)
        self._up_b(16, b['du0'], b['dc1'], B, N, False)
        self._wgrad('c13', b['a12'], b['dc1'], B, n1, b)
        self._dgrad('c13', b['dc1'], b['da12'], B, n1)
        self._gelu_b(b['z12'], b['da12'], b['dz12'])
        self._wgrad('c12', b['u1'], b['dz12'], B, n1, b)
        self._dgrad('c12', b['dz12'], b['du1'], B, n1)
        self._up_b(32, b['du1'], b['dc2'], B, n1, False)
        self._wgrad('c22', b['a21'], b['dc2'], B, n2, b)
        self._dgrad('c22', b['dc2'], b['da21'], B, n2)
        self._gelu_b(b['z21'], b['da21'], b['dz21'])
        self._wgrad('c21', b['u2'], b['dz21'], B, n2, b)
        self._dgrad('c21', b['dz21'], b['du2'], B, n2)
        self._up_b(64, b['du2'], b['da31'], B, n2, True)
        self._gelu_b(b['z31'], b['da31'], b['dz31'])
        self._wgrad('c31', b['a30'], b['dz31'], B, n3, b)
        self._dgrad('c31', b['dz31'], b['da30'], B, n3)
        self._gelu_b(b['z30'], b['da30'], b['dz30'])
        self._wgrad('c30', b['p3'], b['dz30'], B, n3, b)
        self._dgrad('c30', b['dz30'], b['dp3'], B, n3)
        self._pool_b(64, b['dp3'], b['du2'], B, n2, True)   # du2 = da20
        self._gelu_b(b['z20'], b['du2'], b['dz20'])
        self._wgrad('c20', b['p2'], b['dz20'], B, n2, b)
        self._dgrad('c20', b['dz20'], b['dp2'], B, n2)
        self._pool_b(32, b['dp2'], b['du1'], B, n1, True)   # du1 = da11
        self._gelu_b(b['z11'], b['du1'], b['dz11'])
        self._wgrad('c11', b['a10'], b['dz11'], B, n1, b)
        self._dgrad('c11', b['dz11'], b['da10'], B, n1)
        self._gelu_b(b['z10'], b['da10'], b['dz10'])
        self._wgrad('c10', b['p1'], b['dz10'], B, n1, b)
        self._dgrad('c10', b['dz10'], b['dp1'], B, n1)
        self._pool_b(16, b['dp1'], b['du0'], B, N, True)    # du0 = da01
        self._gelu_b(b['z01'], b['du0'], b['dz01'])
        self._wgrad('c01', b['a00'], b['dz01'], B, N, b)
        self._dgrad('c01', b['dz01'], b['da00'], B, N)
        self._gelu_b(b['z00'], b['da00'], b['dz00'])
        self._wgrad('c00', b['x'], b['dz00'], B, N, b)

    def loss_and_grad(self, x, target, tscale, n):
        """Forward + backward on packed inputs x (B, N, N, N, 16) against
        float64 targets (B, n, n, n) scaled by tscale (B,): returns the
        loss; gradients in self.g32."""
        B, N = x.shape[0], x.shape[1]
        b = self.forward_input(x, training=True)
        b['tscale'].copy_(tscale)
        _chk(self.lib.gpw_nn_mse(b['pred'].data_ptr(), target.data_ptr(),
                                 b['tscale'].data_ptr(), B, n, N,
                                 b['dpred'].data_ptr(), b['loss'].data_ptr(),
                                 b['loss'].numel(), arrays.stream()))
        self._backward(b, B, N)
        return b['loss']

    def adam_step(self, lr, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        _chk(self.lib.gpw_nn_adam(self.nparam, self.p32.data_ptr(),
                                  self.g32.data_ptr(), self.m.data_ptr(),
                                  self.v.data_ptr(), lr, b1, b2, eps,
                                  self.step_count, self.p16.data_ptr(),
                                  arrays.stream()))
        self._wt = {}

    # ------------------------------------------------------------ solver glue
    def pack(self, rho, N, B=None):
        """Packed network input for densities rho (B, n, n, n) float64 on
        the device: returns (x buffer, per-member scale 1/rms(rho))."""
        B = rho.shape[0]
        n = rho.shape[1]
        sums = blas.vector_dots(rho, rho, B)
        rms = np.sqrt(sums / n ** 3)
        s = 1.0 / np.where(rms > 0, rms, 1.0)
        b = self._buffers(B, N, False)
        b['scale'].copy_(self.torch.from_numpy(s))
        _chk(self.lib.gpw_nn_pack_input(rho.data_ptr(), b['scale'].data_ptr(),
                                        B, n, N, b['x'].data_ptr(),
                                        arrays.stream()))
        return b['x'], s

    def predict(self, rho, N=None):
        """Initial potentials (B, n, n, n) float64 on the device."""
        torch = self.torch
        B, n = rho.shape[0], rho.shape[1]
        N = N or _padded(n)
        x, s = self.pack(rho, N)
        b = self.forward_input(x, training=False)
        out = torch.empty_like(rho)
        b['scale'].copy_(torch.from_numpy(self.K / s))
        _chk(self.lib.gpw_nn_unpack_output(b['pred'].data_ptr(),
                                           b['scale'].data_ptr(), B, n, N,
                                           out.data_ptr(), arrays.stream()))
        return out


def _padded(n):
    return int(np.ceil(n / 8.0) * 8)


# ---------------------------------------------------------------- data
class DensitySampler:
    """Seeded random neutral Gaussian-sum densities generated on the device
    (widths log-uniform in [0.3, 2.0] A, 8-64 Gaussians, centres uniform in
    the cell, charges N(0, 1) re-centred to a neutral density), on the
    zero-boundary grid with N_c points per axis and spacing h_ang."""

    def __init__(self, N_c=128, h_ang=0.2, ngauss=(8, 64),
                 sigma_ang=(0.3, 2.0), seed=6):
        self.N_c = N_c
        self.n = N_c - 1
        self.h = h_ang * BOHR_PER_ANGSTROM
        self.L = N_c * self.h
        self.ng = ngauss
        self.sig = (sigma_ang[0] * BOHR_PER_ANGSTROM,
                    sigma_ang[1] * BOHR_PER_ANGSTROM)
        self.rng = np.random.default_rng(seed)
        self.lib = _lib.load()

    def sample(self, B):
        import torch
        maxg = self.ng[1]
        counts = self.rng.integers(self.ng[0], self.ng[1] + 1, B).astype(
            np.int32)
        params = np.zeros((B, maxg, 5))
        for b in range(B):
            k = counts[b]
            params[b, :k, :3] = self.rng.uniform(0.0, self.L, (k, 3))
            params[b, :k, 3] = np.exp(self.rng.uniform(np.log(self.sig[0]),
                                                       np.log(self.sig[1]),
                                                       k))
            params[b, :k, 4] = self.rng.standard_normal(k)
        n = self.n
        rho = torch.empty((B, n, n, n), dtype=torch.float64, device='cuda')
        c = torch.from_numpy(counts).cuda()
        p = torch.from_numpy(params).cuda()
        _chk(self.lib.gpw_nn_gaussians(B, n, self.h, 1.0, maxg, c.data_ptr(),
                                       p.data_ptr(), rho.data_ptr(),
                                       arrays.stream()))
        # re-centre to a neutral density (sum rho dv = 0 exactly)
        sums = blas.vector_sums(rho, B)
        for b in range(B):
            blas.add_scalar(rho[b], -sums[b] / n ** 3)
        return rho


def make_solver(N_c=128, h_ang=0.2, batch=1, precision='fp32', maxiter=1000):
    from .grid_descriptor import GridDescriptor
    from .poisson import PoissonSolver
    h = h_ang * BOHR_PER_ANGSTROM
    gd = GridDescriptor((N_c,) * 3, (N_c * h,) * 3, 0)
    ps = PoissonSolver(nn=3, relax='J', maxiter=maxiter, precision=precision,
                       batch=batch)
    ps.set_grid_descriptor(gd)
    ps.initialize()
    return ps


def rel_eps(rho, dv, rel):
    """Per-member eps of the reference's test sum(r^2) dv <= eps that means
    ||A phi - rho|| / ||rho|| <= rel."""
    sums = blas.vector_dots(rho, rho, rho.shape[0])
    return rel ** 2 * sums * dv


def train(net, pairs=20000, batch=4, N_c=128, lr=1e-3, seed=6,
          target_rel=1e-6, log_every=100, time_limit=None, logger=print):
    """Train on `pairs` fresh (density, potential) pairs: densities from
    DensitySampler, potentials from the float32 multigrid solver to relative
    residual `target_rel`.  Cosine learning-rate decay.  Returns a history
    of (pairs seen, mean loss)."""
    torch = net.torch
    sampler = DensitySampler(N_c=N_c, seed=seed)
    ps = make_solver(N_c, batch=batch)
    n = N_c - 1
    N = _padded(n)
    steps = max(1, pairs // batch)
    hist, acc, cnt = [], 0.0, 0
    t0 = time.time()
    for step in range(steps):
        rho = sampler.sample(batch)
        phi = torch.zeros_like(rho)
        ps.solve_batch(phi, rho, eps=rel_eps(rho, ps.gd.dv, target_rel))
        x, s = net.pack(rho, N)
        if net.step_count == 0 and step == 0:
            # K: the data's rms(phi) / rms(rho)
            r = np.sqrt(blas.vector_dots(phi, phi, batch) / n ** 3)
            net.K = float(np.mean(r * s))
        tscale = torch.from_numpy(s / net.K)
        loss = net.loss_and_grad(x, phi, tscale, n)
        frac = step / steps
        net.adam_step(lr * 0.5 * (1 + np.cos(np.pi * frac)))
        acc += float(loss.sum().item()) if (step + 1) % 10 == 0 or \
            step == steps - 1 else 0.0
        cnt += 1 if (step + 1) % 10 == 0 or step == steps - 1 else 0
        if (step + 1) % log_every == 0 or step == steps - 1:
            hist.append(((step + 1) * batch, acc / max(cnt, 1)))
            if logger:
                logger('pairs %6d  loss %.4e  %.1fs' % ((step + 1) * batch,
                                                        acc / max(cnt, 1),
                                                        time.time() - t0))
            acc, cnt = 0.0, 0
        if time_limit and time.time() - t0 > time_limit:
            hist.append(((step + 1) * batch, float('nan')))
            break
    torch.cuda.synchronize()
    return hist


def warm_start(net, ps, rho, judge=True):
    """Initial potentials for the batch rho (device, (B, n, n, n) float64)
    from the network, judged by the plain multigrid: one outer iteration is
    run from the guess, and a member whose error sum(r^2) dv after it is
    larger than the zero start's initial error (sum(rho^2) dv: the residual
    grew) falls back to phi = 0.  Returns (phi, used, k): the potentials to
    continue from (after the judging iteration where the guess was kept),
    the members that kept it, and the iterations already spent (1, or 0
    without judging)."""
    phi = net.predict(rho)
    B = rho.shape[0]
    if not judge:
        return phi, np.ones(B, bool), 0
    err1 = ps.iterate_batch(phi, rho, 1)
    err0 = blas.vector_dots(rho, rho, B) * ps.gd.dv
    used = err1 <= err0
    for b in np.nonzero(~used)[0]:
        phi[b].zero_()
    return phi, used, 1
