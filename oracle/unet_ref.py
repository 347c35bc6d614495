"""CPU float64 oracle of the learned warm start's U-Net (test infrastructure
only: the GPU kernels' gradients are checked against torch CPU autograd).

Mirrors gpawdft_b200/learned.py layer by layer in NCDHW float64: 3x3x3
convolutions with zero padding 1 (weights given as [27][cout][cin], tap =
(kd * 3 + kh) * 3 + kw), GELU (erf form), 2x2x2 average pooling, nearest
upsampling, the 1x1x1 heads, pred = head_f(a02) + up8(head_c(a31)) and the
mean squared error on the n^3 interior.  The reference (GPAW) has no
network; this oracle is the definition the kernels are tested against.
"""
import numpy as np
import torch
import torch.nn.functional as F

CONVS = [('c00', 16, 16), ('c01', 16, 16), ('c10', 16, 32), ('c11', 32, 32),
         ('c20', 32, 64), ('c30', 64, 64), ('c31', 64, 64), ('c21', 64, 64),
         ('c22', 64, 32), ('c12', 32, 32), ('c13', 32, 16), ('c02', 16, 16)]
LINEAR = ('c22', 'c13')


def torch_weight(w):
    """[27][cout][cin] -> torch conv3d layout (cout, cin, 3, 3, 3)."""
    w = torch.as_tensor(np.asarray(w, np.float64))
    cout, cin = w.shape[1], w.shape[2]
    return w.reshape(3, 3, 3, cout, cin).permute(3, 4, 0, 1, 2).contiguous()


def conv3(x, w, b=None):
    """x (B, cin, D, H, W); w [27][cout][cin] (numpy or tensor)."""
    wt = w if isinstance(w, torch.Tensor) and w.dim() == 5 else torch_weight(w)
    return F.conv3d(x, wt, b, padding=1)


def ndhwc_to_ncdhw(a):
    return torch.as_tensor(np.asarray(a, np.float64)).permute(0, 4, 1, 2, 3)


def up(x, f=2):
    return x.repeat_interleave(f, 2).repeat_interleave(f, 3).repeat_interleave(
        f, 4)


def forward(params, x):
    """params: dict name -> float64 tensors (requires_grad as needed);
    x: (B, 16, N, N, N).  Returns pred (B, N, N, N)."""
    def c(name, inp):
        z = F.conv3d(inp, params[name + '.w'], params[name + '.b'], padding=1)
        return z if name in LINEAR else F.gelu(z)
    a00 = c('c00', x)
    a01 = c('c01', a00)
    a10 = c('c10', F.avg_pool3d(a01, 2))
    a11 = c('c11', a10)
    a20 = c('c20', F.avg_pool3d(a11, 2))
    a30 = c('c30', F.avg_pool3d(a20, 2))
    a31 = c('c31', a30)
    a21 = c('c21', up(a31) + a20)
    c2 = c('c22', a21)
    a12 = c('c12', up(c2) + a11)
    c1 = c('c13', a12)
    a02 = c('c02', up(c1) + a01)
    pf = (a02 * params['hf.w'].view(1, -1, 1, 1, 1)).sum(1) + params['hf.b']
    pc = (a31 * params['hc.w'].view(1, -1, 1, 1, 1)).sum(1) + params['hc.b']
    return pf + up(pc.unsqueeze(1), 8).squeeze(1)


def torch_params(flat_params, requires_grad=True):
    """learned.PoissonUNet.params() (numpy, conv weights [27][cout][cin]) ->
    float64 torch tensors in conv3d layout."""
    out = {}
    for k, v in flat_params.items():
        t = torch_weight(v) if k.endswith('.w') and v.ndim == 3 else \
            torch.as_tensor(np.asarray(v, np.float64))
        out[k] = t.clone().requires_grad_(requires_grad)
    return out


def grads_as_flat_layout(params):
    """Gradients back in the network's layout ([27][cout][cin] for convs)."""
    out = {}
    for k, t in params.items():
        g = t.grad.detach()
        if k.endswith('.w') and g.dim() == 5:
            g = g.permute(2, 3, 4, 0, 1).reshape(27, g.shape[0], g.shape[1])
        out[k] = g.numpy()
    return out


def loss_fn(pred, target, tscale, n):
    """mean over b and the n^3 interior of (pred - target * tscale)^2."""
    B = pred.shape[0]
    diff = pred[:, :n, :n, :n] - torch.as_tensor(target) * torch.as_tensor(
        tscale).view(B, 1, 1, 1)
    return (diff ** 2).mean()
