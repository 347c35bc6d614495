"""GPU tests of the learned warm start (no reference counterpart; oracle:
the float64 CPU network of oracle/unet_ref.py under torch autograd).

Tolerances: activations and activation gradients are stored in bf16 (8
significant bits), so kernel outputs are compared at 1e-2 relative (max
norm) and gradients at 3e-2 / 5e-2 relative (L2 norm per tensor).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(16, 16, 1), (16, 32, 1), (32, 16, 0), (32, 32, 1), (32, 64, 1),
         (64, 32, 0), (64, 64, 1)]


def _bf16(a):
    import torch
    return torch.as_tensor(np.asarray(a, np.float32)).to(torch.bfloat16)


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def _rel2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize('cin,cout,epi', CASES)
def test_conv_forward(cuda, cin, cout, epi):
    """bf16 tensor-core 3x3x3 convolution (+ bias, GELU) vs float64."""
    import torch
    import torch.nn.functional as F
    from gpawdft_b200 import _lib, arrays
    from oracle import unet_ref
    lib = _lib.load()
    rng = np.random.default_rng(cin + cout)
    B, D, H, W = 2, 6, 10, 20   # not multiples of the 16 x 8 x 2 block
    x = _bf16(rng.standard_normal((B, D, H, W, cin)))
    w = _bf16(rng.standard_normal((27, cout, cin)) / np.sqrt(27 * cin))
    bias = torch.as_tensor(rng.standard_normal(cout).astype(np.float32))
    xd, wd, bd = x.cuda(), w.cuda(), bias.cuda()
    out = torch.empty((B, D, H, W, cout), dtype=torch.bfloat16, device='cuda')
    z = torch.empty_like(out)
    _lib.check(lib.gpw_nn_conv3(cin, cout, epi, xd.data_ptr(), wd.data_ptr(),
                                bd.data_ptr(), None, z.data_ptr(),
                                out.data_ptr(), B, D, H, W, arrays.stream()))
    ref = unet_ref.conv3(unet_ref.ndhwc_to_ncdhw(x.float().numpy()),
                         w.float().numpy(),
                         torch.as_tensor(bias.numpy(), dtype=torch.float64))
    if epi:
        assert _rel(z.float().cpu().permute(0, 4, 1, 2, 3), ref) < 1e-2
        ref = F.gelu(ref)
    assert _rel(out.float().cpu().permute(0, 4, 1, 2, 3), ref) < 1e-2


@pytest.mark.parametrize('cin,cout,epi', CASES)
def test_conv_gradients(cuda, cin, cout, epi):
    """Data gradient (flipped-weight convolution) and weight / bias
    gradients vs torch autograd in float64."""
    import torch
    from gpawdft_b200 import _lib, arrays
    from oracle import unet_ref
    lib = _lib.load()
    rng = np.random.default_rng(7 * cin + cout)
    B, D, H, W = 2, 6, 10, 20
    x = _bf16(rng.standard_normal((B, D, H, W, cin)))
    w = _bf16(rng.standard_normal((27, cout, cin)) / np.sqrt(27 * cin))
    dz = _bf16(rng.standard_normal((B, D, H, W, cout)))
    xd, wd, dzd = x.cuda(), w.cuda(), dz.cuda()
    wt = torch.empty(27 * cin * cout, dtype=torch.bfloat16, device='cuda')
    _lib.check(lib.gpw_nn_flip_weights(cin, cout, wd.data_ptr(),
                                       wt.data_ptr(), arrays.stream()))
    dx = torch.empty((B, D, H, W, cin), dtype=torch.bfloat16, device='cuda')
    _lib.check(lib.gpw_nn_conv3(cout, cin, 0, dzd.data_ptr(), wt.data_ptr(),
                                None, None, None, dx.data_ptr(), B, D, H, W,
                                arrays.stream()))
    ns = lib.gpw_nn_wgrad_scratch(cin, cout)
    scratch = torch.empty(ns, dtype=torch.float32, device='cuda')
    dw = torch.empty((27, cout, cin), dtype=torch.float32, device='cuda')
    _lib.check(lib.gpw_nn_conv3_wgrad(cin, cout, xd.data_ptr(),
                                      dzd.data_ptr(), dw.data_ptr(),
                                      scratch.data_ptr(), ns, B, D, H, W,
                                      arrays.stream()))
    npart = lib.gpw_nn_partials()
    ps = torch.empty(npart * cout, dtype=torch.float32, device='cuda')
    db = torch.empty(cout, dtype=torch.float32, device='cuda')
    _lib.check(lib.gpw_nn_channel_sum(cout, B * D * H * W, dzd.data_ptr(),
                                      db.data_ptr(), ps.data_ptr(), ps.numel(),
                                      arrays.stream()))
    xr = unet_ref.ndhwc_to_ncdhw(x.float().numpy()).clone().requires_grad_()
    wr = unet_ref.torch_weight(w.float().numpy()).requires_grad_()
    br = torch.zeros(cout, dtype=torch.float64, requires_grad=True)
    y = unet_ref.conv3(xr, wr, br)
    y.backward(unet_ref.ndhwc_to_ncdhw(dz.float().numpy()))
    assert _rel2(dx.float().cpu().permute(0, 4, 1, 2, 3), xr.grad) < 3e-2
    wg = wr.grad.permute(2, 3, 4, 0, 1).reshape(27, cout, cin)
    assert _rel2(dw.cpu(), wg) < 1e-3      # fp32 accumulation of bf16 inputs
    assert _rel2(db.cpu(), br.grad) < 1e-3


def test_network_gradients(cuda):
    """The whole U-Net (16^3 grids, batch 2): prediction, loss and every
    parameter gradient vs CPU float64 autograd."""
    import torch
    from gpawdft_b200 import learned
    from oracle import unet_ref
    net = learned.PoissonUNet(seed=3)
    rng = np.random.default_rng(4)
    B, n, N = 2, 15, 16
    rho = torch.as_tensor(rng.standard_normal((B, n, n, n))).cuda()
    target = torch.as_tensor(rng.standard_normal((B, n, n, n))).cuda()
    x, s = net.pack(rho, N)
    tscale = torch.as_tensor(np.array([0.7, 1.3]))
    loss = float(net.loss_and_grad(x, target, tscale, n).sum().item())
    pred = net._bufs[(B, N, True)]['pred'].cpu().numpy()
    grads = net.g32.cpu().numpy()
    # oracle with the bf16-rounded conv weights the kernels use
    params = net.params()
    for name, _, _ in learned.CONVS:
        params[name + '.w'] = _bf16(params[name + '.w']).double().numpy()
    tp = unet_ref.torch_params(params)
    xin = unet_ref.ndhwc_to_ncdhw(x.float().cpu().numpy())
    pr = unet_ref.forward(tp, xin)
    lr = unet_ref.loss_fn(pr, target.cpu().numpy(), tscale.numpy(), n)
    lr.backward()
    assert _rel(pred, pr.detach().numpy()) < 3e-2
    assert abs(loss - lr.item()) < 3e-2 * lr.item()
    ref = unet_ref.grads_as_flat_layout(tp)
    for k, (off, shape) in net.layout.items():
        g = grads[off:off + int(np.prod(shape))].reshape(shape)
        if k == 'c00.w':   # only input channel 0 carries data
            g, r = g[:, :, :1], ref[k][:, :, :1]
            assert np.abs(grads[off:off + int(np.prod(shape))].reshape(
                shape)[:, :, 1:]).max() == 0.0
        else:
            r = ref[k]
        assert _rel2(g, r) < 5e-2, k


def test_training_reduces_loss(cuda):
    """A short training run on 32^3 grids lowers the loss."""
    from gpawdft_b200 import learned
    net = learned.PoissonUNet(seed=1)
    hist = learned.train(net, pairs=256, batch=4, N_c=32, lr=2e-3, seed=11,
                         log_every=16, logger=None)
    first = hist[0][1]
    last = hist[-1][1]
    assert np.isfinite(last) and last < 0.5 * first, hist


def test_warm_start_measured_and_safeguarded(cuda):
    """The trained network on held-out densities (32^3 grids, float32 defect
    correction to relative residual 1e-10): what it gives is measured here,
    not claimed.  Asserted: the network has learned the potential (held-out
    prediction error below 50%); the multigrid finishes every solve to the
    tolerance; judging each guess after one iteration bounds the cost of a
    bad guess to that iteration; and the fallback to the zero start engages
    for a guess that makes the residual grow (the prediction scaled by -50:
    one V-cycle, contracting errors by ~0.15, leaves more residual than the
    zero start had).  The network does not reduce the iteration count
    on average at this precision (its bf16 activations leave grid-scale
    noise), so no gain is asserted; the counts are printed."""
    import torch
    from gpawdft_b200 import blas, learned
    net = learned.PoissonUNet(seed=2)
    learned.train(net, pairs=1200, batch=4, N_c=32, lr=2e-3, seed=12,
                  log_every=100, logger=None)
    sampler = learned.DensitySampler(N_c=32, seed=99)   # held out
    ps = learned.make_solver(32, batch=8)
    rho = sampler.sample(8)
    eps = learned.rel_eps(rho, ps.gd.dv, 1e-10)
    phi_zero = torch.zeros_like(rho)
    n_zero = ps.solve_batch(phi_zero, rho, eps=eps)
    pred = net.predict(rho)
    d = pred - phi_zero
    err = np.sqrt(blas.vector_dots(d, d, 8) /
                  blas.vector_dots(phi_zero, phi_zero, 8))
    phi0, used, k = learned.warm_start(net, ps, rho)
    n_warm = ps.solve_batch(phi0, rho, eps=eps) + k
    assert (ps.last_errors <= eps).all()
    assert err.max() < 0.5, err
    assert (n_warm <= n_zero + 1).all(), (n_warm, n_zero)
    # a guess worse than zero is caught by the judging iteration
    good_predict = net.predict
    net.predict = lambda r, N=None: -50.0 * good_predict(r, N)
    try:
        phi_bad, used_bad, kb = learned.warm_start(net, ps, rho)
    finally:
        net.predict = good_predict
    assert not used_bad.any()
    assert float(phi_bad.abs().max().item()) == 0.0
    n_bad = ps.solve_batch(phi_bad, rho, eps=eps) + kb
    assert (n_bad == n_zero + 1).all(), (n_bad, n_zero)
    print('held-out prediction error %s; outer iterations zero start %s, '
          'warm start %s (guess kept: %s, mean change %+.2f)'
          % (np.round(err, 3), n_zero, n_warm, used,
             float(np.mean(n_warm - n_zero))))
