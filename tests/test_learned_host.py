"""CPU checks of the learned warm start's host logic and of its oracle."""
import numpy as np


def test_oracle_conv_layout():
    """oracle conv3 (weights [27][cout][cin], tap = (kd*3+kh)*3+kw, zero
    padding 1, cross-correlation) equals a direct 27-tap loop."""
    import torch
    from oracle import unet_ref
    rng = np.random.default_rng(0)
    B, cin, cout, D, H, W = 1, 3, 2, 4, 5, 6
    x = rng.standard_normal((B, cin, D, H, W))
    w = rng.standard_normal((27, cout, cin))
    out = unet_ref.conv3(torch.as_tensor(x), w).numpy()
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1), (1, 1)))
    ref = np.zeros((B, cout, D, H, W))
    for kd in range(3):
        for kh in range(3):
            for kw in range(3):
                t = (kd * 3 + kh) * 3 + kw
                sl = xp[:, :, kd:kd + D, kh:kh + H, kw:kw + W]
                ref += np.einsum('oc,bcdhw->bodhw', w[t], sl)
    assert np.abs(out - ref).max() < 1e-12


def test_oracle_network_shapes_and_grad():
    """The oracle U-Net runs forward / backward on a 16^3 batch."""
    import torch
    from oracle import unet_ref
    rng = np.random.default_rng(1)
    params = {}
    for name, cin, cout in unet_ref.CONVS:
        params[name + '.w'] = rng.standard_normal((27, cout, cin)) * 0.05
        params[name + '.b'] = np.zeros(cout)
    params['hf.w'] = rng.standard_normal(16) * 0.1
    params['hf.b'] = np.zeros(1)
    params['hc.w'] = rng.standard_normal(64) * 0.1
    params['hc.b'] = np.zeros(1)
    tp = unet_ref.torch_params(params)
    x = torch.as_tensor(rng.standard_normal((2, 16, 16, 16, 16)))
    pred = unet_ref.forward(tp, x)
    assert pred.shape == (2, 16, 16, 16)
    loss = unet_ref.loss_fn(pred, np.zeros((2, 15, 15, 15)), np.ones(2), 15)
    loss.backward()
    g = unet_ref.grads_as_flat_layout(tp)
    assert g['c31.w'].shape == (27, 64, 64)
    assert np.isfinite(g['c00.w']).all()


def test_network_layout_consistent():
    """The GPU network's layer table matches the oracle's."""
    from gpawdft_b200 import learned
    from oracle import unet_ref
    assert learned.CONVS == unet_ref.CONVS
    assert tuple(learned.LINEAR) == tuple(unet_ref.LINEAR)
