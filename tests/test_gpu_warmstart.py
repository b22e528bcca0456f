"""GPU tests of the learned warm start: the tensor-core convolutions (forward, input gradient, weight gradient)
against the float64 oracle of the convolution (oracle/conv_oracle.py) on BF16 inputs, the autograd wrapper's
gradients against the same oracle, and a small end-to-end run: a U-Net trained on steady states of small obstacle
channels makes the steady solves of held-out channels faster, and they converge to the fields of the cold solves.

Tolerances: the forward output is rounded to BF16 (relative 2^-9 per element), so 1e-2 of the largest output; the
weight gradient accumulates exact BF16 products in FP32, so 1e-4 of the largest entry."""
import numpy as np
import pytest
import torch

from lbm_b200 import warmstart as ws
import conv_oracle

pytestmark = pytest.mark.gpu


def bf16(a):
    return torch.as_tensor(a, dtype=torch.float32).to(torch.bfloat16)


def volume(a):
    """(n, d, h, w, c) numpy -> (n, c, d, h, w) BF16 channels-last CUDA tensor."""
    return ws._volume(bf16(a).permute(0, 4, 1, 2, 3).cuda())


def as_numpy(t):
    """(n, c, d, h, w) tensor -> (n, d, h, w, c) float64 numpy."""
    return t.detach().float().permute(0, 2, 3, 4, 1).cpu().numpy().astype(np.float64)


def rounded(a):
    return bf16(a).float().numpy().astype(np.float64)


CASES = [(1, (5, 6, 7), 8, 16), (2, (6, 9, 10), 16, 32), (1, (8, 8, 8), 64, 224), (1, (4, 5, 3), 48, 16)]


@pytest.mark.parametrize('n,shape,cin,cout', CASES)
def test_forward_matches_oracle(n, shape, cin, cout):
    rng = np.random.default_rng(cin*cout)
    x = rounded(rng.standard_normal((n,) + shape + (cin,)))
    w = rounded(rng.standard_normal((cout, 27, cin))*0.2)
    b = rng.standard_normal(cout).astype(np.float32)
    for relu in (False, True):
        y = ws.conv3d_forward(volume(x), bf16(w).cuda(), torch.as_tensor(b).cuda(), relu)
        ws.conv_status()
        ref = conv_oracle.conv3d_forward(x, w, b, relu)
        assert abs(as_numpy(y) - ref).max() <= 1e-2*abs(ref).max()


@pytest.mark.parametrize('n,shape,cin,cout', CASES)
def test_weight_grad_matches_oracle(n, shape, cin, cout):
    rng = np.random.default_rng(cin + cout)
    x = rounded(rng.standard_normal((n,) + shape + (cin,)))
    dy = rounded(rng.standard_normal((n,) + shape + (cout,)))
    g = ws.conv3d_weight_grad(volume(x), volume(dy))
    ws.conv_status()
    ref = conv_oracle.conv3d_weight_grad(x, dy)
    assert abs(g.cpu().numpy() - ref).max() <= 1e-4*abs(ref).max()


@pytest.mark.parametrize('n,shape,cin,cout', [c for c in CASES if c[2] % 16 == 0])
def test_input_grad_matches_oracle(n, shape, cin, cout):
    rng = np.random.default_rng(7*cin + cout)
    dy = rounded(rng.standard_normal((n,) + shape + (cout,)))
    w = rounded(rng.standard_normal((cout, 27, cin))*0.2)
    g = ws.conv3d_input_grad(volume(dy), bf16(w).cuda())
    ws.conv_status()
    ref = conv_oracle.conv3d_input_grad(dy, w)
    assert abs(as_numpy(g) - ref).max() <= 1e-2*abs(ref).max()


def test_autograd_gradients_match_oracle():
    """Gradients of L = sum(r * relu(conv(x, W) + b)) through the autograd wrapper, against the oracle."""
    rng = np.random.default_rng(3)
    n, shape, cin, cout = 1, (6, 5, 7), 16, 32
    x = rounded(rng.standard_normal((n,) + shape + (cin,)))
    w = rounded(rng.standard_normal((cout, 27, cin))*0.1)
    b = rng.standard_normal(cout)*0.1
    r = rounded(rng.standard_normal((n,) + shape + (cout,)))
    xt = volume(x).requires_grad_(True)
    wt = torch.tensor(w, dtype=torch.float32, device='cuda', requires_grad=True)
    bt = torch.tensor(b, dtype=torch.float32, device='cuda', requires_grad=True)
    y = ws.Conv3dFunction.apply(xt, wt, bt, True)
    (y.float()*volume(r).float()).sum().backward()
    ws.conv_status()
    pre = conv_oracle.conv3d_forward(x, w, b)
    yref = np.maximum(pre, 0)
    # The mask of the ReLU is taken from the BF16 output: compare where the two agree on the sign.
    dpre = r*(as_numpy(y) > 0)
    assert abs(as_numpy(y) - yref).max() <= 1e-2*abs(yref).max()
    gw = conv_oracle.conv3d_weight_grad(x, rounded(dpre))
    assert abs(wt.grad.cpu().numpy() - gw).max() <= 1e-4*abs(gw).max()
    gx = conv_oracle.conv3d_input_grad(rounded(dpre), w)
    assert abs(as_numpy(xt.grad) - gx).max() <= 1e-2*abs(gx).max()
    assert abs(bt.grad.cpu().numpy() - dpre.sum(axis=(0, 1, 2, 3))).max() <= 1e-3*abs(dpre).sum()


def test_trained_network_speeds_up_steady_solves():
    """Small obstacle channels (64x32x32, spheres of radius 2-5): the network trained on 96 steady states makes the
    solves of 6 held-out channels take fewer steps than from rest, and they reach the same steady fields (both
    solves stop at the residual 1e-6, so their fields differ by what that residual leaves: measured up to 2.1e-3,
    bound 5e-3)."""
    shape, inlet = (64, 32, 32), 0.02
    train = ws.solve_cases(range(1, 97), shape, inlet, 1e-3, threads=4, radius=(2.0, 5.0))
    test = ws.solve_cases(range(1001, 1007), shape, inlet, 1e-3, threads=1, radius=(2.0, 5.0))
    net = ws.WarmStartNet(widths=(16, 32, 64)).cuda()
    history = ws.train(net, train, epochs=40, batch=4, lr=3e-3)
    assert history[-1] < 0.2*history[0]
    rows = ws.evaluate(net, test, shape, inlet)
    cold = sum(r['cold_steps'] for r in rows)
    warm = sum(r['warm_steps'] for r in rows)
    print('steps cold %d warm %d; final velocity errors %s' % (cold, warm, [round(r['final_velocity_error'], 6) for r in rows]))
    # The stated margin: at least 15% fewer steps in all (measured on B200: 17,300 against 24,400, 29% fewer).
    assert warm <= 0.85*cold
    assert max(r['final_velocity_error'] for r in rows) <= 5e-3


@pytest.mark.skipif(not __import__('os').path.exists(__import__('os').path.join(
    __import__('os').path.dirname(ws.__file__), 'warmstart_net', 'weights.pt')), reason='the trained network is not committed')
def test_committed_network_speeds_up_held_out_channels():
    """The committed network of the 128x64x64 obstacle channel (openmm-lbm_b200/warmstart_net/train.py) on two
    channels it never saw: both reach the steady residual 1e-6 faster than from rest, in total at least 1.3 times
    faster in wall time, and end within 5e-3 of the cold solves' fields."""
    import os
    net = ws.load_network(os.path.join(os.path.dirname(ws.__file__), 'warmstart_net', 'weights.pt'))
    rows = ws.time_to_steady(net, [400001, 400002])
    cold = sum(r['cold_seconds'] for r in rows)
    warm = sum(r['warm_seconds'] for r in rows)
    print('held-out: cold %.2f s warm %.2f s (%.2fx), steps %s' % (cold, warm, cold/warm,
                                                                  [(r['cold_steps'], r['warm_steps']) for r in rows]))
    assert all(r['warm_steps'] < r['cold_steps'] for r in rows)
    assert cold >= 1.3*warm
    assert max(r['final_velocity_error'] for r in rows) <= 5e-3
