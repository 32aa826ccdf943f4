"""The free-form window path on the GPU: a caller's window through
soi_init_window_status, the window proposer's CUDA gradients against the CPU
reference network, and the trained proposer's windows meeting their targets
(verified by the method itself against the FP64 direct FFT)."""
import ctypes
import os

import numpy as np
import pytest

import soi_fft_b200 as sb
from soi_fft_b200 import window_cheb as wc
from oracle import mlp_ref
from tests.conftest import rel_l2
from tests import signals

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("prec,tol", [(sb.PRECISION_FP64, 1e-12), (sb.PRECISION_SPLIT_FP32, 1e-6)])
@pytest.mark.parametrize("tau,sigma,B", [(928 / 1024., 373.7314, 72), (512 / 1024., 121.0936, 44)])
def test_caller_window_with_the_straight_profile_is_the_analytic_window(prec, tol, tau, sigma, B):
    N, S = 1 << 18, 16
    dt = np.complex128 if prec == sb.PRECISION_FP64 else np.complex64
    x = torch.from_numpy(signals.gaussian(N, 11, dt)).cuda()
    d = sb.SoiDescriptor(N=N, B=B, tau=tau, sigma=sigma, precision=prec).init(S)
    ya = torch.empty_like(x)
    d.compute_into(x, ya)
    d.free()
    c = wc.analytic_coeffs(tau, sigma, 5, 4)
    d = wc.init_descriptor(c, N, S, 5, 4, B, precision=prec)
    yc = torch.empty_like(x)
    d.compute_into(x, yc)
    d.free()
    err = rel_l2(yc.cpu().numpy().astype(np.complex128), ya.cpu().numpy().astype(np.complex128))
    # the two differ by the window's rounding (long-double closed form against
    # double quadrature, ~1e-15) amplified by the demodulation's gain, as any
    # two evaluations of one window do (the narrow window's gain is ~2e4)
    if prec == sb.PRECISION_FP64:
        tol = max(tol, 1e-14 * wc.conditioning(c, 5, 4))
    assert err <= tol, err


def test_caller_window_rejects_a_vanishing_transform():
    N, S = 1 << 16, 8
    c = wc.analytic_coeffs(928 / 1024., 373.7314, 5, 4)
    yt, yf = wc.window_arrays(c, N, S, 5, 4, 72)
    yf[3] = 0.0
    L = sb.lib()
    L.soi_init_window_status.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                         ctypes.c_void_p]
    d = sb.SoiDescriptor(N=N)
    rc = L.soi_init_window_status(ctypes.byref(d._d), None, S, yt.ctypes.data_as(ctypes.c_void_p),
                                  yf.ctypes.data_as(ctypes.c_void_p))
    assert rc == 1


def test_a_bent_profile_is_a_consistent_window():
    # any admissible profile gives a transform pair: the method's error with it
    # is set by truncation and conditioning, and stays small for a mild bend
    N, S, B = 1 << 18, 16, 72
    c = wc.analytic_coeffs(928 / 1024., 373.7314, 5, 4)
    c[2] += 0.3
    c[3] += 0.2
    assert wc.profile_ok(c, 5, 4)
    x = wc.gaussian(N, 5)
    X = torch.fft.fft(x)
    assert wc.measure(c, x, X, S, 5, 4, B) < 1e-8


def test_proposer_gradient_matches_the_cpu_network():
    net_ref = mlp_ref.Net(2, 32)
    rng = np.random.default_rng(0)
    p = (rng.standard_normal(net_ref.nparams) * 0.2).astype(np.float32)
    x = rng.standard_normal((96, 2)).astype(np.float32)
    y = rng.standard_normal((96, 32)).astype(np.float32)
    net = wc.WindowProposer(params=p)
    out = net.forward(x).cpu().numpy()
    assert np.allclose(out, net_ref.forward(p, x), rtol=1e-4, atol=1e-4)
    loss, g = net.grad(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda())
    lr, gr = net_ref.loss_and_grad(p, x, y)
    assert abs(float(loss.item()) - lr) <= 1e-4 * abs(lr)
    gd = g.cpu().numpy()
    assert np.linalg.norm(gd - gr) <= 1e-4 * np.linalg.norm(gr)


def test_proposer_training_reduces_the_loss():
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, (512, 2)).astype(np.float32)
    y = np.stack([np.sin(x[:, 0] * (1 + k / 16)) + 0.5 * x[:, 1] * np.cos(k) for k in range(32)], 1)
    net = wc.WindowProposer(seed=2)
    hist = net.train(x, y.astype(np.float32), steps=1500, lr=3e-3)
    assert hist[-1] < 0.1 * hist[0]


@pytest.mark.skipif(not os.path.exists(wc.WEIGHTS), reason="the trained proposer is not in the package")
@pytest.mark.parametrize("n,d,target", [(5, 4, 10 ** -9.5), (5, 4, 10 ** -6.5), (9, 8, 10 ** -7.5)])
def test_trained_proposer_window_meets_its_target(n, d, target):
    from soi_fft_b200.window_mlp import length_for
    net, sc, z = wc.load()
    c = net.propose(n, d, target, sc)
    assert wc.profile_ok(c, n, d)
    N, S = length_for(n, d, 20), 16
    x = wc.gaussian(N, 77)
    X = torch.fft.fft(x)
    got = wc.fewest_taps(c, x, X, S, n, d, target, wc.start_taps(z["table"], n, d, target))
    assert got is not None and got[1] <= target
