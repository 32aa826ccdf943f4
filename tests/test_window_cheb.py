"""The free-form window representation (soi_fft_b200/window_cheb.py) on the
CPU: the reference's analytic window (pfft.c:42-82) is the straight erfc
profile, and the quadrature reproduces the library's own window taps; the
window proposer's parameter count matches the CPU reference network."""
import numpy as np
import pytest

import soi_fft_b200 as sb
from soi_fft_b200 import window_cheb as wc
from oracle import mlp_ref


@pytest.mark.parametrize("n,d,tau,sigma", [(5, 4, 928 / 1024., 373.7314), (5, 4, 512 / 1024., 121.0936),
                                           (9, 8, 0.7238, 476.8683)])
def test_analytic_window_is_the_straight_profile(n, d, tau, sigma):
    N, S, B = 1 << 14, 16, 48
    c = wc.analytic_coeffs(tau, sigma, n, d)
    edge = wc.band_edge(n, d)
    xi = np.linspace(0, 0.999 * edge, 1001)
    ref = tau * wc.analytic_freq(xi, tau, sigma)
    assert np.max(np.abs(wc.freq(c, xi, edge) / ref - 1)) < 1e-12
    # the library's taps: filt[kk][theta][s] = (-1)^kk y(t) / mu
    filt = np.asarray(sb.window_tables(N, S, n_mu=n, d_mu=d, B=B, tau=tau, sigma=sigma)[0]).reshape(B, n, S)
    ylib = filt * (n / d) * np.where(np.arange(B) % 2 == 1, -1, 1)[:, None, None]
    y = wc.time_window(c, wc.tap_points(B, n, d, S), edge) / tau
    assert np.max(np.abs(y - ylib)) < 5e-13 * np.max(np.abs(ylib))


def test_time_window_is_the_inverse_transform():
    # a bent profile: y(t) from the quadrature against a fine trapezoid rule
    c = wc.analytic_coeffs(0.8, 250.0, 5, 4)
    c[2] += 0.6
    c[3] += 0.4
    edge = wc.band_edge(5, 4)
    assert wc.profile_ok(c, 5, 4)
    t = np.array([0.0, 0.37, 3.3, 11.8, 25.1])
    xi = np.linspace(0, edge, 400001)
    f = wc.freq(c, xi, edge)
    direct = np.array([2 * np.trapezoid(f * np.cos(2 * np.pi * xi * tt), xi) for tt in t])
    assert np.max(np.abs(wc.time_window(c, t, edge) - direct)) < 1e-9 * abs(direct[0])


def test_window_arrays_shapes_and_positivity():
    c = wc.analytic_coeffs(928 / 1024., 373.7314, 5, 4)
    yt, yf = wc.window_arrays(c, 1 << 14, 8, 5, 4, 72)
    assert yt.shape == (72 * 5 * 8,) and yf.shape == ((1 << 11) // 2 + 1,)
    assert np.all(yf > 0)


def test_profile_check_rejects_a_transform_that_vanishes_inside():
    c = wc.analytic_coeffs(928 / 1024., 373.7314, 5, 4)
    c[0] = 4.0                       # even part positive: Y negative near 0
    assert not wc.profile_ok(c, 5, 4)


def test_proposer_layout_matches_the_cpu_network():
    assert sb.lib().soi_wmlp_param_count() == mlp_ref.Net(2, 32).nparams
