"""Learned windows in free form: a network proposes the window's frequency
response as 32 Chebyshev coefficients (no counterpart in the reference, whose
windows are the two-parameter analytic family of pfft.c:42-82).

Representation.  For oversampling mu the window's band edge is
Xi = mu - 1/2: a window whose Fourier transform vanishes beyond it aliases
nothing into the segment of interest.  The transform is given by a profile g
on [-Xi, Xi] with 32 Chebyshev coefficients,

    Y(xi) = (erfc(g(xi)) - erfc(-g(-xi))) / 2,  g(xi) = sum_k c[k] T_k(xi / Xi),  |xi| < Xi,
    Y(xi) = 0,                                                               |xi| >= Xi,

even by construction and positive where the even part of g is negative; the
time window is its inverse transform,

    y(t) = 2 int_0^Xi Y(xi) cos(2 pi xi t) dxi,

evaluated by Gauss-Legendre quadrature at the taps' points.  The library takes
both through soi_init_window_status; its error sources are then the truncation
of y to B taps and the conditioning of 1/Y over the segment (plus the cut at
the edge, which the measurement of each window includes).  The reference's analytic
window (pfft.c:42-82: a Gaussian-smoothed sinc, whose transform is
(erfc(sqrt(sigma)(xi - tau/2)) - erfc(sqrt(sigma)(xi + tau/2))) / (2 tau)) is
the straight profile g(xi) = sqrt(sigma) (xi - tau/2), two nonzero
coefficients (`analytic_coeffs`), times tau; the other 30 orders bend the
profile into shapes outside that family.

Learning.  Windows around the analytic family (its Pareto points and the
error surrogate's picks, perturbed in the low Chebyshev orders) are measured
by the method itself: the FP64 SOI transform of an i.i.d. Gaussian input
against an FP64 direct FFT (N = 2^20, S = 16).  For each (mu, target) the
measurements give the fewest-taps window that met the target; the network
(2-64-64-32 GELU, CUDA forward/backward/Adam in csrc/mlp_kernels.cuh) learns
(mu, log10 target) -> coefficients.  A proposal is synthesised, its taps B are
the fewest whose measured error meets the target (verification), and the
analytic window stays the fallback.
"""
import ctypes
import math
import os

import numpy as np
from numpy.polynomial import chebyshev as C

from . import lib, SoiDescriptor, PRECISION_FP64, _check

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "window_cheb.npz")
NCHEB = 32
QNODES = 1024
MU_PAIRS = [(5, 4), (8, 7), (9, 8)]
LOG_EPS = (-13.0, -5.0)


def band_edge(n_mu, d_mu):
    return n_mu / d_mu - 0.5


# ---------------------------------------------------------- representation --

def profile(c, xi, edge):
    """g(xi) = sum_k c[k] T_k(xi / edge) on [-edge, edge]."""
    return C.chebval(np.asarray(xi, np.float64) / edge, c)


def freq(c, xi, edge):
    """Y(xi) = (erfc(g(xi)) - erfc(-g(-xi))) / 2 inside the edge, 0 beyond."""
    from scipy.special import erfc
    xi = np.abs(np.asarray(xi, np.float64))
    x = np.minimum(xi, edge)
    y = 0.5 * (erfc(profile(c, x, edge)) - erfc(-profile(c, -x, edge)))
    return np.where(xi < edge, y, 0.0)


_GL = {}


def _gauss_legendre(q):
    """Composite Gauss-Legendre on [-1, 1]: q // 32 panels of 32 points (a
    single rule of high order loses digits in its nodes and weights)."""
    if q not in _GL:
        x32, w32 = np.polynomial.legendre.leggauss(32)
        p = max(1, q // 32)
        lo = -1.0 + 2.0 * np.arange(p) / p
        x = (lo[:, None] + (x32[None, :] + 1.0) / p).ravel()
        w = np.tile(w32 / p, p)
        _GL[q] = (x, w)
    return _GL[q]


def _frac_product(a, b, xp):
    """frac(a * b) for float64 arrays to ~1e-16 absolute: the product split
    exactly into hi + lo (Veltkamp splitting, Dekker's two-product), so that
    cos(2 pi a b) keeps full accuracy when a * b is large (up to ~40 here)."""
    def split(v):
        c = 134217729.0 * v
        hi = c - (c - v)
        return hi, v - hi
    p = a * b
    ah, al = split(a)
    bh, bl = split(b)
    err = ((ah * bh - p) + ah * bl + al * bh) + al * bl
    return (p - xp.round(p)) + err


def time_window(c, t, edge, q=QNODES):
    """y(t) = 2 int_0^edge Y(xi) cos(2 pi xi t) dxi (Gauss-Legendre, q nodes)."""
    x, w = _gauss_legendre(q)
    xi = 0.5 * edge * (x + 1.0)
    wy = 0.5 * edge * w * freq(c, xi, edge)
    t = np.asarray(t, np.float64)
    out = np.empty(t.shape)
    flat = t.ravel()
    res = out.ravel()
    for i in range(0, flat.size, 4096):
        tt = flat[i:i + 4096][:, None]
        res[i:i + 4096] = 2.0 * np.cos(2.0 * np.pi * _frac_product(tt, xi[None, :], np)) @ wy
    return out


def time_window_gpu(c, t, edge, q=QNODES, device="cuda"):
    """time_window in FP64 on the GPU (the same quadrature)."""
    import torch
    x, w = _gauss_legendre(q)
    xi = 0.5 * edge * (x + 1.0)
    wy = torch.tensor(0.5 * edge * w * freq(c, xi, edge), device=device)
    xit = torch.tensor(xi, device=device)[None, :]
    tt = torch.tensor(np.asarray(t, np.float64).ravel(), device=device)
    out = torch.empty_like(tt)
    for i in range(0, tt.numel(), 1 << 15):
        ph = _frac_product(tt[i:i + (1 << 15)][:, None], xit, torch)
        out[i:i + (1 << 15)] = 2.0 * torch.cos(2.0 * math.pi * ph) @ wy
    return out.cpu().numpy().reshape(np.shape(t))


def tap_points(B, n_mu, d_mu, S):
    """t[kk][theta][s] = theta*d/n - kk - s/S + (B - d)/2: where the library
    evaluates the window (the reference's w_f arguments, pfft.c:52)."""
    kk = np.arange(B)[:, None, None]
    th = np.arange(n_mu)[None, :, None]
    s = np.arange(S)[None, None, :]
    return th * d_mu / n_mu - kk - s / S + (B - d_mu) / 2.0


def window_arrays(c, N, S, n_mu, d_mu, B, device=None):
    """(y_time [B*n*S], y_freq [M/2 + 1]) for soi_init_window_status (the
    quadrature on the GPU when a device is given)."""
    edge = band_edge(n_mu, d_mu)
    M = N // S
    t = tap_points(B, n_mu, d_mu, S)
    yt = (time_window_gpu(c, t, edge, device=device) if device is not None else time_window(c, t, edge)).ravel()
    yf = freq(c, np.arange(M // 2 + 1) / M - 0.5, edge)
    return np.ascontiguousarray(yt), np.ascontiguousarray(yf)


def analytic_freq(xi, tau, sigma):
    """The reference's y_W (pfft.c:68-82): (erfc(sqrt(s)(xi - tau/2)) - erfc(sqrt(s)(xi + tau/2))) / (2 tau)."""
    from scipy.special import erfc
    sq = math.sqrt(sigma)
    xi = np.asarray(xi, np.float64)
    return (erfc(sq * (xi - tau / 2)) - erfc(sq * (xi + tau / 2))) / (2 * tau)


def analytic_coeffs(tau, sigma, n_mu, d_mu):
    """The reference's window as a profile: g(xi) = sqrt(sigma) (xi - tau/2),
    c[0] = -sqrt(sigma) tau / 2, c[1] = sqrt(sigma) Xi; its transform is
    tau * y_W (pfft.c:68-82), cut at the edge."""
    edge = band_edge(n_mu, d_mu)
    sq = math.sqrt(sigma)
    c = np.zeros(NCHEB)
    c[0] = -sq * tau / 2.0
    c[1] = sq * edge
    return c


def conditioning(c, n_mu, d_mu):
    """max over the segment of interest of Y(0) / Y(xi) (the demodulation's gain)."""
    edge = band_edge(n_mu, d_mu)
    xi = np.linspace(0, 0.5, 257)
    f = freq(c, xi, edge)
    return float(f[0] / f.min())


def profile_ok(c, n_mu, d_mu):
    """Y is positive inside the edge (the even part of g is negative there)
    and has fallen by the edge (Y(Xi) < 0.08: what the cut there costs in
    accuracy, the measurement shows)."""
    edge = band_edge(n_mu, d_mu)
    xi = np.linspace(0, edge, 513)
    gp, gm = profile(c, xi, edge), profile(c, -xi, edge)
    return bool(np.all(np.isfinite(gp)) and np.all(gp[:-1] + gm[:-1] < 0) and gp[-1] >= 1.0 and -gm[-1] >= 1.0)


# -------------------------------------------------------------- measuring --

def init_descriptor(c, N, S, n_mu, d_mu, B, precision=PRECISION_FP64, device=0, gpu_quadrature=True):
    """A descriptor initialised with the synthesised window (soi_init_window_status)."""
    L = lib()
    L.soi_init_window_status.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                         ctypes.c_void_p]
    yt, yf = window_arrays(c, N, S, n_mu, d_mu, B, device=("cuda:%d" % device) if gpu_quadrature else None)
    d = SoiDescriptor(N=N, n_mu=n_mu, d_mu=d_mu, B=B, precision=precision, device=device)
    _check(L.soi_init_window_status(ctypes.byref(d._d), None, S, yt.ctypes.data_as(ctypes.c_void_p),
                                    yf.ctypes.data_as(ctypes.c_void_p)), "soi_init_window_status")
    return d


def measure(c, x, X, S, n_mu, d_mu, B, precision=PRECISION_FP64):
    """rel-L2 of the SOI transform of the CUDA tensor x with window c and B
    taps against the FP64 direct FFT X (1.0 for a window the library refuses)."""
    import torch
    xin = x if precision == PRECISION_FP64 else x.to(torch.complex64)
    try:
        d = init_descriptor(c, x.numel(), S, n_mu, d_mu, B, precision, x.device.index or 0)
    except Exception:
        return 1.0
    try:
        y = torch.empty_like(xin)
        d.compute_into(xin, y)
    finally:
        d.free()
    e = float(torch.linalg.norm(y.to(torch.complex128) - X) / torch.linalg.norm(X))
    return e if math.isfinite(e) else 1.0


def gaussian(N, seed, device="cuda"):
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    return torch.complex(torch.randn(N, generator=g, device=device, dtype=torch.float64),
                         torch.randn(N, generator=g, device=device, dtype=torch.float64))


def time_transform(c, x, S, n_mu, d_mu, B, reps=5):
    """Median device time (ms) of the FP64 transform of x with window c and B taps."""
    import torch
    d = init_descriptor(c, x.numel(), S, n_mu, d_mu, B, device=x.device.index or 0)
    try:
        y = torch.empty_like(x)
        d.compute_into(x, y)
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record()
            d.compute_into(x, y)
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
    finally:
        d.free()
    return float(np.median(ts))


# ----------------------------------------------------------- data and search --

def candidate_windows(rng, n_mu, d_mu, seeds, count, scale=0.6, orders=8):
    """Coefficient vectors around analytic windows: each seed (tau, sigma)'s
    straight profile with its low Chebyshev orders perturbed (random
    amplitudes decaying with the order)."""
    out = []
    for _ in range(count):
        tau, sigma = seeds[rng.integers(len(seeds))]
        c = analytic_coeffs(tau, sigma, n_mu, d_mu)
        amp = scale * rng.uniform(0, 1) / (1.0 + np.arange(orders)) ** 1.5
        c[:orders] += amp * rng.standard_normal(orders)
        out.append(c)
    return out


def _seeds(n_mu, d_mu, B, surrogate_best):
    from .window_mlp import PARETO
    mu = n_mu / d_mu
    s = [(t, sg) for (m, t, sg, b, _) in PARETO if abs(m - mu) < 1e-9]
    s += [(t, sg) for (b, t, sg, _) in surrogate_best if abs(b - B) <= 4]
    s.append((928 / 1024., 373.7314))
    return s


def run_search(out, per_b=48, log2n=20, S=16, seed=0):
    """Measure candidate windows for every oversampling pair and B; store the
    rows (mu pair, B, coefficients, error) in `out`."""
    import torch
    from .window_mlp import WindowMLP, length_for
    surrogate = WindowMLP.load()
    rows = []
    for (n_mu, d_mu) in MU_PAIRS:
        best = surrogate.predict_best(n_mu, d_mu)
        N = length_for(n_mu, d_mu, log2n)
        x = gaussian(N, 1000 + n_mu)
        X = torch.fft.fft(x)
        rng = np.random.default_rng(seed + n_mu)
        for B in range(max(12, d_mu + 2), 85, 3):
            seeds = _seeds(n_mu, d_mu, B, best)
            cands = [analytic_coeffs(t, sg, n_mu, d_mu) for (t, sg) in seeds]
            cands += candidate_windows(rng, n_mu, d_mu, seeds, 4 * per_b)
            cands = [c for c in cands if profile_ok(c, n_mu, d_mu)][:len(seeds) + per_b]
            errs = []
            for c in cands:
                errs.append(measure(c, x, X, S, n_mu, d_mu, B))
                rows.append((n_mu, d_mu, B, c, errs[-1]))
            print("mu %d/%d B %d: %d windows, best %s" % (n_mu, d_mu, B, len(cands),
                  "%.3e" % min(errs) if errs else "-"), flush=True)
        del x, X
        torch.cuda.empty_cache()
    np.savez(out, mu=np.array([(r[0], r[1]) for r in rows]), B=np.array([r[2] for r in rows]),
             coeffs=np.array([r[3] for r in rows]), err=np.array([r[4] for r in rows]))
    return rows


def load_rows(path):
    z = np.load(path)
    return [(int(m[0]), int(m[1]), int(b), c, float(e)) for m, b, c, e in zip(z["mu"], z["B"], z["coeffs"], z["err"])]


def best_for(rows, n_mu, d_mu, target):
    """The fewest-taps measured window that met the target (ties: the smaller error)."""
    ok = [r for r in rows if r[:2] == (n_mu, d_mu) and r[4] <= target]
    return min(ok, key=lambda r: (r[2], r[4])) if ok else None


def training_set(rows, grid=np.linspace(LOG_EPS[0], LOG_EPS[1], 81)):
    """(features, coefficients, taps table) for every (mu, log10 target) on the
    grid: the fewest-taps measured window that met the target."""
    feats, coefs, table = [], [], []
    for (n_mu, d_mu) in MU_PAIRS:
        for le in grid:
            r = best_for(rows, n_mu, d_mu, 10.0 ** le)
            if r is None:
                continue
            feats.append(features(n_mu, d_mu, le))
            coefs.append(r[3])
            table.append((n_mu, d_mu, 10.0 ** le, r[2]))
    return np.array(feats, np.float32), np.array(coefs), np.array(table, np.float64)


# ---------------------------------------------------------------- network --

def features(n_mu, d_mu, log_eps):
    mu = np.asarray(n_mu, np.float64) / np.asarray(d_mu, np.float64)
    return np.stack(np.broadcast_arrays((mu - 1.17) / 0.06, (np.asarray(log_eps, np.float64) + 9.0) / 2.5),
                    axis=-1).astype(np.float32)


class CoeffScaler:
    """Per-coefficient affine normalisation of the network's targets."""

    def __init__(self, coeffs):
        a = np.asarray(coeffs, np.float64)
        self.mean = a.mean(0)
        self.std = a.std(0) + 1e-6

    def to_net(self, c):
        return ((np.asarray(c) - self.mean) / self.std).astype(np.float32)

    def from_net(self, z):
        return np.asarray(z, np.float64) * self.std + self.mean


class WindowProposer:
    """The 2-64-64-32 network; parameters and Adam state in device memory."""

    def __init__(self, params=None, seed=0, device="cuda"):
        import torch
        self.device = device
        n = lib().soi_wmlp_param_count()
        if params is None:
            rng = np.random.default_rng(seed)
            p = np.zeros(n, np.float32)
            H, IN, OUT = 64, 2, NCHEB
            p[0:H * IN] = rng.normal(0, np.sqrt(2.0 / (IN + H)), H * IN)
            o = H * IN + H
            p[o:o + H * H] = rng.normal(0, np.sqrt(2.0 / (2 * H)), H * H)
            o += H * H + H
            p[o:o + OUT * H] = rng.normal(0, np.sqrt(2.0 / (H + OUT)), OUT * H)
            params = p
        self.p = torch.tensor(np.asarray(params, np.float32), device=device)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.g = torch.zeros_like(self.p)
        self.loss = torch.zeros(1, dtype=torch.float32, device=device)
        self.step = 0

    @staticmethod
    def _ptr(t):
        return ctypes.c_void_p(t.data_ptr())

    def forward(self, x):
        import torch
        L = lib()
        L.soi_wmlp_forward_device.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_void_p]
        x = torch.as_tensor(np.asarray(x, np.float32), device=self.device).contiguous()
        y = torch.empty((x.shape[0], NCHEB), dtype=torch.float32, device=self.device)
        _check(L.soi_wmlp_forward_device(self._ptr(self.p), self._ptr(x), self._ptr(y), x.shape[0], None),
               "soi_wmlp_forward_device")
        return y

    def grad(self, x, y):
        L = lib()
        L.soi_wmlp_grad_device.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] + [ctypes.c_void_p] * 3
        _check(L.soi_wmlp_grad_device(self._ptr(self.p), self._ptr(x), self._ptr(y), x.shape[0],
                                      self._ptr(self.g), self._ptr(self.loss), None), "soi_wmlp_grad_device")
        return self.loss, self.g

    def train(self, x, y, steps=4000, lr=3e-3, lr_end=1e-4, batch=256, seed=0):
        import torch
        L = lib()
        L.soi_adam_device.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                                              ctypes.c_void_p]
        xd = torch.as_tensor(np.asarray(x, np.float32), device=self.device).contiguous()
        yd = torch.as_tensor(np.asarray(y, np.float32), device=self.device).contiguous()
        n = xd.shape[0]
        gen = torch.Generator(device="cpu").manual_seed(seed)
        hist = []
        for i in range(steps):
            idx = torch.randint(0, n, (min(batch, n),), generator=gen).to(self.device)
            self.grad(xd[idx].contiguous(), yd[idx].contiguous())
            self.step += 1
            a = lr * (lr_end / lr) ** (i / max(1, steps - 1))
            _check(L.soi_adam_device(self._ptr(self.p), self._ptr(self.m), self._ptr(self.v), self._ptr(self.g),
                                     self.p.numel(), a, self.step, None), "soi_adam_device")
            if i % 200 == 0 or i == steps - 1:
                hist.append(float(self.loss.item()))
        return hist

    def propose(self, n_mu, d_mu, target, scaler):
        z = self.forward(features(n_mu, d_mu, math.log10(target))[None, :]).cpu().numpy()[0]
        return scaler.from_net(z)


def save(path, net, scaler, **extra):
    np.savez(path, params=net.p.cpu().numpy(), mean=scaler.mean, std=scaler.std, **extra)


def load(path=WEIGHTS, device="cuda"):
    z = np.load(path)
    net = WindowProposer(params=z["params"], device=device)
    sc = CoeffScaler.__new__(CoeffScaler)
    sc.mean, sc.std = z["mean"], z["std"]
    return net, sc, z


def start_taps(table, n_mu, d_mu, target):
    """The taps of the training table's nearest target (the verification's start)."""
    le = math.log10(target)
    near = [(abs(math.log10(r[2]) - le), int(r[3])) for r in table if (int(r[0]), int(r[1])) == (n_mu, d_mu)]
    return min(near)[1] if near else 48


def fewest_taps(c, x, X, S, n_mu, d_mu, target, B0, Bmax=96, precision=PRECISION_FP64):
    """The fewest taps with which window c meets the target, searched from B0
    (down while it meets it, else up); (B, error) or None."""
    e = measure(c, x, X, S, n_mu, d_mu, B0, precision)
    B = B0
    if e <= target:
        while B - 1 > d_mu:
            e2 = measure(c, x, X, S, n_mu, d_mu, B - 1, precision)
            if e2 > target:
                break
            B, e = B - 1, e2
        return B, e
    while B < Bmax:
        B += 1
        e = measure(c, x, X, S, n_mu, d_mu, B, precision)
        if e <= target:
            return B, e
    return None


def evaluate(net, scaler, table, log2n=26, S=32,
             targets=(10 ** -12.5, 10 ** -11.5, 10 ** -10.5, 10 ** -9.5, 10 ** -8.5, 10 ** -7.5, 10 ** -6.5,
                      10 ** -5.5), seed=4321):
    """Held-out targets (between the training grid's points) at N ~ 2^log2n:
    the proposed window (taps by verification), the analytic window (Pareto
    points, else the default) and the error surrogate's verified window; taps,
    errors and FP64 times.  Yields one dict per case."""
    import torch
    from .window_mlp import length_for, analytic_window, learned_window, WindowMLP, measure_error
    from .window_mlp import time_transform as time_analytic
    surrogate = WindowMLP.load()
    for (n_mu, d_mu) in MU_PAIRS:
        N = length_for(n_mu, d_mu, log2n)
        x = gaussian(N, seed + n_mu)
        X = torch.fft.fft(x)
        meas = lambda B, tau, sigma: measure_error(x, S, n_mu, d_mu, int(B), tau, sigma, X)
        for tgt in targets:
            rec = {"mu": "%d/%d" % (n_mu, d_mu), "N": N, "S": S, "target": tgt}
            c = net.propose(n_mu, d_mu, tgt, scaler)
            rec["profile_ok"] = profile_ok(c, n_mu, d_mu)
            got = fewest_taps(c, x, X, S, n_mu, d_mu, tgt, start_taps(table, n_mu, d_mu, tgt)) \
                if rec["profile_ok"] else None
            if got:
                rec["proposed"] = {"B": got[0], "err": got[1], "conditioning": conditioning(c, n_mu, d_mu)}
            base = analytic_window(n_mu, d_mu, tgt, meas)
            rec["analytic"] = {"B": base[0], "err": base[3], "meets": base[3] <= tgt}
            sur = learned_window(surrogate, n_mu, d_mu, tgt, meas)
            if sur:
                rec["surrogate"] = {"B": sur[0], "err": sur[3]}
            if got and base[3] <= tgt:
                tp = time_transform(c, x, S, n_mu, d_mu, got[0])
                ta = time_analytic(x, S, n_mu, d_mu, *base[:3])
                rec.update(taps_saved_vs_analytic=base[0] - got[0], ms_proposed=tp, ms_analytic=ta,
                           speedup_vs_analytic=ta / tp)
            if got and sur:
                rec["taps_saved_vs_surrogate"] = sur[0] - got[0]
            yield rec
        del x, X
        torch.cuda.empty_cache()


def main():
    import argparse
    import json
    ap = argparse.ArgumentParser(description="the free-form window proposer: measure, train, evaluate (GPU)")
    ap.add_argument("--search", default=None, metavar="ROWS.npz", help="measure candidate windows into ROWS.npz")
    ap.add_argument("--per-b", type=int, default=48)
    ap.add_argument("--train", default=None, metavar="ROWS.npz", help="train the proposer on measured rows")
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--evaluate", action="store_true")
    ap.add_argument("--eval-log2n", type=int, default=26)
    a = ap.parse_args()
    if a.search:
        rows = run_search(a.search, per_b=a.per_b)
        print(json.dumps({"measurements": len(rows)}))
    if a.train:
        rows = load_rows(a.train)
        x, c, table = training_set(rows)
        sc = CoeffScaler(c)
        net = WindowProposer(seed=3)
        hist = net.train(x, sc.to_net(c), steps=a.steps)
        save(a.out, net, sc, table=table, loss_history=np.array(hist), measurements=len(rows))
        print(json.dumps({"samples": int(len(x)), "loss_first": hist[0], "loss_last": hist[-1],
                          "measurements": len(rows)}))
    if a.evaluate:
        net, sc, z = load(a.out)
        for rec in evaluate(net, sc, z["table"], log2n=a.eval_log2n):
            print(json.dumps(rec), flush=True)


if __name__ == "__main__":
    main()
