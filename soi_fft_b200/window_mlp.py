"""Learned window proposals for the SOI transform (no counterpart in the
reference, whose windows are the analytic family of pfft.c:42-82 with the
Pareto points of pfft.c:111-137).

A small MLP (4 -> 64 -> 64 -> 1, GELU; CUDA forward/backward/Adam kernels in
csrc/mlp_kernels.cuh) predicts log10 of the transform's relative L2 error
from a window description (oversampling mu = n_mu/d_mu, taps B, tau, sigma).
It is trained on errors that the method itself measures: the FP64 SOI
transform of i.i.d. Gaussian inputs against an FP64 direct FFT.  Given a
target accuracy, `propose` scans the network over (B, tau, sigma), takes the
smallest B whose best predicted error beats the target with a margin, and
`verify` runs the actual transform on a fresh input: the proposal is accepted
only if the measured error meets the target.  Otherwise the analytic window
(the reference's default, or its Pareto table) is used.

Training and evaluation run on the GPU; torch provides device memory and the
FP64 direct FFT used as the judge.
"""
import ctypes
import math
import os

import numpy as np

from . import lib, SoiDescriptor, PRECISION_FP64

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "window_mlp.npz")

# oversampling pairs the network covers, and the N each is measured at
# (M' = n_mu*M/d_mu must be integral: for 8/7 the length carries a factor 7)
MU_PAIRS = [(5, 4), (8, 7), (9, 8)]
NPARAMS = None

# The reference's Pareto table, pfft.c:111-137: (mu, tau, sigma, B, SNR dB)
PARETO = [
    (1.25, 872 / 1024, 313.1715, 76, 289.2718), (1.25, 928 / 1024, 373.7314, 72, 288.1844),
    (1.25, 818 / 1024, 267.4513, 64, 284.7614), (1.25, 0.899, 352.7647081, 60, 282),
    (1.25, 764 / 1024, 213.2893, 60, 275.246), (1.25, 709 / 1024, 201.8235, 56, 266.6957),
    (1.25, 0.782, 245.8927353, 54, 259), (1.25, 652 / 1024, 176.9743, 54, 258.2814),
    (1.25, 591 / 1024, 154.7071, 50, 247.7459), (1.25, 512 / 1024, 121.0936, 44, 241.8972),
    (1.25, 0.664, 182.5254421, 46, 239), (1.25, 0.578, 155.3322, 44, 233),
    (1.25, 0.531, 136.5983707, 41, 220), (1.25, 383 / 1024, 104.1262, 42, 219.777),
    (1.25, 0.4476, 119.2272, 38, 213), (1.25, 299 / 1024, 90.5391, 38, 210.1298),
    (1.25, 0.373, 102.1115361, 36, 200), (1.25, 0.2927, 90.7306, 32, 193),
    (1.25, 0.154, 73.2102363, 30, 179),
    (1.125, 0.7238, 476.8683, 76, 213), (1.125, 0.6476, 363.891, 66, 193),
    (1.5, 931 / 1024, 109.0712, 36, 289.6294), (1.5, 832 / 1024, 93.4329, 38, 289.4688),
    (1.5, 0.0554, 36.6513, 22, 235),
]

TAU_RANGE = (0.08, 0.97)
# training targets are log10(error) clipped to [-16.5, 1]: every window whose
# error is above 10 is equally useless, and the clip keeps the blown-up ones
# (errors up to 1e15 where the window's frequency response nearly vanishes)
# from taking the network's capacity
Y_CLIP = (-16.5, 1.0)


def clip_target(y):
    return np.clip(y, *Y_CLIP)

SIGMA_RANGE = (25.0, 800.0)
B_RANGE = (12, 84)


def nparams():
    global NPARAMS
    if NPARAMS is None:
        NPARAMS = lib().soi_mlp_param_count()
    return NPARAMS


def features(n_mu, d_mu, B, tau, sigma):
    """Normalised network inputs (arrays broadcast)."""
    mu = np.asarray(n_mu, np.float64) / np.asarray(d_mu, np.float64)
    return np.stack(np.broadcast_arrays((mu - 1.17) / 0.06, (np.asarray(B, np.float64) - 48.0) / 20.0,
                                        (np.asarray(tau, np.float64) - 0.55) / 0.25,
                                        (np.log(np.asarray(sigma, np.float64)) - 5.3) / 0.7), axis=-1)


def length_for(n_mu, d_mu, log2n):
    """A transform length near 2^log2n for which n_mu*M/d_mu is integral."""
    return (1 << log2n) if d_mu in (1, 2, 4, 8, 16) else d_mu * (1 << (log2n - 3))


# ------------------------------------------------------------ measurement --

def measure_error(x, S, n_mu, d_mu, B, tau, sigma, X=None, precision=PRECISION_FP64):
    """rel-L2 of the SOI transform of the CUDA complex128 tensor x against the
    FP64 direct FFT X (computed when not given), in the given precision form
    (the split form transforms x rounded once to complex64)."""
    import torch
    if X is None:
        X = torch.fft.fft(x)
    xin = x if precision == PRECISION_FP64 else x.to(torch.complex64)
    d = SoiDescriptor(N=x.numel(), n_mu=n_mu, d_mu=d_mu, B=B, tau=float(tau), sigma=float(sigma),
                      precision=precision, device=x.device.index or 0)
    try:
        d.init(S)
        y = torch.empty_like(xin)
        d.compute_into(xin, y)
    finally:
        d.free()
    e = float(torch.linalg.norm(y.to(torch.complex128) - X) / torch.linalg.norm(X))
    if not math.isfinite(e):
        e = 1.0
    return e


def conditioning(tau, sigma):
    """max |W_inv| of the window: 1 / y_W(t) at the band edge |t| = 1/2, where
    y_W(t) = (erfc(sqrt(sigma)(t - tau/2)) - erfc(sqrt(sigma)(t + tau/2))) / (2 tau)
    (pfft.c:68-82) is smallest.  The demodulation multiplies by it, so it
    amplifies the working precision's rounding: in the split form a window's
    error is about its FP64 error plus SPLIT_ROUNDING * conditioning."""
    sq = math.sqrt(sigma)
    y = (math.erfc(sq * (0.5 - tau / 2)) - math.erfc(sq * (0.5 + tau / 2))) / (2 * tau)
    return 1.0 / y if y > 0 else float("inf")


# measured: the default window (conditioning 9.1) has split error 3.4e-7 and a
# tau = 0.345, sigma = 56 window (conditioning ~1200) 5.2e-5 -> ~0.6 * 2^-24 each
SPLIT_ROUNDING = 0.6 * 2.0 ** -24


def sample_windows(rng, n, n_mu, d_mu):
    B = rng.integers(max(B_RANGE[0], d_mu + 1), B_RANGE[1] + 1, size=n)
    tau = rng.uniform(*TAU_RANGE, size=n)
    sigma = np.exp(rng.uniform(np.log(SIGMA_RANGE[0]), np.log(SIGMA_RANGE[1]), size=n))
    return B, tau, sigma


def make_dataset(per_mu=1200, log2n=20, S=16, seed=0, device="cuda"):
    """Measured (features, log10 error) pairs over the three oversampling pairs."""
    import torch
    rng = np.random.default_rng(seed)
    feats, ys, raw = [], [], []
    for (n, d) in MU_PAIRS:
        N = length_for(n, d, log2n)
        g = torch.Generator(device=device).manual_seed(seed + n)
        x = torch.complex(torch.randn(N, generator=g, device=device, dtype=torch.float64),
                          torch.randn(N, generator=g, device=device, dtype=torch.float64))
        X = torch.fft.fft(x)
        B, tau, sigma = sample_windows(rng, per_mu, n, d)
        for b, t, s in zip(B, tau, sigma):
            e = measure_error(x, S, n, d, int(b), t, s, X)
            raw.append((n, d, int(b), t, s, e))
            feats.append(features(n, d, b, t, s))
            ys.append(clip_target(np.log10(max(e, 1e-300))))
    return np.array(feats, np.float32), np.array(ys, np.float32), raw


# ---------------------------------------------------------------- network --

class WindowMLP:
    """Parameters and Adam state in device memory; kernels from the C ABI."""

    def __init__(self, params=None, seed=0, device="cuda"):
        import torch
        self.device = device
        n = nparams()
        if params is None:
            rng = np.random.default_rng(seed)
            p = np.zeros(n, np.float32)
            # W1 64x4, W2 64x64, W3 64 (Glorot-style scale); biases zero
            p[0:256] = rng.normal(0, np.sqrt(2.0 / 68), 256)
            p[320:320 + 4096] = rng.normal(0, np.sqrt(2.0 / 128), 4096)
            p[320 + 4096 + 64:320 + 4096 + 128] = rng.normal(0, np.sqrt(2.0 / 65), 64)
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
        x = torch.as_tensor(np.asarray(x, np.float32), device=self.device).contiguous()
        y = torch.empty(x.shape[0], dtype=torch.float32, device=self.device)
        rc = lib().soi_mlp_forward_device(self._ptr(self.p), self._ptr(x), self._ptr(y), x.shape[0], None)
        if rc:
            raise RuntimeError("soi_mlp_forward_device: %d" % rc)
        return y

    def grad(self, x, y):
        """(loss, gradient) of mean squared error on device tensors x [n,4], y [n]."""
        rc = lib().soi_mlp_grad_device(self._ptr(self.p), self._ptr(x), self._ptr(y), x.shape[0],
                                       self._ptr(self.g), self._ptr(self.loss), None)
        if rc:
            raise RuntimeError("soi_mlp_grad_device: %d" % rc)
        return self.loss, self.g

    def train(self, x, y, steps=3000, lr=3e-3, lr_end=2e-4, batch=1024, seed=0):
        import torch
        xd = torch.as_tensor(np.asarray(x, np.float32), device=self.device).contiguous()
        yd = torch.as_tensor(np.asarray(y, np.float32), device=self.device).contiguous()
        n = xd.shape[0]
        gen = torch.Generator(device="cpu").manual_seed(seed)
        hist = []
        for i in range(steps):
            idx = torch.randint(0, n, (min(batch, n),), generator=gen).to(self.device)
            xb, yb = xd[idx].contiguous(), yd[idx].contiguous()
            self.grad(xb, yb)
            self.step += 1
            a = lr * (lr_end / lr) ** (i / max(1, steps - 1))
            rc = lib().soi_mlp_adam_device(self._ptr(self.p), self._ptr(self.m), self._ptr(self.v),
                                           self._ptr(self.g), ctypes.c_float(a), self.step, None)
            if rc:
                raise RuntimeError("soi_mlp_adam_device: %d" % rc)
            if i % 200 == 0 or i == steps - 1:
                hist.append(float(self.loss.item()))
        return hist

    def params_numpy(self):
        return self.p.cpu().numpy()

    def save(self, path=WEIGHTS, **meta):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, params=self.params_numpy(), **meta)

    @classmethod
    def load(cls, path=WEIGHTS, device="cuda"):
        z = np.load(path)
        return cls(params=z["params"], device=device)

    # ---------------------------------------------------------- proposals --

    def predict_grid(self, n_mu, d_mu, ntau=48, nsig=48):
        """Predicted log10 error over the (B, tau, sigma) grid: (Bs, taus, sigmas, pred[B][tau][sigma])."""
        Bs = np.arange(max(B_RANGE[0], d_mu + 1), B_RANGE[1] + 1)
        taus = np.linspace(*TAU_RANGE, ntau)
        sigs = np.exp(np.linspace(np.log(SIGMA_RANGE[0]), np.log(SIGMA_RANGE[1]), nsig))
        BB, TT, SS = np.meshgrid(Bs, taus, sigs, indexing="ij")
        f = features(n_mu, d_mu, BB.ravel(), TT.ravel(), SS.ravel())
        pred = self.forward(f).cpu().numpy().reshape(BB.shape)
        return Bs, taus, sigs, pred

    def predict_best(self, n_mu, d_mu, ntau=48, nsig=48):
        """For every B, the (tau, sigma) with the lowest predicted error."""
        Bs, taus, sigs, pred = self.predict_grid(n_mu, d_mu, ntau, nsig)
        out = []
        for i, b in enumerate(Bs):
            it, isg = np.unravel_index(pred[i].argmin(), pred[i].shape)
            out.append((int(b), float(taus[it]), float(sigs[isg]), float(pred[i, it, isg])))
        return out

    def propose(self, n_mu, d_mu, target, slack=0.3, per_b=3, precision=PRECISION_FP64):
        """Candidates (B, tau, sigma, predicted log10 error) in increasing B:
        for each B the `per_b` best-predicted (tau, sigma) whose prediction is
        within `slack` decades of the target (the measurement decides).  For the
        split form the prediction is the FP64 one plus the window's
        conditioning times the FP32 rounding."""
        lt = math.log10(target)
        Bs, taus, sigs, pred = self.predict_grid(n_mu, d_mu)
        if precision != PRECISION_FP64:
            cond = np.array([[conditioning(t, sg) for sg in sigs] for t in taus])
            pred = np.log10(10.0 ** pred + SPLIT_ROUNDING * cond[None, :, :])
        out = []
        for i, b in enumerate(Bs):
            flat = pred[i].ravel()
            for j in np.argsort(flat)[:per_b]:
                if flat[j] > lt + slack:
                    break
                it, isg = np.unravel_index(j, pred[i].shape)
                out.append((int(b), float(taus[it]), float(sigs[isg]), float(flat[j])))
        return out


def analytic_window(n_mu, d_mu, target, measure):
    """The method without the network: the smallest-B Pareto point of the
    reference's table for this mu whose measured error meets the target, else
    the default window (pfft.c:87-91).  `measure(B, tau, sigma)` returns the
    error."""
    mu = n_mu / d_mu
    for (m, tau, sigma, B, snr) in sorted((p for p in PARETO if abs(p[0] - mu) < 1e-9), key=lambda p: p[3]):
        e = measure(B, tau, sigma)
        if e <= target:
            return B, tau, sigma, e
    e = measure(72, 928 / 1024., 373.7314)
    return 72, 928 / 1024., 373.7314, e


def learned_window(net, n_mu, d_mu, target, measure, tries=24, precision=PRECISION_FP64):
    """A verified proposal: the first candidate (smallest B) whose measured
    error (in `measure`'s precision form) meets the target; None when none of
    the first `tries` does."""
    for (B, tau, sigma, pred) in net.propose(n_mu, d_mu, target, precision=precision)[:tries]:
        e = measure(B, tau, sigma)
        if e <= target:
            return B, tau, sigma, e, pred
    return None


def time_transform(x, S, n_mu, d_mu, B, tau, sigma, reps=5):
    """Median device time (ms) of the FP64 transform with this window."""
    import torch
    d = SoiDescriptor(N=x.numel(), n_mu=n_mu, d_mu=d_mu, B=B, tau=float(tau), sigma=float(sigma),
                      precision=PRECISION_FP64, device=x.device.index or 0)
    try:
        d.init(S)
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


def evaluate(net, log2n=26, S=32, targets=(1e-12, 1e-11, 1e-10, 1e-9, 1e-8, 1e-7), seed=1234):
    """Held-out evaluation: for each oversampling pair and target, the
    learned (verified) window against the analytic one at N ~ 2^log2n: taps,
    measured errors and FP64 transform times.  Yields one dict per case."""
    import torch
    for (n_mu, d_mu) in MU_PAIRS:
        N = length_for(n_mu, d_mu, log2n)
        g = torch.Generator(device="cuda").manual_seed(seed + n_mu)
        x = torch.complex(torch.randn(N, generator=g, device="cuda", dtype=torch.float64),
                          torch.randn(N, generator=g, device="cuda", dtype=torch.float64))
        X = torch.fft.fft(x)
        measure = lambda B, tau, sigma: measure_error(x, S, n_mu, d_mu, int(B), tau, sigma, X)
        for tgt in targets:
            base = analytic_window(n_mu, d_mu, tgt, measure)
            learned = learned_window(net, n_mu, d_mu, tgt, measure)
            rec = {"mu": "%d/%d" % (n_mu, d_mu), "N": N, "S": S, "target": tgt,
                   "analytic": {"B": base[0], "tau": base[1], "sigma": base[2], "err": base[3],
                                "meets": base[3] <= tgt}}
            if learned is not None:
                rec["learned"] = {"B": learned[0], "tau": learned[1], "sigma": learned[2], "err": learned[3],
                                  "pred": 10 ** learned[4]}
            if learned is not None and base[3] <= tgt:
                tb = time_transform(x, S, n_mu, d_mu, *base[:3])
                tl = time_transform(x, S, n_mu, d_mu, *learned[:3])
                rec.update(taps_saved=base[0] - learned[0], ms_analytic=tb, ms_learned=tl, speedup=tb / tl)
            yield rec


def evaluate_split(net, log2n=26, S=128, target=1e-6, seed=99, reps=5):
    """The split form at one accuracy target: the default window (B = 72), the
    analytic window and the learned window, each with its measured rel-L2 of the
    split transform against the FP64 direct FFT and its median time.  Windows
    are proposed with the split form's conditioning term and accepted only if
    the split transform itself meets the target.  Yields one dict per
    oversampling pair."""
    import torch
    from . import PRECISION_SPLIT_FP32

    def run(x32, X, n_mu, d_mu, B, tau, sigma):
        d = SoiDescriptor(N=x32.numel(), n_mu=n_mu, d_mu=d_mu, B=int(B), tau=float(tau), sigma=float(sigma),
                          precision=PRECISION_SPLIT_FP32, device=x32.device.index or 0)
        try:
            d.init(S)
            y = torch.empty_like(x32)
            d.compute_into(x32, y)
            ts = []
            for _ in range(reps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                a.record()
                d.compute_into(x32, y)
                b.record()
                torch.cuda.synchronize()
                ts.append(a.elapsed_time(b))
        finally:
            d.free()
        e = float(torch.linalg.norm(y.to(torch.complex128) - X) / torch.linalg.norm(X))
        return e, float(np.median(ts))

    for (n_mu, d_mu) in MU_PAIRS:
        N = length_for(n_mu, d_mu, log2n)
        g = torch.Generator(device="cuda").manual_seed(seed + n_mu)
        x = torch.complex(torch.randn(N, generator=g, device="cuda", dtype=torch.float64),
                          torch.randn(N, generator=g, device="cuda", dtype=torch.float64))
        X = torch.fft.fft(x)
        x32 = x.to(torch.complex64)
        # windows are chosen and verified in the split form itself: a window that
        # is accurate in FP64 can fail in FP32 when its demodulation is
        # ill-conditioned
        measure = lambda B, tau, sigma: measure_error(x, S, n_mu, d_mu, int(B), tau, sigma, X,
                                                      precision=PRECISION_SPLIT_FP32)
        rec = {"mu": "%d/%d" % (n_mu, d_mu), "N": N, "S": S, "target": target}
        wins = {"default": (72, 928 / 1024., 373.7314)}
        base = analytic_window(n_mu, d_mu, target, measure)
        if base[3] <= target:
            wins["analytic"] = base[:3]
        learned = learned_window(net, n_mu, d_mu, target, measure, precision=PRECISION_SPLIT_FP32)
        if learned is not None:
            wins["learned"] = learned[:3]
        for name, (B, tau, sigma) in wins.items():
            e, ms = run(x32, X, n_mu, d_mu, B, tau, sigma)
            rec[name] = {"B": int(B), "tau": tau, "sigma": sigma, "split_rel_l2": e, "ms": ms, "meets": e <= target}
        del x, X, x32
        torch.cuda.empty_cache()
        yield rec


def main():
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the learned-window surrogate on the GPU")
    ap.add_argument("--per-mu", type=int, default=1200)
    ap.add_argument("--log2n", type=int, default=20)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--from-dataset", default=None,
                    help="retrain on the measurements stored in a weights file instead of measuring")
    ap.add_argument("--evaluate", action="store_true",
                    help="evaluate the weights in --out against the analytic window instead of training")
    ap.add_argument("--eval-log2n", type=int, default=26)
    ap.add_argument("--evaluate-split", type=float, default=None, metavar="TARGET",
                    help="time the split form with the default, analytic and learned windows at TARGET")
    a = ap.parse_args()
    if a.evaluate:
        net = WindowMLP.load(a.out)
        for rec in evaluate(net, log2n=a.eval_log2n):
            print(json.dumps(rec), flush=True)
        return
    if a.evaluate_split is not None:
        net = WindowMLP.load(a.out)
        for rec in evaluate_split(net, log2n=a.eval_log2n, target=a.evaluate_split):
            print(json.dumps(rec), flush=True)
        return
    if a.from_dataset:
        z = np.load(a.from_dataset)
        x, y = z["dataset_x"], z["dataset_y"]
    else:
        x, y, raw = make_dataset(per_mu=a.per_mu, log2n=a.log2n)
    y = clip_target(y).astype(np.float32)
    net = WindowMLP(seed=1)
    hist = net.train(x, y, steps=a.steps)
    net.save(a.out, dataset_x=x, dataset_y=y, loss_history=np.array(hist))
    print(json.dumps({"samples": int(len(y)), "loss_first": hist[0], "loss_last": hist[-1]}))


if __name__ == "__main__":
    main()
