"""Parity of the CUDA path (through the C ABI) with the oracle.

Plain FP64: rel-L2 <= 1e-12 against the oracle (the reference's algorithm,
bit-identical to the reference's own sources).  Split precision (complex64
storage, FP32 arithmetic): rel-L2 <= 1e-6 against an FP64 direct FFT."""
import numpy as np
import pytest

import soi_fft_b200 as sb
from oracle import oracle
from tests.conftest import rel_l2
from tests import signals

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

FP64_TOL = 1e-12
SPLIT_TOL = 1e-6


def on_gpu(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def max_err(y, ref):
    # compute_normalized_inf_norm, input.c:395-425
    return float(np.sqrt(np.max(np.abs(y - ref) ** 2) / np.max(np.abs(ref) ** 2)))


CASES = [  # N, S, n_mu, d_mu, B, tau, sigma
    (1 << 14, 4, 5, 4, 72, None, None),
    (1 << 16, 8, 5, 4, 72, None, None),
    (1 << 18, 16, 5, 4, 72, None, None),
    (1 << 18, 64, 5, 4, 72, None, None),
    (1 << 20, 8, 5, 4, 72, None, None),      # the reference's CPU case: N=2^20, S=8
    (1 << 20, 128, 5, 4, 72, None, None),
    (1 << 17, 32, 5, 4, 44, 512 / 1024, 121.0936),   # Pareto point pfft.c:121
    (1 << 17, 16, 5, 4, 60, 0.899, 352.7647081),     # pfft.c:115
    (7 << 14, 8, 8, 7, 72, None, None),      # mu = 8/7 (.cpp:540)
    (1 << 18, 16, 9, 8, 72, 0.7238, 476.8683),   # mu = 9/8 (not dispatched by the reference)
    (3 << 16, 12, 5, 4, 72, None, None),     # S not a power of two
]


def _kw(n, d, B, tau, sigma):
    kw = dict(n_mu=n, d_mu=d, B=B)
    if tau is not None:
        kw.update(tau=tau, sigma=sigma)
    return kw


def _winv_conditioning(N, S, n, d, B, tau, sigma):
    kw = _kw(n, d, B, tau, sigma)
    return float(np.abs(sb.window_tables(N, S, **kw)[2]).max())


@pytest.mark.parametrize("case", CASES, ids=lambda c: "N%d_S%d_mu%d-%d_B%d" % c[:5])
def test_fp64_matches_oracle(case):
    N, S, n, d, B, tau, sigma = case
    x = signals.gaussian(N, N ^ S)
    kw = _kw(n, d, B, tau, sigma)
    ref = oracle.compute_soi(x, S, **kw)
    y = sb.soi_fft(on_gpu(x), S, **kw).cpu().numpy()
    X = np.fft.fft(x)
    # never less accurate than the reference against the exact DFT
    assert rel_l2(y, X) <= 1.05 * rel_l2(ref, X) + 1e-14
    if _winv_conditioning(N, S, n, d, B, tau if tau else 928 / 1024., sigma if sigma else 373.7314) <= 1e3:
        assert rel_l2(y, ref) <= FP64_TOL
        assert max_err(y, ref) <= 10 * FP64_TOL
    else:
        # Narrow windows (max|W_inv| > 1e3): the reference rounds t in double
        # when tabulating w (pfft.c:52); W_inv amplifies that ~1e-15 error to
        # >1e-12 at the segment edges.  The tables here use the exact rational
        # t, so the difference is the reference's rounding, not ours.
        assert rel_l2(y, ref) <= 1e-10


SPLIT_CASES = [c for c in CASES[:8] if c[4] != 44]


@pytest.mark.parametrize("case", SPLIT_CASES, ids=lambda c: "N%d_S%d_B%d" % (c[0], c[1], c[4]))
def test_split_fp32_vs_fp64_direct_fft(case):
    # The split form's error is about eps32 * max|W_inv|: the demodulation
    # multiplies by W_inv (pfft.c:653-660), up to 9 for the default window but
    # 1e4 for B=44/tau=0.5 (pfft.c:121), where FP32 cannot reach 1e-6; those
    # narrow windows are for the FP64 form only.
    N, S, n, d, B, tau, sigma = case
    x = signals.gaussian_plus_tones(N, 3 * N + S)
    X = np.fft.fft(x)
    y = sb.soi_fft(on_gpu(x.astype(np.complex64)), S, **_kw(n, d, B, tau, sigma)).cpu().numpy()
    assert y.dtype == np.complex64
    # the input itself is rounded to complex64 once; the bound covers that too
    assert rel_l2(y.astype(np.complex128), X) <= SPLIT_TOL


@pytest.mark.parametrize("prec", [sb.PRECISION_FP64, sb.PRECISION_SPLIT_FP32])
def test_host_pointer_equals_device_pointer(prec):
    N, S = 1 << 18, 16
    dt = np.complex128 if prec == sb.PRECISION_FP64 else np.complex64
    x = signals.gaussian(N, 5, dt)
    d = sb.SoiDescriptor(N=N, precision=prec).init(S)
    yh = d.compute(x.copy())
    yd = d.compute(on_gpu(x)).cpu().numpy()
    d.free()
    assert np.array_equal(yh, yd)


def test_stage1_transposed_matches_oracle():
    N, S = 1 << 18, 32
    x = signals.gaussian(N, 17)
    d = sb.SoiDescriptor(N=N).init(S)
    T = d.filter_subsampling(x.copy())
    d.free()
    Tref = oracle.transposed(x, S)
    assert T.shape == Tref.shape
    assert rel_l2(T, Tref) <= 1e-13


def test_repeated_compute_is_deterministic():
    N, S = 1 << 18, 16
    x = signals.gaussian(N, 8)
    d = sb.SoiDescriptor(N=N).init(S)
    a = d.compute(on_gpu(x)).cpu().numpy()
    b = d.compute(on_gpu(x)).cpu().numpy()
    d.free()
    assert np.array_equal(a, b)


def test_edge_inputs():
    N, S = 1 << 16, 8
    d = sb.SoiDescriptor(N=N).init(S)
    z = d.compute(np.zeros(N, np.complex128))
    assert not np.any(z)
    # a delta at 0 transforms to all ones
    e = np.zeros(N, np.complex128)
    e[0] = 1
    assert rel_l2(d.compute(e), np.ones(N, np.complex128)) <= FP64_TOL
    # a pure on-bin tone transforms to a single spike
    k0 = 12345
    t = np.exp(2j * np.pi * ((k0 * np.arange(N)) % N) / N)   # phase reduced exactly
    Y = d.compute(t)
    ref = np.zeros(N, np.complex128)
    ref[k0] = N
    assert rel_l2(Y, ref) <= FP64_TOL
    d.free()


def test_split_error_scales_with_window_conditioning():
    # documents the limit stated above: a narrow window in FP32
    N, S = 1 << 17, 32
    x = signals.gaussian(N, 1)
    X = np.fft.fft(x)
    kw = dict(B=44, tau=512 / 1024, sigma=121.0936)
    y = sb.soi_fft(on_gpu(x.astype(np.complex64)), S, **kw).cpu().numpy().astype(np.complex128)
    cond = float(np.abs(sb.window_tables(N, S, **kw)[2]).max())
    assert cond > 1e3
    assert rel_l2(y, X) <= 50 * cond * 6e-8


def test_smallest_and_largest_segment_counts():
    for N, S in ((1 << 13, 2), (1 << 20, 256)):
        x = signals.gaussian(N, S)
        y = sb.soi_fft(on_gpu(x), S).cpu().numpy()
        assert rel_l2(y, oracle.compute_soi(x, S)) <= FP64_TOL


@pytest.mark.parametrize("N,S", [(1 << 24, 64), (1 << 26, 128)])
def test_large_sizes_against_cufft(N, S):
    # size-independent checks at sizes the CPU oracle is slow for: the FP64
    # direct FFT is cuFFT's Z2Z (called as a library, as the checker only)
    xd = signals.gaussian_plus_tones_torch(N, N + 1)
    X = torch.fft.fft(xd)
    y64 = sb.soi_fft(xd, S)
    assert float(torch.linalg.norm(y64 - X) / torch.linalg.norm(X)) <= FP64_TOL
    y32 = sb.soi_fft(xd.to(torch.complex64), S).to(torch.complex128)
    assert float(torch.linalg.norm(y32 - X) / torch.linalg.norm(X)) <= SPLIT_TOL
    # linearity of the FP64 path: T(a x + b u) = a T(x) + b T(u)
    u = signals.gaussian_plus_tones_torch(N, 2)
    a, b = 0.3 - 1.1j, 2.0 + 0.5j
    lhs = sb.soi_fft(a * xd + b * u, S)
    rhs = a * y64 + b * sb.soi_fft(u, S)
    assert float(torch.linalg.norm(lhs - rhs) / torch.linalg.norm(rhs)) <= FP64_TOL


@pytest.mark.parametrize("N,S,prec", [(1 << 28, 64, "fp64"), (1 << 29, 128, "split")])
def test_configured_sizes_against_cufft(N, S, prec):
    # the configured workloads at full size: plain FP64 at N = 2^28, P = 64 and
    # the split form at N = 2^29, P = 128, on Gaussian + 64 tones, against the
    # FP64 direct FFT (cuFFT Z2Z, the checker)
    xd = signals.gaussian_plus_tones_torch(N, 7)
    X = torch.fft.fft(xd)
    nX = torch.linalg.norm(X)
    if prec == "fp64":
        y = sb.soi_fft(xd, S)
        assert float(torch.linalg.norm(y - X) / nX) <= FP64_TOL
    else:
        x32 = xd.to(torch.complex64)
        del xd
        y = sb.soi_fft(x32, S).to(torch.complex128)
        assert float(torch.linalg.norm(y - X) / nX) <= SPLIT_TOL
    del X, y
    torch.cuda.empty_cache()


def test_timings_reported():
    N, S = 1 << 20, 16
    d = sb.SoiDescriptor(N=N, precision=sb.PRECISION_SPLIT_FP32).init(S)
    d.set_timing(True)
    d.compute(on_gpu(signals.gaussian(N, 1, np.complex64)))
    t = d.timings()
    d.free()
    assert t["stage1_ms"] > 0 and t["stage2_ms"] > 0 and t["total_ms"] >= t["stage1_ms"]


@pytest.mark.parametrize("prec", [sb.PRECISION_FP64, sb.PRECISION_SPLIT_FP32])
def test_out_of_place_leaves_input_and_matches_in_place(prec):
    N, S = 1 << 18, 32
    dt = np.complex128 if prec == sb.PRECISION_FP64 else np.complex64
    x = signals.gaussian(N, 9, dt)
    d = sb.SoiDescriptor(N=N, precision=prec).init(S)
    xd = on_gpu(x)
    out = torch.empty_like(xd)
    d.compute_into(xd, out)
    assert np.array_equal(xd.cpu().numpy(), x)
    inplace = d.compute(on_gpu(x)).cpu().numpy()
    host_out = np.empty_like(x)
    d.compute_into(x, host_out)
    d.free()
    assert np.array_equal(out.cpu().numpy(), inplace)
    assert np.array_equal(host_out, inplace)


@pytest.mark.parametrize("prec,tol", [(sb.PRECISION_FP64, 1e-13), (sb.PRECISION_SPLIT_FP32, 2e-6)])
@pytest.mark.parametrize("N,S", [(1 << 20, 8), (1 << 22, 128), (1 << 18, 64)])
def test_fast_paths_agree_with_fallback_kernels(prec, tol, N, S, monkeypatch):
    dt = np.complex128 if prec == sb.PRECISION_FP64 else np.complex64
    x = on_gpu(signals.gaussian(N, 21, dt))
    outs = []
    for fast in ("1", "0"):
        monkeypatch.setenv("SOI_STAGE1_FAST", fast)
        monkeypatch.setenv("SOI_STAGE2_FAST", fast)
        d = sb.SoiDescriptor(N=N, precision=prec).init(S)
        outs.append(d.compute(x.clone()).cpu().numpy().astype(np.complex128))
        d.free()
    assert rel_l2(outs[0], outs[1]) <= tol


@pytest.mark.parametrize("prec,tol", [(sb.PRECISION_FP64, 1e-13), (sb.PRECISION_SPLIT_FP32, 2e-6)])
@pytest.mark.parametrize("N,S,n,d", [(7 << 23, 128, 8, 7), (1 << 26, 128, 9, 8)])
def test_other_oversampling_persistent_stage2_agrees_with_fallback(prec, tol, N, S, n, d, monkeypatch):
    # mu = 8/7 (M' = 512 x 1024) and 9/8 (M' = 1152 x 512, a radix-9 register
    # stage) on the persistent stage 2, against the two-kernel stage 2; both
    # against the FP64 direct FFT at the default window's own accuracy for
    # these oversamplings (~1e-7 for 8/7, ~1e-6 for 9/8)
    dt = np.complex128 if prec == sb.PRECISION_FP64 else np.complex64
    xh = signals.gaussian(N, 23, dt)
    x = on_gpu(xh)
    X = torch.fft.fft(x.to(torch.complex128)).cpu().numpy()
    outs = []
    for fast in ("1", "0"):
        monkeypatch.setenv("SOI_STAGE2_FAST", fast)
        desc = sb.SoiDescriptor(N=N, precision=prec, n_mu=n, d_mu=d).init(S)
        outs.append(desc.compute(x.clone()).cpu().numpy().astype(np.complex128))
        desc.free()
    errs = [rel_l2(o, X) for o in outs]
    assert max(errs) <= 3e-6, errs
    assert rel_l2(outs[0], outs[1]) <= tol


@pytest.mark.parametrize("side_stream", [False, True])
def test_input_written_just_before_the_call_is_read_complete(side_stream):
    # the input is filled by an asynchronous device copy queued right before
    # the call (on torch's default stream, or on a side stream) over a buffer
    # that held NaN; the library's own stream must not start stage 1 before the
    # copy ends.  A first compute loads the kernels, so nothing delays the
    # launches that follow.
    N, S, prec = 1 << 26, 128, sb.PRECISION_SPLIT_FP32
    x = on_gpu(signals.gaussian(N, 31, np.complex64))
    X = torch.fft.fft(x.to(torch.complex128))
    buf = torch.empty_like(x)
    desc = sb.SoiDescriptor(N=N, precision=prec).init(S)
    try:
        desc.compute(x.clone())
        s = torch.cuda.Stream() if side_stream else torch.cuda.current_stream()
        for _ in range(3):
            torch.view_as_real(buf).fill_(float("nan"))
            torch.cuda.synchronize()
            with torch.cuda.stream(s):
                buf.copy_(x)
                desc.compute(buf)
            torch.cuda.synchronize()
            e = float(torch.linalg.norm(buf.to(torch.complex128) - X) / torch.linalg.norm(X))
            assert e <= 1e-6, e
    finally:
        desc.free()


def test_fp64_first_plan_in_a_fresh_process():
    # every plan must set up all device tables it uses: an FP64 plan made
    # first in a process (no split-form plan before it) must be exact
    import subprocess
    import sys
    import os
    code = ("import numpy as np, soi_fft_b200 as sb\n"
            "from oracle import oracle\n"
            "from tests import signals\n"
            "for N, S in ((1 << 16, 8), (1 << 18, 32), (1 << 18, 64)):\n"
            "    x = signals.gaussian(N, 5)\n"
            "    y = sb.soi_fft(x, S)\n"
            "    r = oracle.compute_soi(x, S)\n"
            "    e = np.linalg.norm(y - r) / np.linalg.norm(r)\n"
            "    assert e < 1e-12, (N, S, e)\n"
            "print('ok')\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-2000:]
