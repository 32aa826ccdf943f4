"""Segments of interest (soi_compute_segments_status), the non-waiting compute
(soi_compute_async_status + soi_check_status) and its capture into a CUDA
graph.  The segment outputs must be bit-identical to the same segments of a
full compute (same kernels, same arithmetic), and nothing outside the band
may be written."""
import numpy as np
import pytest

import soi_fft_b200 as sb
from tests import signals

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

# (N, S, precision): the two-kernel stage 2 (small M'), and the persistent
# stage 2 in both precisions (M' = 320 x 256 and 320 x 512)
SHAPES = [
    (1 << 16, 8, sb.PRECISION_FP64),
    (1 << 20, 16, sb.PRECISION_SPLIT_FP32),
    (1 << 20, 8, sb.PRECISION_FP64),
    (1 << 22, 32, sb.PRECISION_SPLIT_FP32),
]


def _input(N, prec, seed=7):
    x = signals.gaussian(N, seed)
    if prec == sb.PRECISION_SPLIT_FP32:
        x = x.astype(np.complex64)
    return torch.from_numpy(x).cuda()


def _desc(N, S, prec, **kw):
    return sb.SoiDescriptor(N=N, precision=prec, **kw).init(S)


@pytest.mark.parametrize("N,S,prec", SHAPES)
@pytest.mark.parametrize("band", [(0, 1), (3, 5), "last", "all"])
def test_segments_are_bit_identical_to_full_compute(N, S, prec, band):
    x = _input(N, prec)
    d = _desc(N, S, prec)
    try:
        full = torch.empty_like(x)
        d.compute_into(x, full)
        lo, hi = (S - 2, S) if band == "last" else (0, S) if band == "all" else band
        M = N // S
        sentinel = torch.full_like(x, complex(1234.5, -77.25))
        part = sentinel.clone()
        d.compute_segments(x, part, lo, hi)
        torch.cuda.synchronize()
        assert torch.equal(part[lo * M:hi * M], full[lo * M:hi * M])
        assert torch.equal(part[:lo * M], sentinel[:lo * M])
        assert torch.equal(part[hi * M:], sentinel[hi * M:])
        # a full compute after a band compute is unaffected by the band's state
        again = torch.empty_like(x)
        d.compute_into(x, again)
        assert torch.equal(again, full)
    finally:
        d.free()


def test_segments_with_host_buffers():
    N, S, prec = 1 << 18, 16, sb.PRECISION_SPLIT_FP32
    x = signals.gaussian(N, 3).astype(np.complex64)
    d = _desc(N, S, prec)
    try:
        full = np.empty_like(x)
        d.compute_into(x, full)
        part = np.zeros_like(x)
        d.compute_segments(x, part, 5, 9)
        M = N // S
        assert np.array_equal(part[5 * M:9 * M], full[5 * M:9 * M])
        assert not part[:5 * M].any() and not part[9 * M:].any()
    finally:
        d.free()


def test_segment_range_is_checked():
    N, S, prec = 1 << 16, 8, sb.PRECISION_FP64
    x = _input(N, prec)
    d = _desc(N, S, prec)
    try:
        y = torch.empty_like(x)
        for lo, hi in [(-1, 2), (3, 3), (5, 4), (0, S + 1)]:
            with pytest.raises(sb.SoiError):
                d.compute_segments(x, y, lo, hi)
    finally:
        d.free()


@pytest.mark.parametrize("N,S,prec", SHAPES)
def test_async_compute_matches_and_checks(N, S, prec):
    x = _input(N, prec)
    d = _desc(N, S, prec)
    try:
        ref = torch.empty_like(x)
        d.compute_into(x, ref)
        y = torch.empty_like(x)
        d.compute_async(x, y)
        d.check()
        assert torch.equal(y, ref)
    finally:
        d.free()


@pytest.mark.parametrize("N,S,prec", [(1 << 20, 16, sb.PRECISION_SPLIT_FP32), (1 << 20, 8, sb.PRECISION_FP64)])
def test_async_compute_captures_into_a_cuda_graph(N, S, prec):
    s = torch.cuda.Stream()
    x = _input(N, prec)
    d = _desc(N, S, prec, stream=s.cuda_stream)
    try:
        ref = torch.empty_like(x)
        d.compute_into(x, ref)
        torch.cuda.synchronize()
        y = torch.zeros_like(x)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            d.compute_async(x, y)
        for _ in range(3):
            y.zero_()
            g.replay()
            torch.cuda.synchronize()
            d.check()
            assert torch.equal(y, ref)
        del g
    finally:
        d.free()


def test_stage2_wait_that_runs_out_reports_timeout_and_leaves_the_gpu_usable(monkeypatch):
    # failure detection without a fault: the plan is told to wait for one more
    # pass-1 completion than exists, so every pass-2 wait gives up after its
    # iteration limit; the kernel returns, the host reads the error flag
    N, S, prec = 1 << 20, 16, sb.PRECISION_SPLIT_FP32
    x = _input(N, prec)
    monkeypatch.setenv("SOI_TEST_STAGE2_WAIT_EXTRA", "1")
    d = _desc(N, S, prec)
    monkeypatch.delenv("SOI_TEST_STAGE2_WAIT_EXTRA")
    try:
        y = torch.empty_like(x)
        with pytest.raises(sb.SoiError) as e:
            d.compute_into(x, y)
        assert e.value.status == 5          # SOI_ERR_TIMEOUT
    finally:
        d.free()
    d2 = _desc(N, S, prec)
    try:
        y = torch.empty_like(x)
        d2.compute_into(x, y)
        X = torch.fft.fft(x.to(torch.complex128))
        assert float(torch.linalg.norm(y.to(torch.complex128) - X) / torch.linalg.norm(X)) < 1e-6
    finally:
        d2.free()


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("N,S,prec", [(1 << 20, 16, sb.PRECISION_SPLIT_FP32), (1 << 18, 8, sb.PRECISION_FP64)])
def test_streamed_host_transforms_equal_single_computes(N, S, prec, pinned):
    dt = np.complex64 if prec == sb.PRECISION_SPLIT_FP32 else np.complex128
    tdt = torch.complex64 if prec == sb.PRECISION_SPLIT_FP32 else torch.complex128

    def host(a):
        if not pinned:
            return np.ascontiguousarray(a)
        t = torch.empty(a.size, dtype=tdt, pin_memory=True)
        v = t.numpy()
        v[:] = a
        return v

    xs = [host(signals.gaussian(N, 20 + i).astype(dt)) for i in range(5)]
    ys = [host(np.zeros(N, dt)) for _ in range(5)]
    d = _desc(N, S, prec)
    try:
        d.compute_stream(xs, ys)
        for x, y in zip(xs, ys):
            ref = np.empty_like(x)
            d.compute_into(x, ref)
            assert np.array_equal(y, ref)
    finally:
        d.free()


@pytest.mark.parametrize("N,S,prec,tol", [(1 << 20, 16, sb.PRECISION_SPLIT_FP32, 1e-6),
                                          (1 << 18, 8, sb.PRECISION_FP64, 1e-12),
                                          (1 << 22, 32, sb.PRECISION_SPLIT_FP32, 1e-6)])
def test_inverse_matches_direct_inverse_fft_and_round_trips(N, S, prec, tol):
    x = _input(N, prec)
    d = _desc(N, S, prec)
    try:
        y = torch.empty_like(x)
        d.compute_inverse(x, y)
        ref = torch.fft.ifft(x.to(torch.complex128))
        assert float(torch.linalg.norm(y.to(torch.complex128) - ref) / torch.linalg.norm(ref)) <= tol
        # forward then inverse returns the input
        X = torch.empty_like(x)
        d.compute_into(x, X)
        back = torch.empty_like(x)
        d.compute_inverse(X, back)
        assert float(torch.linalg.norm((back - x).to(torch.complex128)) / torch.linalg.norm(x.to(torch.complex128))) <= 2 * tol
        # host buffers
        xh = x.cpu().numpy()
        yh = np.empty_like(xh)
        d.compute_inverse(xh, yh)
        assert np.array_equal(yh, y.cpu().numpy())
    finally:
        d.free()


def test_misaligned_device_input_is_rejected():
    N, S, prec = 1 << 16, 8, sb.PRECISION_SPLIT_FP32
    d = _desc(N, S, prec)
    try:
        big = torch.zeros(N + 1, dtype=torch.complex64, device="cuda")
        x = big[1:]                                   # 8-byte aligned only
        y = torch.empty(N, dtype=torch.complex64, device="cuda")
        with pytest.raises(sb.SoiError) as e:
            d.compute_into(x, y)
        assert e.value.status == 1                    # SOI_ERR_INVALID
        x2 = big[:N]
        d.compute_into(x2, y)                         # the aligned view works
    finally:
        d.free()


@pytest.mark.parametrize("N,S,prec,nt", [(1 << 16, 8, sb.PRECISION_SPLIT_FP32, "512"),
                                         (1 << 18, 8, sb.PRECISION_SPLIT_FP32, "256"),
                                         (1 << 20, 16, sb.PRECISION_SPLIT_FP32, "512"),
                                         (1 << 22, 128, sb.PRECISION_SPLIT_FP32, "512"),
                                         (1 << 22, 128, sb.PRECISION_SPLIT_FP32, "256"),
                                         (1 << 24, 256, sb.PRECISION_SPLIT_FP32, "512"),
                                         (1 << 18, 8, sb.PRECISION_FP64, "512"),
                                         (1 << 22, 128, sb.PRECISION_FP64, "512"),
                                         (1 << 20, 64, sb.PRECISION_FP64, "256")])
def test_bulk_copy_staging_equals_cp_async_staging(N, S, prec, nt, monkeypatch):
    # the two ways of staging stage 1's input rows (per-thread cp.async, or a
    # tensor copy per phase with row-by-row bulk copies for the tiles whose
    # rows wrap around the input) feed identical arithmetic
    x = _input(N, prec)
    outs = []
    monkeypatch.setenv("SOI_STAGE1_NT", nt)
    for bulk in ("0", "1"):
        monkeypatch.setenv("SOI_STAGE1_BULK", bulk)
        d = _desc(N, S, prec)
        try:
            y = torch.empty_like(x)
            d.compute_into(x, y)
            torch.cuda.synchronize()
            outs.append(y)
        finally:
            d.free()
    assert torch.equal(outs[0], outs[1])


@pytest.mark.parametrize("N,S,prec", [(1 << 20, 16, sb.PRECISION_SPLIT_FP32), (1 << 22, 32, sb.PRECISION_SPLIT_FP32),
                                      (1 << 26, 128, sb.PRECISION_SPLIT_FP32), (1 << 20, 8, sb.PRECISION_FP64),
                                      (1 << 24, 64, sb.PRECISION_FP64)])
@pytest.mark.parametrize("band", ["all", (3, 7)])
def test_tensor_copy_staging_equals_cp_async_staging(N, S, prec, band, monkeypatch):
    # the persistent stage 2 stages pass-1 tiles by tensor copies (a swizzled
    # dense tile) or by cp.async (a padded tile): the same arithmetic on the
    # same values, so the outputs are identical (pass 2 with one row per
    # thread in both; its row-pair threads are compared to rounding elsewhere)
    x = _input(N, prec)
    lo, hi = (0, S) if band == "all" else band
    outs = []
    monkeypatch.setenv("SOI_STAGE2_ROWS2", "0")
    for tma in ("1", "0"):
        monkeypatch.setenv("SOI_STAGE2_TMA", tma)
        d = _desc(N, S, prec)
        try:
            y = torch.zeros_like(x)
            d.compute_segments(x, y, lo, hi)
            torch.cuda.synchronize()
            outs.append(y)
        finally:
            d.free()
    assert torch.equal(outs[0], outs[1])


@pytest.mark.parametrize("N,S,prec", [(1 << 22, 32, sb.PRECISION_SPLIT_FP32), (1 << 20, 8, sb.PRECISION_FP64)])
@pytest.mark.parametrize("band", ["all", (2, 5)])
def test_stage2_schedule_does_not_change_results(N, S, prec, band, monkeypatch):
    # the persistent stage 2's task order (how pass 1 of the next segment is
    # interleaved with pass 2 of the current one) only moves work in time
    x = _input(N, prec)
    lo, hi = (0, S) if band == "all" else band
    outs = []
    for tail in ("0", "7", None):
        if tail is None:
            monkeypatch.delenv("SOI_STAGE2_TAIL", raising=False)
        else:
            monkeypatch.setenv("SOI_STAGE2_TAIL", tail)
        d = _desc(N, S, prec)
        try:
            y = torch.zeros_like(x)
            d.compute_segments(x, y, lo, hi)
            torch.cuda.synchronize()
            outs.append(y)
        finally:
            d.free()
    assert torch.equal(outs[0], outs[2]) and torch.equal(outs[1], outs[2])


@pytest.mark.parametrize("N,S,prec", [(1 << 20, 16, sb.PRECISION_SPLIT_FP32), (1 << 22, 32, sb.PRECISION_SPLIT_FP32),
                                      (1 << 27, 32, sb.PRECISION_SPLIT_FP32), (1 << 20, 8, sb.PRECISION_FP64),
                                      (1 << 22, 16, sb.PRECISION_FP64), (1 << 26, 16, sb.PRECISION_FP64)])
@pytest.mark.parametrize("band", ["all", (3, 7)])
def test_bulk_copied_pass2_rows_equal_cp_async_rows(N, S, prec, band, monkeypatch):
    # pass-2 rows by bulk copies (dense rows, the last radix reading in an XOR
    # order) or by cp.async (a padded tile): the same arithmetic on the same
    # values, so the outputs are identical
    x = _input(N, prec)
    lo, hi = (0, S) if band == "all" else band
    outs = []
    for bulk in ("1", "0"):
        monkeypatch.setenv("SOI_STAGE2_BULK2", bulk)
        monkeypatch.setenv("SOI_STAGE2_ROWS2", "0")
        d = _desc(N, S, prec)
        try:
            y = torch.zeros_like(x)
            d.compute_segments(x, y, lo, hi)
            torch.cuda.synchronize()
            outs.append(y)
        finally:
            d.free()
    assert torch.equal(outs[0], outs[1])


@pytest.mark.parametrize("N,S", [(1 << 20, 16), (1 << 22, 32), (1 << 27, 32)])
@pytest.mark.parametrize("band", ["all", (3, 7)])
def test_row_pair_pass2_agrees_with_single_rows(N, S, band, monkeypatch):
    # FP32 pass 2 with each thread on a pair of rows (tile_fft_rows2) against
    # one row per thread: the same products, whose fused multiply-adds the
    # compiler may pair differently, so the outputs agree to rounding (the
    # split form's own error against the exact DFT is ~3.6e-7), and both meet
    # the split tolerance against the FP64 oracle
    prec = sb.PRECISION_SPLIT_FP32
    x = _input(N, prec)
    lo, hi = (0, S) if band == "all" else band
    outs = []
    for rows2 in ("0", "1"):
        monkeypatch.setenv("SOI_STAGE2_ROWS2", rows2)
        d = _desc(N, S, prec)
        try:
            y = torch.zeros_like(x)
            d.compute_segments(x, y, lo, hi)
            torch.cuda.synchronize()
            outs.append(y.to(torch.complex128))
        finally:
            d.free()
    M = N // S
    a, b = outs[0][lo * M:hi * M], outs[1][lo * M:hi * M]
    assert float(torch.linalg.norm(a - b) / torch.linalg.norm(a)) <= 5e-7
    assert torch.equal(outs[0][:lo * M], outs[1][:lo * M]) and torch.equal(outs[0][hi * M:], outs[1][hi * M:])
    X = torch.fft.fft(x.to(torch.complex128))[lo * M:hi * M]
    for y in (a, b):
        assert float(torch.linalg.norm(y - X) / torch.linalg.norm(X)) <= 1e-6


def test_output_aligned_to_eight_bytes_only_is_written_by_single_rows():
    # pass-2 row pairs store 16 bytes at a time; an output view aligned to 8
    # bytes only takes the one-row-per-thread stores (results equal to
    # rounding, both within the split tolerance)
    N, S, prec = 1 << 22, 32, sb.PRECISION_SPLIT_FP32
    x = _input(N, prec)
    d = _desc(N, S, prec)
    try:
        y = torch.empty_like(x)
        d.compute_into(x, y)
        big = torch.zeros(N + 1, dtype=torch.complex64, device="cuda")
        y8 = big[1:]
        d.compute_into(x, y8)
        torch.cuda.synchronize()
        a, b = y.to(torch.complex128), y8.to(torch.complex128)
        assert float(torch.linalg.norm(a - b) / torch.linalg.norm(a)) <= 5e-7
        X = torch.fft.fft(x.to(torch.complex128))
        assert float(torch.linalg.norm(b - X) / torch.linalg.norm(X)) <= 1e-6
    finally:
        d.free()
