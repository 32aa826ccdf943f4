"""The batch driver (soi_batch_*): a band-limited batch of transforms of
mixed lengths replayed as one CUDA graph.  Untuned batches must equal the
single-descriptor segments-of-interest compute bit for bit (same kernels);
tuned batches may pick other kernel variants, so they are checked against the
FP64 direct FFT on the band's segments at the precision's tolerance."""
import numpy as np
import pytest

import soi_fft_b200 as sb

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from soi_fft_b200 import batch as sbb  # noqa: E402

SPLIT_TOL, FP64_TOL = 1e-6, 1e-12


def _items(wl, inplace=False):
    outs = []
    for w in wl:
        y = w["x"] if inplace else torch.full_like(w["x"], complex(-3.0, 5.0))
        outs.append(y)
    return outs


def _single(w, prec, use_vlc=False):
    """The same band through one descriptor (reference for untuned batches)."""
    d = sb.SoiDescriptor(N=w["N"], precision=prec, use_vlc=int(use_vlc)).init(w["k"])
    try:
        y = torch.full_like(w["x"], complex(-3.0, 5.0))
        d.compute_segments(w["x"], y, w["seg_lo"], w["seg_hi"])
        torch.cuda.synchronize()
        return y
    finally:
        d.free()


@pytest.mark.parametrize("prec", [sb.PRECISION_SPLIT_FP32, sb.PRECISION_FP64])
def test_untuned_batch_equals_single_transforms(prec):
    wl = sbb.band_workload(24, 14, 19, seed=3, precision=prec)
    outs = _items(wl)
    b = sbb.SoiBatch([(w["x"], y, w["k"], w["seg_lo"], w["seg_hi"]) for w, y in zip(wl, outs)],
                     precision=prec, chains=3, tune=False)
    try:
        info = b.info()
        assert info["transforms"] == len(wl) and info["chains"] == 3 and info["graph_nodes"] > len(wl)
        for rep in range(2):
            for y in outs:
                y.fill_(complex(-3.0, 5.0))
            b.execute()
            b.check()
            for w, y in zip(wl, outs):
                assert torch.equal(y, _single(w, prec)), (w["N"], w["k"], rep)
    finally:
        b.free()


@pytest.mark.parametrize("prec,tol", [(sb.PRECISION_SPLIT_FP32, SPLIT_TOL), (sb.PRECISION_FP64, FP64_TOL)])
def test_tuned_batch_matches_direct_fft_on_the_band(prec, tol):
    wl = sbb.band_workload(16, 14, 20, seed=5, precision=prec)
    outs = _items(wl, inplace=True)
    refs = [torch.fft.fft(w["x"].to(torch.complex128)) for w in wl]
    b = sbb.SoiBatch([(w["x"], y, w["k"], w["seg_lo"], w["seg_hi"]) for w, y in zip(wl, outs)],
                     precision=prec, chains=4, tune=True)
    try:
        plans = b.plans()
        assert len(plans) == len({(w["N"], w["k"]) for w in wl})
        b.execute()
        b.check()
        for w, y, X in zip(wl, outs, refs):
            M = w["N"] // w["k"]
            sl = slice(w["seg_lo"] * M, w["seg_hi"] * M)
            e = float(torch.linalg.norm(y[sl].to(torch.complex128) - X[sl]) / torch.linalg.norm(X[sl]))
            assert e <= tol, (w["N"], w["k"], e)
    finally:
        b.free()


def test_vlc_batch_equals_single_transforms():
    prec = sb.PRECISION_FP64
    wl = sbb.band_workload(6, 14, 17, seed=9, precision=prec)
    outs = _items(wl)
    b = sbb.SoiBatch([(w["x"], y, w["k"], w["seg_lo"], w["seg_hi"]) for w, y in zip(wl, outs)],
                     precision=prec, chains=2, tune=False, use_vlc=True)
    try:
        assert b.info()["chains"] == 1
        b.execute()
        b.check()
        for w, y in zip(wl, outs):
            assert torch.equal(y, _single(w, prec, use_vlc=True))
    finally:
        b.free()


def test_full_segment_items_and_mixed_shapes():
    prec = sb.PRECISION_SPLIT_FP32
    wl = sbb.band_workload(5, 16, 22, seed=11, precision=prec)
    outs = _items(wl)
    b = sbb.SoiBatch([(w["x"], y, w["k"], 0, 0) for w, y in zip(wl, outs)], precision=prec, chains=2, tune=False)
    try:
        b.execute()
        b.check()
        for w, y in zip(wl, outs):
            d = sb.SoiDescriptor(N=w["N"], precision=prec).init(w["k"])
            try:
                ref = torch.empty_like(w["x"])
                d.compute_into(w["x"], ref)
                torch.cuda.synchronize()
            finally:
                d.free()
            assert torch.equal(y, ref)
    finally:
        b.free()


def test_batch_rejects_bad_items():
    x = torch.zeros(1 << 14, dtype=torch.complex64, device="cuda")
    for k, lo, hi in [(4, 3, 2), (4, 0, 5), (7, 0, 0)]:
        with pytest.raises(sb.SoiError):
            sbb.SoiBatch([(x, x, k, lo, hi)], tune=False)
