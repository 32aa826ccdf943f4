"""The allocation-free VLC round trip, soi_vlc_roundtrip_noalloc_device.

Some callers cannot call cudaMalloc: a process whose device memory is already
reserved by its own pool allocator, or a latency-critical loop that must not
pay cudaMalloc's device-wide synchronisation.  For them the library offers one
entry point whose scratch is a static device array.  This test calls it through
the C ABI twice in a row, on different inputs, and checks each result against
the round trip built from the existing entry points (max_exponent, compress,
decompress with caller-provided buffers).  The VLC stream is bit-exact, so the
comparison is bit-for-bit.  This file is named to be collected last."""
import ctypes

import numpy as np
import pytest

import soi_fft_b200 as sb

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def existing_round_trip(xd, ln, nchunks):
    L = sb.lib()
    emax = torch.zeros(nchunks, dtype=torch.int32, device="cuda")
    assert L.soi_vlc_max_exponent_device(ptr(xd), ln, nchunks, ptr(emax), None) == 0
    torch.cuda.synchronize()
    g = int(emax.max().item())
    stride = L.soi_vlc_words(ln, 0, 0)
    words = torch.zeros(nchunks * stride, dtype=torch.int32, device="cuda")
    nw = torch.zeros(nchunks, dtype=torch.int32, device="cuda")
    assert L.soi_vlc_compress_device(ptr(xd), ln, nchunks, g, ptr(emax), ptr(words), stride, ptr(nw), None) == 0
    out = torch.empty_like(xd)
    assert L.soi_vlc_decompress_device(ptr(words), stride, ln, nchunks, g, ptr(emax), ptr(out), None) == 0
    torch.cuda.synchronize()
    return out


def test_noalloc_round_trip_matches_existing_entry_points_twice():
    L = sb.lib()
    L.soi_vlc_roundtrip_noalloc_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                   ctypes.c_int, ctypes.c_void_p]
    # two small calls, then the two capacity corners: the most chunks (2047,
    # the per-chunk header full) and exactly the 8388608-word scratch
    cases = [(40960, 16, 1), (4096, 37, 2), (16, 2047, 3), (74896, 64, 4)]
    assert L.soi_vlc_words(74896, 0, 0) * 64 == 8388608
    for call, (ln, nchunks, seed) in enumerate(cases):
        rng = np.random.default_rng(seed)
        x = rng.standard_normal((nchunks, ln)) * 2.0 ** rng.integers(-12, 12, size=(nchunks, 1))
        xd = torch.from_numpy(x).cuda()
        ref = existing_round_trip(xd, ln, nchunks)
        out = torch.full_like(xd, float("nan"))
        assert L.soi_vlc_roundtrip_noalloc_device(ptr(xd), ptr(out), ln, nchunks, None) == 0
        torch.cuda.synchronize()
        assert torch.equal(out.view(torch.int64), ref.view(torch.int64)), "call %d differs" % call
        # and the round trip is the quantisation it should be
        assert float((out - xd).abs().max()) <= float(xd.abs().max()) * 2.0 ** -51


def test_noalloc_rejects_requests_beyond_its_scratch():
    L = sb.lib()
    L.soi_vlc_roundtrip_noalloc_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                   ctypes.c_int, ctypes.c_void_p]
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    too_long = 1 << 23                       # 8M doubles in one chunk
    assert L.soi_vlc_roundtrip_noalloc_device(ptr(x), ptr(x), too_long, 1, None) == 1
    assert L.soi_vlc_roundtrip_noalloc_device(ptr(x), ptr(x), 16, 5000, None) == 1
    # one past each capacity corner
    assert L.soi_vlc_roundtrip_noalloc_device(ptr(x), ptr(x), 16, 2048, None) == 1
    assert L.soi_vlc_roundtrip_noalloc_device(ptr(x), ptr(x), 74896, 65, None) == 1
    assert L.soi_vlc_roundtrip_noalloc_device(ptr(x), ptr(x), 74896 + 16, 64, None) == 1
    assert L.soi_vlc_roundtrip_noalloc_device(ptr(x), ptr(x), 1 << 30, 1, None) == 1
    assert L.soi_vlc_roundtrip_noalloc_device(ptr(x), ptr(x), 17, 1, None) == 2
