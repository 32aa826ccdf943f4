"""The VLC kernels against compress.c semantics (via the oracle, which is
bit-identical to the reference's compress.c, tests/test_oracle.py)."""
import ctypes

import numpy as np
import pytest

import soi_fft_b200 as sb
from oracle import oracle
from tests.conftest import rel_l2
from tests import signals

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("ln,nchunks,shift", [(16, 3, 0), (160, 4, 5), (4096, 8, 12), (65536, 2, 30),
                                              (1024, 5, 60)])
def test_vlc_kernels_bit_exact(ln, nchunks, shift):
    rng = np.random.default_rng(ln + shift)
    x = rng.standard_normal((nchunks, ln)) * 2.0 ** rng.integers(-20, 20, size=(nchunks, 1))
    x[0, : ln // 4] = np.round(x[0, : ln // 4] * 8) / 8          # halfway cases
    xd = torch.from_numpy(x).cuda()
    emax = torch.zeros(nchunks, dtype=torch.int32, device="cuda")
    assert sb.lib().soi_vlc_max_exponent_device(ptr(xd), ln, nchunks, ptr(emax), None) == 0
    torch.cuda.synchronize()
    e_ref = [oracle.max_exponent(x[c]) for c in range(nchunks)]
    assert emax.cpu().tolist() == e_ref
    g = max(e_ref) + shift
    stride = 4 * ln + 64
    words = torch.zeros(nchunks * stride, dtype=torch.int32, device="cuda")
    nw = torch.zeros(nchunks, dtype=torch.int32, device="cuda")
    assert sb.lib().soi_vlc_compress_device(ptr(xd), ln, nchunks, g, ptr(emax), ptr(words), stride,
                                            ptr(nw), None) == 0
    torch.cuda.synchronize()
    wc = words.cpu().numpy().reshape(nchunks, stride)
    out = torch.zeros_like(xd)
    assert sb.lib().soi_vlc_decompress_device(ptr(words), stride, ln, nchunks, g, ptr(emax), ptr(out),
                                              None) == 0
    dec = out.cpu().numpy()
    for c in range(nchunks):
        ref_w = oracle.compress(x[c], g, e_ref[c])
        assert nw[c].item() == ref_w.size
        assert np.array_equal(wc[c, : ref_w.size], ref_w)
        ref_d = oracle.decompress(ref_w, ln, g, e_ref[c]) if ref_w.size else np.zeros(ln)
        assert np.array_equal(dec[c].view(np.int64), ref_d.view(np.int64))


def test_soi_with_vlc_matches_oracle():
    N, S = 1 << 18, 16
    x = signals.band_limited(N, 4)
    d = sb.SoiDescriptor(N=N, use_vlc=1).init(S)
    y = d.compute(torch.from_numpy(x).cuda()).cpu().numpy()
    d.free()
    Mh = 5 * (N // S) // 4
    ref = oracle.compute_soi(x, S, vlc_chunk=Mh)
    assert rel_l2(y, ref) <= 1e-12
    assert rel_l2(y, np.fft.fft(x)) <= 1e-12
