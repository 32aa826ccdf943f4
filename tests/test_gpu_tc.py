"""The tensor-core stage 1 (k_conv_sfft_tc: tcgen05 3xTF32 convolution with
accumulators in tensor memory, SOI_STAGE1_TC=1) against the oracle and the
FP64 direct FFT.  Split form only; rel-L2 <= 1e-6 like every split result."""
import numpy as np
import pytest

import soi_fft_b200 as sb
from oracle import oracle
from tests.conftest import rel_l2
from tests import signals

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SPLIT_TOL = 1e-6


@pytest.fixture
def tc_stage1(monkeypatch):
    monkeypatch.setenv("SOI_STAGE1_TC", "1")
    yield


def _desc(N, S, **kw):
    return sb.SoiDescriptor(N=N, precision=sb.PRECISION_SPLIT_FP32, **kw).init(S)


@pytest.mark.parametrize("N,S", [(1 << 16, 32), (1 << 18, 64), (1 << 20, 128), (1 << 18, 128)])
def test_tc_transposed_matches_oracle(tc_stage1, N, S):
    x = signals.gaussian(N, 31).astype(np.complex64)
    d = _desc(N, S)
    T = d.filter_subsampling(x.copy())
    d.free()
    Tref = oracle.transposed(x.astype(np.complex128), S)
    assert T.shape == Tref.shape
    err = rel_l2(T.astype(np.complex128), Tref)
    assert err <= SPLIT_TOL, err


@pytest.mark.parametrize("N,S", [(1 << 16, 32), (1 << 20, 128), (1 << 21, 64)])
def test_tc_transform_matches_fp64_direct_fft(tc_stage1, N, S):
    x = signals.gaussian_plus_tones(N, 7)
    x64 = x.astype(np.complex64)
    ref = np.fft.fft(x64.astype(np.complex128))
    d = _desc(N, S)
    y = d.compute(torch.from_numpy(x64).cuda()).cpu().numpy()
    d.free()
    err = rel_l2(y.astype(np.complex128), ref)
    assert err <= SPLIT_TOL, err


def test_tc_differs_in_rounding_from_the_fma_kernel(monkeypatch):
    # the two stage-1 kernels sum in different orders: both within tolerance
    # of each other, not bit-equal (so the switch does select another kernel)
    N, S = 1 << 18, 64
    x = signals.gaussian(N, 3).astype(np.complex64)
    outs = []
    for tc in ("0", "1"):
        monkeypatch.setenv("SOI_STAGE1_TC", tc)
        d = _desc(N, S)
        outs.append(d.compute(torch.from_numpy(x).cuda()).cpu().numpy())
        d.free()
    assert not np.array_equal(outs[0], outs[1])
    assert rel_l2(outs[1].astype(np.complex128), outs[0].astype(np.complex128)) <= SPLIT_TOL


def test_tc_segments_of_interest_equal_full_compute(tc_stage1):
    N, S = 1 << 18, 32
    x = torch.from_numpy(signals.gaussian(N, 9).astype(np.complex64)).cuda()
    d = _desc(N, S)
    full = torch.empty_like(x)
    d.compute_into(x, full)
    part = torch.zeros_like(x)
    d.compute_segments(x, part, 5, 11)
    d.free()
    M = N // S
    assert torch.equal(part[5 * M:11 * M], full[5 * M:11 * M])
    assert not part[:5 * M].any() and not part[11 * M:].any()
