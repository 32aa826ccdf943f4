"""CPU tests of the C ABI boundary: the library loads, exports every function
include/soi_b200.h declares, validates arguments before touching a GPU, and
its host-side tables equal the reference's window (pfft.c:42-82)."""
import ctypes
import os
import re

import numpy as np
import pytest

import soi_fft_b200 as sb
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "soi_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                       src, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "defined")))


def test_library_exports_every_declared_symbol():
    lib = sb.lib()
    names = declared_functions()
    assert "compute_soi" in names and "init_soi_descriptor" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_entry_points_present():
    # soi.h:272-280
    for n in ("set_default_soi_descriptor", "init_soi_descriptor", "compute_soi",
              "free_soi_descriptor", "parallel_filter_subsampling"):
        assert hasattr(sb.lib(), n)


def test_defaults_match_reference():
    d = sb.SoiDescriptor()
    # pfft.c:87-94
    assert (d.n_mu, d.d_mu, d.B) == (5, 4, 72)
    assert d.tau == 928 / 1024.
    assert d.sigma == 373.7314
    assert d.use_vlc == 0 and d.comm_to_comp_cost_ratio == 1
    assert d.P == 1 and d.rank == 0


@pytest.mark.parametrize("fields,k,status", [
    (dict(N=1 << 16, P=2), 8, 2),            # multi-rank: not built here
    (dict(N=1 << 16), 0, 1),                 # k = 0
    (dict(N=1000), 8, 1),                    # S does not divide N
    (dict(N=1 << 16, n_mu=7, d_mu=4), 8, 2),  # oversampling pair not built
    (dict(N=1 << 8), 8, 1),                  # M < B (.cpp:89-94)
    (dict(N=1 << 16, precision=5), 8, 1),
])
def test_init_rejects_before_touching_the_gpu(fields, k, status):
    d = sb.SoiDescriptor(**fields)
    with pytest.raises(sb.SoiError) as e:
        d.init(k)
    assert e.value.status == status


def test_void_entry_point_exits_like_the_reference(tmp_path):
    # init_soi_descriptor on an invalid descriptor prints and exits(-1), as the
    # reference does for unsupported sizes (.cpp:543-548)
    import subprocess
    import sys
    code = ("import ctypes, soi_fft_b200 as sb\n"
            "d = sb.SoiDescriptor(N=1000)\n"
            "sb.lib().init_soi_descriptor.argtypes=[ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]\n"
            "sb.lib().init_soi_descriptor(ctypes.byref(d._d), None, 8)\n"
            "print('survived')\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True)
    assert r.returncode == 255 and "survived" not in r.stdout
    assert "invalid parameters" in r.stderr


@pytest.mark.parametrize("N,S,n,d,B,tau,sigma", [
    (1 << 16, 8, 5, 4, 72, 928 / 1024., 373.7314),
    (1 << 18, 64, 5, 4, 72, 928 / 1024., 373.7314),
    (1 << 16, 16, 5, 4, 44, 512 / 1024., 121.0936),
    (7 << 14, 8, 8, 7, 72, 928 / 1024., 373.7314),
])
def test_factorised_window_equals_reference_window(N, S, n, d, B, tau, sigma):
    filt, phase, winv = sb.window_tables(N, S, n, d, B, tau, sigma)
    w = oracle.w_table(N, S, n, d, B, tau, sigma)            # [theta][kk][s]
    wf = np.transpose(phase[None, :, :] * filt, (1, 0, 2))
    # the reference rounds t in double before evaluating the window; the
    # exact-rational tables differ from it by that rounding, ~1e-14
    assert np.abs(wf - w).max() <= 5e-14 * np.abs(w).max()
    W = oracle.W_inv_table(N, S, n, d, B, tau, sigma)
    # W_inv = 1/y with y a difference of two erfc values (pfft.c:75); near the
    # segment edges y ~ 1e-4 and the reference's double erfc loses ~1e-12
    # relative there, the long-double tables do not
    assert np.abs(winv - W).max() <= 1e-11 * np.abs(W).max()
    assert np.linalg.norm(winv - W) <= 1e-12 * np.linalg.norm(W)


@pytest.mark.parametrize("ln,emax,emaxi", [(16, 3, 3), (64, 10, 2), (4096, 20, -10), (160, 5, -40),
                                            (32, 0, -60), (17, 3, 1)])
def test_vlc_word_count_matches_oracle(ln, emax, emaxi):
    assert sb.lib().soi_vlc_words(ln, emax, emaxi) == oracle.vlc_words(ln, emax, emaxi)


def test_vlc_words_reports_overflow_instead_of_wrapping():
    L = sb.lib()
    # 1.75 words per double at full width (56 bits): 2^30 doubles fit in an
    # int count, 2^31 - 16 (3.76e9 words) do not
    assert L.soi_vlc_words(1 << 29, 0, 0) == (1 << 29) // 16 * 28
    assert L.soi_vlc_words(1 << 30, 0, 0) == (1 << 30) // 16 * 28
    assert L.soi_vlc_words((1 << 31) - 16, 0, 0) == -1


@pytest.mark.parametrize("ln,nchunks", [
    ((1 << 31) - 16, 1),          # the word count overflows an int
    ((1 << 31) - 16, 2047),
    (1 << 30, 2),                 # fits an int per chunk; the product does not fit the scratch
    (74896 + 16, 64),             # over the 8388608-word scratch by one group per chunk
    (4793488 + 16, 1),
    (16, 2048),                   # too many chunks
])
def test_noalloc_rejects_oversized_requests_before_touching_the_gpu(ln, nchunks):
    L = sb.lib()
    fn = L.soi_vlc_roundtrip_noalloc_device
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    # non-null stand-in pointers: the size check comes before any device access,
    # so without a GPU the call returns SOI_ERR_INVALID, not SOI_ERR_CUDA
    assert fn(ctypes.c_void_p(256), ctypes.c_void_p(256), ln, nchunks, None) == 1


def test_plan_variant_picks_the_measured_defaults(monkeypatch):
    # host logic only: the kernels a plan would launch
    v = sb.plan_variant(1 << 29, 128, sb.PRECISION_SPLIT_FP32)
    assert v == {"stage1": "compile-time S", "stage1_threads": 256, "stage1_staging": "tensor copies",
                 "stage2": "persistent", "pass2_staging": "bulk copies"}
    assert sb.plan_variant(1 << 28, 64, sb.PRECISION_FP64)["stage1_threads"] == 256
    assert sb.plan_variant(1 << 28, 128, sb.PRECISION_FP64)["stage1_threads"] == 512
    assert sb.plan_variant(1 << 28, 64, sb.PRECISION_FP64)["pass2_staging"] == "bulk copies"
    monkeypatch.setenv("SOI_STAGE1_BULK", "0")
    v = sb.plan_variant(1 << 29, 128, sb.PRECISION_SPLIT_FP32)
    assert (v["stage1_staging"], v["stage1_threads"]) == ("cp.async", 512)
    monkeypatch.setenv("SOI_STAGE1_NT", "256")
    assert sb.plan_variant(1 << 29, 128, sb.PRECISION_SPLIT_FP32)["stage1_threads"] == 256
    monkeypatch.setenv("SOI_STAGE2_BULK2", "0")
    assert sb.plan_variant(1 << 29, 128, sb.PRECISION_SPLIT_FP32)["pass2_staging"] == "cp.async"


@pytest.mark.parametrize("N,S,prec", [(1 << 20, 16, sb.PRECISION_SPLIT_FP32), (1 << 26, 16, sb.PRECISION_SPLIT_FP32),
                                      (1 << 22, 8, sb.PRECISION_FP64), (1 << 29, 128, sb.PRECISION_SPLIT_FP32),
                                      (1 << 24, 256, sb.PRECISION_SPLIT_FP32)])
@pytest.mark.parametrize("nt", ["256", "512"])
def test_tensor_copy_tiles_fit_one_box(N, S, prec, nt, monkeypatch):
    # a stage-1 phase's rows travel as one tensor-copy box of at most 256
    # rows of at most 256 eight-byte values: the plan keeps JT + B/d - 1
    # within it whenever it stages by tensor copies
    monkeypatch.setenv("SOI_STAGE1_NT", nt)
    v = sb.plan_variant(N, S, prec)
    g = sb.plan_geometry(N, S, prec)
    if v["stage1_staging"] == "tensor copies":
        elem = 8 if prec == sb.PRECISION_SPLIT_FP32 else 16
        assert g["JT"] + g["taps_per_phase"] - 1 <= 256
        assert S * elem // 8 <= 256 and S * elem >= 128


def test_sixty_four_byte_rows_stage_by_cp_async():
    assert sb.plan_variant(1 << 20, 8, sb.PRECISION_SPLIT_FP32)["stage1_staging"] == "cp.async"
    assert sb.plan_variant(1 << 20, 8, sb.PRECISION_FP64)["stage1_staging"] == "tensor copies"
