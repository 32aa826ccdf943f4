"""The header as a C program sees it: tests/c_caller/soi_caller.c calls
libsoi_b200.so the way the reference's driver calls soi.h (test.c:373-429),
including the struct fields test.c frees and sets to NULL after each compute.
It is compiled with the system C compiler against include/soi_b200.h alone.
The CPU test runs the defaults and init's argument validation; the GPU test
runs a transform and compares it with the oracle."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import soi_fft_b200 as sb
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_caller", "soi_caller.c")


@pytest.fixture(scope="module")
def caller(tmp_path_factory):
    cc = shutil.which("cc") or shutil.which("gcc")
    if cc is None:
        pytest.skip("no C compiler")
    out = str(tmp_path_factory.mktemp("c_caller") / "soi_caller")
    libdir = os.path.dirname(sb.LIB)
    subprocess.run([cc, "-std=c99", "-D_POSIX_C_SOURCE=200112L", "-Wall", "-Wextra", "-Werror", "-O1",
                    "-I", os.path.join(ROOT, "include"), SRC, "-o", out, "-L", libdir, "-lsoi_b200",
                    "-Wl,-rpath," + libdir, "-lm"], check=True)
    return out


def test_c_caller_compiles_and_init_validates_without_a_gpu(caller):
    r = subprocess.run([caller, "validate"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "validate ok" in r.stdout


def splitmix_input(n, seed):
    # the C caller's input generator, restated: splitmix64 -> [-1, 1)
    mask = (1 << 64) - 1
    s = seed
    vals = np.empty(2 * n)
    for i in range(2 * n):
        s = (s + 0x9E3779B97F4A7C15) & mask
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z ^= z >> 31
        vals[i] = (z >> 11) * 2.0 ** -52 - 1.0
    return vals[0::2] + 1j * vals[1::2]


@pytest.mark.gpu
def test_c_caller_transform_matches_oracle(caller, tmp_path):
    N, k, seed = 1 << 16, 8, 7
    out = str(tmp_path / "y.bin")
    r = subprocess.run([caller, "compute", str(N), str(k), str(seed), out], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    y = np.fromfile(out, dtype=np.complex128)
    x = splitmix_input(N, seed)
    ref = oracle.compute_soi(x, k)
    assert y.shape == ref.shape
    err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
    assert err < 1e-12, err
