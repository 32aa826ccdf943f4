"""ctypes bindings to the CPU checker (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It loads oracle/_build/liboracle.so (the C restatement of the
reference's algorithm, oracle/soi_oracle.c) and runs oracle/_ref/soi_ref_run
(the reference's own sources compiled by oracle/Makefile).
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_RUN = os.path.join(HERE, "_ref", "soi_ref_run")
REF_COMPRESS = os.path.join(HERE, "_ref", "libcompress_ref.so")

_P = ctypes.c_void_p


class Params(ctypes.Structure):
    _fields_ = [("N", ctypes.c_size_t), ("S", ctypes.c_size_t), ("n_mu", ctypes.c_int),
                ("d_mu", ctypes.c_int), ("B", ctypes.c_size_t), ("tau", ctypes.c_double),
                ("sigma", ctypes.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "_build/liboracle.so"], check=True,
                           capture_output=True)
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_max_exponent.restype = ctypes.c_int
        _lib.oracle_compress.restype = ctypes.c_int
        _lib.oracle_vlc_words.restype = ctypes.c_int
    return _lib


def params(N, S, n_mu=5, d_mu=4, B=72, tau=None, sigma=None):
    p = Params()
    lib().oracle_defaults(ctypes.byref(p))
    p.N, p.S, p.n_mu, p.d_mu, p.B = N, S, n_mu, d_mu, B
    if tau is not None:
        p.tau = tau
    if sigma is not None:
        p.sigma = sigma
    return p


def _ptr(a):
    return a.ctypes.data_as(_P)


def compute_soi(x, S, n_mu=5, d_mu=4, B=72, tau=None, sigma=None, vlc_chunk=0):
    """Full SOI transform of complex128 x (natural-order output)."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    p = params(x.size, S, n_mu, d_mu, B, tau, sigma)
    out = np.zeros(x.size, np.complex128)
    if vlc_chunk:
        lib().oracle_compute_soi_vlc(ctypes.byref(p), ctypes.c_size_t(vlc_chunk), _ptr(x), _ptr(out))
    else:
        lib().oracle_compute_soi(ctypes.byref(p), _ptr(x), _ptr(out))
    return out


def w_table(N, S, n_mu=5, d_mu=4, B=72, tau=None, sigma=None):
    p = params(N, S, n_mu, d_mu, B, tau, sigma)
    w = np.zeros(n_mu * B * S, np.complex128)
    lib().oracle_w_table(ctypes.byref(p), _ptr(w))
    return w.reshape(n_mu, B, S)


def W_inv_table(N, S, n_mu=5, d_mu=4, B=72, tau=None, sigma=None):
    p = params(N, S, n_mu, d_mu, B, tau, sigma)
    w = np.zeros(N // S, np.complex128)
    lib().oracle_W_inv_table(ctypes.byref(p), _ptr(w))
    return w


def transposed(x, S, n_mu=5, d_mu=4, B=72, tau=None, sigma=None):
    """alpha_tilde after conv + S-point FFT + transpose: (S, M') complex128."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    N = x.size
    p = params(N, S, n_mu, d_mu, B, tau, sigma)
    Mh = n_mu * (N // S) // d_mu
    w = w_table(N, S, n_mu, d_mu, B, tau, sigma)
    G = np.zeros(Mh * S, np.complex128)
    T = np.zeros(Mh * S, np.complex128)
    lib().oracle_conv(ctypes.byref(p), _ptr(w), _ptr(x), _ptr(G))
    lib().oracle_row_fft(ctypes.byref(p), _ptr(G))
    lib().oracle_transpose(ctypes.byref(p), _ptr(G), _ptr(T))
    return T.reshape(S, Mh)


def aligned(n, dtype):
    buf = np.zeros(n + 64, dtype)
    off = (-buf.ctypes.data % 64) // buf.itemsize
    return buf[off:off + n]


def max_exponent(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    return lib().oracle_max_exponent(_ptr(x), x.size)


def compress(x, e_max, e_max_i):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = aligned(4 * x.size + 64, np.int32)
    n = lib().oracle_compress(_ptr(out), _ptr(x), x.size, e_max, e_max_i)
    return out[:n].copy()


def decompress(words, length, e_max, e_max_i):
    words = np.ascontiguousarray(words, dtype=np.int32)
    out = np.zeros(length, np.float64)
    lib().oracle_decompress(_ptr(out), _ptr(words), words.size, length, e_max, e_max_i)
    return out


def vlc_words(length, e_max, e_max_i):
    return lib().oracle_vlc_words(length, e_max, e_max_i)


def ref_available():
    return os.path.exists(REF_RUN)


def run_reference(x, P, k, threads=None, repeat=1, n_mu=5, d_mu=4, B=72, tau=None, sigma=None,
                  vlc=False, return_times=False):
    """Run the reference's own compute_soi on P forked ranks x `threads` OpenMP
    threads each.  Returns (output complex128 natural order, best seconds)."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    S = P * k
    ntg = min(S // 4, 8)
    if threads is None:
        threads = ntg
    d = tempfile.mkdtemp(prefix="soi_ref_")
    fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
    x.tofile(fin)
    cmd = [REF_RUN, "--N", str(x.size), "--P", str(P), "--k", str(k), "--threads", str(threads),
           "--repeat", str(repeat), "--n_mu", str(n_mu), "--d_mu", str(d_mu), "--B", str(B),
           "--in", fin, "--out", fout]
    if tau is not None:
        cmd += ["--tau", repr(tau)]
    if sigma is not None:
        cmd += ["--sigma", repr(sigma)]
    if vlc:
        cmd += ["--vlc"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    try:
        if r.returncode != 0:
            raise RuntimeError("reference run failed: %s" % r.stderr[-500:])
        line = [l for l in r.stdout.splitlines() if l.startswith("SOI_REF_RESULT")][-1]
        best = float(line.split("best_s=")[1].split()[0])
        times = [float(t) for t in line.split("times=")[1].split(",") if t]
        y = np.fromfile(fout, dtype=np.complex128)
    finally:
        for f in (fin, fout):
            if os.path.exists(f):
                os.remove(f)
        os.rmdir(d)
    return (y, best, times) if return_times else (y, best)
