"""Batched transforms: many SOI transforms of different lengths, segment
counts and bands, replayed as one CUDA graph (soi_batch_* in the C ABI).

The reference transforms one signal per call (pfft.c:276); this is the
batched/banded driver built on the same kernels.  `band_workload` makes the
synthetic band-limited batch: N log-uniform over powers of two, each input's
spectrum confined to a random band of a given fraction of the bins, and the
segments of interest those that overlap the band.
"""
import ctypes
import math

import numpy as np

from . import lib, _Desc, _check, PRECISION_FP64, PRECISION_SPLIT_FP32


class _Item(ctypes.Structure):
    _fields_ = [("N", ctypes.c_size_t), ("k", ctypes.c_size_t), ("seg_lo", ctypes.c_int),
                ("seg_hi", ctypes.c_int), ("inp", ctypes.c_void_p), ("out", ctypes.c_void_p)]


def _bind():
    L = lib()
    if getattr(L, "_batch_bound", False):
        return L
    P = ctypes.c_void_p
    L.soi_batch_create.argtypes = [ctypes.POINTER(P), ctypes.POINTER(_Desc), ctypes.POINTER(_Item), ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int]
    L.soi_batch_execute.argtypes = [P, P]
    L.soi_batch_check.argtypes = [P]
    L.soi_batch_info.argtypes = [P, ctypes.POINTER(ctypes.c_longlong)]
    L.soi_batch_plan_info.argtypes = [P, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
    L.soi_batch_destroy.argtypes = [P]
    L._batch_bound = True
    return L


class SoiBatch:
    """A fixed batch of transforms on CUDA tensors.

    items: list of (x, out, k, seg_lo, seg_hi) with x/out contiguous CUDA
    tensors of the precision's dtype (out may be x: in place); seg_hi <= 0
    computes all k segments.  Window and oversampling as for SoiDescriptor.
    """

    def __init__(self, items, precision=PRECISION_SPLIT_FP32, chains=4, tune=True, n_mu=5, d_mu=4, B=72,
                 tau=None, sigma=None, use_vlc=False, device=0):
        import torch
        L = _bind()
        d = _Desc()
        L.set_default_soi_descriptor(ctypes.byref(d))
        d.n_mu, d.d_mu, d.B, d.precision, d.device, d.use_vlc = n_mu, d_mu, B, precision, device, int(use_vlc)
        if tau is not None:
            d.tau = tau
        if sigma is not None:
            d.sigma = sigma
        want = torch.complex128 if precision == PRECISION_FP64 else torch.complex64
        arr = (_Item * len(items))()
        self._keep = []
        for i, (x, out, k, lo, hi) in enumerate(items):
            for t in (x, out):
                if not (t.is_cuda and t.dtype == want and t.is_contiguous()):
                    raise ValueError("batch buffers must be contiguous CUDA %s tensors" % want)
            arr[i] = _Item(x.numel(), int(k), int(lo), int(hi), x.data_ptr(), out.data_ptr())
            self._keep.append((x, out))
        self._b = ctypes.c_void_p()
        _check(L.soi_batch_create(ctypes.byref(self._b), ctypes.byref(d), arr, len(items), int(chains), int(tune)),
               "soi_batch_create")

    def execute(self, stream=None):
        """Launch the graph on `stream` (a torch.cuda.Stream; default: the current stream)."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        _check(_bind().soi_batch_execute(self._b, ctypes.c_void_p(s.cuda_stream)), "soi_batch_execute")

    def check(self):
        _check(_bind().soi_batch_check(self._b), "soi_batch_check")

    def info(self):
        a = (ctypes.c_longlong * 8)()
        _check(_bind().soi_batch_info(self._b, a), "soi_batch_info")
        keys = ["transforms", "plans", "chains", "graph_nodes", "kernels_per_execute", "scratch_bytes"]
        return dict(zip(keys, list(a)[:6]))

    def plans(self):
        out = []
        for i in range(self.info()["plans"]):
            a = (ctypes.c_longlong * 8)()
            _check(_bind().soi_batch_plan_info(self._b, i, a), "soi_batch_plan_info")
            out.append({"N": a[0], "k": a[1], "stage1_threads": a[2], "persistent_stage2": bool(a[3]),
                        "M1": a[4], "M2": a[5], "tuned_us": a[6], "variant": a[7]})
        return out

    def free(self):
        if self._b:
            _bind().soi_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def segments_for(N):
    """Segment count for a length: 4 at 2^14 up to 64 at 2^24, a power of
    two growing with log N."""
    lg = int(round(math.log2(N)))
    return 1 << int(min(6, max(2, round((lg - 14) * 0.4) + 2)))


def band_workload(count, log2_lo=14, log2_hi=24, band=0.05, seed=0, precision=PRECISION_SPLIT_FP32,
                  device="cuda", max_total=None):
    """Synthetic band-limited batch.  Returns a list of dicts with the input
    tensor `x`, its segment count `k`, the band [b0, b1) of output bins, the
    segments of interest [seg_lo, seg_hi) and N.  Inputs are generated in FP64
    (random complex spectrum on the band, inverse FFT) and rounded once to
    the working precision."""
    import torch
    rng = np.random.default_rng(seed)
    cdt = torch.complex128 if precision == PRECISION_FP64 else torch.complex64
    out, total = [], 0
    for i in range(count):
        lg = int(rng.integers(log2_lo, log2_hi + 1))
        N = 1 << lg
        if max_total is not None and total + N > max_total:
            break
        k = segments_for(N)
        width = max(1, int(band * N))
        b0 = int(rng.integers(0, N - width + 1))
        g = torch.Generator(device=device).manual_seed(seed * 100003 + i)
        X = torch.zeros(N, dtype=torch.complex128, device=device)
        X[b0:b0 + width] = torch.complex(torch.randn(width, generator=g, device=device, dtype=torch.float64),
                                         torch.randn(width, generator=g, device=device, dtype=torch.float64))
        x = torch.fft.ifft(X) * math.sqrt(N / width)
        M = N // k
        out.append({"N": N, "k": k, "band": (b0, b0 + width), "seg_lo": b0 // M,
                    "seg_hi": min(k, -(-(b0 + width) // M)), "x": x.to(cdt).contiguous()})
        total += N
    return out
