"""soi_fft_b200 -- the SOI FFT (IntelLabs/SOI_FFT's soi.h API) on one B200.

Host-side mirror of the reference interface over the C ABI of
libsoi_b200.so (include/soi_b200.h).  The reference's entry points are kept
with their names and argument meaning (soi.h:272-280):

    d = SoiDescriptor()                 # set_default_soi_descriptor
    d.N = 1 << 20; d.n_mu, d.d_mu = 5, 4
    d.init(k=8)                         # init_soi_descriptor(&d, comm, k)
    y = d.compute(x)                    # compute_soi(&d, alpha_dt), in place
    d.free()                            # free_soi_descriptor

x may be a numpy array (host memory, copied in and out by the library) or a
CUDA torch tensor (device memory).  complex128 selects the plain FP64 method,
complex64 the split-precision form.  Errors raise SoiError carrying the
library's status; the library itself never falls back to a CPU path.
"""
import ctypes
import os

import numpy as np

from .build import LIB

__all__ = ["SoiDescriptor", "SoiError", "soi_fft", "lib", "window_tables",
           "PRECISION_FP64", "PRECISION_SPLIT_FP32"]

PRECISION_FP64 = 0
PRECISION_SPLIT_FP32 = 1


class SoiError(RuntimeError):
    def __init__(self, status, what):
        super().__init__("%s: %s (status %d)" % (what, _status_string(status), status))
        self.status = status


class _Desc(ctypes.Structure):
    _fields_ = [("comm", ctypes.c_void_p), ("P", ctypes.c_int), ("rank", ctypes.c_int),
                ("k", ctypes.c_size_t), ("N", ctypes.c_size_t),
                # soi.h:243-251, kept NULL (the library never touches them)
                ("W_inv", ctypes.c_void_p), ("w", ctypes.c_void_p), ("w_dup", ctypes.c_void_p),
                ("gamma_tilde", ctypes.c_void_p), ("alpha_tilde", ctypes.c_void_p),
                ("beta_tilde", ctypes.c_void_p), ("alpha_ghost", ctypes.c_void_p),
                ("delta", ctypes.POINTER(ctypes.c_int)), ("epsilon", ctypes.POINTER(ctypes.c_int)),
                ("n_mu", ctypes.c_int),
                ("d_mu", ctypes.c_int), ("B", ctypes.c_size_t), ("tau", ctypes.c_double),
                ("sigma", ctypes.c_double), ("use_vlc", ctypes.c_int),
                ("segmentBoundaries", ctypes.POINTER(ctypes.c_int)),
                ("comm_to_comp_cost_ratio", ctypes.c_double), ("precision", ctypes.c_int),
                ("device_ptr", ctypes.c_int), ("device", ctypes.c_int), ("stream", ctypes.c_void_p),
                ("last_status", ctypes.c_int), ("plan", ctypes.c_void_p)]


_lib = None


def lib():
    """The loaded libsoi_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise OSError("libsoi_b200.so is not built (python -m soi_fft_b200.build)")
        L = ctypes.CDLL(LIB)
        P = ctypes.POINTER(_Desc)
        for name in ("soi_init_status",):
            getattr(L, name).argtypes = [P, ctypes.c_void_p, ctypes.c_size_t]
        for name in ("soi_compute_status", "soi_filter_subsampling_status", "soi_get_transposed"):
            getattr(L, name).argtypes = [P, ctypes.c_void_p]
        L.soi_compute_oop_status.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p]
        L.soi_compute_segments_status.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.soi_compute_async_status.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p]
        L.soi_check_status.argtypes = [P]
        L.soi_compute_inverse_status.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p]
        L.soi_compute_stream_status.argtypes = [P, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                                                ctypes.c_int]
        L.soi_free_status.argtypes = [P]
        L.set_default_soi_descriptor.argtypes = [P]
        L.soi_status_string.restype = ctypes.c_char_p
        L.soi_b200_version.restype = ctypes.c_char_p
        L.soi_set_timing.argtypes = [P, ctypes.c_int]
        L.soi_kernels_per_compute.argtypes = [P]
        L.soi_last_timings.argtypes = [P, ctypes.POINTER(ctypes.c_float)]
        L.soi_filter_subsample_device.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p]
        L.soi_segment_fft_demod_device.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p]
        L.soi_window_tables.argtypes = [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_size_t, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.soi_vlc_words.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.soi_vlc_max_exponent_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_void_p, ctypes.c_void_p]
        L.soi_vlc_compress_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
                                              ctypes.c_void_p, ctypes.c_void_p]
        L.soi_vlc_decompress_device.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p]
        V = ctypes.c_void_p
        L.soi_mlp_param_count.restype = ctypes.c_int
        L.soi_mlp_forward_device.argtypes = [V, V, V, ctypes.c_int, V]
        L.soi_mlp_grad_device.argtypes = [V, V, V, ctypes.c_int, V, V, V]
        L.soi_mlp_adam_device.argtypes = [V, V, V, V, ctypes.c_float, ctypes.c_int, V]
        _lib = L
    return _lib


def _status_string(s):
    try:
        return lib().soi_status_string(s).decode()
    except OSError:
        return "status %d" % s


def _check(rc, what):
    if rc != 0:
        raise SoiError(rc, what)


def _is_torch_cuda(x):
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


class SoiDescriptor:
    """soi_desc_t (soi.h:236-270) with the reference's lifecycle."""

    def __init__(self, **fields):
        self._d = _Desc()
        lib().set_default_soi_descriptor(ctypes.byref(self._d))
        for k, v in fields.items():
            setattr(self, k, v)

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        return getattr(self._d, name)

    def __setattr__(self, name, value):
        if name.startswith("_"):
            object.__setattr__(self, name, value)
        else:
            setattr(self._d, name, value)

    @property
    def S(self):
        return self._d.k * self._d.P

    @property
    def M(self):
        return self._d.N // self.S

    @property
    def M_hat(self):
        return self._d.n_mu * self.M // self._d.d_mu

    def init(self, k, comm=None):
        """init_soi_descriptor (pfft.c:140-232)."""
        _check(lib().soi_init_status(ctypes.byref(self._d), comm, k), "init_soi_descriptor")
        return self

    def free(self):
        """free_soi_descriptor (pfft.c:234-267)."""
        if self._d.plan:
            lib().soi_free_status(ctypes.byref(self._d))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def _dtype(self):
        return np.complex128 if self._d.precision == PRECISION_FP64 else np.complex64

    def _ptr(self, x):
        if _is_torch_cuda(x):
            import torch
            want = torch.complex128 if self._d.precision == PRECISION_FP64 else torch.complex64
            if x.dtype != want or not x.is_contiguous() or x.numel() != self._d.N:
                raise ValueError("device array must be contiguous %s of length N" % want)
            if not self._d.stream:
                # the library's own stream is ordered with the legacy default
                # stream only: work queued on a torch side stream (the tensor's
                # producer) must finish before the library reads the tensor
                cur = torch.cuda.current_stream(x.device)
                if cur.cuda_stream != 0 and not torch.cuda.is_current_stream_capturing():
                    cur.synchronize()
            self._d.device_ptr = 1
            return ctypes.c_void_p(x.data_ptr())
        if x.dtype != self._dtype() or not x.flags.c_contiguous or x.size != self._d.N:
            raise ValueError("host array must be contiguous %s of length N" % self._dtype())
        self._d.device_ptr = 0
        return x.ctypes.data_as(ctypes.c_void_p)

    def compute(self, x):
        """compute_soi (pfft.c:276-721): in-place; returns x."""
        _check(lib().soi_compute_status(ctypes.byref(self._d), self._ptr(x)), "compute_soi")
        return x

    def compute_into(self, x, out):
        """Out-of-place transform: x is left untouched, out receives the
        result (both host arrays or both CUDA tensors)."""
        px = self._ptr(x)
        dev = self._d.device_ptr
        po = self._ptr(out)
        if self._d.device_ptr != dev:
            raise ValueError("x and out must both be host arrays or both CUDA tensors")
        _check(lib().soi_compute_oop_status(ctypes.byref(self._d), px, po), "soi_compute_oop")
        return out

    def compute_segments(self, x, out, seg_lo, seg_hi):
        """Segments of interest: outputs of segments [seg_lo, seg_hi) only
        (out[seg_lo*M : seg_hi*M]); the rest of out is left as it was."""
        px = self._ptr(x)
        dev = self._d.device_ptr
        po = self._ptr(out)
        if self._d.device_ptr != dev:
            raise ValueError("x and out must both be host arrays or both CUDA tensors")
        _check(lib().soi_compute_segments_status(ctypes.byref(self._d), px, po, int(seg_lo), int(seg_hi)),
               "soi_compute_segments")
        return out

    def compute_async(self, x, out):
        """Enqueue the transform of CUDA tensors x -> out on the descriptor's
        stream without waiting (capturable); check() reports a stage-2 wait
        that gave up."""
        if not (_is_torch_cuda(x) and _is_torch_cuda(out)):
            raise ValueError("compute_async takes CUDA tensors")
        px, po = self._ptr(x), self._ptr(out)
        _check(lib().soi_compute_async_status(ctypes.byref(self._d), px, po), "soi_compute_async")
        return out

    def compute_inverse(self, x, out):
        """Inverse transform x -> out, (1/N) sum_k x[k] exp(+2 pi i k n/N);
        x is left untouched (both host arrays or both CUDA tensors)."""
        px = self._ptr(x)
        dev = self._d.device_ptr
        po = self._ptr(out)
        if self._d.device_ptr != dev:
            raise ValueError("x and out must both be host arrays or both CUDA tensors")
        _check(lib().soi_compute_inverse_status(ctypes.byref(self._d), px, po), "soi_compute_inverse")
        return out

    def compute_stream(self, xs, ys):
        """Transforms of several host arrays, ys[i] <- transform of xs[i], with
        the uploads, kernels and downloads of neighbours overlapped (pinned
        host memory makes the copies overlap)."""
        if len(xs) != len(ys) or not xs:
            raise ValueError("xs and ys must be non-empty lists of the same length")
        ins = (ctypes.c_void_p * len(xs))()
        outs = (ctypes.c_void_p * len(ys))()
        for i, (x, y) in enumerate(zip(xs, ys)):
            if _is_torch_cuda(x) or _is_torch_cuda(y):
                raise ValueError("compute_stream takes host arrays")
            ins[i] = self._ptr(x)
            outs[i] = self._ptr(y)
        _check(lib().soi_compute_stream_status(ctypes.byref(self._d), ins, outs, len(xs)), "soi_compute_stream")
        return ys

    def check(self):
        """Wait for the descriptor's stream; raise if a stage-2 wait gave up."""
        _check(lib().soi_check_status(ctypes.byref(self._d)), "soi_check_status")

    def filter_subsampling(self, x):
        """parallel_filter_subsampling (.cpp:535): stage 1 only; returns the
        transposed data (S, M') as a numpy array."""
        _check(lib().soi_filter_subsampling_status(ctypes.byref(self._d), self._ptr(x)),
               "parallel_filter_subsampling")
        dev = self._d.device_ptr
        self._d.device_ptr = 0
        T = np.empty(self.S * self.M_hat, self._dtype())
        _check(lib().soi_get_transposed(ctypes.byref(self._d), T.ctypes.data_as(ctypes.c_void_p)),
               "soi_get_transposed")
        self._d.device_ptr = dev
        return T.reshape(self.S, self.M_hat)

    def set_timing(self, on=True):
        _check(lib().soi_set_timing(ctypes.byref(self._d), int(on)), "soi_set_timing")

    def kernels_per_compute(self):
        """How many of the library's kernels one compute launches."""
        n = lib().soi_kernels_per_compute(ctypes.byref(self._d))
        if n < 0:
            _check(-n, "soi_kernels_per_compute")
        return n

    def timings(self):
        a = (ctypes.c_float * 4)()
        _check(lib().soi_last_timings(ctypes.byref(self._d), a), "soi_last_timings")
        return {"stage1_ms": a[0], "stage2_ms": a[1], "vlc_ms": a[2], "total_ms": a[3]}


def soi_fft(x, S, n_mu=5, d_mu=4, B=72, tau=None, sigma=None, use_vlc=False, device=0):
    """One-shot SOI transform of x (numpy or CUDA torch tensor, complex128 for
    the plain FP64 method, complex64 for the split-precision form)."""
    is_dev = _is_torch_cuda(x)
    dt = x.dtype
    if is_dev:
        import torch
        prec = PRECISION_FP64 if dt == torch.complex128 else PRECISION_SPLIT_FP32
        y = x.clone()
    else:
        prec = PRECISION_FP64 if dt == np.complex128 else PRECISION_SPLIT_FP32
        y = np.array(x, copy=True)
    d = SoiDescriptor(N=y.numel() if is_dev else y.size, n_mu=n_mu, d_mu=d_mu, B=B,
                      precision=prec, device=device, use_vlc=int(use_vlc))
    if tau is not None:
        d.tau = tau
    if sigma is not None:
        d.sigma = sigma
    d.init(S)
    try:
        d.compute(y)
    finally:
        d.free()
    return y


def window_tables(N, S, n_mu=5, d_mu=4, B=72, tau=928 / 1024., sigma=373.7314):
    """Host tables of the factorised window: (filt[B][n_mu][S] real,
    phase[n_mu][S] complex, W_inv[N/S] complex), FP64."""
    filt = np.zeros(B * n_mu * S, np.float64)
    phase = np.zeros(n_mu * S, np.complex128)
    winv = np.zeros(N // S, np.complex128)
    _check(lib().soi_window_tables(N, S, n_mu, d_mu, B, tau, sigma, filt.ctypes.data_as(ctypes.c_void_p),
                                   phase.ctypes.data_as(ctypes.c_void_p), winv.ctypes.data_as(ctypes.c_void_p)),
           "soi_window_tables")
    return filt.reshape(B, n_mu, S), phase.reshape(n_mu, S), winv


def plan_variant(N, S, precision=PRECISION_FP64, n_mu=5, d_mu=4, B=72):
    """Host-side choice of kernels (no GPU): stage-1 kernel, its threads and
    staging, the stage-2 form and its pass-2 staging."""
    d = _Desc()
    lib().set_default_soi_descriptor(ctypes.byref(d))
    d.N, d.n_mu, d.d_mu, d.B, d.precision = N, n_mu, d_mu, B, precision
    info = (ctypes.c_int * 5)()
    lib().soi_plan_variant.argtypes = [ctypes.POINTER(_Desc), ctypes.c_size_t, ctypes.c_void_p]
    _check(lib().soi_plan_variant(ctypes.byref(d), S, info), "soi_plan_variant")
    kinds = {0: "general", 1: "staged", 2: "compile-time S", 3: "tensor cores"}
    return {"stage1": kinds[info[0]], "stage1_threads": info[1],
            "stage1_staging": "tensor copies" if info[2] else "cp.async",
            "stage2": "persistent" if info[3] else "two kernels",
            "pass2_staging": "bulk copies" if info[4] else "cp.async"}


def plan_geometry(N, S, precision=PRECISION_FP64, n_mu=5, d_mu=4, B=72):
    """Host-side plan geometry (no GPU): dict of tile shapes and splits."""
    d = _Desc()
    lib().set_default_soi_descriptor(ctypes.byref(d))
    d.N, d.n_mu, d.d_mu, d.B, d.precision = N, n_mu, d_mu, B, precision
    info = (ctypes.c_longlong * 16)()
    lib().soi_plan_geometry.argtypes = [ctypes.POINTER(_Desc), ctypes.c_size_t, ctypes.c_void_p]
    _check(lib().soi_plan_geometry(ctypes.byref(d), S, info), "soi_plan_geometry")
    keys = ["S", "M", "M_hat", "JT", "taps_per_phase", "JR", "smem_stage1", "M1", "M2", "C1", "C2",
            "smem_pass1", "smem_pass2", "stages_S", "stages_M1", "stages_M2"]
    return dict(zip(keys, list(info)))
