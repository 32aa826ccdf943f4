#!/usr/bin/env python
"""bench.py -- SOI FFT on B200: GFLOP/s (5 N log2 N) at N=2^29.

Workload (one step = one SOI transform of one synthetic batch):
    N = 2^29 complex64 (4 GiB), S = 128 segments, mu = 5/4, B = 72 taps,
    split-precision form (FP32 arithmetic, complex64 storage,
    FP64-generated tables rounded once).  Input: seeded complex Gaussian plus
    64 pure tones at random bin + fractional offsets with amplitudes
    log-uniform in [1e-6, 1] (synthetic stand-in; the reference names no
    dataset).  Inputs (4 GiB) are larger than L2 (126 MB), so no L2 flush is
    needed between steps.

value   : device-resident inputs, out-of-place transform through the C ABI's
          non-waiting entry point (soi_compute_async_status with device
          pointers), K steps back to back on the library's stream timed by
          CUDA events, soi_check_status after them.
e2e     : the same transform through the C ABI with host (pinned) buffers,
          the host->device copy of the input and the device->host copy of the
          output inside every timed step; the streamed call overlaps a step's
          upload with its neighbours' kernels and downloads (the one-at-a-time
          call is reported beside it).
fp64_plain : the plain FP64 method on the same signal at the same N.
accuracy   : rel-L2 and max error of both forms against cuFFT's FP64 Z2Z
             transform of the same input (the FP64 direct-FFT checker).
roofline   : the slower of the two kernels (stage 1: convolution + S-point
             FFTs + transposed store; stage 2: M'-point FFT + demodulation),
             algorithmic bytes over its event-timed duration, against the
             measured HBM bandwidth.
cpu_baseline : the reference's own compute_soi (oracle/_ref, compiled from the
               reference sources) on the host cores, bounded sample.

--impl reference times the reference's CPU implementation alone.
Multi-GPU (torchrun): independent replicas, one per GPU (the transform does
not shard without an all-to-all, which this build does not use); value =
transforms of all ranks / max-over-ranks time.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(N=1 << 29, S=128, n_mu=5, d_mu=4, B=72)
METRIC = "GFLOP/s (5N log2 N) at N=2^29, split-FP32 vs plain FP64 GPU, at rel-L2 <=1e-6"
CPU_SAMPLE_LOG2N = 26

# The two kernels of the split-precision path at this workload, their DRAM
# traffic per launch as a multiple of the algorithmic bytes (dram__bytes_read
# + dram__bytes_write from one ncu capture of the same kernel instance on the
# same per-segment geometry, which carries to N = 2^29 in proportion to the
# segments), and where that capture is summarised.  Stage 1: N = 2^26, S = 128
# (the same instance; its traffic per output does not depend on N).  Stage 2:
# N = 2^28, S = 64, the same M' = 2560 x 2048 tiles as N = 2^29, S = 128 (its
# L2 residency depends on the segment size, so a smaller M' would not carry).
KERNELS = {
    "stage1": ("k_conv_sfft_tS (stage 1: convolution + S-point FFTs + transposed store)", 1160.1 / 1208.0,
               "ncu at N=2^26, S=128 (same kernel instance), scaled by the units processed"),
    "stage2": ("k_stage2_ct (stage 2: M'-point four-step FFT + demodulation + discard)", 4378.3 / 2415.9,
               "ncu at N=2^27, S=32 (same M' tiles), scaled by the segments"),
}


# FP64 kernels of the configured plain workload (N = 2^28, S = 64): figures
# from ncu captures of the same instances (stage 1 at N = 2^26, S = 64, whose
# per-output behaviour does not depend on N; stage 2 at N = 2^26, S = 16, the
# same M' = 2560 x 2048 tiles).
FP64_PROFILE = {
    "stage1": {"fp64_pipe_frac": 0.565, "traffic_ratio": 2.369 / 2.416,
               "profile": "ncu --set full at N=2^26, S=64, same instance"},
    "stage2": {"fp64_pipe_frac": 0.245, "traffic_ratio": 5.790 / 2.416,
               "profile": "ncu --set full at N=2^26, S=16, same M' tiles"},
}


def flop(N):
    return 5.0 * N * math.log2(N)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--log2n", type=int, default=29)
    ap.add_argument("--segments", type=int, default=128)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="headline", choices=["headline", "batched"],
                    help="batched: the band-limited batch of mixed lengths (its own JSON line)")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--batch-chains", type=int, default=16)
    ap.add_argument("--vlc", action="store_true",
                    help="with the VLC round trip between the stages (use_vlc = 1, pfft.c:316-353,618-632)")
    ap.add_argument("--precision", default="split", choices=["split", "fp64"],
                    help="precision of the main leg (fp64: the plain method, for per-kernel profiling runs)")
    ap.add_argument("--no-config2", action="store_true",
                    help="skip the plain FP64 leg at N=2^28, S=64 (the configured FP64 workload)")
    ap.add_argument("--ref-log2n", type=int, default=None,
                    help="reference arm: transform size (default: the headline --log2n)")
    return ap.parse_args()


# ---------------------------------------------------------------- helpers --

def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML polled from a thread every `period` seconds (read-only
    queries), else nvidia-smi at its 200 ms minimum."""
    # NVML clock-event reason bits (nvml.h): sw power cap 0x4, hw slowdown
    # 0x8, sw thermal 0x20, hw thermal 0x40, hw power brake 0x80
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index, period=0.005):
        self.index = index
        self.period = period
        self.proc = None
        self.lines = []
        self.samples = []          # (sm_mhz, reason bits)
        self.max_mhz = None
        self.stop = threading.Event()
        self.t = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _poll(self, nv, h):
        while not self.stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                try:
                    bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                except AttributeError:
                    bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.samples.append((float(mhz), int(bits)))
            except Exception:
                pass
            self.stop.wait(self.period)

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.t.start()
            return self
        except Exception:
            self.t = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        elif self.t is not None:
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], self.max_mhz, set()
        if self.samples:
            for mhz, bits in self.samples:
                sm.append(mhz)
                for n, b in self.BITS.items():
                    if bits & b:
                        reasons.add(n)
            src = "nvml"
        else:
            src = "nvidia-smi"
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for l in self.lines:
                f = [v.strip() for v in l.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "sm_mhz_min": min(sm), "source": src}


def gpu_local_cpus(index):
    """The host CPUs NVML lists as local to GPU `index` (its NUMA node), or
    None.  Read-only query."""
    try:
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(index)
        bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
        h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        words = pynvml.nvmlDeviceGetCpuAffinity(h, (os.cpu_count() + 63) // 64)
        cpus = {64 * w + b for w, m in enumerate(words) for b in range(64) if (m >> b) & 1}
        cpus &= os.sched_getaffinity(0)
        return cpus or None
    except Exception:
        return None


def dist_setup(args):
    """One process per GPU (torchrun's RANK/LOCAL_RANK/WORLD_SIZE); NCCL for
    the barrier and the max-over-ranks time, gloo where there is no GPU."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            backend = "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, v, device=None):
    """The largest of the ranks' values (the job's time is its slowest rank's)."""
    if not pg:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def job_value(world, flop_per_step, steps, ms):
    """Whole-job throughput: every rank's steps over the slowest rank's time."""
    return world * flop_per_step * steps / (ms / 1e3) / 1e9


def make_signal(N, seed, device):
    """complex128 Gaussian + 64 tones, built on the GPU in FP64."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    x = torch.complex(torch.randn(N, generator=g, device=device, dtype=torch.float64),
                      torch.randn(N, generator=g, device=device, dtype=torch.float64))
    n = torch.arange(N, device=device, dtype=torch.int64)
    gc = torch.Generator().manual_seed(seed + 1)
    for _ in range(64):
        k0 = int(torch.randint(0, N, (1,), generator=gc))
        frac = float(torch.rand(1, generator=gc, dtype=torch.float64))
        amp = 10.0 ** float(torch.empty(1, dtype=torch.float64).uniform_(-6, 0, generator=gc))
        ph0 = float(torch.rand(1, generator=gc, dtype=torch.float64)) * 2 * math.pi
        m = torch.remainder(n * k0, N).to(torch.float64)
        ph = (m + frac * n.to(torch.float64)) * (2 * math.pi / N) + ph0
        x += amp * torch.polar(torch.ones_like(ph), ph)
        del m, ph
    del n
    return x


def cpu_baseline(log2n, S, repeat=4, threads=None, ranks=1):
    """The reference's compute_soi compiled from its own sources (oracle/_ref),
    `ranks` forked ranks x T OpenMP threads each, best of `repeat` runs as the
    reference's driver reports (test.c:217, REPEAT = 4)."""
    from oracle import oracle
    import numpy as np
    if not oracle.ref_available():
        return None
    N = 1 << log2n
    ncpu = os.cpu_count() or 8
    k = S // ranks
    ntg = min(S // 4, 8)
    T = threads or max(ntg, (ncpu // ranks) // ntg * ntg)
    r = np.random.default_rng(1)
    x = r.standard_normal(N) + 1j * r.standard_normal(N)
    _, best, times = oracle.run_reference(x, ranks, k, threads=T, repeat=repeat, return_times=True)
    del x
    return {"value": flop(N) / best / 1e9, "mean_value": flop(N) / statistics.mean(times) / 1e9,
            "unit": "GFLOP/s", "cores": ranks * T, "kind": "reference",
            "sample": "reference compute_soi (pfft.c + parallel_filter_subsampling.cpp built here, "
                      "DFTI backed by the oracle FFT, not MKL) at N=2^%d, S=%d, mu=5/4, B=72, FP64, "
                      "%d rank%s x %d threads on %d host cores, best of %d runs (test.c:217)"
                      % (log2n, S, ranks, "s" if ranks > 1 else "", T, ncpu, repeat),
            "seconds_per_transform": best, "seconds_all": times}


# ------------------------------------------------------------- reference ---

def run_reference(args):
    # the reference's CPU path runs once, on rank 0; other ranks exit without
    # work (no process group is needed)
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # the headline transform itself (N = 2^29, S = 128: ~14 s per run on 16
    # host threads); the reference's driver times REPEAT = 4 runs and reports
    # the best (test.c:217), so the arm runs 1 + min(steps, 3) and reports the
    # best of the runs after the first
    log2n = args.ref_log2n or args.log2n
    repeat = 1 + max(1, min(args.steps, 3))
    res = cpu_baseline(log2n, args.segments, repeat=repeat)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/soi_ref_run is not built"}))
        return
    timed_runs = res["seconds_all"][1:] or res["seconds_all"]
    best = min(timed_runs)
    N = 1 << log2n
    value = flop(N) / best / 1e9
    cb = {k: res[k] for k in ("unit", "cores", "kind")}
    cb.update(value=value, sample="%s; the first run untimed" % res["sample"])
    # the reference's own CPU configuration (N = 2^20, 8 ranks x 2 threads, best of 4)
    try:
        c1 = cpu_baseline(20, 8, repeat=4, threads=2, ranks=8)
        config1 = {k: c1[k] for k in ("value", "unit", "cores", "kind", "sample")} if c1 else None
    except Exception as e:
        config1 = {"error": str(e)[:200]}
    line = {"metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": args.gpus,
            "steps": len(timed_runs), "warmup": 1,
            "ms_per_step": best * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
            "data": "synthetic: seeded i.i.d. complex Gaussian",
            "config": {"workload": "SOI FFT, reference CPU path (FP64), N=2^%d, S=%d, mu=5/4, B=72"
                                   % (log2n, args.segments),
                       "N": N, "S": args.segments, "mu": "5/4", "B": 72,
                       "same_size_as_gpu_arm": log2n == args.log2n},
            "cpu_baseline": cb,
            "cpu_config1": config1,
            "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ------------------------------------------------------------------- ours ---

def run_ours(args):
    import numpy as np
    import torch
    import soi_fft_b200 as sb

    world, rank, local, pg = dist_setup(args)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    N, S = 1 << args.log2n, args.segments
    # a dedicated stream, handed to the library so its kernels and the timing
    # events share one stream
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)

    x128 = make_signal(N, 1234, dev)
    split = args.precision == "split"
    PREC = sb.PRECISION_SPLIT_FP32 if split else sb.PRECISION_FP64
    ELEM = 8 if split else 16
    x32 = x128.to(torch.complex64) if split else x128

    def new_desc(prec):
        d = sb.SoiDescriptor(N=N, precision=prec, device=local, stream=stream.cuda_stream, use_vlc=int(args.vlc))
        d.init(S)
        return d

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks_(v):
        return max_over_ranks(pg, v, dev)

    def timed(d, src, dst, steps, warmup, per_stage=False):
        # device-resident steps go through the non-waiting entry point
        # (soi_compute_async_status): the K transforms run back to back on the
        # descriptor's stream, and soi_check_status reads the stage-2 error
        # word once after them, so host round trips between steps stay out
        # of the device time; the per-stage leg waits after every step to
        # read the library's stage events
        for _ in range(warmup):
            d.compute_into(src, dst)
        if per_stage:
            d.set_timing(True)
        st = []
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            if per_stage:
                d.compute_into(src, dst)
                st.append(d.timings())
            else:
                d.compute_async(src, dst)
        e1.record(stream)
        if not per_stage:
            d.check()
        barrier()
        d.set_timing(False)
        return e0.elapsed_time(e1), st

    # ---- split precision, device-resident (the headline `value`; with
    # --precision fp64 the plain method in its place, for profiling runs)
    d32 = new_desc(PREC)
    y32 = torch.empty_like(x32)
    peaks = measured_peaks()
    launches_per_step = d32.kernels_per_compute() if hasattr(d32, "kernels_per_compute") else None
    with ClockSampler(local) as clk:
        ms, _ = timed(d32, x32, y32, args.steps, args.warmup)
    clocks = clk.summary()
    ms = max_over_ranks_(ms)
    ms_step = ms / args.steps
    value = world * flop(N) * args.steps / (ms / 1e3) / 1e9

    # per-kernel timing (events recorded by the library on the same stream)
    _, st = timed(d32, x32, y32, max(2, args.steps // 2), 0, per_stage=True)
    stage1 = statistics.mean(s["stage1_ms"] for s in st)
    stage2 = statistics.mean(s["stage2_ms"] for s in st)
    vlc_ms = statistics.mean(s["vlc_ms"] for s in st)

    # ---- accuracy vs the FP64 direct FFT (cuFFT Z2Z, checker only)
    X = torch.fft.fft(x128)
    nX = torch.linalg.norm(X)
    acc32 = {"rel_l2": float(torch.linalg.norm(y32.to(torch.complex128) - X) / nX),
             "max_err": float(torch.sqrt(torch.max((y32.to(torch.complex128) - X).abs() ** 2) /
                                         torch.max(X.abs() ** 2)))}

    # ---- end to end through the C ABI with pinned host buffers: every step
    # uploads its input and downloads its result.  The streamed call overlaps
    # one step's upload with the previous step's kernels and download; the
    # one-at-a-time call (compute_soi's form) is reported beside it.
    # pinned buffers on the GPU's own NUMA node (allocated and first touched
    # from its local CPUs, as a deployment pins its host threads), the
    # previous affinity restored after the e2e runs
    old_aff = os.sched_getaffinity(0)
    local_cpus = gpu_local_cpus(local)
    if local_cpus:
        os.sched_setaffinity(0, local_cpus)
    h_in = torch.empty(N, dtype=x32.dtype, pin_memory=True)
    h_in.copy_(x32)
    h_out = torch.empty(N, dtype=x32.dtype, pin_memory=True)
    e2e_steps = max(3, min(args.steps, 20))
    hi, ho = h_in.numpy(), h_out.numpy()
    d32.compute_stream([hi], [ho])
    e2e_matches = bool(torch.equal(h_out, y32.cpu()))
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    d32.compute_stream([hi] * e2e_steps, [ho] * e2e_steps)
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks_(e0.elapsed_time(e1) / e2e_steps)
    e2e_value = world * flop(N) / (e2e_ms / 1e3) / 1e9
    e0.record(stream)
    for _ in range(2):
        d32.compute_into(hi, ho)
    e1.record(stream)
    barrier()
    single_ms = max_over_ranks_(e0.elapsed_time(e1) / 2)
    # the host link's own time for one step's bytes: the same upload and
    # download at once on two streams, no kernels (the streamed call's floor)
    s_up, s_dn = torch.cuda.Stream(local), torch.cuda.Stream(local)
    d_tmp = torch.empty_like(x32)
    link = []
    for _ in range(3):
        torch.cuda.synchronize()
        e0.record(s_up)
        s_dn.wait_event(e0)
        with torch.cuda.stream(s_up):
            d_tmp.copy_(h_in, non_blocking=True)
        with torch.cuda.stream(s_dn):
            h_out.copy_(y32, non_blocking=True)
        s_up.wait_stream(s_dn)
        e1.record(s_up)
        e1.synchronize()
        link.append(e0.elapsed_time(e1))
    link_ms = max_over_ranks_(min(link))
    del d_tmp
    d32.free()
    del h_in, h_out
    os.sched_setaffinity(0, old_aff)

    # ---- plain FP64 method at the same N
    fp64 = None
    if not args.no_fp64 and split:
        d64 = new_desc(sb.PRECISION_FP64)
        y64 = torch.empty_like(x128)
        ms64, _ = timed(d64, x128, y64, max(2, min(args.steps, 5)), 2)
        ms64 = max_over_ranks_(ms64) / max(2, min(args.steps, 5))
        acc64 = float(torch.linalg.norm(y64 - X) / nX)
        fp64 = {"value": world * flop(N) / (ms64 / 1e3) / 1e9, "unit": "GFLOP/s", "ms_per_step": ms64,
                "rel_l2_vs_fp64_direct_fft": acc64}
        d64.free()
        del y64

    # ---- roofline of the dominant kernel.  Both stages move the same
    # algorithmic bytes: stage 1 reads the N inputs and writes the S*M'
    # transposed values, stage 2 reads those and writes the N outputs.
    geom = sb.plan_geometry(N, S, PREC)
    alg_bytes = (N + geom["M_hat"] * S) * ELEM
    hbm = peaks["hbm_gbs"] if peaks else 6650.0
    dom_ms = max(stage1, stage2)
    achieved = alg_bytes / (dom_ms / 1e3) / 1e9
    name, traffic_ratio, traffic_source = KERNELS["stage1" if stage1 >= stage2 else "stage2"]
    if not split or N != 1 << 29 or S != 128:
        traffic_ratio, traffic_source = None, None          # the captures cover the headline instance only
    roofline = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": "measured" if peaks else "fallback",
                "traffic": traffic_ratio * alg_bytes if traffic_ratio else None,
                "traffic_source": traffic_source if traffic_ratio else None,
                "algorithmic_bytes_per_launch": alg_bytes,
                "stage1_ms": stage1, "stage2_ms": stage2, "vlc_ms": vlc_ms if args.vlc else None,
                "pipeline_achieved_gbs": 2 * alg_bytes / (ms_step / 1e3) / 1e9}

    # ---- the configured plain-FP64 workload: N = 2^28 complex128, S = 64,
    # Gaussian + 64 tones; per-kernel CUDA-event times and HBM GB/s against
    # the measured peak (algorithmic bytes: each kernel reads and writes
    # (1 + mu) N complex128 values between them), accuracy against cuFFT Z2Z
    config2 = None
    if not args.no_config2 and split and not args.no_fp64:
        del X
        N2, S2 = 1 << 28, 64
        x2 = make_signal(N2, 2828, dev)
        d2 = sb.SoiDescriptor(N=N2, precision=sb.PRECISION_FP64, device=local, stream=stream.cuda_stream).init(S2)
        y2 = torch.empty_like(x2)
        k2 = max(3, min(args.steps, 10))
        ms2, _ = timed(d2, x2, y2, k2, 3)
        ms2 = max_over_ranks_(ms2) / k2
        _, st2 = timed(d2, x2, y2, k2, 0, per_stage=True)
        g2 = sb.plan_geometry(N2, S2, sb.PRECISION_FP64)
        b2 = (N2 + g2["M_hat"] * S2) * 16
        X2 = torch.fft.fft(x2)
        acc2 = float(torch.linalg.norm(y2 - X2) / torch.linalg.norm(X2))
        del X2
        kern = {}
        var = sb.plan_variant(N2, S2, sb.PRECISION_FP64)
        s1name = ("k_conv_sfft_tS<double, 5, 4, 8, 8, %d, %s> (convolution + 64-point FFTs + transposed store, "
                  "staged by %s)" % (var["stage1_threads"], "true" if var["stage1_staging"] == "tensor copies"
                                     else "false", var["stage1_staging"]))
        for key, kname in (("stage1", s1name),
                           ("stage2", "k_stage2_ct<double, 10, 16, 16, 8, 16, 16, 256, 2, 2> (M'-point four-step "
                                      "FFT + demodulation + discard)")):
            kms = statistics.mean(t[key + "_ms"] for t in st2)
            gbs = b2 / (kms / 1e3) / 1e9
            kern[key] = dict(kernel=kname, ms=kms, algorithmic_bytes=b2, achieved_gbs=gbs, peak_gbs=hbm,
                             frac_hbm=gbs / hbm, **FP64_PROFILE.get(key, {}))
            if "traffic_ratio" in kern[key]:
                kern[key]["traffic"] = kern[key]["traffic_ratio"] * b2
        config2 = {"workload": "plain FP64, N=2^28 complex128, S=64, mu=5/4, B=72, Gaussian + 64 tones",
                   "value": world * flop(N2) / (ms2 / 1e3) / 1e9, "unit": "GFLOP/s", "ms_per_step": ms2,
                   "steps": k2, "rel_l2_vs_fp64_direct_fft": acc2, "kernels": kern}
        d2.free()
        del x2, y2

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(min(args.log2n, CPU_SAMPLE_LOG2N), S, repeat=4)
        except Exception as e:  # the checker failing must not hide the measurement
            cpu = {"error": str(e)[:200]}
        if cpu and "value" in cpu:
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32" if split else "f64",
                "data": "synthetic: seeded complex Gaussian + 64 tones, amplitudes log-uniform [1e-6, 1]",
                "config": {"workload": "SOI FFT %s, N=2^%d %s, S=%d, mu=5/4, B=72%s"
                                       % ("split-precision" if split else "plain FP64", args.log2n,
                                          "complex64" if split else "complex128", S,
                                          ", VLC round trip" if args.vlc else ""),
                           "use_vlc": bool(args.vlc),
                           "N": N, "S": S, "mu": "5/4", "B": 72, "precision": "split_fp32" if split else "fp64",
                           "l2": "inputs (%d MiB) larger than L2 (126 MB), no flush" % (N * ELEM >> 20),
                           "parallelism": "replicas x%d" % world},
                "accuracy_vs_fp64_direct_fft": acc32,
                "fp64_plain": fp64,
                "fp64_config2": config2,
                "split_over_fp64": (value / fp64["value"]) if fp64 else None,
                "roofline": roofline,
                "cpu_baseline": cpu,
                "e2e": {"value": e2e_value, "unit": "GFLOP/s", "ms_per_step": e2e_ms,
                        "h2d_bytes_per_step": N * ELEM, "d2h_bytes_per_step": N * ELEM,
                        "api": "soi_compute_stream_status, %d transforms per call, pinned host buffers" % e2e_steps,
                        "matches_device_result": e2e_matches,
                        "host_link_ms": link_ms,
                        "host_link_note": "one step's upload and download at once on two streams, no kernels: "
                                          "the streamed call's floor",
                        "host_cpus": "%d NUMA-local to the GPU" % len(local_cpus) if local_cpus else "unpinned",
                        "one_at_a_time": {"api": "soi_compute_oop_status", "ms_per_step": single_ms,
                                          "value": world * flop(N) / (single_ms / 1e3) / 1e9}},
                "gpu_launches": launches_per_step * args.steps,
                "clocks": clocks}
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()


# ---------------------------------------------------------------- batched ---

def run_batched(args):
    """The band-limited batch: --batch-count transforms, N log-uniform over
    2^14..2^24 (powers of two), k from 4 to 64 growing with N, complex64,
    each input's spectrum on a random 5 % band, only the segments that
    overlap the band computed; one CUDA graph per execute.  value = nominal
    5 N log2 N over the batch's transforms per second (the work skipped outside
    the band is credited, as a banded transform's user would count it);
    also transforms/s and the band's accuracy against the FP64 direct FFT."""
    import torch
    import soi_fft_b200 as sb
    from soi_fft_b200 import batch as sbb
    world, rank, local, pg = dist_setup(args)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    # out of place; inputs and outputs together capped to fit HBM with room
    # for the chains' scratch
    free, _ = torch.cuda.mem_get_info(dev)
    cap = int(0.4 * free) // 8
    wl = sbb.band_workload(args.batch_count, 14, 24, band=0.05, seed=42 + rank, device=dev, max_total=cap)
    outs = [torch.empty_like(w["x"]) for w in wl]
    t0 = time.perf_counter()
    b = sbb.SoiBatch([(w["x"], y, w["k"], w["seg_lo"], w["seg_hi"]) for w, y in zip(wl, outs)],
                     precision=sb.PRECISION_SPLIT_FP32, chains=args.batch_chains, tune=True, device=local)
    build_s = time.perf_counter() - t0
    info = b.info()
    for _ in range(args.warmup):
        b.execute(stream)
    b.check()
    # accuracy: the first 32 transforms' bands against the FP64 direct FFT
    errs = []
    for w, y in zip(wl[:32], outs):
        X = torch.fft.fft(w["x"].to(torch.complex128))
        M = w["N"] // w["k"]
        sl = slice(w["seg_lo"] * M, w["seg_hi"] * M)
        errs.append(float(torch.linalg.norm(y[sl].to(torch.complex128) - X[sl]) / torch.linalg.norm(X[sl])))
        del X
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            b.execute(stream)
        e1.record(stream)
        e1.synchronize()
    b.check()
    clocks = clk.summary()
    ms = max_over_ranks(pg, e0.elapsed_time(e1), dev)
    nominal = sum(flop(w["N"]) for w in wl)
    band_frac = sum((w["seg_hi"] - w["seg_lo"]) / w["k"] * w["N"] for w in wl) / sum(w["N"] for w in wl)
    if rank == 0:
        line = {"metric": "GFLOP/s (5N log2 N, nominal) over a band-limited batch of mixed lengths",
                "value": world * nominal * args.steps / (ms / 1e3) / 1e9, "unit": "GFLOP/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic: band-limited complex Gaussian (random 5 %% band), inverse FFT in FP64, rounded "
                        "once to complex64",
                "config": {"workload": "batched banded SOI: %d transforms, N = 2^14..2^24 log-uniform, k = 4..64, "
                                       "mu=5/4, B=72, split precision, segments of interest only" % len(wl),
                           "transforms": len(wl), "total_points": sum(w["N"] for w in wl),
                           "segments_computed_fraction": band_frac,
                           "l2": "batch (%d MiB) larger than L2, no flush" % (sum(w["N"] for w in wl) * 8 >> 20),
                           "parallelism": "replicas x%d" % world},
                "transforms_per_s": world * len(wl) * args.steps / (ms / 1e3),
                "accuracy_vs_fp64_direct_fft": {"band_rel_l2_max": max(errs), "band_rel_l2_median":
                                                statistics.median(errs), "sample": len(errs)},
                "batch": dict(info, build_and_tune_s=build_s, plans=b.plans()),
                "gpu_launches": info["kernels_per_execute"] * args.steps,
                "clocks": clocks}
        print(json.dumps(line))
    b.free()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
