#!/usr/bin/env python
"""Benchmark of the batched FFT engine on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workloads (synthetic, seeded; shapes from the reference benchmark configs):
  cfft2g      (default) CFFT<float> orders 14/16/20, 2 GiB each, forward +
              backward, autotuned plans; per-order plain / fast / TC comparison.
  rfft12      RFFT<float> order 12 (N = 4096), 8192 Hann-windowed frames of
              3 sinusoids + N(0, 0.1^2) noise; one step = forward to AoS,
              forward to split SoA and forward_sqr_mag over the whole batch
              (plain FP32 CUDA-core form).
  cfft10      one CFFT<float> order-10 transform, forward + backward (latency).
  mixed       20,000 transforms of orders 6..16, CFFT and RFFT, one graph.
  cfft64      CFFT<double> order 16 x 512, forward + backward.
  stft        fused STFT front end (framing, Hann window, forward_sqr_mag).
  istft       fused inverse STFT (filter, RFFT backward, window, overlap-add).

Metric: algorithmic HBM bytes (one read of each input, one write of each
output; twiddles excluded) per second, in GB/s; roofline = the measured HBM
copy bandwidth in MEASURED_PEAKS.json. Inputs: two rotating buffer sets, each
step touching > 2x the 126 MB L2, so no step starts with its data in L2.

--impl reference times the reference's own CPU code (zldsp::fft compiled
against the project's Highway-API shim, oracle/_ref) on all host cores, on a
bounded sample of the same workload, and prints the same metric.

Multi-GPU: replicas only (every transform is independent): each rank runs
the whole workload on its own GPU; value = bytes of all ranks / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Batched FFT HBM GB/s (% of roofline), TC-split vs plain FP32 at equal error"
FORMS = {
    "plain": "plain (the reference's Stockham radix-4/8 DIT on CUDA cores, bit-identical results)",
    "fast": "fast-twiddle plain form: CUDA cores, radix-16 groups' twiddles from two table values per butterfly",
    "tc": "tensor-core split FP16 hi/lo, FP32 accumulate (256-point passes), plain elsewhere",
    "tuned": "autotuned per order among plain, fast-twiddle and tensor-core split forms (see schedules)",
    "macro": "the reference's macro path (DIF macro stages + per-segment Stockham + transposed store) as a "
             "small-cache host runs it, bit-identical to the reference there",
}


# ------------------------------------------------------------------ helpers
def pcie_probe(nbytes=256 << 20, reps=5):
    """Pinned-memory copy rates of this box (GB/s): host->device, device->host,
    and both at once on two streams. They bound the host-API (e2e) figure."""
    import torch
    h1 = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    h2 = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d1 = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    d2 = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def h2d():
        with torch.cuda.stream(s1):
            d1.copy_(h1, non_blocking=True)

    def d2h():
        with torch.cuda.stream(s2):
            h2.copy_(d2, non_blocking=True)

    def both():
        h2d()
        d2h()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps

    th, td, tb = timed(h2d), timed(d2h), timed(both)
    del h1, h2, d1, d2
    return {"h2d": round(nbytes / th / 1e9, 2), "d2h": round(nbytes / td / 1e9, 2),
            "both_directions": round(2 * nbytes / tb / 1e9, 2)}


class SlicePipe:
    """Host-path pipeline over slices of a step: slice s's H2D copy runs on one
    stream, its work on a second once the copy is in, and the D2H copy of its
    result on a third once the work is done, so copies in both directions
    overlap each other and the work of neighbouring slices."""

    def __init__(self, device):
        import torch
        self.streams = [torch.cuda.Stream(device) for _ in range(3)]

    def run(self, slices):
        """slices: (h2d, work, d2h) callables, each taking the stream it runs on."""
        import torch
        sh, sc, sd = self.streams
        start = torch.cuda.Event()
        start.record(torch.cuda.current_stream())
        for st in self.streams:
            st.wait_event(start)
        for h2d, work, d2h in slices:
            with torch.cuda.stream(sh):
                h2d(sh)
            e = torch.cuda.Event()
            e.record(sh)
            sc.wait_event(e)
            with torch.cuda.stream(sc):
                work(sc)
            e = torch.cuda.Event()
            e.record(sc)
            sd.wait_event(e)
            with torch.cuda.stream(sd):
                d2h(sd)
        for st in self.streams:
            st.synchronize()


def e2e_bound(bytes_per_step, h2d_bytes, d2h_bytes, pcie):
    """Highest e2e GB/s the copies allow: the step takes at least the longest of
    its H2D copy, its D2H copy, and both sharing the link."""
    t = max(h2d_bytes / (pcie["h2d"] * 1e9), d2h_bytes / (pcie["d2h"] * 1e9),
            (h2d_bytes + d2h_bytes) / (pcie["both_directions"] * 1e9))
    return bytes_per_step / t / 1e9 if t > 0 else None


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        if d.get("hbm_gbs"):
            return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel_key: str):
    """DRAM bytes per launch from the committed ncu summary (profiles/ncu_traffic.json)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    v = d.get(kernel_key)
    return None if v is None else float(v.get("dram_bytes_per_launch")) if isinstance(v, dict) else float(v)


class ClockSampler:
    """Samples SM clock, power and throttle reasons through NVML in a thread."""

    REASONS = {
        "gpu_idle": 0x1, "applications_clocks_setting": 0x2, "sw_power_cap": 0x4, "hw_slowdown": 0x8,
        "sync_boost": 0x10, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
        "hw_power_brake_slowdown": 0x80, "display_clock_setting": 0x100,
    }

    def __init__(self, device_index: int, period_s: float = 0.002):
        self.idx = device_index
        self.period = period_s
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.ok = False

    def _sample(self):
        nv = self.nv
        sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
        try:
            reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        except Exception:
            reasons = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
        try:
            pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
        except Exception:
            pw = None
        self.samples.append((sm, reasons, pw))

    def _run(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception:
                pass
            time.sleep(self.period)

    def start(self):
        if self.ok:
            self._sample()
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()

    def stop(self):
        if self.ok and self._t:
            self._stop.set()
            self._t.join()
            self._sample()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"], "samples": 0}
        mhz = [s[0] for s in self.samples]
        mask = 0
        for s in self.samples:
            mask |= int(s[1])
        reasons = [k for k, v in self.REASONS.items() if mask & v and k != "gpu_idle"]
        pw = [s[2] for s in self.samples if s[2] is not None]
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.samples), "power_w_max": max(pw) if pw else None}


def host_info():
    """The CPU a baseline runs on: model, hardware threads, cache sizes, and the
    reference's algorithm switch there (get_switch_order<F>,
    src/common/zldsp_fft_common_system.hpp:132-157), which decides whether the
    reference timed its micro-only Stockham path or its macro DIF path."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    # The reference reads these through sysconf(_SC_LEVEL{1_DCACHE,2_CACHE,3_CACHE}_SIZE); Python's
    # os.sysconf does not know those names, so libc is asked directly (glibc's values of the three
    # constants on Linux: 188, 191, 194).
    caches = {}
    try:
        import ctypes
        libc = ctypes.CDLL(None)
        libc.sysconf.restype = ctypes.c_long
        libc.sysconf.argtypes = [ctypes.c_int]
        for key, code in (("l1d_bytes", 188), ("l2_bytes", 191), ("l3_bytes", 194)):
            v = int(libc.sysconf(code))
            caches[key] = v if v >= 0 else None
    except (OSError, AttributeError):
        caches = {"l1d_bytes": None, "l2_bytes": None, "l3_bytes": None}
    switch = {}
    try:
        from oracle import oracle as O
        for prec in ("f32", "f64"):
            l1, sw = O.ref_switch_order(prec) if O.ref_available() else (None, None)
            switch[prec] = {"max_l1_order": l1, "switch_order": sw,
                            "source": "the reference's own code" if O.ref_available() else "unavailable"}
    except Exception as e:  # reported, never required
        switch = {"error": str(e)[:120]}
    return {"cpu_model": model, "hw_threads": os.cpu_count(), **caches, "reference_switch_order": switch}


# ------------------------------------------------------------------ workloads
def hann_frames(b, n, seed):
    """3 sinusoids (f ~ U(0, 0.5) cycles/sample, A ~ U[0.1, 1], phase ~ U[0, 2pi))
    + N(0, 0.1^2) noise, times a periodic Hann window."""
    rng = np.random.default_rng(seed)
    t = np.arange(n, dtype=np.float64)
    w = 0.5 - 0.5 * np.cos(2 * np.pi * t / n)
    out = np.empty((b, n), np.float32)
    chunk = 1024
    for s in range(0, b, chunk):
        e = min(b, s + chunk)
        m = e - s
        f = rng.uniform(0, 0.5, (m, 3, 1))
        a = rng.uniform(0.1, 1, (m, 3, 1))
        ph = rng.uniform(0, 2 * np.pi, (m, 3, 1))
        sig = (a * np.sin(2 * np.pi * f * t + ph)).sum(1) + rng.normal(0, 0.1, (m, n))
        out[s:e] = (sig * w).astype(np.float32)
    return out


class Rfft12:
    name = "rfft12"
    desc = "RFFT<float> order 12 (N=4096) x 8192 frames: forward AoS + forward SoA + forward_sqr_mag"
    order, n, batch = 12, 4096, 8192
    dtype = "f32"

    def __init__(self):
        n, nb, b = self.n, self.n // 2 + 1, self.batch
        self.nb = nb
        self.op_bytes = {  # algorithmic bytes of one op over the batch
            "r2c_fwd_aos": b * (4 * n + 8 * nb),
            "r2c_fwd_soa": b * (4 * n + 8 * nb),
            "r2c_sqr_mag": b * (4 * n + 4 * nb),
        }
        self.bytes_per_step = sum(self.op_bytes.values())

    # ---- GPU (ours)
    def setup(self, device):
        import torch
        import zldsp_fft_b200 as Z
        self.Z = Z
        self.plan = Z.Plan(Z.R2C, self.order, np.float32, device=device)
        host = hann_frames(self.batch, self.n, 1002)
        self.host_in = host
        b, n, nb = self.batch, self.n, self.nb
        self.sets = []
        for _ in range(2):  # rotating sets: each step reads/writes > 2x L2
            d = {
                "in": torch.from_numpy(host).to(device),
                "aos": torch.empty((b, nb, 2), dtype=torch.float32, device=device),
                "re": torch.empty((b, nb), dtype=torch.float32, device=device),
                "im": torch.empty((b, nb), dtype=torch.float32, device=device),
                "sqr": torch.empty((b, nb), dtype=torch.float32, device=device),
            }
            self.sets.append(d)
        torch.cuda.synchronize(device)

    def ops(self, step):
        """[(op_name, launch_fn)] for one step on rotating set step % 2."""
        Z, p, d = self.Z, self.plan, self.sets[step % 2]
        b = self.batch

        def fwd_aos(st):
            p.exec_device(Z.FORWARD, Z.AOS, Z.AOS, d["in"].data_ptr(), None, d["aos"].data_ptr(), None, b, stream=st)

        def fwd_soa(st):
            p.exec_device(Z.FORWARD, Z.AOS, Z.SOA, d["in"].data_ptr(), None, d["re"].data_ptr(), d["im"].data_ptr(),
                          b, stream=st)

        def sqr(st):
            p.exec_device(Z.FORWARD_SQR_MAG, Z.AOS, Z.AOS, d["in"].data_ptr(), None, d["sqr"].data_ptr(), None, b,
                          stream=st)

        return [("r2c_fwd_aos", fwd_aos), ("r2c_fwd_soa", fwd_soa), ("r2c_sqr_mag", sqr)]

    def take_launches(self):
        return self.plan.take_launch_count()

    def cpu_sample_desc(self, frames):
        return f"{frames} of {self.batch} frames, same ops as one step"

    # ---- end to end through the host API (pinned host buffers)
    def setup_e2e(self):
        import torch
        b, n, nb = self.batch, self.n, self.nb
        self.h_in = torch.from_numpy(self.host_in).pin_memory()
        self.h_aos = torch.empty((b, nb, 2), dtype=torch.float32).pin_memory()
        self.h_re = torch.empty((b, nb), dtype=torch.float32).pin_memory()
        self.h_im = torch.empty((b, nb), dtype=torch.float32).pin_memory()
        self.h_sqr = torch.empty((b, nb), dtype=torch.float32).pin_memory()
        self.e2e_h2d = 3 * self.h_in.numel() * 4
        self.e2e_d2h = (self.h_aos.numel() + self.h_re.numel() + self.h_im.numel() + self.h_sqr.numel()) * 4

    def e2e_step(self):
        Z, p, b = self.Z, self.plan, self.batch
        p.exec_host(Z.FORWARD, Z.AOS, Z.AOS, self.h_in.data_ptr(), None, self.h_aos.data_ptr(), None, b)
        p.exec_host(Z.FORWARD, Z.AOS, Z.SOA, self.h_in.data_ptr(), None, self.h_re.data_ptr(), self.h_im.data_ptr(), b)
        p.exec_host(Z.FORWARD_SQR_MAG, Z.AOS, Z.AOS, self.h_in.data_ptr(), None, self.h_sqr.data_ptr(), None, b)

    # ---- CPU: the reference's own code (or the oracle restatement)
    def cpu_run(self, frames, threads, kind):
        from oracle import oracle as O
        x = self.host_in[:frames]
        frames = x.shape[0]
        if kind == "reference":
            plan = O.RefPlan("r2c", self.order, "f32", threads)
            outs = (np.empty((frames, self.nb), np.complex64),
                    (np.empty((frames, self.nb), np.float32), np.empty((frames, self.nb), np.float32)),
                    np.empty((frames, self.nb), np.float32))
            t0 = time.perf_counter()
            plan.rfft_forward(x, O.AOS, out=outs[0])
            plan.rfft_forward(x, O.SOA, out=outs[1])
            plan.rfft_forward(x, sqr_mag=True, out=outs[2])
            dt = time.perf_counter() - t0
            plan.close()
        else:
            t0 = time.perf_counter()
            O.rfft_forward_port(x)
            O.rfft_forward_port(x)
            O.rfft_forward_port(x, sqr_mag=True)
            dt = time.perf_counter() - t0
        return self.bytes_per_step * frames / self.batch, dt


class Cfft2G:
    """CFFT<float> orders 14, 16 and 20, each batched to 2 GiB of complex64
    input (batch 16384 / 4096 / 256); one step = forward then backward of all
    three (plain FP32 form). re, im ~ U[-1, 1), seed 1003."""
    name = "cfft2g"
    l2 = "each op reads 2 GiB and writes 2 GiB, > 16x L2 (no L2 flush needed)"
    desc = "CFFT<float> orders 14/16/20 x 2 GiB complex64 each (batch 16384/4096/256), forward + backward"
    orders = (14, 16, 20)
    total = 1 << 28  # complex elements per order (2 GiB)
    dtype = "f32"

    def __init__(self, total_log2=28, form="tuned"):
        self.total = 1 << total_log2
        self.form = form
        self.desc = self.desc + {"tc": ", tensor-core split FP16 hi/lo form", "fast": ", fast-twiddle form",
                                 "plain": ", plain form (the reference's arithmetic, bit-identical)",
                                 "tuned": ", autotuned form per order",
                                 "macro": ", the reference's macro DIF path (small-cache host switch)"}[form]
        self.op_bytes = {}
        for o in self.orders:
            for d in ("fwd", "bwd"):
                self.op_bytes[f"c2c_{d}_order{o}"] = 2 * 8 * self.total  # read + write
        self.bytes_per_step = sum(self.op_bytes.values())

    def setup(self, device):
        import torch
        import zldsp_fft_b200 as Z
        self.Z = Z
        mode = {"tc": Z.MODE_TC_FP16, "fast": Z.MODE_FAST, "plain": Z.MODE_PLAIN, "tuned": Z.MODE_TUNED,
                "macro": Z.MODE_PLAIN}[self.form]
        self.tuning = None
        if self.form == "tuned":  # set-up, outside the timed region
            for o in self.orders:
                Z.autotune(Z.C2C, o, o, np.float32, device=device)
            self.tuning = {f"order{o}": Z.tuning(Z.C2C, o, np.float32, device=device) for o in self.orders}
        sw = (10, 14) if self.form == "macro" else None
        self.plans = {o: Z.Plan(Z.C2C, o, np.float32, mode=mode, device=device, switch=sw) for o in self.orders}
        g = torch.Generator(device=device)
        g.manual_seed(1003)
        # A: input (never overwritten), B: forward output, C: backward output
        self.A = (torch.rand((self.total, 2), generator=g, device=device) * 2 - 1).contiguous()
        self.B = torch.empty_like(self.A)
        self.C = torch.empty_like(self.A)
        torch.cuda.synchronize(device)
        self.host_in = None

    def ops(self, step):
        Z = self.Z
        out = []
        for o in self.orders:
            p = self.plans[o]
            b = self.total >> o

            def fwd(st, p=p, b=b):
                p.exec_device(Z.FORWARD, Z.AOS, Z.AOS, self.A.data_ptr(), None, self.B.data_ptr(), None, b, stream=st)

            def bwd(st, p=p, b=b):
                p.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, self.B.data_ptr(), None, self.C.data_ptr(), None, b, stream=st)

            out += [(f"c2c_fwd_order{o}", fwd), (f"c2c_bwd_order{o}", bwd)]
        return out

    def take_launches(self):
        return sum(p.take_launch_count() for p in self.plans.values())

    def compare(self, stream, reps):
        """Both forms at every order: GB/s of forward+backward and the relative
        L2 error of forward against numpy's FP64 FFT on 8 transforms."""
        import torch
        Z = self.Z
        out = {}
        # "macro": the reference's own algorithm on a small-cache host (its switch at order 14 with
        # micro order 10: DIF macro stages + per-segment Stockham + transposed store), bit-identical
        # to the reference built there
        for form, mode in (("plain", Z.MODE_PLAIN), ("fast", Z.MODE_FAST), ("tc_fp16", Z.MODE_TC_FP16),
                           ("macro", None)):
            res = {}
            for o in self.orders:
                if mode is None:
                    p = Z.Plan(Z.C2C, o, np.float32, device=self.A.device.index, switch=(10, 14))
                else:
                    p = Z.Plan(Z.C2C, o, np.float32, mode=mode, device=self.A.device.index)
                b = self.total >> o

                def step():
                    p.exec_device(Z.FORWARD, Z.AOS, Z.AOS, self.A.data_ptr(), None, self.B.data_ptr(), None, b,
                                  stream=stream.cuda_stream)
                    p.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, self.B.data_ptr(), None, self.C.data_ptr(), None, b,
                                  stream=stream.cuda_stream)
                for _ in range(2):
                    step()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(reps):
                    step()
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / reps
                n = 1 << o
                k = min(8, b)
                x = self.A[:k * n].cpu().numpy().astype(np.float64).view(np.complex128).reshape(k, n)
                y = self.B[:k * n].cpu().numpy().astype(np.float64).view(np.complex128).reshape(k, n)
                ref = np.fft.fft(x, axis=-1)
                err = np.linalg.norm(y - ref, axis=-1) / np.linalg.norm(ref, axis=-1)
                res[f"order{o}"] = {"gbs": round(2 * 16 * self.total / (ms / 1e3) / 1e9, 1),
                                    "max_rel_l2": float(err.max()), "tolerance": 4 * o * 2.0 ** -24}
            out[form] = res
        out["macro_host_switch"] = {"max_l1_order": 10, "switch_order": 14,
                                    "what": "the reference's macro path as a host with a 48 KiB L1d, 1 MiB L2 and "
                                            "no L3 runs it"}
        if self.tuning is not None:
            out["autotuned_plans"] = self.tuning
        return out

    batch = 1 << 14  # largest per-order batch (order 14), for sample sizing

    def cpu_sample_desc(self, frames):
        cnt = [max(1, min(frames >> max(0, o - 14), self.total >> o)) for o in self.orders]
        return (f"forward+backward of {cnt[0]}/{cnt[1]}/{cnt[2]} transforms of orders 14/16/20 "
                f"(of 16384/4096/256 per step)")

    def setup_e2e(self):
        import torch
        # host copies of A, pinned; forward into hB, backward in place in hB
        self.hA = self.A.cpu().pin_memory()
        self.hB = torch.empty_like(self.hA).pin_memory()
        self.e2e_h2d = 2 * 8 * self.total * len(self.orders)
        self.e2e_d2h = 2 * 8 * self.total * len(self.orders)

    def e2e_step(self):
        Z = self.Z
        for o in self.orders:
            p = self.plans[o]
            b = self.total >> o
            p.exec_host(Z.FORWARD, Z.AOS, Z.AOS, self.hA.data_ptr(), None, self.hB.data_ptr(), None, b)
            p.exec_host(Z.BACKWARD, Z.AOS, Z.AOS, self.hB.data_ptr(), None, self.hB.data_ptr(), None, b)

    def cpu_run(self, frames, threads, kind):
        """`frames` transforms of each order (forward + backward) on the CPU."""
        from oracle import oracle as O
        rng = np.random.default_rng(1003)
        nbytes, dt = 0.0, 0.0
        for o in self.orders:
            n = 1 << o
            cnt = max(1, min(frames >> max(0, o - 14), self.total >> o))
            x = (rng.uniform(-1, 1, (cnt, n)) + 1j * rng.uniform(-1, 1, (cnt, n))).astype(np.complex64)
            if kind == "reference":
                plan = O.RefPlan("c2c", o, "f32", threads)
                y = np.empty_like(x)
                z = np.empty_like(x)
                t0 = time.perf_counter()
                plan.cfft(x, True, out=y)
                plan.cfft(y, False, out=z)
                dt += time.perf_counter() - t0
                plan.close()
            else:
                t0 = time.perf_counter()
                O.cfft_port(O.cfft_port(x, True), False)
                dt += time.perf_counter() - t0
            nbytes += 2 * 2 * 8 * n * cnt
        return nbytes, dt


class Mixed:
    """Mixed-order batch: 20,000 transforms, order ~ U{6..16}, half CFFT<float>
    forward AoS and half RFFT<float> forward AoS, lengths and data from seed
    1004 (entries ~ U[-1, 1)). Inputs are packed back to back in one device
    buffer and outputs in another (each transform 256-byte aligned), so the
    batch is addressed through per-transform pointers. One step runs the whole
    batch with the persistent schedule replayed from a CUDA graph; the
    per-order launch loop and the un-captured persistent schedule are timed
    beside it."""
    name = "mixed"
    l2 = "each step reads 1.42 GB and writes 1.42 GB, > 10x L2 (no L2 flush needed)"
    desc = ("mixed batch: 20,000 transforms, order U{6..16}, 50% CFFT<float> forward AoS / 50% RFFT<float> "
            "forward AoS, seed 1004; persistent schedule replayed from a CUDA graph")
    count = 20000
    dtype = "f32"

    def __init__(self, autotune=True):
        self.autotune = autotune
        rng = np.random.default_rng(1004)
        self.orders = rng.integers(6, 17, self.count)
        self.is_c = rng.random(self.count) < 0.5
        n = (1 << self.orders).astype(np.int64)
        self.in_sz = np.where(self.is_c, 8 * n, 4 * n)
        self.out_sz = np.where(self.is_c, 8 * n, 8 * (n // 2 + 1))
        up = lambda v: (v + 255) // 256 * 256  # noqa: E731
        self.in_off = np.concatenate([[0], np.cumsum(up(self.in_sz))[:-1]])
        self.out_off = np.concatenate([[0], np.cumsum(up(self.out_sz))[:-1]])
        self.in_total = int(up(self.in_sz).sum())
        self.out_total = int(up(self.out_sz).sum())
        self.bytes_per_step = int(self.in_sz.sum() + self.out_sz.sum())
        self.op_bytes = {"mixed_graph": self.bytes_per_step}
        self.batch = self.count
        self.host_in = None

    def setup(self, device):
        import torch
        import zldsp_fft_b200 as Z
        self.Z = Z
        g = torch.Generator(device=device)
        g.manual_seed(1004)
        self.A = (torch.rand(self.in_total // 4, generator=g, device=device) * 2 - 1).contiguous()
        self.B = torch.zeros(self.out_total // 4, dtype=torch.float32, device=device)
        a, b = self.A.data_ptr(), self.B.data_ptr()
        # autotuned plan per order (set-up, outside the timed region): the batch's
        # plans are created in the tuned mode
        if self.autotune:
            Z.autotune(Z.C2C, 6, 16, np.float32, device=device)
            Z.autotune(Z.R2C, 6, 16, np.float32, device=device)
        self.tuning = {f"{'c2c' if k == Z.C2C else 'r2c'}{o}": Z.tuning(k, o, np.float32, device=device)
                       for k in (Z.C2C, Z.R2C) for o in range(14, 17)}
        descs = [(Z.C2C if c else Z.R2C, int(o), Z.FORWARD, a + int(io), b + int(oo))
                 for c, o, io, oo in zip(self.is_c, self.orders, self.in_off, self.out_off)]
        self.mb = Z.MixedBatch(descs, np.float32, device=device)
        torch.cuda.synchronize(device)

    def ops(self, step):
        Z = self.Z
        return [("mixed_graph", lambda st: self.mb.run(Z.SCHED_GRAPH, st))]

    def take_launches(self):
        return self.mb.take_launch_count()

    def compare(self, stream, reps):
        """GB/s and launches per step of every schedule; max relative-L2 error
        of a sample (two transforms per (kind, order)) against numpy FP64."""
        import torch
        Z = self.Z
        out = {}
        for name, sched in (("per_order_loop", Z.SCHED_PER_ORDER), ("persistent", Z.SCHED_PERSISTENT),
                            ("graph", Z.SCHED_GRAPH)):
            for _ in range(2):
                self.mb.run(sched, stream.cuda_stream)
            torch.cuda.synchronize()
            self.mb.take_launch_count()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                self.mb.run(sched, stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            out[name] = {"gbs": round(self.bytes_per_step / (ms / 1e3) / 1e9, 1), "ms": round(ms, 4),
                         "launches": self.mb.take_launch_count() // reps}
        A, B = self.A.cpu().numpy(), self.B.cpu().numpy()
        worst, seen = 0.0, {}
        for i in range(self.count):
            key = (bool(self.is_c[i]), int(self.orders[i]))
            if seen.get(key, 0) >= 2:
                continue
            seen[key] = seen.get(key, 0) + 1
            n = 1 << key[1]
            io, oo = int(self.in_off[i]) // 4, int(self.out_off[i]) // 4
            if key[0]:
                x = A[io:io + 2 * n].astype(np.float64).view(np.complex128)
                ref = np.fft.fft(x)
                y = B[oo:oo + 2 * n].astype(np.float64).view(np.complex128)
            else:
                ref = np.fft.rfft(A[io:io + n].astype(np.float64))
                y = B[oo:oo + 2 * (n // 2 + 1)].astype(np.float64).view(np.complex128)
            worst = max(worst, float(np.linalg.norm(y - ref) / np.linalg.norm(ref)))
        out["max_rel_l2_vs_fp64"] = worst
        out["tolerance_order16"] = 4 * 16 * 2.0 ** -24
        out["autotuned_multipass_plans"] = self.tuning
        return out

    def cpu_sample_desc(self, frames):
        return f"the first {frames} of the 20,000 transforms, grouped by (kind, order)"

    e2e_slices = 4
    e2e_api = ("zlfft_exec_mixed_device on 4 slices of the batch (a MixedBatch each, graph schedule), "
               "pinned host buffers, H2D / run / D2H pipelined on three streams")

    def setup_e2e(self):
        import torch
        Z = self.Z
        self.hA = self.A.cpu().pin_memory()
        self.hB = torch.empty_like(self.B, device="cpu").pin_memory()
        self.e2e_h2d = self.hA.numel() * 4
        self.e2e_d2h = self.hB.numel() * 4
        # slices of the packed batch: contiguous index ranges are contiguous
        # ranges of both buffers (floats)
        up = lambda v: (v + 255) // 256 * 256  # noqa: E731
        a, b = self.A.data_ptr(), self.B.data_ptr()
        cuts = [self.count * k // self.e2e_slices for k in range(self.e2e_slices + 1)]
        self.slices = []
        for i0, i1 in zip(cuts[:-1], cuts[1:]):
            lo_in, hi_in = int(self.in_off[i0]) // 4, int(self.in_off[i1 - 1] + up(self.in_sz[i1 - 1])) // 4
            lo_out, hi_out = int(self.out_off[i0]) // 4, int(self.out_off[i1 - 1] + up(self.out_sz[i1 - 1])) // 4
            descs = [(Z.C2C if self.is_c[i] else Z.R2C, int(self.orders[i]), Z.FORWARD, a + int(self.in_off[i]),
                      b + int(self.out_off[i])) for i in range(i0, i1)]
            mb = Z.MixedBatch(descs, np.float32, device=self.A.device.index)
            mb.run(Z.SCHED_GRAPH, torch.cuda.current_stream().cuda_stream)  # capture the graph (set-up)
            self.slices.append((mb, lo_in, hi_in, lo_out, hi_out))
        torch.cuda.synchronize()
        self.pipe = SlicePipe(self.A.device)

    def e2e_step(self):
        Z = self.Z

        def item(mb, li, hi, lo, ho):
            return (lambda st: self.A[li:hi].copy_(self.hA[li:hi], non_blocking=True),
                    lambda st: mb.run(Z.SCHED_GRAPH, st.cuda_stream),
                    lambda st: self.hB[lo:ho].copy_(self.B[lo:ho], non_blocking=True))
        self.pipe.run([item(*sl) for sl in self.slices])

    def cpu_run(self, frames, threads, kind):
        """The first `frames` transforms, one reference object per (kind, order)."""
        from oracle import oracle as O
        rng = np.random.default_rng(1004)
        frames = min(frames, self.count)
        nbytes, dt = 0.0, 0.0
        groups = {}
        for i in range(frames):
            groups.setdefault((bool(self.is_c[i]), int(self.orders[i])), []).append(i)
        for (is_c, o), idx in sorted(groups.items()):
            n, cnt = 1 << o, len(idx)
            if is_c:
                x = (rng.uniform(-1, 1, (cnt, n)) + 1j * rng.uniform(-1, 1, (cnt, n))).astype(np.complex64)
            else:
                x = rng.uniform(-1, 1, (cnt, n)).astype(np.float32)
            if kind == "reference":
                plan = O.RefPlan("c2c" if is_c else "r2c", o, "f32", threads)
                t0 = time.perf_counter()
                if is_c:
                    plan.cfft(x, True, out=np.empty_like(x))
                else:
                    plan.rfft_forward(x, O.AOS, out=np.empty((cnt, n // 2 + 1), np.complex64))
                dt += time.perf_counter() - t0
                plan.close()
            else:
                t0 = time.perf_counter()
                O.cfft_port(x, True) if is_c else O.rfft_forward_port(x)
                dt += time.perf_counter() - t0
            nbytes += float(self.in_sz[idx].sum() + self.out_sz[idx].sum())
        return nbytes, dt


class Cfft64:
    """CFFT<double> order 16, batch 512, re, im ~ U[-1, 1) (seed 1005): one
    step = forward then backward of the batch on the FP64 path (FP64
    twiddles and butterflies). CFFT<float> at the same shape is timed beside
    it, and a sample's error against numpy's FP64 FFT is reported."""
    name = "cfft64"
    desc = "CFFT<double> order 16 (N=65536) x 512, forward + backward, full FP64 path"
    l2 = "each op reads 512 MiB and writes 512 MiB, > 4x L2 (no L2 flush needed)"
    order, batch = 16, 512
    dtype = "f64"
    form = "tuned"

    def __init__(self):
        n = 1 << self.order
        self.op_bytes = {"c2c_f64_fwd": 2 * 16 * n * self.batch, "c2c_f64_bwd": 2 * 16 * n * self.batch}
        self.bytes_per_step = sum(self.op_bytes.values())
        self.host_in = None

    def setup(self, device):
        import torch
        import zldsp_fft_b200 as Z
        self.Z = Z
        n = 1 << self.order
        Z.autotune(Z.C2C, self.order, self.order, np.float64, device=device)  # set-up: per-order plan choice
        self.tuning = Z.tuning(Z.C2C, self.order, np.float64, device=device)
        self.plan = Z.Plan(Z.C2C, self.order, np.float64, mode=Z.MODE_TUNED, device=device)
        g = torch.Generator(device=device)
        g.manual_seed(1005)
        self.A = (torch.rand((self.batch, n, 2), generator=g, device=device, dtype=torch.float64) * 2 - 1)
        self.B = torch.empty_like(self.A)
        self.C = torch.empty_like(self.A)
        torch.cuda.synchronize(device)

    def ops(self, step):
        Z, p, b = self.Z, self.plan, self.batch
        return [("c2c_f64_fwd", lambda st: p.exec_device(Z.FORWARD, Z.AOS, Z.AOS, self.A.data_ptr(), None,
                                                         self.B.data_ptr(), None, b, stream=st)),
                ("c2c_f64_bwd", lambda st: p.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, self.B.data_ptr(), None,
                                                         self.C.data_ptr(), None, b, stream=st))]

    def take_launches(self):
        return self.plan.take_launch_count()

    def compare(self, stream, reps):
        """CFFT<float> at the same shape, and the FP64 error of a sample."""
        import torch
        Z = self.Z
        n, b = 1 << self.order, self.batch
        Z.autotune(Z.C2C, self.order, self.order, np.float32, device=self.A.device.index)
        p32 = Z.Plan(Z.C2C, self.order, np.float32, mode=Z.MODE_TUNED, device=self.A.device.index)
        a32 = self.A.float()
        b32 = torch.empty_like(a32)
        c32 = torch.empty_like(a32)

        def f32_step():
            p32.exec_device(Z.FORWARD, Z.AOS, Z.AOS, a32.data_ptr(), None, b32.data_ptr(), None, b,
                            stream=stream.cuda_stream)
            p32.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, b32.data_ptr(), None, c32.data_ptr(), None, b,
                            stream=stream.cuda_stream)
        for _ in range(2):
            f32_step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            f32_step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms32 = e0.elapsed_time(e1) / reps
        f32_bytes = self.bytes_per_step // 2  # complex64 moves half the bytes
        x = self.A[:8].cpu().numpy().view(np.complex128)[..., 0]
        y64 = self.B[:8].cpu().numpy().view(np.complex128)[..., 0]
        y32 = b32[:8].cpu().numpy().astype(np.float64).view(np.complex128)[..., 0]
        ref = np.fft.fft(x, axis=-1)
        nrm = np.linalg.norm(ref, axis=-1)
        return {
            "autotuned_plan": self.tuning,
            "cfft_float_same_shape": {"gbs": round(f32_bytes / (ms32 / 1e3) / 1e9, 1), "ms_per_step": round(ms32, 4),
                                      "transforms_per_s": round(2 * b / (ms32 / 1e3))},
            "max_rel_l2_vs_numpy_fp64": {"f64": float((np.linalg.norm(y64 - ref, axis=-1) / nrm).max()),
                                         "f32": float((np.linalg.norm(y32 - ref, axis=-1) / nrm).max())},
            "tolerance": {"f64": 4 * 16 * 2.0 ** -53, "f32": 4 * 16 * 2.0 ** -24},
        }

    def cpu_sample_desc(self, frames):
        return f"forward+backward of {frames} of the 512 transforms"

    def setup_e2e(self):
        import torch
        self.hA = self.A.cpu().pin_memory()
        self.hB = torch.empty_like(self.hA).pin_memory()
        self.e2e_h2d = 2 * self.hA.numel() * 8
        self.e2e_d2h = 2 * self.hA.numel() * 8

    def e2e_step(self):
        Z, p, b = self.Z, self.plan, self.batch
        p.exec_host(Z.FORWARD, Z.AOS, Z.AOS, self.hA.data_ptr(), None, self.hB.data_ptr(), None, b)
        p.exec_host(Z.BACKWARD, Z.AOS, Z.AOS, self.hB.data_ptr(), None, self.hB.data_ptr(), None, b)

    def cpu_run(self, frames, threads, kind):
        from oracle import oracle as O
        rng = np.random.default_rng(1005)
        n = 1 << self.order
        cnt = max(1, min(frames, self.batch))
        x = rng.uniform(-1, 1, (cnt, n)) + 1j * rng.uniform(-1, 1, (cnt, n))
        if kind == "reference":
            plan = O.RefPlan("c2c", self.order, "f64", threads)
            y, z = np.empty_like(x), np.empty_like(x)
            t0 = time.perf_counter()
            plan.cfft(x, True, out=y)
            plan.cfft(y, False, out=z)
            dt = time.perf_counter() - t0
            plan.close()
        else:
            t0 = time.perf_counter()
            O.cfft_port(O.cfft_port(x, True), False)
            dt = time.perf_counter() - t0
        return 2 * 2 * 16 * n * cnt, dt


class Cfft10:
    """CFFT<float> order 10 (N = 1024), one transform, AoS, re, im ~ U[-1, 1)
    (seed 1001): one step = forward then backward of the single transform,
    the pair recorded into one CUDA graph (two kernels) and replayed, as a
    caller repeating that pair would. Latency-bound (16 KiB per direction):
    the line reports microseconds per step beside the GB/s; L2 is flushed (a
    256 MiB write) between steps, outside the timed ops."""
    name = "cfft10"
    desc = ("CFFT<float> order 10 (N=1024), single transform, forward then backward, AoS; the pair "
            "replayed from one CUDA graph")
    l2 = "L2 flushed between steps by a 256 MiB write, outside the timed ops"
    order, batch = 10, 1
    dtype = "f32"

    def __init__(self):
        n = 1 << self.order
        self.op_bytes = {"c2c_fwd_bwd": 32 * n}
        self.bytes_per_step = sum(self.op_bytes.values())
        self.host_in = None

    def setup(self, device):
        import torch
        import zldsp_fft_b200 as Z
        self.Z = Z
        n = 1 << self.order
        rng = np.random.default_rng(1001)
        x = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(np.complex64)
        self.host_x = x
        self.plan = Z.Plan(Z.C2C, self.order, np.float32, device=device)
        self.A = torch.from_numpy(x.view(np.float32).copy()).to(device)
        self.B = torch.empty_like(self.A)
        self.C = torch.empty_like(self.A)
        self.flush_buf = torch.empty(64 << 20, dtype=torch.float32, device=device)
        # The forward + backward pair recorded into one CUDA graph (two
        # kernels), so the timed op is the device's own latency, not the
        # host's enqueue time per call.
        p = self.plan
        fwd = lambda st: p.exec_device(Z.FORWARD, Z.AOS, Z.AOS, self.A.data_ptr(), None,  # noqa: E731
                                       self.B.data_ptr(), None, 1, stream=st)
        bwd = lambda st: p.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, self.B.data_ptr(), None,  # noqa: E731
                                       self.C.data_ptr(), None, 1, stream=st)
        s = torch.cuda.Stream(device)
        with torch.cuda.stream(s):
            fwd(s.cuda_stream)
            bwd(s.cuda_stream)
        torch.cuda.synchronize(device)
        self.graphs = {}
        self.graph_kernels = {}  # kernels recorded in each graph (the plan's launch counter)
        self.launches = 0
        p.take_launch_count()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            fwd(s.cuda_stream)
            bwd(s.cuda_stream)
        self.graphs["c2c_fwd_bwd"] = g
        self.graph_kernels["c2c_fwd_bwd"] = p.take_launch_count()
        torch.cuda.synchronize(device)

    def flush(self, st):
        self.flush_buf.fill_(1.0)

    def _replay(self, name):
        self.graphs[name].replay()
        self.launches += self.graph_kernels[name]

    def ops(self, step):
        return [(name, lambda st, n=name: self._replay(n)) for name in self.graphs]

    def take_launches(self):
        n = self.launches + self.plan.take_launch_count()
        self.launches = 0
        return n

    def compare(self, stream, reps):
        """Microseconds per transform and the error of forward (vs numpy FP64)
        and of the round trip (backward(forward(x)) / N vs x)."""
        x = self.host_x.astype(np.complex128)
        y = self.B.cpu().numpy().view(np.complex64)
        z = self.C.cpu().numpy().view(np.complex64)
        ref = np.fft.fft(x)
        n = 1 << self.order
        return {
            "fwd_rel_l2_vs_fp64": float(np.linalg.norm(y - ref) / np.linalg.norm(ref)),
            "roundtrip_rel_l2": float(np.linalg.norm(z / n - x) / np.linalg.norm(x)),
            "tolerance": 4 * self.order * 2.0 ** -24,
        }

    def cpu_sample_desc(self, frames):
        return f"{frames} repetitions of the single forward+backward transform in one call, one thread"

    e2e_steps = 2000  # forward + backward pairs timed through the drop-in class
    e2e_api = ("zldsp::fft::CFFT<float>(10).forward then .backward on host numpy buffers (the drop-in "
               "class, ZLFFT_MODE_HOST): one transform per call, synchronous, as the reference's callers make them")

    def cpp_dropin_latency(self):
        """The same pairs through the C++ drop-in class (tests/cpp/dropin_latency.cpp,
        compiled here against include/ and libzlfft_cuda.so): the reference's
        callers are C++, so this is their per-call cost without Python."""
        import shutil
        import subprocess
        import tempfile
        if shutil.which("g++") is None:
            return {"error": "g++ not available"}
        libdir = os.path.join(ROOT, "zldsp_fft_b200", "lib")
        with tempfile.TemporaryDirectory() as td:
            exe = os.path.join(td, "dropin_latency")
            r = subprocess.run(["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"),
                                os.path.join(ROOT, "tests", "cpp", "dropin_latency.cpp"), "-L", libdir,
                                "-lzlfft_cuda", "-o", exe], capture_output=True, text=True)
            if r.returncode != 0:
                return {"error": r.stderr[-200:]}
            env = dict(os.environ)
            env["LD_LIBRARY_PATH"] = libdir + ":" + env.get("LD_LIBRARY_PATH", "")
            r = subprocess.run([exe, str(self.order), "2000", "7"], capture_output=True, text=True, env=env,
                               timeout=300)
            if r.returncode != 0:
                return {"error": (r.stdout + r.stderr)[-200:]}
            return json.loads(r.stdout.strip().splitlines()[-1])

    def setup_e2e(self):
        n = 1 << self.order
        self.cf = self.Z.CFFT(self.order, np.float32)
        self.hx = self.host_x.copy()
        self.hy = np.empty_like(self.hx)
        self.hz = np.empty_like(self.hx)
        self.e2e_h2d = 2 * 8 * n
        self.e2e_d2h = 2 * 8 * n

    def e2e_step(self):
        self.cf.forward(self.hx, self.hy)
        self.cf.backward(self.hy, self.hz)

    def cpu_run(self, frames, threads, kind):
        from oracle import oracle as O
        n = 1 << self.order
        rng = np.random.default_rng(1001)
        x = (rng.uniform(-1, 1, (1, n)) + 1j * rng.uniform(-1, 1, (1, n))).astype(np.complex64)
        reps = max(1, frames)
        if kind == "reference":
            plan = O.RefPlan("c2c", self.order, "f32", 1)
            t0 = time.perf_counter()
            plan.cfft_roundtrip_repeat(x[0], reps)
            dt = time.perf_counter() - t0
            plan.close()
        else:
            t0 = time.perf_counter()
            for _ in range(reps):
                O.cfft_port(O.cfft_port(x, True), False)
            dt = time.perf_counter() - t0
        return 2 * 16 * n * reps, dt

    batch_for_cpu = 1 << 30  # repetitions the CPU sample may grow to
    cpu_threads = 1          # one transform: the reference runs it on one thread


class Stft:
    """STFT front end: a 2^27-sample real signal (U[-1, 1), seed 1006),
    4096-point frames at hop 1024 (131,069 frames), periodic Hann window, power
    spectrum (forward_sqr_mag) of every frame, in one zlfft_stft_device launch.
    Algorithmic bytes: the signal read once plus the spectrogram written.
    Beside it: the same spectrogram from frames cut and windowed by torch into a
    buffer first (unfold * window), then the batched RFFT."""
    name = "stft"
    desc = ("STFT: 2^27-sample float signal, 4096-point Hann frames at hop 1024 (131,069 frames), "
            "forward_sqr_mag, fused framing + window + RFFT")
    l2 = "each step reads 512 MiB and writes 1.07 GB, > 10x L2 (no L2 flush needed)"
    order, hop = 12, 1024
    dtype = "f32"

    def __init__(self, total_log2=27):
        self.total = 1 << total_log2
        n = 1 << self.order
        self.frame_n = n
        self.nf = (self.total - n) // self.hop + 1
        self.nb = n // 2 + 1
        self.op_bytes = {"stft_sqr_mag": 4 * self.total + 4 * self.nb * self.nf}
        self.bytes_per_step = self.op_bytes["stft_sqr_mag"]
        self.batch = self.nf
        self.host_in = None

    def setup(self, device):
        import torch
        import zldsp_fft_b200 as Z
        self.Z = Z
        g = torch.Generator(device=device)
        g.manual_seed(1006)
        self.sig = (torch.rand(self.total, generator=g, device=device) * 2 - 1).contiguous()
        t = torch.arange(self.frame_n, dtype=torch.float64, device=device)
        self.win = (0.5 - 0.5 * torch.cos(2 * np.pi * t / self.frame_n)).float().contiguous()
        self.out = torch.empty((self.nf, self.nb), dtype=torch.float32, device=device)
        self.plan = Z.Plan(Z.R2C, self.order, np.float32, device=device)
        torch.cuda.synchronize(device)

    def ops(self, step):
        Z = self.Z

        def run(st):
            self.plan.stft(Z.FORWARD_SQR_MAG, Z.AOS, self.sig.data_ptr(), self.hop, self.win.data_ptr(),
                           self.out.data_ptr(), None, self.nf, stream=st)
        return [("stft_sqr_mag", run)]

    def take_launches(self):
        return self.plan.take_launch_count()

    def compare(self, stream, reps):
        """The unfused path (frames materialised by torch, then the batched
        RFFT) and the fused result's equality with it."""
        import torch
        Z = self.Z
        ref_out = torch.empty_like(self.out)

        def unfused():
            with torch.cuda.stream(stream):
                fr = (self.sig.unfold(0, self.frame_n, self.hop) * self.win).contiguous()
                self.plan.exec_device(Z.FORWARD_SQR_MAG, Z.AOS, Z.AOS, fr.data_ptr(), None, ref_out.data_ptr(), None,
                                      self.nf, stream=stream.cuda_stream)
            return fr
        for _ in range(2):
            unfused()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            unfused()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        self.ops(0)[0][1](stream.cuda_stream)
        torch.cuda.synchronize()
        return {"unfused_frames_then_rfft": {"gbs": round(self.bytes_per_step / (ms / 1e3) / 1e9, 1), "ms": round(ms, 3)},
                "fused_equals_unfused_bitwise": bool(torch.equal(self.out, ref_out))}

    def cpu_sample_desc(self, frames):
        return f"{frames} of {self.nf} frames: numpy framing + window, then the reference's forward_sqr_mag"

    e2e_slices = 8
    e2e_api = ("zlfft_stft_device on 8 slices of the frames, pinned host buffers, each slice's new signal "
               "samples H2D / its frames / its spectrogram rows D2H pipelined on three streams")

    def setup_e2e(self):
        import torch
        self.h_sig = self.sig.cpu().pin_memory()
        self.h_out = torch.empty((self.nf, self.nb), dtype=torch.float32).pin_memory()
        self.e2e_h2d = self.h_sig.numel() * 4
        self.e2e_d2h = self.h_out.numel() * 4
        self.pipe = SlicePipe(self.sig.device)

    def e2e_step(self):
        Z = self.Z
        n, hop = self.frame_n, self.hop
        cuts = [self.nf * k // self.e2e_slices for k in range(self.e2e_slices + 1)]
        items, done = [], 0
        for f0, f1 in zip(cuts[:-1], cuts[1:]):
            end = (f1 - 1) * hop + n if f1 < self.nf else self.total  # samples the slice's frames need

            def h2d(st, a=done, b=end):
                self.sig[a:b].copy_(self.h_sig[a:b], non_blocking=True)

            def work(st, f0=f0, f1=f1):
                self.plan.stft(Z.FORWARD_SQR_MAG, Z.AOS, self.sig.data_ptr() + 4 * f0 * hop, hop,
                               self.win.data_ptr(), self.out[f0].data_ptr(), None, f1 - f0, stream=st.cuda_stream)

            def d2h(st, f0=f0, f1=f1):
                self.h_out[f0:f1].copy_(self.out[f0:f1], non_blocking=True)
            items.append((h2d, work, d2h))
            done = end
        self.pipe.run(items)

    def cpu_run(self, frames, threads, kind):
        from oracle import oracle as O
        n, hop = self.frame_n, self.hop
        frames = max(1, min(frames, self.nf))
        rng = np.random.default_rng(1006)
        sig = rng.uniform(-1, 1, (frames - 1) * hop + n).astype(np.float32)
        win = (0.5 - 0.5 * np.cos(2 * np.pi * np.arange(n) / n)).astype(np.float32)
        view = np.lib.stride_tricks.sliding_window_view(sig, n)[::hop]  # frames as views of the signal
        out = np.empty((frames, self.nb), np.float32)
        if kind == "reference":
            plan = O.RefPlan("r2c", self.order, "f32", threads)
            t0 = time.perf_counter()
            fr = view * win  # the windowed copy a caller of forward_sqr_mag makes
            plan.rfft_forward(fr, sqr_mag=True, out=out)
            dt = time.perf_counter() - t0
            plan.close()
        else:
            t0 = time.perf_counter()
            O.rfft_forward_port(view * win, sqr_mag=True)
            dt = time.perf_counter() - t0
        return float(4 * ((frames - 1) * hop + n) + 4 * self.nb * frames), dt


class Istft:
    """Inverse STFT / overlap-add: the bins of 131,069 frames of 4096 points
    (the stft workload's shape; complex U[-1, 1), seed 1007, real DC and
    Nyquist bins), times a spectral filter (a delayed low-pass), RFFT backward,
    periodic Hann synthesis window, and overlap-add at hop 1024 into a
    2^27-sample signal, in one zlfft_istft_device launch. Algorithmic bytes:
    the bins read once plus the signal written. Beside it: the same synthesis
    unfused (torch filter multiply, the batched RFFT backward into a frames
    buffer, torch window multiply and strided overlap-add)."""
    name = "istft"
    desc = ("inverse STFT: 131,069 frames of 4096-point bins (complex64 AoS), spectral filter, RFFT backward, "
            "Hann synthesis window, overlap-add at hop 1024 into a 2^27-sample signal, fused")
    l2 = "each step reads 2.15 GB and writes 512 MiB, > 20x L2 (no L2 flush needed)"
    order, hop = 12, 1024
    dtype = "f32"

    def __init__(self, total_log2=27):
        self.total = 1 << total_log2
        n = 1 << self.order
        self.frame_n = n
        self.nf = (self.total - n) // self.hop + 1
        self.nb = n // 2 + 1
        self.op_bytes = {"istft_filter_window": 8 * self.nb * self.nf + 4 * self.total}
        self.bytes_per_step = self.op_bytes["istft_filter_window"]
        self.batch = self.nf
        self.host_in = None

    @staticmethod
    def filter_bins(nb, n, xp, dtype):
        """H[k] = exp(-2 pi i 64 k / n) / (1 + (k / 256)^2): a 64-sample delay and a low-pass."""
        k = xp.arange(nb, dtype=dtype)
        mag = 1.0 / (1.0 + (k / 256.0) ** 2)
        ph = -2.0 * np.pi * 64.0 * k / n
        return mag * xp.cos(ph), mag * xp.sin(ph)

    def setup(self, device):
        import torch
        import zldsp_fft_b200 as Z
        self.Z = Z
        g = torch.Generator(device=device)
        g.manual_seed(1007)
        self.bins = (torch.rand((self.nf, self.nb, 2), generator=g, device=device) * 2 - 1).contiguous()
        self.bins[:, 0, 1] = 0
        self.bins[:, -1, 1] = 0
        t = torch.arange(self.frame_n, dtype=torch.float64, device=device)
        self.win = (0.5 - 0.5 * torch.cos(2 * np.pi * t / self.frame_n)).float().contiguous()
        hr, hi = self.filter_bins(self.nb, self.frame_n, torch, torch.float64)
        self.filt = torch.stack([hr, hi], -1).to(device).float().contiguous()
        self.sig = torch.empty(self.total, dtype=torch.float32, device=device)
        self.plan = Z.Plan(Z.R2C, self.order, np.float32, device=device)
        torch.cuda.synchronize(device)

    def ops(self, step):
        Z = self.Z

        def run(st):
            self.plan.istft(Z.AOS, self.bins.data_ptr(), None, self.hop, self.nf, self.sig.data_ptr(),
                            filter=self.filt.data_ptr(), window=self.win.data_ptr(), stream=st)
        return [("istft_filter_window", run)]

    def take_launches(self):
        return self.plan.take_launch_count()

    def compare(self, stream, reps):
        """The unfused path and its relative L2 distance from the fused result
        (the unfused overlap-add sums the frames in another order)."""
        import torch
        Z = self.Z
        n, hop, nf = self.frame_n, self.hop, self.nf
        k = n // hop
        frames = torch.empty((nf, n), dtype=torch.float32, device=self.bins.device)
        ref = torch.empty_like(self.sig)
        b = torch.view_as_complex(self.bins)
        h = torch.view_as_complex(self.filt)

        def unfused():
            with torch.cuda.stream(stream):
                fb = torch.view_as_real(b * h).contiguous()
                self.plan.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, fb.data_ptr(), None, frames.data_ptr(), None, nf,
                                      stream=stream.cuda_stream)
                fw = frames * self.win
                ref.zero_()
                for r in range(k):  # frames r, r + K, ... tile the signal from r * hop without overlap
                    cnt = (nf - r + k - 1) // k
                    ref[r * hop:r * hop + cnt * n] += fw[r::k].reshape(-1)
        for _ in range(2):
            unfused()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            unfused()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        self.ops(0)[0][1](stream.cuda_stream)
        torch.cuda.synchronize()
        d = (torch.linalg.vector_norm((self.sig - ref).double()) / torch.linalg.vector_norm(ref.double())).item()
        return {"unfused_filter_rfft_window_overlap_add": {"gbs": round(self.bytes_per_step / (ms / 1e3) / 1e9, 1),
                                                           "ms": round(ms, 3)},
                "fused_vs_unfused_rel_l2": d}

    def cpu_sample_desc(self, frames):
        return (f"{frames} of {self.nf} frames: numpy filter multiply, the reference's RFFT backward, numpy window "
                f"and sequential overlap-add")

    e2e_slices = 8
    e2e_api = ("zlfft_istft_device on 8 slices of the frames (each also given the K - 1 frames before it, "
               "its signal into its own buffer, its final blocks copied back), pinned host buffers, "
               "H2D / run / D2H pipelined on three streams")

    def setup_e2e(self):
        import torch
        self.h_bins = self.bins.cpu().pin_memory()
        self.h_sig = torch.empty(self.total, dtype=torch.float32).pin_memory()
        self.e2e_h2d = self.h_bins.numel() * 4
        self.e2e_d2h = self.h_sig.numel() * 4
        n, hop, k = self.frame_n, self.hop, self.frame_n // self.hop
        self.cuts = [self.nf * j // self.e2e_slices for j in range(self.e2e_slices + 1)]
        # slice [f0, f1) runs frames [g0, f1), g0 = f0 - (K - 1): its blocks [f0, f1) then
        # hold their final sums (the same terms, in the same order, as one launch)
        self.slice_sig = [torch.empty((f1 - max(0, f0 - k + 1) - 1) * hop + n, dtype=torch.float32,
                                      device=self.bins.device) for f0, f1 in zip(self.cuts[:-1], self.cuts[1:])]
        self.pipe = SlicePipe(self.bins.device)

    def e2e_step(self):
        Z = self.Z
        hop, k = self.hop, self.frame_n // self.hop
        items = []
        for j, (f0, f1) in enumerate(zip(self.cuts[:-1], self.cuts[1:])):
            g0 = max(0, f0 - k + 1)
            last = f1 == self.nf
            buf = self.slice_sig[j]

            def h2d(st, f0=f0, f1=f1):
                self.bins[f0:f1].copy_(self.h_bins[f0:f1], non_blocking=True)

            def work(st, g0=g0, f1=f1, buf=buf):
                self.plan.istft(Z.AOS, self.bins[g0].data_ptr(), None, hop, f1 - g0, buf.data_ptr(),
                                filter=self.filt.data_ptr(), window=self.win.data_ptr(), stream=st.cuda_stream)

            def d2h(st, f0=f0, f1=f1, g0=g0, buf=buf, last=last):
                a, b = f0 * hop, (self.total if last else f1 * hop)
                self.h_sig[a:b].copy_(buf[a - g0 * hop:b - g0 * hop], non_blocking=True)
            items.append((h2d, work, d2h))
        self.pipe.run(items)

    def cpu_run(self, frames, threads, kind):
        from oracle import oracle as O
        n, hop = self.frame_n, self.hop
        frames = max(1, min(frames, self.nf))
        rng = np.random.default_rng(1007)
        X = (rng.uniform(-1, 1, (frames, self.nb)) + 1j * rng.uniform(-1, 1, (frames, self.nb))).astype(np.complex64)
        X[:, 0], X[:, -1] = X[:, 0].real, X[:, -1].real
        hr, hi = self.filter_bins(self.nb, n, np, np.float64)
        H = (hr + 1j * hi).astype(np.complex64)
        win = (0.5 - 0.5 * np.cos(2 * np.pi * np.arange(n) / n)).astype(np.float32)
        if kind == "reference":
            plan = O.RefPlan("r2c", self.order, "f32", threads)
            t0 = time.perf_counter()
            Y = np.empty_like(X)
            Y.real = X.real * H.real - X.imag * H.imag
            Y.imag = X.real * H.imag + X.imag * H.real
            x = plan.rfft_backward(Y) * win
            y = np.zeros((frames - 1) * hop + n, np.float32)
            for f in range(frames):
                y[f * hop:f * hop + n] += x[f]
            dt = time.perf_counter() - t0
            plan.close()
        else:
            t0 = time.perf_counter()
            O.istft_port(X, hop, H, win)
            dt = time.perf_counter() - t0
        return float(8 * self.nb * frames + 4 * ((frames - 1) * hop + n)), dt


WORKLOADS = {"rfft12": Rfft12, "cfft2g": Cfft2G, "mixed": Mixed, "cfft64": Cfft64, "cfft10": Cfft10, "stft": Stft,
             "istft": Istft}


# ------------------------------------------------------------------ CPU baseline
CPU_SAMPLE_S = 1.0     # seconds of CPU work per sample (the baseline takes the median of 3)
CPU_FRAMES_CAP = 2048  # rfft12: frames generated for the CPU sample


def cpu_sample_frames(wl, threads, kind, target_s=CPU_SAMPLE_S):
    """The one sampling rule of both CPU figures (the cpu_baseline of the GPU
    arm and every step of the reference arm): from 16 transforms (or frames),
    doubled until one sample takes target_s or covers the workload."""
    avail = getattr(wl, "batch_for_cpu", wl.batch) if wl.host_in is None else wl.host_in.shape[0]
    frames = 16
    _, dt = wl.cpu_run(frames, threads, kind)
    while dt < target_s and frames < avail:
        frames = min(avail, frames * 2)
        _, dt = wl.cpu_run(frames, threads, kind)
    return frames


def cpu_threads_kind(wl):
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    threads = (getattr(wl, "cpu_threads", None) or os.cpu_count() or 1) if kind == "reference" else 1
    return threads, kind


def cpu_baseline(wl):
    threads, kind = cpu_threads_kind(wl)
    if hasattr(wl, "n") and wl.host_in is not None:
        wl.host_in = wl.host_in[:CPU_FRAMES_CAP]
    frames = cpu_sample_frames(wl, threads, kind)
    runs = [wl.cpu_run(frames, threads, kind) for _ in range(3)]
    gbs = statistics.median(b / t / 1e9 for b, t in runs)
    return {
        "value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": kind,
        "sample": wl.cpu_sample_desc(frames) + ", median of 3 samples", "host": host_info(),
    }


def config_of(wl, world):
    """The config object of both arms' lines (identical keys and values)."""
    return {"workload": wl.desc,
            "form": FORMS.get(getattr(wl, "form", "plain"), FORMS["plain"]),
            "l2": getattr(wl, "l2", "rotating input/output sets, each step > 2x L2 (no L2 flush needed)"),
            "parallelism": f"replicas x{world}"}


# ------------------------------------------------------------------ the other configurations
OTHER_CONFIGS = (("rfft12", "cfg 2"), ("mixed", "cfg 4"), ("cfft64", "cfg 5"), ("cfft10", "cfg 1"))


def quick_measure(wl, device, steps=5, warmup=3):
    """One configuration measured the way the main line is (rotating sets or
    L2 flush as the workload defines, CUDA events on the launching stream,
    clocks sampled), with fewer steps and without the host-API and CPU legs:
    the evidence for the benchmark configurations other than the default."""
    import torch
    wl.setup(device)
    stream = torch.cuda.current_stream()
    st = stream.cuda_stream
    for w in range(warmup):
        for _, fn in wl.ops(w):
            fn(st)
    torch.cuda.synchronize()
    wl.take_launches()
    names = [name for name, _ in wl.ops(0)]
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(names) + 1)] for _ in range(steps)]
    flush = getattr(wl, "flush", None)
    clocks = ClockSampler(device)
    clocks.start()
    for s in range(steps):
        if flush is not None:
            flush(st)
        ops = wl.ops(s)
        ev[s][0].record(stream)
        for i, (_, fn) in enumerate(ops):
            fn(st)
            ev[s][i + 1].record(stream)
    torch.cuda.synchronize()
    clocks.stop()
    launches = wl.take_launches()
    elapsed_ms = sum(ev[s][0].elapsed_time(ev[s][-1]) for s in range(steps))
    per_op_ms = {name: statistics.mean(ev[s][i].elapsed_time(ev[s][i + 1]) for s in range(steps))
                 for i, name in enumerate(names)}
    peak, peak_kind = measured_hbm_peak()
    dom = max(per_op_ms, key=per_op_ms.get)
    achieved = wl.op_bytes[dom] / (per_op_ms[dom] / 1e3) / 1e9
    res = {"workload": wl.desc, "dtype": wl.dtype, "steps": steps, "warmup": warmup,
           "value": round(wl.bytes_per_step * steps / (elapsed_ms / 1e3) / 1e9, 2), "unit": "GB/s",
           "ms_per_step": round(elapsed_ms / steps, 4),
           "roofline": {"kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                        "frac": round(achieved / peak, 4), "peak_source": peak_kind},
           "per_op_gbs": {k: round(wl.op_bytes[k] / (v / 1e3) / 1e9, 1) for k, v in per_op_ms.items()},
           "per_op_us": {k: round(v * 1e3, 2) for k, v in per_op_ms.items()},
           "gpu_launches": launches, "clocks": clocks.summary()}
    if hasattr(wl, "compare"):
        res["schedules"] = wl.compare(stream, 3)
    return res


def measure_other_configs(device):
    out = {}
    for name, label in OTHER_CONFIGS:
        try:
            r = quick_measure(WORKLOADS[name](), device)
            r["config"] = label
            out[name] = r
        except Exception as e:  # reported, never required: the main line stands on its own
            out[name] = {"config": label, "error": str(e)[:200]}
    return out


# ------------------------------------------------------------------ arms
def run_reference_arm(args, wl_cls):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = wl_cls()
    threads, kind = cpu_threads_kind(wl)
    wl.host_in = hann_frames(min(wl.batch, CPU_FRAMES_CAP), wl.n, 1002) if hasattr(wl, "n") else None
    # each step: a bounded sample of the workload on all host cores, sized by
    # the same rule as the GPU arm's cpu_baseline
    frames = cpu_sample_frames(wl, threads, kind)
    for _ in range(args.warmup):
        wl.cpu_run(frames, threads, kind)
    tot_b, tot_t = 0.0, 0.0
    for _ in range(args.steps):
        b, t = wl.cpu_run(frames, threads, kind)
        tot_b += b
        tot_t += t
    v = tot_b / tot_t / 1e9
    line = {
        "metric": METRIC, "value": round(v, 3), "unit": "GB/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * tot_t / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl.dtype, "data": "synthetic",
        "config": config_of(wl, args.gpus),
        "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "cores": threads, "kind": kind,
                         "sample": wl.cpu_sample_desc(frames) + " per step", "host": host_info()},
        "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, wl_cls):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    device = torch.cuda.current_device()
    wl = wl_cls()
    wl.setup(device)
    stream = torch.cuda.current_stream()
    st = stream.cuda_stream

    def barrier():
        if dist is not None:
            dist.barrier()

    for w in range(args.warmup):
        for _, fn in wl.ops(w):
            fn(st)
    torch.cuda.synchronize()
    wl.take_launches()

    names = [name for name, _ in wl.ops(0)]
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(names) + 1)] for _ in range(args.steps)]
    clocks = ClockSampler(device)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    flush = getattr(wl, "flush", None)
    for s in range(args.steps):
        if flush is not None:
            flush(st)  # outside the op events
        ops = wl.ops(s)
        ev[s][0].record(stream)
        for i, (_, fn) in enumerate(ops):
            fn(st)
            ev[s][i + 1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    clocks.stop()
    barrier()
    launches = wl.take_launches()
    elapsed_ms = t_start.elapsed_time(t_end)
    if flush is not None:  # the steps' own time, without the flushes between them
        elapsed_ms = sum(ev[s][0].elapsed_time(ev[s][-1]) for s in range(args.steps))
    per_op_ms = {name: statistics.mean(ev[s][i].elapsed_time(ev[s][i + 1]) for s in range(args.steps))
                 for i, name in enumerate(names)}
    from zldsp_fft_b200 import replicas
    elapsed_ms = replicas.max_over_ranks(elapsed_ms, dist, device="cuda")
    value = replicas.aggregate_gbs(wl.bytes_per_step * args.steps, world, elapsed_ms / 1e3)

    # end to end through the host API, pinned host buffers, copies inside the region
    wl.setup_e2e()
    e2e_steps = getattr(wl, "e2e_steps", max(3, min(args.steps, 10)))
    wl.e2e_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        wl.e2e_step()
    e2e_s = time.perf_counter() - t0
    e2e_s = replicas.max_over_ranks(e2e_s, dist, device="cuda")
    e2e_val = replicas.aggregate_gbs(wl.bytes_per_step * e2e_steps, world, e2e_s)
    wl.take_launches()
    pcie = pcie_probe()
    bound = e2e_bound(wl.bytes_per_step, wl.e2e_h2d, wl.e2e_d2h, pcie)
    schedules = wl.compare(stream, max(3, min(args.steps, 10))) if hasattr(wl, "compare") else None
    cpp_latency = wl.cpp_dropin_latency() if (rank == 0 and hasattr(wl, "cpp_dropin_latency")) else None

    peak, peak_kind = measured_hbm_peak()
    dom = max(per_op_ms, key=per_op_ms.get)  # the op with the largest share of the step's time
    achieved = wl.op_bytes[dom] / (per_op_ms[dom] / 1e3) / 1e9
    traffic = ncu_traffic(dom)
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(elapsed_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": wl.dtype, "data": "synthetic",
        "config": config_of(wl, world),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "kernel": dom, "time_share": round(per_op_ms[dom] / sum(per_op_ms.values()), 3),
                     "algorithmic_bytes_per_launch": wl.op_bytes[dom],
                     "traffic": traffic},
        "per_op_gbs": {k: round(wl.op_bytes[k] / (v / 1e3) / 1e9, 1) for k, v in per_op_ms.items()},
        "per_op_us": {k: round(v * 1e3, 2) for k, v in per_op_ms.items()},
        "e2e": {"value": round(e2e_val, 2), "unit": "GB/s", "h2d_bytes_per_step": wl.e2e_h2d,
                "d2h_bytes_per_step": wl.e2e_d2h, "us_per_step": round(e2e_s / e2e_steps * 1e6, 2),
                "api": getattr(wl, "e2e_api", "zlfft_exec_host_batched, pinned host buffers"),
                "pcie_gbs": pcie, "pcie_bound": round(bound, 2) if bound else None,
                "frac_of_pcie_bound": round(e2e_val / bound, 3) if bound else None},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    if schedules is not None:
        line["schedules"] = schedules
    if cpp_latency is not None:
        line["e2e"]["cpp_dropin"] = cpp_latency
    if rank == 0 and world == 1 and args.workload == "cfft2g" and not args.no_configs:
        line["other_configs"] = measure_other_configs(device)
    if rank == 0:
        if world == 1 and not args.no_cpu:
            try:
                line["cpu_baseline"] = cpu_baseline(wl)
            except Exception as e:  # the baseline is reported, never required
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="cfft2g")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-configs", action="store_true",
                    help="default workload only: skip the short measurement of the other benchmark configurations "
                         "(other_configs in the line)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="mixed only: skip the per-order autotuning in set-up (for profiling runs)")
    ap.add_argument("--form", choices=["tuned", "plain", "fast", "tc", "macro"], default="tuned",
                    help="cfft2g only: the autotuned form per order (default), the plain form (the reference's "
                         "arithmetic), the fast-twiddle form, the tensor-core split FP16 hi/lo form, or the "
                         "reference's macro DIF path as a small-cache host runs it")
    ap.add_argument("--total-log2", type=int, default=None,
                    help="cfft2g: complex elements per order = 2^k (default 28 = 2 GiB); stft / istft: signal "
                         "samples = 2^k (default 27); smaller cases are for profiling and are not the benchmark "
                         "configuration")
    args = ap.parse_args()
    wl_cls = WORKLOADS[args.workload]
    if args.workload == "cfft2g" and (args.total_log2 is not None or args.form != "tuned"):
        base = wl_cls
        tl = args.total_log2 if args.total_log2 is not None else 28
        wl_cls = lambda: base(total_log2=tl, form=args.form)  # noqa: E731
        wl_cls.__name__ = base.__name__
    if args.workload in ("stft", "istft") and args.total_log2 is not None:
        base_s = wl_cls
        wl_cls = lambda: base_s(total_log2=args.total_log2)  # noqa: E731
        wl_cls.__name__ = base_s.__name__
    if args.workload == "mixed" and args.no_autotune:
        base_m = wl_cls
        wl_cls = lambda: base_m(autotune=False)  # noqa: E731
        wl_cls.__name__ = base_m.__name__
    if args.impl == "reference":
        return run_reference_arm(args, wl_cls)
    return run_ours(args, wl_cls)


if __name__ == "__main__":
    sys.exit(main())
