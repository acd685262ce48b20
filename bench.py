#!/usr/bin/env python
"""Throughput of the EPIC 3-D parcel step on B200s (parcel-steps/s).

One step = one iteration of the reference run loop (epic3d.f90:135-153):
vorticity correction, 5-stage low-storage RK4 (par2grid, vor2vel,
vorticity tendency, grid2par per stage), merge, split and two correction
passes.  parcel-steps = sum over timed steps of the parcels at step start.

Default workload: the rising thermal, 128^3 grid, 8 parcels per cell
(16,777,216 parcels), plain FP64.  With N GPUs (torchrun) every rank runs
an independent replica of the workload (replicas only: a single EPIC run
has no data-parallel shard without halos), and the reported value is the
whole-job parcel-steps/s over the max-over-ranks device time.

--impl reference times the CPU restatement of the reference step
(oracle/, OpenMP build, all host threads) on the same workload; the
reference Fortran cannot be built on this image (no Fortran compiler, MPI
or NetCDF).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "parcel-steps/s at 1 B200 (FP64 plain vs mixed vs served), p50/p99 at fixed error"
UNIT = "parcel-steps/s"


def peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region (nvidia-smi sampling)
class ClockSampler:
    """SM clock and clock-event reasons during the timed region: NVML polled
    every 10 ms on the device torch uses (found by its PCI bus id), else
    nvidia-smi every 200 ms.  Reads only; changes no setting."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.nvml = None
        self.samples = []
        self.max_mhz = None
        self.stop_flag = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            h = None
            try:
                import torch
                props = torch.cuda.get_device_properties(gpu_index)
                bus = "%08X:%02X:%02X.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(gpu_index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                         "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                         "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                         "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
            self.nvml, self.handle = pynvml, h
        except Exception:
            self.nvml = None

    def _poll(self):
        nv, h = self.nvml, self.handle
        while not self.stop_flag.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                self.samples.append((mhz, r))
            except Exception:
                pass
            self.stop_flag.wait(0.01)

    def start(self):
        if self.nvml is not None:
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_flag.set()
            self.thread.join(timeout=2)
            sm = [m for m, _ in self.samples]
            reasons = {nm for nm, bit in self.bits.items() for _, r in self.samples if r & bit}
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml, 10 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


# ---------------------------------------------------------------------------
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_timing(ms: float, work: float, device: str = "cuda"):
    """Max of the device times and sum of the work over ranks (replicas)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms, work], dtype=torch.float64, device=device)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(t[0]), float(t[1])
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = t.clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(sm[1])


def stage_launch_bytes(n: int, nx: int, ny: int, nz: int, form: str = "plain", later_only: bool = False) -> float:
    """Minimal DRAM bytes of one stage-kernel launch (grid2par + LS-RK update),
    averaged over the 5 stages of a step (later_only: of one of stages 2-5):
    per parcel the attributes read (position, Veta, Vtau, B, volume,
    vorticity; stages 2-5 also delta_pos, delta_vor, delta_b; stage 1 the
    buoyancy for the diagnostics) and written (position, vorticity, B,
    delta_pos, delta_vor, delta_b), plus one read of the gather records (16
    values per grid point)."""
    gh = nx * ny * (nz + 3)
    if form == "mixed":
        # FP64: position, volume, delta_pos; FP32: the rest
        first, later, rec = 96 + 112, 144 + 112, 64.0
    else:
        first, later, rec = (19 + 22) * 8, (29 + 22) * 8, 128.0
    if later_only:
        return later * n + rec * gh
    return (first + 4 * later) / 5.0 * n + rec * gh


# Minimal compulsory HBM traffic of one whole step per parcel (8 parcels per
# cell): the parcel attributes each call of the reference step must read and
# write (288 FP64 values = 2304 B plain; 1536 B with the mixed form's FP32
# attributes) plus the grid transforms (about 0.4 KB plain, 0.2 KB mixed per
# parcel).
STEP_BYTES_PER_PARCEL = {"plain": 2700.0, "mixed": 1740.0}


def step_roofline(value: float, form: str, peak_gbs: float, peak_kind: str) -> dict:
    """The whole step against HBM: parcel-steps/s x compulsory bytes per
    parcel-step, as a fraction of the measured copy bandwidth."""
    b = STEP_BYTES_PER_PARCEL[form]
    achieved = value * b / 1e9
    return {"bound": "hbm", "unit": "GB/s", "bytes_per_parcel_step": b, "achieved": achieved,
            "peak": peak_gbs, "peak_source": peak_kind, "frac": achieved / peak_gbs if peak_gbs else None,
            "meaning": "whole step: parcel-steps/s x the step's compulsory HBM bytes per parcel-step"}


def algorithmic_bytes(kernel: str, n: int, nx: int, ny: int, nz: int, form: str = "plain") -> float:
    """Minimal compulsory DRAM bytes of one launch."""
    gh = nx * ny * (nz + 3)
    if kernel == "stage" and form == "mixed":
        # state read: x3 V (FP64) + w3 B5 b q (FP32) = 72 B; accumulators
        # dx3 (FP64) + dw3 dB5 (FP32) = 56 B read and written; state written:
        # x3 (FP64) + w3 B5 (FP32) = 56 B.  Fields as in the plain form.
        return (72 + 56 + 56 + 56) * n + 14 * 8.0 * gh + 7 * 8.0 * gh + 2 * 4.0 * gh
    if kernel == "p2g":
        # read x3 w3 B5 V b q per parcel; write 7 scattered fields + 2 int counts
        return 14 * 8.0 * n + 7 * 8.0 * gh + 2 * 4.0 * gh
    if kernel == "g2p":
        # read x3 w3 B5 V + dx3 dw3 dB5; write x3 w3 B5 + dx3 dw3 dB5; read 14 fields
        return (23 + 22) * 8.0 * n + 14 * 8.0 * gh
    if kernel == "stage":
        # fused grid2par + RK update + next par2grid: read state (14) and
        # accumulators (11), write state (11) and accumulators (11) per parcel;
        # read 14 gathered fields, write 7 scattered fields + 2 int counts
        return 47 * 8.0 * n + 14 * 8.0 * gh + 7 * 8.0 * gh + 2 * 4.0 * gh
    if kernel == "fft":
        # one pass over a (nz+1) x ny x nx field: read + write
        return 2 * 8.0 * nx * ny * (nz + 1)
    raise KeyError(kernel)


class Timer:
    """The library's own CUDA-event timers around a window of steps: the
    window on the context's stream, one named kernel (every launch of it),
    the launch count and the SM clocks sampled meanwhile."""

    def __init__(self, lib, ctx, stream, dev):
        import ctypes as C
        self.C, self.lib, self.ctx, self.stream, self.dev = C, lib, ctx, stream, dev
        L = lib.lib
        L.epic_gpu_profile_kernel.argtypes = [C.c_void_p, C.c_char_p]
        L.epic_gpu_kernel_time.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.epic_gpu_launch_count.argtypes = [C.POINTER(C.c_int64)]

    def window(self, t, steps, kernel="stage", barrier=lambda: None):
        import torch
        C, L, ctx = self.C, self.lib.lib, self.ctx
        L.epic_gpu_profile_kernel(ctx.h, kernel.encode())
        clocks = ClockSampler(self.dev)
        barrier()
        torch.cuda.synchronize()
        ctx.sync()
        clocks.start()
        l0 = C.c_int64()
        L.epic_gpu_launch_count(C.byref(l0))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        psteps, infos = 0, []
        nmin = nmax = ctx.num_parcels()
        for _ in range(steps):
            psteps += ctx.num_parcels()
            t, info = ctx.step(t)
            infos.append(info)
            nmin, nmax = min(nmin, info.n_parcels), max(nmax, info.n_parcels)
        e1.record(self.stream)
        ctx.sync()
        torch.cuda.synchronize()
        barrier()
        clk = clocks.stop()
        l1 = C.c_int64()
        L.epic_gpu_launch_count(C.byref(l1))
        kms, kl = C.c_double(), C.c_int64()
        L.epic_gpu_kernel_time(ctx.h, C.byref(kms), C.byref(kl))
        L.epic_gpu_profile_kernel(ctx.h, b"")
        return t, {"ms": e0.elapsed_time(e1), "psteps": psteps, "nmin": int(nmin), "nmax": int(nmax),
                   "kernel_ms": kms.value, "kernel_launches": kl.value, "clocks": clk,
                   "launches": int(l1.value - l0.value), "infos": infos}


def stage_roofline(w: dict, steps: int, setup, form: str) -> dict:
    """The dominant kernel against HBM: one k_stage launch (grid2par + LS-RK
    update of every parcel), its algorithmic bytes over its average
    CUDA-event duration in the timed window."""
    peak, peak_kind = peaks()
    avg_n = w["psteps"] / steps
    unit_ms = w["kernel_ms"] / max(w["kernel_launches"], 1)
    alg = stage_launch_bytes(int(avg_n), setup.nx, setup.ny, setup.nz, form)
    achieved = alg / (unit_ms * 1e-3) / 1e9 if w["kernel_launches"] else None
    r = {"bound": "hbm", "kernel": "stage",
         "unit_of_work": "one k_stage launch (grid2par + LS-RK update of every parcel), averaged over the 5 stages",
         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": (achieved / peak if achieved else None),
         "traffic": None, "peak_source": peak_kind, "ms_per_unit": unit_ms, "launches": w["kernel_launches"],
         "share_of_step_time": w["kernel_ms"] / w["ms"] if w["ms"] else None, "algorithmic_bytes_per_unit": alg}
    # DRAM bytes of one k_stage launch of stages 2-5 from ncu captures of
    # the stage kernel (64^3, 2,097,152 parcels, early flow: plain 536.6 MB
    # read + 319.2 MB written = 408.1 B per parcel; mixed 337.3 + 184.7 MB =
    # 248.9 B), scaled by the parcels of this run (the traffic grows with
    # them), against the algorithmic bytes of the same stages.  Lines still
    # dirty in L2 when the launch ends (up to its 126 MB) are not counted,
    # which puts the captures a little below their algorithmic bytes.
    per_parcel = 248.9 if form == "mixed" else 408.1
    r["traffic"] = per_parcel * avg_n
    r["traffic_source"] = (f"ncu dram__bytes_read+write of k_stage<0,{'float' if form == 'mixed' else 'double'},0> "
                           "(stages 2-5), 64^3 capture scaled by parcels")
    r["traffic_over_algorithmic"] = r["traffic"] / stage_launch_bytes(int(avg_n), setup.nx, setup.ny, setup.nz, form,
                                                                      later_only=True)
    return r


def form_line(w: dict, steps: int, setup, form: str, extra: dict | None = None) -> dict:
    """The summary of one timed window of a form (parcel-steps/s on the
    device, with its roofline, clocks and launches)."""
    value = w["psteps"] / (w["ms"] * 1e-3)
    peak, peak_kind = peaks()
    out = {"value": value, "unit": UNIT, "ms_per_step": w["ms"] / steps, "steps": steps,
           "parcels_range_timed": [w["nmin"], w["nmax"]], "grid": [setup.nx, setup.ny, setup.nz],
           "roofline": stage_roofline(w, steps, setup, form), "step_roofline": step_roofline(value, form, peak, peak_kind),
           "clocks": w["clocks"], "gpu_launches": w["launches"]}
    if extra:
        out.update(extra)
    return out


def context_stream(lib, ctx, dev):
    import ctypes as C
    import torch
    sp = C.c_void_p()
    lib.lib.epic_gpu_get_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    lib.lib.epic_gpu_get_stream(ctx.h, C.byref(sp))
    return torch.cuda.ExternalStream(sp.value, device=dev)


def run_ours(args):
    import torch
    import epic_b200
    from epic_b200 import initial

    world, rank, local = dist_setup()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    lib = epic_b200.load()
    # keep_order = 0: the device keeps the parcels ordered by boxes of cells
    # and carries each one's index in the reference's container, so merges and
    # splits take the reference's decisions
    mixed = args.form == "mixed"
    large = args.workload == "thermal2-512x512x256"
    if args.device_init or large or args.parcels_per_cell:
        # parcels generated on the device (the same state as the host generator)
        setup = initial.device_spec(args.workload)
        if args.parcels_per_cell:
            # the grid's kernels at full size on a smaller device footprint
            setup.n_per_cell = args.parcels_per_cell
        extra = dict(capacity=int(1.15 * setup.n)) if large else {}
        ctx = epic_b200.make_context_device(setup, lib, keep_order=args.keep_order, precision=1 if mixed else 0,
                                            **extra)
        if large:
            args.no_e2e = True
    else:
        setup = initial.config(args.workload)
        ctx = epic_b200.make_context(setup, lib, keep_order=args.keep_order, precision=1 if mixed else 0)
    tuning = ctx.autotune() if not args.no_autotune else None
    if args.scatter_groups is not None:
        # lanes per group of consecutive parcels in the scatters, 2^lg
        import ctypes as C
        f = lib.lib.epic_gpu_test_set_scatter_groups
        f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        lg = args.scatter_groups
        assert f(ctx.h, lg, lg, lg) == 0
    if args.fft_path is not None:
        # horizontal FFT implementation (overrides the tuner)
        import ctypes as C
        f = lib.lib.epic_gpu_test_set_fft_path
        f.argtypes = [C.c_void_p, C.c_int]
        assert f(ctx.h, args.fft_path) == 0
    stream = context_stream(lib, ctx, dev)
    timer = Timer(lib, ctx, stream, dev if world == 1 else local)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    t = 0.0
    done = 0
    # optional untimed spin-up to a developed flow (deformed parcels, splits)
    for _ in range(args.spinup + args.warmup):
        t, _info = ctx.step(t)
        done += 1
    t, w = timer.window(t, args.steps, args.roofline_kernel, barrier)
    done += args.steps
    ms, psteps = w["ms"], w["psteps"]
    infos = w["infos"]

    # per-kernel CUDA-event times over one extra (untimed) step each
    kernel_times = {}
    import ctypes as C
    for kname in [k for k in args.profile_kernels.split(",") if k]:
        lib.lib.epic_gpu_profile_kernel(ctx.h, kname.encode())
        t, _ = ctx.step(t)
        done += 1
        km, kn = C.c_double(), C.c_int64()
        lib.lib.epic_gpu_kernel_time(ctx.h, C.byref(km), C.byref(kn))
        kernel_times[kname] = {"ms_per_step": km.value, "launches_per_step": kn.value}
    lib.lib.epic_gpu_profile_kernel(ctx.h, b"")

    free_b, total_b = torch.cuda.mem_get_info()
    used_gb = (total_b - free_b) / 1e9
    # max over ranks, sum of work
    ms_max, ps_total = reduce_timing(ms, float(psteps))
    value = ps_total / (ms_max * 1e-3)
    peak, peak_kind = peaks()
    if args.roofline_kernel == "stage":
        roofline = stage_roofline(w, args.steps, setup, args.form)
    else:
        avg_n = psteps / args.steps
        unit_ms = w["kernel_ms"] / max(w["kernel_launches"], 1)
        alg = algorithmic_bytes(args.roofline_kernel, int(avg_n), setup.nx, setup.ny, setup.nz, args.form)
        achieved = alg / (unit_ms * 1e-3) / 1e9 if w["kernel_launches"] else None
        roofline = {"bound": "hbm", "kernel": args.roofline_kernel, "unit_of_work": f"one {args.roofline_kernel} launch",
                    "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": (achieved / peak if achieved else None),
                    "traffic": args.traffic, "peak_source": peak_kind, "ms_per_unit": unit_ms,
                    "launches": w["kernel_launches"], "algorithmic_bytes_per_unit": alg}

    # ---- end-to-end through the C ABI with host buffers (drop-in serial step:
    # the host container owns the parcels; every step copies them in, steps,
    # and copies them back, like a caller keeping the reference's container)
    e2e = None
    if not args.no_e2e:
        cap = int(ctx.num_parcels() * 1.5) + 1024
        host = {k: torch.empty((cap, c), dtype=torch.float64, pin_memory=True).numpy()
                for k, c in (("pos", 3), ("vor", 3), ("B", 5), ("vol", 1), ("buoy", 1), ("hum", 1))}
        n_now = ctx.num_parcels()
        st = ctx.get_parcels()
        for k in host:
            host[k][:n_now] = st[k].reshape(n_now, -1)
        P = C.POINTER(C.c_double)
        fn_set = lib.fn["set_parcels"]
        fn_get = lib.fn["get_parcels"]
        names = ("pos", "vor", "B", "vol", "buoy", "hum")

        def e2e_step(t, n_now):
            rc = fn_set(ctx.h, C.c_int64(n_now), *(host[k].ctypes.data_as(P) for k in names))
            assert rc == 0, ctx.lib.fn["last_error"](ctx.h)
            t, info = ctx.step(t)
            nn = C.c_int64()
            rc = fn_get(ctx.h, C.c_int64(cap), C.byref(nn), *(host[k].ctypes.data_as(P) for k in names))
            assert rc == 0
            return t, nn.value

        # one untimed step warms the pinned copies and the reloaded store
        t, n_now = e2e_step(t, n_now)
        done += 1
        barrier()
        torch.cuda.synchronize()
        h2d = d2h = 0
        eps = 0
        w0 = time.perf_counter()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.e2e_steps):
            h2d += n_now * 14 * 8
            eps += n_now
            t, n_now = e2e_step(t, n_now)
            d2h += n_now * 14 * 8
            done += 1
        f1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
        ems = f0.elapsed_time(f1)
        ems_max, eps_total = reduce_timing(ems, float(eps))
        e2e = {"value": eps_total / (ems_max * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": h2d // args.e2e_steps, "d2h_bytes_per_step": d2h // args.e2e_steps,
               "steps": args.e2e_steps, "warmup_steps": 1, "wall_s": wall,
               "mode": "host-owned parcel container: set_parcels (pinned H2D) + step + get_parcels (D2H) every step"}

    store_gb = int(setup.n) * (184 if mixed else 312) / 1e9
    field_gb = 21 * 8 * setup.nx * setup.ny * (setup.nz + 3) / 1e9
    precision = ("mixed: FP32 vorticity, B, buoyancy, humidity, delta_vor, delta_b, support vectors, "
                 "par2grid sums and grid2par interpolation; FP64 positions, volume, delta_pos, B33 and fields"
                 if mixed else "fp64-plain")
    kind = "rising thermal" if args.workload.startswith("thermal") else "Beltrami flow"
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64" if mixed else "f64", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {kind}, {setup.nx}x{setup.ny}x{setup.nz} grid, "
                               f"{int(setup.n):,} parcels at t=0, seeded, {args.form} form, "
                               "merge/split/corrections on",
                   "form": args.form,
                   "grid": [setup.nx, setup.ny, setup.nz], "parcels_at_start": int(setup.n),
                   "parcels_range_timed": [w["nmin"], w["nmax"]], "precision": precision,
                   "timed_steps": f"steps {args.spinup + args.warmup + 1}-{args.spinup + args.warmup + args.steps} from t = 0",
                   "store_order": ("box-ordered store with container indices (keep_order 0)" if args.keep_order == 0
                                   else "reference container order (keep_order 1)"),
                   "spinup_steps": args.spinup, "autotune": tuning,
                   "fft_path_override": args.fft_path,
                   "device_memory_used_gb": round(used_gb, 2), "device_memory_total_gb": round(total_b / 1e9, 2),
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": f"inputs larger than L2 (parcel state {store_gb:.2f} GB, fields {field_gb:.2f} GB)"},
        "roofline": roofline,
        "step_roofline": step_roofline(value, args.form, peak, peak_kind),
        "clocks": w["clocks"],
        "e2e": e2e,
        "gpu_launches": w["launches"],
        "kernel_times": kernel_times,
        "dt_last": infos[-1].dt if infos else None,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    all_forms = (world == 1 and not args.no_forms and args.form == "plain" and args.workload == "thermal-128"
                 and args.spinup == 0)
    if all_forms:
        # the same run later in its life: deformed parcels, splits and merges
        forms = {}
        while done < args.developed_at:
            t, _ = ctx.step(t)
            done += 1
        t, wd = timer.window(t, args.steps, "stage")
        forms["plain_developed"] = form_line(wd, args.steps, setup, "plain", {
            "workload": f"the same thermal-128 run, steps {done + 1}-{done + args.steps}",
            "timed_steps": [done + 1, done + args.steps]})
        ctx.close()
        forms["mixed"] = mixed_form(args, lib, dev)
        forms["served"] = served_form(args, lib, dev)
        line["forms"] = forms
    else:
        ctx.close()
    if mixed and rank == 0 and not args.no_error:
        line["error"] = mixed_error(lib)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def mixed_form(args, lib, dev) -> dict:
    """The mixed-precision form on its own workload: the thermal on
    256x256x128 (67,108,864 parcels, 6.28 x 6.28 x 3.14), parcels generated on
    the device, warm-up then the timed window; with its errors against FP64."""
    import epic_b200
    from epic_b200 import initial
    spec = initial.device_spec("thermal-256x256x128")
    ctx = epic_b200.make_context_device(spec, lib, keep_order=0, precision=1)
    tuning = ctx.autotune() if not args.no_autotune else None
    timer = Timer(lib, ctx, context_stream(lib, ctx, dev), dev)
    t = 0.0
    for _ in range(args.warmup):
        t, _ = ctx.step(t)
    t, w = timer.window(t, args.steps, "stage")
    ctx.close()
    out = form_line(w, args.steps, spec, "mixed", {
        "workload": f"thermal-256x256x128: rising thermal, 256x256x128 grid, {spec.n:,} parcels at t=0, "
                    f"mixed form, steps {args.warmup + 1}-{args.warmup + args.steps}",
        "precision": "FP32 vorticity, B, buoyancy, humidity, delta_vor, delta_b, support vectors, par2grid sums "
                     "and grid2par interpolation, FFTs and z transforms; FP64 positions, volume, delta_pos, "
                     "B33, tridiagonal solve and fields",
        "autotune": tuning})
    if not args.no_error:
        out["error"] = mixed_error_at_size(lib, args)
    return out


def run_pair(lib, spec, steps, *overrides, fields=True):
    """Runs from the same device-generated state, one after the other:
    kinetic energy, enstrophy, parcel counts and (optionally) the gridded
    velocity, vorticity and buoyancy after `steps` steps."""
    from epic_b200 import make_context_device, abi
    out = []
    for ov in overrides:
        c = make_context_device(spec, lib, **ov)
        t = 0.0
        for _ in range(steps):
            t, info = c.step(t)
        f = None
        if fields:
            c.par2grid(False)
            c.vor2vel()
            f = {"velocity": np.stack([c.get_field(abi.VELOG[k])[:, :, 1:-1] for k in range(3)]),
                 "vorticity": np.stack([c.get_field(abi.VORTG[k])[:, :, 1:-1] for k in range(3)]),
                 "buoyancy": c.get_field(abi.TBUOYG)[:, :, 1:-1]}
        out.append((info.parcel_stats[1], info.parcel_stats[12], f, int(info.n_parcels), t))
        c.close()
    return out


def pair_errors(a, b) -> dict:
    ke1, en1, f1, n1, t1 = a
    ke0, en0, f0, n0, t0 = b
    out = {"ke_rel_drift": abs(ke1 - ke0) / abs(ke0), "enstrophy_rel_drift": abs(en1 - en0) / abs(en0),
           "parcels": [n0, n1], "t": [t0, t1]}
    if f0 is not None:
        for k in f0:
            x, y = f1[k], f0[k]
            out[k + "_l2_rel"] = float(np.sqrt(((x - y) ** 2).sum() / max((y ** 2).sum(), 1e-300)))
            out[k + "_linf_rel"] = float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-300))
    return out


def mixed_error_at_size(lib, args) -> dict:
    """Errors of the mixed form against the plain FP64 form from the same
    seed.  On its own workload (256x256x128): 100 steps at the fixed dt 0.05
    (both runs at the same times; merge, split and corrections on).  With the
    adaptive dt (thermal 64^3, 100 steps): mixed against plain, and, as the
    flow's own sensitivity, plain against plain in the reference's container
    order (the same FP64 arithmetic with other summation orders)."""
    from epic_b200 import initial
    steps = args.error_steps
    spec = initial.device_spec("thermal-256x256x128")
    fixed = dict(use_fixed_dt=1, fixed_dt=0.05, keep_order=0)
    m, p = run_pair(lib, spec, steps, dict(fixed, precision=1), dict(fixed, precision=0))
    out = {"fixed_dt": dict(pair_errors(m, p), workload=f"thermal-256x256x128, {steps} steps at fixed dt 0.05, "
                                                          "mixed vs plain FP64 from the same seed"),
           "target": 1e-5}
    spec64 = initial.device_spec("thermal-64")
    m, p, q = run_pair(lib, spec64, steps, dict(precision=1, keep_order=0), dict(precision=0, keep_order=0),
                       dict(precision=0, keep_order=1), fields=False)
    out["adaptive_dt"] = {"workload": f"thermal-64, {steps} steps, adaptive dt",
                          "mixed_vs_plain": pair_errors(m, p), "plain_vs_plain_other_order": pair_errors(q, p)}
    out["within_target"] = bool(out["fixed_dt"]["ke_rel_drift"] < 1e-5 and out["fixed_dt"]["enstrophy_rel_drift"] < 1e-5)
    return out


def served_form(args, lib, dev) -> dict:
    """The served ensemble as a form of the default run (see run_served)."""
    return run_served(args, lib=lib, dev=dev, emit=False)


# ---------------------------------------------------------------------------
def mixed_error(lib, steps: int = 100, dt: float = 0.05) -> dict:
    """Errors of the mixed form against the plain FP64 form from the same
    seeded state (the rising thermal on 32^3, 262,144 parcels, merge / split /
    corrections on): relative drift of kinetic energy and enstrophy
    (parcel_diagnostics.f90:139-143) after `steps` steps at a fixed dt, and the
    relative L2 and Linf errors of the gridded velocity, vorticity and
    buoyancy (par2grid + vor2vel of the final parcels).  The step is fixed so
    that both runs compare the same times."""
    from epic_b200 import initial
    spec = initial.device_spec("thermal-32")
    fixed = dict(use_fixed_dt=1, fixed_dt=dt, keep_order=0)
    m, p = run_pair(lib, spec, steps, dict(fixed, precision=1), dict(fixed, precision=0))
    out = pair_errors(m, p)
    out.update({"workload": f"thermal 32^3, {steps} steps at fixed dt {dt}, mixed vs plain FP64 from the same seed",
                "target": 1e-5})
    out["within_target"] = bool(out["ke_rel_drift"] < 1e-5 and out["enstrophy_rel_drift"] < 1e-5)
    return out


def served_requests(args, lib):
    """The served ensemble: requests with seeded Poisson arrivals, grids drawn
    uniformly from {32^3, 48^3, 64^3, 96x96x48}, a Beltrami (k, l, m in {1, 2})
    or thermal initial state of its own seed, mixed precision."""
    from epic_b200 import serve
    rng = np.random.default_rng(args.served_seed)
    grids = [(32, 32, 32), (48, 48, 48), (64, 64, 64), (96, 96, 48)]
    reqs, arrivals, meta = [], [], []
    t = 0.0
    for r in range(args.served_requests):
        t += float(rng.exponential(1.0 / args.served_rate))
        g = grids[int(rng.integers(0, len(grids)))]
        kind = "beltrami" if rng.random() < 0.5 else "thermal"
        klm = tuple(int(v) for v in rng.integers(1, 3, size=3))
        reqs.append(serve.request(kind, g, seed=1000 + r, klm=klm, steps=args.served_steps, precision=1, lib=lib,
                                  tune=not args.no_autotune))
        arrivals.append(t)
        meta.append({"grid": list(g), "kind": kind, "klm": list(klm) if kind == "beltrami" else None})
    return reqs, arrivals, meta


def run_served(args, lib=None, dev=None, emit=True):
    import torch
    import epic_b200
    from epic_b200 import serve

    world, rank, local = dist_setup()
    if dev is None:
        torch.cuda.set_device(local if world > 1 else 0)
        dev = torch.cuda.current_device()
    lib = lib or epic_b200.load()
    reqs, arrivals, meta = served_requests(args, lib)
    clocks = ClockSampler(dev)
    srv = serve.Server(slots=args.served_slots, hbm_fraction=0.8, lib=lib, policy=args.served_policy)
    ids = []
    clocks.start()
    w0 = time.perf_counter()
    for req, ta in zip(reqs, arrivals):
        delay = ta - (time.perf_counter() - w0)
        if delay > 0:
            time.sleep(delay)
        ids.append(srv.submit(req))
    res = [srv.wait(i) for i in ids]
    wall = time.perf_counter() - w0
    clk = clocks.stop()
    srv.close()
    failed = [r for r in res if r["status"] != 0]
    lat = np.array([r["t_done"] - r["t_submit"] for r in res if r["status"] == 0])
    ps = sum(r["parcel_steps"] for r in res if r["status"] == 0)
    span = max(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
    value = ps / span
    ps_total = value
    if world > 1 and emit:
        # replicas: every rank serves its own copy of the ensemble
        _, ps_total = reduce_timing(span * 1e3, float(ps))
        ps_total = ps_total / span
    req_bytes = C_sizeof_request()
    workload = (f"served ensemble: {len(reqs)} requests, Poisson arrivals {args.served_rate}/s "
                f"(seed {args.served_seed}), grids 32^3/48^3/64^3/96x96x48, Beltrami (k,l,m in 1..2) "
                f"or thermal, {args.served_steps} mixed-precision steps each, "
                f"{args.served_slots} slots, admission by free HBM, {args.served_policy} order")
    latency = {"p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
               "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
               "mean_s": float(lat.mean()) if len(lat) else None,
               "max_s": float(lat.max()) if len(lat) else None}
    timing = ("host steady clock of the server: submit to completion per request; "
              "aggregate = parcel-steps / (last completion - first submission)")
    if not emit:
        return {"value": value, "unit": UNIT, "workload": workload, "latency": latency, "failed": len(failed),
                "clocks": clk, "wall_s": wall, "span_s": span, "parcel_steps": ps, "timing": timing,
                "arrival_span_s": arrivals[-1] if arrivals else 0.0}
    line = {
        "metric": METRIC, "value": ps_total, "unit": UNIT, "n_gpus": world, "steps": args.served_steps,
        "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32/f64", "data": "synthetic",
        "config": {"workload": workload,
                   "form": "served", "requests": len(reqs), "slots": args.served_slots,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "timing": timing},
        "latency": latency,
        "failed": len(failed),
        "failures": [dict(meta[k], message=r["message"]) for k, r in enumerate(res) if r["status"] != 0][:8],
        "clocks": clk,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": req_bytes * len(reqs) / max(1, args.served_steps * len(reqs)),
                "d2h_bytes_per_step": 0, "mode": "requests submitted through the server's C ABI; "
                "initial states generated on the device; results (diagnostics) read back"},
        "wall_s": wall, "span_s": span, "parcel_steps": ps,
    }
    if rank == 0 and not args.no_error:
        line["error"] = mixed_error(lib)
    if rank == 0:
        print(json.dumps(line))


def C_sizeof_request():
    import ctypes
    from epic_b200 import serve
    return ctypes.sizeof(serve.EpicRequest)


def oracle_sample_workload():
    """The bounded CPU sample: the same rising thermal on a 64^3 grid
    (2,097,152 parcels, same parcel density and physics), one step."""
    from epic_b200 import initial
    return initial.thermal(64, name="thermal-64")


def cpu_baseline(args):
    import oracle
    lib = oracle.load(threads=True)
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    from epic_b200 import make_context
    s = oracle_sample_workload()
    ctx = make_context(s, lib)
    t = 0.0
    t0 = time.perf_counter()
    n0 = ctx.num_parcels()
    t, info = ctx.step(t)
    el = time.perf_counter() - t0
    return {"value": n0 / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"1 step of the rising thermal on a 64^3 grid ({n0} parcels, same density and physics), "
                      f"{el:.1f} s wall, oracle OpenMP build",
            "seconds": el}


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return
    import oracle
    lib = oracle.load(threads=True)
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    from epic_b200 import initial, make_context
    s = oracle_sample_workload()
    ctx = make_context(s, lib)
    t = 0.0
    for _ in range(args.warmup):
        t, _ = ctx.step(t)
    ps = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ps += ctx.num_parcels()
        t, _ = ctx.step(t)
    el = time.perf_counter() - t0
    ctx.close()
    v = ps / el
    # the per-parcel-step rate of the sample against the full workload: one
    # step of the 128^3 thermal itself (16,777,216 parcels)
    full = None
    if not args.no_full_check:
        sf = initial.config("thermal-128")
        cf = make_context(sf, lib)
        n0 = cf.num_parcels()
        t1 = time.perf_counter()
        cf.step(0.0)
        ef = time.perf_counter() - t1
        cf.close()
        full = {"workload": "thermal-128 (the GPU arm's workload), first step", "parcels": n0, "seconds": ef,
                "value": n0 / ef, "unit": UNIT, "ratio_to_sample": (n0 / ef) / v}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": args.workload, "sample": "each step is one step of the rising thermal on a "
                       "64^3 grid (2,097,152 parcels, 8/cell, same physics) as a bounded sample of the workload; "
                       "parcel-steps/s per parcel-step is size-independent (full_size_check: one step of the "
                       "128^3 workload itself)",
                       "full_size_check": full},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": "64^3 rising thermal, one step per timed step"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference Fortran not buildable here (no Fortran compiler, MPI or NetCDF); "
                    "timed the CPU restatement of its step (oracle/, OpenMP)"}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="thermal-128")
    ap.add_argument("--form", default="plain", choices=["plain", "mixed", "served"],
                    help="plain FP64, the mixed-precision form (FP32 attributes and interpolation), "
                         "or the served ensemble")
    ap.add_argument("--served-requests", type=int, default=64)
    ap.add_argument("--served-rate", type=float, default=4.0, help="mean arrivals per second")
    ap.add_argument("--served-steps", type=int, default=100)
    ap.add_argument("--served-slots", type=int, default=8)
    ap.add_argument("--served-seed", type=int, default=2024)
    ap.add_argument("--served-policy", default="arrival", choices=["arrival", "shortest-first"],
                    help="admission order of the server's queue")
    ap.add_argument("--roofline-kernel", default="stage", choices=["stage", "p2g", "g2p", "fft"])
    ap.add_argument("--traffic", type=float, default=None, help="ncu DRAM bytes per launch of that kernel")
    ap.add_argument("--profile-kernels", default="", help="comma list of kernels to time over one extra step each")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-forms", action="store_true",
                    help="default plain run: skip the developed-flow window and the mixed and served forms")
    ap.add_argument("--developed-at", type=int, default=100,
                    help="the developed-flow window of the default run starts after this many steps")
    ap.add_argument("--error-steps", type=int, default=100)
    ap.add_argument("--no-full-check", action="store_true",
                    help="reference arm: skip the one step of the full 128^3 workload")
    ap.add_argument("--spinup", type=int, default=0, help="untimed steps before the warm-up (developed flow)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--scatter-groups", type=int, default=None, choices=range(6),
                    help="log2 of the consecutive parcels a lane group of the scatters takes (overrides the tuner)")
    ap.add_argument("--fft-path", type=int, default=None, choices=range(4),
                    help="horizontal FFT: 0 plane, 1 tiled lines, 2 Stockham lines, 3 half-plane clusters "
                         "(overrides the tuner)")
    ap.add_argument("--parcels-per-cell", type=int, default=0,
                    help="device-generated initial state with this many parcels per cell (profiling the grid "
                         "kernels on a small device footprint); 0: the workload's 8")
    ap.add_argument("--keep-order", type=int, default=0, choices=[0, 1],
                    help="1: keep the reference's container order (no box sort)")
    ap.add_argument("--device-init", action="store_true",
                    help="generate the initial parcels on the device (always for thermal2-512x512x256)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-error", action="store_true",
                    help="mixed and served forms: skip the error report against the plain FP64 form")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.form == "served":
        run_served(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
