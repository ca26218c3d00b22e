"""Delay-and-sum benchmark: one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the 3-D diverging-wave volume (32x32 = 1024-channel matrix array,
16 diverging transmits, 4096 samples, batch 1, 128^3 voxels, FP32), seeded
synthetic channel data built on the device.  A step is one ffdas das call on
that volume (ingest + delay-and-sum kernel); its inputs (268 MB of channel
data, 2 x 134 MB of delays/weights) exceed the 126 MB L2, so no flush is
needed between steps.  Metric: voxel x channel x transmit x batch units per
second (Gvox.ch.tx/s), whole job, all ranks.

N > 1 (torchrun): every rank beamforms its own volume (independent frames,
weak scaling, no collective on the data path); the timed region is bracketed
by a barrier and synchronize on both sides and the time is the max over ranks.

Extra keys: `roofline` for the delay-and-sum kernel (FP32 work, 5 flop/unit,
against the FP32 FMA peak measured on this GPU; the HBM figure beside it),
`cpu_baseline` (the FP32 C/OpenMP loop of the same formula on a voxel subset,
all host threads), `e2e` (one ffdas_das_from_host call per step on the
channel data in pinned host memory, whose upload overlaps the beamforming
inside the call, and the image read back; `e2e.serial` copies in, calls
ffdas_das and copies out in series, as the reference arm does;
`e2e.pipelined` overlaps consecutive steps through DASStream), `bf16` /
`fp16` (reduced-precision pair storage: throughput, speed-up over FP32 and
error against this library's FP64-pair pipeline), `bwd_fwd` (backward /
forward time on the differentiable 128-channel, 8-plane-wave, batch-4
workload, with the kernels that ran), `configs` (the 2-D plane-wave frame
under graph replay, the 200-frame FP16 ensemble, uneven das_sparse, the
GPU selection of das_sparse lists and the truncate_rank clutter filter on
beamformed ensembles), `in_record_fraction` (share of the units
whose tap lies inside the record) and `clocks` (SM clock and throttle reasons
sampled through NVML during the timed region).
`--impl reference` times the reference implementation (its CUDA das, built
from its sources into oracle/_ref) on the same workloads and GPU; that arm
never loads libffdas_b200.so (the workload generators are loaded from their
file, not through the package).
`--section bwd|configs` runs one part alone (for profiling).
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
from pathlib import Path

import numpy as np
import torch
import torch.distributed as dist

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DAS Gvox·ch·tx/s: bf16-in vs plain FP32 at ≤1e-3 rel err; bwd/fwd time ratio"
UNIT = "Gvox·ch·tx/s"
FLOP_PER_UNIT = 5.0


# ----------------------------------------------------------------- clocks ---
class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region.

    NVML is polled every 10 ms from a thread (read-only queries), so that even
    a timed region of a few hundred milliseconds yields tens of samples; when
    NVML is unavailable, nvidia-smi is polled every 200 ms instead.
    """
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int, period_s: float = 0.01):
        self.index = index
        self.period = period_s
        self.rows = []          # (sm_mhz, sm_max_mhz, set of reasons)
        self.proc = None
        self.thread = None
        self.stop_evt = threading.Event()
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID("GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            nv, hd = self._nvml_handle()
            smax = float(nv.nvmlDeviceGetMaxClockInfo(hd, nv.NVML_CLOCK_SM))
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}

            def poll():
                while not self.stop_evt.is_set():
                    try:
                        sm = float(nv.nvmlDeviceGetClockInfo(hd, nv.NVML_CLOCK_SM))
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(hd)
                        self.rows.append((sm, smax, {n for n, b in bits.items() if r & b}))
                    except Exception:
                        pass
                    self.stop_evt.wait(self.period)

            self.source = "nvml 10 ms"
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.source = "nvidia-smi 200 ms"
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            r = [c.strip() for c in line.split(",")]
            try:
                self.rows.append((float(r[1]), float(r[2]),
                                  {n for n, v in zip(self.NAMES, r[5:9]) if v.lower() == "active"}))
            except (ValueError, IndexError):
                continue

    def stop(self) -> dict:
        if self.thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi and NVML unavailable"]}
        self.stop_evt.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        self.thread.join(timeout=2)
        sm = [r[0] for r in self.rows]
        smax = [r[1] for r in self.rows]
        reasons = set().union(*[r[2] for r in self.rows]) if self.rows else set()
        load = [s for s in sm if smax and s > 0.5 * max(smax)] or sm
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": self.source}


# ------------------------------------------------------------------ utils ---
def workloads():
    """The seeded workload generators, loaded from their file.

    Importing them as `ffdas_b200.workloads` would run the package's
    `__init__`, which loads libffdas_b200.so; the reference arm must not map
    this library, so it loads the module on its own (it imports only numpy
    and torch)."""
    import importlib.util
    mod = sys.modules.get("_ffdas_workloads")
    if mod is None:
        spec = importlib.util.spec_from_file_location("_ffdas_workloads", ROOT / "ffdas_b200" / "workloads.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules["_ffdas_workloads"] = mod
        spec.loader.exec_module(mod)
    return mod


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured (MEASURED_PEAKS.json hbm_gbs)"}
    return {"hbm_gbs": 6650.0, "source": "fallback (MEASURED_PEAKS.json absent: the pool's earlier copy measurement)"}


def profile_field(name: str, key: str):
    """A figure of the committed ncu summary of the kernel (profiles/<name>.json), if any."""
    p = ROOT / "profiles" / f"{name}.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get(key)
        except Exception:
            return None
    return None


def profile_traffic(name: str):
    """Per-launch DRAM bytes of the kernel from the committed ncu summary, if any."""
    return profile_field(name, "dram_bytes_per_launch")


def timed(fn, steps: int, warmup: int, stream, world: int):
    for _ in range(warmup):
        fn()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = a.elapsed_time(b) / steps
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms


def in_record_fraction(wl, every: int = 8) -> float:
    """Share of units whose tap lies inside the record (0 <= floor(tau) < N-1),
    from every `every`-th voxel (all channels, events): the metric counts all
    units, like the reference, and this says how many of them are real taps."""
    x, dst, src, offs = wl["x"], wl["dstpos"], wl["srcpos"], wl["offsets"]
    N = x.shape[-1]
    d = dst.reshape(-1, 3)[::every].float()
    o = offs.reshape(offs.shape[0], -1)[:, ::every].float()
    inside = 0
    total = 0
    for c0 in range(0, src.shape[0], 64):
        r = torch.cdist(d, src[c0:c0 + 64].float())                 # (v, c)
        tau = r[None] + o.t()[None].permute(2, 1, 0)                # (s, v, c)
        k = torch.floor(tau)
        inside += int(((k >= 0) & (k < N - 1)).sum())
        total += tau.numel()
    return inside / max(total, 1)


def algorithmic_bytes(wl, x_bytes_per_sample: int) -> int:
    x = wl["x"]
    V = int(np.prod(wl["dstpos"].shape[:-1]))
    C, S = x.shape[-3], x.shape[-2]
    B = x.shape[0]
    n_ev = wl["offsets"].shape[0]
    return int(x.numel() * x_bytes_per_sample + 2 * n_ev * V * 4 + V * 12 + C * 12 + B * V * 4)


# ------------------------------------------------------------ CPU baseline ---
def cpu_baseline(wl, budget_s: float = 12.0) -> dict:
    from oracle import oracle
    x = wl["x"][0].cpu().numpy()
    srcpos = wl["srcpos"].cpu().numpy()
    dst = wl["dstpos"].cpu().numpy()
    offs = wl["offsets"].cpu().numpy()
    w = wl["weights"].cpu().numpy()
    nz = dst.shape[0]
    C, S = x.shape[0], x.shape[1]
    threads = oracle.num_threads()
    per_plane = int(np.prod(dst.shape[1:-1])) * C * S

    def run(planes):
        t0 = time.perf_counter()
        oracle.das_f32(x[None], srcpos, dst[:planes], offs[:, :planes], w[:, :planes])
        return time.perf_counter() - t0

    run(1)                                   # warm-up (page-in, thread pool)
    t1 = run(1)
    planes = int(max(1, min(nz, budget_s / max(t1, 1e-3))))
    # take planes spread over depth so near and far voxels are both sampled
    sel = np.linspace(0, nz - 1, planes).astype(int)
    t0 = time.perf_counter()
    oracle.das_f32(x[None], srcpos, dst[sel], offs[:, sel], w[:, sel])
    dt = time.perf_counter() - t0
    units = planes * per_plane
    return {"value": units / dt / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{planes} of {nz} depth planes ({units:.3g} units), FP32 C/OpenMP loop, "
                      f"{threads} threads, {dt:.1f} s"}


# ------------------------------------------------------------ reference ---
def run_reference(args, rank, world) -> dict:
    W = workloads()
    from oracle import reference
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    wl = W.diverging3d(device=dev)
    units = wl["units"]
    if not reference.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libffdas_ref.so was not built "
                "(the reference sources were absent at build time)"}
    call = reference.Prepared(wl["x"], wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"], alg=1)
    stream = torch.cuda.current_stream(dev)
    clocks = ClockSampler(dev.index)
    clocks.start()
    ms = timed(call, args.steps, args.warmup, stream, 1)
    ck = clocks.stop()
    # e2e: channel data from pinned host memory, image back, every step
    xh = wl["x"].cpu().pin_memory()
    out_h = torch.empty(call.out.shape, dtype=torch.float32).pin_memory()

    def e2e():
        call.x.copy_(xh, non_blocking=True)
        call()
        out_h.copy_(call.out, non_blocking=True)
    ms_e2e = timed(e2e, args.steps, args.warmup, stream, 1)
    call.close()
    value = units / (ms * 1e-3) / 1e9
    cpu = cpu_baseline(wl) if args.cpu_baseline else None
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "diverging3d: 32x32 matrix array (1024 ch), 16 diverging transmits, "
                       "4096 samples, batch 1, 128^3 voxels, FP32", "units_per_step": units,
                       "l2": "inputs larger than L2 (no flush)", "reference": "ffdas ALG1 (DEFAULT) "
                       "built for sm_100a from the reference sources, run on the same GPU"},
            "device": "gpu",
            "e2e": {"value": units / (ms_e2e * 1e-3) / 1e9, "unit": UNIT,
                    "h2d_bytes_per_step": int(wl["x"].numel() * 4), "d2h_bytes_per_step": int(call.out.numel() * 4),
                    "api": "reference ffdas_das per step: pinned host copy in, call, copy out (serial)"},
            "clocks": ck}
    if cpu:
        line["cpu_baseline"] = cpu
    if not args.quick:
        line.update(config_extras(args, "reference"))
    return line


# ------------------------------------------------------------------ ours ---
def run_ours(args, rank, world) -> dict:
    import ffdas_b200
    from ffdas_b200 import workloads as W
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    wl = W.diverging3d(device=dev, seed=1 + rank)
    x, srcpos, dstpos, offs, w = wl["x"], wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"]
    units = wl["units"]
    stream = torch.cuda.current_stream(dev)
    out = torch.empty((1, *dstpos.shape[:-1]), device=dev)
    h = ffdas_b200.get_library_handle(dev)
    # schedule picked by the autotuner on these inputs (not timed)
    from ffdas_b200.tune import autotune
    if args.schedule:
        tuned = {"config": json.loads(args.schedule), "ms": None, "table": []}
    else:
        tuned = autotune(x, srcpos, dstpos, offs, w, reps=2, use_cache=False)
    h.set_config(tuned["config"])

    def step():
        ffdas_b200.das(x, srcpos, dstpos, offs, w, out=out)

    clocks = ClockSampler(dev.index)
    clocks.start()
    ms = timed(step, args.steps, args.warmup, stream, world)
    ck = clocks.stop()
    value = units * world / (ms * 1e-3) / 1e9

    # kernel-only duration of the delay-and-sum kernel (events inside the library)
    h.set_kernel_timing(True)
    kms = []
    for _ in range(max(3, args.steps)):
        step()
        kms.append(h.last_kernel_ms())
    # units the kernel actually evaluated: it skips passes and stages whose
    # every tap lies outside the record (they add exactly nothing)
    units_eval = h.last_kernel_units()
    h.set_kernel_timing(False)
    info = h.last_kernel_info()
    kernel_ms = statistics.mean(kms[1:]) if len(kms) > 1 else kms[0]
    fp32_peak = h.measure_fp32_peak()
    pk = peaks()
    work_units = units_eval if units_eval is not None else units
    achieved_tf = FLOP_PER_UNIT * work_units / (kernel_ms * 1e-3) / 1e12
    bytes_alg = algorithmic_bytes(wl, 4)
    tile_voxels = info["tile_x"] * info["tile_y"] * info["tile_z"]
    if info["variant"] == 2 and tile_voxels == 512:
        kname, pname = "das_staged2_kernel<f32 pairs>", "das_staged2_diverging3d"
    elif info["variant"] == 2:
        kname, pname = "das_staged_kernel<f32 pairs>", "das_staged_diverging3d"
    else:
        kname, pname = "das_gather_kernel<f32 pairs>", "das_gather_diverging3d"
    # secondary ceilings of the same kernel, in units per second: the shared-
    # memory data path (128 B per clock per SM; one 8-byte f32 pair per tap)
    # and instruction issue (4 warp instructions per clock per SM, at the
    # thread instructions per unit of the committed ncu summary)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    clk_hz = (ck.get("sm_mhz") or ck.get("sm_max_mhz") or 1965.0) * 1e6
    ups = work_units / (kernel_ms * 1e-3)
    smem_ceiling = sms * (128 / 8) * clk_hz
    ceilings = {"smem_f32_pairs": {"units_per_s": smem_ceiling, "achieved_frac": ups / smem_ceiling,
                                   "basis": f"{sms} SMs x 16 taps/clk (128 B/clk, 8-B pairs) x {clk_hz / 1e9:.3f} GHz"}}
    ipu = profile_field(pname, "thread_instr_per_unit")
    if ipu:
        issue_ceiling = sms * 128 * clk_hz / ipu
        ceilings["issue"] = {"units_per_s": issue_ceiling, "achieved_frac": ups / issue_ceiling,
                             "basis": f"{sms} SMs x 128 thread-instr/clk / {ipu:.2f} instr per unit (ncu summary)"}
    roofline = {"bound": "fp32", "achieved": achieved_tf, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved_tf / fp32_peak, "traffic": profile_traffic(pname),
                "kernel": kname, "kernel_ms": kernel_ms,
                "peak_source": "FP32 FMA throughput measured on this GPU by ffdas_measure_fp32_peak "
                               "(faster of scalar FFMA and packed FFMA2)",
                "flop_per_unit": FLOP_PER_UNIT, "units_per_launch": units,
                "units_evaluated": work_units, "evaluated_fraction": work_units / units,
                "achieved_basis": "5 flop x units the kernel evaluated / kernel time (out-of-record passes and "
                                  "stages it skips are not counted as work)",
                "ceilings": ceilings,
                "hbm": {"algorithmic_bytes": bytes_alg, "achieved_gbs": bytes_alg / (kernel_ms * 1e-3) / 1e9,
                        "peak_gbs": pk["hbm_gbs"], "peak_source": pk["source"]}}

    # e2e through the public API: pinned host channel data in, image out
    xh = x.cpu().pin_memory()
    xd = torch.empty_like(x)
    out_h = torch.empty(out.shape, dtype=torch.float32).pin_memory()

    def e2e():
        xd.copy_(xh, non_blocking=True)
        ffdas_b200.das(xd, srcpos, dstpos, offs, w, out=out)
        out_h.copy_(out, non_blocking=True)
    ms_e2e_serial = timed(e2e, args.steps, args.warmup, stream, world)

    # e2e through the host-data entry point (ffdas_das_from_host): one call
    # per step takes the pinned host channel data; inside the call the upload
    # runs in channel runs on a second stream, each run beamformed as it lands,
    # and the image is read back after the call (no overlap between steps)
    def e2e_host():
        ffdas_b200.das_from_host(xh, srcpos, dstpos, offs, w, out=out)
        out_h.copy_(out, non_blocking=True)
    ms_e2e_host = timed(e2e_host, args.steps, args.warmup, stream, world)

    # e2e through the streaming API (DASStream): the same per-step copies and
    # call, with frame i+1's upload and frame i-1's download overlapping frame
    # i's delay-and-sum on separate streams; device-timed from before the first
    # upload to after the last download
    from ffdas_b200.runner import DASStream
    pipe = DASStream(x, srcpos, dstpos, offs, w, tune=False, config=tuned["config"])
    outs = [torch.empty(out.shape, dtype=torch.float32).pin_memory() for _ in range(max(args.steps, args.warmup))]
    pipe.run([xh] * args.warmup, outs[:args.warmup])
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ea = torch.cuda.Event(enable_timing=True)
    eb = torch.cuda.Event(enable_timing=True)
    ea.record(stream)
    pipe.run([xh] * args.steps, outs[:args.steps])
    stream.wait_stream(pipe.download_stream)
    eb.record(stream)
    torch.cuda.synchronize()
    ms_e2e = ea.elapsed_time(eb) / args.steps
    if world > 1:
        t = torch.tensor([ms_e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
        dist.barrier()

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "diverging3d: 32x32 matrix array (1024 ch), 16 diverging transmits, "
                       "4096 samples, batch 1, 128^3 voxels, FP32", "units_per_step": units * world,
                       "parallelism": f"replicas x{world} (independent volumes)" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (no flush)", "schedule": info,
                       "autotune": {"best": tuned["config"], "top": tuned["table"][:5]}},
            "roofline": roofline,
            # e2e: one C-ABI call per step with the channel data in pinned
            # host memory (ffdas_das_from_host), the image copied back; the
            # reference arm's only API is copy in, call, copy out, which is
            # `serial` here (same per-step bytes); `pipelined` overlaps steps
            "e2e": {"value": units * world / (ms_e2e_host * 1e-3) / 1e9, "unit": UNIT,
                    "h2d_bytes_per_step": int(x.numel() * 4), "d2h_bytes_per_step": int(out.numel() * 4),
                    "api": "ffdas_b200.das_from_host (C-ABI ffdas_das_from_host) per step on pinned host channel "
                           "data, upload overlapping the beamforming inside the call; image copied out",
                    "serial": {"value": units * world / (ms_e2e_serial * 1e-3) / 1e9,
                               "api": "per step: pinned host copy in, ffdas_b200.das, copy out, in series "
                                      "(the reference arm's protocol)"},
                    "pipelined": {"value": units * world / (ms_e2e * 1e-3) / 1e9,
                                  "api": "ffdas_b200.runner.DASStream (frame i+1's upload and frame i-1's "
                                         "download overlapping frame i)"}},
            "gpu_launches": 2 * args.steps,
            "in_record_fraction": in_record_fraction(wl),
            "clocks": ck}

    if rank == 0 and world == 1 and not args.quick:
        line.update(extras(args, wl, ms, h))
        line.update(bwd_extras(args, h))
        line.update(config_extras(args, "ours"))
        if args.cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(wl)
    return line


def error_report(img: np.ndarray, ref: np.ndarray) -> dict:
    d = img.astype(np.float64) - ref
    peak = float(np.abs(ref).max()) or 1.0
    rel = float(np.linalg.norm(d) / max(np.linalg.norm(ref), 1e-300))
    pa = float(np.abs(d).max())
    return {"rel_l2": rel, "peak_abs": pa, "peak_db_below_max": float(20 * np.log10(max(pa, 1e-300) / peak))}


def extras(args, wl, ms_fp32, h) -> dict:
    """16-bit channel data: throughput (kernel and end to end) and error.

    `bf16` / `fp16`: the channel data arrives as 16-bit values (default
    compute type: widened exactly to FP32 pairs on ingest); `e2e` copies the
    16-bit data from pinned host memory each step, so it moves half the bytes
    of the FP32 e2e.  `bf16_pairs` / `fp16_pairs`: FP32 data stored as 16-bit
    pairs (the fp16 / bf16 compute types), which halves the workspace.  The
    error reference is this library's own FP64 pipeline (FP64 pairs and
    accumulation, the same FP32 delays) on the FP32 data, six depth planes
    spread over the volume, so the figure includes quantising the data to 16
    bits; the test suite holds the same claims against the FP64 CPU oracle.
    """
    import ffdas_b200
    from ffdas_b200 import workloads as W
    dev = wl["x"].device
    srcpos, dstpos, offs, w = wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"]
    units = wl["units"]
    xn = W.normalize_channels(wl["x"])          # per-channel peak 1
    stream = torch.cuda.current_stream(dev)
    res = {}
    nz = dstpos.shape[0]
    sel = torch.from_numpy(np.linspace(0, nz - 1, 6).astype(np.int64)).to(dev)
    h.set_config(None)
    ref = ffdas_b200.das(xn.double(), srcpos, dstpos[sel].contiguous(), offs[:, sel].contiguous(),
                         w[:, sel].contiguous()).cpu().numpy()

    from ffdas_b200.tune import autotune
    out = torch.empty((1, *dstpos.shape[:-1]), device=dev)

    def measure(x, **kw):
        tkw = {k: v for k, v in kw.items() if k != "channel_scale"}
        cfg = autotune(x, srcpos, dstpos, offs, w, reps=2, use_cache=False, **tkw)["config"]
        h.set_config(cfg)
        ms = timed(lambda: ffdas_b200.das(x, srcpos, dstpos, offs, w, out=out, **kw), args.steps, args.warmup,
                   stream, 1)
        img = out[:, sel].cpu().numpy()
        return ms, error_report(img, ref), cfg

    def measure_e2e(x):
        xh = x.cpu().pin_memory()
        xd = torch.empty_like(x)
        out_h = torch.empty(out.shape, dtype=torch.float32).pin_memory()

        def e2e():
            xd.copy_(xh, non_blocking=True)
            ffdas_b200.das(xd, srcpos, dstpos, offs, w, out=out)
            out_h.copy_(out, non_blocking=True)
        return timed(e2e, args.steps, args.warmup, stream, 1), int(x.numel() * x.element_size())

    ms32, err32, _ = measure(xn)
    e2e32, b32 = measure_e2e(xn)
    res["fp32_error_vs_fp64_pairs"] = err32
    res["fp32_normalised"] = {"ms_per_step": ms32, "e2e": {"value": units / (e2e32 * 1e-3) / 1e9, "unit": UNIT,
                                                          "h2d_bytes_per_step": b32}}
    for name, dt in (("bf16", torch.bfloat16), ("fp16", torch.float16)):
        x = xn.to(dt)
        msr, err, cfg = measure(x)
        e2e, bb = measure_e2e(x)
        res[name] = {"value": units / (msr * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": msr,
                     "speedup_vs_fp32": ms32 / msr, "error_vs_fp64_pairs": err, "schedule": cfg,
                     "e2e": {"value": units / (e2e * 1e-3) / 1e9, "unit": UNIT, "h2d_bytes_per_step": bb,
                             "speedup_vs_fp32_e2e": e2e32 / e2e},
                     "input": f"channel data given as {name} (per-channel peak 1), widened to FP32 pairs on ingest"}
        flag = "use_bf16" if dt == torch.bfloat16 else "use_fp16"
        msp, errp, cfgp = measure(xn, **{flag: True})
        res[name + "_pairs"] = {"value": units / (msp * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": msp,
                                "speedup_vs_fp32": ms32 / msp, "error_vs_fp64_pairs": errp, "schedule": cfgp,
                                "input": f"FP32 channel data stored as {name} pairs ({flag}), half the workspace"}
        # the same with the per-channel normalisation done by the library's
        # ingest (ffdas_set_channel_scale, scale = 1 / peak) on the raw data
        xr = wl["x"]
        inv_peak = 1.0 / xr.abs().amax(dim=(0, 2, 3)).clamp_min(1e-30)
        mss, errs, cfgs = measure(xr, **{flag: True, "channel_scale": inv_peak})
        res[name + "_pairs_channel_scale"] = {
            "value": units / (mss * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": mss, "speedup_vs_fp32": ms32 / mss,
            "error_vs_fp64_pairs": errs, "schedule": cfgs,
            "input": f"raw FP32 channel data, normalised per channel (1 / peak) and stored as {name} pairs "
                     f"by the ingest (channel_scale)"}
    h.set_config(None)
    return res


def bwd_extras(args, h) -> dict:
    """Backward / forward time on the differentiable workload (autofocus).

    The forward is autotuned; the backward is timed under its planner default
    and a few staged-adjoint tiles plus the gather adjoint, and the fastest is
    reported together with the kernel that ran.
    """
    import ffdas_b200
    from ffdas_b200 import workloads as W, _lib
    from ffdas_b200._lib import DataType
    from ffdas_b200.tune import autotune
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    af = W.autofocus(device=dev)
    xa = af["x"]
    args_f = (af["srcpos"], af["dstpos"], af["offsets"], af["weights"])
    gout = torch.randn((xa.shape[0], *af["dstpos"].shape[:-1]), device=dev)
    fcfg = autotune(xa, *args_f, reps=2, use_cache=False)["config"]
    h.set_config(fcfg)
    xdsc = _lib.TensorDesc(list(xa.shape), list(xa.stride()), DataType.R_32F)
    # as in the autograd forward: the pair rows go into a buffer that the
    # backward then reads instead of building them again
    nbytes = _lib.pair_bytes(xdsc, 0)
    pairs = torch.empty(nbytes, dtype=torch.uint8, device=dev)

    def fwd():
        h.set_pair_buffer(pairs.data_ptr(), nbytes)
        ffdas_b200.das(xa, *args_f)
        h.set_pair_buffer(None, 0)

    msf = timed(fwd, args.steps, args.warmup, stream, 1)
    finfo = h.last_kernel_info()

    gx = torch.zeros(xa.shape, device=dev)
    go = torch.empty_like(af["offsets"])
    gw = torch.empty_like(af["weights"])
    gd = torch.empty_like(af["dstpos"])
    gs = torch.empty_like(af["srcpos"])
    gdsc = _lib.TensorDesc(list(gout.shape), None, DataType.R_32F)
    L = _lib.load()
    reuse = [True]
    every_grad = [True]

    def bwd():
        h.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        if reuse[0]:
            h.set_pair_buffer(pairs.data_ptr(), nbytes)
        # every_grad False: the gradients an autofocus step takes (the delays
        # and both position sets scale with the sound speed; x and the
        # weights do not), as the autograd function passes them
        gxp, gwp = (gx.data_ptr(), gw.data_ptr()) if every_grad[0] else (None, None)
        _lib.check(L.ffdas_das_backward(h.h, af["srcpos"].data_ptr(), None, 0.0, xdsc.desc, xa.data_ptr(),
                                        af["dstpos"].data_ptr(), af["offsets"].data_ptr(), af["weights"].data_ptr(),
                                        0, None, gdsc.desc, gout.data_ptr(), gxp, go.data_ptr(),
                                        gwp, gd.data_ptr(), gs.data_ptr()))
        h.set_pair_buffer(None, 0)

    table = []
    bcands = [None] + [dict(variant=2, tile_x=tx, tile_y=256 // tx, window=wb)
                       for tx in (8, 16, 32) for wb in (32, 64)] + [dict(variant=3)]
    if args.schedule_bwd:
        bcands = [json.loads(args.schedule_bwd)]
    for cfg in bcands:
        h.set_config(cfg)
        ms = timed(bwd, args.steps, args.warmup, stream, 1)
        table.append((ms, cfg, h.last_kernel_info()))
    table.sort(key=lambda t: t[0])
    msb, bcfg, binfo = table[0]
    # the same backward building its own pair rows (a backward without the
    # forward's buffer, e.g. called on its own through the C-ABI)
    reuse[0] = False
    h.set_config(bcfg)
    msb_own = timed(bwd, args.steps, args.warmup, stream, 1)
    reuse[0], every_grad[0] = True, False
    msb_af = timed(bwd, args.steps, args.warmup, stream, 1)
    h.set_config(None)

    # das_sparse: the focused 64-transmit frame (uneven lists of 1..32
    # transmits), planner schedules, the adjoint of every input and without
    # the weight gradient (padding entries then need no work)
    sf = W.sparse_focus(device=dev)
    xs, idx_s = sf["x"], sf["sparse_indices"]
    geo_s = (sf["srcpos"], sf["dstpos"], sf["offsets"], sf["weights"])
    msf_s = timed(lambda: ffdas_b200.das_sparse(xs, *geo_s, idx_s), args.steps, args.warmup, stream, 1)
    gout_s = torch.randn((1, *sf["dstpos"].shape[:-1]), device=dev)
    gxs, gos, gws = torch.zeros_like(xs), torch.empty_like(sf["offsets"]), torch.empty_like(sf["weights"])
    gds, gss = torch.empty_like(sf["dstpos"]), torch.empty_like(sf["srcpos"])
    xdsc_s = _lib.TensorDesc(list(xs.shape), None, DataType.R_32F)
    gdsc_s = _lib.TensorDesc(list(gout_s.shape), None, DataType.R_32F)
    with_w, with_x = [True], [True]

    def bwd_s():
        h.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(L.ffdas_das_backward(h.h, sf["srcpos"].data_ptr(), None, 0.0, xdsc_s.desc, xs.data_ptr(),
                                        sf["dstpos"].data_ptr(), sf["offsets"].data_ptr(),
                                        sf["weights"].data_ptr(), int(idx_s.shape[0]), idx_s.data_ptr(),
                                        gdsc_s.desc, gout_s.data_ptr(), gxs.data_ptr() if with_x[0] else None,
                                        gos.data_ptr(), gws.data_ptr() if with_w[0] else None, gds.data_ptr(),
                                        gss.data_ptr()))
    msb_s = timed(bwd_s, args.steps, args.warmup, stream, 1)
    binfo_s = h.last_kernel_info()
    with_w[0] = False
    msb_s_nw = timed(bwd_s, args.steps, args.warmup, stream, 1)
    # the gradients an autofocus step takes (delays and both position sets)
    with_x[0] = False
    msb_s_af = timed(bwd_s, args.steps, args.warmup, stream, 1)

    # complex IQ data with the phase rotation: the autofocus workload's
    # channel data as its analytic signal (complex64), wavenum 0.05, every
    # gradient (the complex adjoint, a thread per voxel)
    xc = W.analytic_signal(xa).to(torch.complex64)
    wn = 0.05
    msf_c = timed(lambda: ffdas_b200.das(xc, *args_f, wavenum=wn), args.steps, args.warmup, stream, 1)
    gout_c = torch.complex(gout, torch.roll(gout, 1, dims=-1)).contiguous()
    gxc = torch.zeros(xc.shape, dtype=torch.complex64, device=dev)
    xdsc_c = _lib.TensorDesc(list(xc.shape), None, DataType.C_32F)
    gdsc_c = _lib.TensorDesc(list(gout_c.shape), None, DataType.C_32F)

    def bwd_c():
        h.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(L.ffdas_das_backward(h.h, af["srcpos"].data_ptr(), None, wn, xdsc_c.desc, xc.data_ptr(),
                                        af["dstpos"].data_ptr(), af["offsets"].data_ptr(), af["weights"].data_ptr(),
                                        0, None, gdsc_c.desc, gout_c.data_ptr(), gxc.data_ptr(), go.data_ptr(),
                                        gw.data_ptr(), gd.data_ptr(), gs.data_ptr()))
    msb_c = timed(bwd_c, args.steps, args.warmup, stream, 1)
    binfo_c = h.last_kernel_info()
    return {"bwd_fwd": {"ratio": msb / msf, "fwd_ms": msf, "bwd_ms": msb,
                        "bwd_ms_own_pairs": msb_own, "ratio_own_pairs": msb_own / msf,
                        "pairs": "the backward reads the pair rows the forward built (ffdas_set_pair_buffer), as "
                                 "the autograd function does; ratio_own_pairs: it builds them itself",
                        "bwd_ms_autofocus_grads": msb_af, "ratio_autofocus_grads": msb_af / msf,
                        "autofocus_grads": "the gradients an autofocus step takes: delays, voxel and channel "
                                           "positions (x and the weights do not depend on the sound speed, so "
                                           "the autograd function passes no buffers for them)",
                        "fwd_schedule": finfo, "bwd_schedule": binfo, "bwd_config": bcfg,
                        "bwd_table": [[m, c, i["variant"]] for m, c, i in table],
                        "workload": "autofocus: 128 ch, 8 plane waves, batch 4, 2048 samples, 256x256 voxels; "
                                    "backward = grads of x, offsets, weights, voxel and channel positions"},
            "bwd_fwd_sparse": {"ratio": msb_s / msf_s, "fwd_ms": msf_s, "bwd_ms": msb_s,
                               "bwd_ms_without_weight_grad": msb_s_nw, "ratio_without_weight_grad": msb_s_nw / msf_s,
                               "bwd_ms_autofocus_grads": msb_s_af, "ratio_autofocus_grads": msb_s_af / msf_s,
                               "bwd_kernel": binfo_s,
                               "workload": "das_sparse, 128 ch, 64 focused transmits, 1536 samples, 400x256 "
                                           "pixels, lists of 1..32 transmits padded to 32; backward = grads of x, "
                                           "offsets, weights, voxel and channel positions (and the same "
                                           "without the weight gradient; autofocus_grads: offsets and the "
                                           "two position sets only)"},
            "bwd_fwd_complex": {"ratio": msb_c / msf_c, "fwd_ms": msf_c, "bwd_ms": msb_c, "bwd_kernel": binfo_c,
                                "workload": "autofocus channel data as its analytic signal (complex64), wavenum "
                                            "0.05; backward = grads of x, offsets, weights, voxel and channel "
                                            "positions"}}



def config_extras(args, impl: str) -> dict:
    """The other benchmark configurations, one entry each, for either arm.

    plane2d: 128-element linear array, 1 plane wave, 2048 samples, 256x128
      pixels, FP32; ours replays a captured CUDA graph (DASRunner), the
      reference is called through its API; time per call in microseconds.
    ensemble: 200-frame FP16 ensemble, 128 ch, 11 plane waves, 1536 samples,
      400x256 pixels (frames batched in one call).  The reference arm times
      both of its batched algorithms and reports the faster as the entry:
      ALG1 with its 16-frame register tile (its default tile of 32 has no
      float-output kernel, src/das/das_alg1.cu:219-239), and ALG2 on three
      64-frame calls plus ALG1 on the last 8 frames -- ALG2 sums correctly
      only when a call's batch equals its 64-frame batch block (see
      `reference_alg2_ok`).
    sparse_focus: das_sparse, 64 focused transmits, 1..32 events per pixel
      (padding repeats an index with zero weight); units count real events.
    Parity of the two arms on these inputs is held by the test suite.
    """
    W = workloads()
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    out = {}
    steps, warm = max(args.steps, 5), args.warmup
    for name in ("plane2d", "ensemble", "sparse_focus"):
        wl = W.CONFIGS[name](device=dev)
        geo = (wl["x"], wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
        idx = wl.get("sparse_indices")
        units = wl.get("real_units", wl["units"])
        reps = 50 if name == "plane2d" else 1
        if impl == "reference":
            from oracle import reference
            if not reference.available():
                out[name] = {"unavailable": "oracle/_ref/libffdas_ref.so not built"}
                continue
            B = wl["x"].shape[0]
            # the reference's default ALG1 batch tile for B >= 32 FP32 has no kernel; 16 is its largest
            call = reference.Prepared(*geo, sparse_indices=idx, alg=1, tile=16 if B >= 32 else None)

            def fn():
                for _ in range(reps):
                    call()
            ms = timed(fn, steps, warm, stream, 1) / reps
            call.close()
            kind = "reference ALG1 through ffdas_das" + ("_sparse" if idx is not None else "")
            alg_table = {"alg1": ms}
            if name == "ensemble":
                ms2 = reference_alg2_ensemble(wl, steps, warm, stream)
                if ms2 is not None:
                    alg_table["alg2_64_frame_calls"] = ms2
                    if ms2 < ms:
                        ms = ms2
                        kind = "reference ALG2 on 3 x 64 frames + ALG1 on the last 8 (the faster of its algorithms)"
        else:
            from ffdas_b200.runner import DASRunner
            run = DASRunner(*geo, sparse_indices=idx)

            def fn():
                for _ in range(reps):
                    run.replay()
            ms = timed(fn, steps, warm, stream, 1) / reps
            kind = f"ffdas_b200 CUDA graph replay, schedule {run.config}"
            alg_table = None
            del run
        e = {"value": units / (ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_call": ms, "units_per_call": units,
             "x_dtype": str(wl["x"].dtype).replace("torch.", ""), "impl": kind}
        if alg_table:
            e["reference_ms_by_algorithm"] = alg_table
        if name == "plane2d":
            e["us_per_call"] = ms * 1e3
        out[name] = e
        del wl, geo
        torch.cuda.empty_cache()
    out["sparse_select"] = select_extra(args, impl, dev, stream)
    out["rank_filter"] = rank_filter_extra(args, impl, dev, stream)
    return {"configs": out}


ALG2_FRAMES = 64


def reference_alg2_ok(B: int) -> bool:
    """Batch sizes on which the reference's ALG2 sums correctly.

    Its launcher sets the frames per batch block to min(roundup(B, 16), 64)
    (src/das/das_alg2.cu:405-408), while its kernel keeps (M * N) / 32
    accumulators per thread (das_alg2_kernels.cuh:38, 77) and fills them over
    n < N (:144) but writes them out over n < B (:169).  The two loops agree
    only when B equals the block, 64 frames, for 4-byte and 2-byte samples
    alike (with fewer frames the vector loads fill more accumulators than the
    array holds; with more, each block writes frames of the other blocks from
    accumulators it never filled).  The harness calls ALG2 only at B = 64."""
    return B == ALG2_FRAMES


def reference_alg2_ensemble(wl, steps: int, warm: int, stream):
    """The 200-frame ensemble through the reference's ALG2: three calls of 64
    frames and ALG1 (tile 8) on the last 8 frames, per call in ms; None when
    ALG2 cannot be driven safely (a tap outside the record: ALG2 reads an
    internal copy of x that cannot be guarded)."""
    from oracle import reference
    x = wl["x"]
    B = x.shape[0]
    geo = (wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
    calls = []
    try:
        for b0 in range(0, B - B % ALG2_FRAMES, ALG2_FRAMES):
            calls.append(reference.Prepared(x[b0:b0 + ALG2_FRAMES].contiguous(), *geo, alg=2))
        if B % ALG2_FRAMES:
            calls.append(reference.Prepared(x[B - B % ALG2_FRAMES:].contiguous(), *geo, alg=1, tile=8))
    except ValueError:
        for c in calls:
            c.close()
        return None

    def fn():
        for c in calls:
            c()
    ms = timed(fn, steps, warm, stream, 1)
    for c in calls:
        c.close()
    return ms


def rank_filter_extra(args, impl: str, dev, stream) -> dict:
    """The clutter filter that follows beamforming: truncate_rank with the 5
    leading (tissue) ranks removed, on a 200-frame 400x256 FP32 image
    ensemble (the ensemble configuration's output shape) and on a 64-frame
    64^3 complex64 volume (the reference's clutter_filter example).  Ours:
    ffdas_truncate_rank; reference: its ffdas_truncate_rank built from its
    sources (cuBLAS GEMM, cuSOLVER syevd, SYRK + SYMM).  Both calls return
    with the stream drained (the solver status is read on the host)."""
    W = workloads()
    out = {}
    steps, warm = max(args.steps, 5), args.warmup
    for name, (m, shape, dtype, seed) in {"ensemble_f32": (200, (400, 256), torch.float32, 51),
                                          "volume_c64": (64, (64, 64, 64), torch.complex64, 52)}.items():
        x = W.slow_time_ensemble(m, shape, dtype, dev, seed)
        if impl == "reference":
            from oracle import reference
            if not reference.available():
                out[name] = {"unavailable": "oracle/_ref/libffdas_ref.so not built"}
                continue
            call = reference.PreparedRank(x.view(m, -1), 5)
            ms = timed(call, steps, warm, stream, 1)
            call.close()
            kind = "reference ffdas_truncate_rank"
        else:
            import ffdas_b200
            res = torch.empty_like(x)
            ms = timed(lambda: ffdas_b200.truncate_rank(x, 5, out=res), steps, warm, stream, 1)
            kind = "ffdas_b200 ffdas_truncate_rank"
        out[name] = {"ms_per_call": ms, "shape": [m, *shape], "dtype": str(dtype).replace("torch.", ""),
                     "start": 5, "impl": kind}
        del x
        torch.cuda.empty_cache()
    return out


def select_extra(args, impl: str, dev, stream) -> dict:
    """Choosing the das_sparse lists: per voxel the 32 of 64 events with the
    largest weight (a seeded 0/1 beam mask plus jitter, 400x256 pixels), with
    weights and delays gathered.  Ours: ffdas_sparse_select on the GPU.  The
    reference does this step with host-array calls in its example
    (sparse_compounding.py:141-144, through CuPy, which is not installed here):
    the reference arm times the same numpy calls on the host."""
    g = torch.Generator().manual_seed(41)
    S, k, shape = 64, 32, (400, 256)
    w = (torch.rand((S, *shape), generator=g) < 0.3).float() + torch.rand((S, *shape), generator=g) * 1e-3
    o = torch.rand((S, *shape), generator=g) * 1000
    if impl == "reference":
        import time
        wn, on = w.numpy(), o.numpy()
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            i = np.argpartition(wn, -k, axis=0)[-k:]
            np.take_along_axis(wn, i, axis=0)
            np.take_along_axis(on, i, axis=0)
            ts.append(time.perf_counter() - t0)
        return {"us_per_call": min(ts) * 1e6, "impl": "host numpy argpartition + take_along_axis (the reference "
                "example's calls; CuPy absent)", "shape": [S, *shape], "k": k}
    import ffdas_b200
    wd, od = w.to(dev), o.to(dev)
    ms = timed(lambda: ffdas_b200.sparse_select(wd, k, offsets=od), max(args.steps, 5), args.warmup, stream, 1)
    return {"us_per_call": ms * 1e3, "impl": "ffdas_sparse_select (GPU)", "shape": [S, *shape], "k": k}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--quick", action="store_true", help="main metric only")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--schedule", default=None,
                    help="JSON schedule (ffdas_das_config_t fields) instead of autotuning, e.g. for profiling")
    ap.add_argument("--schedule-bwd", dest="schedule_bwd", default=None,
                    help="JSON schedule for the backward instead of trying several")
    ap.add_argument("--section", choices=["all", "bwd", "configs"], default="all",
                    help="bwd / configs: only that part, printed as its own JSON object (for profiling)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    try:
        if args.section != "all":
            if world > 1 or (args.impl == "reference" and args.section == "bwd"):
                return 0
            if args.section == "bwd":
                import ffdas_b200
                part = bwd_extras(args, ffdas_b200.get_library_handle(torch.device("cuda", 0)))
            else:
                part = config_extras(args, args.impl)
            print(json.dumps({"section": args.section, "impl": args.impl, **part}), flush=True)
            return 0
        if args.impl == "reference":
            if rank != 0:
                line = None
            else:
                line = run_reference(args, rank, world)
        else:
            line = run_ours(args, rank, world)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
