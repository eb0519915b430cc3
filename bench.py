#!/usr/bin/env python3
"""Throughput of delta.subtract on a 4096x4096 spatially varying field, one B200 per rank.

A step is one full subtract of one frame: stamp selection -> kernel fit (GCV) ->
subtract -> ZOGY decorrelation -> PSF estimate + matched-filter score -> CCL
catalog. Workload: 4096x4096 float32 pair, 20000 stars (dN/dF ~ F^-2.5 on
1e3..1e6 e-), elliptical Moffat (beta 3, q 0.85, PA 30 deg) science PSF whose
FWHM rises 3.0 -> 4.5 px along the diagonal, Gaussian FWHM 2.5 reference, 50
transients at S/N 5-50, 1% masked; n_max 6, 4x4 thin-plate knots, GCV,
stamp radius 15, decorrelate + score + catalog at 5 sigma. Inputs are seeded
synthetic frames (each rank its own seed: weak scaling, no collective on the
data path).

  value   Mpix/s of the mixed-precision path, layers resident in HBM
  plain   the same with the plain FP32 normal equations (one frame, and
          the same frames in flight as `value`)
  e2e     the public delta_b200.subtract() call from pinned host arrays
          (host->device upload and device->host products inside the timing)
  uneven  the batch of uneven frames below, mixed and plain FP32

`--impl reference` times the CPU chain of the same workload instead (the
reference's own detect/catalog/convolve code compiled from source plus the
C / NumPy restatements of its fit, subtract, decorrelation and score).

`--workload uneven` runs the batch of uneven frames instead: 64 frames of
2048x4096, 2048x2048 and 1024x4096 (science FWHM ~ U(2, 5) px, 500-20000 stars,
0-3% masked), 16 distinct seeded frames each queued four times in a seeded
order, through the end-to-end API with `--batch` frames in flight; it reports
aggregate Mpix/s and the per-frame p50 / p99 latency. Ranks take frames by
longest-processing-time dealing (descending pixel count).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "subtract Mpix/s on 1 B200: mixed-prec+batched vs plain, at stated FP64 error"
UNIT = "Mpix/s"
WORKLOAD = ("4096x4096 spatially varying Moffat field, 20000 stars, 50 transients; n_max 6, 16 TPS knots, GCV, "
            "decorrelate + score + CCL at 5 sigma; one frame per step per GPU")
# Algorithmic HBM bytes per science pixel of the fused model-convolve kernel:
# science + reference (float32), reference mask (u8), difference (float32).
MODEL_CONVOLVE_BYTES_PER_PX = 13
# FP32 FMA peak of the part (148 SMs x 128 FMA lanes x 1.965 GHz), for the
# compute side of the model convolve's roofline.
FP32_FMA_PEAK_TFMA = 148 * 128 * 1.965e9 / 1e12


def model_convolve_fma_per_px(n_max: int, radius: int, tile_h: int = 64) -> float:
    """Algorithmic FP32 FMAs per pixel of the fused model convolve: the NX
    shared x passes over the tile plus its y halo, the nc y passes, the blend."""
    nx = n_max + 1
    nc = (n_max + 1) * (n_max + 2) // 2
    ks = 2 * radius + 1
    return nx * ks * (tile_h + 2 * radius) / tile_h + nc * ks + nc
MODEL_CONVOLVE_STAGE = "subtract: model convolve"


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("delta_b200", "reference"), default="delta_b200")
    ap.add_argument("--size", type=int, default=4096, help="frame side (default: the 4096^2 workload)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--batch", type=int, default=4, help="frames in flight per GPU (each its own stream)")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU leg (rank 0, N=1)")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-batch leg of the default run")
    ap.add_argument("--workload", choices=("frame", "uneven", "precision", "grad"), default="frame",
                    help="frame: the 4096^2 workload (default); uneven: 64 frames of mixed sizes; "
                         "precision: the normal-equation precision study at 725 unknowns, ~4e6 rows; "
                         "grad: the gradient evaluations on 8 fields of 2048^2")
    return ap.parse_args(argv)


def frame_config(size: int) -> dict:
    scale = (size / 4096.0) ** 2
    return {"size": size, "n_stars": max(50, int(round(20000 * scale))),
            "n_transients": max(1, int(round(50 * scale)))}


def make_frame(size: int, seed: int):
    from delta_b200 import validation

    fc = frame_config(size)
    return validation.config2_pair(seed=seed, size=size, n_stars=fc["n_stars"], n_transients=fc["n_transients"])


UNEVEN_SHAPES = ((2048, 4096), (2048, 2048), (1024, 4096))  # (height, width)
UNEVEN_FRAMES, UNEVEN_DISTINCT = 64, 16


def uneven_specs(seed: int, n_distinct: int = UNEVEN_DISTINCT) -> list[dict]:
    """Seeded parameters of the distinct frames of the uneven batch: shapes in
    turn, science FWHM ~ U(2, 5) px, stars ~ U(500, 20000), masked ~ U(0, 3%)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_distinct):
        h, w = UNEVEN_SHAPES[i % len(UNEVEN_SHAPES)]
        specs.append({"height": h, "width": w, "n_stars": int(rng.uniform(500, 20000)),
                      "sci_fwhm": float(rng.uniform(2.0, 5.0)), "mask_fraction": float(rng.uniform(0.0, 0.03)),
                      "seed": seed * 1000 + i})
    return specs


def uneven_queue(seed: int, n_distinct: int = UNEVEN_DISTINCT, n_frames: int = UNEVEN_FRAMES) -> list[int]:
    """Distinct-frame index of every queued frame: whole seeded permutations of
    the distinct frames, repeated until n_frames are queued."""
    rng = np.random.default_rng(seed + 1)
    q: list[int] = []
    while len(q) < n_frames:
        q.extend(int(j) for j in rng.permutation(n_distinct))
    return q[:n_frames]


def lpt_deal(pixels: list[int], world: int) -> list[int]:
    """Owner rank of every item: items by descending pixel count (ties by
    index), each to the rank with the least pixels so far (lowest rank on ties)."""
    loads = [0] * max(1, world)
    owner = [0] * len(pixels)
    for i in sorted(range(len(pixels)), key=lambda i: (-pixels[i], i)):
        r = min(range(len(loads)), key=lambda k: (loads[k], k))
        owner[i] = r
        loads[r] += pixels[i]
    return owner


def subtract_kwargs(pair, precision: str | None = None) -> dict:
    kw = dict(n_max=6, n_knots=4, cv_folds=0, stamp_radius=15, threshold_sigma=5.0, decorrelate=True, score=True,
              source_catalog=True, saturation=pair.saturation)
    if precision is not None:
        kw["precision"] = precision
    return kw


# ---------------------------------------------------------------- clocks -------

_REASON_BITS = {
    "sw_power_cap": 0x4, "hw_slowdown": 0x8, "sync_boost": 0x10, "sw_thermal_slowdown": 0x20,
    "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80, "applications_clocks_setting": 0x2,
}


def summarise_clocks(samples: list[tuple[float, float, int]]) -> dict:
    """samples: (sm_mhz, sm_max_mhz, reasons bitmask) taken while the timed loop ran."""
    if not samples:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
    seen = 0
    for _, _, r in samples:
        seen |= int(r)
    return {"sm_mhz": float(statistics.median(s[0] for s in samples)),
            "sm_max_mhz": float(max(s[1] for s in samples)),
            "reasons": sorted(name for name, bit in _REASON_BITS.items() if seen & bit),
            "samples": len(samples)}


_SAMPLER_CHILD = r"""
import sys, time
import pynvml
pynvml.nvmlInit()
uuid, period = sys.argv[1], float(sys.argv[2])
h = pynvml.nvmlDeviceGetHandleByUUID(uuid) if uuid else pynvml.nvmlDeviceGetHandleByIndex(int(sys.argv[3]))
while True:
    try:
        r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
    except Exception:
        r = pynvml.nvmlDeviceGetCurrentClocksThrottleReasons(h)
    sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
    mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
    print(f"{time.time():.6f} {sm} {mx} {int(r)}", flush=True)
    time.sleep(period)
"""


class ClockSampler:
    """SM clock, max clock and clock-event reasons (read-only NVML queries)
    sampled every `period` seconds by a small child process, so the sampling
    does not compete for the interpreter with the bench's worker threads. It
    is started ahead of time (start()); the context manager marks the timed
    window and only samples inside it are kept. Falls back to a thread when
    the child cannot start."""

    def __init__(self, device_index: int, period: float = 0.01):
        self.period = period
        self.device_index = device_index
        self.samples: list[tuple[float, float, int]] = []
        self.error = None
        self._proc = None
        self._lines: list[str] = []
        self._reader = None
        self._t0 = self._t1 = None
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None

    @staticmethod
    def _uuid(device_index: int) -> str:
        try:
            import torch

            u = str(torch.cuda.get_device_properties(device_index).uuid)
            return u if u.startswith("GPU-") else "GPU-" + u
        except Exception:
            return ""

    def start(self):
        import subprocess

        try:
            self._proc = subprocess.Popen(
                [sys.executable, "-c", _SAMPLER_CHILD, self._uuid(self.device_index), str(self.period),
                 str(self.device_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._reader = threading.Thread(target=self._drain, daemon=True)
            self._reader.start()
            deadline = time.time() + 15.0
            while not self._lines and self._proc.poll() is None and time.time() < deadline:
                time.sleep(0.01)
            if not self._lines:
                raise RuntimeError("clock sampler produced no sample")
        except Exception as exc:
            self._stop_child()
            self.error = f"sampler process: {exc}"
            self._start_thread()
        return self

    def _drain(self):
        for line in self._proc.stdout:
            self._lines.append(line)

    def _stop_child(self):
        if self._proc is not None:
            if self._proc.poll() is None:
                self._proc.terminate()
                try:
                    self._proc.wait(timeout=5)
                except Exception:
                    self._proc.kill()
            self._proc = None

    # Thread fallback (NVML in-process).
    def _start_thread(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            self._nvml = pynvml
            uuid = self._uuid(self.device_index)
            self._handle = (pynvml.nvmlDeviceGetHandleByUUID(uuid) if uuid
                            else pynvml.nvmlDeviceGetHandleByIndex(self.device_index))
        except Exception as exc:
            self._nvml = None
            self.error = f"nvml unavailable: {exc}"
            return
        self._thread = threading.Thread(target=self._loop, daemon=True)
        self._thread.start()

    def _read(self):
        n = self._nvml
        sm = n.nvmlDeviceGetClockInfo(self._handle, n.NVML_CLOCK_SM)
        mx = n.nvmlDeviceGetMaxClockInfo(self._handle, n.NVML_CLOCK_SM)
        try:
            reasons = n.nvmlDeviceGetCurrentClocksEventReasons(self._handle)
        except Exception:
            reasons = n.nvmlDeviceGetCurrentClocksThrottleReasons(self._handle)
        return float(sm), float(mx), int(reasons)

    def _loop(self):
        while not self._stop.is_set():
            try:
                self._lines.append(f"{time.time():.6f} " + " ".join(str(int(v)) for v in self._read()))
            except Exception as exc:
                self.error = str(exc)
                return
            self._stop.wait(self.period)

    def __enter__(self):
        if self._proc is None and self._thread is None:
            self.start()
        self._t0 = time.time()
        return self

    def __exit__(self, *exc):
        self._t1 = time.time()
        time.sleep(2 * self.period)
        self._stop_child()
        self._stop.set()
        if self._thread is not None:
            self._thread.join()
        for line in list(self._lines):
            parts = line.split()
            if len(parts) != 4:
                continue
            t = float(parts[0])
            if self._t0 <= t <= self._t1:
                self.samples.append((float(parts[1]), float(parts[2]), int(parts[3])))

    def summary(self) -> dict:
        out = summarise_clocks(self.samples)
        if self.error:
            out["error"] = self.error
        return out


# ---------------------------------------------------------------- ranks --------


def rank_env() -> tuple[int, int, int]:
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar over the process group (identity without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(device=None) -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        if device is not None and device.type == "cuda":
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


def timed_steps(fn, steps: int, device) -> float:
    """Device milliseconds of `steps` calls of fn, barrier + synchronize on both
    sides, CUDA events on the current stream; max over ranks."""
    import torch

    barrier(device)
    torch.cuda.synchronize(device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize(device)
    barrier(device)
    return max_over_ranks(e0.elapsed_time(e1), device)


# ---------------------------------------------------------------- pieces -------


def load_peaks() -> tuple[dict, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def load_traffic(stage: str, size: int):
    """DRAM bytes per launch of the roofline kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        rows = json.loads(p.read_text())
    except ValueError:
        return None
    for row in rows:
        if row.get("stage") == stage:
            return float(row["bytes_per_px"]) * size * size
    return None


def drain_stage_seconds(ctx) -> dict:
    import ctypes

    from delta_b200 import _lib

    cap = 64
    labels = (ctypes.c_char * 64 * cap)()
    secs = (ctypes.c_double * cap)()
    n = ctypes.c_int()
    _lib.check(_lib.lib().dgpu_drain_timing(ctx.handle, labels, secs, cap, ctypes.byref(n)), ctx.handle)
    return {bytes(labels[i]).split(b"\0", 1)[0].decode(): float(secs[i]) for i in range(min(n.value, cap))}


def launch_count() -> int:
    import ctypes

    from delta_b200 import _lib

    c = ctypes.c_ulonglong()
    _lib.check(_lib.lib().dgpu_launch_count(ctypes.byref(c)))
    return int(c.value)


def pinned_copy(a):
    import torch

    t = torch.empty(a.shape, dtype=torch.from_numpy(a[:1].copy()).dtype, pin_memory=True)
    out = t.numpy()
    out[...] = a
    return out


def error_vs_fp64(out, ref) -> dict:
    """Errors of one precision's products against the FP64 normal-equation path."""
    th, th64 = np.asarray(out["solution"].theta), np.asarray(ref["solution"].theta)
    d = out["difference"].double().cpu().numpy()
    d64 = ref["difference"].double().cpu().numpy()
    v64 = ref["variance"].double().cpu().numpy()
    m64 = ref["mask"].cpu().numpy()
    good = (v64 > 0) & (m64 == 0) & np.isfinite(d) & np.isfinite(d64)
    z = (d - d64)[good] / np.sqrt(v64[good])
    s = out["score"].double().cpu().numpy()
    s64 = ref["score"].double().cpu().numpy()
    ok = np.isfinite(s) & np.isfinite(s64)
    cat, cat64 = out["catalog"], ref["catalog"]
    return {"theta_rel": float(np.linalg.norm(th - th64) / max(np.linalg.norm(th64), 1e-300)),
            "lambda_equal": bool(out["solution"].lam == ref["solution"].lam),
            "diff_rms_sigma": float(np.sqrt(np.mean(z * z))) if z.size else None,
            "diff_max_sigma": float(np.max(np.abs(z))) if z.size else None,
            "score_max_abs": float(np.max(np.abs(s - s64)[ok])) if ok.any() else None,
            "catalog_rows": [len(cat), len(cat64)]}


def error_vs_oracle(out, want) -> dict:
    """Errors of one GPU run's products against the oracle chain's on the same
    frame: theta, the (whitened) difference in units of the local sigma, the
    score, mask and CCL label equality (the reference's own CCL, compiled from
    source, run on both scores)."""
    from oracle import numpy_ref as nr
    from oracle import refbuild

    th, th0 = np.asarray(out["solution"].theta), np.asarray(want["fit"]["theta"])
    d = out["difference"].double().cpu().numpy()
    d0 = np.asarray(want["difference"], np.float64)
    v0 = np.asarray(want["variance"], np.float64)
    ok = (v0 > 0) & np.isfinite(d) & np.isfinite(d0)
    z = (d - d0)[ok] / np.sqrt(v0[ok])
    mask = out["mask"].cpu().numpy()
    s = out["score"].float().cpu().numpy()
    s0 = np.asarray(want["score"], np.float32)
    fin = np.isfinite(s) & np.isfinite(s0)
    lab = refbuild.label_components(nr.seed_mask(s, 5.0, +1, mask, True))[0]
    lab0 = refbuild.label_components(nr.seed_mask(s0, 5.0, +1, want["mask"], True))[0]
    return {"theta_rel": float(np.linalg.norm(th - th0) / max(np.linalg.norm(th0), 1e-300)),
            "lambda_equal": bool(out["solution"].lam == want["fit"]["lambda"]),
            "diff_rms_sigma": float(np.sqrt(np.mean(z * z))) if z.size else None,
            "diff_max_sigma": float(np.max(np.abs(z))) if z.size else None,
            "score_max_abs": float(np.max(np.abs(s.astype(np.float64) - s0)[fin])) if fin.any() else None,
            "mask_equal": bool(np.array_equal(mask, want["mask"])),
            "labels_equal": bool(np.array_equal(lab, lab0)), "components": int(lab0.max()),
            "catalog_rows": [len(out["catalog"]), len(want["catalog"]["x"])]}


def cpu_baseline(pair, size: int) -> tuple[dict, dict | None]:
    """The CPU chain on one full frame of the workload (rank 0, N=1); returns
    the baseline entry and the chain's products (the oracle for error_vs_oracle)."""
    from oracle import chain

    if not chain.available():
        return {"value": None, "unit": UNIT, "cores": None, "kind": "port",
                "unavailable": "oracle/_ref (the reference sources compiled by oracle/Makefile) is not built"}, None
    kw = subtract_kwargs(pair)
    kw.pop("saturation")
    t0 = time.perf_counter()
    stages: dict = {}
    want = chain.run(pair.science, pair.reference, pair.science_var, pair.reference_var, pair.science_mask,
                     pair.reference_mask, saturation=pair.saturation, timings=stages,
                     **{k: v for k, v in kw.items() if k not in ("precision",)})
    dt = time.perf_counter() - t0
    return {"value": size * size / 1e6 / dt, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"1 full {size}x{size} frame of the workload, one pass ({dt:.1f} s): {chain.DESCRIPTION}",
            "stage_seconds": {k: round(v, 3) for k, v in stages.items()}}, want


# ---------------------------------------------------------------- arms ---------


def run_reference(args) -> int:
    rank, world, _ = rank_env()
    if rank != 0:
        return 0
    from oracle import chain

    if not chain.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref is not built (make -C oracle ref)"}))
        return 0
    # Each step is one full frame of the same workload as the GPU arm (about
    # 7 s on 16 host cores), so both arms time the same configuration.
    size = args.size
    pair = make_frame(size, args.seed)
    kw = {k: v for k, v in subtract_kwargs(pair).items() if k != "saturation"}

    def step():
        chain.run(pair.science, pair.reference, pair.science_var, pair.reference_var, pair.science_mask,
                  pair.reference_mask, saturation=pair.saturation, **kw)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = args.steps * size * size / 1e6 / dt
    sample = f"one full {size}x{size} frame of the workload per step: {chain.DESCRIPTION}"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, **frame_config(args.size), "precision": "fp64 (CPU)",
                       "frames_per_rank": 1, "frames_in_flight": 1},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_gpu(args) -> int:
    import torch
    import torch.distributed as dist

    rank, world, local = rank_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (the product path has no CPU fallback)")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=device)

    import delta_b200 as delta
    from delta_b200 import _device, _lib
    from delta_b200.pipeline import Subtractor

    B = max(1, args.batch)
    size = args.size
    pairs = [make_frame(size, args.seed + rank * B + i) for i in range(B)]
    pair = pairs[0]
    frames = [_device.DeviceFrame.from_numpy(p.science, p.reference, p.science_var, p.reference_var, p.science_mask,
                                             p.reference_mask) for p in pairs]
    frame = frames[0]
    subs = {p: Subtractor(**subtract_kwargs(pair, p)) for p in ("mixed", "fp32", "fp64")}
    batch_subs = [Subtractor(**subtract_kwargs(p, "mixed")) for p in pairs]
    plain_subs = [Subtractor(**subtract_kwargs(p, "fp32")) for p in pairs]
    ctx = _lib.context()
    ex = _device.runner(B)

    def batch_step(subs_=batch_subs):
        futs = [ex.submit(_device.on_own_stream, _device.run, sb, f) for sb, f in zip(subs_, frames, strict=True)]
        for f in futs:
            f.result()

    # value: B frames in flight, mixed precision, layers resident in HBM.
    for _ in range(args.warmup):
        batch_step()
    torch.cuda.synchronize(device)
    clocks = ClockSampler(local).start()
    l0 = launch_count()
    with clocks:
        ms = timed_steps(batch_step, args.steps, device)
    launches = launch_count() - l0

    # one frame at a time, mixed: stage timers on for the roofline kernel.
    for _ in range(args.warmup):
        _device.run(subs["mixed"], frame)
    _lib.lib().dgpu_set_timing(ctx.handle, 1)
    drain_stage_seconds(ctx)
    ms_single = timed_steps(lambda: _device.run(subs["mixed"], frame), args.steps, device)
    stages = drain_stage_seconds(ctx)
    _lib.lib().dgpu_set_timing(ctx.handle, 0)

    # plain: FP32 normal equations, one frame at a time and B frames in flight
    for _ in range(args.warmup):
        _device.run(subs["fp32"], frame)
    ms_plain = timed_steps(lambda: _device.run(subs["fp32"], frame), args.steps, device)
    for _ in range(args.warmup):
        batch_step(plain_subs)
    ms_plain_batched = timed_steps(lambda: batch_step(plain_subs), args.steps, device)

    # end to end through the public batch API from pinned host arrays
    layer_names = ("science", "reference", "science_var", "reference_var", "science_mask", "reference_mask")
    host_items = [{k: pinned_copy(getattr(p, k)) for k in layer_names} for p in pairs]
    h2d = sum(a.nbytes for it in host_items for a in it.values())
    kw = subtract_kwargs(pair, "mixed")  # every frame of the generator has the same saturation level
    res_holder = {}

    def e2e_step():
        res_holder["r"] = delta.subtract_batch([dict(it) for it in host_items], max_in_flight=B, **kw)

    for _ in range(args.warmup):
        e2e_step()
    ms_e2e = timed_steps(e2e_step, args.steps, device)
    d2h = sum(a.nbytes for r in res_holder["r"] for a in (r.difference, r.variance, r.mask, r.score)
              if a is not None)
    # The same call from ordinary (pageable) NumPy arrays, as a caller without
    # pinned buffers would make it.
    page_items = [{k: np.array(getattr(p, k), copy=True) for k in layer_names} for p in pairs]

    def e2e_pageable_step():
        delta.subtract_batch([dict(it) for it in page_items], max_in_flight=B, **kw)

    for _ in range(max(1, args.warmup // 2)):
        e2e_pageable_step()
    ms_e2e_page = timed_steps(e2e_pageable_step, args.steps, device)

    # errors of mixed and plain against the FP64 normal-equation path (outside the timing)
    out64 = _device.run(subs["fp64"], frame)
    out_mixed = _device.run(subs["mixed"], frame)
    out_plain = _device.run(subs["fp32"], frame)
    errors = {"mixed": error_vs_fp64(out_mixed, out64), "plain": error_vs_fp64(out_plain, out64)}

    uneven = None
    if not args.no_uneven:
        uneven = uneven_batch(args, rank, world, device, precisions=("mixed", "fp32"))

    mpix = size * size / 1e6
    value = world * args.steps * B * mpix / (ms / 1e3)
    line = None
    if rank == 0:
        peaks, peak_kind = load_peaks()
        t_conv = stages.get(MODEL_CONVOLVE_STAGE)
        roofline = None
        sol = out64.get("solution")
        if t_conv and sol is not None:
            from delta_b200 import _core

            # The model convolve is FP32-FMA bound (about 68 FMA per HBM byte),
            # so its FP32 rate is the primary roofline; its HBM rate sits beside it.
            per_launch = t_conv / args.steps
            radius = int(_core._resolve_radius(float(sol.beta), int(sol.n_max), int(sol.radius)))
            fma = model_convolve_fma_per_px(int(sol.n_max), radius) * size * size
            tflops = 2.0 * fma / per_launch / 1e12
            peak_tflops = 2.0 * FP32_FMA_PEAK_TFMA
            bytes_launch = MODEL_CONVOLVE_BYTES_PER_PX * size * size
            gbs = bytes_launch / per_launch / 1e9
            roofline = {"bound": "fp32", "kernel": "k_model_convolve", "achieved": tflops, "peak": peak_tflops,
                        "unit": "TFLOP/s", "frac": tflops / peak_tflops,
                        "traffic": load_traffic(MODEL_CONVOLVE_STAGE, size),
                        "peak_source": "nominal FP32 (148 SMs x 128 lanes x 2 FLOP x 1.965 GHz); no measured FP32 peak",
                        "algorithmic_flop_per_launch": 2.0 * fma, "ms_per_launch": 1e3 * per_launch,
                        "timed_in": "the one-frame-at-a-time mixed pass",
                        "hbm": {"achieved": gbs, "peak": float(peaks["hbm_gbs"]), "unit": "GB/s",
                                "frac": gbs / float(peaks["hbm_gbs"]), "peak_source": peak_kind,
                                "algorithmic_bytes_per_launch": bytes_launch}}
        cpu, oracle_errors = None, None
        if world == 1 and not args.no_cpu_baseline:
            cpu, want = cpu_baseline(pair, size)
            if want is not None:
                oracle_errors = {"fp64": error_vs_oracle(out64, want),
                                 "mixed": error_vs_oracle(out_mixed, want),
                                 "plain": error_vs_oracle(out_plain, want)}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator of the workload)",
            "config": {"workload": WORKLOAD, **frame_config(size), "precision": "mixed", "frames_per_rank": B,
                       "frames_in_flight": B, "l2": "inputs larger than L2 (about 300 MB of layers per frame)"},
            "single": {"value": world * args.steps * mpix / (ms_single / 1e3), "ms_per_step": ms_single / args.steps,
                       "precision": "mixed", "frames_in_flight": 1},
            "plain": {"value": world * args.steps * mpix / (ms_plain / 1e3), "ms_per_step": ms_plain / args.steps,
                      "precision": "fp32", "frames_in_flight": 1},
            "plain_batched": {"value": world * args.steps * B * mpix / (ms_plain_batched / 1e3),
                              "ms_per_step": ms_plain_batched / args.steps, "precision": "fp32",
                              "frames_in_flight": B},
            "uneven": None if uneven is None else {"workload": UNEVEN_WORKLOAD, **uneven},
            "error_vs_fp64": errors,
            "error_vs_oracle": oracle_errors,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": world * args.steps * B * mpix / (ms_e2e / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e / args.steps,
                    "api": "delta_b200.subtract_batch", "inputs": "pinned host arrays"},
            "e2e_pageable": {"value": world * args.steps * B * mpix / (ms_e2e_page / 1e3), "unit": UNIT,
                             "ms_per_step": ms_e2e_page / args.steps, "inputs": "pageable NumPy arrays"},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "stage_ms_per_step": {k: round(1e3 * v / args.steps, 4) for k, v in sorted(stages.items())},
        }
    if world > 1:
        barrier(device)
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))
    return 0


def uneven_batch(args, rank: int, world: int, device, precisions=("mixed",), native: bool = True) -> dict:
    """The uneven batch through delta_b200's Subtractor.subtract (the call
    subtract_batch makes per frame) on `--batch` worker streams, from pinned
    host arrays; wall clock with a device synchronize and barrier on both
    sides, per precision; with `native`, also through the native batch
    scheduler with graph replay ("native_graphs"). Returns {name: stats}
    (rank 0's latencies)."""
    import torch

    from delta_b200 import _device, validation
    from delta_b200.pipeline import Subtractor

    specs = uneven_specs(args.seed)
    queue = uneven_queue(args.seed)
    owner = lpt_deal([specs[j]["height"] * specs[j]["width"] for j in queue], world)
    mine = [q for q in range(len(queue)) if owner[q] == rank]
    needed = sorted({queue[q] for q in mine})
    names = ("science", "reference", "science_var", "reference_var", "science_mask", "reference_mask")
    host = {}
    first = None
    for j in needed:
        sp = specs[j]
        p = validation.synthetic_pair(sp["width"], sp["height"], sp["n_stars"], sp["seed"], sci_fwhm=sp["sci_fwhm"],
                                      mask_fraction=sp["mask_fraction"])
        host[j] = {k: pinned_copy(getattr(p, k)) for k in names}
        first = first or p
    total_px = sum(specs[j]["height"] * specs[j]["width"] for j in queue)
    ex = _device.runner(max(1, args.batch))
    out = {}
    for prec in precisions:
        # Every frame of the generator has the same gain and saturation level.
        sub = Subtractor(**subtract_kwargs(first, prec)) if first is not None else None
        lat = {}

        def one(q, record):
            t0 = time.perf_counter()
            sub.subtract(**host[queue[q]])
            if record:
                lat[q] = (time.perf_counter() - t0) * 1e3

        warm: dict[int, int] = {}
        for q in mine:
            warm.setdefault(queue[q], q)
        # Untimed: each distinct frame once on the workers (workspace grows
        # stream-ordered inside the library, so no largest-frame-first warm-up
        # is needed to keep growth out of the timed pass).
        for f in [ex.submit(_device.on_own_stream, one, q, False) for q in warm.values()]:
            f.result()
        barrier(device)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        for f in [ex.submit(_device.on_own_stream, one, q, True) for q in mine]:
            f.result()
        torch.cuda.synchronize(device)
        wall = (time.perf_counter() - t0) * 1e3
        barrier(device)
        wall = max_over_ranks(wall, device)
        ls = sorted(lat.values())
        pct = (lambda f: ls[min(len(ls) - 1, int(round(f * (len(ls) - 1))))]) if ls else (lambda f: None)
        out[prec] = {"value": total_px / 1e6 / (wall / 1e3), "unit": UNIT, "wall_ms": wall, "frames": len(queue),
                     "latency_ms": {"p50": pct(0.5), "p99": pct(0.99), "max": ls[-1] if ls else None},
                     "frames_in_flight": max(1, args.batch), "precision": prec}
    if native:
        # The same queue through the native batch scheduler (dgpu_subtract_batch:
        # C++ workers over pooled contexts, longest frame first, each frame's
        # post-fit device work replayed as a recorded CUDA graph once its
        # worker has run that shape), from the same pinned host arrays.
        from delta_b200 import _core

        nkw = dict(n_max=6, n_knots=4, cv_folds=0, stamp_radius=15, threshold_sigma=5.0, decorrelate=True, score=True,
                   catalog=True, saturation=first.saturation if first is not None else 0.0, precision="mixed")
        B = max(1, args.batch)
        items = [host[queue[q]] for q in mine]
        # Products land in pinned host memory (one arena for the whole batch,
        # allocated before the timing; slices handed out inside it).
        need = sum(64 + 13 * it["science"].size for it in items) + 4096
        arena = torch.empty(need, dtype=torch.uint8, pin_memory=True).numpy()
        off = [0]

        def alloc(shape, dtype):
            nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
            o = (off[0] + 63) & ~63
            off[0] = o + nbytes
            return arena[o : o + nbytes].view(dtype).reshape(shape)

        _core.subtract_batch_native([host[j] for j in needed], frames_in_flight=B, graphs=True, alloc=alloc,
                                    **nkw)  # untimed
        off[0] = 0
        barrier(device)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        res = _core.subtract_batch_native(items, frames_in_flight=B, graphs=True, alloc=alloc, **nkw) if items else []
        torch.cuda.synchronize(device)
        wall = (time.perf_counter() - t0) * 1e3
        barrier(device)
        wall = max_over_ranks(wall, device)
        ls = sorted(r["seconds"] * 1e3 for r in res)
        pct = (lambda f: ls[min(len(ls) - 1, int(round(f * (len(ls) - 1))))]) if ls else (lambda f: None)
        out["native_graphs"] = {"value": total_px / 1e6 / (wall / 1e3), "unit": UNIT, "wall_ms": wall,
                                "frames": len(queue), "graph_replays": int(sum(r["graph_replayed"] for r in res)),
                                "latency_ms": {"p50": pct(0.5), "p99": pct(0.99), "max": ls[-1] if ls else None},
                                "frames_in_flight": B, "precision": "mixed",
                                "api": "delta_b200._core.subtract_batch_native (dgpu_subtract_batch, graphs on)"}
    return out


UNEVEN_WORKLOAD = ("64 frames: 16 distinct seeded frames of 2048x4096, 2048x2048, 1024x4096, each queued 4 times; "
                   "FWHM U(2,5), 500-20000 stars, 0-3% masked; n_max 6, 4x4 knots, GCV, decorrelate + score + CCL")


def run_uneven(args) -> int:
    import torch
    import torch.distributed as dist

    rank, world, local = rank_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (the product path has no CPU fallback)")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=device)
    both = uneven_batch(args, rank, world, device)
    stats = both["mixed"]
    if rank == 0:
        print(json.dumps({
            "metric": "uneven batch: aggregate Mpix/s over 64 frames of mixed sizes, end to end", "unit": UNIT,
            "value": stats["value"], "n_gpus": world, "frames": stats["frames"], "wall_ms": stats["wall_ms"],
            "latency_ms": {**stats["latency_ms"], "rank": 0}, "frames_in_flight": stats["frames_in_flight"],
            "higher_is_better": True, "scaling": "strong", "dtype": "f32", "data": "synthetic (seeded generator)",
            "native_graphs": both.get("native_graphs"),
            "config": {"workload": UNEVEN_WORKLOAD, "precision": "mixed",
                       "timing": "wall clock, device synchronize and barrier on both sides; untimed first: one "
                                 "pass over the distinct frames"}}), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def precision_study(seed: int = 0, size: int = 4096, n_stamps: int = 4200, n_max: int = 6, n_knots: int = 5,
                    stamp_radius: int = 15) -> dict:
    """Normal-equation arithmetic at the 725-unknown shape (n_max 6: 28
    components, 5 x 5 knots) over about 4e6 stamp rows of the 4096^2 field:
    FP32 SIMT, TF32 and BF16x3 tensor-core builds (the latter two with their
    FP64 refinement step, without and with the FP64 fallback) and the device
    FP64 path, each against the FP64
    oracle's fit of the same rows (oracle.numpy_ref.fit_kernel with the C GLS
    solve, B_n through the reference's own convolve.cpp). Reported per
    precision: ||theta - theta0|| / ||theta0||, the selected lambda, and the
    difference image and matched-filter score of its theta against those of
    the oracle's theta (RMS and max of dD / sigma, max |dscore|), where both
    images come from the same device subtraction so only theta differs."""
    import torch

    from delta_b200 import _core, _lib
    from oracle import cref, refbuild
    from oracle import numpy_ref as nr

    pair = make_frame(size, seed)
    edge = stamp_radius + 25
    xy, flux = pair.star_xy, pair.star_flux
    inside = (xy[:, 0] > edge) & (xy[:, 0] < size - 1 - edge) & (xy[:, 1] > edge) & (xy[:, 1] < size - 1 - edge)
    order = np.argsort(-flux[inside], kind="stable")
    pick = xy[inside][order][:n_stamps]
    sx = np.rint(pick[:, 0]).astype(np.int32)
    sy = np.rint(pick[:, 1]).astype(np.int32)
    sel = _core.select_stamps(pair.science, pair.reference, pair.science_mask, pair.reference_mask,
                              stamp_radius=stamp_radius, saturation=pair.saturation)
    beta = nr.default_beta(sel["median_fwhm_science"], sel["median_fwhm_reference"])
    knots = nr.grid_knots(0.0, 0.0, size - 1.0, size - 1.0, n_knots, n_knots)
    grid = np.logspace(-6.0, 6.0, 25)
    layers = dict(science_var=pair.science_var, reference_var=pair.reference_var, science_mask=pair.science_mask,
                  reference_mask=pair.reference_mask)
    r = nr.resolve_radius(beta, n_max, 0)
    t0 = time.perf_counter()
    want = nr.fit_kernel(pair.science, pair.reference, knots, sx, sy, stamp_radius, beta, n_max, grid, radius=r,
                         clip_iterations=0, basis_convolve_fn=lambda patch: refbuild.basis_convolve(patch, beta, n_max, r),
                         gcv_solver=cref.gls_gcv, **layers)
    oracle_s = time.perf_counter() - t0
    theta0 = np.asarray(want["theta"])
    sub0 = _core.subtract(pair.science, pair.reference, knots, theta0, beta, n_max, r, pair.saturation, **layers)
    var0 = sub0["variance"].astype(np.float64)
    good = (var0 > 0) & (sub0["mask"] == 0)
    psf = _core.estimate_psf(pair.science, sel["x"], sel["y"], 8)
    score0 = _core.matched_filter(sub0["difference"], psf, sub0["variance"]).astype(np.float64)
    out = {"P": int(theta0.size), "n_stamps": int(sx.size), "n_rows": int(want["n_pixels"]),
           "lambda_oracle": float(want["lambda"]), "oracle_seconds": round(oracle_s, 1), "modes": {}}
    ctx = _lib.context()
    # Each build's own error: the reduced-precision modes run without their
    # FP64 fallback ("tf32", "mixed"), then "mixed" once more as a fit runs by
    # default ("mixed+fallback": redone in FP64 when its refinement step shows
    # the BF16x3 system too far from the FP64 one).
    for mode in ("fp64", "fp32", "tf32", "mixed", "mixed+fallback"):
        prec = mode.split("+")[0]
        ctx.set_precision_fallback(mode.endswith("+fallback"))
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        try:
            got = _core.fit_kernel(pair.science, pair.reference, knots, sx, sy, stamp_radius, beta, n_max, grid,
                                   radius=r, clip_iterations=0, precision=prec, **layers)
        finally:
            ctx.set_precision_fallback(True)
        fit_ms = (time.perf_counter() - t1) * 1e3
        th = np.asarray(got["theta"])
        sub = _core.subtract(pair.science, pair.reference, knots, th, beta, n_max, r, pair.saturation, **layers)
        z = (sub["difference"].astype(np.float64) - sub0["difference"])[good] / np.sqrt(var0[good])
        sc = _core.matched_filter(sub["difference"], psf, sub["variance"]).astype(np.float64)
        fin = np.isfinite(sc) & np.isfinite(score0)
        out["modes"][mode] = {
            "theta_rel": float(np.linalg.norm(th - theta0) / np.linalg.norm(theta0)),
            "lambda_equal": bool(got["lambda"] == want["lambda"]), "precision_used": got["precision_used"],
            "refine_correction": float(got["refine_correction"]),
            "diff_rms_sigma": float(np.sqrt(np.mean(z * z))), "diff_max_sigma": float(np.max(np.abs(z))),
            "score_max_abs": float(np.max(np.abs(sc - score0)[fin])), "fit_wall_ms": round(fit_ms, 1)}
    return out


def run_precision(args) -> int:
    import torch

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (the product path has no CPU fallback)")
    rank, _, local = rank_env()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    study = precision_study(seed=args.seed, size=args.size)
    print(json.dumps({"metric": "normal-equation precision study (errors against the FP64 oracle)",
                      "config": {"workload": f"{args.size}x{args.size} spatially varying field, n_max 6, 5x5 knots, "
                                             "stamps of radius 15 at the brightest catalogue stars, GCV, one pass"},
                      **study}), flush=True)
    return 0


def run_grad(args) -> int:
    """Throughput of the gradient evaluations on the differentiation workload:
    8 fields of 2048 x 2048 (each its own seeded misregistration and scale),
    layers resident on the device. A step evaluates, on every field, chi^2 of
    the full-frame kernel model with its gradient in theta, (dx, dy) and the
    scale (dgpu_kernel_chi2) and the stamp-fit GCV with its gradient in
    (log lambda, dx, dy, scale) (dgpu_stamp_gcv). theta is the FP64 fit of
    each field's aligned exposure (n_max 6, 4 x 4 knots)."""
    import torch

    import delta_b200 as delta
    from delta_b200 import validation
    from delta_b200.autograd import KernelProblem, StampProblem

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (the product path has no CPU fallback)")
    rank, world, local = rank_env()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    size, n_fields = min(args.size, 2048), 8
    fields = []
    for i in range(n_fields):
        rng = np.random.default_rng(4000 + i)
        dx, dy = rng.uniform(-0.5, 0.5, 2)
        s = rng.uniform(0.8, 1.2)
        aligned = validation.synthetic_pair(size, size, 5000, 500 + i, mask_fraction=0.01)
        moved = validation.synthetic_pair(size, size, 5000, 500 + i, science_shift=(dx, dy), science_scale=s,
                                          mask_fraction=0.01)
        sol = delta.subtract(aligned.science, aligned.reference, science_var=aligned.science_var,
                             reference_var=aligned.reference_var, science_mask=aligned.science_mask,
                             reference_mask=aligned.reference_mask, n_max=6, n_knots=4, cv_folds=0, score=False,
                             decorrelate=False, saturation=aligned.saturation).solution
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        good = (moved.science_mask == 0) & (moved.reference_mask == 0)
        wt = np.where(good, 1.0 / (moved.science_var + moved.reference_var), 0.0).astype(np.float32)
        kp = KernelProblem(t(moved.science), t(wt), sol.knots, sol.beta, sol.n_max, sol.radius,
                           reference_mask=t(moved.reference_mask))
        sp = StampProblem(t(moved.science), t(moved.reference), sol.knots, sol.stamp_x, sol.stamp_y, 15, sol.beta,
                          sol.n_max, sol.radius, target_var=t(moved.science_var), convolved_var=t(moved.reference_var),
                          target_mask=t(moved.science_mask), convolved_mask=t(moved.reference_mask))
        fields.append((kp, sp, t(moved.reference), torch.tensor(np.asarray(sol.theta)), float(np.log(sol.lam))))
    z2 = torch.zeros(2, dtype=torch.float64)
    one = torch.ones((), dtype=torch.float64)

    def chi2_step():
        for kp, _, ref, th, _ in fields:
            kp.evaluate(th, z2, one, ref, grad=True)

    def gcv_step():
        for _, sp, _, _, ll in fields:
            sp.evaluate(torch.tensor(ll), z2, one, grad=True)

    out = {}
    for name, fn in (("chi2_grad", chi2_step), ("gcv_grad", gcv_step)):
        for _ in range(max(1, args.warmup)):
            fn()
        ms = timed_steps(fn, args.steps, dev)
        per_field = ms / args.steps / n_fields
        out[name] = {"ms_per_field": per_field, "fields_per_s": 1e3 / per_field,
                     "mpix_per_s": size * size / 1e6 / (per_field / 1e3)}
    print(json.dumps({"metric": "gradient evaluations on 8 fields of 2048x2048 (device-resident)", "unit": "ms/field",
                      "steps": args.steps, "warmup": args.warmup,
                      "config": {"workload": f"{n_fields} fields of {size}x{size}, n_max 6, 4x4 knots, chi^2 "
                                             "gradient in theta/shift/scale and GCV gradient in "
                                             "log lambda/shift/scale"}, **out}), flush=True)
    return 0


def main(argv=None) -> int:
    args = parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "uneven":
        return run_uneven(args)
    if args.workload == "precision":
        return run_precision(args)
    if args.workload == "grad":
        return run_grad(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
