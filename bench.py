"""Benchmark of the per-grain tracking path: grains per second per frame pair.

One step = one frame pair tracked through the whole per-frame pipeline of
particle_tracking (precompute, integer pixel + rotation search, subpixel
refinement, increments) for every grain of the workload.  Default workload:
the 16-bit 5616x3744 pair with 2000 bimodal grains (search +-15 px, 21
rotation steps), seeded synthetic data.

Forms, all on the same pair:
  headline  BF16 tensor-core candidate ranking (tcgen05) with exact integer
            rescoring of the kept candidates, then the adjoint
            Levenberg-Marquardt subpixel refinement;
  plain     exact integer search + FP64 Powell (the reference's method);
  exact_search+adjoint_lm.

  value  headline, device-resident: frames already in HBM, grain state
         restored on the device before each step; L2 flushed (256 MiB write)
         before every timed step; CUDA events on the context stream.
  e2e    headline through the C ABI with pinned host buffers: both frames and
         the grain records uploaded, the frame tracked, the records read back,
         every step; consecutive steps timed together, the next pair's frames
         handed over before the current pair's records are read back.
  roofline  k_search_bf16 timed with CUDA events between the search kernels
         (ptk_search_timed): 6 flops per pattern-pixel-candidate, against the
         measured dense BF16 peak; its tensor-core flops reported beside.

Multi-GPU (torchrun): one process per GPU; grains are independent, so each rank
tracks its own pair (different seed) with no data-path collective; time is the
max over ranks and value = all ranks' grains / that time ("scaling": "weak").

--impl reference runs the reference's own CPU implementation (compiled from its
sources into oracle/_ref, else the CPU port) on a bounded sample of the same
workload with all host threads (<= 48, the reference's MAX_NUMBER_THREADS).
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "grains/s per frame pair at <=0.01px vs FP64; plain vs BF16-search+adjoint-LM"
UNIT = "grains/s"
FLUSH_BYTES = 256 << 20


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def cpu_threads() -> int:
    try:
        n = len(os.sched_getaffinity(0))
    except Exception:
        n = os.cpu_count() or 1
    return max(1, min(48, n))


def rank_seed(rank: int) -> int:
    """Each rank tracks its own pair: grains are independent (weak scaling)."""
    return 1000 + rank


def reduce_max(values, world: int, device="cpu") -> list:
    """Max over ranks of per-rank timings (the only collective of the bench)."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def aggregate_rate(units_per_rank: int, world: int, ms_per_step: float) -> float:
    """Whole-job rate: units of all ranks over the slowest rank's step time."""
    return units_per_rank * world / (ms_per_step * 1e-3)


def ref_sample_size(n: int, threads: int) -> int:
    """Grains per timed step of the reference arm: 32 per host thread (so the
    reference's schedule(dynamic) OpenMP loops stay balanced over the bimodal
    radii), at most the whole workload."""
    return min(n, 32 * threads)


def baseline_sample_size(n: int, threads: int) -> int:
    """Grains of the one-off CPU baseline beside the GPU line: the whole
    workload when it is at most 200 grains per host thread (cfg2 on 16 host
    cores: all 2000 grains, about 17 s), else 200 per thread."""
    return n if n <= 200 * threads else 200 * threads


def pair_config(p: dict, n: int, zone, nsteps: int, world: int) -> dict:
    """The `config` of a frame-pair workload, the same for both arms."""
    return {"workload": f"{p['name']}: {p['dimx']}x{p['dimy']} {'u16' if p['maxval'] > 255 else 'u8'}, {n} grains "
                        f"per GPU, search +-{zone[0]} px, {nsteps} rotation steps",
            "grains_per_gpu": n, "l2": "flushed (256 MiB write) before each timed step",
            "parallelism": f"grain shards x{world}"}


def rotation_step_count(zone) -> int:
    """Steps of the reference's rotation loop (double accumulation)."""
    nsteps = 0
    drot = -abs(zone[5] * zone[4])
    while drot <= abs(zone[5] * zone[4]):
        nsteps += 1
        drot += zone[5]
    return nsteps


def sample_indices(n: int, k: int) -> np.ndarray:
    """Evenly spaced sample of k grains (keeps the radius mix)."""
    k = min(n, k)
    return np.unique(np.linspace(0, n - 1, k).round().astype(int))


def subset_pair(pair: dict, idx: np.ndarray) -> dict:
    out = dict(pair)
    out["rec"] = pair["rec"][idx]
    out["truth"] = pair["truth"][idx]
    return out


def cpu_track(pair: dict, wl, idx: np.ndarray, threads: int, steps: int = 1, warmup: int = 0):
    """Times the CPU checker (compiled reference when present) on a sample."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import bind
    kind = "reference" if bind.have_reference() else "port"
    if not bind.PORT_SO.exists():
        bind.build(ref=False)
    cls = bind.Reference if kind == "reference" else bind.Port
    sub = subset_pair(pair, idx)
    opts = wl.tracker_options(pair["params"])
    times = []
    for it in range(warmup + steps):
        t = bind.setup(cls, sub, threads=threads, zones=opts["zones"],
                       params={"rescue_level": opts["rescue_level"], "NCC_min": opts["NCC_min"], "iraz": 1 << 30})
        t0 = time.perf_counter()
        t.track_frame(1)
        dt = time.perf_counter() - t0
        if it >= warmup:
            times.append(dt)
        rec = t.get_grains()
        t.close()
    return kind, times, rec


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.proc = None
        self.out = None
        if gpu_id is None:
            return
        try:
            self.out = open(os.devnull if False else "/tmp/ptk_clocks.csv", "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", gpu_id], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        rows = []
        for line in open("/tmp/ptk_clocks.csv"):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smax=float(parts[2]), power=float(parts[3]),
                                 hw=parts[5], hwt=parts[6], swt=parts[7], swp=parts[8]))
            except ValueError:
                continue
        if not rows:
            return None
        load = [r for r in rows if r["power"] > 200.0] or rows
        reasons = set()
        for r in load:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                              ("swp", "sw_power_cap")):
                if r[key].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in load), "sm_max_mhz": max(r["smax"] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows), "samples_under_load": len(load)}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "bf16_tflops": d.get("bf16_tflops", 1590.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def recorded_traffic(summary: str):
    """DRAM bytes (read + write) per launch of a kernel on the default
    workload, as its committed ncu summary records them
    (`traffic_bytes_per_launch: N`); None when there is none."""
    import re
    p = ROOT / "profiles" / summary
    if not p.exists():
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", p.read_text())
    return float(m.group(1)) if m else None


def search_ppc(tracker, rec: np.ndarray, zone, nsteps: int) -> int:
    """Pattern-pixel-candidate evaluations of one pixel-stage search."""
    P = sum(tracker.pattern_size(g) for g in range(rec.shape[0]))
    left, right, up, down = zone[:4]
    return P * nsteps * (left + right + 1) * (up + down + 1)


def run_reference_arm(args, rank: int, world: int):
    if rank != 0:
        return 0
    wl = importlib.import_module("p-tracker_b200.workloads")
    pair = wl.make_pair(args.workload, seed=rank_seed(rank))
    n = pair["rec"].shape[0]
    threads = cpu_threads()
    idx = sample_indices(n, args.ref_sample if args.ref_sample > 0 else ref_sample_size(n, threads))
    kind, times, _ = cpu_track(pair, wl, idx, threads, steps=args.steps, warmup=args.warmup)
    per_step = statistics.mean(times)
    value = len(idx) / per_step
    zone = wl.tracker_options(pair["params"])["zones"][0]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": pair_config(dict(pair["params"], name=args.workload), n, zone, rotation_step_count(zone), world),
        "form": "the reference's own CPU path (precompute, exact pixel search, Powell subpixel), OpenMP",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{len(idx)} of {n} grains ({len(idx) / threads:.0f} per host thread, evenly "
                                   f"spaced over the radius mix), the whole frame pipeline per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


DISTO_METRIC = "equiprojectivity residuals/s (distortion-fit objective)"
DISTO_UNIT = "residuals/s"


def _disto_setup(ptk, wl, seed: int):
    case = wl.make_disto_case(seed)
    pairs = ptk.disto_pairs(case["refx"], case["refy"], 0.0, 1000.0)  # equiProj_dist_range defaults
    X0 = case["X"].copy()
    X0[2] = X0[3] = 0.0  # centres at the frame centre, no distortion
    return case, pairs, X0


def _disto_cpu(case, pairs, X0, reference: bool, budget_s: float = 10.0):
    """Seconds per objective evaluation of the CPU checker (single-threaded,
    as the reference's objective loop): the oracle restatement, or the loop
    around the reference's own undistor."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import bind
    if not reference and not bind.PORT_SO.exists():
        bind.build(ref=False)
    times, v = [], None
    while not times or (sum(times) < budget_s and len(times) < 5):
        t0 = time.perf_counter()
        v = bind.disto_objective(X0, case["refx"], case["refy"], case["dx"], case["dy"], case["ncc"], 0.7, pairs,
                                 reference=reference)
        times.append(time.perf_counter() - t0)
    return statistics.mean(times), v, len(times)


def run_disto(args, rank: int, world: int, local: int) -> int:
    """Distortion-parameter fit workload (correction_distortion's
    minimisation): 2000 grains of a 5616x3744 frame tracked into 3 images,
    pairs 0..1000 px apart (268,944 pairs, 806,832 residuals per objective
    evaluation).  One step = one objective evaluation.  A fit is one small
    problem, so N > 1 runs nothing on ranks other than 0 (replicas only).

      value  device time of the objective's kernels (per-point undistortion,
             pair residuals, fixed-order sum), inputs resident, L2 flushed
             before every step (the inputs are smaller than L2);
      e2e    ptk_disto_objective from the host: parameters in, value out;
      fit    one POWELL fit of K1 and K2 through ptk_disto_fit, wall time."""
    if rank != 0:
        return 0
    import torch
    torch.cuda.set_device(local)
    ptk = importlib.import_module("p-tracker_b200")
    wl = importlib.import_module("p-tracker_b200.workloads")
    case, pairs, X0 = _disto_setup(ptk, wl, seed=rank_seed(rank))
    n, nimg1, P = case["refx"].shape[0], case["dx"].shape[0], pairs.shape[0]
    m = nimg1 * P
    if args.impl == "reference":
        sec, _, k = _disto_cpu(case, pairs, X0, reference=True)
        line = {"metric": DISTO_METRIC, "value": m / sec, "unit": DISTO_UNIT, "n_gpus": world, "steps": k,
                "warmup": 0, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "replicas",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": f"disto: {n} grains of a 5616x3744 frame, {nimg1} tracked images, {P} "
                                       f"pairs 0..1000 px apart, {m} residuals per evaluation"},
                "cpu_baseline": {"value": m / sec, "unit": DISTO_UNIT, "cores": 1, "kind": "reference",
                                 "sample": f"{k} objective evaluations"},
                "e2e": {"value": m / sec, "unit": DISTO_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    fit = ptk.DistoFit(case["dimx"], case["dimy"], case["refx"], case["refy"], case["dx"], case["dy"], case["ncc"],
                       0.7, pairs)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    try:
        pr = torch.cuda.get_device_properties(local)
        gpu_id = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
    except Exception:
        gpu_id = str(local)
    sampler = ClockSampler(gpu_id)
    # the timed steps last well under the sampler's 200 ms period: the clocks
    # are sampled over a warm-up of at least 1.5 s of evaluations before them
    t_w = time.perf_counter()
    k = 0
    while k < args.warmup or time.perf_counter() - t_w < 1.5:
        fit.objective_timed(X0, 200)
        k += 1
    ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ms.append(fit.objective_timed(X0, 1))
    ms_step = statistics.mean(ms)
    clocks = sampler.stop()
    gpu_value = fit.objective(X0)
    e2e = []
    for it in range(args.warmup + max(args.e2e_steps, args.steps)):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fit.objective(X0)
        if it >= args.warmup:
            e2e.append(time.perf_counter() - t0)
    e2e_ms = statistics.mean(e2e) * 1e3
    DX = np.zeros(14)
    DX[2], DX[3] = 1e-10, 1e-17
    t0 = time.perf_counter()
    x, ini, end, _ = fit.fit(X0, DX, ptk.DISTO_POWELL)
    fit_s = time.perf_counter() - t0
    fit.close()
    # compulsory bytes of one evaluation after an L2 flush: the pair list, the
    # per-(image, grain) inputs, the undistorted points written and read back
    alg_bytes = 8 * P + (8 + 16) * nimg1 * n + 8 * n + 2 * 16 * (nimg1 + 1) * n
    peaks = measured_peaks()
    achieved = alg_bytes / (ms_step * 1e-3) / 1e9
    line = {
        "metric": DISTO_METRIC, "value": m / (ms_step * 1e-3), "unit": DISTO_UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "replicas", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"disto: {n} grains of a 5616x3744 frame, {nimg1} tracked images, {P} pairs "
                               f"0..1000 px apart, {m} residuals per evaluation",
                   "l2": "flushed (256 MiB write) before each timed step",
                   "clocks": "sampled over 1.5 s of evaluations right before the timed steps"},
        "e2e": {"value": m / (e2e_ms * 1e-3), "unit": DISTO_UNIT, "h2d_bytes_per_step": 14 * 8,
                "d2h_bytes_per_step": 8, "ms_per_step": e2e_ms},
        "gpu_launches": 2 * args.steps,
        "roofline": {"kernel": "k_disto_points + k_disto_residuals (one evaluation)", "bound": "hbm",
                     "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": None, "algorithmic_bytes_per_launch": alg_bytes,
                     "peak_source": peaks["source"] + " copy bandwidth"},
        "fit": {"algo": "POWELL over K1, K2", "seconds": fit_s, "index_ini": ini, "index_end": end,
                "K1": x[2], "K2": x[3], "K1_rendered": case["X"][2], "K2_rendered": case["X"][3]},
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        sec, cpu_v, k = _disto_cpu(case, pairs, X0, reference=False)
        line["cpu_baseline"] = {"value": m / sec, "unit": DISTO_UNIT, "cores": 1, "kind": "port",
                                "sample": f"{k} full objective evaluations"}
        line["accuracy"] = {"objective_rel_diff_vs_oracle": abs(gpu_value - cpu_v) / cpu_v}
    print(json.dumps(line), flush=True)
    return 0


RAW_METRIC = "RAW frames demosaiced/s (5616x3744, DemosaicModel -2 + rescaleGrayLevels)"
RAW_UNIT = "frames/s"


def run_raw(args, rank: int, world: int, local: int) -> int:
    """RAW ingest workload: a 5616x3744 frame in a 5680x3760 16-bit sensor
    mosaic (margins 24 / 8), DemosaicModel -2 (3x3 binomial) with the grey
    rescale, into a frame slot of the context.  One step = one frame.  Frames
    are independent: N > 1 runs nothing on ranks other than 0 (replicas).

      value  ptk_load_frame_raw_device on a device-resident mosaic: the
             demosaic pass (with MinGray/MaxGray) and the rescale pass, CUDA
             events on the context stream, L2 flushed before each step;
      e2e    ptk_load_frame_raw from a pinned host mosaic (upload included)
             returning MinGray/MaxGray to the host."""
    if rank != 0:
        return 0
    import torch
    torch.cuda.set_device(local)
    ptk = importlib.import_module("p-tracker_b200")
    W, H, RW, RH, L, T, MODE = 5616, 3744, 5680, 3760, 24, 8, -2
    rng = np.random.default_rng(rank_seed(rank))
    raw = rng.integers(0, 16384, (RH, RW)).astype(np.uint16)
    raw_pin = torch.from_numpy(raw.view(np.int16)).pin_memory()
    if args.impl == "reference":
        sys.path.insert(0, str(ROOT / "oracle"))
        import bind
        ref = bind.have_reference()
        times = []
        for _ in range(max(1, min(args.steps, 5))):
            t0 = time.perf_counter()
            bind.raw_demosaic(raw, W, H, L, T, MODE, True, reference=ref)
            times.append(time.perf_counter() - t0)
        sec = statistics.mean(times)
        line = {"metric": RAW_METRIC, "value": 1.0 / sec, "unit": RAW_UNIT, "n_gpus": world, "steps": len(times),
                "warmup": 0, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "replicas",
                "vs_baseline": None, "dtype": "u16", "data": "synthetic", "impl": "reference",
                "config": {"workload": "raw: 5616x3744 frame of a 5680x3760 u16 mosaic, mode -2, rescale"},
                "cpu_baseline": {"value": 1.0 / sec, "unit": RAW_UNIT, "cores": 1,
                                 "kind": "reference" if ref else "port", "sample": f"{len(times)} whole frames"},
                "e2e": {"value": 1.0 / sec, "unit": RAW_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    stream = torch.cuda.Stream()
    t = ptk.Tracker(W, H)
    t.set_stream(stream.cuda_stream)
    d_raw = raw_pin.cuda()
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    try:
        pr = torch.cuda.get_device_properties(local)
        gpu_id = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
    except Exception:
        gpu_id = str(local)
    with torch.cuda.stream(stream):
        sampler = ClockSampler(gpu_id)
        t_w = time.perf_counter()
        k = 0
        while k < args.warmup or time.perf_counter() - t_w < 1.5:  # clocks sampled over >= 1.5 s of frames
            t.load_frame_raw_device(0, d_raw.data_ptr(), RW, RH, L, T, MODE, True)
            stream.synchronize()
            k += 1
        ms = []
        l0 = t.launches()
        for _ in range(args.steps):
            flush.zero_()
            stream.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t.load_frame_raw_device(0, d_raw.data_ptr(), RW, RH, L, T, MODE, True)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        launches = t.launches() - l0
        clocks = sampler.stop()
        e2e = []
        for it in range(args.warmup + max(args.e2e_steps, args.steps)):
            flush.zero_()
            stream.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            mm = t.load_frame_raw(0, raw_pin.numpy().view(np.uint16), L, T, MODE, True)
            e1.record(stream)
            e1.synchronize()
            if it >= args.warmup:
                e2e.append(e0.elapsed_time(e1))
        frame = t.read_frame(0)
    t.close()
    ms_step, e2e_ms = statistics.mean(ms), statistics.mean(e2e)
    alg_bytes = 2 * W * H * 2 + 2 * W * H * 2  # demosaic: mosaic read + frame write; rescale: frame read + write
    peaks = measured_peaks()
    achieved = alg_bytes / (ms_step * 1e-3) / 1e9
    line = {
        "metric": RAW_METRIC, "value": 1e3 / ms_step, "unit": RAW_UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "replicas",
        "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": f"raw: {W}x{H} frame of a {RW}x{RH} u16 mosaic (margins {L}/{T}), DemosaicModel "
                               f"{MODE}, rescaleGrayLevels", "l2": "flushed (256 MiB write) before each timed step",
                   "clocks": "sampled over 1.5 s of frames right before the timed steps"},
        "e2e": {"value": 1e3 / e2e_ms, "unit": RAW_UNIT, "h2d_bytes_per_step": int(raw.nbytes),
                "d2h_bytes_per_step": 8, "ms_per_step": e2e_ms},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "k_raw_demosaic + k_raw_rescale (one frame)", "bound": "hbm", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                     "algorithmic_bytes_per_launch": alg_bytes, "peak_source": peaks["source"] + " copy bandwidth"},
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import bind
        if not bind.PORT_SO.exists():
            bind.build(ref=False)
        t0 = time.perf_counter()
        want, mm_want = bind.raw_demosaic(raw, W, H, L, T, MODE, True)
        sec = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": 1.0 / sec, "unit": RAW_UNIT, "cores": 1, "kind": "port",
                                "sample": "one whole frame"}
        line["accuracy"] = {"frame_equal_to_oracle": bool(np.array_equal(frame, want)),
                            "min_max_equal_to_oracle": list(mm) == list(mm_want)}
    print(json.dumps(line), flush=True)
    return 0


def run_sequence(args, rank: int, world: int, local: int) -> int:
    """Full-sequence workload (cfg5): every frame of the sequence is brought
    into the current slot, resampled by the on-device lens-distortion remap and
    tracked (BF16 search + adjoint LM, +-40 px rescue, reference change after
    every frame).  value: grains x frames per second with the frames resident
    in HBM (each step copies its frame into the context slot); e2e: frames
    uploaded from pinned host memory and the records read back every step."""
    import torch
    ptk = importlib.import_module("p-tracker_b200")
    wl = importlib.import_module("p-tracker_b200.workloads")
    torch.cuda.set_device(local)
    s = wl.make_sequence(args.workload, seed=rank_seed(rank))
    p = s["params"]
    frames = s["frames"]
    nf = len(frames)
    n = s["rec"].shape[0]
    o = wl.tracker_options(p)
    stream = torch.cuda.Stream()
    dev = [torch.from_numpy(f.view(np.int16)).to("cuda") for f in frames]
    pinned = [torch.from_numpy(f).pin_memory().numpy() for f in frames]

    def tracker(**form):
        t = ptk.Tracker(p["dimx"], p["dimy"], rescue_level=o["rescue_level"], NCC_min=o["NCC_min"], iraz=0, **form)
        t.set_stream(stream.cuda_stream)
        for lvl, z in enumerate(o["zones"]):
            if z is not None:
                t.set_zone(lvl, *z)
        t.set_grains(s["rec"])
        t.make_patterns("grain_diameter", 1.0, 1.0)
        t.set_distortion(s["disto"])
        return t

    def device_run(t):
        t.set_grains(s["rec"])
        t.set_iref(0)
        t.load_frame_device(0, dev[0].data_ptr(), p["dimx"] * 2)
        t.remap(0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        stream.synchronize()
        e0.record(stream)
        for k in range(1, nf):
            t.load_frame_device(1, dev[k].data_ptr(), p["dimx"] * 2)
            t.remap(1)
            t.track_frame(k)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / (nf - 1)

    def host_run(t):
        t.set_grains(s["rec"])
        t.set_iref(0)
        t.load_frame(0, pinned[0])
        t.remap(0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        stream.synchronize()
        e0.record(stream)
        # the next frame is handed over before the current one's records are
        # read back: its upload (into the old reference's buffer) overlaps the
        # tracking from the end of the precompute on
        t.load_frame(1, pinned[1])
        for k in range(1, nf):
            t.remap(1)
            t.track_frame(k)
            if k + 1 < nf:
                t.load_frame(1, pinned[k + 1])
            out = t.get_grains()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / (nf - 1), out

    # the CPU reference's sample through the sequence: 20 grains per host thread, so that its
    # schedule(dynamic) loops stay balanced (320 of 5000 grains on 16 threads, about 2 min per pass)
    idx = sample_indices(n, args.cpu_sample if args.cpu_sample > 0 else min(n, 20 * cpu_threads()))
    levels = range(o["rescue_level"] + 1)

    def pos(rec):  # positions and rotations: refcoord + d (a reference change may split them differently)
        return np.stack([rec[:, 0] + rec[:, 4], rec[:, 1] + rec[:, 5], rec[:, 2] + rec[:, 6]], 1)

    def lockstep(t):
        """One-step parity along the plain trajectory: every frame is tracked
        by the headline form and by the plain form from the same grain state,
        and the plain result carries the sequence on.  Returns the largest
        differences, the sampled grains' states and results per frame, and the
        remapped frames (the device remap is bit-exact to the oracle's)."""
        t.set_grains(s["rec"])
        t.set_iref(0)
        t.load_frame_device(0, dev[0].data_ptr(), p["dimx"] * 2)
        t.remap(0)
        remapped = [t.read_frame(0)]
        worst = np.zeros(3)
        over = 0
        over_closer = 0  # of those: the headline no farther from the synthetic truth than the plain form
        per = []
        eh, ep = [], []  # one-step position errors against the synthetic motion, per grain-frame
        rh_rad, rp_rad = [], []
        for k in range(1, nf):
            t.load_frame_device(1, dev[k].data_ptr(), p["dimx"] * 2)
            t.remap(1)
            remapped.append(t.read_frame(1))
            t.precompute()
            t.snapshot_grains()
            before = t.get_grains()
            t.configure(search_method=ptk.SEARCH_BF16, subpix_method=ptk.SUBPIX_ADJOINT_LM)
            for lvl in levels:
                t.search(lvl)
            t.subpixel(ptk.SUBPIX_ADJOINT_LM)
            rh = t.get_grains()
            t.restore_grains()
            t.configure(search_method=ptk.SEARCH_EXACT, subpix_method=ptk.SUBPIX_POWELL)
            for lvl in levels:
                t.search(lvl)
            t.subpixel(ptk.SUBPIX_POWELL)
            rp = t.get_grains()
            t.end_frame(k)
            d = np.abs(rh[:, 4:7] - rp[:, 4:7])
            worst = np.maximum(worst, [d[:, 0].max(), d[:, 1].max(), d[:, 2].max()])
            # The step's dx, dy is the displacement of the pattern anchored at the
            # integer refcoord of the reference frame (the reference's pixel search
            # restarts from round(dx) and drops its fraction, src/p-tracker.cpp:666-669,
            # 739): its truth is that material point's motion from frame k - 1 to k,
            # the grain's translation plus the rotation increment about its centre.
            m0, m1 = s["motion"][k - 1], s["motion"][k]
            at_k1 = {"cx": s["grains"]["cx"] + m0[0], "cy": s["grains"]["cy"] + m0[1]}
            tr = wl.anchor_truth(at_k1, before, m1[0] - m0[0], m1[1] - m0[1], m1[2] - m0[2])
            eh.append(np.abs(rh[:, 4:6] - tr[:, :2]).max(1))
            ep.append(np.abs(rp[:, 4:6] - tr[:, :2]).max(1))
            e_h, e_p = eh[-1], ep[-1]
            rh_rad.append(np.abs(rh[:, 6] - tr[:, 2]))
            rp_rad.append(np.abs(rp[:, 6] - tr[:, 2]))
            big = d[:, :2].max(1) > 0.01
            over += int(big.sum())
            over_closer += int((big & (e_h <= e_p)).sum())
            per.append((before[idx], rh[idx], rp[idx]))
        return {"worst": worst, "over": over, "over_closer": over_closer, "per": per, "remapped": remapped,
                "truth_h": np.concatenate(eh), "truth_p": np.concatenate(ep),
                "truth_h_rad": np.concatenate(rh_rad), "truth_p_rad": np.concatenate(rp_rad)}

    try:
        pr = torch.cuda.get_device_properties(local)
        gpu_id = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
    except Exception:
        gpu_id = str(local)
    with torch.cuda.stream(stream):
        head = tracker(search_method=ptk.SEARCH_BF16, subpix_method=ptk.SUBPIX_ADJOINT_LM)
        for _ in range(max(1, args.warmup // 3)):
            device_run(head)
        sampler = ClockSampler(gpu_id if rank == 0 else None)
        ms_head = min(device_run(head) for _ in range(max(1, args.steps // 5)))
        clocks = sampler.stop()
        head_rec = head.get_grains()
        res_counts = head.rescue_counts()
        # the undistortion remap of one frame (map gather + cubic, copy back), L2 flushed before each
        flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
        rm = []
        for it in range(6):
            flush.zero_()
            head.load_frame_device(1, dev[1].data_ptr(), p["dimx"] * 2)
            stream.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            head.remap(1)
            e1.record(stream)
            e1.synchronize()
            if it > 0:
                rm.append(e0.elapsed_time(e1))
        del flush
        e2e_ms, _ = host_run(head)
        plain = tracker()
        device_run(plain)
        ms_plain = device_run(plain)
        plain_rec = plain.get_grains()
        step = lockstep(plain) if rank == 0 else None

    if rank == 0:
        block = 16 * 8 * n + 2 * 8 * n + ((12 * n + 15) // 16) * 16 + ((2 * n + 15) // 16) * 16
        line = {
            "metric": METRIC, "value": n * world / (ms_head * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": nf - 1, "warmup": max(1, args.warmup // 3), "ms_per_step": ms_head, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 ranking (f32 accumulate) + int64 exact rescoring + f32/f64 adjoint LM", "data": "synthetic",
            "config": {"workload": f"{args.workload}: {nf} frames {p['dimx']}x{p['dimy']} u16, {n} grains, "
                                   f"search +-{p['zone']} px, rescue +-{p['rescue_zone']} px, lens distortion "
                                   f"remapped on device, reference change every frame",
                       "form": "BF16 tensor-core search + exact rescoring + adjoint LM",
                       "step": "one frame: copy into the current slot, remap, track",
                       "l2": "a new 42 MB frame per step"},
            "e2e": {"value": n * world / (e2e_ms * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": int(frames[0].nbytes), "d2h_bytes_per_step": int(block)},
            "forms": {"plain": {"value": n * world / (ms_plain * 1e-3), "ms_per_step": ms_plain},
                      "speedup_headline_vs_plain": ms_plain / ms_head},
            "accuracy": {"one_step_max_abs_err_px_vs_plain": float(step["worst"][:2].max()),
                         "one_step_max_abs_err_rad_vs_plain": float(step["worst"][2]),
                         "one_step_grain_frames_over_0.01px_vs_plain": step["over"],
                         "one_step_over_0.01px_headline_no_farther_from_truth": step["over_closer"],
                         "one_step_median_abs_err_px_vs_truth": float(np.median(step["truth_h"])),
                         "one_step_max_abs_err_px_vs_truth": float(step["truth_h"].max()),
                         "plain_one_step_median_abs_err_px_vs_truth": float(np.median(step["truth_p"])),
                         "plain_one_step_max_abs_err_px_vs_truth": float(step["truth_p"].max()),
                         "one_step_median_abs_err_rad_vs_truth": float(np.median(step["truth_h_rad"])),
                         "plain_one_step_median_abs_err_rad_vs_truth": float(np.median(step["truth_p_rad"])),
                         "truth_note": "one-step dx, dy against the motion of the material point at the integer "
                                       "refcoord (the reference's definition of dx after a reference change); "
                                       "maxima include grains that are lost",
                         "grain_frames": n * (nf - 1),
                         "trajectory_max_abs_dev_px_vs_plain_after_sequence":
                         float(np.abs(pos(head_rec)[:, :2] - pos(plain_rec)[:, :2]).max()),
                         "rescued_last_frame": int(res_counts[0]), "jumping_grains": int(s["jumpers"].sum())},
            "clocks": clocks,
            "remap": {"ms": statistics.median(rm),
                      # map 16 B + output 2 B + copy back 2 + 2 B per pixel; the 4x4 source gathers hit L2
                      "algorithmic_gb_s": 22.0 * p["dimx"] * p["dimy"] / (statistics.median(rm) * 1e-3) / 1e9},
        }
        if not args.no_cpu_baseline:
            sys.path.insert(0, str(ROOT / "oracle"))
            import bind
            kind = "reference" if bind.have_reference() else "port"
            cls = bind.Reference if kind == "reference" else bind.Port
            threads = cpu_threads()
            remapped = step["remapped"]
            pair = dict(params=p, ref=remapped[0], cur=remapped[1], rec=s["rec"][idx])
            c = bind.setup(cls, pair, threads=threads, zones=o["zones"],
                           params={"rescue_level": o["rescue_level"], "NCC_min": o["NCC_min"], "iraz": 0})
            t0 = time.perf_counter()
            for k in range(1, nf):
                if k > 1:
                    c.load_current(remapped[k])
                c.track_frame(k)
            dt = time.perf_counter() - t0
            cr_seq = c.get_grains()
            c.close()
            line["cpu_baseline"] = {"value": len(idx) / (dt / (nf - 1)), "unit": UNIT, "cores": threads, "kind": kind,
                                    "sample": f"{len(idx)} of {n} grains (evenly spaced) through all {nf} frames"}
            # one step of the FP64 reference from the plain trajectory's state, every frame
            wh, wp = np.zeros(3), np.zeros(3)
            for k in range(1, nf):
                before, rh, rp = step["per"][k - 1]
                c = cls(p["dimx"], p["dimy"], threads)
                c.load_reference(remapped[k - 1])
                c.load_current(remapped[k])
                c.set_grains(before)
                c.grain_diameter_patterns(before, 1.0, 1.0)
                for lvl, z in enumerate(o["zones"]):
                    if z is not None:
                        c.set_zone(lvl, *z)
                for key, v in (("rescue_level", o["rescue_level"]), ("NCC_min", o["NCC_min"]), ("iraz", 0)):
                    c.set_param(key, v)
                c.precompute()
                c.pixel_all()
                if o["rescue_level"] >= 1:
                    c.rescue_all()
                c.subpixel_all()
                cr = c.get_grains()
                c.close()
                wh = np.maximum(wh, np.abs(rh[:, 4:7] - cr[:, 4:7]).max(0))
                wp = np.maximum(wp, np.abs(rp[:, 4:7] - cr[:, 4:7]).max(0))
            line["accuracy"]["one_step_max_abs_err_px_vs_fp64_reference"] = float(wh[:2].max())
            line["accuracy"]["one_step_max_abs_err_rad_vs_fp64_reference"] = float(wh[2])
            line["accuracy"]["plain_one_step_max_abs_err_px_vs_fp64_reference"] = float(wp[:2].max())
            line["accuracy"]["plain_one_step_max_abs_err_rad_vs_fp64_reference"] = float(wp[2])
            line["accuracy"]["fp64_reference_sample"] = f"{len(idx)} grains x {nf - 1} frames"
            d = np.abs(pos(plain_rec[idx]) - pos(cr_seq))
            line["accuracy"]["plain_trajectory_max_abs_dev_px_vs_fp64_reference"] = float(d[:, :2].max())
        print(json.dumps(line), flush=True)
    head.close()
    plain.close()
    return 0


def gemm_flops(rec: np.ndarray, inc_rot: float = 0.005, num_rot: int = 10) -> float:
    """Tensor-core flops of one BF16 search launch over the 32x32 candidate
    tile of each grain: per footprint row, the 16-column chunks that touch a
    block holding a point of some rotation step, 2 MMAs each (cross terms and
    second moments) of M=128 (4 x-shifts x 32 rotation slots) x N=256 x K=16,
    rotation-slot and chunk padding included (grain_diameter 1.0 discs at
    reference rotation 0, rotated as rotate_pixel_pattern rotates them)."""
    rotmax = abs(inc_rot * num_rot)
    steps, a = [], -rotmax
    while a <= rotmax:
        steps.append(a)
        a += inc_rot
    per_radius = {}
    total = 0.0
    for r in rec[:, 3]:
        R = max(int(r), 1)
        if R not in per_radius:
            half = R + 1
            fw = 2 * half + 1
            nbf = (fw + 7) // 8
            nch = (nbf + 4) // 2
            yy, xx = np.mgrid[-R:R + 1, -R:R + 1]
            inside = xx * xx + yy * yy <= R * R
            px, py = xx[inside].astype(float), yy[inside].astype(float)
            lo = np.full(fw, 10 ** 6)
            hi = np.full(fw, -1)
            for t in steps:
                c, sn = np.cos(t), np.sin(t)
                qx = np.sign(c * px + sn * py) * np.floor(np.abs(c * px + sn * py) + 0.5)
                qy = np.sign(-sn * px + c * py) * np.floor(np.abs(-sn * px + c * py) + 0.5)
                row = (qy + half).astype(int)
                blk = ((qx + half).astype(int)) // 8
                np.minimum.at(lo, row, blk)
                np.maximum.at(hi, row, blk)
            n = 0
            for y in range(fw):
                if hi[y] >= 0:
                    n += max(0, min(nch - 1, (hi[y] + 3) // 2) - lo[y] // 2 + 1)
            per_radius[R] = n
        total += per_radius[R] * 2 * 2.0 * 128 * 256 * 16
    return total


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg2")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--ref-sample", type=int, default=0, help="grains per reference-arm step (0: 32 per host thread)")
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="grains of the CPU baseline (0: all, up to 200 per host thread; cfg5: 20 per host thread)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)
    if args.workload == "disto":
        return run_disto(args, rank, world, local)
    if args.workload == "raw":
        return run_raw(args, rank, world, local)
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if args.workload == "cfg5":
        return run_sequence(args, rank, world, local)

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    ptk = importlib.import_module("p-tracker_b200")
    wl = importlib.import_module("p-tracker_b200.workloads")

    pair = wl.make_pair(args.workload, seed=rank_seed(rank))
    p = pair["params"]
    n = pair["rec"].shape[0]
    opts = wl.tracker_options(p)
    stream = torch.cuda.Stream()
    head = dict(search_method=ptk.SEARCH_BF16, subpix_method=ptk.SUBPIX_ADJOINT_LM)
    t = ptk.Tracker(p["dimx"], p["dimy"], rescue_level=opts["rescue_level"], NCC_min=opts["NCC_min"], iraz=1 << 30,
                    autotune=1, **head)
    t.set_stream(stream.cuda_stream)
    for lvl, z in enumerate(opts["zones"]):
        if z is not None:
            t.set_zone(lvl, *z)
    ref_pin = torch.from_numpy(np.ascontiguousarray(pair["ref"])).pin_memory().numpy()
    cur_pin = torch.from_numpy(np.ascontiguousarray(pair["cur"])).pin_memory().numpy()
    t.set_grains(pair["rec"])
    t.make_patterns("grain_diameter", 1.0, 1.0)
    t.load_frame(0, ref_pin)
    t.load_frame(1, cur_pin)
    t.snapshot_grains()
    tune = {"headline": t.autotune()}  # search shapes timed on this pair, before any timing
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def time_frames(steps):
        """Device-resident frames: grain state restored on the device, L2
        flushed, then one frame timed with events on the context stream."""
        for _ in range(args.warmup):
            t.restore_grains()
            t.track_frame(1)
        stream.synchronize()
        total = 0.0
        l0 = t.launches()
        for _ in range(steps):
            flush.zero_()
            t.restore_grains()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t.track_frame(1)
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        return total / steps, t.launches() - l0

    def pixel_stage():
        t.restore_grains()
        t.precompute()
        t.search(0)
        return t.get_grains()

    with torch.cuda.stream(stream):
        # ---- headline: BF16 tensor-core search + exact rescoring + adjoint LM
        barrier()
        try:
            pr = torch.cuda.get_device_properties(local)
            gpu_id = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        except Exception:
            gpu_id = str(local)
        sampler = ClockSampler(gpu_id if rank == 0 else None)
        ms_step, launches = time_frames(args.steps)
        barrier()
        head_rec = t.get_grains()

        # ---- per-kernel roofline of the BF16 search (CUDA events between its kernels)
        kms = []
        for _ in range(max(3, args.steps // 2)):
            flush.zero_()
            t.restore_grains()
            t.precompute()
            kms.append(t.search_timed(0))
        kms = np.median(np.array(kms), axis=0).tolist()
        bf16_pix = pixel_stage()

        # ---- the other forms on the same pair
        t.configure(search_method=ptk.SEARCH_EXACT, subpix_method=ptk.SUBPIX_POWELL)
        t.restore_grains()
        tune["plain"] = t.autotune()
        plain_ms, _ = time_frames(args.steps)
        plain_rec = t.get_grains()
        exact_pix = pixel_stage()
        t.configure(subpix_method=ptk.SUBPIX_ADJOINT_LM)
        lm_ms, _ = time_frames(args.steps)
        lm_rec = t.get_grains()
        t.configure(**head)
        clocks = sampler.stop()  # sampled over the timed frames of all three forms

        # ---- e2e: the headline form through the C ABI with host buffers, as a
        # host loop runs it: every step uploads both frames from pinned memory,
        # tracks them and reads the records back; the next pair's frames are
        # handed to the library before the current pair's records are read, so
        # that the upload into the buffer the current frame no longer reads (the
        # old reference, after its precompute) overlaps the tracking.  Every
        # step's inputs come from host memory, so no L2 flush is needed.
        rec_host = pair["rec"]

        def e2e_run(k_steps):
            t.load_frame(0, ref_pin)
            t.load_frame(1, cur_pin)
            out = None
            for k in range(k_steps):
                t.set_grains(rec_host)
                t.track_frame(1)
                if k + 1 < k_steps:
                    t.load_frame(0, ref_pin)
                    t.load_frame(1, cur_pin)
                out = t.get_grains()
            return out

        e2e_run(max(args.warmup, 1))
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_run(args.e2e_steps)
        e1.record(stream)
        e1.synchronize()
        e2e_ms = [e0.elapsed_time(e1) / args.e2e_steps]

    e2e_step = statistics.mean(e2e_ms)
    ms_step, e2e_step, plain_ms, lm_ms = reduce_max([ms_step, e2e_step, plain_ms, lm_ms], world, device="cuda")

    if rank == 0:
        zone = opts["zones"][0]
        nsteps = rotation_step_count(zone)
        ppc = search_ppc(t, pair["rec"], zone, nsteps)
        peaks = measured_peaks()
        k_search_ms = kms[1]
        alg = 6.0 * ppc / (k_search_ms * 1e-3) / 1e12
        gemm = gemm_flops(pair["rec"]) / (k_search_ms * 1e-3) / 1e12
        truth_err = np.abs(head_rec[:, 4:6] - pair["truth"][:, :2])
        plain_err = np.abs(plain_rec[:, 4:6] - pair["truth"][:, :2])
        agree = np.all(bf16_pix[:, 4:7] == exact_pix[:, 4:7], axis=1)
        frame_bytes = pair["ref"].nbytes + pair["cur"].nbytes
        nn = n
        block = 16 * 8 * nn + 2 * 8 * nn + ((12 * nn + 15) // 16) * 16 + ((2 * nn + 15) // 16) * 16
        line = {
            "metric": METRIC, "value": aggregate_rate(n, world, ms_step), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 ranking (f32 accumulate) + int64 exact rescoring + f32/f64 adjoint LM",
            "data": "synthetic",
            "config": pair_config(dict(p, name=args.workload), n, zone, nsteps, world),
            "form": "BF16 tensor-core search + exact rescoring + adjoint LM (headline)",
            "autotune": tune,
            "e2e": {"value": aggregate_rate(n, world, e2e_step), "unit": UNIT,
                    "h2d_bytes_per_step": int(frame_bytes + block), "d2h_bytes_per_step": int(block)},
            "gpu_launches": int(launches),
            "roofline": {"kernel": "k_search_bf16 (tcgen05 candidate ranking)", "bound": "tensor",
                         "achieved": alg, "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
                         "frac": alg / peaks["bf16_tflops"],
                         "traffic": recorded_traffic("k_search_bf16_cfg2.md") if args.workload == "cfg2" else None,
                         "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of this "
                                           "kernel on this workload (profiles/k_search_bf16_cfg2.md)",
                         "algorithmic_flop_per_launch": 6.0 * ppc, "ppc_per_launch": int(ppc),
                         "tensor_flop_per_launch": gemm_flops(pair["rec"]), "tensor_tflops": gemm,
                         "tensor_frac": gemm / peaks["bf16_tflops"], "launch_ms": k_search_ms,
                         "search_kernels_ms": {"k_weights_bf16": kms[0], "k_search_bf16": kms[1],
                                               "k_rescore_bf16": kms[2]},
                         "peak_source": peaks["source"] + " bf16 dense (burst)"},
            "accuracy": {"median_abs_err_px_vs_truth": float(np.median(truth_err)),
                         "max_abs_err_px_vs_truth": float(truth_err.max()),
                         "plain_median_abs_err_px_vs_truth": float(np.median(plain_err)),
                         "plain_max_abs_err_px_vs_truth": float(plain_err.max()),
                         "integer_argmax_agreement_vs_exact_search": float(agree.mean()),
                         "max_abs_err_px_vs_plain": float(np.abs(head_rec[:, 4:6] - plain_rec[:, 4:6]).max()),
                         "max_abs_err_rad_vs_plain": float(np.abs(head_rec[:, 6] - plain_rec[:, 6]).max())},
            "clocks": clocks,
            "forms": {
                "bf16_search+adjoint_lm": {"value": aggregate_rate(n, world, ms_step), "ms_per_step": ms_step},
                "plain": {"value": aggregate_rate(n, world, plain_ms), "ms_per_step": plain_ms,
                          "search": "exact integer/FP64", "subpixel": "FP64 Powell"},
                "exact_search+adjoint_lm": {"value": aggregate_rate(n, world, lm_ms), "ms_per_step": lm_ms,
                                            "max_abs_err_px_vs_plain": float(np.abs(lm_rec[:, 4:6] -
                                                                                    plain_rec[:, 4:6]).max())},
                "speedup_headline_vs_plain": plain_ms / ms_step,
            },
        }
        if not args.no_cpu_baseline:
            threads = cpu_threads()
            idx = sample_indices(n, args.cpu_sample if args.cpu_sample > 0 else baseline_sample_size(n, threads))
            kind, times, cpu_rec = cpu_track(pair, wl, idx, threads, steps=1)
            cpu_value = len(idx) / times[0]
            line["cpu_baseline"] = {"value": cpu_value, "unit": UNIT, "cores": threads, "kind": kind,
                                    "sample": f"{len(idx)} of {n} grains, the whole frame pipeline"}
            line["accuracy"]["fp64_oracle_grains"] = int(len(idx))
            line["accuracy"]["max_abs_err_px_vs_fp64_oracle"] = float(np.abs(head_rec[idx][:, 4:6] -
                                                                             cpu_rec[:, 4:6]).max())
            line["accuracy"]["max_abs_err_rad_vs_fp64_oracle"] = float(np.abs(head_rec[idx][:, 6] -
                                                                              cpu_rec[:, 6]).max())
            line["accuracy"]["plain_max_abs_err_px_vs_fp64_oracle"] = float(np.abs(plain_rec[idx][:, 4:6] -
                                                                                   cpu_rec[:, 4:6]).max())
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    t.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
