"""Benchmark of the per-grain tracking path: grains per second per frame pair.

One step = one frame pair tracked through the whole per-frame pipeline of
particle_tracking (precompute, exact pixel + rotation search, Powell subpixel,
increments) for every grain of the workload.  Default workload: the 16-bit
5616x3744 pair with 2000 bimodal grains (search +-15 px, 21 rotation steps),
seeded synthetic data.

  value  device-resident: frames already in HBM, grain state restored on the
         device before each step; L2 flushed (256 MiB write) before every
         timed step; CUDA events on the context stream.
  e2e    through the C ABI with pinned host buffers: both frames and the grain
         records uploaded, the frame tracked, the records read back, every step.

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


def search_ppc(tracker, rec: np.ndarray, zone, nsteps: int) -> int:
    """Pattern-pixel-candidate evaluations of one pixel-stage search."""
    P = sum(tracker.pattern_size(g) for g in range(rec.shape[0]))
    left, right, up, down = zone[:4]
    return P * nsteps * (left + right + 1) * (up + down + 1)


def run_reference_arm(args, rank: int, world: int):
    if rank != 0:
        return 0
    wl = importlib.import_module("p-tracker_b200.workloads")
    pair = wl.make_pair(args.workload, seed=1000)
    n = pair["rec"].shape[0]
    idx = sample_indices(n, args.ref_sample)
    threads = cpu_threads()
    kind, times, _ = cpu_track(pair, wl, idx, threads, steps=args.steps, warmup=args.warmup)
    per_step = statistics.mean(times)
    value = len(idx) / per_step
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": args.workload, "grains": n, "sample_grains": int(len(idx)), "frame": "5616x3744 u16"
                   if args.workload != "cfg1" else "2048x1536 u8", "pipeline": "precompute+pixel search+Powell"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{len(idx)} of {n} grains (evenly spaced), full frame pipeline per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg2")
    ap.add_argument("--form", default="plain", choices=["plain"])
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--ref-sample", type=int, default=48)
    ap.add_argument("--cpu-sample", type=int, default=48)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)

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
    t = ptk.Tracker(p["dimx"], p["dimy"], rescue_level=opts["rescue_level"], NCC_min=opts["NCC_min"], iraz=1 << 30)
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
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    # ---- value: device-resident steps --------------------------------------
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            t.restore_grains()
            t.track_frame(1)
        stream.synchronize()
        barrier()
        try:
            pr = torch.cuda.get_device_properties(local)
            gpu_id = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        except Exception:
            gpu_id = str(local)
        sampler = ClockSampler(gpu_id if rank == 0 else None)
        launches0 = t.launches()
        total_ms = 0.0
        for _ in range(args.steps):
            flush.zero_()
            t.restore_grains()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t.track_frame(1)
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
        launches = t.launches() - launches0
        barrier()
        clocks = sampler.stop()
        gpu_rec = t.get_grains()

        # ---- differentiation form: same exact search, adjoint-LM subpixel ------
        t.configure(subpix_method=ptk.SUBPIX_ADJOINT_LM)
        for _ in range(args.warmup):
            t.restore_grains()
            t.track_frame(1)
        lm_ms = 0.0
        for _ in range(args.steps):
            flush.zero_()
            t.restore_grains()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t.track_frame(1)
            e1.record(stream)
            e1.synchronize()
            lm_ms += e0.elapsed_time(e1)
        lm_rec = t.get_grains()
        t.configure(subpix_method=ptk.SUBPIX_POWELL)

        # ---- roofline: the pixel search stage alone (k_search dominates) ----
        zone = opts["zones"][0]
        search_ms = []
        for _ in range(max(3, args.steps // 2)):
            flush.zero_()
            t.restore_grains()
            t.precompute()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t.search(0)
            e1.record(stream)
            e1.synchronize()
            search_ms.append(e0.elapsed_time(e1))

        # ---- e2e through the C ABI with host buffers --------------------------
        e2e_ms = []
        rec_host = pair["rec"]
        for it in range(args.warmup + args.e2e_steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            flush.zero_()
            stream.synchronize()
            e0.record(stream)
            t.load_frame(0, ref_pin)
            t.load_frame(1, cur_pin)
            t.set_grains(rec_host)
            t.track_frame(1)
            out = t.get_grains()
            e1.record(stream)
            e1.synchronize()
            if it >= args.warmup:
                e2e_ms.append(e0.elapsed_time(e1))

    ms_step = total_ms / args.steps
    e2e_step = statistics.mean(e2e_ms)
    s_ms = statistics.median(search_ms)
    lm_step = lm_ms / args.steps
    ms_step, e2e_step, s_ms, lm_step = reduce_max([ms_step, e2e_step, s_ms, lm_step], world, device="cuda")

    if rank == 0:
        sys.path.insert(0, str(ROOT / "oracle"))
        import bind
        steps_list = bind.rotation_steps(zone[5], zone[4]) if bind.PORT_SO.exists() else None
        nrot = len(steps_list) if steps_list is not None else 2 * zone[4] + 1
        ppc = search_ppc(t, pair["rec"], zone, nrot)
        flops = 6.0 * ppc
        peaks = measured_peaks()
        achieved = flops / (s_ms * 1e-3) / 1e12
        truth_err = np.abs(gpu_rec[:, 4:6] - pair["truth"][:, :2])
        frame_bytes = pair["ref"].nbytes + pair["cur"].nbytes
        nn = n
        block = 16 * 8 * nn + 2 * 8 * nn + ((12 * nn + 15) // 16) * 16 + ((2 * nn + 15) // 16) * 16
        line = {
            "metric": METRIC, "value": aggregate_rate(n, world, ms_step), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64+f64", "data": "synthetic",
            "config": {"workload": f"{args.workload}: {p['dimx']}x{p['dimy']} "
                                   f"{'u16' if p['maxval'] > 255 else 'u8'}, {n} grains per GPU, search +-{zone[0]} px,"
                                   f" {nrot} rotation steps, Powell subpixel",
                       "form": "plain (exact integer search + FP64 Powell)", "grains_per_gpu": n,
                       "l2": "flushed (256 MiB write) before each timed step", "parallelism": f"grain shards x{world}"},
            "e2e": {"value": aggregate_rate(n, world, e2e_step), "unit": UNIT,
                    "h2d_bytes_per_step": int(frame_bytes + block), "d2h_bytes_per_step": int(block)},
            "gpu_launches": int(launches),
            "roofline": {"kernel": "k_search (pixel + rotation stage)", "bound": "tensor", "achieved": achieved,
                         "peak": peaks["bf16_tflops"], "unit": "TFLOP/s", "frac": achieved / peaks["bf16_tflops"],
                         "traffic": None, "algorithmic_flop_per_launch": flops, "ppc_per_launch": int(ppc),
                         "launch_ms": s_ms, "peak_source": peaks["source"] + " bf16 dense (burst)"},
            "accuracy": {"median_abs_err_px_vs_truth": float(np.median(truth_err)),
                         "max_abs_err_px_vs_truth": float(truth_err.max())},
            "clocks": clocks,
            "forms": {
                "plain": {"value": aggregate_rate(n, world, ms_step), "ms_per_step": ms_step,
                          "search": "exact integer/FP64", "subpixel": "FP64 Powell"},
                "exact_search+adjoint_lm": {"value": aggregate_rate(n, world, lm_step), "ms_per_step": lm_step,
                                            "search": "exact integer/FP64",
                                            "subpixel": "adjoint LM (FP32 samples, FP64 3x3 solve)",
                                            "max_abs_err_px_vs_plain": float(np.abs(lm_rec[:, 4:6] -
                                                                                    gpu_rec[:, 4:6]).max()),
                                            "max_abs_err_rad_vs_plain": float(np.abs(lm_rec[:, 6] -
                                                                                     gpu_rec[:, 6]).max())},
            },
        }
        if not args.no_cpu_baseline:
            idx = sample_indices(n, args.cpu_sample)
            threads = cpu_threads()
            kind, times, cpu_rec = cpu_track(pair, wl, idx, threads, steps=1)
            cpu_value = len(idx) / times[0]
            dpos = np.abs(gpu_rec[idx][:, 4:6] - cpu_rec[:, 4:6])
            line["cpu_baseline"] = {"value": cpu_value, "unit": UNIT, "cores": threads, "kind": kind,
                                    "sample": f"{len(idx)} of {n} grains (evenly spaced), full frame pipeline"}
            line["accuracy"]["max_abs_err_px_vs_fp64_oracle"] = float(dpos.max())
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    t.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
