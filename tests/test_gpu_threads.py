"""Contexts created and run from several host threads at once.

Each context is independent (one per host thread); the shared-memory limits
its kernels need are raised per device behind a lock, so contexts that are
created concurrently all launch their large-shared-memory kernels (the BF16
search and its weights kernel, the register-tiled exact search, Powell).
The threads run in a fresh process, so no earlier context has raised a
limit for them; every thread's results must equal those of a context run
alone afterwards."""
from __future__ import annotations

import importlib
import json
import subprocess
import sys
import threading
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _track(ptk, wl, pair, **form):
    p = pair["params"]
    o = wl.tracker_options(p)
    t = ptk.Tracker(p["dimx"], p["dimy"], rescue_level=o["rescue_level"], NCC_min=0.7, iraz=1 << 30, **form)
    for lvl, z in enumerate(o["zones"]):
        if z is not None:
            t.set_zone(lvl, *z)
    t.set_grains(pair["rec"])
    t.make_patterns("grain_diameter", 1.0, 1.0)
    t.load_frame(0, pair["ref"])
    t.load_frame(1, pair["cur"])
    t.track_frame(1)
    out = t.get_grains()
    t.close()
    return out


def _run_threads(form: str, nthreads: int = 4) -> dict:
    sys.path.insert(0, str(ROOT))
    ptk = importlib.import_module("p-tracker_b200")
    wl = importlib.import_module("p-tracker_b200.workloads")
    pair = wl.make_pair("small16", seed=3)
    kw = (dict(search_method=ptk.SEARCH_BF16, subpix_method=ptk.SUBPIX_ADJOINT_LM) if form == "bf16_lm"
          else dict(search_method=ptk.SEARCH_EXACT, subpix_method=ptk.SUBPIX_POWELL))
    results, errors = [None] * nthreads, []
    start = threading.Barrier(nthreads)

    def work(i):
        try:
            start.wait(timeout=60)
            results[i] = _track(ptk, wl, pair, **kw)
        except Exception as e:  # reported to the parent
            errors.append(repr(e))

    # ctypes releases the GIL around library calls: the contexts are created
    # and launched concurrently
    threads = [threading.Thread(target=work, args=(i,)) for i in range(nthreads)]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=300)
    alone = _track(ptk, wl, pair, **kw)
    same = [r is not None and bool(np.array_equal(r, alone)) for r in results]
    return {"errors": errors, "same": same, "grains": int(alone.shape[0])}


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["bf16_lm", "exact_powell"])
def test_concurrent_contexts(ptk, cuda_device, form):
    r = subprocess.run([sys.executable, __file__, form], capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert r.returncode == 0, r.stdout + r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert not out["errors"], out["errors"]
    assert out["grains"] > 0
    assert all(out["same"]), out["same"]


if __name__ == "__main__":
    print(json.dumps(_run_threads(sys.argv[1])))
