"""The autotuner (ptk_autotune / ptk_config.autotune) on the GPU: it times
the level-0 search shapes, keeps one of them, leaves the grain state as it
found it, and the tuned context tracks a frame pair to exactly the results of
an untuned one, in the BF16 and the exact form."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _tracker(ptk, wl, pair, **opts):
    p = pair["params"]
    o = wl.tracker_options(p)
    t = ptk.Tracker(p["dimx"], p["dimy"], rescue_level=o["rescue_level"], NCC_min=o["NCC_min"], **opts)
    for lvl, z in enumerate(o["zones"]):
        if z is not None:
            t.set_zone(lvl, *z)
    t.set_grains(pair["rec"])
    t.make_patterns("grain_diameter", 1.0, 1.0)
    t.load_frame(0, pair["ref"])
    t.load_frame(1, pair["cur"])
    return t


@pytest.mark.parametrize("form", [dict(search_method=1, subpix_method=1), dict(search_method=0)])
def test_autotune_keeps_results(ptk, wl, pair_cache, cuda_device, form):
    pair = pair_cache("small16", seed=31)
    plain = _tracker(ptk, wl, pair, **form)
    plain.track_frame(1)
    want = plain.get_grains()
    plain.close()
    t = _tracker(ptk, wl, pair, **form)
    before = t.get_grains()
    rep = t.autotune()
    np.testing.assert_array_equal(t.get_grains(), before)  # the trials leave the grains as they were
    assert rep["method"] == ("bf16" if form["search_method"] == 1 else "exact")
    assert rep["choice"] in rep["candidates"] and len(rep["candidates"]) >= 1
    assert all(ms > 0.0 for ms in rep["candidates"].values())
    if rep["method"] == "bf16":
        assert set(rep["candidates"]) <= {2, 3, 4, 6} and 4 in rep["candidates"]
    else:
        assert set(rep["candidates"]) <= {1, 2}
    t.track_frame(1)
    np.testing.assert_array_equal(t.get_grains(), want)
    t.close()
    auto = _tracker(ptk, wl, pair, autotune=1, **form)  # tuned inside the first track_frame
    auto.track_frame(1)
    np.testing.assert_array_equal(auto.get_grains(), want)
    auto.close()


def test_autotune_cache(ptk, wl, pair_cache, cuda_device, tmp_path):
    """With a tune cache, the first context times the candidates and records
    its choice under the workload's signature; a second context on the same
    workload takes the recorded choice without timing, and tracks to the same
    results."""
    pair = pair_cache("small16", seed=31)
    form = dict(search_method=1, subpix_method=1)
    cache = tmp_path / "tune.json"
    t = _tracker(ptk, wl, pair, **form)
    t.set_tune_cache(cache)
    sig = t.tune_signature()
    assert sig.startswith("sm_") and "|bf16|" in sig and "|grains " in sig
    rep = t.autotune()
    assert not rep["cached"] and rep["candidates"]
    assert ptk.tune_cache_lookup(cache, sig) == (1, rep["choice"])
    t.track_frame(1)
    want = t.get_grains()
    t.close()
    u = _tracker(ptk, wl, pair, **form)
    u.set_tune_cache(cache)
    assert u.tune_signature() == sig
    rep2 = u.autotune()
    assert rep2["cached"] and rep2["choice"] == rep["choice"] and not rep2["candidates"]
    u.track_frame(1)
    np.testing.assert_array_equal(u.get_grains(), want)
    u.close()
    # an entry for another form is not taken: the exact form times its own candidates
    e = _tracker(ptk, wl, pair, search_method=0)
    e.set_tune_cache(cache)
    assert "|exact|" in e.tune_signature()
    assert not e.autotune()["cached"]
    e.close()
    data = __import__("json").loads(cache.read_text())
    assert len(data["entries"]) == 2
