"""The precision form's integer search: BF16 tensor-core candidate ranking
(tcgen05, FP32 accumulation in tensor memory) followed by exact integer
rescoring of every rotation step at the kept candidates.

Bar: the exact search's own - the same integer offset and rotation step as the
CPU oracle on every grain whose two best NCC values differ by more than 1e-6,
NCC within 1e-5 - on 8- and 16-bit frames, noisy frames, multi-tile zones,
rescue levels and irregular patterns.  The launch count shows that the
tensor-core kernels ran (6 launches per level instead of 2)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import assert_pixel_parity

pytestmark = pytest.mark.gpu

THREADS = max(1, min(32, os.cpu_count() or 1))


def _gpu(ptk, pair, zones, pattern=("grain_diameter", 1.0, 1.0), **opts):
    p = pair["params"]
    t = ptk.Tracker(p["dimx"], p["dimy"], search_method=ptk.SEARCH_BF16, **opts)
    for lvl, z in enumerate(zones):
        if z is not None:
            t.set_zone(lvl, *z)
    t.set_grains(pair["rec"])
    if pattern[0] == "patterns":
        t.set_patterns(pattern[1])
    else:
        t.make_patterns(pattern[0], pattern[1], pattern[2])
    t.load_frame(0, pair["ref"])
    t.load_frame(1, pair["cur"])
    return t


def _cpu(oracle, pair, zones, params, pattern=("grain_diameter", 1.0, 1.0)):
    t = oracle.setup(oracle.Port, pair, threads=THREADS, zones=zones, params=params,
                     pattern=pattern if pattern[0] != "patterns" else ("circ", 1))
    if pattern[0] == "patterns":
        for g, pts in enumerate(pattern[1]):
            t.set_pattern(g, pts)
    return t


def _pixel_case(ptk, oracle, pair, zones, pattern=("grain_diameter", 1.0, 1.0), **opts):
    g = _gpu(ptk, pair, zones, pattern, rescue_level=0, **opts)
    g.precompute()
    before = g.launches()
    g.search(0)
    assert g.launches() - before == 7, ("stage begin, weights, tensor-core search, rescore, finalize, "
                                        "exact re-search of rejected grains, finalize")
    c = _cpu(oracle, pair, zones, {"rescue_level": 0, "NCC_min": 0.7}, pattern)
    c.precompute()
    c.pixel_all()
    gr, cr = g.get_grains(), c.get_grains()
    n = assert_pixel_parity(gr, cr, c.top2())
    return gr, cr, n


@pytest.mark.parametrize("preset,seed", [("tiny", 5), ("small16", 7), ("small16", 8)])
def test_bf16_pixel_stage(ptk, wl, oracle, cuda_device, pair_cache, preset, seed):
    pair = pair_cache(preset, seed)
    zones = wl.tracker_options(pair["params"])["zones"]
    gr, cr, n = _pixel_case(ptk, oracle, pair, zones)
    assert n >= pair["rec"].shape[0] - 1
    np.testing.assert_array_equal(gr[:, 7:10], cr[:, 7:10])


def test_bf16_pixel_stage_noisy(ptk, wl, oracle, cuda_device):
    p = dict(wl.PRESETS["small16"], noise=0.05 * 65535)
    pair = wl.make_pair(p, seed=12)
    zones = wl.tracker_options(p)["zones"]
    _pixel_case(ptk, oracle, pair, zones)


def test_bf16_multi_tile_zone(ptk, wl, oracle, cuda_device):
    """A 41 x 41 zone (2 x 2 candidate tiles per grain, partial edge tiles).
    Grains are placed with a margin for the zone: the oracle, like the
    reference, does not guard reads past the frame edge."""
    pair = wl.make_pair(dict(wl.PRESETS["small16"], zone=22), seed=9)
    zones = [(20, 20, 18, 22, 3, 0.005)]
    gr, _, n = _pixel_case(ptk, oracle, pair, zones)
    assert n >= pair["rec"].shape[0] - 1


@pytest.mark.parametrize("keep", [1, 3])
def test_bf16_fewer_kept_candidates(ptk, wl, oracle, cuda_device, pair_cache, keep):
    pair = pair_cache("small16", 7)
    zones = wl.tracker_options(pair["params"])["zones"]
    _pixel_case(ptk, oracle, pair, zones, topk=keep)


@pytest.mark.parametrize("dups", [1, 3, 9], ids=["unique", "few_repeats", "many_repeats"])
def test_bf16_custom_patterns(ptk, wl, oracle, cuda_device, pair_cache, dups):
    pair = pair_cache("tiny", 5)
    rng = np.random.default_rng(3 + dups)
    pats = []
    for _ in range(pair["rec"].shape[0]):
        k = rng.integers(20, 120)
        base = np.stack([rng.integers(-8, 9, k), rng.integers(-8, 9, k)], 1).astype(np.int32)
        pats.append(np.concatenate([base] + [base[:5]] * (dups - 1)) if dups > 1 else base)
    zones = wl.tracker_options(pair["params"])["zones"]
    _pixel_case(ptk, oracle, pair, zones, pattern=("patterns", pats))


def test_bf16_rescue_levels(ptk, wl, oracle, cuda_device):
    p = dict(wl.PRESETS["small16"], disp=7.0, n=30)
    pair = wl.make_pair(p, seed=21)
    zones = [(2, 2, 2, 2, 2, 0.01), (5, 5, 5, 5, 2, 0.01), (9, 9, 9, 9, 3, 0.01)]
    params = {"rescue_level": 2, "NCC_min": 0.8, "NCC_min_super": 0.75}
    g = _gpu(ptk, pair, zones, rescue_level=2, NCC_min=0.8, NCC_min_super=0.75, subpixel=0)
    g.precompute()
    g.search(0)
    g.search(1)
    g.search(2)
    c = _cpu(oracle, pair, zones, params)
    c.precompute()
    nres = c.pixel_all()
    nsup = c.rescue_all()
    c.super_rescue_all()
    assert nres > 0 and nsup > 0, "workload must exercise both rescue levels"
    assert g.rescue_counts() == (nres, nsup)
    gr, cr = g.get_grains(), c.get_grains()
    assert_pixel_parity(gr, cr, c.top2())
    assert np.abs(gr[:, 11] - cr[:, 11]).max() <= 1e-5


def test_bf16_too_many_steps_runs_exact(ptk, wl, oracle, cuda_device, pair_cache):
    """More than 32 rotation steps: the level runs the exact kernels."""
    pair = pair_cache("tiny", 5)
    zones = [(3, 3, 3, 3, 20, 0.0025)]  # 41 steps
    g = _gpu(ptk, pair, zones, rescue_level=0)
    g.precompute()
    before = g.launches()
    g.search(0)
    assert g.launches() - before == 3
    c = _cpu(oracle, pair, zones, {"rescue_level": 0, "NCC_min": 0.7})
    c.precompute()
    c.pixel_all()
    assert_pixel_parity(g.get_grains(), c.get_grains(), c.top2())


def test_bf16_full_frame_with_lm(ptk, wl, oracle, cuda_device, pair_cache):
    """The precision form end to end: BF16 search + adjoint LM, against the
    FP64 Powell oracle at the form's tolerance (0.01 px, 1e-4 rad)."""
    pair = pair_cache("small16", 11)
    o = wl.tracker_options(pair["params"])
    g = _gpu(ptk, pair, o["zones"], rescue_level=o["rescue_level"], NCC_min=o["NCC_min"], iraz=1 << 30,
             subpix_method=ptk.SUBPIX_ADJOINT_LM)
    g.track_frame(1)
    gr = g.get_grains()
    c = oracle.setup(oracle.Port, pair, threads=THREADS, zones=o["zones"],
                     params={"rescue_level": o["rescue_level"], "NCC_min": o["NCC_min"], "iraz": 1 << 30})
    c.track_frame(1)
    cr = c.get_grains()
    np.testing.assert_array_equal(gr[:, :2], cr[:, :2])
    assert np.abs(gr[:, 4:6] - cr[:, 4:6]).max() <= 0.01
    assert np.abs(gr[:, 6] - cr[:, 6]).max() <= 1e-4


def test_bf16_wait_timeout_is_reported(ptk, wl, oracle, cuda_device, pair_cache):
    """A bounded wait of the tensor-core search that runs out is reported by
    ptk_synchronize as PTK_ERR_TIMEOUT, without a fault: the test hook makes the
    kernel wait on a barrier nothing arrives on, before any copy or MMA is
    issued, with a limit of 1000 polls.  Afterwards the same context (hook off)
    and a fresh one track the pair as an untouched context does."""
    pair = pair_cache("small16", 3)
    p = pair["params"]
    o = wl.tracker_options(p)

    def make():
        t = ptk.Tracker(p["dimx"], p["dimy"], rescue_level=o["rescue_level"], NCC_min=0.7, iraz=1 << 30,
                        search_method=ptk.SEARCH_BF16, subpix_method=ptk.SUBPIX_ADJOINT_LM)
        for lvl, z in enumerate(o["zones"]):
            if z is not None:
                t.set_zone(lvl, *z)
        t.set_grains(pair["rec"])
        t.make_patterns("grain_diameter", 1.0, 1.0)
        t.load_frame(0, pair["ref"])
        t.load_frame(1, pair["cur"])
        return t

    want = make()
    want.track_frame(1)
    expect = want.get_grains()
    want.close()
    L = ptk.lib()
    t = make()
    t.snapshot_grains()
    assert L.ptk_test_bf16_wait_timeout(t.h, 1000) == ptk.PTK_OK
    t.precompute()
    t.search(0)
    assert L.ptk_synchronize(t.h) == ptk.PTK_ERR_TIMEOUT
    assert b"gave up" in L.ptk_last_error(t.h)
    assert L.ptk_synchronize(t.h) == ptk.PTK_OK  # the flag is cleared once reported
    assert L.ptk_test_bf16_wait_timeout(t.h, 0) == ptk.PTK_OK
    t.restore_grains()
    t.track_frame(1)
    assert L.ptk_synchronize(t.h) == ptk.PTK_OK
    np.testing.assert_array_equal(t.get_grains(), expect)
    t.close()
    fresh = make()
    fresh.track_frame(1)
    np.testing.assert_array_equal(fresh.get_grains(), expect)
    fresh.close()
