"""Frame uploads that overlap the tracking (ptk_load_frame waits only for the
last reader of the buffer it fills when the last queued work is a frame
graph): a host loop that hands over the next pair's frames before reading the
current pair's records back gets exactly the records of a loop that reads
them back first, with different frames every step, 16-bit and 8-bit, in the
BF16 + LM and the exact + Powell forms, with and without reference changes."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _tracker(ptk, wl, p, rec, iraz, **form):
    o = wl.tracker_options(p)
    t = ptk.Tracker(p["dimx"], p["dimy"], rescue_level=o["rescue_level"], NCC_min=o["NCC_min"], iraz=iraz, **form)
    for lvl, z in enumerate(o["zones"]):
        if z is not None:
            t.set_zone(lvl, *z)
    t.set_grains(rec)
    t.make_patterns("grain_diameter", 1.0, 1.0)
    return t


def _run(t, pairs, rec, pipelined):
    out = []
    t.load_frame(0, pairs[0][0])
    t.load_frame(1, pairs[0][1])
    for k in range(len(pairs)):
        t.set_grains(rec)
        t.track_frame(k + 1)
        if pipelined and k + 1 < len(pairs):
            t.load_frame(0, pairs[k + 1][0])
            t.load_frame(1, pairs[k + 1][1])
        out.append(t.get_grains())
        if not pipelined and k + 1 < len(pairs):
            t.load_frame(0, pairs[k + 1][0])
            t.load_frame(1, pairs[k + 1][1])
    return out


@pytest.mark.parametrize("form", ["bf16_lm", "exact_powell"])
@pytest.mark.parametrize("iraz", [0, 1000])
@pytest.mark.parametrize("preset", ["small16", "tiny"])
def test_pipelined_loads_give_the_same_records(ptk, wl, pair_cache, cuda_device, form, iraz, preset):
    kw = (dict(search_method=ptk.SEARCH_BF16, subpix_method=ptk.SUBPIX_ADJOINT_LM) if form == "bf16_lm"
          else dict(search_method=ptk.SEARCH_EXACT, subpix_method=ptk.SUBPIX_POWELL))
    cases = [pair_cache(preset, seed=s) for s in (41, 42, 43, 44)]
    p, rec = cases[0]["params"], cases[0]["rec"]
    # the same grains tracked through four different frame pairs (the other
    # seeds' frames, pinned so that the uploads are asynchronous)
    pairs = [(ptk.pinned_copy(c["ref"]), ptk.pinned_copy(c["cur"])) for c in cases]
    seq = _tracker(ptk, wl, p, rec, iraz, **kw)
    want = _run(seq, pairs, rec, pipelined=False)
    seq.close()
    pip = _tracker(ptk, wl, p, rec, iraz, **kw)
    got = _run(pip, pairs, rec, pipelined=True)
    pip.close()
    for k, (a, b) in enumerate(zip(want, got)):
        np.testing.assert_array_equal(a, b, err_msg=f"pair {k}")
    # the four pairs give four different results (the uploads matter)
    assert not np.array_equal(want[0], want[1])


def test_stagewise_calls_wait_for_the_uploads(ptk, wl, pair_cache, cuda_device):
    """The stage-by-stage calls (precompute, search, subpixel) issued right
    after asynchronous uploads from page-locked memory read the new frames:
    the same records as with the frames uploaded from ordinary memory."""
    cases = [pair_cache("small16", seed=s) for s in (51, 52, 53)]
    p, rec = cases[0]["params"], cases[0]["rec"]
    kw = dict(search_method=ptk.SEARCH_EXACT, subpix_method=ptk.SUBPIX_POWELL)

    def run(pinned):
        t = _tracker(ptk, wl, p, rec, 1000, **kw)
        out = []
        for c in cases:
            ref, cur = (ptk.pinned_copy(c["ref"]), ptk.pinned_copy(c["cur"])) if pinned else (c["ref"], c["cur"])
            t.set_grains(rec)
            t.load_frame(0, ref)
            t.load_frame(1, cur)
            t.precompute()
            t.search(0)
            t.subpixel(ptk.SUBPIX_POWELL)
            out.append(t.get_grains())
        t.close()
        return out

    for k, (a, b) in enumerate(zip(run(False), run(True))):
        np.testing.assert_array_equal(a, b, err_msg=f"pair {k}")


def test_slots_read_back_what_was_loaded(ptk, wl, pair_cache, cuda_device):
    """With uploads moving slots between the three frame buffers, each slot
    reads back the frame last loaded into it - right after the load, after a
    tracked frame and after reference changes - and the records match a loop
    that waits for every step."""
    cases = [pair_cache("small16", seed=s) for s in (61, 62, 63, 64, 65)]
    p, rec = cases[0]["params"], cases[0]["rec"]
    frames = [(ptk.pinned_copy(c["ref"]), ptk.pinned_copy(c["cur"])) for c in cases]
    kw = dict(search_method=ptk.SEARCH_BF16, subpix_method=ptk.SUBPIX_ADJOINT_LM)
    t = _tracker(ptk, wl, p, rec, 0, **kw)
    want = _run(_tracker(ptk, wl, p, rec, 0, **kw), frames, rec, pipelined=False)
    t.load_frame(0, frames[0][0])
    t.load_frame(1, frames[0][1])
    for k in range(len(frames)):
        t.set_grains(rec)
        t.track_frame(k + 1)
        if k + 1 < len(frames):
            t.load_frame(0, frames[k + 1][0])
            t.load_frame(1, frames[k + 1][1])
        np.testing.assert_array_equal(t.get_grains(), want[k], err_msg=f"pair {k}")
        if k + 1 < len(frames):
            # stage-by-stage reads of both slots: the frames just handed over
            np.testing.assert_array_equal(t.read_frame(0), np.asarray(frames[k + 1][0]))
            np.testing.assert_array_equal(t.read_frame(1), np.asarray(frames[k + 1][1]))
    t.close()
