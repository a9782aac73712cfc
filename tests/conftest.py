"""Shared fixtures: the package (in-tree libptk.so), the CPU checkers, and
seeded workloads.  GPU tests are marked `gpu`; everything else runs on CPU."""
from __future__ import annotations

import importlib
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ptk():
    build = importlib.import_module("p-tracker_b200.build")
    build.build()
    return importlib.import_module("p-tracker_b200")


@pytest.fixture(scope="session")
def wl(ptk):
    return importlib.import_module("p-tracker_b200.workloads")


@pytest.fixture(scope="session")
def oracle():
    import bind
    bind.build()
    return bind


@pytest.fixture(scope="session")
def cuda_device():
    if not _cuda_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    import torch
    torch.cuda.init()
    return 0


_PAIRS: dict = {}


@pytest.fixture(scope="session")
def pair_cache(wl):
    def get(name: str, seed: int = 1, n: int | None = None):
        key = (name, seed, n)
        if key not in _PAIRS:
            _PAIRS[key] = wl.make_pair(name, seed=seed, n=n)
        return _PAIRS[key]
    return get


def assert_pixel_parity(gpu_rec: np.ndarray, cpu_rec: np.ndarray, top2: np.ndarray, ncc_tol: float = 1e-5,
                        gap: float = 1e-6):
    """Same integer offset / rotation step on every grain whose best NCC and
    best distinct NCC differ by more than `gap`; NCC within `ncc_tol`
    everywhere.  Returns the number of grains that were checked."""
    clear = (top2[:, 0] - top2[:, 1]) > gap
    for col in (4, 5, 6):
        bad = clear & (np.abs(gpu_rec[:, col] - cpu_rec[:, col]) > 1e-9)
        assert not bad.any(), f"column {col} differs on grains {np.nonzero(bad)[0][:10]}"
    d = np.abs(gpu_rec[:, 10] - cpu_rec[:, 10])
    assert np.nanmax(d) <= ncc_tol, f"NCC differs by {np.nanmax(d)}"
    return int(clear.sum())
