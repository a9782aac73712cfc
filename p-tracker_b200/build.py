"""Builds the in-tree shared libraries of the package.

    libptk.so        C-ABI tracking path (CUDA kernels for sm_100a + host runtime)
    libptk_synth.so  seeded synthetic frame generator (host, OpenMP)
    ptracker_b200    command-file driver of the tracking procedure (links libptk.so)

Every .cu file is compiled by nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a); the remap kernels are compiled with
-fmad=false so their FP64 arithmetic repeats the CPU restatement's operations
exactly (the remap is checked bit for bit), and so are the distortion fit's
objective and the plain form's subpixel objective and Powell minimiser (the
reference is built without FMA contraction).  Objects go to _build/ next to
this file; a source is recompiled only when it or a header is newer than its
object.  Run `python p-tracker_b200/build.py` or call build().
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
ROOT = HERE.parent
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-O3", "--expt-relaxed-constexpr"]
NO_FMA = {"ptk_remap.cu", "ptk_disto.cu", "ptk_raw.cu", "ptk_subpix.cu"}
CU_SOURCES = ["ptk_search.cu", "ptk_search_tiled.cu", "ptk_search_bf16.cu", "ptk_subpix_lm.cu", "ptk_subpix.cu", "ptk_remap.cu", "ptk_api.cu", "ptk_noalloc.cu", "ptk_disto.cu", "ptk_raw.cu"]
CXX_SOURCES = ["grainfile.cpp", "imageio.cpp", "tunecache.cpp"]


def _host_cxx() -> str:
    # an inherited $CXX may be a wrapper without OpenMP support
    for c in ("/usr/bin/g++", shutil.which("g++") or "g++"):
        if c and os.path.exists(c):
            return c
    return "g++"


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _headers() -> list[Path]:
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(verbose: bool = False, ptxas_verbose: bool = False) -> dict:
    BUILD.mkdir(exist_ok=True)
    hdrs = _headers()
    nvcc = _nvcc()
    cxx = _host_cxx()
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            flags = list(NVCC_FLAGS) + (["-fmad=false"] if src in NO_FMA else [])
            if ptxas_verbose:
                flags += ["-Xptxas", "-v"]
            jobs.append([nvcc, *ARCH, *flags, "-ccbin", cxx, "-I", str(INCLUDE), "-c", str(s), "-o", str(o)])
    for src in CXX_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            jobs.append([cxx, "-O2", "-std=c++17", "-fPIC", "-I", str(INCLUDE), "-c", str(s), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        list(ex.map(_run, jobs))
    lib = HERE / "libptk.so"
    if jobs or _stale(lib, objs):
        _run([nvcc, *ARCH, "-shared", "-ccbin", cxx, "-o", str(lib), *map(str, objs), "-lcudart", "-lz"])
    synth = HERE / "libptk_synth.so"
    s = CSRC / "synth.cpp"
    if _stale(synth, [s]):
        _run([cxx, "-O3", "-fopenmp", "-std=c++17", "-fPIC", "-shared", str(s), "-o", str(synth)])
    cli = HERE / "ptracker_b200"
    s = CSRC / "ptracker_cli.cpp"
    if _stale(cli, [s, lib] + hdrs):
        _run([cxx, "-O2", "-std=c++17", "-I", str(INCLUDE), str(s), "-o", str(cli), "-L", str(HERE), "-lptk",
              "-Wl,-rpath,$ORIGIN", "-pthread"])
    if verbose:
        print(f"built {lib}, {synth} and {cli} ({len(jobs)} objects recompiled)")
    return {"libptk": str(lib), "libptk_synth": str(synth), "cli": str(cli), "recompiled": len(jobs)}


if __name__ == "__main__":
    build(verbose=True, ptxas_verbose="-v" in sys.argv)
