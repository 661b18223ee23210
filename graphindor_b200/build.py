"""Builds libgraphindor_b200.so in-tree for sm_100a.

Host C++ (the planner and the C ABI) is compiled with g++ without FMA
contraction so that the analytic schedule model rounds exactly like the
reference planner; CUDA sources are compiled by nvcc for
``-gencode arch=compute_100a,code=sm_100a``.  Objects go to
``graphindor_b200/_build`` and the library to ``graphindor_b200/lib``.
Re-running only recompiles sources newer than their objects.

Usage: ``python -m graphindor_b200.build [--force] [-v]``
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libgraphindor_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    # The system g++ (the /opt wrapper some images put first on CC/CXX lacks
    # the OpenMP spec files).
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("g++ not found")


def _sources():
    return sorted(CSRC.glob("*.cpp")) + sorted(CSRC.glob("*.cu"))


def _headers():
    return sorted(CSRC.glob("*.hpp")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _compile_cmd(src: Path, obj: Path) -> list[str]:
    if src.suffix == ".cpp":
        return [_host_cxx(), "-std=c++17", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-Wall",
                "-Wno-unused-function", f"-I{INCLUDE}", "-c", str(src), "-o", str(obj)]
    return [_nvcc(), *ARCH, "-std=c++17", "-O3", "-lineinfo", "-Xptxas", "-v", "--use_fast_math",
            "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off", "-ccbin", _host_cxx(),
            f"-I{INCLUDE}", "-c", str(src), "-o", str(obj)]


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0.0)
    jobs = []
    objs = []
    for src in _sources():
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        stale = force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header)
        if stale:
            jobs.append((src, obj))

    def run(job):
        src, obj = job
        cmd = _compile_cmd(src, obj)
        res = subprocess.run(cmd, capture_output=True, text=True)
        return src, cmd, res

    failed = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for src, cmd, res in ex.map(run, jobs):
            if verbose or res.returncode != 0:
                sys.stderr.write(f"$ {' '.join(cmd)}\n{res.stdout}{res.stderr}\n")
            if res.returncode != 0:
                failed.append(src.name)
    if failed:
        raise RuntimeError(f"compilation failed: {', '.join(failed)}")
    newest_obj = max(o.stat().st_mtime for o in objs)
    if force or jobs or not LIB.exists() or LIB.stat().st_mtime < newest_obj:
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-Xcompiler", "-fopenmp",
               "-ccbin", _host_cxx(), "-lgomp"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or res.returncode != 0:
            sys.stderr.write(f"$ {' '.join(cmd)}\n{res.stdout}{res.stderr}\n")
        if res.returncode != 0:
            raise RuntimeError("link failed")
    build_tools(force=force, verbose=verbose)
    return LIB


TOOLS = {"gpu_graph": 1, "gpu_clique": 2, "gpu_kclique": 3, "gpu_mc": 4, "gpu_fsm": 5}
BINDIR = PKG / "bin"


def build_tools(force: bool = False, verbose: bool = False) -> None:
    """The reference-compatible command-line tools, linked against the library."""
    BINDIR.mkdir(exist_ok=True)
    src = CSRC / "cli" / "gi_cli.cpp"
    for name, tool in TOOLS.items():
        out = BINDIR / name
        if not force and out.exists() and out.stat().st_mtime >= max(src.stat().st_mtime, LIB.stat().st_mtime):
            continue
        cmd = [_host_cxx(), "-std=c++17", "-O2", f"-DGI_TOOL={tool}", f"-I{INCLUDE}", str(src), "-o", str(out),
               f"-L{LIBDIR}", "-lgraphindor_b200", f"-Wl,-rpath,$ORIGIN/../lib"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or res.returncode != 0:
            sys.stderr.write(f"$ {' '.join(cmd)}\n{res.stdout}{res.stderr}\n")
        if res.returncode != 0:
            raise RuntimeError(f"building {name} failed")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
