"""Build recipe of the CUDA library: nvcc for sm_100a, in-tree output.

``python -m pulse_b200.build`` (or ``__graft_entry__.build()``) compiles
``pulse_b200/csrc/*.cu`` into ``pulse_b200/libpulse_cuda.so``.  The tracer is
compiled with ``-fmad=false`` and IEEE division/sqrt so its arithmetic matches
the restated reference operation for operation.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
OUT = PKG / "libpulse_cuda.so"
BUILD = PKG / "_build"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr",
         f"-I{INCLUDE}"]


def sources():
    return sorted(CSRC.glob("*.cu"))


def _deps():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + \
        sorted(INCLUDE.glob("*.h"))


def needs_build() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _deps())


def _compile(src: Path, extra) -> Path:
    obj = BUILD / (src.stem + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if "-v" in extra:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False, extra=()) -> Path:
    if not force and not needs_build():
        return OUT
    BUILD.mkdir(exist_ok=True)
    extra = list(extra) + (["-Xptxas", "-v"] if verbose else [])
    with ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), sources()))
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *[str(o) for o in objs], "-o", str(tmp)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, OUT)
    build_plugin(force=True)
    return OUT


HOST = PKG / "host"
PLUGIN = PKG / "libpulse_plugin.so"


def build_plugin(force: bool = False) -> Path:
    """The C++ plugin surface (pulse_b200/host) as libpulse_plugin.so, linked
    against libpulse_cuda.so in the same directory."""
    srcs = sorted(HOST.glob("*.cpp"))
    deps = srcs + sorted(HOST.glob("*.hpp")) + [OUT]
    if not force and PLUGIN.exists() and all(p.stat().st_mtime <= PLUGIN.stat().st_mtime for p in deps):
        return PLUGIN
    tmp = PLUGIN.with_suffix(".so.tmp")
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", *[str(s) for s in srcs], "-o", str(tmp),
           f"-L{PKG}", "-lpulse_cuda", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"plugin build failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, PLUGIN)
    return PLUGIN


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    build_plugin()
    print(OUT)
