"""Build the B200 library and its Python binding in-tree.

    libh3g.so     hyphy-3_b200/lib/      CUDA kernels + C ABI (nvcc, sm_100a) and host C++20 drivers (g++)
    _hyphy3*.so   hyphy-3_b200/python/   pybind11 module over include/hyphy/core/likelihood_gpu.hpp

Objects go to hyphy-3_b200/_build/.  Rebuilds only what is older than its
sources.  Usage: python hyphy-3_b200/build.py [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import subprocess
import sys
import sysconfig

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib"
PYDIR = PKG / "python"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOSTCXX = os.environ.get("H3G_HOSTCXX", "/usr/bin/g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills",
                  "-ccbin", HOSTCXX, f"-I{ROOT / 'include'}"]


def _stale(target: pathlib.Path, deps: list[pathlib.Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(force: bool = False) -> dict[str, pathlib.Path]:
    BUILD.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "h3g.h"]
    sources = sorted(CSRC.glob("*.cu"))
    host_sources = sorted(CSRC.glob("*.cpp"))       # host-only parts (C++20), built by the host compiler
    objs = []
    jobs = []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append([NVCC] + NVFLAGS + ["-c", str(src), "-o", str(obj)])
    for src in host_sources:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append([HOSTCXX, "-O2", "-std=c++20", "-fPIC", "-Wall", "-Wextra", "-I/usr/local/cuda/include",
                         f"-I{ROOT / 'include'}", "-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        list(ex.map(_run, jobs))
    lib = LIB / "libh3g.so"
    if force or _stale(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-ccbin", HOSTCXX, "-o", str(lib)] + [str(o) for o in objs] + ["-lcudart"])
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    mod = PYDIR / f"_hyphy3{ext}"
    mod_src = PYDIR / "_hyphy3_module.cpp"
    # every host header the module compiles against (shims, analyses, optimisers)
    mod_deps = [mod_src, lib, ROOT / "include" / "h3g.h"] + sorted((ROOT / "include" / "hyphy").rglob("*.hpp"))
    if force or _stale(mod, mod_deps):
        import pybind11
        _run([HOSTCXX, "-O2", "-std=c++20", "-fPIC", "-shared", "-Wall", "-Wno-unused-parameter",
              f"-I{pybind11.get_include()}", f"-I{sysconfig.get_paths()['include']}", f"-I{ROOT / 'include'}",
              str(mod_src), "-o", str(mod), f"-L{LIB}", "-lh3g", f"-Wl,-rpath,{LIB}", "-Wl,-rpath,$ORIGIN/../lib"])
    return {"lib": lib, "module": mod}


if __name__ == "__main__":
    out = build(force="--force" in sys.argv)
    for k, v in out.items():
        print(k, v)
