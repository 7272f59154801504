"""Builds the in-tree shared libraries.

``build_library()`` compiles the CUDA kernels for sm_100a (nvcc) and the host
C++ (g++, OpenMP) into ``optixrender_b200/_lib/liboptixrender_b200.so``.
``build_oracle()`` runs ``oracle/Makefile`` (the CPU checker and, when the
reference tree is present, its host build).  Both skip work whose outputs are
newer than their inputs.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "_lib"
BUILD = PKG / "_build"
LIBNAME = "liboptixrender_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("RT_CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-ftz=true", "-prec-div=false", "-prec-sqrt=false",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fopenmp", "-Wall", "-Wno-unused-function", "-Wno-unknown-pragmas",
             "-I/usr/local/cuda/include"]

CU_SOURCES = ["rt_kernels.cu", "rt_trace_scratch.cu", "rt_guide.cu", "rt_guide_api.cu", "rt_bvh_gpu.cu"]
CPP_SOURCES = ["rt_capi.cpp", "rt_renderer.cpp", "rt_bvh.cpp", "rt_tables.cpp", "rt_scene_io.cpp", "rt_server.cpp",
               "rt_png.cpp", "rt_jpeg.cpp"]
HEADERS = ["rt_device.cuh", "rt_shading.cuh", "rt_traverse.cuh", "rt_kernels.cuh", "rt_internal.h", "rt_bvh.h",
           "rt_media.cuh", "rt_guide.cuh", "rt_guide_host.h", "rt_image.h", "rt_schedule.h"]


def _newer(out: Path, inputs) -> bool:
    if not out.exists():
        return False
    t = out.stat().st_mtime
    return all(not Path(i).exists() or Path(i).stat().st_mtime <= t for i in inputs)


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(map(str, cmd)) + "\n" + r.stdout)
    return r.stdout


def library_path() -> Path:
    return LIBDIR / LIBNAME


def build_library(force: bool = False, verbose: bool = False) -> Path:
    LIBDIR.mkdir(exist_ok=True)
    BUILD.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS if (CSRC / h).exists()] + [ROOT / "include" / "rt_capi.h"]
    objs = []
    jobs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if force or not _newer(o, [s] + headers):
            jobs.append([NVCC] + ARCH + NVCC_FLAGS + ["-c", str(s), "-o", str(o)])
    for src in CPP_SOURCES:
        s = CSRC / src
        if not s.exists():
            continue
        o = BUILD / (src + ".o")
        objs.append(o)
        if force or not _newer(o, [s] + headers):
            jobs.append([CXX] + CXX_FLAGS + ["-c", str(s), "-o", str(o)])
    procs = [subprocess.Popen(j, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True) for j in jobs]
    errors = []
    for j, p in zip(jobs, procs):
        out, _ = p.communicate()
        if p.returncode != 0:
            errors.append(" ".join(j) + "\n" + out)
        elif verbose and out:
            print(out)
    if errors:
        raise RuntimeError("build failed:\n" + "\n".join(errors))
    lib = library_path()
    if force or jobs or not _newer(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", str(lib)] + [str(o) for o in objs] +
             ["-Xcompiler", "-fopenmp", "-lgomp", "-cudart", "static"])
    cli = LIBDIR / "render_json"
    src = PKG / "cpp" / "render_json.cpp"
    if src.exists() and (force or not _newer(cli, [src, lib, ROOT / "include" / "optixrender.hpp"])):
        _run([CXX, "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(src), "-o", str(cli), "-L", str(LIBDIR),
              "-loptixrender_b200", "-Wl,-rpath,$ORIGIN"])
    return lib


def build_oracle(verbose: bool = False) -> None:
    out = _run(["make", "-s", "-C", str(ROOT / "oracle")])
    if verbose and out:
        print(out)


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    force = "--force" in argv
    lib = build_library(force=force, verbose=True)
    print("built", lib)
    build_oracle(verbose=True)
    print("built oracle")
    return 0


if __name__ == "__main__":
    sys.exit(main())
