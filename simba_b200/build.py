"""Build recipe for the native library and the drop-in executables.

Compiles every CUDA source for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) and links, in-tree:

    simba_b200/libsimba_b200.so   the C ABI of include/simba_b200.h
    simba_b200/bin/simba          drop-in for the reference `simba` executable
    simba_b200/bin/simba_rtid     drop-in for the reference `simba_rtid` executable
    simba_b200/bin/vfb            drop-in for the reference `vfb` executable

Usage: python -m simba_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
BIN = PKG / "bin"
LIB = PKG / "libsimba_b200.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-O3",
              "--expt-relaxed-constexpr"] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra", f"-I{CUDA_HOME / 'include'}"]

CU_SOURCES = ["search_u64.cu", "search_u32.cu", "search_static.cu", "peak.cu", "vfb.cu",
              "mlp.cu", "ext.cu"]
CPP_SOURCES = ["capi.cpp"]
HEADERS = ["grammar.h", "ext_grammar.h", "engine.h", "cuda_util.h", "json_lite.h",
           "search_impl.cuh"]


def _host_cxx() -> str:
    # The system g++ (an overriding $CXX wrapper may lack runtime pieces).
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps if Path(d).exists())


def _run(cmd, verbose: bool) -> None:
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(str(c) for c in cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    BIN.mkdir(exist_ok=True)
    hdrs = [CSRC / h for h in HEADERS] + [ROOT / "include" / "simba_b200.h"]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = CSRC / src
        if not s.exists():
            continue
        o = OBJ / (src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            jobs.append([NVCC] + NVCC_FLAGS + ["-c", s, "-o", o])
    for src in CPP_SOURCES:
        s = CSRC / src
        o = OBJ / (src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            jobs.append([_host_cxx()] + CXX_FLAGS + ["-c", s, "-o", o])
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    if force or jobs or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs
             + ["-cudart", "static", "-lpthread", "-ldl", "-lrt"], verbose)
    for cli, name, defs in (("cli_simba.cpp", "simba", []),
                            ("cli_simba.cpp", "simba_rtid", ["-DSIMBA_CLI_RTID=1"]),
                            ("cli_vfb.cpp", "vfb", [])):
        s = CSRC / cli
        if not s.exists():
            continue
        out = BIN / name
        if force or _newer(out, [s, LIB] + hdrs):
            _run([_host_cxx()] + CXX_FLAGS + defs + [s, "-o", out, f"-L{PKG}", "-lsimba_b200",
                                                      "-Wl,-rpath,$ORIGIN/.."], verbose)
    return LIB


def clean() -> None:
    shutil.rmtree(OBJ, ignore_errors=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
