"""Build the B200 engine in-tree: relaxmap_b200/librelaxmap_b200.so (C ABI) and
relaxmap_b200/ompRelaxmap (the drop-in command line), sm_100a only.

    python -m relaxmap_b200.build [--force]

RMX_NVCC_EXTRA adds compiler flags, e.g. RMX_NVCC_EXTRA="-DRMX_DELTA_MINB=5" to
build a variant of a compile-time launch bound; every object is rebuilt when
the flags differ from the previous build's.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "librelaxmap_b200.so"
CLI = PKG / "ompRelaxmap"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3,-Wall", "-diag-suppress", "177",
         *os.environ.get("RMX_NVCC_EXTRA", "").split()]
CU = ["rmx_prims.cu", "rmx_flow.cu", "rmx_moves.cu", "rmx_coarsen.cu", "rmx_engine.cu", "rmx_adjoint.cu", "rmx_noalloc.cu"]
CPP = ["rmx_io.cpp", "rmx_abi.cpp", "rmx_cli.cpp", "rmx_batch.cpp"]
CUDA_CPP = {"rmx_abi.cpp", "rmx_batch.cpp"}
HEADERS = ["rmx_common.cuh", "rmx_prims.cuh", "rmx_engine.cuh", "rmx_graph.hpp", "rmx_io.hpp", "rmx_batch.hpp"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    stamp = OBJ / "flags.txt"  # the flags the objects were built with
    flags = " ".join([NVCC, *ARCH, *FLAGS])
    if not stamp.exists() or stamp.read_text() != flags:
        force = True
    hdrs = [CSRC / h for h in HEADERS] + [PKG.parent / "include" / "relaxmap_b200.h"]
    jobs = []
    objs = []
    for src in CU + CPP:
        s = CSRC / src
        o = OBJ / (src.rsplit(".", 1)[0] + ".o")
        objs.append(o)
        if force or _stale(o, [s, *hdrs]):
            # C++ sources that see device types go through the CUDA front end
            lang = ["-x", "cu"] if src in CUDA_CPP else []
            jobs.append([NVCC, *ARCH, *FLAGS, *lang, "-c", str(s), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for r in ex.map(_run, jobs):
            if verbose and r.stderr:
                print(r.stderr, file=sys.stderr)
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lpthread", "-ldl", "-lrt"])
    main_o = OBJ / "ompRelaxmap_main.o"
    if force or _stale(main_o, [CSRC / "ompRelaxmap_main.cpp", *hdrs]):
        _run([NVCC, *ARCH, *FLAGS, "-c", str(CSRC / "ompRelaxmap_main.cpp"), "-o", str(main_o)])
    if force or _stale(CLI, [main_o, LIB]):
        _run([NVCC, *ARCH, "-o", str(CLI), str(main_o), *map(str, objs), "-lpthread", "-ldl", "-lrt"])
    stamp.write_text(flags)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
