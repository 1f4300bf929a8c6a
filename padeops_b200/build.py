"""Build the padeops_b200 CUDA library in-tree (sm_100a).

    python -m padeops_b200.build          # builds padeops_b200/_lib/libpado.so

nvcc cross-compiles for sm_100a without a GPU.  The library is placed inside
the package directory so it travels with the source tree.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libpado.so")
SOURCES = ["pado_api.cu", "pado_batch.cu", "pado_tables.cpp", "pado_inst.cu", "pado_stagg.cu"]
HEADERS = ["pado_common.h", "pado_tables.h", "pado_kernels.cuh", "pado_batch.cuh", "pado_internal.h", "pado_params.h",
           "pado_stream.cuh", "pado_resident.cuh"]
# pado_inst.cu is compiled once per stencil (-DPADO_RK=n) into pado_inst_rkN.o
STENCILS = 4
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build padeops_b200")
    return cand


def _digest() -> str:
    h = hashlib.sha256()
    for name in SOURCES + HEADERS + ["../../include/pado.h"]:
        p = os.path.join(CSRC, name)
        if os.path.exists(p):
            with open(p, "rb") as fh:
                h.update(fh.read())
    h.update(" ".join(ARCH + NVCC_FLAGS).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source for sm_100a and link libpado.so (skipped when up to date)."""
    os.makedirs(LIBDIR, exist_ok=True)
    stamp = os.path.join(LIBDIR, "libpado.sha256")
    digest = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp):
        with open(stamp) as fh:
            if fh.read().strip() == digest:
                return LIB
    objs = []
    procs = []
    units = []
    for src in SOURCES:
        stem = os.path.splitext(src)[0]
        if src == "pado_inst.cu":
            units += [(src, f"{stem}_rk{rk}.o", [f"-DPADO_RK={rk}"]) for rk in range(STENCILS)]
        else:
            units.append((src, stem + ".o", []))
    for src, oname, defs in units:
        path = os.path.join(CSRC, src)
        obj = os.path.join(LIBDIR, oname)
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *defs, "-I", os.path.join(HERE, "..", "include"), "-c", path, "-o", obj]
        if verbose:
            cmd.append("-Xptxas=-v")
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed ({' '.join(cmd)}):\n{out}")
        if verbose and out:
            print(out)
    link = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
    subprocess.run(link, check=True)
    with open(stamp, "w") as fh:
        fh.write(digest)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
