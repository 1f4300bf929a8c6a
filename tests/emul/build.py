"""Builds the CPU emulator of the line kernel (TEST ONLY): tests/emul/_build/libpado_emul.so."""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_build", "libpado_emul.so")
SRCS = [os.path.join(HERE, "pado_emul.cu"), os.path.join(ROOT, "padeops_b200", "csrc", "pado_tables.cpp")]
DEPS = SRCS + [os.path.join(ROOT, "padeops_b200", "csrc", h) for h in ("pado_kernels.cuh", "pado_common.h",
                                                                        "pado_tables.h", "pado_params.h",
                                                                        "pado_stream.cuh", "pado_resident.cuh")]


def build() -> str:
    if os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d) for d in DEPS):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-O1", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
           "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT, *SRCS]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build())
