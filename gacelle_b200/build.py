"""In-tree build of libgacelle_b200.so for sm_100a.

``build()`` compiles every CUDA translation unit of ``gacelle_b200/csrc``
with nvcc into ``gacelle_b200/libgacelle_b200.so`` (static CUDA runtime, no
torch dependency) unless the library is newer than all its sources.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libgacelle_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -ftz=true: FP32 subnormals flush to zero, so ex2/rcp/rsqrt are single
# hardware approximations; no quantity in these fits is subnormal.
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-ftz=true", "-Xcompiler", "-fPIC,-O2", "-Xptxas", "-O3",
         "-diag-suppress", "177"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) \
        + glob.glob(os.path.join(INCLUDE, "*.h"))
    return os.path.getmtime(LIB) < max(os.path.getmtime(p) for p in deps)


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objs = []
    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)
    procs = []
    for src in sources():
        obj = os.path.join(build_dir, os.path.basename(src) + ".o")
        cmd = [nvcc()] + ARCH + FLAGS + ["-I", INCLUDE, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), src))
        objs.append(obj)
    for p, src in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{out.decode(errors='replace')}")
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
