"""Build the engine's shared library in-tree with nvcc for sm_100a (B200).

    python -m flyzero_b200._build            # from can-the-fly-play-f-zero-_b200/

The library is C-ABI only (include/flybrain.h); nothing in it links against PyTorch.
"""

from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(ROOT, "csrc")
OUT_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(OUT_DIR, "libflybrain.so")
SOURCES = ["flybrain.cu", "static_run.cu", "mlp.cu"]
HEADERS = ["common.cuh", "engine.cuh", "persist.cuh", "host_prep.hpp", "plastic.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _digest(deps: list) -> str:
    """SHA-256 over the sources' names and contents: what the library was built from."""
    import hashlib

    h = hashlib.sha256()
    for d in sorted(set(os.path.abspath(x) for x in deps)):
        h.update(os.path.basename(d).encode())
        with open(d, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def _stale(out: str, deps: list) -> bool:
    """True unless ``out`` exists and its stamp records the current sources' digest (a build that
    read the sources before they changed leaves an old stamp, whatever the file times say)."""
    stamp = out + ".sha256"
    if not os.path.exists(out) or not os.path.exists(stamp):
        return True
    with open(stamp) as f:
        return f.read().strip() != _digest(deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "..", "include", h) for h in ("flybrain.h", "flysurrogate.h")]
    deps += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh"))]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-O2",
           "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills", "-o", LIB + ".tmp"]
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    digest = _digest(deps)                     # taken before nvcc reads the sources
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    with open(LIB + ".sha256", "w") as f:
        f.write(digest + "\n")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
