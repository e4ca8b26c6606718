"""Build oracle/_ref/libref_gpu.so: the reference's own CUDA kernels with a host launcher.

    python oracle/make_ref_gpu.py [--reference PATH]

Extracts the `_SRC` string of flyzero/gpu.py (gpu.py:26-119) with `ast` (no import: the module needs
CuPy), writes it to oracle/_ref/ref_gpu_src.cu and compiles it with oracle/ref_gpu_host.cu for
sm_100a with `--use_fast_math`, the option the reference compiles it with (gpu.py:125). Output only
under oracle/_ref/ (git-ignored); test infrastructure, never shipped.
"""

from __future__ import annotations

import argparse
import ast
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libref_gpu.so")


def extract(reference: str) -> str:
    path = os.path.join(reference, "flyzero", "gpu.py")
    tree = ast.parse(open(path).read(), path)
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(isinstance(t, ast.Name) and t.id == "_SRC" for t in node.targets):
            return ast.literal_eval(node.value)
    raise RuntimeError(f"no _SRC in {path}")


def build(reference: str = "/root/reference", nvcc: str = "nvcc") -> str:
    src = extract(reference)
    os.makedirs(OUT, exist_ok=True)
    cu = os.path.join(OUT, "ref_gpu_src.cu")
    with open(cu, "w") as f:
        f.write(src)
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--use_fast_math", "-shared", "-Xcompiler",
           "-fPIC", f"-DREF_SRC=\"{cu}\"", os.path.join(HERE, "ref_gpu_host.cu"), "-o", LIB + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    print(build(ap.parse_args().reference))
