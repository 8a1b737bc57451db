"""Builds libbonsai_b200.so in-tree with nvcc for sm_100a.

    python -m bonsai_b200.build            # build if any source is newer
    python -m bonsai_b200.build --force    # rebuild

-fmad=false is load-bearing: the plain form is bit-identical to the
reference's CPU grower, which is compiled without floating contraction.
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libbonsai_b200.so")
BUILD_DIR = os.path.join(ROOT, "_build")

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(
        os.path.join(INCLUDE, "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, "-I", INCLUDE, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                       stderr=subprocess.STDOUT), src))
        objs.append(obj)
    for p, src in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{out.decode()}")
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs,
           "-o", tmp, "-lcudart", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


def build_oracle(ref: str | None = None) -> None:
    """Compiles the oracle checkers (test infrastructure): the C restatement
    always, the reference's own CPU grower when `ref` (or BONSAI_REFERENCE)
    names its source tree."""
    ref = ref or os.environ.get("BONSAI_REFERENCE", "")
    args = [f"REF={ref}"] if ref else []
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all", *args], check=True)
    if ref and os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_driver.o")):
        # the drop-in check links the product library: build it after
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "dropin", *args],
                       check=True)


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
