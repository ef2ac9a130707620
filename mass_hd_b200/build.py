"""Build the sm_100a library libmass_lb.so in-tree (mass_hd_b200/lib/).

    python -m mass_hd_b200.build [--verbose]

Each .cu is compiled for sm_100a only. unfused.cu is compiled twice: its
FP64 half (the oracle mode) with --fmad=false, so that no multiply-add is
contracted and every operation rounds as the reference's double-precision
build rounds it, and its FP32 half with contraction on, like the other units.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libmass_lb.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
          "-I", INCLUDE, "-I", CSRC]
# object -> (source, flags)
UNITS = {
    "unfused": ("unfused.cu", ["--fmad=false", "-DMLB_UNFUSED_PART=64"]),
    "unfused_f32": ("unfused.cu", ["-DMLB_UNFUSED_PART=32"]),
    "masks": ("masks.cu", ["--fmad=false"]),
    "fused32": ("fused32.cu", []),
    "fused_warp": ("fused_warp.cu", []),
    "reduce": ("reduce.cu", []),
    "stats": ("stats.cu", []),
    "api": ("api.cu", []),
    "noalloc": ("noalloc.cu", []),
    "conv_tc": ("conv_tc.cu", []),
    "surrogate_ops": ("surrogate_ops.cu", []),
}


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources_hash(extra: list[str]) -> str:
    h = hashlib.sha256()
    for d in (CSRC, INCLUDE):
        for f in sorted(os.listdir(d)):
            with open(os.path.join(d, f), "rb") as fh:
                h.update(f.encode() + fh.read())
    h.update(" ".join(extra).encode())
    return h.hexdigest()


def build(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False) -> str:
    """Compile every unit and link libmass_lb.so; skipped when the sources
    have not changed since the last build."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    units = {u: sf for u, sf in UNITS.items() if os.path.exists(os.path.join(CSRC, sf[0]))}
    stamp = os.path.join(BUILD, "stamp")
    digest = _sources_hash(ARCH + COMMON + [f"{u}:{sf[0]}:{' '.join(sf[1])}" for u, sf in sorted(units.items())])
    if not force and os.path.exists(LIB) and os.path.exists(stamp):
        with open(stamp) as fh:
            if fh.read().strip() == digest:
                return LIB
    objs = []
    for unit, (src, flags) in units.items():
        obj = os.path.join(BUILD, unit + ".o")
        cmd = [nvcc()] + ARCH + COMMON + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    with open(stamp, "w") as fh:
        fh.write(digest)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print registers/spills")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force, ptxas_verbose=a.ptxas))
    sys.exit(0)
