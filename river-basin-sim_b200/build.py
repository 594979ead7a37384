"""Build librbsim.so (the CUDA kernels + C ABI) in-tree for sm_100a.

    python river-basin-sim_b200/build.py [--verbose-ptxas] [--force]

The library is written next to the Python package (``rbsim/librbsim.so``) so it
travels with the source tree. Each source compiles to its own object (in
parallel, under ``_build/``), then one link. Flags that carry meaning:

* ``-gencode arch=compute_100a,code=sm_100a`` -- B200 only, no other targets;
* the **exact** translation units (every ``csrc/*.cu``): ``--fmad=false`` with the
  default IEEE division and square root -- one rounding per operation in source
  order, the arithmetic contract the kernels share with the CPU oracle
  (``include/rb_detmath.h`` supplies the fractional powers);
* the **fast** translation unit (``csrc/fast/*.cu``: the same step kernels again,
  in namespace ``rb::fast``, with ``RB_FAST_MATH`` defined): contracted
  multiply-adds and the hardware's approximate division and square root, the
  arithmetic a GPU build of the reference uses; selected at run time with
  ``rb_set_arith_mode`` and held to the solver tolerance instead of bit equality;
* ``-cudart static`` -- the library carries its own runtime and only needs the
  driver, so it does not depend on which CUDA runtime the host process loaded.
"""

from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "rbsim", "librbsim.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2"]
EXACT = ["--fmad=false"]
FAST = ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-DRB_FAST_MATH=1"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build librbsim.so")


def units() -> list[tuple[str, list[str]]]:
    """(source, arithmetic flags) of every translation unit."""
    exact = [(p, EXACT) for p in sorted(glob.glob(os.path.join(CSRC, "*.cu")))]
    fast = [(p, FAST) for p in sorted(glob.glob(os.path.join(CSRC, "fast", "*.cu")))]
    return exact + fast


def sources() -> list[str]:
    return [p for p, _ in units()]


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = (sources() + glob.glob(os.path.join(CSRC, "*.h*")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
            + [os.path.abspath(__file__)])  # fmt: skip
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, flags: list[str], verbose_ptxas: bool) -> str:
    rel = os.path.relpath(src, CSRC).replace(os.sep, "__")
    obj = os.path.join(OBJ, rel[:-3] + ".o")
    cmd = [nvcc(), *ARCH, *COMMON, *flags, "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-c", src, "-o", obj]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    subprocess.run(cmd, check=True)
    return obj


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    with ThreadPoolExecutor(max_workers=max(1, min(len(units()), os.cpu_count() or 1))) as pool:
        objs = list(pool.map(lambda u: _compile(u[0], u[1], verbose_ptxas), units()))
    subprocess.run([nvcc(), *ARCH, "-cudart", "static", "-shared", *objs, "-o", OUT + ".tmp"], check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    print(build(args.verbose_ptxas, force=True if args.verbose_ptxas else args.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
