"""Build librbsim.so (the CUDA kernels + C ABI) in-tree for sm_100a.

    python river-basin-sim_b200/build.py [--verbose-ptxas]

The library is written next to the Python package (``rbsim/librbsim.so``) so it
travels with the source tree. Flags that carry meaning:

* ``-gencode arch=compute_100a,code=sm_100a`` -- B200 only, no other targets;
* ``--fmad=false`` with the default IEEE division and square root -- one rounding
  per operation in source order, the arithmetic contract the kernels share with
  the CPU oracle (``include/rb_detmath.h`` supplies the fractional powers);
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

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "rbsim", "librbsim.so")


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build librbsim.so")


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.h*")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    cmd = [
        nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "--fmad=false",
        "-std=c++17", "-cudart", "static", "-Xcompiler", "-fPIC,-O2", "-shared",
        "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-o", OUT + ".tmp",
    ]  # fmt: skip
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    cmd += sources()
    subprocess.run(cmd, check=True)
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
