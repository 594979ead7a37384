"""The product package never reaches the oracle, and has no CPU fallback.

The oracle is the checker. Nothing under river-basin-sim_b200/ may import it, link
it or run it. The solver path must refuse to run, loudly, when its CUDA library or a
CUDA device is missing, rather than fall back to anything else.
"""

from __future__ import annotations

import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "river-basin-sim_b200")


def test_no_product_source_names_the_oracle():
    pattern = re.compile(r"^\s*(import\s+oracle|from\s+oracle\b)|librbo_|rbo_[a-z_]+_f(32|64)", re.M)
    hits = []
    for dirpath, _, files in os.walk(PKG):
        if "_build" in dirpath:
            continue
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".c")):
                path = os.path.join(dirpath, f)
                with open(path, encoding="utf-8") as fh:
                    if pattern.search(fh.read()):
                        hits.append(os.path.relpath(path, ROOT))
    assert hits == []


def test_importing_every_product_module_loads_no_oracle():
    """In a fresh interpreter: the whole package imports without pulling in the oracle."""
    mods = ["rbsim", "rbsim.run", "rbsim.serve", "rbsim.ensemble", "rbsim.device_clock", "rbsim.replicas",
            "rbsim.arith", "rbsim.channels", "rbsim.sediment", "rbsim.massbalance", "rbsim.config",
            "rbsim.processes.inflow", "rbsim.processes.morphology", "rbsim.processes.reservoir",
            "rbsim.io.zarr_writer", "rbsim.io.status", "rbsim.io.viewer_export", "rbsim.schemes.hllc",
            "rbsim.schemes.local_inertial"]  # fmt: skip
    code = ("import importlib, sys\n"
            f"sys.path.insert(0, {PKG!r})\n"
            f"for m in {mods!r}: importlib.import_module(m)\n"
            "bad = sorted(m for m in sys.modules if m == 'oracle' or m.startswith('oracle.'))\n"
            "print(bad)\n")  # fmt: skip
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "[]"


def test_the_library_links_no_oracle():
    from rbsim import _lib

    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("librbsim.so is not built")
    deps = subprocess.run(["ldd", _lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "librbo" not in deps


def test_a_missing_library_is_an_error_not_a_fallback(monkeypatch):
    from rbsim import _lib

    monkeypatch.setattr(_lib, "_LIB", None)
    monkeypatch.setattr(_lib, "LIB_PATH", os.path.join(ROOT, "no_such_dir", "librbsim.so"))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.lib()


def test_a_state_refuses_the_cpu_device():
    import torch

    import rbsim

    with pytest.raises((ValueError, RuntimeError), match="CUDA|no CPU fallback"):
        rbsim.State.from_bed(np.zeros((4, 4), np.float32), 10.0, device="cpu")
    if not torch.cuda.is_available():  # with no device, the default CUDA state refuses too
        with pytest.raises(RuntimeError, match="no CPU fallback"):
            rbsim.State.from_bed(np.zeros((4, 4), np.float32), 10.0)
