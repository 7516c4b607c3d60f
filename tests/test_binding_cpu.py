"""The reference-side binding builds: tests/binding/gate.cpp and online-physics-cuda_b200/binding/B200Solver.cpp
compiled against the reference's headers and linked with its objects and libfe_b200.so (oracle/Makefile `binding`).
No device needed: the gate's usage answer, and that it resolves this repository's library."""
import os
import subprocess

import pytest

from conftest import ROOT

GATE = os.path.join(ROOT, "oracle", "_ref", "b200_gate")


def test_gate_links_this_backend():
    if not os.path.exists(GATE):
        pytest.skip("oracle/_ref/b200_gate is not built (the reference's sources were not at hand when building)")
    res = subprocess.run([GATE], capture_output=True, text=True, timeout=60)
    assert res.returncode == 2 and "usage" in res.stderr
    libs = subprocess.run(["ldd", GATE], capture_output=True, text=True).stdout
    want = os.path.realpath(os.path.join(ROOT, "online-physics-cuda_b200", "libfe_b200.so"))
    assert any(want in os.path.realpath(line.split("=>")[1].split()[0]) for line in libs.splitlines()
               if "libfe_b200" in line and "=>" in line), libs
