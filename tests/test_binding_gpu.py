"""The drop-in boundary at the C++ level: the reference's own Solver (its src/field/Solver.cpp, unmodified) running on
this backend through the reference's LawBackend interface, with online-physics-cuda_b200/binding/B200Solver.cpp in
place of the reference's CUDA backend, held to the reference's CPU Solver (tests/binding/gate.cpp, built against the
reference's headers and objects by `make -C oracle binding` into oracle/_ref/b200_gate).

Checks: every golden law from its golden starting state within the reference's gates (1e-6 heat, 2e-5 one op, 1e-4 a
whole law: src/tests/cuda_parity_smoke.cpp:114-117, 159-160) with the same substeps and two runs equal to the bit; the
reference's shipped world law on its fire_test scene (its own gate, 1e-4); every op alone; a moved window (only the
arriving boxes uploaded) equal to the bit to the window uploaded whole; lazy readback equal to the bit to fetching
every step; the idle-term bounds never short."""
import glob
import json
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GATE = os.path.join(ROOT, "oracle", "_ref", "b200_gate")
ASSETS = os.path.join(ROOT, "oracle", "_ref", "assets")
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))
TOLERANCE = {"heat_24": 1e-6, "ops_stencil": 2e-5, "ops_stencil_wide": 2e-5, "ops_matter": 2e-5, "cn_64": 2e-5,
             "implicit_yz": 2e-5, "op_distance": 2e-5, "op_poisson": 2e-5}
# Nets declared `half` are not in these laws; the fp32 nets' tanh/exp differ from the C library's by a few ulps.


def gate(*args):
    if not os.path.exists(GATE):
        pytest.skip("oracle/_ref/b200_gate is not built (the reference's sources were not at hand when building)")
    res = subprocess.run([GATE, *args], capture_output=True, text=True, cwd=ROOT, timeout=900)
    checks = [json.loads(line) for line in res.stdout.splitlines() if line.startswith("{")]
    assert checks, res.stdout + res.stderr
    bad = [c for c in checks if not c["ok"]]
    assert not bad and res.returncode == 0, (bad, res.stderr[-2000:])
    return checks


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_reference_solver_on_this_backend_matches_its_cpu_solver(cuda, path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    work = tempfile.mkdtemp(prefix="fe_gate_")
    try:
        for k in z.files:
            if k.startswith("init_"):
                np.ascontiguousarray(z[k], np.float32).tofile(os.path.join(work, k[5:] + ".bin"))
        nz, ny, nx = meta["shape"]
        tol = TOLERANCE.get(meta["name"], 1e-4)
        checks = gate("parity", os.path.join("tests", "laws", meta["law"]), "--grid", str(nx), str(ny), str(nz),
                      repr(meta["h"]), "--dt", repr(meta["dt"]), "--steps", str(meta["steps"]), "--tol", repr(tol),
                      "--init", work)
        assert {c["check"] for c in checks} == {"parity", "deterministic"}
    finally:
        shutil.rmtree(work, ignore_errors=True)


def test_reference_world_law_on_this_backend(cuda):
    if not os.path.exists(os.path.join(ASSETS, "world.law")):
        pytest.skip("the reference's world law was not copied into oracle/_ref/assets when building")
    checks = gate("world", ASSETS)
    assert any(c["check"].startswith("world law within") for c in checks)


@pytest.mark.parametrize("mode", ["ops", "window", "lazy", "bounds"])
def test_reference_solver_scenarios_on_this_backend(cuda, mode):
    gate(mode)
