"""Every law of the golden cases on degenerate lattices, the CUDA path against the oracle: one cell, one row, a single
row 128 cells wide (the TMA slab pass with one live row), x extents that leave a partial 128-cell tile, and flat axes.
The starting values are drawn from the case's own starting state, so they lie where the law was exercised."""
import glob
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CASES = [p for p in sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz"))) if not p.endswith("_wide.npz")]
SHAPES = [(1, 1, 1), (2, 1, 128), (1, 3, 132), (3, 2, 7)]
TOLERANCE = 1e-4  # the reference's whole-law gate (src/tests/cuda_parity_smoke.cpp:159-160)


@pytest.mark.parametrize("shape", SHAPES, ids=str)
@pytest.mark.parametrize("path", CASES, ids=lambda p: os.path.basename(p)[:-4])
def test_degenerate_lattices_match_the_oracle(cuda, path, shape, monkeypatch):
    from fieldcuda.solver import Solver
    from oracle import law_cpu
    monkeypatch.chdir(ROOT)  # net weight files are repository paths
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    rng = np.random.default_rng(sum(shape) + len(meta["name"]))
    init = {k[5:]: rng.choice(z[k].ravel(), size=shape).astype(np.float32) for k in z.files if k.startswith("init_")}
    text = open(os.path.join(ROOT, "tests", "laws", meta["law"])).read()
    ir = json.load(open(os.path.join(ROOT, "tests", "golden", "ir", meta["law"][:-4] + ".json")))
    nz, ny, nx = shape
    s = Solver(text, nx, ny, nz, meta["h"], meta["law"])
    o = law_cpu.Solver(law_cpu.Law(ir), shape, meta["h"])
    for k, v in init.items():
        s.set_field(k, v)
        o.fields[k] = v.copy()
    for _ in range(2):
        s.step(meta["dt"])
        o.step(meta["dt"])
    # A term whose bounds say it is idle (a lone cell's diffusion) reports one substep and is skipped, as the reference's
    # Solver does (src/field/Solver.cpp:341-347); the oracle restates the arithmetic only and counts substeps anyway.
    want_substeps = [1 if idle else n for idle, n in zip(s.idle_terms(), o.substeps)]
    assert s.last_substeps() == want_substeps, (s.last_substeps(), o.substeps, s.idle_terms())
    for name in s.field_names:
        if name not in o.fields:
            continue
        got = s.values(name).astype(np.float64)
        want = o.fields[name].astype(np.float64)
        scale = max(float(np.abs(want).max()), 1e-6)
        assert float(np.abs(got - want).max()) <= TOLERANCE * scale, (meta["name"], name, float(np.abs(got - want).max()), scale)
    s.close()
