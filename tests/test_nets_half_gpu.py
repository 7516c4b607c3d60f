"""Nets declared `half` on the tensor cores (tcgen05, BF16 operands, FP32 accumulators), against the same laws' fp32
nets and the reference's CPU solver. The reference's gate for its tensor-core nets (src/tests/nets_smoke.cpp:154-190):
after a step, |T_gpu - T_cpu| <= 0.03 * (what the step moved) + 1e-3, and a conserving learned flux keeps the total
to 1e-6 relative."""
import glob
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CASES = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "nets_*.npz")))


def half(text):
    """The law with every net declared `half` (net NAME ... act A half file PATH)."""
    out = []
    for line in text.splitlines():
        if line.startswith("net ") and " half" not in line:
            line = line.replace(" file ", " half file ") if " file " in line else line + " half"
        out.append(line)
    return "\n".join(out) + "\n"


def load(path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    init = {k[5:]: z[k] for k in z.files if k.startswith("init_")}
    final = {k[6:]: z[k] for k in z.files if k.startswith("final_")}
    return meta, init, final


def solve(text, meta, init, steps):
    from fieldcuda.solver import Solver
    nz, ny, nx = meta["shape"]
    s = Solver(text, nx, ny, nz, meta["h"], meta["law"])
    for name, arr in init.items():
        s.set_field(name, arr)
    for _ in range(steps):
        s.step(meta["dt"])
    return s


@pytest.mark.parametrize("path", CASES, ids=lambda p: os.path.basename(p)[:-4])
def test_half_nets_hold_to_the_cpu_to_bf16(cuda, path, monkeypatch):
    from fieldcuda.solver import cuda_source
    monkeypatch.chdir(ROOT)  # the laws' weight files are repository paths
    meta, init, final = load(path)
    text = open(os.path.join(ROOT, "tests", "laws", meta["law"])).read()
    nz, ny, nx = meta["shape"]
    assert "fe_net_pass<" in cuda_source(half(text), nx, ny, nz, meta["h"])
    # One step against the fp32 nets on the card.
    a, b = solve(half(text), meta, init, 1), solve(text, meta, init, 1)
    for name in init:
        before = init[name].astype(np.float64)
        want = b.values(name).astype(np.float64)
        moved = float(np.abs(want - before).max())
        worst = float(np.abs(a.values(name).astype(np.float64) - want).max())
        assert worst <= 0.03 * moved + 1e-3, f"{name}: {worst:.3g} of a step that moved {moved:.3g}"
    assert a.violations() == [] and a.last_substeps() == meta["substeps"]
    a.close()
    b.close()
    # The fixture's steps against the reference's CPU solver.
    s = solve(half(text), meta, init, meta["steps"])
    for name, want in final.items():
        want = want.astype(np.float64)
        moved = float(np.abs(want - init[name]).max())
        worst = float(np.abs(s.values(name).astype(np.float64) - want).max())
        assert worst <= 0.03 * moved + 1e-3, f"{name}: {worst:.3g} of steps that moved {moved:.3g}"
    assert s.violations() == []
    s.close()


@pytest.mark.parametrize("law", ["nets_flux.law", "nets_ldiffuse.law"])
def test_half_learned_fluxes_keep_the_total(cuda, law, monkeypatch):
    monkeypatch.chdir(ROOT)
    meta, init, _ = load(os.path.join(ROOT, "tests", "golden", law[:-4] + "_wide.npz"))
    text = half(open(os.path.join(ROOT, "tests", "laws", law)).read())
    s = solve(text, meta, init, 5)
    t0 = float(init["T"].astype(np.float64).sum())
    t1 = float(s.values("T").astype(np.float64).sum())
    assert abs(t1 - t0) / abs(t0) < 1e-6, (t0, t1)
    assert s.violations() == []
    s.close()


def test_half_step_is_deterministic(cuda, monkeypatch):
    monkeypatch.chdir(ROOT)
    meta, init, _ = load(os.path.join(ROOT, "tests", "golden", "nets_ldiffuse_wide.npz"))
    text = half(open(os.path.join(ROOT, "tests", "laws", "nets_ldiffuse.law")).read())
    a, b = solve(text, meta, init, 3), solve(text, meta, init, 3)
    assert a.digest() == b.digest()
    a.close()
    b.close()


@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 2, 3), (3, 5, 7), (2, 3, 130), (2, 1, 129)], ids=str)
def test_half_nets_on_ragged_lattices(cuda, shape, monkeypatch):
    """Lattices smaller than one 128-cell tile, partial last tiles and flat axes (closed faces): the tensor-core stage
    against the fp32 one, the same gate."""
    monkeypatch.chdir(ROOT)
    rng = np.random.default_rng(sum(shape))
    for law in ("nets_mlp.law", "nets_flux.law", "nets_ldiffuse.law"):
        text = open(os.path.join(ROOT, "tests", "laws", law)).read()
        meta = {"shape": list(shape), "h": 0.5, "law": law, "dt": 0.02}
        init = {"T": (290 + 600 * rng.random(shape)).astype(np.float32)}
        if "fuel" in text:
            init["fuel"] = rng.random(shape).astype(np.float32)
        a, b = solve(half(text), meta, init, 1), solve(text, meta, init, 1)
        before = init["T"].astype(np.float64)
        want = b.values("T").astype(np.float64)
        moved = float(np.abs(want - before).max())
        worst = float(np.abs(a.values("T").astype(np.float64) - want).max())
        assert worst <= 0.03 * moved + 1e-3, (law, worst, moved)
        assert a.violations() == []
        a.close()
        b.close()
