"""Pins the oracle: its restatement of the reference's CPU solver against the reference's own outputs (golden fixtures
made by the reference's lawc), bit for bit, and the heat restatement against it."""
import glob
import json
import os

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))


def load(path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    return meta, {k[5:]: z[k] for k in z.files if k.startswith("init_")}, {k[6:]: z[k] for k in z.files if k.startswith("final_")}


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_reproduces_reference_solver(path, monkeypatch):
    from oracle import law_cpu
    monkeypatch.chdir(ROOT)  # net weight files are found from the repository root, as the fixtures were made
    meta, init, final = load(path)
    ir = json.load(open(os.path.join(ROOT, "tests", "golden", "ir", meta["law"][:-4] + ".json")))
    law = law_cpu.Law(ir)
    s = law_cpu.Solver(law, tuple(meta["shape"]), meta["h"])
    for k, v in init.items():
        s.fields[k] = v.copy()
    for _ in range(meta["steps"]):
        s.step(meta["dt"])
    assert s.substeps == meta["substeps"]
    # A net's tanh/exp come from numpy here and from the C library there: a net law is held to a few units in the last
    # place, every other law to the bit.
    ulps = 4 if meta["law"].startswith("nets_") else 0
    for name, want in final.items():
        got = s.fields[name]
        apart = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64)).max()
        assert apart <= ulps, f"{meta['name']}:{name} differs by {np.abs(got.astype(np.float64) - want).max()} ({apart} ulps)"


def test_heat_restatement_matches_the_law_oracle():
    from oracle import heat as oh
    from oracle import law_cpu
    ir = json.load(open(os.path.join(ROOT, "tests", "golden", "ir", "heat.json")))
    n, h = 20, 1.0 / 20
    dt = 0.4 * h * h / 6.0
    T0 = oh.gaussian_blobs(n, h, seed=5)
    s = law_cpu.Solver(law_cpu.Law(ir), (n, n, n), h)
    s.fields["T"] = T0.copy()
    s.step(dt)
    assert np.array_equal(s.fields["T"].view(np.uint32), oh.cpu_step(T0, 1.0, h, dt).view(np.uint32))


def test_c1_fixture_against_the_fp32_restatement():
    """The full-size heat fixture (128^3, 100 steps; tests/golden/large/c1_heat_128.npz, made by the reference's lawc)
    against the restatement of the generated kernel's FP32 arithmetic over the same 100 steps: within the 1e-6 the GPU
    test holds the engine to, and the FP64 solve in the fixture within the same bound of both."""
    from oracle import heat as oh
    z = np.load(os.path.join(ROOT, "tests", "golden", "large", "c1_heat_128.npz"))
    meta = json.loads(str(z["meta"]))
    n, h, dt = meta["n"], meta["h"], meta["dt"]
    T = oh.gaussian_blobs(n, h, seed=0)
    for _ in range(meta["steps"]):
        T = oh.gpu_order_step(T, 1.0, h, dt)
    p = z["pick"]
    ix = np.ix_(p, p, p)
    assert float(np.abs(T[ix].astype(np.float64) - z["ref_T"]).max()) / meta["max_abs"]["T"] <= 1e-6
    assert float(np.abs(T[z["planes"]].astype(np.float64) - z["refplanes_T"]).max()) / meta["max_abs"]["T"] <= 1e-6
    assert float(np.abs(T[ix].astype(np.float64) - z["fp64_T"]).max()) / meta["max_abs"]["fp64_T"] <= 1e-6
    assert float(np.abs(z["ref_T"].astype(np.float64) - z["fp64_T"]).max()) / meta["max_abs"]["fp64_T"] <= 1e-6


def test_reverse_pass_reproduces_the_reference_vjp():
    """The adjoint law this backend builds (fe_law_adjoint), run by the oracle back over every kept state, against the
    reference's own lawc --vjp on the same scene and seed (tests/golden/scene/heat_vjp.npz): bit for bit, for the
    state's cotangent and the param's."""
    from fieldcuda import _lib, lawc
    from fieldcuda.adjoint import adjoint_law
    from oracle import law_cpu
    z = np.load(os.path.join(ROOT, "tests", "golden", "scene", "heat_vjp.npz"))
    meta = json.loads(str(z["meta"]))
    scene = lawc.load_scene(os.path.join(ROOT, "tests", "scenes", meta["scene"]))
    nx, ny, nz, h = scene.grid
    law = open(os.path.join(ROOT, "tests", "laws", "heat.law")).read()

    def solver(text, fields):
        s = law_cpu.Solver(law_cpu.Law(json.loads(_lib.text_call("fe_law_ir_json", text.encode()))), (nz, ny, nx), h)
        for k, v in fields.items():
            s.fields[k] = np.asarray(v, law_cpu.F32).copy()
        return s
    start = lawc.scene_fields(scene, ["T"], {"T": 0.0})
    o = solver(law, start)
    states = []
    for _ in range(meta["steps"]):
        states.append(o.fields["T"].copy())
        o.step(meta["dt"])
    a = solver(adjoint_law(law), dict(start, T__adj=z["seed"]))
    for s in range(meta["steps"] - 1, -1, -1):
        a.fields["T"] = states[s]
        a.step(meta["dt"])
    for name in ("T__adj", "D__adj"):
        assert np.array_equal(a.fields[name].view(np.uint32), z[name].view(np.uint32)), name
