"""The lawc command line on this backend, end to end on the GPU: a scene in the reference's format run for a few steps,
dumped in its format, against the reference's lawc on the same scene (tests/golden/scene/)."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_scene_run_matches_the_reference_lawc(cuda, tmp_path, monkeypatch):
    from fieldcuda import lawc
    z = np.load(os.path.join(ROOT, "tests", "golden", "scene", "ops.npz"))
    meta = json.loads(str(z["meta"]))
    monkeypatch.chdir(ROOT)  # the scene's law path is the repository's
    dump, js = tmp_path / "dump", tmp_path / "t.json"
    rc = lawc.main(["--scene", "tests/scenes/ops.scene", "--steps", str(meta["steps"]), "--dt", repr(meta["dt"]), "--dump", str(dump),
                    "--json", str(js)])
    assert rc == 0
    out = json.loads(js.read_text())
    assert out["substeps"] == meta["substeps"] and out["violations"] == meta["violations"] == 0
    dmeta = json.loads((dump / "step_0" / "meta.json").read_text())
    assert dmeta["fields"] == meta["fields"] and (dmeta["nx"], dmeta["ny"], dmeta["nz"]) == (20, 14, 9)
    for name in meta["fields"]:
        start = np.fromfile(dump / "step_0" / f"{name}.bin", np.float32).reshape(9, 14, 20)
        assert np.array_equal(start.view(np.uint32), z[f"step0_{name}"].view(np.uint32)), name
        got = np.fromfile(dump / f"step_{meta['steps']}" / f"{name}.bin", np.float32).reshape(9, 14, 20).astype(np.float64)
        want = z[f"step{meta['steps']}_{name}"].astype(np.float64)
        assert np.abs(got - want).max() <= 1e-4 * max(np.abs(want).max(), 1e-6), name


def test_learned_run_counts_the_undone_steps(cuda, tmp_path, monkeypatch, capsys):
    from fieldcuda import lawc
    monkeypatch.chdir(ROOT)
    js = tmp_path / "g.json"
    rc = lawc.main(["--scene", "tests/scenes/guarded.scene", "--steps", "30", "--dt", "0.3", "--learned", "--profile",
                    "--json", str(js)])
    assert rc == 0
    out = json.loads(js.read_text())
    printed = capsys.readouterr().out
    assert "1 fields, 1 terms, 1 nets" in printed
    assert out["violations"] == 0 and 0 < out["fallbacks"] <= 30
    assert "learned step(s) undone" in printed
    rc = lawc.main(["--scene", "tests/scenes/guarded.scene", "--steps", "5", "--dt", "0.3", "--json", str(js)])
    assert rc == 0 and json.loads(js.read_text())["fallbacks"] == 0


def test_vjp_matches_the_oracle_reverse_pass(cuda, tmp_path, monkeypatch):
    """lawc --vjp (the native checkpointed driver) against the oracle keeping every state and running the same adjoint
    law back over them, as the reference's lawc --vjp does."""
    from fieldcuda import _lib, lawc
    from fieldcuda.adjoint import adjoint_law
    from oracle import law_cpu
    monkeypatch.chdir(ROOT)
    scene = lawc.load_scene("tests/scenes/heat_vjp.scene")
    nx, ny, nz, h = scene.grid
    law = open("tests/laws/heat.law").read()
    steps, dt = 12, 0.4 * h * h / 6.0 * 0.9
    rng = np.random.default_rng(11)
    seed = rng.normal(size=(nz, ny, nx)).astype(np.float32)
    (tmp_path / "seed").mkdir()
    seed.tofile(tmp_path / "seed" / "T__adj.bin")
    rc = lawc.main(["--scene", "tests/scenes/heat_vjp.scene", "--steps", str(steps), "--dt", repr(dt), "--vjp",
                    str(tmp_path / "seed"), "--dump", str(tmp_path / "out")])
    assert rc == 0
    got = np.fromfile(tmp_path / "out" / "adjoint" / "T__adj.bin", np.float32).reshape(nz, ny, nx).astype(np.float64)

    def solver(text, fields):
        ir = json.loads(_lib.text_call("fe_law_ir_json", text.encode()))
        s = law_cpu.Solver(law_cpu.Law(ir), (nz, ny, nx), h)
        for k, v in fields.items():
            s.fields[k] = np.asarray(v, law_cpu.F32).copy()
        return s
    start = lawc.scene_fields(scene, ["T"], {"T": 0.0})
    o = solver(law, start)
    states = []
    for _ in range(steps):
        states.append(o.fields["T"].copy())
        o.step(dt)
    a = solver(adjoint_law(law), dict(start, T__adj=seed))
    for s in range(steps - 1, -1, -1):
        a.fields["T"] = states[s]
        a.step(dt)
    want = a.fields["T__adj"].astype(np.float64)
    assert float(np.abs(got - want).max()) <= 1e-4 * float(np.abs(want).max())


def test_guarded_scene_matches_the_reference_lawc(cuda, tmp_path, monkeypatch):
    """lawc --learned on the guarded scene against the reference's lawc --learned (tests/golden/scene/guarded.npz): the
    guard undoes the same learned steps (the count), and the state they leave agrees to the whole-law gate."""
    from fieldcuda import lawc
    z = np.load(os.path.join(ROOT, "tests", "golden", "scene", "guarded.npz"))
    meta = json.loads(str(z["meta"]))
    monkeypatch.chdir(ROOT)
    dump, js = tmp_path / "dump", tmp_path / "g.json"
    rc = lawc.main(["--scene", "tests/scenes/guarded.scene", "--steps", str(meta["steps"]), "--dt", repr(meta["dt"]), "--learned",
                    "--dump", str(dump), "--every", str(meta["steps"]), "--json", str(js)])
    assert rc == 0
    out = json.loads(js.read_text())
    assert out["fallbacks"] == meta["fallbacks"] and out["violations"] == meta["violations"] == 0
    got = np.fromfile(dump / f"step_{meta['steps']}" / "T.bin", np.float32).reshape(z["step30_T"].shape).astype(np.float64)
    want = z["step30_T"].astype(np.float64)
    assert float(np.abs(got - want).max()) <= 1e-4 * float(np.abs(want).max())
