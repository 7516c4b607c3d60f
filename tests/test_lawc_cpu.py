"""The lawc command line on this backend (fieldcuda.lawc), without a GPU: scenes in the reference's text format make
the same starting state as the reference's lawc (bit for bit, tests/golden/scene/ made by it), the IR outputs, and what
it refuses."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT


def fixture(name):
    z = np.load(os.path.join(ROOT, "tests", "golden", "scene", name + ".npz"))
    return json.loads(str(z["meta"])), z


def test_scene_ops_make_the_reference_starting_state():
    from fieldcuda import lawc
    from fieldcuda.solver import ir_json
    meta, z = fixture("ops")
    scene = lawc.load_scene(os.path.join(ROOT, "tests", "scenes", "ops.scene"))
    assert scene.grid == (20, 14, 9, 0.5) and len(scene.ops) == 5
    law = open(os.path.join(ROOT, scene.laws[0])).read()
    inits = {f["name"]: f["init"] for f in json.loads(ir_json(law))["fields"]}
    got = lawc.scene_fields(scene, list(inits), inits)
    for name in meta["fields"]:
        want = z[f"step0_{name}"]
        assert np.array_equal(got[name].view(np.uint32), want.view(np.uint32)), name


def test_scene_guarded_makes_the_reference_starting_state():
    from fieldcuda import lawc
    from fieldcuda.solver import ir_json
    meta, z = fixture("guarded")
    scene = lawc.load_scene(os.path.join(ROOT, "tests", "scenes", "guarded.scene"))
    law = open(os.path.join(ROOT, scene.laws[0])).read()
    inits = {f["name"]: f["init"] for f in json.loads(ir_json(law))["fields"]}
    got = lawc.scene_fields(scene, list(inits), inits)
    assert np.array_equal(got["T"].view(np.uint32), z["step0_T"].view(np.uint32))


def test_noise_is_a_pure_function_of_seed_and_cell():
    from fieldcuda.lawc import cell_noise
    idx = np.arange(1000, dtype=np.uint64)
    a, b = cell_noise(7, idx), cell_noise(7, idx)
    assert np.array_equal(a, b) and 0.0 <= a.min() and a.max() < 1.0 and abs(a.mean() - 0.5) < 0.05
    assert not np.array_equal(a, cell_noise(8, idx))


def test_ir_outputs_and_refusals(tmp_path):
    from fieldcuda import lawc
    law = os.path.join(ROOT, "tests", "laws", "ops_fields.law")
    out = tmp_path / "ir.json"
    assert lawc.main(["--ir-json", str(out), law]) == 0
    want = open(os.path.join(ROOT, "tests", "golden", "ir", "ops_fields.json")).read()
    assert json.loads(out.read_text()) == json.loads(want)
    adj = tmp_path / "adj.law"
    assert lawc.main(["--adjoint", str(adj), os.path.join(ROOT, "tests", "laws", "heat.law")]) == 0
    assert "T__adj" in adj.read_text()
    assert lawc.main(["--backend", "cpu", law]) == 1
    assert lawc.main(["--compare", "--steps", "1", law]) == 2
    bad = tmp_path / "bad.scene"
    bad.write_text("grid 4 4 4 1\nsprinkle T 1\n")
    with pytest.raises(ValueError, match="unknown line 'sprinkle'"):
        lawc.load_scene(str(bad))


def test_untrained_nets_are_noted(capsys):
    from fieldcuda import lawc
    assert lawc.main(["--ir", os.path.join(ROOT, "tests", "laws", "guarded_heat.law")]) == 0
    assert "note: net 'lh' has no weights at none (it starts untrained: its output is 0)" in capsys.readouterr().err
