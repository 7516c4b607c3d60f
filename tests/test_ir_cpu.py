"""The law front-end and IR lowering against the reference's own IR (golden JSON from the reference's lawc), and the
generated CUDA compiling for sm_100a under NVRTC. No GPU needed."""
import glob
import json
import os

import pytest

from conftest import ROOT

LAWS = sorted(glob.glob(os.path.join(ROOT, "tests", "laws", "*.law")))


@pytest.mark.parametrize("law", LAWS, ids=lambda p: os.path.basename(p))
def test_ir_json_matches_reference(law, monkeypatch):
    from fieldcuda import solver
    monkeypatch.chdir(ROOT)  # a net's weight file path is relative to the working directory (loaded: true there)
    mine = json.loads(solver.ir_json(open(law).read()))
    ref = json.load(open(os.path.join(ROOT, "tests", "golden", "ir", os.path.basename(law)[:-4] + ".json")))
    assert mine == ref


@pytest.mark.parametrize("law", LAWS, ids=lambda p: os.path.basename(p))
def test_generated_cuda_compiles_for_sm100a(law):
    from fieldcuda import solver
    solver.compile_check(open(law).read(), 20, 14, 9, 0.5)


def test_reference_bench_laws_lower_identically():
    """Where the reference's sources are at hand (this build's container), its own benchmark laws and its 43-term world
    law lower to the same IR as its lawc prints."""
    import subprocess
    lawc = os.path.join(ROOT, "oracle", "_ref", "lawc")
    where = os.path.join(ROOT, "oracle", "_ref", "REFERENCE")  # the checkout oracle/Makefile built lawc from
    ref_root = open(where).read().strip() if os.path.exists(where) else ""
    if not (os.path.exists(lawc) and ref_root and os.path.isdir(ref_root)):
        pytest.skip("the reference's sources and lawc are not here")
    from fieldcuda import solver
    sets = [[p] for p in sorted(glob.glob(os.path.join(ref_root, "bench", "laws", "*.law")))]
    sets.append([os.path.join(ref_root, "assets", "law", "world.law"), os.path.join(ref_root, "assets", "law", "magic.law")])
    for paths in sets:
        out = "/tmp/fe_ref_ir.json"
        subprocess.run([lawc, "--ir-json", out] + paths, check=True, capture_output=True)
        ref = json.load(open(out))
        for n in ref["nets"]:
            n["loaded"] = False
        mine = json.loads(solver.ir_json("".join(open(p).read() + "\n" for p in paths)))
        assert mine == ref, paths
        # The same IR taken in as IR (fe_law_create_ir's ingest) is the same law.
        assert ir_check(json.dumps(ref)) == ref, paths


IRS = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "ir", "*.json")))


def ir_check(text):
    import ctypes
    from fieldcuda import _lib
    lib = _lib.lib()
    need = ctypes.c_size_t()
    _lib.check(lib.fe_law_ir_check(text.encode(), None, 0, ctypes.byref(need)))
    buf = ctypes.create_string_buffer(need.value)
    _lib.check(lib.fe_law_ir_check(text.encode(), buf, need.value, ctypes.byref(need)))
    return json.loads(buf.value.decode())


@pytest.mark.parametrize("path", IRS, ids=lambda p: os.path.basename(p))
def test_law_given_as_the_references_ir_is_the_same_law(path, monkeypatch):
    """fe_law_create_ir's ingest: the reference's IR JSON (made by its lawc) rebuilt into a law and lowered again gives
    that JSON back, instruction for instruction (folded-away numbers included) and program for program."""
    monkeypatch.chdir(ROOT)  # net weight files named in the IR are repository paths
    text = open(path).read()
    assert ir_check(text) == json.loads(text)


def test_ir_ingest_refuses_what_it_cannot_take():
    from fieldcuda import _lib
    text = open(os.path.join(ROOT, "tests", "golden", "ir", "heat.json")).read()
    for bad in ("{", "[]", text.replace('"version":1', '"version":2'), text.replace('"op":"diffuse"', '"op":"sprinkle"')):
        with pytest.raises(_lib.FeError) as e:
            ir_check(bad)
        assert e.value.code == _lib.FE_ELAW
    # An edited program (its stage list) no longer matches what its instructions lower to.
    doc = json.loads(open(os.path.join(ROOT, "tests", "golden", "ir", "heston_douglas.json")).read())
    doc["terms"][0]["stages"] = doc["terms"][0]["stages"][:-1]
    with pytest.raises(_lib.FeError, match="does not lower back"):
        ir_check(json.dumps(doc))


def test_law_errors_match_the_reference_word_for_word():
    """Malformed laws give the reference lawc's own error lines, in its order (tests/golden/law_errors.json, made by
    it): the messages are part of the language's interface."""
    from fieldcuda import _lib, solver
    cases = json.load(open(os.path.join(ROOT, "tests", "golden", "law_errors.json")))
    assert len(cases) >= 20
    for case in cases:
        assert case["rc"] != 0 and case["errors"]
        with pytest.raises(_lib.FeError) as e:
            solver.ir_json(case["law"])
        got = [line for line in str(e.value).splitlines() if line.startswith("law:") or "] law:" in line]
        got = [line[line.index("law:"):] for line in got]
        assert got == case["errors"], case["law"]


def test_law_errors_name_the_line():
    from fieldcuda import _lib, solver
    with pytest.raises(_lib.FeError) as e:
        solver.ir_json("field T init 0\nterm t\n  d T = nosuch(T)\n")
    assert e.value.code == _lib.FE_ELAW and "law:3" in str(e.value) and "unknown function" in str(e.value)
    with pytest.raises(_lib.FeError):
        solver.ir_json("field T init 0 static\nterm t\n  d T = 1\n")  # writes a static field


def test_bad_net_files_are_refused_not_faked(monkeypatch):
    from fieldcuda import _lib, solver
    monkeypatch.chdir(ROOT)
    # fx's file holds a 2-16-16-1 net: a law declaring another shape for it does not compile
    law = "field T init 290 range 0 6000\nnet fx in 2 hidden 8 out 1 act tanh file tests/laws/nets/fx\nterm t\n  d T = mlp(fx, T, T)\n"
    with pytest.raises(_lib.FeError) as e:
        solver.compile_check(law, 8, 8, 8, 1.0)
    assert e.value.code == _lib.FE_ELAW and "sizes" in str(e.value)
    # distance, poisson and the net ops are run (not refused); a net without a file starts untrained
    solver.compile_check("field s init 0\nfield q init 0\nterm t\n  d q = distance(s) - q + poisson(s, 5)\n", 8, 8, 8, 1.0)
    law = "field T init 290 range 0 6000\nnet ld in 5 hidden 8 out 4 act tanh file none\nterm t\n  d T = ldiffuse(ld, 0.8, T)\n"
    solver.compile_check(law, 8, 8, 8, 1.0)