"""The benchmarked configurations pinned at their full size, not only on toy lattices.

C1 as stated: the heat law on 128^3 (h = 1/128, dt = 0.4 h^2 / 6, one substep), four seeded Gaussian blobs, 100 steps
with the contracts checked every step. The engine's generated step must equal the hand-written kernel's to the bit
after every one of the 100 steps (the reference's own engine-vs-kernel check, bench/stencil_bench.cpp:291-294), stay
within 1e-6 relative (max |difference| / max |T|, as src/tests/cuda_parity_smoke.cpp:56-71) of the reference's CPU
solver (tests/golden/large/c1_heat_128.npz, made by its lawc; the whole field too when that lawc is built in
oracle/_ref), and two runs must agree to the bit. Its error against the same scheme solved in FP64 is stated and bounded.

The 43-term, 6-field law on 128^3 over 3 steps, against the reference's CPU solver within its whole-law gate (1e-4,
src/tests/cuda_parity_smoke.cpp:114-117).
"""
import json
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(ROOT, "tests", "golden", "large")
LAWC = os.path.join(ROOT, "oracle", "_ref", "lawc")


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return json.loads(str(z["meta"])), z


def reference_full(meta, fields):
    """The reference's lawc run on the whole lattice (when it is built in oracle/_ref), else None."""
    if not os.path.exists(LAWC):
        return None
    n, h = meta["n"], meta["h"]
    work = tempfile.mkdtemp(prefix="fe_c1_")
    try:
        scene = os.path.join(work, "scene")
        with open(scene, "w") as f:
            f.write(f"grid {n} {n} {n} {h!r}\nlaw {os.path.join(ROOT, 'tests', 'laws', meta['law'])}\n")
        init = os.path.join(work, "init")
        os.makedirs(init)
        for k, v in fields.items():
            np.ascontiguousarray(v, np.float32).tofile(os.path.join(init, k + ".bin"))
        dump = os.path.join(work, "dump")
        subprocess.run([LAWC, "--scene", scene, "--init", init, "--steps", str(meta["steps"]), "--dt", repr(meta["dt"]),
                        "--dump", dump, "--every", str(meta["steps"])], check=True, capture_output=True,
                       env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 4)))
        last = os.path.join(dump, f"step_{meta['steps']}")
        return {k: np.fromfile(os.path.join(last, k + ".bin"), np.float32).reshape(n, n, n) for k in fields}
    finally:
        shutil.rmtree(work, ignore_errors=True)


def test_c1_heat_128_engine_equals_handwritten_every_step_and_reference(cuda):
    import torch
    from fieldcuda import kernels
    from fieldcuda.solver import Solver
    from oracle.heat import gaussian_blobs

    meta, z = load("c1_heat_128")
    n, h, dt, steps = meta["n"], meta["h"], meta["dt"], meta["steps"]
    assert (n, steps) == (128, 100) and dt == 0.4 * h * h / 6.0
    T0 = gaussian_blobs(n, h, seed=0)
    law = open(os.path.join(ROOT, "tests", "laws", "heat.law")).read()
    digests = []
    for run in range(2):
        s = Solver(law, n, n, n, h, "heat.law")
        s.set_field("T", T0)
        if run == 0:
            a = torch.from_numpy(T0).cuda()
            b = torch.empty_like(a)
            eng = torch.empty_like(a)
            ws = kernels.heat7_workspace(T0.shape, 0, 16)
        for k in range(steps):
            s.step(dt)
            assert s.last_substeps() == [1]
            assert not s.violations(), (k, s.violations())
            if run == 0:
                kernels.heat7_step(a, b, 1.0, h, dt, variant=0, zchunk=16, check=0, workspace=ws)
                a, b = b, a
                s.fetch_device("T", eng)
                torch.cuda.synchronize()
                assert torch.equal(eng.view(torch.int32), a.view(torch.int32)), f"engine and hand-written kernel differ after step {k + 1}"
        digests.append(s.digest())
        got = s.values("T")
        s.close()
    assert digests[0] == digests[1], "two runs of 100 steps differ"

    # Against the reference's CPU solver: the sampled cells and two full planes of the committed fixture.
    p, planes = z["pick"], z["planes"]
    ix = np.ix_(p, p, p)
    scale = meta["max_abs"]["T"]
    rel = max(float(np.abs(got[ix].astype(np.float64) - z["ref_T"]).max()),
              float(np.abs(got[planes].astype(np.float64) - z["refplanes_T"]).max())) / scale
    assert rel <= 1e-6, f"relative difference {rel:.3g} from the reference's CPU solver (sampled cells)"
    full = reference_full(meta, {"T": T0})
    if full is not None:
        rel_full = float(np.abs(got.astype(np.float64) - full["T"]).max()) / float(np.abs(full["T"]).max())
        assert rel_full <= 1e-6, f"relative difference {rel_full:.3g} from the reference's CPU solver (whole field)"
    # Against the same scheme in FP64: FP32 rounding over 100 steps (the FP32 restatement of this arithmetic is 2.4e-8
    # of max |T| from it).
    err64 = float(np.abs(got[ix].astype(np.float64) - z["fp64_T"]).max()) / meta["max_abs"]["fp64_T"]
    assert err64 <= 1e-6, f"error {err64:.3g} against the FP64 solve"


def test_multifield43_128_matches_reference(cuda):
    from fieldcuda.solver import Solver

    meta, z = load("multifield43_128")
    n, h, dt, steps = meta["n"], meta["h"], meta["dt"], meta["steps"]
    rng = np.random.default_rng(4343)
    init = {f"f{i}": rng.uniform(-1, 1, (n, n, n)).astype(np.float32) for i in range(6)}
    s = Solver(open(os.path.join(ROOT, "tests", "laws", meta["law"])).read(), n, n, n, h, meta["law"])
    for k, v in init.items():
        s.set_field(k, v)
    for _ in range(steps):
        s.step(dt)
    assert s.last_substeps() == meta["substeps"]
    assert not s.violations(), s.violations()
    got = {k: s.values(k) for k in init}
    s.close()
    p = z["pick"]
    ix = np.ix_(p, p, p)
    for k in init:
        rel = float(np.abs(got[k][ix].astype(np.float64) - z[f"ref_{k}"]).max()) / max(meta["max_abs"][k], 1e-6)
        assert rel <= 1e-4, f"{k}: relative difference {rel:.3g} from the reference's CPU solver"
    full = reference_full(meta, init)
    if full is not None:
        for k in init:
            rel = float(np.abs(got[k].astype(np.float64) - full[k]).max()) / max(float(np.abs(full[k]).max()), 1e-6)
            assert rel <= 1e-4, f"{k}: relative difference {rel:.3g} from the reference's CPU solver (whole field)"
