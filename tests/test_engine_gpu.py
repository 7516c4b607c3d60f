"""The law backend on the GPU against the reference's own CPU solver (golden fixtures made by its lawc), the hand-written
kernel, itself (determinism) and the contracts it must catch."""
import glob
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))
# Relative tolerance against the reference's CPU solver (which computes every op in double and stores float): the
# reference's own gate holds one op to 2e-5 and a whole law to 1e-4 (src/tests/cuda_parity_smoke.cpp:114-117, 159-160).
TOLERANCE = {"heat_24": 1e-6, "ops_stencil": 2e-5, "ops_matter": 2e-5, "cn_64": 2e-5, "implicit_yz": 2e-5, "op_distance": 2e-5,
             "op_poisson": 2e-5}


def load(path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    init = {k[5:]: z[k] for k in z.files if k.startswith("init_")}
    final = {k[6:]: z[k] for k in z.files if k.startswith("final_")}
    return meta, init, final


def run_case(meta, init, steps=None):
    from fieldcuda.solver import Solver
    os.chdir(ROOT)  # net weight files (tests/laws/nets/) are read from the repository root
    nz, ny, nx = meta["shape"]
    s = Solver(open(os.path.join(ROOT, "tests", "laws", meta["law"])).read(), nx, ny, nz, meta["h"], meta["law"])
    for name, arr in init.items():
        s.set_field(name, arr)
    for _ in range(steps or meta["steps"]):
        s.step(meta["dt"])
    return s


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_matches_reference_cpu_solver(cuda, path):
    meta, init, final = load(path)
    s = run_case(meta, init)
    tol = TOLERANCE.get(meta["name"], 1e-4)
    for name, want in final.items():
        got = s.values(name)
        scale = max(float(np.abs(want).max()), 1e-6)
        rel = float(np.abs(got.astype(np.float64) - want).max()) / scale
        assert rel <= tol, f"{meta['name']}:{name} relative difference {rel:.3g} > {tol}"
    assert s.last_substeps() == meta["substeps"], (s.last_substeps(), meta["substeps"])
    assert len(s.violations()) == 0 and meta["violations"] == 0, s.violations()
    s.close()


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_two_runs_are_bit_identical(cuda, path):
    meta, init, _ = load(path)
    a = run_case(meta, init)
    b = run_case(meta, init)
    assert a.digest() == b.digest()
    a.close()
    b.close()


def test_engine_heat_bit_identical_to_handwritten_kernel(cuda):
    """The generated step of `d T = diffuse(D, T)` and the hand-written kernel do the same arithmetic in the same order:
    equal to the bit (the reference's own check: bench/stencil_bench.cpp:291-294). 64^3 and 96^3 take the plain pass,
    the rest the TMA slab pass with the plane carry: one plane a chunk up to 160^3, then chunks of several planes whose
    later planes read plane z - 1 from the registers (256^3: 4 planes; 203 x 256 x 384: 5, the last chunk 3; 256 x 512
    x 512: the length the fullest-last-wave rule picks)."""
    import torch
    from fieldcuda import kernels
    from fieldcuda.solver import Solver
    from oracle import heat as oh
    shapes = [(64, 64, 64), (96, 96, 96), (128, 128, 128), (160, 160, 160), (256, 256, 256), (203, 256, 384),
              (256, 512, 512)]
    for shape in shapes:
        nz, ny, nx = shape
        h = 1.0 / nx
        dt = 0.4 * h * h / 6.0
        if nz == ny == nx:
            T0 = oh.gaussian_blobs(nx, h, seed=3)
        else:
            T0 = np.random.default_rng(nz).uniform(0.0, 1.0, shape).astype(np.float32)
        s = Solver(open(os.path.join(ROOT, "tests", "laws", "heat.law")).read(), nx, ny, nz, h)
        s.set_field("T", T0)
        a = torch.from_numpy(T0).cuda()
        b = torch.empty_like(a)
        ws = kernels.heat7_workspace(T0.shape, 0, 16)
        for _ in range(7):
            s.step(dt)
            kernels.heat7_step(a, b, 1.0, h, dt, variant=0, zchunk=16, check=0, workspace=ws)
            a, b = b, a
        torch.cuda.synchronize()
        got = s.values("T")
        assert np.array_equal(got.view(np.uint32), a.cpu().numpy().view(np.uint32)), shape
        s.close()
        del a, b, ws
        torch.cuda.empty_cache()


def test_conservation_violation_is_reported(cuda):
    from fieldcuda.solver import Solver
    law = ("field T init 1 range -1e6 1e6\nparam leak = 0.5\nterm leaky\n  d T = diffuse(1, T) - leak * T\n  conserves T\n")
    s = Solver(law, 16, 12, 8, 0.1)
    s.set_field("T", np.random.default_rng(0).uniform(1, 2, (8, 12, 16)).astype(np.float32))
    s.step(0.001)
    v = s.violations()
    assert any(x.kind == "conservation" and x.term == "leaky" and x.field == "T" for x in v), v
    s.set_param("leak", 0.0)
    s.step(0.001)
    assert not s.violations()
    s.close()


def test_range_and_nan_violations_are_reported(cuda):
    from fieldcuda.solver import Solver
    law = "field a init 0 range 0 1\nterm grow\n  d a = 2 * a + 1\n"
    s = Solver(law, 8, 8, 4, 1.0)
    s.step(0.25)  # 0 -> 0.25: in range
    assert not s.violations()
    s.step(1.0)   # 0.25 -> 1.75: out of range everywhere
    v = s.violations()
    assert len(v) == 1 and v[0].kind == "range" and v[0].count == 8 * 8 * 4 and v[0].first_cell == 0
    bad = np.zeros((4, 8, 8), np.float32)
    bad[1, 2, 3] = np.nan
    s.set_field("a", bad)
    s.step(0.0)
    v = s.violations()
    assert len(v) == 1 and v[0].kind == "not-finite" and v[0].first_cell == 3 + 8 * (2 + 8 * 1)
    s.close()


@pytest.mark.parametrize("nx", [16, 128])
def test_conserved_totals_carry_from_step_to_step(cuda, nx):
    """The totals before a term are those after the checked pass that last wrote the field (carried, exactly), or
    summed afresh on the first step and after an edit; either way they are the field's FP64 sums (plain pass at 16 wide,
    TMA slab pass with ragged rows at 128)."""
    from fieldcuda.solver import Solver
    law = ("field T init 1 range -1e6 1e6\nparam leak = 0.5\nterm leaky\n  d T = diffuse(1, T) - leak * T\n  conserves T\n")
    s = Solver(law, nx, 12, 8, 0.1)
    T0 = np.random.default_rng(0).uniform(1, 2, (8, 12, nx)).astype(np.float32)
    s.set_field("T", T0)

    def leak_record():
        v = [x for x in s.violations() if x.kind == "conservation"]
        assert len(v) == 1, s.violations()
        return v[0]

    s.step(0.001)
    first = leak_record()
    assert abs(first.before - T0.astype(np.float64).sum()) <= 1e-7 * abs(first.before)
    T1 = s.values("T")
    assert abs(first.after - T1.astype(np.float64).sum()) <= 1e-7 * abs(first.after)
    s.step(0.001)
    second = leak_record()
    assert second.before == first.after
    s.set_param("leak", 0.0)
    s.step(0.001)
    assert not s.violations()
    s.set_param("leak", 0.5)
    s.set_field("T", T0)  # an edit: the totals are summed again
    s.step(0.001)
    again = leak_record()
    assert abs(again.before - T0.astype(np.float64).sum()) <= 1e-7 * abs(again.before)
    s.check_contracts_every(2)  # steps 4 and 6 checked, 5 not: step 6 sums its totals again
    s.step(0.001)
    s.step(0.001)
    T5 = s.values("T")
    s.step(0.001)
    late = leak_record()
    assert abs(late.before - T5.astype(np.float64).sum()) <= 1e-7 * abs(late.before)
    s.close()


@pytest.mark.parametrize("nx", [16, 128])
def test_range_cells_are_counted_once_across_planes(cuda, nx):
    """Out-of-range and NaN cells scattered over several planes: each counted once, the first one named (on the slab
    pass the test runs per plane, and a plane that fails it is read back)."""
    from fieldcuda.solver import Solver
    law = "field a init 0 range -1 1\nfield b init 0 range -1e30 1e30 static\nterm t\n  d a = b\n"
    shape = (6, 20, nx)
    s = Solver(law, nx, 20, 6, 1.0)
    b = np.zeros(shape, np.float32)
    bad = [(1, 3, 5), (1, 19, nx - 1), (4, 0, 7), (5, 11, nx - 2)]
    for z, y, x in bad:
        b[z, y, x] = 5.0
    b[3, 7, 2] = np.nan
    s.set_field("b", b)
    s.step(1.0)
    v = sorted(s.violations(), key=lambda x: x.kind)
    kinds = {x.kind: x for x in v}
    assert set(kinds) == {"not-finite"}, v
    nan = kinds["not-finite"]
    assert nan.count == len(bad) + 1
    assert nan.first_cell == 5 + nx * (3 + 20 * 1)
    b[3, 7, 2] = 0.0
    s.set_field("b", b)
    s.set_field("a", np.zeros(shape, np.float32))
    s.step(1.0)
    v = s.violations()
    assert len(v) == 1 and v[0].kind == "range" and v[0].count == len(bad) and v[0].first_cell == 5 + nx * (3 + 20 * 1), v
    s.close()


def test_substep_cap_and_ignoring_max_dt(cuda):
    from fieldcuda.solver import Solver
    law = "field T init 0 range -1e9 1e9\nterm c\n  d T = diffuse(1, T)\n  max_dt = 0.1 * h * h\n"
    s = Solver(law, 8, 8, 8, 0.01)
    s.set_field("T", np.random.default_rng(1).uniform(0, 1, (8, 8, 8)).astype(np.float32))
    s.step(1e-6)
    assert s.last_substeps() == [1]
    s.step(1e-4)  # max_dt = 1e-5: 10 substeps
    assert s.last_substeps() == [10]
    s.step(1.0)   # 100000 substeps wanted: capped
    assert s.last_substeps() == [4096]
    assert any(v.kind == "substep-cap" for v in s.violations())
    s.set_respect_max_dt(False)
    s.step(1e-4)
    assert s.last_substeps() == [1]
    s.close()


def test_idle_term_is_not_dispatched(cuda):
    """A term whose every equation is zero given the fields' bounds does nothing (LawBounds.cpp; CudaSolver.cpp:590)."""
    from fieldcuda.solver import Solver
    law = "field T init 5 range -1e9 1e9\nfield m init 0 range -1e9 1e9\nterm heat\n  d T = diffuse(1, T)\nterm mana\n  d T = 3 * m\n"
    s = Solver(law, 8, 8, 8, 1.0)
    s.step(0.1)
    assert s.idle_terms() == [True, True]  # T uniform: no flux; m all zero
    T = np.full((8, 8, 8), 5, np.float32)
    T[4, 4, 4] = 6
    s.set_field("T", T)
    s.step(0.01)
    assert s.idle_terms() == [False, True]
    s.close()


def test_deferred_judging_keeps_steps_off_the_host(cuda):
    from fieldcuda.solver import Solver
    law = "field T init 1 range -1e6 1e6\nparam leak = 0\nterm t\n  d T = diffuse(1, T) - leak * T\n  conserves T\n"
    s = Solver(law, 16, 8, 8, 0.1)
    s.set_field("T", np.random.default_rng(2).uniform(1, 2, (8, 8, 16)).astype(np.float32))
    s.set_deferred(True)
    for i in range(5):
        if i == 3:
            s.set_param("leak", 1.0)
        s.step(0.001)
    s.sync()
    v = s.violations()
    assert [x.step for x in v if x.kind == "conservation"] == [3, 4], v
    s.close()


def test_wider_staging_changes_no_bit(cuda):
    """On a lattice of 2M cells and more the code generator stores values stencils read at several offsets (here the
    FHN law's third RK4 stage); each z-plane is a sample of its own, so the first planes of such a lattice must match,
    bit for bit, a small lattice of the same samples planned without it."""
    from fieldcuda.solver import Solver
    law = open(os.path.join(ROOT, "tests", "laws", "fhn_rk4.law")).read()
    rng = np.random.default_rng(8)
    big_nz, small_nz, n = 128, 8, 128
    u = rng.normal(size=(big_nz, n, n)).astype(np.float32)
    v = rng.normal(size=(big_nz, n, n)).astype(np.float32)
    out = []
    for nz in (big_nz, small_nz):
        s = Solver(law, n, n, nz, 2.0 / n)
        s.set_field("u", u[:nz])
        s.set_field("v", v[:nz])
        for _ in range(3):
            s.step(0.05)
        out.append((s.values("u")[:small_nz], s.values("v")[:small_nz]))
        s.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_two_source_plane_carry_matches_the_oracle(cuda):
    """`d T = diffuse(k, T)` with k a field: both sources are read one plane down at the cell's own column, so both ride
    the plane carry; on 128 x 256 x 256 the pass's z-chunks hold several planes. Against the oracle (the reference's CPU
    arithmetic restated) within the reference's per-op gate (2e-5, src/tests/cuda_parity_smoke.cpp:114-117)."""
    from fieldcuda import solver as sv
    from fieldcuda.solver import Solver
    from oracle import law_cpu
    law = ("field T init 0 range -1e9 1e9\nfield k init 1 range 0 10 static\nterm t\n  d T = diffuse(k, T)\n"
           "  conserves T\n")
    src = sv.cuda_source(law, 128, 256, 256, 1.0 / 128)
    assert "NCARRY = 2;" in src
    shape = (256, 256, 128)
    rng = np.random.default_rng(21)
    init = {"T": rng.uniform(-1, 1, shape).astype(np.float32), "k": rng.uniform(0.5, 2.0, shape).astype(np.float32)}
    h, dt = 1.0 / 128, 0.05 / 128 ** 2
    s = Solver(law, 128, 256, 256, h)
    o = law_cpu.Solver(law_cpu.Law(json.loads(sv.ir_json(law))), shape, h)
    for name, v in init.items():
        s.set_field(name, v)
        o.fields[name] = v.copy()
    for _ in range(2):
        s.step(dt)
        o.step(dt)
    got, want = s.values("T").astype(np.float64), o.fields["T"].astype(np.float64)
    s.close()
    assert float(np.abs(got - want).max()) <= 2e-5 * float(np.abs(want).max())
