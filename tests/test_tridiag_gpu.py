"""The laws' tridiagonal solves along x by the partition method (a warp a line: per-lane Thomas sweeps, parallel
cyclic reduction of the lanes' first and last unknowns over shuffles; fe_tridiag_x_warp), on lines of 33 to 512 cells
(2 to 16 rows a lane, ragged ends padded with identity rows), against the oracle (the reference's CPU solver restated)
within the reference's per-op gate (2e-5, src/tests/cuda_parity_smoke.cpp:114-117) or whole-law gate (1e-4), two runs
equal to the bit; the transposed solves of an adjoint law the same way; and each solve's kernel timed by itself."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CASES = [
    # (law, tolerance)
    ("crank_nicolson.law", 2e-5),
    ("heston_douglas.law", 1e-4),
    ("heston_hv.law", 1e-4),
]
WIDTHS = [33, 40, 64, 100, 136, 256, 512]


def start(law, shape, seed):
    """(meta with h and dt, starting fields) for a law on a lattice (nz, ny, nx): Crank-Nicolson from a cosine with
    seeded noise, the Heston laws from seeded options laid out as the batch benchmark lays them (one a z-plane)."""
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    if law.startswith("heston"):
        from fieldcuda.heston import lattice_fields, sample_options
        fields, h = lattice_fields(sample_options(nz, seed, sizes=((nx, ny),)), nx, ny)
        return {"h": h, "dt": 0.01}, fields
    x = (np.arange(nx) + 0.5) / nx
    T = (1 + np.cos(4 * np.pi * x))[None, None, :] + 0.01 * rng.normal(size=shape)
    return {"h": 1.0 / nx, "dt": 0.01}, {"T": T.astype(np.float32)}


def run_both(law, meta, init, shape, steps=2):
    from fieldcuda import solver as sv
    from fieldcuda.solver import Solver
    from oracle import law_cpu
    text = open(os.path.join(ROOT, "tests", "laws", law)).read()
    ir = json.loads(sv.ir_json(text))
    nz, ny, nx = shape
    s = Solver(text, nx, ny, nz, meta["h"], law)
    o = law_cpu.Solver(law_cpu.Law(ir), shape, meta["h"])
    for k, v in init.items():
        s.set_field(k, v)
        o.fields[k] = v.copy()
    for _ in range(steps):
        s.step(meta["dt"])
        o.step(meta["dt"])
    return s, o


@pytest.mark.parametrize("nx", WIDTHS)
@pytest.mark.parametrize("law,tol", CASES, ids=[c[0] for c in CASES])
def test_x_solves_match_the_oracle(cuda, law, tol, nx):
    shape = (2, 16, nx)
    meta, init = start(law, shape, nx)
    s, o = run_both(law, meta, init, shape)
    for name in s.field_names:
        if name not in o.fields:
            continue
        got = s.values(name).astype(np.float64)
        want = o.fields[name].astype(np.float64)
        scale = max(float(np.abs(want).max()), 1e-6)
        assert float(np.abs(got - want).max()) <= tol * scale, (law, nx, name, float(np.abs(got - want).max()) / scale)
    d = s.digest()
    s.close()
    s2, _ = run_both(law, meta, init, shape, steps=2)
    assert s2.digest() == d, "two runs differ"
    s2.close()


YZ_SHAPES = [(3, 16, 40), (3, 64, 36), (2, 100, 33), (2, 128, 64), (2, 256, 40), (40, 20, 36), (130, 6, 32)]


@pytest.mark.parametrize("shape", YZ_SHAPES, ids=str)
@pytest.mark.parametrize("law,tol", [("implicit_yz.law", 2e-5), ("heston_douglas.law", 1e-4)], ids=["implicit_yz", "heston_douglas"])
def test_yz_solves_match_the_oracle(cuda, law, tol, shape):
    """y and z lines by the segmented partition solve (32 lines a block, each cut into segments of 8 or 16 rows; lines
    of 16 to 256 rows, ragged ends padded with identity rows), or a thread a line where a line is too short to cut."""
    nz, ny, nx = shape
    if law.startswith("heston"):
        meta, init = start(law, shape, sum(shape))
    else:
        rng = np.random.default_rng(sum(shape))
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        T = 1 + 0.5 * np.cos(0.3 * x + 0.2 * y) * np.sin(0.25 * z + 0.1) + 0.01 * rng.normal(size=shape)
        meta, init = {"h": 1.0 / max(ny, nz), "dt": 0.001}, {"T": T.astype(np.float32)}
    s, o = run_both(law, meta, init, shape)
    for name in s.field_names:
        if name not in o.fields:
            continue
        got = s.values(name).astype(np.float64)
        want = o.fields[name].astype(np.float64)
        scale = max(float(np.abs(want).max()), 1e-6)
        assert float(np.abs(got - want).max()) <= tol * scale, (law, shape, name, float(np.abs(got - want).max()) / scale)
    d = s.digest()
    s.close()
    s2, _ = run_both(law, meta, init, shape)
    assert s2.digest() == d, "two runs differ"
    s2.close()


def test_transposed_yz_solves_match_the_oracle(cuda):
    law = ("field A init 0 range -1e9 1e9\nfield B init 0 range -1e9 1e9\nterm t\n"
           "  d A = tridiag_y_t(-0.2 * (1 + B), 1.6 + 0.1 * A, -0.3 + 0.05 * B, A) + tridiag_z_t(-0.1, 1.3 + 0.1 * B, -0.25 * A, B) - A\n")
    from fieldcuda import solver as sv
    from fieldcuda.solver import Solver
    from oracle import law_cpu
    ir = json.loads(sv.ir_json(law))
    rng = np.random.default_rng(4)
    for shape in ((40, 100, 33), (3, 256, 32)):
        nz, ny, nx = shape
        init = {"A": rng.uniform(0, 1, shape).astype(np.float32), "B": rng.uniform(0, 1, shape).astype(np.float32)}
        s = Solver(law, nx, ny, nz, 0.5)
        o = law_cpu.Solver(law_cpu.Law(ir), shape, 0.5)
        for k, v in init.items():
            s.set_field(k, v)
            o.fields[k] = v.copy()
        s.step(0.01)
        o.step(0.01)
        got, want = s.values("A").astype(np.float64), o.fields["A"].astype(np.float64)
        assert float(np.abs(got - want).max()) <= 2e-5 * float(np.abs(want).max()), shape
        s.close()


def test_transposed_x_solve_matches_the_oracle(cuda):
    """tridiag_x_t (the adjoint laws' solve): below the diagonal the previous cell's `up`, above it the next cell's
    `lo`, through the same warp-a-line kernel."""
    law = ("field A init 0 range -1e9 1e9\nfield B init 0 range -1e9 1e9\nterm t\n"
           "  d A = tridiag_x_t(-0.2 * (1 + B), 1.6 + 0.1 * A, -0.3 + 0.05 * B, A) - A\n")
    from fieldcuda import solver as sv
    from fieldcuda.solver import Solver
    from oracle import law_cpu
    ir = json.loads(sv.ir_json(law))
    rng = np.random.default_rng(3)
    for nx in (40, 200):
        shape = (2, 2, nx)
        init = {"A": rng.uniform(0, 1, shape).astype(np.float32), "B": rng.uniform(0, 1, shape).astype(np.float32)}
        s = Solver(law, nx, 2, 2, 0.5)
        o = law_cpu.Solver(law_cpu.Law(ir), shape, 0.5)
        for k, v in init.items():
            s.set_field(k, v)
            o.fields[k] = v.copy()
        s.step(0.01)
        o.step(0.01)
        got, want = s.values("A").astype(np.float64), o.fields["A"].astype(np.float64)
        assert float(np.abs(got - want).max()) <= 2e-5 * float(np.abs(want).max()), nx
        s.close()


def test_solve_kernels_are_timed_alone(cuda):
    """fe_law_time_stage: the Douglas law's x and y solves (its stages after the stored explicit rate) each timed by
    itself on the calibration's lattice, 256 x 128 x 512 (65,536 x lines: 16,384 blocks of the warp-a-line kernel)."""
    from fieldcuda.solver import Solver
    meta, init = start("heston_douglas.law", (512, 128, 256), 5)
    text = open(os.path.join(ROOT, "tests", "laws", "heston_douglas.law")).read()
    s = Solver(text, 256, 128, 512, 6.0 / 256, "heston_douglas.law")
    for k, v in init.items():
        s.set_field(k, v)
    s.step(0.001)
    names = []
    for stage in range(8):
        try:
            name, ms = s.time_stage(0, stage, 5, 0.001)
        except Exception:
            break
        names.append(name)
        assert ms > 0.0
    s.close()
    assert any(n.startswith("fe_tri_") for n in names), names
