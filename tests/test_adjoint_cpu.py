"""The IR-generated adjoint laws (fe_law_adjoint) on the CPU: they compile, refuse what has no adjoint, and — run by the
oracle in double — are the transposes of the primal steps: <A, dU'/dU delta> = <U_bar - A, delta> / dt and the static
fields' and params' cotangents against central differences of the primal."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT


def text(name):
    return open(os.path.join(ROOT, "tests", "laws", name)).read()


def adjoint(law, term=""):
    from fieldcuda import _lib
    return _lib.text_call("fe_law_adjoint", law.encode(), term.encode())


def ir_of(law):
    from fieldcuda import _lib
    return json.loads(_lib.text_call("fe_law_ir_json", law.encode()))


def run(law_cpu, law, shape, h, fields, dt):
    s = law_cpu.Solver(law_cpu.Law(ir_of(law)), shape, h)
    for k, v in fields.items():
        s.fields[k] = np.asarray(v, np.float64).copy()
    s.step(dt)
    assert max(s.substeps) == 1
    return s


@pytest.fixture
def f64_oracle(monkeypatch):
    from oracle import law_cpu
    monkeypatch.setattr(law_cpu, "F32", np.float64)
    return law_cpu


@pytest.mark.parametrize("name", ["heston_douglas.law", "heston_hv.law", "heston_explicit.law", "heat.law", "fhn_rk4.law"])
def test_adjoint_laws_compile(name):
    adj = adjoint(text(name))
    ir = ir_of(adj)
    assert ir["terms"], adj


@pytest.mark.parametrize("name", ["heston_douglas.law", "heston_hv.law", "heston_explicit.law"])
def test_adjoint_laws_generate_and_compile_to_sm100a(name):
    """The backend plans the adjoint law's passes and NVRTC compiles them (no GPU needed)."""
    from fieldcuda.solver import compile_check, cuda_source
    adj = adjoint(text(name))
    src = cuda_source(adj, 32, 16, 3, 6.0 / 32)
    assert "tridiag" in src or "explicit" in name
    compile_check(adj, 32, 16, 3, 6.0 / 32)


def test_adjoint_refuses_what_has_no_adjoint():
    from fieldcuda import _lib
    for eq in ("d a = adv(a, 1, 0, 0)", "d a = maxof(a) * a", "d a = diffuse(a, a)"):
        law = f"field a init 0 range -10 10\nterm t\n  {eq}\n"
        with pytest.raises(_lib.FeError) as e:
            adjoint(law)
        assert e.value.code == _lib.FE_EUNSUP
        assert "adjoint" in str(e.value)


CASES = {
    "shift": "d V = shift(V, 1, 0, 0)", "shift_far": "d V = shift(V, 0, 2, -1) * k", "gx": "d V = gx(V)", "gy": "d V = gy(k * V)",
    "gz": "d V = gz(V)", "mixed": "d V = gx(gy(V)) * k", "lap": "d V = lap(V)", "diffuse": "d V = diffuse(0.7, V)",
    "product": "d V = k * V * V - V / (k + 2)", "tridiag_x": "d V = tridiag_x(0 - k, 3 + k, 0 - 0.5 * k, V) / dt",
    "tridiag_y": "d V = tridiag_y(0 - k, 3 + k * k, 0 - 0.5 * k, V * k) / dt",
    "tridiag_z": "d V = tridiag_z(0 - 0.3 * k, 3, 0 - k, V) / dt",
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_adjoint_is_the_transpose(f64_oracle, case):
    law = f"field V init 0 range -1e30 1e30\nfield k init 1 range -1e30 1e30 static\nterm t\n  {CASES[case]}\n"
    adj = adjoint(law)
    shape, h, dt = (3, 5, 7), 0.5, 0.01
    rng = np.random.default_rng(1)
    V, k = rng.normal(size=shape), rng.uniform(0.5, 1.5, size=shape)
    A, dlt = rng.normal(size=shape), rng.normal(size=shape)
    sa = run(f64_oracle, adj, shape, h, {"V": V, "k": k, "V__adj": A}, dt)
    eps = 1e-4
    for name, base in (("V", V), ("k", k)):
        if name + "__adj" not in sa.fields:
            continue
        got = float(np.sum(sa.fields[name + "__adj"] * dlt))
        fp = {"V": V, "k": k, name: base + eps * dlt}
        fm = {"V": V, "k": k, name: base - eps * dlt}
        up = run(f64_oracle, law, shape, h, fp, dt).fields["V"]
        um = run(f64_oracle, law, shape, h, fm, dt).fields["V"]
        want = float(np.sum(A * (up - um) / (2 * eps)))
        assert abs(got - want) <= 1e-7 * max(1.0, abs(want)), (case, name, got, want)


@pytest.mark.parametrize("law_name", ["heston_douglas.law", "heston_hv.law"])
def test_heston_step_cotangents_match_central_differences(f64_oracle, law_name):
    from fieldcuda.heston import lattice_fields, sample_options
    law = text(law_name)
    adj = adjoint(law)
    nx, ny, nz = 16, 8, 2
    opts = sample_options(nz, 3, sizes=((nx, ny),))
    fields, h = lattice_fields(opts, nx, ny)
    fields = {k: v.astype(np.float64) for k, v in fields.items()}
    rng = np.random.default_rng(0)
    fields["V"] = fields["V"] + rng.uniform(0, 1, fields["V"].shape)
    dt = 0.002
    A = rng.normal(size=fields["V"].shape)
    sa = run(f64_oracle, adj, (nz, ny, nx), h, dict(fields, V__adj=A), dt)
    for name in ("V", "kappa", "theta", "sig_v", "rho", "var"):
        got = float(np.sum(sa.fields[name + "__adj"]))
        if name == "V":
            got = float(np.sum(sa.fields["V__adj"] - A))
        e = 1e-4 * max(1e-3, float(np.abs(fields[name]).mean()))
        up = run(f64_oracle, law, (nz, ny, nx), h, dict(fields, **{name: fields[name] + e}), dt).fields["V"]
        um = run(f64_oracle, law, (nz, ny, nx), h, dict(fields, **{name: fields[name] - e}), dt).fields["V"]
        want = float(np.sum(A * (up - um) / (2 * e)))
        if name == "V":
            want = want - float(np.sum(A))
        # step() of the first-row switch is flat away from its edge: the perturbation stays on one side.
        assert abs(got - want) <= 1e-5 * max(abs(want), 1e-3), (law_name, name, got, want)
