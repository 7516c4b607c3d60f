"""Reverse mode on the GPU: the IR-generated adjoint laws run as generated kernels against the oracle running the same
adjoint law, the sqrt(N)-checkpointed driver against the oracle's keep-every-state reverse pass (and against itself
with other checkpoint spacings, bit for bit), and the Heston calibration gradient against central differences of an
FP64 restatement of the loss."""
import json
import math
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

# The oracle computes every op in double and stores float; the engine computes in fp32 (the same parity bar as the
# primal laws).
TOL = 1e-4


def text(name):
    return open(os.path.join(ROOT, "tests", "laws", name)).read()


def oracle_solver(law_cpu, law, shape, h, fields):
    from fieldcuda import _lib
    ir = json.loads(_lib.text_call("fe_law_ir_json", law.encode()))
    s = law_cpu.Solver(law_cpu.Law(ir), shape, h)
    for k, v in fields.items():
        s.fields[k] = np.asarray(v, law_cpu.F32).copy()
    return s


def heston_case(nx=32, ny=16, nz=3, seed=3):
    from fieldcuda.heston import lattice_fields, sample_options
    opts = sample_options(nz, seed, sizes=((nx, ny),))
    fields, h = lattice_fields(opts, nx, ny)
    return fields, h, (nz, ny, nx)


@pytest.mark.parametrize("law_name", ["heston_douglas.law", "heston_hv.law", "heston_explicit.law"])
def test_adjoint_step_matches_the_oracle(cuda, law_name):
    from fieldcuda.adjoint import adjoint_law
    from fieldcuda.solver import Solver
    from oracle import law_cpu
    adj = adjoint_law(text(law_name))
    fields, h, shape = heston_case()
    rng = np.random.default_rng(4)
    fields = dict(fields, V__adj=rng.normal(size=shape).astype(np.float32))
    dt = 1e-4 if "explicit" in law_name else 0.01
    s = Solver(adj, shape[2], shape[1], shape[0], h, "adj")
    for k, v in fields.items():
        s.set_field(k, v)
    o = oracle_solver(law_cpu, adj, shape, h, fields)
    for _ in range(3):
        s.step(dt)
        o.step(dt)
    for name in s.field_names:
        if not name.endswith("__adj"):
            continue
        got = s.values(name).astype(np.float64)
        want = o.fields[name].astype(np.float64)
        scale = max(float(np.abs(want).max()), 1e-12)
        assert float(np.abs(got - want).max()) / scale <= TOL, (law_name, name)
    s.close()


def test_checkpointed_vjp_matches_the_oracle_and_its_own_spacings(cuda):
    import torch
    from fieldcuda.adjoint import LawVJP
    from oracle import law_cpu
    law = text("heston_douglas.law")
    fields, h, shape = heston_case()
    steps, dt = 20, 0.01
    rng = np.random.default_rng(8)
    seed = rng.normal(size=shape).astype(np.float32)
    tens = {k: torch.tensor(v, device="cuda") for k, v in fields.items()}
    results = []
    for every in (1, 5, 20):
        vjp = LawVJP(law, shape[2], shape[1], shape[0], h)
        vjp.forward(tens, dt, steps, every=every)
        cot = vjp.backward({"V": torch.tensor(seed, device="cuda")})
        results.append({k: v.cpu().numpy() for k, v in cot.items()})
        vjp.close()
    for k in results[0]:
        for r in results[1:]:
            assert np.array_equal(results[0][k].view(np.uint32), r[k].view(np.uint32)), k
    # The oracle keeps every state and runs the same adjoint law back over them.
    from fieldcuda.adjoint import adjoint_law
    o = oracle_solver(law_cpu, law, shape, h, fields)
    states = []
    for _ in range(steps):
        states.append(o.fields["V"].copy())
        o.step(dt)
    adj = adjoint_law(law)
    a = oracle_solver(law_cpu, adj, shape, h, dict(fields, V__adj=seed))
    for s in range(steps - 1, -1, -1):
        a.fields["V"] = states[s]
        a.step(dt)
    for name in ("V", "kappa", "theta", "sig_v", "rho", "var"):
        got = results[0][name].astype(np.float64)
        want = a.fields[name + "__adj"].astype(np.float64)
        rel = float(np.abs(got - want).max()) / max(float(np.abs(want).max()), 1e-12)
        assert rel <= 1e-3, (name, rel)
        tot = abs(got.sum() - want.sum()) / max(abs(want.sum()), 1e-12)
        assert tot <= 1e-4, (name, tot)


def test_calibration_gradient_matches_fp64_central_differences(cuda):
    from fieldcuda.heston import Calibration, calibration_options, lattice_fields
    from oracle import law_cpu
    z = np.load(os.path.join(ROOT, "tests", "golden", "heston", "calib_16.npz"))
    strikes, common, truth = calibration_options(16, int(z["seed"]))
    assert np.allclose(strikes, z["strikes"])
    nx, ny, steps = 64, 32, 32
    law = text("heston_douglas.law")
    cal = Calibration(law, strikes, common["maturity"], common["spot"], common["r"], z["targets"], nx, ny, steps)
    x = np.array([truth["kappa"] * 1.3, truth["theta"] * 0.8, truth["sigma"] * 1.1, truth["rho"] * 0.9, truth["v0"] * 1.2])
    loss, grad = cal.loss_and_grad(x)
    cal.close()

    # The loss restated in FP64 on the oracle (every op and store in double), differenced centrally.
    def loss64(v):
        kappa, theta, sigma, rho, v0 = v
        opts = [dict(nx=nx, ny=ny, strike=k, maturity=common["maturity"], spot=common["spot"], v0=v0, kappa=kappa,
                     theta=theta, sigma=sigma, rho=rho, r=common["r"]) for k in strikes]
        f, h = lattice_fields(opts, nx, ny)
        f["var"] = (sigma * (np.arange(ny) + 0.5) * h)[None, :, None] * np.ones((len(opts), ny, nx))
        old = law_cpu.F32
        law_cpu.F32 = np.float64
        try:
            o = oracle_solver(law_cpu, law, (len(opts), ny, nx), h, f)
            for _ in range(steps):
                o.step(common["maturity"] / steps)
            VT = o.fields["V"]
        finally:
            law_cpu.F32 = old
        from fieldcuda.heston import price_bilinear
        p = np.array([price_bilinear(VT[i].astype(np.float64), o_) for i, o_ in enumerate(opts)], np.float64)
        return float(np.sum((p - z["targets"]) ** 2))

    for i in range(5):
        e = 1e-3 * abs(x[i])
        xp, xm = x.copy(), x.copy()
        xp[i] += e
        xm[i] -= e
        fd = (loss64(xp) - loss64(xm)) / (2 * e)
        assert abs(grad[i] - fd) <= 2e-3 * max(abs(fd), 1e-3 * abs(loss)), (Calibration.NAMES[i], grad[i], fd)
