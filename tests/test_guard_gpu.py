"""Learned schemes under guard (the reference's gate src/tests/guarded_smoke.cpp, on this backend): an unstable learned
step is undone and taken classically, so no broken contract reaches the world and the world stays the classical one;
a stable learned step is kept; off, nothing learned runs."""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SHAPE = (6, 20, 24)


def start():
    T = np.full(SHAPE, 290.0, np.float32)
    z, y, x = np.meshgrid(*(np.arange(n) for n in SHAPE), indexing="ij")
    T[(x - 8) ** 2 + (y - 10) ** 2 + (z - 3) ** 2 <= 9] = 1400.0
    T[(x - 17) ** 2 + (y - 6) ** 2 <= 4] = 900.0
    return T


def solver(learned, half=False):
    from fieldcuda.solver import Solver
    text = open(os.path.join(ROOT, "tests", "laws", "guarded_heat.law")).read()
    if half:
        text = text.replace(" file none", " half file none")
    s = Solver(text, SHAPE[2], SHAPE[1], SHAPE[0], 1.0)
    s.set_field("T", start())
    s.set_learned(learned)
    return s


def test_an_unstable_learned_step_is_undone_and_taken_classically(cuda):
    learned, classical = solver(True), solver(False)
    fallbacks = held = 0
    for _ in range(40):
        learned.step(0.3)
        classical.step(0.3)
        fallbacks += learned.profile()["fallbacks"]
        held += learned.term_learned()[0] == "learned"
        assert learned.violations() == [], learned.violations()
        assert classical.term_learned() == ["classical"]
    T = learned.values("T")
    worst = float(np.abs(T.astype(np.float64) - classical.values("T")).max())
    assert fallbacks > 0, "the guard never caught the unstable step"
    assert T.min() >= 0.0 and T.max() <= 6000.0
    assert worst < 400.0, worst
    assert fallbacks + held == 40
    learned.close()
    classical.close()


def test_a_stable_learned_step_is_kept(cuda):
    learned, classical = solver(True), solver(False)
    for _ in range(10):
        learned.step(0.1)
        classical.step(0.1)
        assert learned.profile()["fallbacks"] == 0 and learned.term_learned() == ["learned"]
        assert learned.last_substeps() == [1]
    # untrained, the learned fluxes are the classical ones (to rounding)
    assert float(np.abs(learned.values("T").astype(np.float64) - classical.values("T")).max()) < 1e-2
    learned.close()
    classical.close()


def test_a_learned_step_on_the_tensor_cores_is_guarded_too(cuda):
    """The same gate with the net declared half: the learned step runs on tcgen05 (BF16), the guard judges it the same
    way, and a kept step stays within BF16 of the classical one."""
    from fieldcuda.solver import cuda_source
    text = open(os.path.join(ROOT, "tests", "laws", "guarded_heat.law")).read().replace(" file none", " half file none")
    assert "fe_net_pass<" in cuda_source(text, SHAPE[2], SHAPE[1], SHAPE[0], 1.0)
    learned, classical = solver(True, half=True), solver(False)
    fallbacks = 0
    for _ in range(40):
        learned.step(0.3)
        classical.step(0.3)
        fallbacks += learned.profile()["fallbacks"]
        assert learned.violations() == [], learned.violations()
    T = learned.values("T")
    assert fallbacks > 0 and T.min() >= 0.0 and T.max() <= 6000.0
    learned.close()
    classical.close()
    kept, classical = solver(True, half=True), solver(False)
    for _ in range(10):
        kept.step(0.1)
        classical.step(0.1)
        assert kept.profile()["fallbacks"] == 0 and kept.term_learned() == ["learned"]
    moved = float(np.abs(classical.values("T").astype(np.float64) - start()).max())
    worst = float(np.abs(kept.values("T").astype(np.float64) - classical.values("T")).max())
    assert worst <= 0.03 * moved + 1e-3, (worst, moved)
    kept.close()
    classical.close()
