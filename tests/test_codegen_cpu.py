"""The generated slab passes' plane carry, decided on the CPU from the generated source (fe_law_source): a pass keeps
plane z - 1 in registers, and its ring holds planes z and z + 1 with two in flight (4 stages, where the full ring holds
three planes and one in flight), exactly when every read it makes below the cell's plane is the cell's own column one
plane down (and at most two sources are read there). Anything that reads the plane
below at another column (a diagonal shift, topple's neighbours, a stencil of a stencil) keeps the full ring."""
import re

import pytest


def passes(law, n=256):
    from fieldcuda.solver import cuda_source
    src = cuda_source(law, n, n, n, 1.0 / n)
    carry = re.findall(r"static constexpr bool ZCARRY = (true|false);", src)
    rings = [int(m) for m in re.findall(r"static constexpr int W = 8, R = \d+, RZ = \d+, NST = (\d+)", src)]
    return carry, rings


HEAD = "field T init 0 range -1e9 1e9\nfield k init 1 range 0 10 static\nfield s init 0 range 0 1 static\n"

CASES = [
    # (expression for d T, carried?)
    ("diffuse(1, T)", True),
    ("diffuse(k, T)", True),               # k read at the faces too: both sources carried
    ("lap(T)", True),
    ("gz(T)", True),
    ("adv(T, 0.5, -0.5, 0.25)", True),
    ("shift(T, 0, 0, -1) - T", True),
    ("shift(T, 1, 0, -1) - T", False),     # the plane below, one column over
    ("shift(T, 0, 0, 1) - T", False),      # nothing below: RZ is 1 but no source needs the carry
    ("shift(T, 0, 0, -2) - T", False),     # two planes down
    ("lap(lap(T))", True),                 # the inner lap is a stage of its own: two passes, each one plane each way
    ("gz(gx(T))", False),                  # gx inside gz reads the plane below at x +- 1
    ("fall(T, s, 2)", True),
    ("topple(T, s, 2)", False),            # reads the room below its neighbours
    ("T * k", False),                      # no other plane at all
]


@pytest.mark.parametrize("expr,carried", CASES, ids=[c[0] for c in CASES])
def test_plane_carry_is_planned_from_the_reads(expr, carried):
    carry, rings = passes(HEAD + "term t\n  d T = " + expr + "\n  conserves T\n")
    assert carry and rings, "no slab pass generated"
    assert all(c == ("true" if carried else "false") for c in carry), (expr, carry)
    if carried:
        assert all(r in (3, 4) for r in rings), (expr, rings)
    if expr == "diffuse(1, T)":
        assert rings == [4], rings


def test_carry_keeps_the_small_lattice_plain_pass_untouched():
    """Below 128 cells along x no slab pass runs; the traits still say no carry for the plain twin's sake."""
    from fieldcuda.solver import cuda_source
    src = cuda_source(HEAD + "term t\n  d T = diffuse(1, T)\n", 64, 64, 64, 1.0 / 64)
    assert "ZCARRY = false" in src
