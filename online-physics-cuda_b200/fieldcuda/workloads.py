"""Seeded synthetic workloads of the benchmark configurations: law texts and starting states.

* :func:`heat_law` — the plain conduction law (one field, `diffuse`, `conserves`, `max_dt = 0.4 h^2 / 6 D`).
* :func:`multifield_law` — a 43-term law over 6 fields: radius-1 stencils (diffuse, lap, gx/gy/gz, shift) and reaction
  products, its params drawn U[0, 1] from a seed. The reference's shipped world law has 43 terms
  (bench/results/perf.md:15); this one is generated so it can be made at any size and seed
  (tests/laws/multifield43.law is seed 0).
* :func:`blobs` — the sum of Gaussian blobs the heat workload starts from.

The algorithmic bytes of a multi-field step (Lie splitting forbids fusing terms): for every term, 4 bytes a cell for
every field it reads or writes, plus 4 for every field it writes.
"""
import numpy as np

HEAT_LAW = """field T init 0 range -1000000 1000000
param D = 1
term conduction
  d T = diffuse(D, T)
  conserves T
  max_dt = 0.4 * h * h / (6 * D)
"""


def heat_law():
    return HEAT_LAW


def blobs(shape, h, seed, count=4, width=0.05):
    """A sum of `count` Gaussians A exp(-|x - c|^2 / (2 width^2)) at cell centres (i + 0.5) h; centres U[0.2, 0.8]^3,
    amplitudes U[0.5, 1], from numpy default_rng(seed). Shape is (nz, ny, nx)."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    c = rng.uniform(0.2, 0.8, size=(count, 3))
    a = rng.uniform(0.5, 1.0, size=count)
    xs = [(np.arange(n) + 0.5) * h for n in (nx, ny, nz)]
    out = np.zeros(shape)
    for b in range(count):
        g = [np.exp(-((xs[i] - c[b, i]) ** 2) / (2 * width * width)) for i in range(3)]
        out += a[b] * g[2][:, None, None] * g[1][None, :, None] * g[0][None, None, :]
    return out.astype(np.float32)


def multifield_law(seed=0, fields=6, terms=43):
    """(law text, per-term (reads, writes) field-name sets). Five term shapes in turn, fields and params chosen by the
    seed. Rates are scaled so a step of dt <= 0.1 h^2 keeps every field bounded for thousands of steps."""
    rng = np.random.default_rng(seed)
    names = [f"f{i}" for i in range(fields)]
    lines = [f"field {n} init 0 range -1000000 1000000" for n in names]
    body = []
    rw = []
    for t in range(terms):
        for p in "abc":
            lines.append(f"param p{t}{p} = {rng.uniform(0.0, 1.0):.6f}")
        x, y, z = (names[i] for i in rng.choice(fields, 3, replace=False))
        kind = t % 5
        body.append(f"term t{t}")
        if kind == 0:
            body.append(f"  d {x} = diffuse(p{t}a, {x})")
            body.append(f"  conserves {x}")
            body.append(f"  max_dt = 0.4 * h * h / (6 * p{t}a + 0.000001)")
            rw.append(({x}, {x}))
        elif kind == 1:
            body.append(f"  d {x} = 0.01 * h * (p{t}a * gx({y}) - p{t}b * gy({z})) / (h * h) * h - 0.1 * p{t}c * {x}")
            rw.append(({x, y, z}, {x}))
        elif kind == 2:
            body.append(f"  d {x} = 0.1 * (p{t}a * {y} - p{t}b * {x} * {z}) - 0.1 * p{t}c * {x}")
            rw.append(({x, y, z}, {x}))
        elif kind == 3:
            body.append(f"  d {x} = 0.1 * p{t}a * h * h * lap({y}) + 0.01 * h * p{t}b * gz({z}) - 0.1 * p{t}c * {x}")
            rw.append(({x, y, z}, {x}))
        else:
            body.append(f"  d {x} = 0.05 * p{t}a * (shift({y}, 1, 0, 0) - shift({y}, -1, 0, 0) + shift({z}, 0, 1, 0) - {z}) - 0.1 * p{t}b * {x}")
            rw.append(({x, y, z}, {x}))
    return "\n".join(lines + body) + "\n", rw


def multifield_bytes_per_cell(rw):
    """Algorithmic bytes a cell a step: per term, its read-or-written fields plus its written fields, 4 bytes each."""
    return sum(4 * (len(r | w) + len(w)) for r, w in rw)
