#!/usr/bin/env python3
"""Writes the test laws' net weight files (tests/laws/nets/fx, fl, ld) in the reference's text format (sections net,
sizes, act, in_shift, in_scale, out_scale, weights; src/field/nn/Net.cpp:335-360 writes the same), from seeded normal
draws: trained-looking nets, so the net ops' parity tests exercise every weight.

    python tests/laws/nets/make_nets.py
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def write(name, sizes, act, shift, scale, out_scale, seed):
    rng = np.random.default_rng(seed)
    weights = []
    for ni, no in zip(sizes[:-1], sizes[1:]):
        weights.extend((rng.normal(size=(no, ni)) / np.sqrt(ni)).astype(np.float32).reshape(-1))
        weights.extend((0.1 * rng.normal(size=no)).astype(np.float32))
    with open(os.path.join(HERE, name), "w") as f:
        f.write(f"net {name}\nsizes {' '.join(str(s) for s in sizes)}\nact {act}\n")
        f.write("in_shift " + " ".join(f"{v:.9g}" for v in shift) + "\n")
        f.write("in_scale " + " ".join(f"{v:.9g}" for v in scale) + "\n")
        f.write(f"out_scale {out_scale:.9g}\nweights\n")
        for i, w in enumerate(weights):
            f.write(f"{float(w):.9g}" + ("\n" if (i + 1) % 8 == 0 else " "))
        f.write("\n")


if __name__ == "__main__":
    write("fx", [2, 16, 16, 1], "tanh", [600.0, 0.3], [1 / 400.0, 2.0], 50.0, 1)
    write("fl", [4, 16, 1], "relu", [600.0, 0.3, 600.0, 0.3], [1 / 400.0, 2.0, 1 / 400.0, 2.0], 20.0, 2)
    write("ld", [5, 8, 8, 4], "silu", [0.0] * 5, [1.0] * 5, 0.2, 3)
