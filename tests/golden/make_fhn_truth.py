#!/usr/bin/env python3
"""Makes tests/golden/fhn/truth.npz: FP64 method-of-lines solutions (oracle/fhn_fp64.py) of the FitzHugh-Nagumo
benchmark on 128 x 128 for a few test seeds (fieldcuda.learned.fhn_initial: u0 then v0 N(0, 1) from default_rng(seed)),
t in [0, 5], averaged 4 x 4 onto 32 x 32 and kept every 10th frame, float32.

    python tests/golden/make_fhn_truth.py [--seeds 1000 1001 1002 1003]
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "online-physics-cuda_b200")]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, nargs="+", default=[1000, 1001, 1002, 1003])
    args = ap.parse_args()
    from fieldcuda.learned import block_mean, fhn_initial
    from oracle import fhn_fp64
    u0, v0 = fhn_initial(args.seeds, 128)
    states = fhn_fp64.solve(u0, v0, 100)
    keep = states[::10]
    coarse = np.stack([[np.stack([block_mean(s[0], 4), block_mean(s[1], 4)]) for s in keep]])[0].astype(np.float32)
    os.makedirs(os.path.join(HERE, "fhn"), exist_ok=True)
    out = os.path.join(HERE, "fhn", "truth.npz")
    np.savez_compressed(out, seeds=np.array(args.seeds), every=10, frame=0.05, states=coarse)
    print("wrote", out, coarse.shape)


if __name__ == "__main__":
    main()
