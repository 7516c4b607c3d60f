#!/usr/bin/env python3
"""Makes tests/golden/heston/calib_<n>.npz: the adjoint calibration's targets, FP64 characteristic-function prices
(oracle/heston_cf.py) of the seeded calibration set (fieldcuda.heston.calibration_options(n, seed)) under its seeded
ground-truth parameters, plus N(0, 1e-4) noise from default_rng(seed + 1).

    python tests/golden/make_heston_calib.py [--n 512] [--seed 5] [--jobs 8]
"""
import argparse
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "online-physics-cuda_b200")]


def price(args):
    from oracle import heston_cf
    k, common, t = args
    return heston_cf.put(common["spot"], k, common["maturity"], t["v0"], t["kappa"], t["theta"], t["sigma"], t["rho"], common["r"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    from fieldcuda.heston import calibration_options
    strikes, common, truth = calibration_options(args.n, args.seed)
    with mp.get_context("spawn").Pool(args.jobs) as pool:
        prices = np.array(pool.map(price, [(k, common, truth) for k in strikes], chunksize=8))
    noise = np.random.default_rng(args.seed + 1).normal(0.0, 1e-4, args.n)
    os.makedirs(os.path.join(HERE, "heston"), exist_ok=True)
    out = os.path.join(HERE, "heston", f"calib_{args.n}.npz")
    np.savez_compressed(out, strikes=strikes, cf=prices, targets=prices + noise, seed=args.seed,
                        **{k: v for k, v in truth.items()}, **common)
    print("wrote", out, "truth", truth)


if __name__ == "__main__":
    main()
