#!/usr/bin/env python3
"""Makes tests/golden/heston/cf_2048.npz: FP64 characteristic-function prices (oracle/heston_cf.py) of the 2048 seeded
options the batched Heston benchmark prices (fieldcuda.heston.sample_options(2048, seed=1)), with the options' numbers,
so the benchmark can report the batch's price error without running the oracle.

    python tests/golden/make_heston_cf.py [--n 2048] [--seed 1] [--jobs 8]
"""
import argparse
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "online-physics-cuda_b200")]

FIELDS = ("nx", "ny", "strike", "maturity", "spot", "v0", "kappa", "theta", "sigma", "rho", "r")


def price(o):
    from oracle import heston_cf
    return heston_cf.put(o["spot"], o["strike"], o["maturity"], o["v0"], o["kappa"], o["theta"], o["sigma"], o["rho"], o["r"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    from fieldcuda.heston import sample_options
    opts = sample_options(args.n, args.seed)
    with mp.get_context("spawn").Pool(args.jobs) as pool:
        prices = pool.map(price, opts, chunksize=8)
    os.makedirs(os.path.join(HERE, "heston"), exist_ok=True)
    out = os.path.join(HERE, "heston", f"cf_{args.n}.npz")
    np.savez_compressed(out, price=np.array(prices, np.float64), seed=args.seed,
                        **{f: np.array([o[f] for o in opts]) for f in FIELDS})
    print("wrote", out, "median price", float(np.median(prices)))


if __name__ == "__main__":
    main()
