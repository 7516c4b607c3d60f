#!/usr/bin/env python3
"""Makes the golden fixtures: the reference's own CPU solver (its lawc, built from the reference's sources by
`make -C oracle ref`) run on this repository's test laws (tests/laws/) from seeded starting states.

    python tests/golden/make_golden.py [--lawc oracle/_ref/lawc]

For each case it writes tests/golden/<case>.npz with the starting fields, the fields after the steps, and a JSON meta
(law file, lattice, dt, steps, the substeps of the last step and the contract violations the reference reported). The
GPU parity tests and the oracle's pin test read these; nothing here runs at test time.
"""
import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LAWS = os.path.join(ROOT, "tests", "laws")
sys.path.insert(0, ROOT)


def blobs(shape, h, seed, count=4, width=0.05):
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


def heston_fields(nx, ny, nz, seed, h_over=None):
    """Per-plane option: x = ln S over ln K +- 3 (h = 6 / nx), var_j = sig_v (j + 1/2) h, put payoff, seeded model."""
    rng = np.random.default_rng(seed)
    h = 6.0 / nx
    f = {k: np.zeros((nz, ny, nx), np.float32) for k in ("V", "var", "kappa", "theta", "sig_v", "rho", "r")}
    for z in range(nz):
        K = rng.uniform(80, 120)
        kappa, theta, sig, rho, r = (rng.uniform(0.5, 5), rng.uniform(0.01, 0.1), rng.uniform(0.1, 1.0),
                                     rng.uniform(-0.9, -0.1), rng.uniform(0.0, 0.05))
        x = np.log(K) - 3 + (np.arange(nx) + 0.5) * h
        f["V"][z] = np.maximum(K - np.exp(x), 0.0)[None, :]
        f["var"][z] = (sig * (np.arange(ny) + 0.5) * h)[:, None]
        f["kappa"][z], f["theta"][z], f["sig_v"][z], f["rho"][z], f["r"][z] = kappa, theta, sig, rho, r
    return f, h


def cases():
    rng = np.random.default_rng(12345)
    out = []
    # Conduction with 3 substeps a step (dt = 2.5 max_dt).
    n = (16, 20, 24)
    h = 1.0 / 24
    out.append(dict(name="heat_24", law="heat.law", shape=n, h=h, dt=2.5 * 0.4 * h * h / 6, steps=5,
                    fields={"T": blobs(n, h, 1)}))
    n = (9, 14, 20)
    out.append(dict(name="ops_stencil", law="ops_stencil.law", shape=n, h=0.5, dt=0.01, steps=4,
                    fields={"a": rng.uniform(-1, 1, n).astype(np.float32),
                            "k": rng.uniform(0.5, 2.0, n).astype(np.float32)}))
    out.append(dict(name="ops_point", law="ops_point.law", shape=n, h=0.5, dt=0.2, steps=4,
                    fields={"a": rng.uniform(-1, 1, n).astype(np.float32),
                            "b": rng.uniform(-1, 1, n).astype(np.float32)}))
    n = (10, 12, 16)
    f = (rng.uniform(0, 1, n) * (rng.uniform(0, 1, n) < 0.4)).astype(np.float32)
    s = (rng.uniform(0, 1, n) < 0.2).astype(np.float32)
    out.append(dict(name="ops_matter", law="ops_matter.law", shape=n, h=0.5, dt=0.01, steps=4, fields={"f": f, "s": s}))
    n = (4, 32, 32)
    out.append(dict(name="fhn_32", law="fhn_rk4.law", shape=n, h=2.0 / 32, dt=0.05, steps=3,
                    fields={"u": rng.normal(size=n).astype(np.float32), "v": rng.normal(size=n).astype(np.float32)}))
    n = (3, 4, 64)
    x = (np.arange(64) + 0.5) / 64
    T = (1 + np.cos(4 * np.pi * x))[None, None, :] + 0.01 * rng.normal(size=n)
    out.append(dict(name="cn_64", law="crank_nicolson.law", shape=n, h=1.0 / 64, dt=0.01, steps=5,
                    fields={"T": T.astype(np.float32)}))
    n = (20, 24, 8)
    out.append(dict(name="implicit_yz", law="implicit_yz.law", shape=n, h=1.0 / 24, dt=0.001, steps=3,
                    fields={"T": blobs(n, 1.0 / 24, 2, width=0.15)}))
    f, h = heston_fields(32, 16, 3, 7)
    out.append(dict(name="heston_douglas", law="heston_douglas.law", shape=(3, 16, 32), h=h, dt=0.01, steps=4, fields=f))
    out.append(dict(name="heston_hv", law="heston_hv.law", shape=(3, 16, 32), h=h, dt=0.01, steps=4, fields=f))
    n = (6, 9, 11)
    rngt = np.random.default_rng(7)
    out.append(dict(name="ops_transposed", law="ops_transposed.law", shape=n, h=0.5, dt=0.01, steps=3,
                    fields={"a": rngt.uniform(-1, 1, n).astype(np.float32), "b": rngt.uniform(-1, 1, n).astype(np.float32)}))
    # Lattices at least one slab tile (128 cells) wide: the generated TMA slab passes rather than the plain ones.
    n = (5, 9, 136)
    rngw = np.random.default_rng(11)
    out.append(dict(name="ops_stencil_wide", law="ops_stencil.law", shape=n, h=0.5, dt=0.01, steps=3,
                    fields={"a": rngw.uniform(-1, 1, n).astype(np.float32),
                            "k": rngw.uniform(0.5, 2.0, n).astype(np.float32)}))
    n = (4, 6, 128)
    out.append(dict(name="multifield43_wide", law="multifield43.law", shape=n, h=1.0 / 128, dt=0.1 * (1.0 / 128) ** 2, steps=2,
                    fields={f"f{i}": rngw.uniform(-1, 1, n).astype(np.float32) for i in range(6)}))
    n = (12, 16, 20)
    rngm = np.random.default_rng(43)
    out.append(dict(name="multifield43", law="multifield43.law", shape=n, h=1.0 / 20, dt=0.1 * (1.0 / 20) ** 2, steps=3,
                    fields={f"f{i}": rngm.uniform(-1, 1, n).astype(np.float32) for i in range(6)}))
    out.append(dict(name="heston_explicit", law="heston_explicit.law", shape=(3, 16, 32), h=h, dt=0.01, steps=3, fields=f))
    # distance and poisson: the per-op starting state of the reference's CUDA gate (a smooth A, B solid in a pattern),
    # then both ops with a drifting source.
    n = (9, 14, 20)
    z, y, x = np.meshgrid(np.arange(9), np.arange(14), np.arange(20), indexing="ij")
    A = (0.5 + 0.4 * np.sin(0.7 * x + 0.3 * y) * np.cos(0.5 * z)).astype(np.float32)
    B = ((x + 2 * y + 3 * z) % 7 < 3).astype(np.float32)
    for name in ("op_distance", "op_poisson"):
        out.append(dict(name=name, law=name + ".law", shape=n, h=0.5, dt=0.02, steps=4, fields={"A": A, "B": B}))
    # The net ops (weights in tests/laws/nets/, read relative to the repository root like the reference's assets/nets).
    rngn = np.random.default_rng(31)
    for shape, tag in (((9, 14, 20), ""), ((4, 6, 136), "_wide")):
        T = (290.0 + 900.0 * rngn.uniform(0, 1, shape) * (rngn.uniform(0, 1, shape) < 0.3)).astype(np.float32)
        fuel = rngn.uniform(0, 1, shape).astype(np.float32)
        out.append(dict(name="nets_mlp" + tag, law="nets_mlp.law", shape=shape, h=0.5, dt=0.02, steps=3, fields={"T": T, "fuel": fuel}))
        out.append(dict(name="nets_flux" + tag, law="nets_flux.law", shape=shape, h=0.5, dt=0.02, steps=3, fields={"T": T, "fuel": fuel}))
        out.append(dict(name="nets_ldiffuse" + tag, law="nets_ldiffuse.law", shape=shape, h=0.5, dt=0.02, steps=3, fields={"T": T}))
    n = (10, 12, 16)
    rngf = np.random.default_rng(21)
    out.append(dict(name="ops_fields", law="ops_fields.law", shape=n, h=0.5, dt=0.05, steps=4,
                    fields={"b": (rngf.uniform(0, 1, n) < 0.3).astype(np.float32)}))
    return out


def run(case, lawc, work):
    law = os.path.join(LAWS, case["law"])
    nz, ny, nx = case["shape"]
    scene = os.path.join(work, "scene")
    with open(scene, "w") as fh:
        fh.write(f"grid {nx} {ny} {nz} {case['h']!r}\nlaw {law}\n")
    init = os.path.join(work, "init")
    os.makedirs(init, exist_ok=True)
    for name, arr in case["fields"].items():
        np.ascontiguousarray(arr, dtype=np.float32).tofile(os.path.join(init, name + ".bin"))
    dump = os.path.join(work, "dump")
    js = os.path.join(work, "t.json")
    cmd = [lawc, "--scene", scene, "--init", init, "--steps", str(case["steps"]), "--dt", repr(case["dt"]), "--dump", dump,
           "--json", js]
    res = subprocess.run(cmd, capture_output=True, text=True, cwd=ROOT, env=dict(os.environ, OMP_NUM_THREADS="4"))
    if res.returncode != 0:
        raise RuntimeError(f"{case['name']}: lawc failed\n{res.stdout}\n{res.stderr}")
    meta_dump = json.load(open(os.path.join(dump, f"step_{case['steps']}", "meta.json")))
    final = {f: np.fromfile(os.path.join(dump, f"step_{case['steps']}", f + ".bin"), dtype=np.float32).reshape(case["shape"])
             for f in meta_dump["fields"]}
    timing = json.load(open(js))
    meta = dict(name=case["name"], law=case["law"], shape=list(case["shape"]), h=case["h"], dt=case["dt"], steps=case["steps"],
                substeps=timing["substeps"], violations=timing["violations"], fields=meta_dump["fields"],
                made_by="the reference's lawc (its OpenMP CPU Solver), OMP_NUM_THREADS=4")
    arrays = {f"init_{k}": np.asarray(v, np.float32) for k, v in case["fields"].items()}
    arrays.update({f"final_{k}": v for k, v in final.items()})
    np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), meta=json.dumps(meta), **arrays)
    return meta


def ir_fixtures(lawc):
    """The reference's IR JSON (lawc --ir-json) of every test law: the lowering's golden vectors."""
    out_dir = os.path.join(HERE, "ir")
    os.makedirs(out_dir, exist_ok=True)
    for name in sorted(os.listdir(LAWS)):
        if not name.endswith(".law"):
            continue
        out = os.path.join(out_dir, name[:-4] + ".json")
        subprocess.run([lawc, "--ir-json", out, os.path.join(LAWS, name)], check=True, capture_output=True, cwd=ROOT)
        print("ir", name)


def scene_fixtures(lawc):
    """lawc --scene on tests/scenes/*.scene (from the repository root, where the scenes' law paths point): the state the
    scene makes (step_0, after refresh_derived) and the state after the steps, for the CLI's parity tests."""
    out_dir = os.path.join(HERE, "scene")
    os.makedirs(out_dir, exist_ok=True)
    # guarded: heat with an untrained learned scheme at twice the stable step, run with --learned: which learned steps
    # the reference's guard undoes, and the state that leaves.
    for name, steps, dt, extra in (("ops", 3, 0.05, []), ("guarded", 30, 0.3, ["--learned"])):
        work = tempfile.mkdtemp(prefix="fe_scene_")
        try:
            dump = os.path.join(work, "dump")
            js = os.path.join(work, "t.json")
            subprocess.run([lawc, "--scene", os.path.join("tests", "scenes", name + ".scene"), "--steps", str(steps), "--dt", repr(dt),
                            "--dump", dump, "--json", js] + extra, check=True, capture_output=True, cwd=ROOT,
                           env=dict(os.environ, OMP_NUM_THREADS="4"))
            meta_dump = json.load(open(os.path.join(dump, "step_0", "meta.json")))
            shape = (meta_dump["nz"], meta_dump["ny"], meta_dump["nx"])
            arrays = {}
            for k in (0, steps):
                for f in meta_dump["fields"]:
                    arrays[f"step{k}_{f}"] = np.fromfile(os.path.join(dump, f"step_{k}", f + ".bin"), np.float32).reshape(shape)
            timing = json.load(open(js))
            meta = dict(scene=name + ".scene", steps=steps, dt=dt, fields=meta_dump["fields"], substeps=timing["substeps"],
                        violations=timing["violations"], fallbacks=timing["fallbacks"], flags=extra,
                        made_by="the reference's lawc --scene (its OpenMP CPU Solver)")
            np.savez_compressed(os.path.join(out_dir, name + ".npz"), meta=json.dumps(meta), **arrays)
            print("scene", name)
        finally:
            shutil.rmtree(work, ignore_errors=True)


def vjp_fixture(lawc):
    """lawc --vjp on tests/scenes/heat_vjp.scene: a seeded cotangent of the state after 12 steps stepped back by the
    reference's own reverse-mode driver (every state kept), and the cotangents of the start it gives (T and the param
    D), for pinning the adjoint law and the oracle's reverse pass."""
    out_dir = os.path.join(HERE, "scene")
    steps, h = 12, 0.05
    dt = 0.4 * h * h / 6.0 * 0.9
    shape = (6, 20, 24)
    seed = np.random.default_rng(11).normal(size=shape).astype(np.float32)
    work = tempfile.mkdtemp(prefix="fe_vjp_")
    try:
        seed_dir, dump = os.path.join(work, "seed"), os.path.join(work, "out")
        os.makedirs(seed_dir)
        seed.tofile(os.path.join(seed_dir, "T__adj.bin"))
        with open(os.path.join(seed_dir, "meta.json"), "w") as f:
            json.dump({"nx": shape[2], "ny": shape[1], "nz": shape[0], "h": h, "fields": ["T__adj"]}, f)
        subprocess.run([lawc, "--scene", os.path.join("tests", "scenes", "heat_vjp.scene"), "--steps", str(steps), "--dt", repr(dt),
                        "--vjp", seed_dir, "--dump", dump], check=True, capture_output=True, cwd=ROOT,
                       env=dict(os.environ, OMP_NUM_THREADS="4"))
        arrays = {f: np.fromfile(os.path.join(dump, "adjoint", f + ".bin"), np.float32).reshape(shape) for f in ("T__adj", "D__adj")}
        meta = dict(scene="heat_vjp.scene", steps=steps, dt=dt, made_by="the reference's lawc --vjp (its CPU Solver)")
        np.savez_compressed(os.path.join(out_dir, "heat_vjp.npz"), meta=json.dumps(meta), seed=seed, **arrays)
        print("vjp heat_vjp")
    finally:
        shutil.rmtree(work, ignore_errors=True)


BAD_LAWS = [
    "field T init 0\nterm t\n  d T = (T + 1\n",
    "field T init 0\nterm t\n  d T = T +* 2\n",
    "field T init 0\nterm t\n  d T = nosuch(T)\n",
    "field T init 0\nterm t\n  d T = shift(T, 0.5, 0, 0)\n",
    "field T init 0\nterm t\n  d T = T 2\n",
    "field T init 0\nparam p = T\nterm t\n  d T = p\n",
    "field T init 0\nterm t\n  let h = 2\n  d T = 1\n",
    "field T init 0\nterm t\n  d T = min(T)\n",
    "field T init 0 range 2 1\nterm t\n  d T = 1\n",
    "field T init 0\nterm t\n  max_dt = dt\n  d T = 1\n",
    "field T init 0\nterm t\n  max_dt = T\n  d T = 1\n",
    "field T init 0\nfield T init 1\nterm t\n  d T = 1\n",
    "field T init 0 static\nterm t\n  d T = 1\n  conserves Q\n",
    "field T init 0\nd T = 1\nterm t\n  learned d T = 2\n  d T = 1 +\n",
    "field T init 0\nderive A = T\nderive A = 2 * T\nterm t\n  d T = 1 ^\n",
    "field T init 0\nnet n1 in 3 out 1 act tanh file none\nterm t\n  d T = mlp(n1, T, T)\n",
    "field T init 0\nnet n1 in 2 hidden 200 out 1 act tanh\nterm t\n  d T = flux(n2, T)\n",
    "field T init 0\nterm t\n  d T = poisson(T, 0) + 1 2\n  bogus line\n",
    "field T init 0\nterm t\n  d T = @\n",
    "field T init 0\nterm t\nterm t\n  d T = 1\n  conserves T + T\n",
]


def error_fixtures(lawc):
    """The reference's lawc on malformed laws: the error lines it prints (source name replaced by 'law'), which the
    law front end must give word for word (tests/test_ir_cpu.py)."""
    out = []
    work = tempfile.mkdtemp(prefix="fe_err_")
    try:
        path = os.path.join(work, "bad.law")
        for text in BAD_LAWS:
            with open(path, "w") as f:
                f.write(text)
            res = subprocess.run([lawc, "--ir", path], capture_output=True, text=True)
            lines = [l.replace(path + ":", "law:") for l in (res.stdout + res.stderr).splitlines() if l.startswith(path + ":")]
            out.append({"law": text, "errors": lines, "rc": res.returncode})
    finally:
        shutil.rmtree(work, ignore_errors=True)
    with open(os.path.join(HERE, "law_errors.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("errors", len(out))


def pick(n):
    """The sampled coordinates along an axis of n cells for the fixtures of large lattices: both edges, the quarter
    points and the middle, each with a neighbour either side (16 values at n = 128)."""
    q = [0, 1, 2, 3, n // 4 - 1, n // 4, n // 4 + 1, n // 2 - 1, n // 2, n // 2 + 1, 3 * n // 4 - 1, 3 * n // 4,
         n - 4, n - 3, n - 2, n - 1]
    return np.array(sorted(set(i for i in q if 0 <= i < n)), np.int64)


def heat_fp64(T, D, h, dt, steps):
    """The heat law's explicit scheme (acc = sum over present faces of (neighbour - cell), T += max(D, 0) acc / h^2 dt)
    in FP64 arithmetic and storage: the FP64 solve the FP32 step's error is stated against."""
    from oracle.heat import _faces
    v = np.asarray(T, np.float64)
    for _ in range(steps):
        acc = np.zeros_like(v)
        for nb, valid in _faces(v):
            acc += np.where(valid, nb - v, 0.0)
        v = v + max(D, 0.0) * acc / (h * h) * dt
    return v


def large_fixtures(lawc):
    """The benchmarked lattices, pinned to the reference (lawc) at their full size: too large to commit whole, so each
    fixture keeps the cells on a 16 x 16 x 16 grid of sampled coordinates (pick(n) per axis: edges, quarter points,
    middle), the reference's FNV-1a digest of its final state and the largest |value|; c1_heat_128 also two full planes
    (z = 0 and 64).

    c1_heat_128: the heat law (tests/laws/heat.law) on 128^3, h = 1/128, dt = 0.4 h^2 / 6 (one substep), the sum of 4
      Gaussian blobs from oracle.heat.gaussian_blobs(128, h, seed=0), 100 steps, contracts on; plus the same scheme in
      FP64 (heat_fp64) sampled the same way.
    multifield43_128: the 43-term law (tests/laws/multifield43.law) on 128^3, h = 1/128, dt = 0.1 h^2, 3 steps, fields
      f0..f5 drawn U[-1, 1] in order from numpy default_rng(4343)."""
    from oracle.heat import gaussian_blobs
    n = 128
    h = 1.0 / n
    p = pick(n)
    ix = np.ix_(p, p, p)
    planes = np.array([0, n // 2], np.int64)
    rng = np.random.default_rng(4343)
    specs = [
        dict(name="c1_heat_128", law="heat.law", dt=0.4 * h * h / 6.0, steps=100,
             fields={"T": gaussian_blobs(n, h, seed=0)}),
        dict(name="multifield43_128", law="multifield43.law", dt=0.1 * h * h, steps=3,
             fields={f"f{i}": rng.uniform(-1, 1, (n, n, n)).astype(np.float32) for i in range(6)}),
    ]
    for spec in specs:
        work = tempfile.mkdtemp(prefix="fe_large_")
        try:
            law = os.path.join(LAWS, spec["law"])
            scene = os.path.join(work, "scene")
            with open(scene, "w") as fh:
                fh.write(f"grid {n} {n} {n} {h!r}\nlaw {law}\n")
            init = os.path.join(work, "init")
            os.makedirs(init)
            for name, arr in spec["fields"].items():
                np.ascontiguousarray(arr, np.float32).tofile(os.path.join(init, name + ".bin"))
            dump, js = os.path.join(work, "dump"), os.path.join(work, "t.json")
            subprocess.run([lawc, "--scene", scene, "--init", init, "--steps", str(spec["steps"]), "--dt", repr(spec["dt"]),
                            "--dump", dump, "--every", str(spec["steps"]), "--json", js], check=True, capture_output=True,
                           cwd=ROOT, env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 4)))
            last = os.path.join(dump, f"step_{spec['steps']}")
            meta_dump = json.load(open(os.path.join(last, "meta.json")))
            timing = json.load(open(js))
            arrays = {"pick": p, "planes": planes}
            digest = 0xcbf29ce484222325
            maxabs = {}
            for f in meta_dump["fields"]:
                final = np.fromfile(os.path.join(last, f + ".bin"), np.float32).reshape(n, n, n)
                arrays[f"ref_{f}"] = final[ix]
                if spec["name"] == "c1_heat_128":
                    arrays[f"refplanes_{f}"] = final[planes]
                maxabs[f] = float(np.abs(final).max())
                digest = _fnv1a(f.encode(), digest)
                digest = _fnv1a(np.ascontiguousarray(final, np.float32).view(np.uint8).tobytes(), digest)
            if spec["name"] == "c1_heat_128":
                v64 = heat_fp64(spec["fields"]["T"], 1.0, h, spec["dt"], spec["steps"])
                arrays["fp64_T"] = v64[ix]
                maxabs["fp64_T"] = float(np.abs(v64).max())
            meta = dict(name=spec["name"], law=spec["law"], n=n, h=h, dt=spec["dt"], steps=spec["steps"],
                        substeps=timing["substeps"], violations=timing["violations"], fields=meta_dump["fields"],
                        ref_digest=f"{digest:016x}", max_abs=maxabs,
                        made_by=f"the reference's lawc (its OpenMP CPU Solver), OMP_NUM_THREADS={os.cpu_count() or 4}")
            os.makedirs(os.path.join(HERE, "large"), exist_ok=True)
            np.savez_compressed(os.path.join(HERE, "large", spec["name"] + ".npz"), meta=json.dumps(meta), **arrays)
            print(spec["name"], "substeps", meta["substeps"], "violations", meta["violations"], "digest", meta["ref_digest"])
        finally:
            shutil.rmtree(work, ignore_errors=True)


def _fnv1a(data, h):
    """FNV-1a 64 over `data` (bytes), continuing from h (FieldSet::digest mixes each field's name, then its values'
    bits, in declaration order)."""
    prime = 0x100000001b3
    mask = (1 << 64) - 1
    for b in data:
        h = ((h ^ b) * prime) & mask
    return h


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--lawc", default=os.path.join(ROOT, "oracle", "_ref", "lawc"))
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    if not os.path.exists(args.lawc):
        sys.exit(f"no reference solver at {args.lawc}: build it with `make -C oracle ref`")
    if args.only == "large":
        large_fixtures(args.lawc)
        return
    if args.only == "errors":
        error_fixtures(args.lawc)
        return
    ir_fixtures(args.lawc)
    error_fixtures(args.lawc)
    scene_fixtures(args.lawc)
    vjp_fixture(args.lawc)
    large_fixtures(args.lawc)
    for case in cases():
        if args.only and case["name"] not in args.only.split(","):
            continue
        work = tempfile.mkdtemp(prefix="fe_golden_")
        try:
            meta = run(case, args.lawc, work)
            print(case["name"], "substeps", meta["substeps"], "violations", meta["violations"])
        finally:
            shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    main()
