"""lawc on the B200 backend: the reference's law command line (tools/lawc/main.cpp:1-20), same options and outputs, so
the scripts that drive it (the bench drivers, tools/lawjax) run unchanged with this backend under them.

    python -m fieldcuda.lawc --ir LAW...                   the IR as a listing
    python -m fieldcuda.lawc --ir-json out.json LAW...     the IR as JSON
    python -m fieldcuda.lawc --cuda out.cu [--scene S | --grid NX NY NZ H] LAW...
                                                           the generated sm_100a translation unit (for that lattice)
    python -m fieldcuda.lawc --scene S --steps N [--dt X] [--dump DIR [--every K]] [--dump-only F,G] [--init DIR]
                             [--param NAME VALUE]... [--json FILE [--warmup N]] [--profile]
    python -m fieldcuda.lawc --adjoint OUT [--term T] LAW...

Scenes are the reference's text format (src/field/Scene.hpp:9-17): grid, law, fill, box, ball, noise, param; dumps
are raw float32 per field plus meta.json (Scene.cpp:112-135). The solves run on the GPU; the reference's CPU solver is
not part of this backend, so --backend cpu and --compare are refused. --vjp SEED_DIR differentiates one term (--term)
over the steps (main.cpp:274-361): the scene is the forward's start, SEED_DIR holds the cotangents of its end
(X__adj.bin, the dump format; a missing one is zero), and --dump DIR writes the cotangents of the start to DIR/adjoint;
the driver is the native one (fe_vjp_*: states kept on the card every ceil(sqrt(N)) steps, not all on the host). --learned runs the terms' learned schemes under guard (main.cpp:260): a learned step that breaks a contract is
undone and taken classically, and the undone steps are counted in --profile and --json as the reference counts them.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

SCENE_COUNTS = {"fill": 0, "box": 6, "ball": 4, "noise": 1}


class Scene:
    """A starting state as text: the lattice, the law files, the field ops in order, the params."""

    def __init__(self):
        self.grid = (64, 64, 1, 1.0)
        self.laws = []
        self.ops = []
        self.params = []


def load_scene(path):
    scene = Scene()
    for number, raw in enumerate(open(path), 1):
        line = raw.split("#", 1)[0].split()
        if not line:
            continue
        kind, words = line[0], line[1:]
        where = f"{path}:{number}: "
        if kind == "grid":
            try:
                nx, ny, nz, h = int(words[0]), int(words[1]), int(words[2]), float(words[3])
            except (IndexError, ValueError):
                raise ValueError(where + "expected 'grid NX NY NZ METRES'")
            if nx < 1 or ny < 1 or nz < 1 or h <= 0.0:
                raise ValueError(where + "expected 'grid NX NY NZ METRES'")
            scene.grid = (nx, ny, nz, h)
        elif kind == "law":
            scene.laws.append(words[0] if words else "")
        elif kind == "param":
            try:
                scene.params.append((words[0], float(words[1])))
            except (IndexError, ValueError):
                raise ValueError(where + "expected 'param NAME VALUE'")
        elif kind in SCENE_COUNTS:
            n = SCENE_COUNTS[kind]
            if len(words) < 2:
                raise ValueError(where + f"expected '{kind} FIELD VALUE ...'")
            try:
                args = [float(w) for w in words[2:2 + n]]
                value = float(words[1])
            except ValueError:
                raise ValueError(where + f"expected '{kind} FIELD VALUE ...'")
            if len(args) < n:
                raise ValueError(where + f"{kind} needs {n} numbers after the value")
            scene.ops.append((kind, words[0], value, args))
        else:
            raise ValueError(where + f"unknown line '{kind}' (grid, law, param, fill, box, ball, noise)")
    return scene


def cell_noise(seed, index):
    """A splitmix64-style mix of (seed, linear cell index) as a float in [0, 1): no generator state, so the same scene
    text gives the same start (Scene.cpp:101-106). `index`: a uint64 array."""
    with np.errstate(over="ignore"):
        h = np.uint64(int(seed) & 0xFFFFFFFFFFFFFFFF) * np.uint64(0x9E3779B97F4A7C15) ^ index * np.uint64(0xBF58476D1CE4E5B9)
        h ^= h >> np.uint64(31)
        h *= np.uint64(0x94D049BB133111EB)
        h ^= h >> np.uint64(29)
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def scene_fields(scene, names, inits):
    """The fields (dict name -> (nz, ny, nx) float32) after the scene's ops, from the law's init values."""
    nx, ny, nz, _ = scene.grid
    fields = {n: np.full((nz, ny, nx), np.float32(inits[n]), np.float32) for n in names}
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    index = (x.astype(np.uint64) + np.uint64(nx) * (y.astype(np.uint64) + np.uint64(ny) * z.astype(np.uint64)))
    for kind, name, value, args in scene.ops:
        if name not in fields:
            raise ValueError(f"the law has no field '{name}'")
        v = fields[name]
        if kind == "fill":
            v[...] = np.float32(value)
        elif kind == "box":
            m = (x >= args[0]) & (y >= args[1]) & (z >= args[2]) & (x < args[3]) & (y < args[4]) & (z < args[5])
            v[m] = np.float32(value)
        elif kind == "ball":
            dx, dy, dz = x - args[0], y - args[1], z - args[2]
            v[dx * dx + dy * dy + dz * dz <= args[3] * args[3]] = np.float32(value)
        else:
            v += (value * cell_noise(args[0], index)).astype(np.float32)
    return fields


def dump_fields(solver, directory, only=""):
    os.makedirs(directory, exist_ok=True)
    names = solver.field_names if not only else [n for n in solver.field_names if n in only.split(",")]
    nz, ny, nx = solver.shape
    for n in names:
        solver.values(n).tofile(os.path.join(directory, n + ".bin"))
    with open(os.path.join(directory, "meta.json"), "w") as f:
        f.write(json.dumps({"nx": nx, "ny": ny, "nz": nz, "h": solver.h, "fields": names}, separators=(",", ":")) + "\n")


def load_fields(solver, directory):
    if not os.path.isdir(directory):
        raise ValueError(f"no state at {directory}")
    cells = int(np.prod(solver.shape))
    for n in solver.field_names:
        path = os.path.join(directory, n + ".bin")
        if not os.path.exists(path):
            continue
        v = np.fromfile(path, np.float32)
        if v.size != cells:
            raise ValueError(f"{path} holds {v.size} floats, the lattice {cells}")
        solver.set_field(n, v.reshape(solver.shape))


def print_profile(solver, step_ms):
    """One step's profile in the reference's layout (main.cpp:71-92): the card's time and launches, the undone learned
    steps, then per running term its substeps and whether its learned scheme was kept or fell back."""
    p = solver.profile()
    line = f"  B200: step {step_ms:.3f} ms (card {p['gpu_ms']:.3f} ms, {p['launches']} launches)"
    if p["fallbacks"] > 0:
        line += f", {p['fallbacks']} learned step(s) undone"
    print(line)
    marks = {"learned": "  learned", "fell back": "  FELL BACK"}
    for name, idle, sub, how in zip(solver.term_names, solver.idle_terms(), solver.last_substeps(), solver.term_learned()):
        if not idle:
            print(f"    {name:<22} x{sub}{marks.get(how, '')}")


def run_vjp(args, scene, text):
    """--vjp: the scene's start stepped forward, then the seed cotangents stepped back; prints the reference's line."""
    import torch
    from . import _lib
    from .adjoint import LawVJP
    nx, ny, nz, h = scene.grid
    try:
        vjp = LawVJP(text, nx, ny, nz, h, term=args.term or None)
    except _lib.FeError as e:
        print(e, file=sys.stderr)
        return 1
    try:
        for name, value in scene.params + [(n, float(v)) for n, v in args.param]:
            vjp.set_param(name, value)
        p = vjp.primal
        inits = {n: p.field_info(n)["init"] for n in p.field_names}
        for name, v in scene_fields(scene, p.field_names, inits).items():
            p.set_field(name, v)
        p.refresh_derived()
        if args.init:
            load_fields(p, args.init)
            p.refresh_derived()
        if not os.path.isdir(args.vjp):
            raise ValueError(f"no seed at {args.vjp}")
        seeds = {}
        for name in vjp.state:
            path = os.path.join(args.vjp, name + "__adj.bin")
            if os.path.exists(path):
                v = np.fromfile(path, np.float32)
                if v.size != nx * ny * nz:
                    raise ValueError(f"{path} holds {v.size} floats, the lattice {nx * ny * nz}")
                seeds[name] = torch.tensor(v.reshape(nz, ny, nx), device="cuda")
        t0 = time.perf_counter()
        vjp.forward({}, args.dt, args.steps)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        vjp.backward(seeds)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
    except (ValueError, _lib.FeError) as e:
        print(e, file=sys.stderr)
        vjp.close()
        return 1
    term = args.term or vjp.primal.term_names[0]
    print(f"vjp of '{term}' over {args.steps} steps on B200: forward {(t1 - t0) * 1e3:g} ms, backward {(t2 - t1) * 1e3:g} ms")
    if args.dump:
        dump_fields(vjp.adj, os.path.join(args.dump, "adjoint"))
    vjp.close()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(prog="lawc", description="the law compiler and runner on the B200 backend")
    ap.add_argument("laws", nargs="*")
    ap.add_argument("--ir", action="store_true")
    ap.add_argument("--ir-json")
    ap.add_argument("--cuda")
    ap.add_argument("--scene")
    ap.add_argument("--grid", nargs=4)
    ap.add_argument("--steps", type=int, default=0)
    ap.add_argument("--dt", type=float, default=0.05)
    ap.add_argument("--backend", default="cuda")
    ap.add_argument("--learned", action="store_true")
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--eager", action="store_true")
    ap.add_argument("--compare", action="store_true")
    ap.add_argument("--dump")
    ap.add_argument("--every", type=int, default=0)
    ap.add_argument("--dump-only", default="")
    ap.add_argument("--init")
    ap.add_argument("--param", nargs=2, action="append", default=[])
    ap.add_argument("--json")
    ap.add_argument("--warmup", type=int, default=0)
    ap.add_argument("--adjoint")
    ap.add_argument("--vjp")
    ap.add_argument("--term", default="")
    args = ap.parse_args(argv)

    if args.backend not in ("cuda", "b200"):
        print(f"no {args.backend} backend here: this lawc runs the B200 backend only", file=sys.stderr)
        return 1
    for flag, what in ((args.compare, "--compare (the reference's CPU solver is not part of this backend)"),):
        if flag:
            print(f"not in this lawc: {what}", file=sys.stderr)
            return 2
    try:
        scene = load_scene(args.scene) if args.scene else Scene()
    except ValueError as e:
        print(e, file=sys.stderr)
        return 1
    paths = args.laws or scene.laws
    if args.grid:
        scene.grid = (int(args.grid[0]), int(args.grid[1]), int(args.grid[2]), float(args.grid[3]))
    texts = []
    for p in paths:
        if not os.path.exists(p):
            print(f"no law at {p}", file=sys.stderr)
            return 1
        texts.append(open(p).read())
    if not texts:
        print("no law: give LAW files or a scene with 'law' lines (--help)", file=sys.stderr)
        return 2
    text = "\n".join(texts)
    source = os.path.basename(paths[0])

    from . import _lib
    from .solver import Solver, cuda_source, ir_json, ir_listing
    try:
        nets = json.loads(ir_json(text))["nets"]
    except _lib.FeError as e:
        print(e, file=sys.stderr)
        return 1
    for net in nets:
        if not net["loaded"]:
            print(f"note: net '{net['name']}' has no weights at {net['file']} (it starts untrained: its output is 0)",
                  file=sys.stderr)
    try:
        if args.ir:
            print(ir_listing(text), end="")
        if args.ir_json:
            with open(args.ir_json, "w") as f:
                f.write(ir_json(text))
            print(f"IR written to {args.ir_json}")
        if args.cuda:
            nx, ny, nz, h = scene.grid
            with open(args.cuda, "w") as f:
                f.write(cuda_source(text, nx, ny, nz, h))
            print(f"CUDA written to {args.cuda}")
        if args.adjoint:
            adj = _lib.text_call("fe_law_adjoint", text.encode(), args.term.encode())
            with open(args.adjoint, "w") as f:
                f.write(adj)
            print(f"adjoint law written to {args.adjoint}")
    except _lib.FeError as e:
        print(e, file=sys.stderr)
        return 1
    if args.steps <= 0:
        return 0

    nx, ny, nz, h = scene.grid
    if args.vjp:
        return run_vjp(args, scene, text)
    try:
        s = Solver(text, nx, ny, nz, h, source)
    except _lib.FeError as e:
        print(e, file=sys.stderr)
        return 1
    try:
        if args.learned:
            s.set_learned(True)
        for name, value in scene.params + [(n, float(v)) for n, v in args.param]:
            if not s.set_param(name, value):
                print(f"the law has no param '{name}'", file=sys.stderr)
                return 1
        inits = {n: s.field_info(n)["init"] for n in s.field_names}
        for name, v in scene_fields(scene, s.field_names, inits).items():
            s.set_field(name, v)
        s.refresh_derived()
        if args.init:
            load_fields(s, args.init)
            s.refresh_derived()
    except ValueError as e:
        print(e, file=sys.stderr)
        return 1
    print(f"{len(s.field_names)} fields, {len(s.term_names)} terms, {len(nets)} nets; grid {nx}x{ny}x{nz} at {h:g} m; {args.steps} steps of "
          f"{args.dt:g} s on B200")
    if args.dump:
        dump_fields(s, os.path.join(args.dump, "step_0"), args.dump_only)
    total = 0.0
    timed, gpu = [], 0.0
    violations = fallbacks = 0
    for step in range(1, args.steps + 1):
        t0 = time.perf_counter()
        s.step(args.dt)
        ms = (time.perf_counter() - t0) * 1e3
        total += ms
        fallbacks += s.profile()["fallbacks"]
        if step > args.warmup:
            timed.append(ms)
            gpu += s.profile()["gpu_ms"]
        found = s.violations()
        violations += len(found)
        for v in found:
            if violations < 12:
                print(f"  step {step}: [{v.term}] {v.field} {v.kind}: {v.detail}", file=sys.stderr)
        if args.dump and args.every > 0 and step % args.every == 0:
            dump_fields(s, os.path.join(args.dump, f"step_{step}"), args.dump_only)
        if args.profile and (step == 1 or step == args.steps):
            print_profile(s, ms)
    if args.dump and (args.every <= 0 or args.steps % args.every != 0):
        dump_fields(s, os.path.join(args.dump, f"step_{args.steps}"), args.dump_only)
    print(f"mean step {total / args.steps:g} ms, {violations} contract violation(s)")
    if args.json:
        out = {"backend": "B200", "cells": nx * ny * nz, "steps": len(timed),
               "mean_ms": (sum(timed) / len(timed)) if timed else 0.0,
               "median_ms": sorted(timed)[len(timed) // 2] if timed else 0.0,
               "gpu_ms": gpu / len(timed) if timed else 0.0, "violations": violations, "fallbacks": fallbacks,
               "substeps": s.last_substeps(), "terms": {t: 0.0 for t in s.term_names}}
        with open(args.json, "w") as f:
            f.write(json.dumps(out) + "\n")
    s.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
