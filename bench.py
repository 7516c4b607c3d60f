#!/usr/bin/env python3
"""Benchmark of the law-step hot path on B200: the 7-point FP32 heat step, d T = diffuse(1, T), conserves T, at 512^3.

One step = one explicit Euler step of the whole 512^3 lattice (one substep: dt = 0.4 h^2 / 6 is exactly max_dt), with
the conserved-total, range/NaN, bounds and change contracts checked on the card in the same pass. Metric: effective
HBM bandwidth at the reference's own unit of 8 bytes a cell a step (one fp32 read and one write), against the measured
copy roof.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--size 512]

Prints ONE JSON line (rank 0). With --gpus N > 1 (torchrun), the lattice is 512 x 512 x 512N, one 512-plane z-slab a
rank (weak scaling): each rank steps its slab plus one halo plane a side, the halo planes are exchanged over NCCL after
every step and conservation is judged over the ranks (fieldcuda/slabs.py); timed with CUDA events, max over ranks.
"""
import argparse
import ctypes
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "online-physics-cuda_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, ROOT)

BYTES_PER_CELL = 8  # one fp32 read of T and one write of the next T (the reference's unit, stencil_bench.cpp:188)
FALLBACK_HBM_GBS = 6650.0


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def heat_workload(n):
    """The headline workload's name, the same on both arms."""
    return (f"heat law d T = diffuse(1, T), conserves T, {n}^3 fp32 a GPU (on N GPUs one {n} x {n} x {n}N lattice in "
            f"z-slabs, halo planes over NCCL), h = 1/{n}, dt = 0.4 h^2/6 (1 substep), contracts checked every step")


def profile_traffic(name):
    """dram bytes per launch of the dominant kernel from the committed ncu summary (profiles/<name>.md), or None."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = None

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                      "-i", str(self.index), "-lms", "100"], stdout=self.out, stderr=subprocess.DEVNULL)
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.strip()]
        os.unlink(self.out.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def init_dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- the reference's CPU solver (the oracle built from the reference's sources), timed on this host ----------------

HEAT_LAW = """field T init 0 range -1000000 1000000
param D = 1
term conduction
  d T = diffuse(D, T)
  conserves T
  max_dt = 0.4 * h * h / (6 * D)
"""


def cpu_reference_heat(n, steps, warmup, threads):
    """Times the reference's own OpenMP CPU solver (oracle/_ref/lawc) on the heat law at n^3. Returns (ms/step, kind,
    cores) or None when the binary is absent. Falls back to nothing: the oracle port is in oracle/heat.py."""
    lawc = os.path.join(ROOT, "oracle", "_ref", "lawc")
    if not os.path.exists(lawc):
        return None
    import numpy as np
    from oracle import heat as oh
    h = 1.0 / n
    dt = 0.4 * h * h / 6.0
    work = tempfile.mkdtemp(prefix="fe_cpu_")
    try:
        law = os.path.join(work, "heat.law")
        open(law, "w").write(HEAT_LAW)
        scene = os.path.join(work, "heat.scene")
        open(scene, "w").write(f"grid {n} {n} {n} {h!r}\nlaw {law}\n")
        init = os.path.join(work, "init")
        os.makedirs(init)
        oh.gaussian_blobs(n, h, seed=0).tofile(os.path.join(init, "T.bin"))
        out = os.path.join(work, "t.json")
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        subprocess.run([lawc, "--scene", scene, "--init", init, "--steps", str(steps + warmup), "--dt", repr(dt),
                        "--json", out, "--warmup", str(warmup)], check=True, env=env, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL)
        ms = json.load(open(out))["mean_ms"]
        return ms, "reference", threads
    finally:
        shutil.rmtree(work, ignore_errors=True)


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    n = args.size
    threads = os.cpu_count() or 1
    steps = args.steps
    # Bounded: each CPU step at 512^3 takes seconds; cap the sample so the run ends within a few minutes.
    cells = n ** 3
    sample_steps = max(1, min(steps, int(60e9 / (cells * 40))))
    res = cpu_reference_heat(n, sample_steps, min(args.warmup, 1), threads)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/lawc (the reference's CPU solver) is not built"}))
        return
    ms, kind, cores = res
    gbs = BYTES_PER_CELL * cells / (ms * 1e-3) / 1e9
    sample = f"{sample_steps} timed steps of the {n}^3 heat law after 1 warm-up, reference lawc, OMP_NUM_THREADS={cores}"
    print(json.dumps({
        "impl": "reference", "metric": "7-pt stencil effective HBM GB/s (8 B/cell/step)", "value": gbs, "unit": "GB/s",
        "n_gpus": world, "steps": sample_steps, "warmup": 1, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": heat_workload(n), "cells_per_gpu": cells},
        "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ---- our arm ---------------------------------------------------------------------------------------------------------

def _events(stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    return e0, e1


def handwritten_ms(n, h, dt, cells, stream, variant=0, zchunk=32, reps=10):
    """The hand-written kernel (same arithmetic, contracts on): ms per step, for comparison."""
    import torch
    from fieldcuda import _lib, kernels
    a = torch.rand((n, n, n), device="cuda")
    b = torch.empty_like(a)
    ws = kernels.heat7_workspace((n, n, n), variant, zchunk)
    flags = dict(lo=-1e6, hi=1e6, variant=variant, zchunk=zchunk, check=_lib.FE_HEAT7_BEFORE | _lib.FE_HEAT7_AFTER)
    with torch.cuda.stream(stream):
        for _ in range(3):
            kernels.check_reset(ws, stream)
            kernels.heat7_step(a, b, 1.0, h, dt, workspace=ws, stream=stream, **flags)
        e0, e1 = _events(stream)
        e0.record(stream)
        for _ in range(reps):
            kernels.check_reset(ws, stream)
            kernels.heat7_step(a, b, 1.0, h, dt, workspace=ws, stream=stream, **flags)
            a, b = b, a
        e1.record(stream)
        stream.synchronize()
    return e0.elapsed_time(e1) / reps


def copy_roof_gbs(cells, stream, reps=10):
    import torch
    from fieldcuda import kernels
    ca = torch.empty(cells, dtype=torch.float32, device="cuda")
    cb = torch.empty_like(ca)
    with torch.cuda.stream(stream):
        for _ in range(3):
            kernels.copy_f32(ca, cb, stream)
        e0, e1 = _events(stream)
        e0.record(stream)
        for _ in range(reps):
            kernels.copy_f32(ca, cb, stream)
        e1.record(stream)
        stream.synchronize()
    return 2 * 4 * cells * reps / (e0.elapsed_time(e1) * 1e-3) / 1e9


def pct(values, q):
    import numpy as np
    return float(np.percentile(np.asarray(values, dtype=np.float64), q))


def step_times(s, dt, steps, stream_sync):
    """Per-step times of `steps` steps of solver `s`: device time of each step (CUDA events on the solver's stream
    around it; contracts checked on the card, judged after the run: lazy readback, nothing fetched) and the host's wall
    time of each step when every step is judged on the host (its contract records read back: the wall time a caller
    that waits for each step sees). Returns (device ms list, wall ms list, violations)."""
    import torch
    st = torch.cuda.ExternalStream(s.stream)
    s.set_deferred(True)
    for _ in range(3):
        s.step(dt)
    s.sync()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    stream_sync()
    ev[0].record(st)
    for i in range(steps):
        s.step(dt)
        ev[i + 1].record(st)
    st.synchronize()
    dev = [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]
    s.sync()
    broken = len(s.violations())
    s.set_deferred(False)
    wall = []
    for _ in range(steps):
        t0 = time.perf_counter()
        s.step(dt)
        wall.append((time.perf_counter() - t0) * 1e3)
        broken += len(s.violations())
    return dev, wall, broken


def stats(ms):
    import numpy as np
    return {"p50_ms": pct(ms, 50), "p99_ms": pct(ms, 99), "mean_ms": float(np.mean(ms))}


C1_FIXTURE = os.path.join(ROOT, "tests", "golden", "large", "c1_heat_128.npz")


def c1_section(stream_sync, peak):
    """BASELINE's first configuration as stated: the heat law on 128^3 (h = 1/128, dt = 0.4 h^2 / 6, one substep),
    4 seeded Gaussian blobs, 100 steps, contracts on. Per-step device and wall times, the engine against the
    hand-written kernel (every step, to the bit), and the final state against the reference's CPU solver and against
    the same scheme in FP64 (tests/golden/large/c1_heat_128.npz: both at its sampled cells and planes); the
    reference's own OpenMP solver timed on the same steps on this host."""
    import numpy as np
    import torch
    from fieldcuda import kernels
    from fieldcuda.solver import Solver
    from oracle import heat as oh
    n, steps = 128, 100
    h = 1.0 / n
    dt = 0.4 * h * h / 6.0
    T0 = oh.gaussian_blobs(n, h, seed=0)
    s = Solver(HEAT_LAW, n, n, n, h, "heat.law")
    s.set_field("T", T0)
    a = torch.from_numpy(T0).cuda()
    b = torch.empty_like(a)
    eng = torch.empty_like(a)
    ws = kernels.heat7_workspace(T0.shape, 0, 16)
    st = torch.cuda.ExternalStream(s.stream)
    dev, wall, same, broken = [], [], True, 0
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream_sync()
        t0 = time.perf_counter()
        e0.record(st)
        s.step(dt)          # judged on the host before it returns
        e1.record(st)
        wall.append((time.perf_counter() - t0) * 1e3)
        st.synchronize()
        dev.append(e0.elapsed_time(e1))
        broken += len(s.violations())
        kernels.heat7_step(a, b, 1.0, h, dt, variant=0, zchunk=16, check=0, workspace=ws)
        a, b = b, a
        s.fetch_device("T", eng)
        torch.cuda.synchronize()
        same = same and bool(torch.equal(eng.view(torch.int32), a.view(torch.int32)))
    got = s.values("T").astype(np.float64)
    d1 = s.digest()
    s.close()
    s = Solver(HEAT_LAW, n, n, n, h, "heat.law")
    s.set_field("T", T0)
    for _ in range(steps):
        s.step(dt)
    deterministic = s.digest() == d1
    s.close()
    out = {"lattice": "128^3", "steps": steps, "dt": dt, "device": stats(dev), "wall_judged_each_step": stats(wall),
           "gbs_device_mean": BYTES_PER_CELL * n ** 3 / (stats(dev)["mean_ms"] * 1e-3) / 1e9,
           "bit_identical_to_handwritten_every_step": same, "deterministic_two_runs": deterministic,
           "violations": broken}
    out["roofline_frac_mean_step"] = out["gbs_device_mean"] / peak
    if os.path.exists(C1_FIXTURE):
        z = np.load(C1_FIXTURE)
        meta = json.loads(str(z["meta"]))
        p = z["pick"]
        ix = np.ix_(p, p, p)
        out["rel_err_vs_reference_cpu"] = max(float(np.abs(got[ix] - z["ref_T"]).max()),
                                              float(np.abs(got[z["planes"]] - z["refplanes_T"]).max())) / meta["max_abs"]["T"]
        out["rel_err_vs_fp64"] = float(np.abs(got[ix] - z["fp64_T"]).max()) / meta["max_abs"]["fp64_T"]
        out["reference_rel_err_vs_fp64"] = float(np.abs(z["ref_T"] - z["fp64_T"]).max()) / meta["max_abs"]["fp64_T"]
        out["err_note"] = ("max |difference| / max |T| at the fixture's 4096 sampled cells (edges, quarter points, middle) "
                           "and two full planes; the FP64 solve is the same scheme in double (tests/golden/make_golden.py)")
    res = cpu_reference_heat(n, steps, 1, os.cpu_count() or 1)
    if res is not None:
        ms, kind, cores = res
        out["cpu_baseline"] = {"value": ms, "unit": "ms/step", "cores": cores, "kind": kind,
                               "sample": f"{steps} timed steps of the 128^3 heat law after 1 warm-up, reference lawc"}
        out["speedup_vs_cpu_device_p50"] = ms / out["device"]["p50_ms"]
    return out


def c2_section(stream_sync, peak, cpu=True):
    """BASELINE's second configuration: the heat law at 256^3 and 512^3 over 1000 steps, and the 43-term, 6-field law
    (tests/laws/multifield43.law, seed 0) at 256^3 (1000 steps) and 512^3 (300 steps), with lazy readback (nothing
    fetched; contracts checked on the card every step, judged after the run): p50/p99 of the per-step device time,
    the wall time of a step judged on the host, effective bandwidth at the algorithmic bytes and its fraction of the
    measured copy roof; the reference's OpenMP solver on the 43-term law at 256^3 on this host."""
    import numpy as np
    from fieldcuda.solver import Solver
    from fieldcuda.workloads import multifield_bytes_per_cell, multifield_law
    from oracle import heat as oh
    out = {}
    for n in (256, 512):
        h = 1.0 / n
        dt = 0.4 * h * h / 6.0
        s = Solver(HEAT_LAW, n, n, n, h, "heat.law")
        s.set_field("T", oh.gaussian_blobs(n, h, seed=0))
        dev, wall, broken = step_times(s, dt, 1000, stream_sync)
        s.close()
        d = stats(dev)
        gbs = BYTES_PER_CELL * n ** 3 / (d["mean_ms"] * 1e-3) / 1e9
        out[f"heat_{n}"] = {"steps": 1000, "device": d, "wall_judged_each_step": stats(wall), "gbs": gbs,
                            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "frac": gbs / peak,
                                         "bytes_per_cell_step": BYTES_PER_CELL}, "violations": broken}
    text, rw = multifield_law(0)
    bpc = multifield_bytes_per_cell(rw)
    for n, steps in ((256, 1000), (512, 300)):
        h = 1.0 / n
        dt = 0.1 * h * h
        s = Solver(text, n, n, n, h, "multifield43.law")
        rng = np.random.default_rng(43)
        for i in range(6):
            s.set_field(f"f{i}", rng.uniform(-1, 1, (n, n, n)).astype(np.float32))
        s.step(dt)
        launches = s.profile()["launches"]
        passes = sum(s.last_substeps())
        dev, wall, broken = step_times(s, dt, steps, stream_sync)
        s.close()
        d = stats(dev)
        gbs = bpc * n ** 3 / (d["mean_ms"] * 1e-3) / 1e9
        out[f"multifield43_{n}"] = {"steps": steps, "device": d, "wall_judged_each_step": stats(wall), "gbs": gbs,
                                    "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "frac": gbs / peak,
                                                 "bytes_per_cell_step": bpc},
                                    "launches_per_step": launches, "term_passes_per_step": passes, "violations": broken}
    if cpu:
        res = cpu_reference_law(text, 256, 0.1 / 256 ** 2, 2, {f"f{i}": ("uniform", 43 + i) for i in range(6)})
        if res is not None:
            ms, cores = res
            out["multifield43_256"]["cpu_baseline"] = {
                "value": ms, "unit": "ms/step", "cores": cores, "kind": "reference",
                "sample": "2 timed steps of the 43-term law at 256^3 after 1 warm-up, reference lawc"}
            out["multifield43_256"]["speedup_vs_cpu_device_p50"] = ms / out["multifield43_256"]["device"]["p50_ms"]
    out["note"] = ("device: CUDA events around every step on the solver's stream; wall: host time of a step judged on the "
                   "host (its records read back). Multi-field bytes: per term 4 B a cell for every field it reads or "
                   "writes plus 4 B for every field it writes (fieldcuda/workloads.py)")
    return out


def cpu_reference_run(law_path, grid, dt, steps, fields):
    """The reference's own OpenMP CPU solver (oracle/_ref/lawc) on a law file: ms a step over `steps` after one warm-up
    step, all host cores. grid = (nx, ny, nz, h); fields: name -> (nz, ny, nx) float32 starting values. None without
    lawc."""
    lawc = os.path.join(ROOT, "oracle", "_ref", "lawc")
    if not os.path.exists(lawc):
        return None
    import numpy as np
    threads = os.cpu_count() or 1
    nx, ny, nz, h = grid
    work = tempfile.mkdtemp(prefix="fe_cpu_")
    try:
        scene = os.path.join(work, "s.scene")
        open(scene, "w").write(f"grid {nx} {ny} {nz} {h!r}\nlaw {law_path}\n")
        init = os.path.join(work, "init")
        os.makedirs(init)
        for k, v in fields.items():
            np.ascontiguousarray(v, np.float32).tofile(os.path.join(init, k + ".bin"))
        out = os.path.join(work, "t.json")
        subprocess.run([lawc, "--scene", scene, "--init", init, "--steps", str(steps + 1), "--dt", repr(dt), "--json", out,
                        "--warmup", "1"], check=True, env=dict(os.environ, OMP_NUM_THREADS=str(threads)),
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        return json.load(open(out))["mean_ms"], threads
    finally:
        shutil.rmtree(work, ignore_errors=True)


def cpu_reference_law(text, n, dt, steps, fields):
    """Times the reference's own OpenMP CPU solver (oracle/_ref/lawc) on law `text` at n^3: ms/step over `steps` after
    one warm-up, all host cores. `fields`: name -> ("uniform", seed) starting states, U[-1, 1]. None without lawc."""
    lawc = os.path.join(ROOT, "oracle", "_ref", "lawc")
    if not os.path.exists(lawc):
        return None
    import numpy as np
    threads = os.cpu_count() or 1
    work = tempfile.mkdtemp(prefix="fe_cpu_")
    try:
        law = os.path.join(work, "law.law")
        open(law, "w").write(text)
        scene = os.path.join(work, "s.scene")
        open(scene, "w").write(f"grid {n} {n} {n} {1.0 / n!r}\nlaw {law}\n")
        init = os.path.join(work, "init")
        os.makedirs(init)
        for name, (_, seed) in fields.items():
            np.random.default_rng(seed).uniform(-1, 1, (n, n, n)).astype(np.float32).tofile(os.path.join(init, name + ".bin"))
        out = os.path.join(work, "t.json")
        subprocess.run([lawc, "--scene", scene, "--init", init, "--steps", str(steps + 1), "--dt", repr(dt), "--json", out,
                        "--warmup", "1"], check=True, env=dict(os.environ, OMP_NUM_THREADS=str(threads)),
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        return json.load(open(out))["mean_ms"], threads
    finally:
        shutil.rmtree(work, ignore_errors=True)


HESTON_EXPLICIT_T_LAW = os.path.join(ROOT, "tests", "laws", "heston_explicit_T.law")
HESTON_DOUGLAS_LAW = os.path.join(ROOT, "tests", "laws", "heston_douglas.law")
HESTON_CF = os.path.join(ROOT, "tests", "golden", "heston", "cf_2048.npz")
HESTON_BUCKETS = ((128, 64), (256, 128), (512, 256))


def err_stats(e):
    import numpy as np
    e = np.asarray(e, np.float64)
    return {"options": int(e.size), "rms": float(np.sqrt(np.mean(e * e))), "median": float(np.median(e)),
            "p90": float(np.percentile(e, 90)), "max": float(e.max())}


def plain_heston_bucket(opts, nx, ny, stream_sync, planes=None):
    """The plain method on one bucket: explicit Euler (tests/laws/heston_explicit_T.law: heston_explicit.law's operator
    with each option's time to maturity scaled onto s in [0, 1]) through fe_law_step, the bucket's options (or the
    first `planes` of them) as the z-planes of one lattice, stepped at the law's stability limit to s = 1. Returns
    (device ms, substeps, prices)."""
    import numpy as np
    import torch
    from fieldcuda.heston import lattice_fields, price_at
    from fieldcuda.solver import Solver
    group = opts if planes is None else opts[:planes]
    fields, h = lattice_fields(group, nx, ny)
    fields["mat"] = np.broadcast_to(np.array([o["maturity"] for o in group], np.float32)[:, None, None],
                                    fields["V"].shape).copy()
    s = Solver(open(HESTON_EXPLICIT_T_LAW).read(), nx, ny, len(group), h, "heston_explicit_T.law")
    for k, v in fields.items():
        s.set_field(k, v)
    # ds = 1 in chunks the substep cap (4096 a step) allows: the limit is 0.25 h^2 / max(T (var + sig_v h / 2)).
    limit = min(0.25 * h * h / (o["maturity"] * o["sigma"] * ny * h) for o in group)
    chunks = int(np.ceil(1.0 / limit / 4000.0))
    st = torch.cuda.ExternalStream(s.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream_sync()
    e0.record(st)
    substeps = 0
    for _ in range(chunks):
        s.step(1.0 / chunks)
        substeps += s.last_substeps()[0]
    e1.record(st)
    st.synchronize()
    ms = e0.elapsed_time(e1)
    V = s.values("V")
    s.close()
    return ms, substeps, np.array([price_at(V[z], o) for z, o in enumerate(group)])


def heston_batch_section(stream_sync):
    """Batched Heston ADI (Douglas, theta = 1/2): 2048 seeded options on their own grids (128 x 64, 256 x 128 or 512 x
    256), 512 steps, priced in one persistent launch (autotuned, CUDA-graph replayed), against the plain method at the
    same grids: explicit Euler (the same operator, tests/laws/heston_explicit_T.law, each option's maturity scaled onto
    one time axis) through the law backend, every bucket's options as the z-planes of one lattice, the reference's way
    of batching. The two smaller buckets run end to end, every option priced by both methods; the 512 x 256 bucket's
    plain time is extrapolated from 128 of its options over 2000 substeps (labelled). Errors are against FP64
    characteristic-function prices of the same options (tests/golden/heston/cf_2048.npz), by bucket and by Feller ratio
    2 kappa theta / sigma^2. The reference's own OpenMP solver is timed on a sample of the 256 x 128 bucket."""
    import numpy as np
    from fieldcuda.heston import DOUGLAS, HestonBatch, sample_options

    n, steps = 2048, 512
    opts = sample_options(n, 1)
    cf = None
    if os.path.exists(HESTON_CF):
        z = np.load(HESTON_CF)
        if int(z["seed"]) == 1 and len(z["price"]) == n and np.allclose(z["strike"], [o["strike"] for o in opts]):
            cf = z["price"]
    with HestonBatch(opts, steps, DOUGLAS) as b:
        split = b.autotune()
        clusters, tasks = b.layout()
        b.run(use_graph=True)
        prices = b.prices().astype(np.float64)
        runs = [b.time(use_graph=True) for _ in range(3)]
    ms = statistics.median(runs)
    cells = sum(o["nx"] * o["ny"] for o in opts)
    out = {"options": n, "steps": steps, "scheme": "Douglas (theta = 1/2)", "ms": ms, "options_per_s": n / (ms * 1e-3),
           "cell_steps_per_s": cells * steps / (ms * 1e-3), "split": {"mx": split[0], "sy": split[1], "threads": split[2]},
           "clusters": clusters, "tasks": tasks, "readout": "bicubic (4 x 4 cell centres, local Lagrange) at (ln S0, v0)",
           "hbm_bytes": 8 * cells, "hbm_note": "each option's state stays in shared memory for all its steps: 8 B a cell a run"}
    buckets = {f"{nx}x{ny}": [i for i, o in enumerate(opts) if (o["nx"], o["ny"]) == (nx, ny)] for nx, ny in HESTON_BUCKETS}
    if cf is not None:
        err = np.abs(prices - cf)
        feller = np.array([2 * o["kappa"] * o["theta"] / o["sigma"] ** 2 for o in opts])
        out["error_vs_cf"] = err_stats(err)
        out["error_vs_cf_by_bucket"] = {k: err_stats(err[idx]) for k, idx in buckets.items()}
        bins = ((0, 0.25), (0.25, 0.5), (0.5, 1.0), (1.0, 1e9))
        out["error_vs_cf_by_feller_ratio"] = {f"[{a}, {b})": err_stats(err[(feller >= a) & (feller < b)])
                                              for a, b in bins if np.any((feller >= a) & (feller < b))}
        below = np.array([o["v0"] < 0.5 * o["sigma"] * 6.0 / o["nx"] for o in opts])
        out["error_vs_cf_v0_below_first_row"] = err_stats(err[below]) if below.any() else None
        worst = np.argsort(err)[-5:][::-1]
        out["worst_options"] = [dict(err=float(err[i]), price=float(prices[i]), cf=float(cf[i]), feller=float(feller[i]),
                                     **{k: opts[i][k] for k in ("nx", "ny", "strike", "maturity", "v0", "kappa", "theta",
                                                                "sigma", "rho", "r")}) for i in worst]

    # The plain method, end to end on the two smaller buckets (every option priced), extrapolated on the largest.
    plain = {}
    measured_idx = []
    plain_ms_measured = 0.0
    for nx, ny in HESTON_BUCKETS:
        key = f"{nx}x{ny}"
        idx = buckets[key]
        group = [opts[i] for i in idx]
        if (nx, ny) != HESTON_BUCKETS[-1]:
            pms, subs, pp = plain_heston_bucket(group, nx, ny, stream_sync)
            row = {"options": len(idx), "substeps": subs, "ms": pms, "measured": True}
            if cf is not None:
                pe = np.abs(pp - cf[idx])
                ae = np.abs(prices[idx] - cf[idx])
                row["plain_error_vs_cf"] = err_stats(pe)
                row["adi_error_vs_cf"] = err_stats(ae)
                row["adi_within_plain_error_1e_3"] = float(np.mean(ae <= pe + 1e-3))
                row["max_abs_adi_minus_plain"] = float(np.abs(prices[idx] - pp).max())
            plain_ms_measured += pms
            measured_idx += idx
        else:
            # 128 of its options over 2000 substeps, scaled by options and by the substeps its longest option needs.
            sample = group[:128]
            limit = min(0.25 * (6.0 / nx) ** 2 / (o["maturity"] * o["sigma"] * ny * (6.0 / nx)) for o in group)
            subs = int(np.ceil(1.0 / limit))
            pms, psub, _ = plain_heston_bucket_sample(sample, nx, ny, stream_sync, 2000)
            row = {"options": len(idx), "substeps": subs, "ms": pms / psub * subs * len(group) / len(sample),
                   "measured": False, "extrapolated_from": f"{len(sample)} options x {psub} substeps in {pms:.1f} ms"}
        plain[key] = row
    plain_ms = sum(r["ms"] for r in plain.values())
    out["plain"] = {"method": "explicit Euler law (tests/laws/heston_explicit_T.law) through fe_law_step, same grids",
                    "ms": plain_ms, "options_per_s": n / (plain_ms * 1e-3), "buckets": plain}
    out["speedup_vs_plain"] = plain_ms / ms
    # A fully measured ratio: the ADI batch of just the measured buckets' options against their plain runs.
    with HestonBatch([opts[i] for i in measured_idx], steps, DOUGLAS) as b2:
        b2.autotune()
        b2.run(use_graph=True)
        ms2 = statistics.median([b2.time(use_graph=True) for _ in range(3)])
    out["measured_buckets"] = {"options": len(measured_idx), "adi_ms": ms2, "plain_ms": plain_ms_measured,
                               "speedup": plain_ms_measured / ms2}
    cpu = cpu_reference_heston(256, 128, [opts[i] for i in buckets["256x128"][:16]], 4)
    if cpu is not None:
        ms_step, cores = cpu
        per_option = ms_step / 16 * steps
        out["cpu_baseline"] = {"value": 1e3 / per_option, "unit": "options/s", "cores": cores, "kind": "reference",
                               "sample": "the reference's lawc on tests/laws/heston_douglas.law, 16 options of the 256 x 128 "
                                         f"bucket as z-planes, 4 timed steps after 1 warm-up ({ms_step:.1f} ms a step), "
                                         f"scaled to {steps} steps an option"}
    return out


def plain_heston_bucket_sample(group, nx, ny, stream_sync, substeps):
    """Device time of `substeps` explicit substeps (heston_explicit_T.law) on these options as the planes of one lattice."""
    import numpy as np
    import torch
    from fieldcuda.heston import lattice_fields
    from fieldcuda.solver import Solver
    fields, h = lattice_fields(group, nx, ny)
    fields["mat"] = np.broadcast_to(np.array([o["maturity"] for o in group], np.float32)[:, None, None],
                                    fields["V"].shape).copy()
    s = Solver(open(HESTON_EXPLICIT_T_LAW).read(), nx, ny, len(group), h, "heston_explicit_T.law")
    for k, v in fields.items():
        s.set_field(k, v)
    limit = min(0.25 * h * h / (o["maturity"] * o["sigma"] * ny * h) for o in group)
    s.step(0.999 * limit * 8)  # warm-up: compile and a few substeps
    st = torch.cuda.ExternalStream(s.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    done = 0
    stream_sync()
    e0.record(st)
    while done < substeps:
        s.step(0.999 * limit * 1000)
        done += s.last_substeps()[0]
    e1.record(st)
    st.synchronize()
    ms = e0.elapsed_time(e1)
    s.close()
    return ms, done, None


def cpu_reference_heston(nx, ny, group, steps):
    """The reference's OpenMP solver (oracle/_ref/lawc) on tests/laws/heston_douglas.law with these options as z-planes:
    ms a step (after one warm-up step), all host cores; None without lawc."""
    lawc = os.path.join(ROOT, "oracle", "_ref", "lawc")
    if not os.path.exists(lawc):
        return None
    import numpy as np
    from fieldcuda.heston import lattice_fields
    threads = os.cpu_count() or 1
    fields, h = lattice_fields(group, nx, ny)
    work = tempfile.mkdtemp(prefix="fe_cpu_")
    try:
        scene = os.path.join(work, "s.scene")
        open(scene, "w").write(f"grid {nx} {ny} {len(group)} {h!r}\nlaw {HESTON_DOUGLAS_LAW}\n")
        init = os.path.join(work, "init")
        os.makedirs(init)
        for k, v in fields.items():
            np.ascontiguousarray(v, np.float32).tofile(os.path.join(init, k + ".bin"))
        out = os.path.join(work, "t.json")
        dt = min(o["maturity"] for o in group) / 512
        subprocess.run([lawc, "--scene", scene, "--init", init, "--steps", str(steps + 1), "--dt", repr(dt), "--json", out,
                        "--warmup", "1"], check=True, env=dict(os.environ, OMP_NUM_THREADS=str(threads)),
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        return json.load(open(out))["mean_ms"], threads
    finally:
        shutil.rmtree(work, ignore_errors=True)


def multifield_section(n, steps, warmup, stream_sync):
    """The 43-term, 6-field generated law (tests/laws/multifield43.law) at n^3 through the law backend: median step
    time and effective bandwidth at its algorithmic bytes (every term reads and writes its fields once)."""
    import numpy as np
    import torch
    from fieldcuda.solver import Solver
    from fieldcuda.workloads import multifield_bytes_per_cell, multifield_law

    text, rw = multifield_law(0)
    h = 1.0 / n
    dt = 0.1 * h * h
    s = Solver(text, n, n, n, h, "multifield43.law")
    rng = np.random.default_rng(43)
    for i in range(6):
        s.set_field(f"f{i}", rng.uniform(-1, 1, (n, n, n)).astype(np.float32))
    s.set_deferred(True)
    for _ in range(warmup):
        s.step(dt)
    s.sync()
    st = torch.cuda.ExternalStream(s.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream_sync()
    e0.record(st)
    launches = 0
    for _ in range(steps):
        s.step(dt)
        launches += s.profile()["launches"]
    e1.record(st)
    st.synchronize()
    ms = e0.elapsed_time(e1) / steps
    s.sync()
    broken = s.violations()
    substeps = sum(s.last_substeps())
    s.close()
    bpc = multifield_bytes_per_cell(rw)
    return {"law": "43 terms, 6 fp32 fields (tests/laws/multifield43.law, seed 0)", "cells": n ** 3, "dt": dt,
            "ms_per_step": ms, "term_passes_per_step": substeps, "launches_per_step": launches / steps,
            "algorithmic_bytes_per_cell_step": bpc, "effective_gbs": bpc * n ** 3 / (ms * 1e-3) / 1e9,
            "violations": len(broken)}


def nets_section(stream_sync):
    """The net ops (tests/laws/nets_mlp.law, nets_flux.law, nets_ldiffuse.law) on 128 x 128 x 64 cells, random state:
    median step time with fp32 nets (per cell on the CUDA cores) and with the nets declared half (tcgen05 stage
    kernels, BF16 operands, FP32 accumulation), and the half step's worst difference from the fp32 one as a fraction of
    what the step moved (the reference's gate for its tensor-core nets: 0.03)."""
    import numpy as np
    import torch
    from fieldcuda.solver import Solver
    here = os.getcwd()
    os.chdir(ROOT)  # the laws' weight files are repository paths
    out = {}
    try:
        n, nz, dt = 128, 64, 0.02
        for law in ("nets_mlp.law", "nets_flux.law", "nets_ldiffuse.law"):
            text = open(os.path.join("tests", "laws", law)).read()
            row, after = {}, {}
            for form, t in (("fp32", text), ("half", text.replace(" file ", " half file "))):
                rng = np.random.default_rng(5)
                T0 = (290 + 600 * rng.random((nz, n, n))).astype(np.float32)
                s = Solver(t, n, n, nz, 0.5, law)
                s.set_field("T", T0)
                if "fuel" in s.field_names:
                    s.set_field("fuel", rng.random((nz, n, n)).astype(np.float32))
                s.step(dt)
                after[form] = s.values("T").astype(np.float64)
                s.set_deferred(True)
                for _ in range(3):
                    s.step(dt)
                st = torch.cuda.ExternalStream(s.stream)
                times = []
                for _ in range(10):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    stream_sync()
                    e0.record(st)
                    s.step(dt)
                    e1.record(st)
                    st.synchronize()
                    times.append(e0.elapsed_time(e1))
                s.sync()
                row[form + "_ms_per_step"] = statistics.median(times)
                row[form + "_violations"] = len(s.violations())
                s.close()
                if form == "fp32":
                    moved = float(np.abs(after["fp32"] - T0).max())
            row["speedup"] = row["fp32_ms_per_step"] / row["half_ms_per_step"]
            row["half_worst_over_moved"] = float(np.abs(after["half"] - after["fp32"]).max()) / max(moved, 1e-30)
            out[law] = row
    finally:
        os.chdir(here)
    return {"cells": n * n * nz, "dt": dt, "laws": out}


HESTON_CALIB = os.path.join(ROOT, "tests", "golden", "heston", "calib_512.npz")


def tridiag_section():
    """The law's tridiagonal solves timed alone (fe_law_time_stage): tests/laws/heston_douglas.law on the calibration's
    lattice (256 x 128 x 512 planes, one option a plane): its stages in launch order (the stored explicit rate, the
    x solve by the partition method, the y solve a thread a line), each launched 10 times back to back. Cells solved a
    second, and the effective bandwidth at 8 B a cell (the right-hand side read, the answer written; the coefficients
    are formed from static fields in the same kernel and read on top of that)."""
    import numpy as np
    from fieldcuda.heston import lattice_fields, sample_options
    from fieldcuda.solver import Solver
    nx, ny, nz = 256, 128, 512
    fields, h = lattice_fields(sample_options(nz, 9, sizes=((nx, ny),)), nx, ny)
    s = Solver(open(HESTON_DOUGLAS_LAW).read(), nx, ny, nz, h, "heston_douglas.law")
    for k, v in fields.items():
        s.set_field(k, v)
    s.step(1.0 / 512)
    out = {"lattice": f"{nx} x {ny} x {nz}", "stages": []}
    cells = nx * ny * nz
    for stage in range(16):
        try:
            name, ms = s.time_stage(0, stage, 10, 1.0 / 512)
        except Exception:
            break
        per = ms / 10
        out["stages"].append({"kernel": name, "ms": per, "cells_per_s": cells / (per * 1e-3),
                              "gbs_at_8_bytes_a_cell": 8 * cells / (per * 1e-3) / 1e9})
    s.close()
    return out


def calibration_section():
    """The adjoint calibration: loss = sum (price - target)^2 over 512 options (one maturity, strikes U[80, 120]) on one
    256 x 128 lattice (the options as its z-planes), 512 Douglas ADI steps, and its gradient with respect to (kappa,
    theta, sigma, rho, v0) by the IR-generated adjoint law with sqrt(N) checkpoints behind torch.autograd; checked
    against central differences (eps = 1e-3 relative) of the same FP32 loss. Targets: FP64 characteristic-function
    prices under a seeded ground truth plus N(0, 1e-4) noise (tests/golden/heston/calib_512.npz)."""
    import numpy as np
    from fieldcuda.heston import Calibration, calibration_options

    z = np.load(HESTON_CALIB)
    strikes, common, truth = calibration_options(512, int(z["seed"]))
    nx, ny, steps = 256, 128, 512
    cal = Calibration(open(HESTON_DOUGLAS_LAW).read(), strikes, common["maturity"], common["spot"], common["r"],
                      z["targets"], nx, ny, steps)
    x = np.array([truth["kappa"] * 1.3, truth["theta"] * 0.8, truth["sigma"] * 1.1, truth["rho"] * 0.9, truth["v0"] * 1.2])
    cal.loss_and_grad(x)
    t0 = time.perf_counter()
    loss, grad = cal.loss_and_grad(x)
    ms_grad = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    cal.loss_only(x)
    ms_fwd = (time.perf_counter() - t0) * 1e3
    fd = []
    for i in range(5):
        e = 1e-3 * abs(x[i])
        xp, xm = x.copy(), x.copy()
        xp[i] += e
        xm[i] -= e
        fd.append((cal.loss_only(xp) - cal.loss_only(xm)) / (2 * e))
    cal.close()
    fd = np.array(fd)
    out_cpu = None
    # The reference cannot differentiate through its tridiagonal solves: its way to this gradient is central
    # differences of its CPU forward (10 losses). Timed on a sample (64 of the 512 options, 4 Douglas steps) and
    # scaled to the whole calibration lattice, its 512 steps and the 11 losses (the base and 10 perturbed).
    from fieldcuda.heston import lattice_fields
    sample = [dict(nx=nx, ny=ny, strike=float(k), maturity=common["maturity"], spot=common["spot"], v0=truth["v0"],
                   kappa=truth["kappa"], theta=truth["theta"], sigma=truth["sigma"], rho=truth["rho"], r=common["r"])
              for k in strikes[:64]]
    fields, h = lattice_fields(sample, nx, ny)
    res = cpu_reference_run(HESTON_DOUGLAS_LAW, (nx, ny, 64, h), common["maturity"] / steps, 4, fields)
    if res is not None:
        ms_step, cores = res
        est_ms = ms_step * (512 / 64) * steps * 11
        out_cpu = {"value": 1e3 / est_ms, "unit": "gradients/s", "cores": cores, "kind": "reference",
                   "sample": f"the reference's lawc on tests/laws/heston_douglas.law, 64 of the options as z-planes of "
                             f"{nx} x {ny}, 4 timed steps after 1 warm-up ({ms_step:.1f} ms a step), scaled to 512 options, "
                             f"{steps} steps and 11 losses (central differences of the 5 parameters)",
                   "estimated_ms_a_gradient": est_ms}
    return {"options": 512, "lattice": f"{nx} x {ny} x 512 planes", "steps": steps,
            "gradients_per_s": 1e3 / ms_grad, "cpu_baseline": out_cpu,
            "speedup_vs_cpu": (out_cpu["estimated_ms_a_gradient"] / ms_grad) if out_cpu else None,
            "checkpoints": int(np.ceil(np.sqrt(steps))), "loss": loss,
            "gradient": dict(zip(Calibration.NAMES, map(float, grad))), "central_fd": dict(zip(Calibration.NAMES, map(float, fd))),
            "fd_rel_err": dict(zip(Calibration.NAMES, map(float, np.abs(grad - fd) / np.maximum(np.abs(fd), 1e-12)))),
            "ms_loss_and_gradient": ms_grad, "ms_loss": ms_fwd,
            "what": "wall clock of one loss + gradient (forward, checkpointed recompute, adjoint law backward)"}


FHN_LAW = os.path.join(ROOT, "tests", "laws", "fhn_rk4.law")
FHN_TRUTH = os.path.join(ROOT, "tests", "golden", "fhn", "truth.npz")


def fhn_learned_section(samples=1000, frames=100, train_samples=64, iters=3000):
    """FitzHugh-Nagumo (u, v) on [-1, 1]^2, t in [0, 5] in 100 frames of 0.05, N(0, 1) starts per cell (seeded), as
    z-planes of one lattice: the learned form (32 x 32 plain law + the tensor-core correction after every frame,
    trained here on the engine's own 128 x 128 solves of 64 other seeds) against the plain law at 32, 64 and 128.
    Errors (RMSE of (u, v) averaged onto 32 x 32, every 10th frame) against the plain 128 x 128 solve (the judge) and,
    for the first 4 seeds, against an FP64 method-of-lines solve (tests/golden/fhn/truth.npz). solves/s = samples over
    the device time of the 100 frames."""
    import numpy as np
    import torch
    import torch.nn.functional as F
    from fieldcuda.learned import Corrector, PlainFHN, block_mean, fhn_initial, fine_frames, init_weights, train_correction

    text = open(FHN_LAW).read()

    def pool(x, f):
        return F.avg_pool2d(x[:, None], f)[:, 0].contiguous() if f > 1 else x

    t0 = time.perf_counter()
    targets = fine_frames(text, list(range(train_samples)), frames)
    torch.cuda.synchronize()
    data_s = time.perf_counter() - t0
    corr = Corrector(init_weights(7))
    t0 = time.perf_counter()
    train_rmse, train_plain_rmse = train_correction(corr, text, targets, iters=iters, rounds=2)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    seeds = list(range(1000, 1000 + samples))
    su, sv = fhn_initial(seeds, 128)
    keep = list(range(10, frames + 1, 10))

    def run(n, learned, snapshots):
        s = PlainFHN(text, n, samples)
        f = 128 // n
        s.set(block_mean(su, f) if f > 1 else su, block_mean(sv, f) if f > 1 else sv)
        st = torch.cuda.ExternalStream(s.solver.stream)
        snaps = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        for t in range(1, frames + 1):
            s.step()
            if learned:
                corr.apply_solver(s.solver, time=t * s.frame)
            if snapshots and t in keep:
                u, v = s.get()
                snaps.append((pool(u, n // 32), pool(v, n // 32)))
        e1.record(st)
        st.synchronize()
        ms = e0.elapsed_time(e1)
        subs = s.substeps()
        s.solver.sync()
        broken = len(s.solver.violations())
        s.close()
        return ms, snaps, subs, broken

    methods = {"plain_32": (32, False), "plain_64": (64, False), "plain_128": (128, False), "learned_32": (32, True)}
    out = {}
    snaps = {}
    for name, (n, learned) in methods.items():
        run(n, learned, False)
        ms, _, subs, broken = run(n, learned, False)
        _, snaps[name], _, _ = run(n, learned, True)
        out[name] = {"lattice": f"{n} x {n} x {samples}", "substeps_per_frame": subs, "ms": ms,
                     "solves_per_s": samples / (ms * 1e-3), "violations": broken}
    judge = snaps["plain_128"]
    truth = np.load(FHN_TRUTH)["states"] if os.path.exists(FHN_TRUTH) else None
    for name in methods:
        err = [float(((a - ja) ** 2 + (b - jb) ** 2).mean() / 2) for (a, b), (ja, jb) in zip(snaps[name], judge)]
        out[name]["rmse_vs_plain_128"] = float(np.sqrt(np.mean(err)))
        if truth is not None:
            e64 = []
            for k, (a, b) in enumerate(snaps[name]):
                ref = truth[k + 1]
                e64.append(float((((a[:4].cpu().numpy() - ref[0]) ** 2 + (b[:4].cpu().numpy() - ref[1]) ** 2) / 2).mean()))
            out[name]["rmse_vs_fp64_4_seeds"] = float(np.sqrt(np.mean(e64)))
    corr.close()
    # The reference's own OpenMP solver on the plain 128 x 128 law (the judge), 16 samples as z-planes over 2 frames,
    # scaled to solves (100 frames) a second.
    cu, cv = fhn_initial(list(range(2000, 2016)), 128)
    res = cpu_reference_run(FHN_LAW, (128, 128, 16, 2.0 / 128), 0.05, 2, {"u": cu, "v": cv})
    cpu = None
    if res is not None:
        ms_frame, cores = res
        cpu = {"value": 16 / (ms_frame * frames * 1e-3), "unit": "solves/s", "cores": cores, "kind": "reference",
               "sample": f"the reference's lawc on tests/laws/fhn_rk4.law, 128 x 128 x 16 samples, 2 timed frames of 0.05 "
                         f"after 1 warm-up ({ms_frame:.1f} ms a frame), scaled to {frames} frames a solve"}
    learned_err = out["learned_32"]["rmse_vs_plain_128"]
    matches = [m for m in ("plain_32", "plain_64", "plain_128") if out[m]["rmse_vs_plain_128"] <= learned_err]
    equal = matches[0] if matches else None
    return {"samples": samples, "frames": frames, "methods": out, "cpu_baseline": cpu,
            "speedup_learned_vs_cpu_plain_128": (out["learned_32"]["solves_per_s"] / cpu["value"]) if cpu else None,
            "training": {"seeds": train_samples, "pairs": frames, "adam_steps": iters * 3, "rounds": "teacher forcing, then 2 rounds on "
                         "the learned solver's own rollouts", "seconds": train_s, "data_seconds": data_s,
                         "rollout_rmse_train": train_rmse, "plain_rollout_rmse_train": train_plain_rmse},
            "equal_error_plain": equal,
            "speedup_at_equal_error": (out["learned_32"]["solves_per_s"] / out[equal]["solves_per_s"]) if equal else None,
            "network": "3x3 conv of (u, v) and the time 2->64, ReLU, 64->64, ReLU, 64->2, BF16 tcgen05, FP32 accumulators "
                       "(10,752 FLOP a cell)"}


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    from fieldcuda import _lib
    from fieldcuda.solver import Solver
    from oracle import heat as oh

    torch.cuda.set_device(local)
    _lib.check(_lib.lib().fe_device_check())
    n = args.size
    h = 1.0 / n
    dt = 0.4 * h * h / 6.0
    cells = n ** 3
    K, W = args.steps, args.warmup
    T0 = oh.gaussian_blobs(n, h, seed=rank)
    pinned_in = torch.from_numpy(T0).pin_memory()
    pinned_out = torch.empty((n, n, n), dtype=torch.float32).pin_memory()

    # The product path: the law compiled by the backend (IR -> sm_100a kernels), stepped through the C ABI. On N GPUs
    # the lattice is n x n x (N n), one z-slab of n planes a rank, halo planes exchanged over NCCL after every step
    # and conservation judged over the ranks (fieldcuda/slabs.py).
    if world > 1:
        from fieldcuda.slabs import DistComm, SlabLaw
        slab = SlabLaw(HEAT_LAW, n, n, n * world, h, rank, world, DistComm(), source_name="heat.law")
        s = slab.solver
        stepper = slab
    else:
        slab = None
        s = Solver(HEAT_LAW, n, n, n, h, "heat.law")
        stepper = s
    local_cells = n * n * s.shape[0]

    def judge():
        if slab is not None:
            return slab.sync()
        s.sync()
        return s.violations()

    def upload():
        if slab is not None:
            slab.set_field("T", pinned_in.numpy())
        else:
            s.set_field("T", pinned_in.numpy())

    upload()
    stream = torch.cuda.ExternalStream(s.stream)
    s.set_deferred(True)  # contracts checked every step, judged after the run: no step waits for the host
    for _ in range(W):
        stepper.step(dt)
    broken = judge()
    assert not broken, broken

    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = _events(stream)
    e0.record(stream)
    launches = 0
    for _ in range(K):
        stepper.step(dt)
        launches += s.profile()["launches"]
    e1.record(stream)
    stream.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms_total = max_over_ranks(world, e0.elapsed_time(e1))
    broken = judge()  # judge every timed step's contracts (conserved total, range, NaN)
    assert not broken, broken

    # The dominant kernel alone: the generated gather pass (one launch a step), timed back to back.
    gather_ms = max_over_ranks(world, s.time_gather(0, 20) / 20)

    # End to end through the public API with host buffers: the state up from pinned host memory, K steps each judged
    # on the host (its contract records read back), the state back down to pinned host memory.
    s.set_deferred(slab is not None)  # one GPU: each step judged on the host; slabs: judged over the ranks at the end
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    upload()
    for _ in range(K):
        stepper.step(dt)
    if slab is not None:
        pinned_out.numpy()[:] = slab.values("T")
    else:
        _lib.check(_lib.lib().fe_law_fetch(s._h, 0, ctypes.c_void_p(pinned_out.data_ptr())))
    broken = judge()
    e2e_ms = max_over_ranks(world, (time.perf_counter() - t0) * 1e3)
    assert not broken, broken

    # Bit-identical across runs: the same start stepped twice gives the same FNV-1a digest of the state.
    digests = []
    for _ in range(2):
        upload()
        for _ in range(10):
            stepper.step(dt)
        judge()
        digests.append(s.digest())
    deterministic = digests[0] == digests[1]
    s.close()

    side = torch.cuda.Stream()
    hand_ms = handwritten_ms(n, h, dt, cells, side)
    copy_gbs = copy_roof_gbs(cells, side)

    ms_step = ms_total / K
    total_cells = cells * world
    value = BYTES_PER_CELL * total_cells * K / (ms_total * 1e-3) / 1e9
    e2e_value = BYTES_PER_CELL * total_cells * K / (e2e_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    achieved = BYTES_PER_CELL * local_cells / (gather_ms * 1e-3) / 1e9
    traffic = profile_traffic("heat_gather_512.md")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        res = cpu_reference_heat(n, 2, 1, threads)
        if res is not None:
            ms, kind, cores = res
            cpu = {"value": BYTES_PER_CELL * cells / (ms * 1e-3) / 1e9, "unit": "GB/s", "cores": cores, "kind": kind,
                   "sample": f"2 timed steps of the {n}^3 heat law after 1 warm-up (the reference's lawc, its OpenMP solver)"}
        else:
            t = time.perf_counter()
            oh.cpu_step(T0, 1.0, h, dt)
            ms = (time.perf_counter() - t) * 1e3
            cpu = {"value": BYTES_PER_CELL * cells / (ms * 1e-3) / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
                   "sample": f"1 step of the {n}^3 heat law, numpy restatement (oracle/heat.py)"}

    c1 = c2 = None
    if world == 1 and not args.no_c1:
        c1 = c1_section(torch.cuda.synchronize, peak)
    if world == 1 and not args.no_c2:
        c2 = c2_section(torch.cuda.synchronize, peak, cpu=not args.no_cpu)
    heston = None
    if not args.no_heston:
        heston = heston_batch_section(torch.cuda.synchronize)
    multifield = None
    if not args.no_multifield:
        multifield = multifield_section(256, 10, 3, torch.cuda.synchronize)
    calibration = tridiag = None
    if not args.no_calibration:
        calibration = calibration_section()
        tridiag = tridiag_section()
    learned = None
    if not args.no_learned:
        learned = fhn_learned_section()
    nets = None
    if not args.no_nets:
        nets = nets_section(torch.cuda.synchronize)

    if rank != 0:
        return
    print(json.dumps({
        "metric": "7-pt stencil effective HBM GB/s (8 B/cell/step)",
        "value": value, "unit": "GB/s", "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: sum of 4 seeded Gaussian blobs (numpy default_rng(rank))",
        "config": {"workload": heat_workload(n), "cells_per_gpu": cells,
                   "path": "fe_law_step (law text -> IR -> generated sm_100a TMA pass)",
                   "l2": "inputs larger than L2 (512 MiB a buffer)",
                   "handwritten_kernel_gbs": BYTES_PER_CELL * cells / (hand_ms * 1e-3) / 1e9},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of the same pass at "
                     "512^3, copied from profiles/heat_gather_512.md (an ncu capture of the same pass; the traffic does "
                     "not depend on the tile or the chunk length beyond the z halo), not measured in this run",
                     "kernel": "generated gather pass fe_pass_t0g (8 B/cell)",
                     "peak_source": f"{peak_kind} copy (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                     "copy_same_run_gbs": copy_gbs},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "GB/s", "h2d_bytes_per_step": 4 * cells // K,
                "d2h_bytes_per_step": 64 + 4 + 4 * cells // K, "ms": e2e_ms,
                "what": "fe_law_upload of the state from pinned host memory, K fe_law_step each judged on the host, "
                        "fe_law_fetch of the state to pinned host memory (wall clock)"},
        "gpu_launches": launches,
        "clocks": clk,
        "deterministic": deterministic,
        "err_vs_fp64": (c1 or {}).get("rel_err_vs_fp64"),
        "err_vs_fp64_note": "C1 (128^3, 100 steps): max |T - T_fp64| / max |T_fp64| at the fixture's sampled cells, "
                            "T_fp64 the same scheme in double",
        "c1_128": c1,
        "c2_lazy": c2,
        "heston_batch": heston,
        "multifield_256": multifield,
        "adjoint_calibration": calibration,
        "tridiag_solves": tridiag,
        "fhn_learned": learned,
        "nets_half": nets,
    }))


def profile_case(name):
    """Small cases of the kernels the profiles under profiles/ summarise, for ncu (one GPU; a few launches):
    heat        the heat law on 512^3 (the bench's lattice; inputs larger than L2), 3 steps: the generated gather;
    heat256     the same law on 256^3 (two 64 MiB fields: still larger than L2 together), 3 steps: the gather's instruction
                mix (more metrics than the 512^3 case should carry);
    heston      36 options on 512 x 256, 16 Douglas steps, split (16, 4, 512): the cluster kernel;
    corrector   3 training steps, one gradient and one guarded apply on 256 x 32 x 32 cells: the tcgen05 kernels;
    multifield  the 43-term law on 128^3, 3 steps: its generated passes;
    calibration the adjoint calibration's lattice (512 options, 256 x 128) over 4 Douglas steps: one loss and gradient
                (the forward, the checkpointed recompute and the adjoint law's steps);
    tridiag     tests/laws/heston_douglas.law on 256 x 128 x 256 (256 options; 32 MiB a buffer, the law's buffers
                together larger than L2), 3 steps: the x solve by the partition method
                (fe_tri_* with fe_tridiag_x_warp) and the y solve;
    nets        the learned-flux and learned-conduction laws (tests/laws/nets_flux.law, nets_ldiffuse.law) on
                128 x 128 x 64, 3 steps each with fp32 nets, then with the nets declared half: the tcgen05 net stages."""
    import numpy as np
    import torch
    if name == "heston":
        from fieldcuda.heston import HestonBatch, sample_options
        with HestonBatch(sample_options(36, 1, sizes=((512, 256),)), 16, 0) as b:
            b.set_split(16, 4, 512)
            b.run()
            b.prices()
            print(json.dumps({"case": name, "ms": b.time(False), "layout": b.layout()}))
    elif name == "corrector":
        from fieldcuda.learned import Corrector, init_weights
        rng = np.random.default_rng(0)
        u, v, tu, tv = (torch.tensor(rng.normal(size=(256, 32, 32)).astype(np.float32), device="cuda") for _ in range(4))
        c = Corrector(init_weights(1))
        for _ in range(3):
            c.train_step(u, v, tu, tv, 1e-3)
        loss, _ = c.grads(u, v, tu, tv)
        c.apply(u, v)
        torch.cuda.synchronize()
        c.close()
        print(json.dumps({"case": name, "loss": loss}))
    elif name in ("heat", "heat256"):
        from fieldcuda.solver import Solver
        from oracle import heat as oh
        n = 512 if name == "heat" else 256
        h = 1.0 / n
        s = Solver(HEAT_LAW, n, n, n, h, "heat.law")
        s.set_field("T", oh.gaussian_blobs(n, h, seed=0))
        for _ in range(3):
            s.step(0.4 * h * h / 6.0)
        s.sync()
        print(json.dumps({"case": name, "violations": len(s.violations())}))
        s.close()
    elif name == "multifield":
        from fieldcuda.solver import Solver
        from fieldcuda.workloads import multifield_law
        text, _ = multifield_law(0)
        n = 128
        s = Solver(text, n, n, n, 1.0 / n, "multifield43.law")
        rng = np.random.default_rng(43)
        for i in range(6):
            s.set_field(f"f{i}", rng.uniform(-1, 1, (n, n, n)).astype(np.float32))
        for _ in range(3):
            s.step(0.1 / (n * n))
        s.sync()
        print(json.dumps({"case": name, "violations": len(s.violations())}))
        s.close()
    elif name == "calibration":
        from fieldcuda.heston import Calibration, calibration_options
        z = np.load(HESTON_CALIB)
        strikes, common, truth = calibration_options(512, int(z["seed"]))
        cal = Calibration(open(HESTON_DOUGLAS_LAW).read(), strikes, common["maturity"], common["spot"], common["r"], z["targets"],
                          256, 128, 4)
        x = [truth["kappa"] * 1.2, truth["theta"] * 0.9, truth["sigma"] * 1.1, truth["rho"] * 0.9, truth["v0"] * 1.1]
        loss, grad = cal.loss_and_grad(x)
        torch.cuda.synchronize()
        cal.close()
        print(json.dumps({"case": name, "loss": loss, "grad": [float(g) for g in grad]}))
    elif name == "tridiag":
        from fieldcuda.heston import lattice_fields, sample_options
        from fieldcuda.solver import Solver
        nx, ny, nz = 256, 128, 256
        fields, h = lattice_fields(sample_options(nz, 9, sizes=((nx, ny),)), nx, ny)
        s = Solver(open(HESTON_DOUGLAS_LAW).read(), nx, ny, nz, h, "heston_douglas.law")
        for k, v in fields.items():
            s.set_field(k, v)
        for _ in range(3):
            s.step(1.0 / 512)
        s.sync()
        print(json.dumps({"case": name, "violations": len(s.violations())}))
        s.close()
    elif name == "nets":
        from fieldcuda.solver import Solver
        os.chdir(ROOT)  # the laws' weight files are repository paths
        rng = np.random.default_rng(5)
        n, nz = 128, 64
        out = {}
        for law in ("nets_flux.law", "nets_ldiffuse.law"):
            text = open(os.path.join("tests", "laws", law)).read()
            for form, t in (("fp32", text), ("half", text.replace(" file ", " half file "))):
                s = Solver(t, n, n, nz, 0.5, law)
                s.set_field("T", (290 + 600 * rng.random((nz, n, n))).astype(np.float32))
                if "fuel" in s.field_names:
                    s.set_field("fuel", rng.random((nz, n, n)).astype(np.float32))
                for _ in range(3):
                    s.step(0.02)
                s.sync()
                out[f"{law}:{form}"] = len(s.violations())
                s.close()
        print(json.dumps({"case": name, "violations": out}))
    else:
        raise SystemExit(f"no profile case {name!r}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-c1", action="store_true", help="skip the 128^3 x 100-step heat section")
    ap.add_argument("--no-c2", action="store_true", help="skip the 256^3 / 512^3 lazy-readback section")
    ap.add_argument("--no-heston", action="store_true", help="skip the batched Heston ADI section")
    ap.add_argument("--no-multifield", action="store_true", help="skip the 43-term multi-field law section")
    ap.add_argument("--no-nets", action="store_true", help="skip the net ops section (fp32 and tensor-core nets)")
    ap.add_argument("--no-calibration", action="store_true", help="skip the adjoint calibration section")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-correction section")
    ap.add_argument("--profile-case", default="", help="run one small case for ncu (heat, heat256, heston, corrector, multifield, calibration, tridiag, nets) and exit")
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args.profile_case)
        return
    world, rank, local = init_dist()
    try:
        if args.impl == "reference":
            run_reference_arm(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
