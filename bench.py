"""Benchmark: derived tuples/s per fixpoint of the B200 Datalog engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config tc_chung_lu_317k|tc_dag_5k|sg_lattice_55]

Default workload (one step = one whole TC fixpoint, init through the last
iteration): transitive closure of a seeded Chung-Lu power-law graph with 317K
nodes, exponent 2.5 and 1.05M edges stored once (~1.9e9 closure tuples), the
com-dblp-scale configuration of the reference's TC results. `value` is
closure tuples per second with the edge relation already in HBM; `e2e` is the
same metric through the public API with host buffers (pinned H2D of the edges,
the fixpoint, D2H of every closure row). Under torchrun every rank runs its own
independent replica (the path is one fixpoint per GPU; no collective on the
data path); timing is on the device (CUDA events) and the max over ranks.

--impl reference times the reference's own CPU program (rough/tc_mpi.cpp, built
unmodified by oracle/Makefile into oracle/_ref/tc_mpi_fork: one MPI rank per
host core over a fork + shared-memory MPI) on a bounded sample of the same
graph family, rank 0 only.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "derived tuples/s per fixpoint"
UNIT = "tuples/s"
L2_FLUSH_BYTES = 256 << 20
CPU_SAMPLE_NODES = 24000     # cpu_baseline sample (~10-20 s over 8-16 cores)
REF_SAMPLE_NODES = 12000     # reference arm sample per step (a few seconds over 16 cores)
HBM_FALLBACK_GBS = 6650.0
TUNING_BATCH = os.path.join(ROOT, "mnmgdatalog_b200", "tuning_batch.json")
SERVE_BUDGET = 150 * 10**9   # HBM budget of the served leg's admission


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def workload(config: str):
    if config == "sg_fe_body":  # the reference's fe_body input (data/data_163734.bin)
        return "sg", load_fixture(SG_DATASET[0])
    from mnmgdatalog_b200 import graphs
    prog, edges = graphs.make(config, seed=0)
    return prog, edges


def describe(config: str, edges: np.ndarray) -> dict:
    d = {"tc_chung_lu_317k": "TC, Chung-Lu n=317000 gamma=2.5 m=1050000 (each edge once, seed 0)",
         "tc_dag_5k": "TC, DAG n=5000 p=0.7 + 2000 short edges (seed 0)",
         "sg_lattice_55": "SG, 55^3 lattice 6-neighbour p=0.15 + 1% long edges (seed 0)",
         "tc_chung_lu_40k": "TC, Chung-Lu n=40000 gamma=2.5 m=132500 (each edge once, seed 0)",
         "tc_chung_lu_80k": "TC, Chung-Lu n=80000 gamma=2.5 m=265000 (each edge once, seed 0)",
         "sg_fe_body": "SG, the reference's fe_body input (data/data_163734.bin, 163,734 edges)"}
    return {"workload": d.get(config, config), "config": config, "input_rows": int(len(edges))}


def measured_peak_gbs() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region.

    nvidia-smi is started before the warm-up (its start-up queries the driver
    for a while, which is kept out of the timed steps); mark() and stop()
    bracket the timed region, and only samples taken in between count (the
    nearest later one if none landed inside)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[tuple[float, str]] = []
        self.t_mark = None

    def start(self):
        exe = shutil.which("nvidia-smi")
        if not exe:
            return
        self.proc = subprocess.Popen([exe, f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def mark(self):
        """The timed region starts."""
        self.t_mark = time.monotonic()

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t_end = time.monotonic()
        # at least one sample from the timed region or just after it
        deadline = t_end + 2.0
        while time.monotonic() < deadline and not any(t >= (self.t_mark or 0) for t, _ in self.lines):
            time.sleep(0.05)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        t0 = self.t_mark or 0.0
        inside = [ln for t, ln in self.lines if t0 <= t <= t_end]
        if not inside:
            inside = [ln for t, ln in self.lines if t >= t0][:1]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in inside:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def run_tc_mpi_sample(nodes: int, seed: int = 0) -> dict:
    """Time the reference CPU program on a Chung-Lu sample of `nodes` nodes,
    as one MPI rank per host core (oracle/_ref/tc_mpi_fork: the unmodified
    rough/tc_mpi.cpp over the fork + shared-memory MPI of oracle/mpi_fork),
    else as one rank (oracle/_ref/tc_mpi), else the oracle's restatement."""
    from mnmgdatalog_b200 import graphs
    e = graphs.chung_lu(n=nodes, m=int(round(nodes * 1_050_000 / 317_000)), seed=seed)
    forked = os.path.join(ROOT, "oracle", "_ref", "tc_mpi_fork")
    single = os.path.join(ROOT, "oracle", "_ref", "tc_mpi")
    binary, ranks = (forked, os.cpu_count() or 1) if os.path.exists(forked) else (single, 1)
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "sample.bin")
        e.astype("<i4").tofile(inp)
        if os.path.exists(binary):
            t0 = time.perf_counter()
            r = subprocess.run([binary, inp], capture_output=True, text=True, timeout=600, check=True,
                               env=dict(os.environ, MPI_FORK_RANKS=str(ranks)))
            wall = time.perf_counter() - t0
            row = [l for l in r.stdout.splitlines() if l.startswith("|") and l[2:3].isdigit()][-1]
            cells = [c.strip().replace(",", "").replace("'", "") for c in row.strip("|").split("|")]
            tuples, secs = int(cells[3]), float(cells[4])
            kind = "reference"
        else:  # the oracle's C restatement (same algorithm as the reference GPU path)
            from oracle import cpu
            t0 = time.perf_counter()
            res = cpu.tc(e)
            secs = wall = time.perf_counter() - t0
            tuples = len(res.rows)
            kind, ranks = "port", 1
    return {"value": tuples / secs, "unit": UNIT, "cores": ranks, "kind": kind,
            "sample": f"TC of Chung-Lu n={nodes} m={len(e)} gamma=2.5 (same generator, seed {seed}): "
                      f"{tuples} tuples in {secs:.2f} s (wall {wall:.2f} s), {ranks} MPI rank(s) of "
                      f"rough/tc_mpi.cpp, one per host core",
            "tuples": tuples, "seconds": secs}


def run_reference_gpu(prog: str, edges: np.ndarray, timeout: int = 600) -> dict:
    """Context figure: the reference's own GPU program (tc.cu / sg.cu built
    unmodified by oracle/Makefile into oracle/_ref/, one MPI rank) on the same
    input on this GPU, job_run=1 (no output file). Its "Total Time" column
    excludes file I/O (tc.cu:387-389); the engine's `value` covers the same
    span (input upload through the unpacked result rows)."""
    binary = os.path.join(ROOT, "oracle", "_ref", f"{prog}.out")
    if not os.path.exists(binary):
        return {"unavailable": f"oracle/_ref/{prog}.out not built"}
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "input.bin")
        edges.astype("<i4").tofile(inp)
        t0 = time.perf_counter()
        r = subprocess.run([binary, inp, "0", "0", "1"], capture_output=True, text=True, timeout=timeout, cwd=td)
        wall = time.perf_counter() - t0
    if r.returncode != 0:
        return {"error": f"exit {r.returncode}: {r.stderr[-300:]}"}
    csv = [l for l in r.stdout.splitlines() if l and l[0].isdigit()][-1].split(",")
    total = float(csv[4])
    return {"program": f"oracle/_ref/{prog}.out <input> 0 0 1 (reference {prog}.cu, unmodified, one MPI rank)",
            "iterations": int(csv[2]), "tuples": int(csv[3]), "total_s": total,
            "tuples_per_s": int(csv[3]) / total if total > 0 else None, "wall_s": round(wall, 2),
            "note": "context only; the reference arm of this benchmark is the CPU program"}


def main_reference(args, rank: int, world: int) -> int:
    if rank != 0:
        return 0
    for _ in range(args.warmup):
        run_tc_mpi_sample(REF_SAMPLE_NODES)
    vals, secs = [], []
    for _ in range(args.steps):
        r = run_tc_mpi_sample(REF_SAMPLE_NODES)
        vals.append(r["value"])
        secs.append(r["seconds"])
    total_tuples = r["tuples"] * args.steps
    value = total_tuples / sum(secs)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": r["sample"], "config": args.config, "l2": "host CPU run"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def timed_fixpoints(eng, prog, d_edges, steps, warmup, dedup, dev, world, barrier, flush, clocks=None):
    """`warmup` untimed and `steps` timed whole fixpoints of one program on
    edges already in HBM; each step ends with the result rows in the
    reference's file order in device memory (the rank -> id unpack the
    reference times as finalization, tc.cu:319-327; the destination is
    allocated once). L2 is flushed between steps, outside the events.
    Returns (per-step ms on this rank, last result, live profile)."""
    import torch
    first = eng.run(prog, d_edges, output="none", dedup=dedup)
    out_rows = torch.empty((max(first.output_tuples, 1), 2), dtype=torch.int32, device=dev)
    del first

    def step():
        return eng.run(prog, d_edges, output="device", out=out_rows, dedup=dedup)

    if clocks:
        clocks.start()  # before the warm-up: nvidia-smi's start-up stays out of the timed steps
    for _ in range(warmup):
        step()
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)
    if clocks:
        clocks.mark()
    eng.profile(True)
    stream = eng._stream_obj
    evs = []
    r = None
    # Python's cyclic garbage collector stays off while steps are timed: a
    # full collection between two of a step's library calls leaves the GPU
    # idle for tens of milliseconds inside the events
    gc.collect()
    gc.disable()
    try:
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)                      # L2 flush, outside the timed events
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
            r = step()
            with torch.cuda.stream(stream):
                b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize(dev)
    finally:
        gc.enable()
    barrier()
    torch.cuda.synchronize(dev)
    prof = eng.profile_read()
    eng.profile(False)
    ms = [a.elapsed_time(b) for a, b in evs]
    r.rows = None
    del out_rows
    return ms, r, prof


def roofline_of(prof: dict, step_s: float) -> tuple[dict, dict, dict, int]:
    """The dominant kernel class by device time: its algorithmic bytes per
    event-timed second against the measured HBM peak."""
    peak, peak_kind = measured_peak_gbs()
    host = {k: v for k, v in prof.items() if k.startswith("host_")}
    prof = {k: v for k, v in prof.items() if not k.startswith("host_")}
    dom_name, dom = max(((k, v) for k, v in prof.items() if v["timed_launches"]), key=lambda kv: kv[1]["seconds"])
    launches = sum(v["launches"] for v in prof.values())
    achieved = dom["bytes"] / dom["seconds"] / 1e9 if dom["seconds"] else 0.0
    roofline = {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": traffic_per_launch(dom_name, dom), "launches": dom["timed_launches"],
                "share_of_step": dom["seconds"] / step_s if step_s else None,
                "algorithmic_bytes_per_launch": dom["bytes"] / max(dom["timed_launches"], 1)}
    kernels = {k: {"launches": v["launches"], "ms": round(1e3 * v["seconds"], 3), "bytes": v["bytes"],
                   "GBps": round(v["bytes"] / v["seconds"] / 1e9, 1) if v["seconds"] else None,
                   "frac": round(v["bytes"] / v["seconds"] / 1e9 / peak, 4) if v["seconds"] else None}
               for k, v in prof.items() if v["launches"]}
    host_costs = {k: {"calls": v["launches"], "ms": round(1e3 * v["seconds"], 3)} for k, v in host.items()}
    return roofline, kernels, host_costs, launches


def release(eng, torch):
    """Hand a context's cached device memory back between legs, so that one
    leg's buffers neither crowd out nor speed up the next."""
    eng.release_memory()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def main_ours(args, rank: int, world: int, local_rank: int) -> int:
    import torch
    import torch.distributed as dist

    from mnmgdatalog_b200 import Engine

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    prog, edges = workload(args.config)

    # The reference's own GPU program on the same input, first, while the
    # device is empty (context figure, rank 0 of a one-GPU run only).
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu and prog in ("tc", "sg"):
        try:
            ref_gpu = run_reference_gpu(prog, edges)
        except Exception as exc:  # report, never hide
            ref_gpu = {"error": f"{type(exc).__name__}: {exc}"}

    stream = torch.cuda.Stream(device=dev)
    eng = Engine(local_rank, stream=stream)
    knobs = {k: (float(v) if "." in v else int(v)) for k, v in (t.split("=", 1) for t in args.tuning)}
    if knobs:
        eng.set_tuning(knobs)
    d_edges = torch.from_numpy(edges).to(dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    clocks = ClockSampler(local_rank)
    ms, r, prof = timed_fixpoints(eng, prog, d_edges, args.steps, args.warmup, args.dedup, dev, world, barrier,
                                  flush, clocks)
    clk = clocks.stop()
    my_ms = sum(ms)
    max_ms, total = combine_ranks(my_ms, float(r.output_tuples * args.steps), world, dev)
    value = total / (max_ms / 1e3)
    roofline, kernels, host_costs, launches = roofline_of(prof, my_ms / 1e3)
    release(eng, torch)

    e2e = None
    if not args.no_e2e:
        try:
            e2e = measure_e2e(eng, prog, edges, args, dev, world, barrier)
        except Exception as exc:  # reported in the line, never hidden
            e2e = {"value": None, "unit": UNIT, "error": f"{type(exc).__name__}: {exc}"}
        release(eng, torch)
    del d_edges

    sg = None
    if args.sg_leg and world == 1:
        try:
            sg = measure_sg_dataset(eng, args, dev, flush)
        except Exception as exc:  # reported in the line, never hidden
            sg = {"error": f"{type(exc).__name__}: {exc}"}
        release(eng, torch)

    sj = None
    if args.single_join_leg and world == 1:
        try:
            sj = measure_single_join(eng, args, dev, flush)
        except Exception as exc:  # reported in the line, never hidden
            sj = {"error": f"{type(exc).__name__}: {exc}"}
        release(eng, torch)

    batched = served = None
    if args.batch_instances > 0:
        try:
            with Engine(local_rank) as beng:
                batched = measure_batched(beng, dev, args)
        except Exception as exc:  # reported in the line, never hidden
            batched = {"error": f"{type(exc).__name__}: {exc}"}
        torch.cuda.empty_cache()
    if args.serve_requests > 0:
        try:
            tuned = batched.get("tuning") if isinstance(batched, dict) else None
            with Engine(local_rank) as seng:
                served = measure_served(seng, args, tuned)
        except Exception as exc:
            served = {"error": f"{type(exc).__name__}: {exc}"}
        torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = run_tc_mpi_sample(CPU_SAMPLE_NODES)
            cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as exc:  # report, never hide
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {exc}"}
        cpu["host_cores"] = os.cpu_count()

    if rank == 0:
        cfg = describe(args.config, edges)
        if knobs:
            cfg["tuning"] = knobs
        cfg.update({"parallelism": f"replicas x{world}", "l2": "256 MiB write between steps (outside timing)",
                    "output_tuples_per_step": int(r.output_tuples), "iterations": int(r.iterations),
                    "join_rows_per_step": int(r.join_rows_total), "join_rows_max_iteration": int(r.join_rows_max),
                    "step": "input edges in HBM -> fixpoint -> result rows (reference file order) in HBM"})
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
                "config": cfg, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches, "clocks": clk, "kernels": kernels, "host": host_costs,
                "step_ms": [round(x, 3) for x in ms], "reference_gpu": ref_gpu, "sg": sg, "single_join": sj,
                "batched": batched, "served": served}
        print(json.dumps(line))
    eng.close()
    return 0


SG_DATASET = ("data_163734.bin", "fe_body", 408_443_204, 125, "logs/small-merged-job-output.txt:212")


def load_fixture(name: str) -> np.ndarray:
    import gzip
    with gzip.open(os.path.join(ROOT, "tests", "golden", "data", name + ".gz"), "rb") as f:
        raw = f.read()
    return np.frombuffer(raw, dtype="<i4")[: (len(raw) // 8) * 2].reshape(-1, 2).copy()


SINGLE_JOIN = (10_000_001, 90_000, 1_037_050_773, "logs/single-join-small-job-output.txt:104-106")


def measure_single_join(eng, args, dev, flush) -> dict:
    """single_join's strong-scaling input on one GPU: 10,000,001 rows of
    glibc srand(1)/rand() values in [1, 90,000] (the reference published
    1,037,050,773 output rows for it on one A100), timed like the main leg,
    with the reference's own GPU program on the same rows."""
    import torch

    from mnmgdatalog_b200 import generate_rows
    rows, rng, pub, cite = SINGLE_JOIN
    data = generate_rows(rows, rng, 1)
    ref = None
    if not args.no_reference_gpu:
        binary = os.path.join(ROOT, "oracle", "_ref", "single_join.out")
        if os.path.exists(binary):
            t0 = time.perf_counter()
            r = subprocess.run([binary, str(rows), "0", "0", str(rng)], capture_output=True, text=True, timeout=600)
            wall = time.perf_counter() - t0
            if r.returncode == 0:
                csv = [l for l in r.stdout.splitlines() if l and l[0].isdigit()][-1].split(",")
                ref = {"program": f"oracle/_ref/single_join.out {rows} 0 0 {rng} (reference single_join.cu, "
                                  "unmodified, one MPI rank)", "tuples": int(csv[3]), "total_s": float(csv[4]),
                       "wall_s": round(wall, 2)}
            else:
                ref = {"error": f"exit {r.returncode}: {r.stderr[-300:]}"}
    d = torch.from_numpy(data).to(dev)
    steps = max(1, min(args.steps, 3))
    ms, res, prof = timed_fixpoints(eng, "single_join", d, steps, 1, "auto", dev, 1, lambda: None, flush)
    roofline, kernels, _, launches = roofline_of(prof, sum(ms) / 1e3)
    return {"workload": f"single_join, {rows} rows, values in [1, {rng}] (the reference's strong-scaling input; "
                        f"published {pub} output rows, {cite})",
            "value": res.output_tuples * steps / (sum(ms) / 1e3), "unit": UNIT, "steps": steps,
            "ms_per_step": sum(ms) / steps, "tuples": int(res.output_tuples),
            "matches_published": bool(res.output_tuples == pub),
            "matches_reference": (bool(res.output_tuples == ref["tuples"]) if ref and "tuples" in ref else None),
            "roofline": roofline, "kernels": kernels,
            "gpu_launches": launches, "reference_gpu": ref}


def measure_sg_dataset(eng, args, dev, flush) -> dict:
    """SG at 10^8+ tuples: the reference's fe_body input (163,734 edges; the
    reference published 408,443,204 tuples in 125 iterations), timed like the
    main leg (device events, result rows in HBM), with the dominant sort-path
    kernel's roofline and the reference's own GPU program on the same input."""
    import torch
    fname, name, pub_tuples, pub_iters, cite = SG_DATASET
    edges = load_fixture(fname)
    ref = None
    if not args.no_reference_gpu:
        ref = run_reference_gpu("sg", edges)
    d_edges = torch.from_numpy(edges).to(dev)
    steps = max(1, min(args.steps, 3))
    ms, r, prof = timed_fixpoints(eng, "sg", d_edges, steps, 1, "auto", dev, 1, lambda: None, flush)
    roofline, kernels, _, launches = roofline_of(prof, sum(ms) / 1e3)
    cpu = None if args.no_cpu_baseline else sg_cpu_sample()
    return {"workload": f"SG on {name} ({fname}, {len(edges)} edges; the reference published {pub_tuples} tuples "
                        f"in {pub_iters} iterations, {cite})",
            "value": r.output_tuples * steps / (sum(ms) / 1e3), "unit": UNIT, "steps": steps,
            "ms_per_step": sum(ms) / steps, "tuples": int(r.output_tuples), "iterations": int(r.iterations),
            "matches_published": bool(r.output_tuples == pub_tuples and r.iterations == pub_iters),
            "roofline": roofline, "kernels": kernels, "gpu_launches": launches, "reference_gpu": ref,
            "cpu_baseline": cpu}


def sg_cpu_sample() -> dict:
    """SG on the host cores: the reference has no CPU SG program, so the
    oracle's single-core restatement of sg.cu is timed (project code, labelled
    "port") on a bounded sample -- the small lattice of the SG generator
    (4,702 edges, 4.4M SG tuples, a few seconds)."""
    from oracle import cpu as oracle_cpu
    e = load_fixture("synth_lattice_small.bin")
    t0 = time.perf_counter()
    r = oracle_cpu.sg(e)
    sec = time.perf_counter() - t0
    return {"value": len(r.rows) / sec, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"SG of the small lattice (tests/golden/data/synth_lattice_small.bin, {len(e)} edges): "
                      f"{len(r.rows)} tuples in {r.iterations} iterations, {sec:.2f} s, the oracle's C restatement "
                      f"of sg.cu on one core (the reference has no CPU SG program)"}


def traffic_per_launch(kernel: str, stat: dict):
    """DRAM bytes per launch: the ncu-measured DRAM/algorithmic byte ratio of
    this kernel class (profiles/ncu_traffic.json) times this run's
    algorithmic bytes per launch; null without a capture."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            ratio = json.load(f)[kernel]["dram_per_algorithmic_byte"]
    except Exception:
        return None
    return ratio * stat["bytes"] / max(stat["timed_launches"], 1)


def measure_e2e(eng, prog, edges, args, dev, world, barrier) -> dict:
    import torch
    h_edges = torch.from_numpy(edges).pin_memory().numpy()
    probe = eng.run(prog, h_edges, output="none", dedup=args.dedup)
    out_rows = probe.output_tuples
    out = torch.empty((out_rows, 2), dtype=torch.int32).pin_memory().numpy()
    steps = max(1, min(args.steps, 3))
    barrier()
    torch.cuda.synchronize(dev)
    gc.collect()
    gc.disable()  # as in the device-timed steps: no collection inside the timing
    try:
        t0 = time.perf_counter()
        tuples = 0
        for _ in range(steps):
            r = eng.run(prog, h_edges, output="host", out=out, dedup=args.dedup)
            tuples += r.output_tuples
        torch.cuda.synchronize(dev)
        sec = time.perf_counter() - t0
    finally:
        gc.enable()
    sec, total = combine_ranks(sec, float(tuples), world, dev)
    return {"value": total / sec, "unit": UNIT,
            "h2d_bytes_per_step": int(edges.nbytes), "d2h_bytes_per_step": int(out_rows * 8),
            "steps": steps, "timer": "host wall clock, synchronized"}


def combine_ranks(seconds: float, units: float, world: int, device=None) -> tuple[float, float]:
    """Whole-job timing over the ranks: the slowest rank's time and the sum
    of the units every rank processed. Every rank must call it (a collective
    when world > 1); `device` is the tensor device of the process group's
    backend (a CUDA device for NCCL, None for gloo)."""
    if world <= 1:
        return seconds, units
    import torch
    import torch.distributed as dist
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


def measure_batched(eng, dev, args) -> dict:
    """The batched form on 1,024 instances (half TC on DAGs, half WCC on
    Chung-Lu graphs with exponent 2.3, edge counts log-uniform in 1K-200K):
    dl_run_batch per program against the plain engine run one instance at a
    time, inputs resident in HBM for both, outputs left on the device."""
    import torch

    from mnmgdatalog_b200 import autotune, graphs
    work = graphs.batched_workload(count=args.batch_instances, seed=0)
    groups = {p: [torch.from_numpy(e).to(dev) for q, e in work if q == p] for p in ("tc", "wcc")}
    torch.cuda.synchronize(dev)
    # The knobs come from the committed record of an autotuner run on this
    # workload (mnmgdatalog_b200/tuning_batch.json), so that every box runs
    # the same configuration; --autotune re-runs the autotuner on a sample
    # (every 4th TC instance; its deltas must not change). Both the batched
    # and the plain runs use them.
    before = eng.tuning()
    if args.autotune:
        tuned = autotune.autotune_batch(eng, "tc", groups["tc"][::4], repeats=2, log=lambda *_: None)["tuning"]
        source = "autotuned in this run"
    else:
        with open(TUNING_BATCH) as f:
            tuned = json.load(f)["tuning"]
        source = "mnmgdatalog_b200/tuning_batch.json"
    eng.set_tuning(tuned)
    for _ in range(max(1, min(args.warmup, 2))):
        for p, g in groups.items():
            eng.run_batch(p, g, output="none")
    eng.synchronize()
    reps = max(5, min(args.steps, 7))
    times = []
    for _ in range(reps):
        gc.collect()
        gc.disable()  # no collection inside a timed repetition
        try:
            t0 = time.perf_counter()
            batched = {p: eng.run_batch(p, g, output="none") for p, g in groups.items()}
            eng.synchronize()
            times.append(time.perf_counter() - t0)
        finally:
            gc.enable()
    t_batch = statistics.median(times)
    # one more batched run under the live profile (outside the timing): the
    # sorted-runs kernels' shares and roofline fractions on this workload
    eng.profile(True)
    t0 = time.perf_counter()
    for p, g in groups.items():
        eng.run_batch(p, g, output="none")
    eng.synchronize()
    t_prof = time.perf_counter() - t0
    prof = eng.profile_read()
    eng.profile(False)
    b_roofline, b_kernels, b_host, b_launches = roofline_of(prof, t_prof)
    gc.collect()
    gc.disable()
    try:
        t0 = time.perf_counter()
        plain = {p: [eng.run(p, x, output="none") for x in g] for p, g in groups.items()}
        eng.synchronize()
        t_plain = time.perf_counter() - t0
    finally:
        gc.enable()
    same = all(a.iterations == b.iterations and a.output_tuples == b.output_tuples
               and a.deltas.tolist() == b.deltas.tolist()
               for p in groups for a, b in zip(batched[p], plain[p]))
    eng.set_tuning(before)
    n = sum(len(g) for g in groups.values())
    tuples = sum(r.output_tuples for p in ("tc",) for r in plain[p])
    return {"workload": f"{n} instances: {len(groups['tc'])} TC on DAGs + {len(groups['wcc'])} WCC on Chung-Lu "
                        f"gamma=2.3, edges log-uniform 1K-200K (seed 0)",
            "edges_total": int(sum(len(e) for _, e in work)), "tc_tuples": int(tuples),
            "queries_per_s": n / t_batch, "plain_queries_per_s": n / t_plain,
            "speedup_vs_plain": t_plain / t_batch, "seconds": t_batch, "plain_seconds": t_plain,
            "reps": reps, "batch_seconds": {"median": t_batch, "min": min(times), "max": max(times)},
            "queries_per_s_range": [n / max(times), n / min(times)],
            "identical_to_plain": bool(same), "tuning": tuned, "tuning_source": source,
            "roofline": b_roofline, "kernels": b_kernels, "host": b_host, "gpu_launches": b_launches,
            "profiled_run": "one extra batched run under the live profile, outside the timing",
            "timer": "host wall clock around dl_run_batch per program (synchronized), inputs in HBM",
            "form": "union fixpoint per program (one launch sequence per iteration for all instances)"}


def measure_served(eng, args, tuning=None) -> dict:
    """The served form: a Poisson stream of mixed TC/SG/WCC requests (edge
    counts log-uniform in 1K-500K) through the continuous-batching server with
    a 150 GB HBM budget, against the plain engine serving the same requests
    one at a time. Capacity is measured with every request queued at t=0;
    the Poisson run uses 80% of it."""
    from mnmgdatalog_b200 import serve
    reqs = serve.mixed_requests(args.serve_requests, lo=1000, hi=500_000, pool=args.serve_pool, seed=0,
                                distinct=True)
    for r in reqs[:6]:  # warm-up of every program
        eng.run(r.program, r.edges, output="none")
    before = eng.tuning()
    if tuning:
        eng.set_tuning(tuning)
    # the plain engine on an evenly spaced sample of the same stream (one at a
    # time it would take minutes for all of it); its rate is the comparison
    every = max(1, len(reqs) // max(1, args.serve_plain_sample))
    sample = reqs[::every]
    t_plain, svc, _ = serve.serve_plain(eng, sample, pinned=True, keep_results=False)
    eng.set_tuning(before)
    eng.release_memory()  # the plain engine's cached buffers would crowd the server's budget
    plain_qps = len(sample) / t_plain

    def fresh():
        return [serve.Request(r.id, r.program, r.edges) for r in reqs]

    # one server for all runs: its sessions and buffers stay warm, like a
    # service that has been up for a while
    srv = serve.Server(eng, budget_bytes=SERVE_BUDGET, keep_results=False, concurrent=True, pinned=True,
                       tuning=tuning)
    # the objects that exist now (requests, graphs, the library) are moved out
    # of the collector's reach, so collections during serving stay short
    gc.collect()
    gc.freeze()
    try:
        srv.serve([serve.Request(r.id, r.program, r.edges) for r in reqs[:120]])  # warm-up
        sats = [srv.serve(fresh()) for _ in range(2)]
        sat = max(sats, key=lambda x: x.queries_per_s)
        # the Poisson load is 80% of the slower saturated run: the faster one
        # is not sustained under arrivals spread over time on every box
        rate = 0.8 * min(x.queries_per_s for x in sats)
        stream = fresh()
        arr = serve.poisson_arrivals(len(stream), rate, np.random.default_rng(1))
        for r, t in zip(stream, arr):
            r.arrival = float(t)
        poi = srv.serve(stream)
    finally:
        srv.close()
        gc.unfreeze()
    sp50, sp95, sp99, _ = serve.percentiles(svc)
    return {"workload": f"{len(reqs)} requests, TC/SG/WCC uniform, edges log-uniform 1K-500K "
                        f"({sum(len(r.edges) for r in reqs)} edges in all); every input distinct: one of "
                        f"{args.serve_pool} seeded graphs per program under the request's own seeded id map; "
                        f"Poisson arrivals at 80% of the slower saturated run",
            "plain_sample": f"every {every}th request ({len(sample)})",
            "capacity_queries_per_s": sat.queries_per_s, "capacity_runs": [x.queries_per_s for x in sats],
            "plain_queries_per_s": plain_qps,
            "speedup_vs_plain": sat.queries_per_s / plain_qps,
            "poisson_rate": rate, "poisson_queries_per_s": poi.queries_per_s,
            "latency_s": {"p50": poi.latency_p50, "p95": poi.latency_p95, "p99": poi.latency_p99,
                          "max": poi.latency_max},
            "saturated_latency_s": {"p50": sat.latency_p50, "p95": sat.latency_p95, "p99": sat.latency_p99},
            "plain_service_s": {"p50": sp50, "p95": sp95, "p99": sp99},
            "max_active": poi.max_active, "peak_device_bytes": poi.peak_device_bytes,
            "budget_bytes": poi.budget_bytes, "budget_waits": poi.waits_on_budget,
            "server": "continuous batching, one union session per program, one worker thread and stream per "
                      "program; warmed with 120 requests; capacity = better of two saturated runs; Poisson load "
                      "at 80% of the slower one",
            "tuning": tuning,
            "delivery": "result rows copied into reused page-locked host buffers (served and plain alike)",
            "timer": "host wall clock; latency = result rows on the host - arrival"}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", default="tc_chung_lu_317k")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU program on the same input (context figure)")
    ap.add_argument("--dedup", choices=["auto", "sort", "hash", "bitmap"], default="auto",
                    help="how TC removes known tuples (same results)")
    ap.add_argument("--no-sg-leg", dest="sg_leg", action="store_false",
                    help="skip the SG leg on the reference's fe_body input")
    ap.add_argument("--no-single-join-leg", dest="single_join_leg", action="store_false",
                    help="skip the single_join leg (10M rows, the reference's strong-scaling input)")
    ap.add_argument("--tuning", action="append", default=[], metavar="KNOB=VALUE",
                    help="engine knob for the main leg (dl_tuning field), e.g. bitmap_result=2; repeatable")
    ap.add_argument("--batch-instances", type=int, default=1024, help="batched form instances (0: skip)")
    ap.add_argument("--autotune", action="store_true",
                    help="re-run the autotuner for the batched leg instead of the committed knobs")
    ap.add_argument("--serve-requests", type=int, default=20000, help="served form requests (0: skip)")
    ap.add_argument("--serve-pool", type=int, default=64, help="seeded base graphs per program")
    ap.add_argument("--serve-plain-sample", type=int, default=1000,
                    help="requests of the stream the plain engine serves one at a time")
    args = ap.parse_args(argv)
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local_rank = _env_int("LOCAL_RANK", 0)
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = "gloo" if args.impl == "reference" else "nccl"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local_rank)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            return main_reference(args, rank, world)
        return main_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    raise SystemExit(main())
