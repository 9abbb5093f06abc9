"""Autotuner of the engine's knobs (dl_tuning) on a sample workload.

    python -m mnmgdatalog_b200.autotune [--config tc_chung_lu_40k] [--out tuning.json]

Times candidate settings on a sample workload -- the radix pass variant
(three-kernel LSD or onesweep, shared-memory or ballot ranking, onesweep
tile), the dense/sparse threshold and the small-run fold threshold of the
semi-naive step, for TC the bit-matrix dedup against the tuned sort path,
and the default load factor of the C-ABI hash table (on a join of the
sample's edges) -- by coordinate descent, keeps the fastest, and
checks that every candidate gives identical results (iterations,
per-iteration deltas, rows). The knobs never change results, only time.
autotune_batch() does the same for the batched form (dl_run_batch of a sample
of the instances). The chosen setting is written as JSON;
Engine.set_tuning(path) applies it to a context.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

SORT_VARIANTS = [  # (sort_algorithm, sort_ranking, sort_keys_per_thread, sort_input_tma, join_first_pass)
    (1, 1, 16, 1, 1), (1, 1, 16, 1, 0), (1, 1, 16, 0, 1), (1, 0, 16, 1, 1), (0, 1, 16, 1, 0), (0, 0, 16, 1, 0),
    (0, 1, 12, 1, 0),
]
RATIOS = [2, 4, 8]
LOAD_FACTORS = [0.25, 0.5, 0.7]
BITMAP_GIB = [48, 0]  # TC dedup: bit matrix when it fits in 48 GiB, or never (sort path)


def candidates(stage: str, best: dict) -> list[dict]:
    """Settings to try in one coordinate-descent stage, around `best`."""
    out = []
    if stage == "sort":
        for a, r, k, t, f in SORT_VARIANTS:
            out.append(dict(best, sort_algorithm=a, sort_ranking=r, sort_keys_per_thread=k, sort_input_tma=t,
                            join_first_pass=f))
    elif stage == "dense_ratio":
        out = [dict(best, dense_ratio=v) for v in RATIOS]
    elif stage == "small_ratio":
        out = [dict(best, small_ratio=v) for v in RATIOS]
    elif stage == "hash_load_factor":
        out = [dict(best, hash_load_factor=v) for v in LOAD_FACTORS]
    elif stage == "bitmap_max_gib":
        out = [dict(best, bitmap_max_gib=v) for v in BITMAP_GIB]
    else:
        raise ValueError(stage)
    uniq = []
    for c in out:
        if c not in uniq:
            uniq.append(c)
    return uniq


def tune(eng, run, *, stages=("sort", "dense_ratio", "small_ratio"), repeats: int = 2, log=print) -> dict:
    """Coordinate descent over `stages` for a workload. `run(eng)` runs it
    once on eng's context and returns (seconds, signature); every setting
    must give the first setting's signature. Leaves the best setting applied
    and returns {"tuning": ..., "trials": [...]}."""
    best = eng.tuning()
    trials = []
    reference = None
    for stage in stages:
        scored = []
        for cand in candidates(stage, best):
            eng.set_tuning(cand)
            run(eng)  # warm-up of this setting
            secs = float("inf")
            for _ in range(repeats):
                t, sig = run(eng)
                secs = min(secs, t)
                if reference is None:
                    reference = sig
                elif sig != reference:
                    raise RuntimeError(f"setting {cand} changed the result")
            scored.append((secs, cand))
            trials.append({"stage": stage, "tuning": cand, "seconds": secs})
            log(f"{stage:16s} {json.dumps(cand)}  {secs * 1e3:9.3f} ms")
        best = min(scored, key=lambda x: x[0])[1]
    eng.set_tuning(best)
    return {"tuning": best, "trials": trials}


def _join_workload(rel):
    """get_hash_table (context default load factor) + get_join of a relation
    with itself; the signature is a checksum of the sorted join."""
    def run(eng):
        import torch
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        ht = eng.get_hash_table(rel)
        j = eng.get_join(ht, rel)
        b.record()
        torch.cuda.synchronize()
        ht.close()
        js = eng.sort_unique(j)
        sig = (len(js), int(js.to(torch.int64).sum().item()), int((js[:, 0].to(torch.int64) * 31 + js[:, 1]).sum()))
        return a.elapsed_time(b) * 1e-3, sig
    return run


def autotune(eng, program: str, edges, *, repeats: int = 2, log=print) -> dict:
    """Tunes eng's context on one plain run of `program` on `edges` (sort
    variant, dense and fold thresholds) and on a self-join of the edges (hash
    table load factor)."""
    import torch
    d_edges = torch.from_numpy(edges).cuda() if not isinstance(edges, torch.Tensor) else edges

    def run(e):
        r = e.run(program, d_edges, output="device")
        rows = r.rows.to(torch.int64)
        sig = (r.iterations, tuple(r.deltas.tolist()), r.output_tuples,
               int((rows[:, 0] * 1000003 + rows[:, 1]).sum().item()) if len(rows) else 0)
        return r.seconds, sig

    # TC: the sort path's knobs first, then bit matrix against the tuned sort path
    stages = ("sort", "dense_ratio", "small_ratio") + (("bitmap_max_gib",) if program == "tc" else ())
    res = tune(eng, run, stages=stages, repeats=repeats, log=log)
    res2 = tune(eng, _join_workload(d_edges.contiguous()), stages=("hash_load_factor",), repeats=repeats, log=log)
    return {"tuning": res2["tuning"], "trials": res["trials"] + res2["trials"]}


def autotune_batch(eng, program: str, edge_sets, *, repeats: int = 2, log=print) -> dict:
    """Tunes eng's context for the batched form: dl_run_batch of `edge_sets`
    (a sample of the instances), wall time; every instance's iterations,
    deltas and tuple count must not change."""
    def run(e):
        t0 = time.perf_counter()
        res = e.run_batch(program, edge_sets, output="none")
        e.synchronize()
        return time.perf_counter() - t0, tuple((r.iterations, tuple(r.deltas.tolist()), r.output_tuples)
                                               for r in res)

    return tune(eng, run, repeats=repeats, log=log)


def main(argv=None) -> int:
    from . import graphs
    from .engine import Engine
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--config", default="tc_chung_lu_40k", choices=sorted(graphs.CONFIGS))
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--repeats", type=int, default=2)
    ap.add_argument("--out", default="")
    args = ap.parse_args(argv)
    program, edges = graphs.make(args.config)
    with Engine(args.device) as eng:
        t0 = time.time()
        res = autotune(eng, program, edges, repeats=args.repeats)
        res.update({"config": args.config, "program": program, "tuning_seconds": time.time() - t0})
        print(json.dumps(res["tuning"]))
        if args.out:
            with open(args.out, "w") as f:
                json.dump(res, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
