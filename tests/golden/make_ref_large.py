"""Golden records of the reference's own GPU programs on its large datasets.

    python tests/golden/make_ref_large.py copy [--ref DIR]   # where the reference tree is
    python tests/golden/make_ref_large.py run [--out FILE]   # on a machine with a B200

`copy` gzip-copies the reference's larger data files (data/*.bin; the inputs
behind its published TC/SG counts) into tests/golden/data/. DIR defaults to
$DL_REFERENCE_TREE.

`run` executes the reference's tc.out / sg.out (built unmodified from its
sources by oracle/Makefile into oracle/_ref/, single-rank MPI stub) on each
input as one rank, and records per case: the CSV's iteration and tuple counts,
the reference's own total time (CSV column "Total Time", which excludes file
I/O, tc.cu:387-389), and the SHA-256 of the output file it writes
(<input>_tc.bin / _sg.bin, rows in the reference file order). Cases whose
output has 2^31 or more int32 values cannot be written by the reference
(parallel_write passes `row_size * total_columns` as an int count,
common/parallel_io.cu:117-119), so those run with job_run=1 and are pinned by
counts and iterations only. The result goes to tests/golden/ref_large.json,
which tests/test_large_parity_gpu.py compares the engine against.
"""
from __future__ import annotations

import argparse
import gzip
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# (case, program, input, published (tuples, iterations) or None, citation of the published count)
CASES = [
    ("gnutella_tc", "tc", "data_147892.bin", (884_179_859, 31), "logs/small-merged-job-output.txt:89"),
    ("usroad_tc", "tc", "data_165435.bin", (871_365_688, 606), "logs/small-merged-job-output.txt:51"),
    ("fe_ocean_tc", "tc", "data_409593.bin", (1_669_750_513, 247), "logs/small-merged-job-output.txt:70"),
    ("sf_cedge_tc", "tc", "data_223001.bin", (80_498_014, 287), "logs/small-merged-job-output.txt:108"),
    ("fe_body_tc", "tc", "data_163734.bin", (156_120_489, 188), "rough/README.md:274"),
    ("sf_cedge_sg", "sg", "data_223001.bin", (382_418_182, 269), "logs/small-merged-job-output.txt:161"),
    ("fe_body_sg", "sg", "data_163734.bin", (408_443_204, 125), "logs/small-merged-job-output.txt:212"),
    ("brightkite_sg", "sg", "data_214078.bin", (92_398_050, 18), "logs/small-merged-job-output.txt:193"),
    ("fe_sphere_sg", "sg", "data_49152.bin", (205_814_096, 127), "logs/small-merged-job-output.txt:231"),
    ("ca_hepth_sg", "sg", "data_51971.bin", (74_618_689, 9), "logs/small-merged-job-output.txt:250"),
    ("ego_facebook_sg", "sg", "data_88234.bin", (15_018_986, 13), "logs/small-merged-job-output.txt:269"),
    ("fe_ocean_sg", "sg", "data_409593.bin", (65_941_441, 77), "README.md:54"),
    ("tc_chung_lu_317k", "tc", "synthetic:tc_chung_lu_317k", None, None),
    # single_join's synthetic rows (glibc srand(1)/rand(), common/parallel_io.cu:79-108): the weak- and
    # strong-scaling inputs of one rank; the reference never writes this program's output file (job_run
    # is fixed at 1, single_join.cu:78), so these are pinned by counts
    # (the log line before each cited result holds the command: rows, cuda_aware, comm_method, rand_range)
    ("single_join_weak", "single_join", "rows:10000000:500000", (199_915_594, 1),
     "logs/single-join-small-job-output.txt:58"),
    ("single_join_strong", "single_join", "rows:10000001:90000", (1_037_050_773, 1),
     "logs/single-join-small-job-output.txt:106"),
    ("single_join_10m_100k", "single_join", "rows:10000000:100000", (950_725_901, 1),
     "logs/single-join-small-job-output.txt:10"),
]

LARGE_FILES = sorted({c[2] for c in CASES if not c[2].startswith(("synthetic:", "rows:"))})
INT_MAX = 2**31 - 1


def load_case_input(name: str) -> np.ndarray:
    """Edges of a case: a gzip fixture under tests/golden/data/ or a seeded
    generator of mnmgdatalog_b200.graphs ("synthetic:<config>")."""
    if name.startswith("synthetic:"):
        from mnmgdatalog_b200 import graphs
        return graphs.make(name.split(":", 1)[1], seed=0)[1]
    if name.startswith("rows:"):  # single_join rows: (count, rand_range) through the library's generator
        from mnmgdatalog_b200 import generate_rows
        _, rows, rng = name.split(":")
        return generate_rows(int(rows), int(rng), 1)
    with gzip.open(os.path.join(HERE, "data", name + ".gz"), "rb") as f:
        raw = f.read()
    return np.frombuffer(raw, dtype="<i4")[: (len(raw) // 8) * 2].reshape(-1, 2).copy()


def copy(ref: str) -> None:
    out = os.path.join(HERE, "data")
    for fname in LARGE_FILES:
        with open(os.path.join(ref, "data", fname), "rb") as f:
            raw = f.read()
        dst = os.path.join(out, fname + ".gz")
        if os.path.exists(dst):
            with gzip.open(dst, "rb") as f:
                if f.read() == raw:
                    continue
        with open(dst, "wb") as f, gzip.GzipFile(fileobj=f, mode="wb", compresslevel=9, mtime=0) as g:
            g.write(raw)
        print(fname, len(raw) // 8, "rows")


def sha_file(path: str) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        while True:
            b = f.read(64 << 20)
            if not b:
                break
            h.update(b)
    return h.hexdigest()


def run(out_path: str, only: list[str], timeout: int) -> None:
    refdir = os.path.join(ROOT, "oracle", "_ref")
    results = {}
    if os.path.exists(out_path):
        with open(out_path) as f:
            results = json.load(f).get("cases", {})
    for case, prog, inp, published, cite in CASES:
        if only and case not in only:
            continue
        binary = os.path.join(refdir, f"{prog}.out")
        if prog == "single_join":  # generates its own rows: argv = rows, cuda_aware, comm_method, rand_range
            _, rows, rng = inp.split(":")
            t0 = time.perf_counter()
            r = subprocess.run([binary, rows, "0", "0", rng], capture_output=True, text=True, timeout=timeout)
            wall = time.perf_counter() - t0
            if r.returncode != 0:
                raise SystemExit(f"{case}: {binary} exited {r.returncode}\n{r.stderr[-2000:]}")
            csv = [l for l in r.stdout.splitlines() if l and l[0].isdigit()][-1].split(",")
            results[case] = {"program": prog, "input": inp, "input_rows": int(csv[0]), "iterations": 1,
                             "tuples": int(csv[3]), "reference_total_s": float(csv[4]), "wall_s": round(wall, 2),
                             "published": list(published), "published_source": cite,
                             "command": f"oracle/_ref/single_join.out {rows} 0 0 {rng}", "rows_sha256": None,
                             "rows_note": "the reference does not write this output (job_run = 1, single_join.cu:78)"}
            print(case, results[case]["tuples"], results[case]["reference_total_s"], flush=True)
            with open(out_path, "w") as f:
                json.dump({"generator": "tests/golden/make_ref_large.py run", "cases": results}, f, indent=1,
                          sort_keys=True)
            continue
        edges = load_case_input(inp)
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "input.bin")
            edges.astype("<i4").tofile(path)
            expect = published[0] if published else None
            # the reference's write passes rows * 2 as an int count
            write = expect is not None and 2 * expect <= INT_MAX
            free = shutil.disk_usage(td).free
            if write and expect * 8 * 1.2 > free:
                write = False
            t0 = time.perf_counter()
            r = subprocess.run([binary, path, "0", "0", "0" if write else "1"], capture_output=True, text=True,
                               timeout=timeout, cwd=td)
            wall = time.perf_counter() - t0
            if r.returncode != 0:
                raise SystemExit(f"{case}: {binary} exited {r.returncode}\n{r.stderr[-2000:]}")
            csv = [l for l in r.stdout.splitlines() if l and l[0].isdigit()][-1].split(",")
            rec = {"program": prog, "input": inp, "input_rows": int(csv[0]), "iterations": int(csv[2]),
                   "tuples": int(csv[3]), "reference_total_s": float(csv[4]), "wall_s": round(wall, 2),
                   "published": list(published) if published else None, "published_source": cite,
                   "command": f"oracle/_ref/{prog}.out <input> 0 0 {0 if write else 1}"}
            outf = path + ("_tc.bin" if prog == "tc" else "_sg.bin")
            if write and os.path.exists(outf):
                size = os.path.getsize(outf)
                if size != rec["tuples"] * 8:
                    raise SystemExit(f"{case}: output file has {size} bytes for {rec['tuples']} tuples")
                rec["rows_sha256"] = sha_file(outf)
                os.remove(outf)
            else:
                rec["rows_sha256"] = None
                rec["rows_note"] = ("output not written: rows * 2 exceeds the int count of the reference's "
                                    "parallel_write" if expect is None or 2 * expect > INT_MAX
                                    else "output not written: disk space")
        results[case] = rec
        print(case, {k: rec[k] for k in ("iterations", "tuples", "reference_total_s", "wall_s")}, flush=True)
        with open(out_path, "w") as f:
            json.dump({"generator": "tests/golden/make_ref_large.py run", "cases": results}, f, indent=1,
                      sort_keys=True)


def main() -> int:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("copy")
    c.add_argument("--ref", default=os.environ.get("DL_REFERENCE_TREE"))
    r = sub.add_parser("run")
    r.add_argument("--out", default=os.path.join(HERE, "ref_large.json"))
    r.add_argument("--only", nargs="*", default=[])
    r.add_argument("--timeout", type=int, default=900)
    a = ap.parse_args()
    if a.cmd == "copy":
        if not a.ref:
            raise SystemExit("give --ref or set DL_REFERENCE_TREE to the reference source tree")
        copy(a.ref)
    else:
        run(a.out, a.only, a.timeout)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
