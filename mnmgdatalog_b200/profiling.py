"""Summaries of Nsight Compute captures of the engine's kernels.

    python -m mnmgdatalog_b200.profiling launches <ncu.csv> [bench.json]

reads an `ncu --csv` launch list (metrics gpu__time_duration.sum and,
optionally, dram__bytes_read.sum / dram__bytes_write.sum) and prints, per
kernel class of the live profile (the names bench.py reports), the launches,
total device time, share, and DRAM bytes. Given the bench JSON line of the
same command, it also prints each class's DRAM bytes per algorithmic byte,
the ratio bench.py scales into `roofline.traffic`
(profiles/ncu_traffic.json).
"""
from __future__ import annotations

import csv
import json
import re
import sys
from collections import defaultdict

# kernel function name (regex on the demangled name) -> live-profile class
CLASSES = [
    (r"diff_merge_kernel", "diff_merge"),
    (r"radix_downsweep_kernel|onesweep_kernel", "sort_scatter_pass"),
    (r"radix_upsweep_kernel|radix_hist_kernel", "sort_histogram"),
    (r"scan_kernel<.*WordValue", "sort_spine_scan"),
    (r"radix_bucket_kernel", "sort_spine_scan"),
    (r"scan_kernel<.*DegreeOp", "join_count_scan"),
    (r"join_emit_kernel<.*WccSrc", "wcc_propagate"),
    (r"join_emit_kernel|join_emit_bucket_kernel", "join_emit"),
    (r"digit0_hist_kernel", "join_count_scan"),
    (r"bucket_starts_kernel", "join_partition"),
    (r"bitmat_unit_step_kernel|bitmat_set_edges_kernel", "bitmap_expand"),
    (r"bitmat_transpose_count|bitmat_column_count|column_offsets", "bitmap_columns"),
    (r"bitmat_extract|bitmat_column_rows|scan_kernel<.*CountValue", "bitmap_extract"),
    (r"lbs_partition_kernel", "join_partition"),
    (r"select_kernel", "select_compact"),
    (r"merge_partition_kernel", "merge_partition"),
    (r"merge_kernel", "merge"),
    (r"sparse_mark_kernel|sample_kernel", "sparse_diff"),
    (r"hash_insert_kernel|extract_values_kernel", "hash_build"),
    (r"wordset_insert_kernel|wordset_rehash_kernel", "hash_insert"),
]


def kernel_class(name: str) -> str | None:
    for pat, cls in CLASSES:
        if re.search(pat, name):
            return cls
    if "dl::" in name or "session_" in name or "_kernel" in name:
        return "prep"
    return None  # not one of ours (e.g. a torch fill)


def read_ncu_csv(path: str) -> list[dict]:
    """Rows of `ncu --csv` output: one dict per (launch, metric)."""
    with open(path, newline="") as f:
        lines = [ln for ln in f if ln.startswith('"')]
    return list(csv.DictReader(lines))


def summarize(rows: list[dict]) -> dict:
    per = defaultdict(lambda: {"launches": set(), "ns": 0.0, "dram": 0.0, "kernels": set()})
    for r in rows:
        cls = kernel_class(r.get("Kernel Name", ""))
        if cls is None:
            continue
        d = per[cls]
        d["launches"].add(r.get("ID"))
        d["kernels"].add(re.sub(r"<.*", "", r.get("Kernel Name", "")))
        name, unit = r.get("Metric Name"), r.get("Metric Unit", "")
        try:
            v = float(r.get("Metric Value", "0").replace(",", ""))
        except ValueError:
            continue
        if name == "gpu__time_duration.sum":
            d["ns"] += v * {"nsecond": 1, "usecond": 1e3, "msecond": 1e6, "second": 1e9}.get(unit, 1)
        elif name in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
            d["dram"] += v * {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "KB": 1e3, "MB": 1e6,
                              "GB": 1e9}.get(unit, 1)
    total = sum(d["ns"] for d in per.values()) or 1.0
    return {c: {"launches": len(d["launches"]), "ms": d["ns"] / 1e6, "share": d["ns"] / total,
                "dram_bytes": d["dram"], "kernels": sorted(d["kernels"])} for c, d in per.items()}


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if len(argv) < 2 or argv[0] != "launches":
        print(__doc__)
        return 2
    s = summarize(read_ncu_csv(argv[1]))
    bench = None
    if len(argv) > 2:
        with open(argv[2]) as f:
            bench = json.loads([ln for ln in f if ln.strip().startswith("{")][-1])
    print(f"{'class':20s} {'launches':>8s} {'ms':>10s} {'share':>7s} {'DRAM GB':>9s} {'DRAM/alg':>9s}")
    for c, d in sorted(s.items(), key=lambda kv: -kv[1]["ms"]):
        ratio = ""
        if bench and c in bench.get("kernels", {}) and bench["kernels"][c].get("bytes"):
            ratio = f"{d['dram_bytes'] / bench['kernels'][c]['bytes']:.3f}" if d["dram_bytes"] else ""
        print(f"{c:20s} {d['launches']:8d} {d['ms']:10.3f} {100 * d['share']:6.1f}% {d['dram_bytes'] / 1e9:9.3f} "
              f"{ratio:>9s}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
