"""The engine against the reference's own GPU programs on the reference's
large datasets and on the headline synthetic configuration.

tests/golden/ref_large.json holds what the reference's tc.out / sg.out (built
unmodified, run as one MPI rank on a B200 by tests/golden/make_ref_large.py)
printed and wrote for each case: iterations, tuple count and the SHA-256 of its
output file (rows in the reference's file order). Every case is also checked
against the count the reference published for that input. TC runs on both of
the engine's dedup paths (the bit matrix and the sorted runs); where the
reference cannot write its output (2^31 or more int32 values), the two paths'
rows are compared with each other instead; single_join's output the
reference never writes (job_run is fixed at 1, single_join.cu:78), so its
weak- and strong-scaling inputs are pinned by counts (rows are compared with
the oracle at smaller sizes in test_programs_gpu.py).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

_REF_PATH = os.path.join(GOLDEN, "ref_large.json")
REF = {}
if os.path.exists(_REF_PATH):
    with open(_REF_PATH) as _f:
        REF = json.load(_f)["cases"]


def _load(case):
    import sys
    sys.path.insert(0, GOLDEN)
    from make_ref_large import load_case_input
    return load_case_input(REF[case]["input"])


def _sha(rows) -> str:
    h = hashlib.sha256()
    flat = np.ascontiguousarray(rows, dtype="<i4").reshape(-1)
    step = 1 << 27
    for i in range(0, flat.size, step):
        h.update(memoryview(flat[i:i + step]).cast("B"))
    return h.hexdigest()


def _check_counts(case, r):
    ref = REF[case]
    assert r.iterations == ref["iterations"], (case, r.iterations, ref["iterations"])
    assert r.output_tuples == ref["tuples"], (case, r.output_tuples, ref["tuples"])
    if ref["published"]:
        assert ref["tuples"] == ref["published"][0], f"{case}: reference on B200 differs from its published count"
        assert r.output_tuples == ref["published"][0]


ROW_CASES = sorted(c for c, v in REF.items() if v["rows_sha256"])
COUNT_CASES = sorted(c for c, v in REF.items() if not v["rows_sha256"])


@pytest.mark.parametrize("case", ROW_CASES)
def test_rows_equal_reference(engine, case):
    ref = REF[case]
    # TC: the bit matrix with its result through the transpose and from its
    # columns, and the sorted runs
    modes = [("auto", 1), ("auto", 2), ("sort", 0)] if ref["program"] == "tc" else [("auto", 0)]
    before = engine.tuning()
    try:
        for dedup, form in modes:
            engine.set_tuning(bitmap_result=form)
            r = engine.run(ref["program"], _load(case), dedup=dedup)
            _check_counts(case, r)
            assert _sha(r.rows) == ref["rows_sha256"], f"{case} ({dedup}, {form}): rows differ from the reference's file"
            del r
    finally:
        engine.set_tuning(before)
    engine.release_memory()


@pytest.mark.parametrize("case", COUNT_CASES)
def test_counts_equal_reference_and_paths_agree(engine, case):
    """Counts and iterations against the reference; for TC the bit-matrix and
    sorted-run paths must give byte-identical rows (the reference cannot
    write this output file)."""
    ref = REF[case]
    edges = _load(case)
    shas = {}
    modes = ["auto", "sort"] if ref["program"] == "tc" else ["auto"]
    for dedup in modes:
        r = engine.run(ref["program"], edges, dedup=dedup, output="host" if len(modes) > 1 else "none")
        _check_counts(case, r)
        if len(modes) > 1:
            shas[dedup] = _sha(r.rows)
        del r
    assert len(set(shas.values())) <= 1, shas
    engine.release_memory()
