"""Fixpoint programs on the GPU against the golden outputs and the live oracle
(bit-exact rows in the reference's file order, iteration counts and the
per-iteration delta sizes)."""
import numpy as np
import pytest

from conftest import load_expected, load_input, sha_rows
from oracle import cpu

pytestmark = pytest.mark.gpu

EXP = load_expected()
CASES = [(f, p) for f, e in EXP["inputs"].items() for p in ("tc", "sg", "wcc") if p in e]


@pytest.mark.parametrize("fname,prog", CASES)
def test_golden(engine, fname, prog):
    e = load_input(fname)
    rec = EXP["inputs"][fname][prog]
    if prog == "wcc":
        for mode in ("reference", "fixpoint"):
            r = engine.wcc(e, wcc_stop=mode, labels=True)
            w = rec[mode]
            assert (r.output_tuples, r.largest_component, r.iterations) == \
                (w["components"], w["largest"], w["iterations"]), mode
            assert r.deltas.tolist() == w["deltas"]
            assert sha_rows(r.rows) == w["rows_sha256"]
            assert sha_rows(np.stack([r.node_ids, r.labels], 1)) == w["labels_sha256"]
    else:
        r = engine.run(prog, e)
        assert len(r.rows) == rec["rows_count"]
        assert r.iterations == rec["iterations"]
        assert r.deltas.tolist() == rec["deltas"]
        assert sha_rows(r.rows) == rec["rows_sha256"]


@pytest.mark.parametrize("case", EXP["single_join"], ids=lambda c: f"{c['rows']}x{c['rand_range']}")
def test_single_join_golden(engine, case):
    from mnmgdatalog_b200 import generate_rows
    rows = generate_rows(case["rows"], case["rand_range"], 1)
    assert sha_rows(rows) == case["generated_sha256"]
    r = engine.single_join(rows)
    assert len(r.rows) == case["rows_count"] and r.iterations == 1
    assert sha_rows(r.rows) == case["rows_sha256"]


def _edge_cases():
    rng = np.random.default_rng(0)
    yield "single_edge", np.array([[1, 2]], np.int32)
    yield "self_loop", np.array([[5, 5]], np.int32)
    yield "two_cycle", np.array([[1, 2], [2, 1]], np.int32)
    yield "duplicates", np.array([[1, 2], [1, 2], [2, 3], [2, 3], [3, 1]], np.int32)
    yield "negative_ids", np.array([[-5, -1], [-1, 3], [3, -7], [-7, -5]], np.int32)
    yield "extreme_ids", np.array([[-2**31, 2**31 - 1], [2**31 - 1, 0], [0, -2**31]], np.int32)
    yield "sparse_ids", (rng.integers(0, 60, (150, 2)) * 35_000_000 - 2**30).astype(np.int32)
    yield "random_dense", rng.integers(0, 400, (1500, 2)).astype(np.int32)
    yield "star_out", np.stack([np.zeros(3000, np.int32), np.arange(1, 3001, dtype=np.int32)], 1)
    yield "star_in", np.stack([np.arange(1, 3001, dtype=np.int32), np.zeros(3000, np.int32)], 1)
    yield "chain", np.stack([np.arange(0, 700), np.arange(1, 701)], 1).astype(np.int32)


EDGE_CASES = list(_edge_cases())


@pytest.mark.parametrize("name,e", EDGE_CASES, ids=[c[0] for c in EDGE_CASES])
@pytest.mark.parametrize("prog", ["tc", "sg"])
def test_against_oracle(engine, name, e, prog):
    want = cpu.tc(e) if prog == "tc" else cpu.sg(e)
    got = engine.run(prog, e)
    assert np.array_equal(got.rows, want.rows)
    assert got.iterations == want.iterations
    assert got.deltas.tolist() == want.deltas.tolist()


@pytest.mark.parametrize("name,e", EDGE_CASES, ids=[c[0] for c in EDGE_CASES])
@pytest.mark.parametrize("mode", ["reference", "fixpoint"])
def test_wcc_against_oracle(engine, name, e, mode):
    want = cpu.wcc(e, cpu.STOP_REFERENCE if mode == "reference" else cpu.STOP_FIXPOINT)
    got = engine.wcc(e, wcc_stop=mode, labels=True)
    assert np.array_equal(got.rows, want.comp_rows)
    assert (got.largest_component, got.iterations) == (want.largest, want.iterations)
    assert got.deltas.tolist() == want.deltas.tolist()
    assert np.array_equal(got.node_ids, want.node_ids) and np.array_equal(got.labels, want.labels)


@pytest.mark.parametrize("prog", ["tc", "sg", "wcc", "single_join"])
def test_empty_input(engine, prog):
    r = engine.run(prog, np.zeros((0, 2), np.int32))
    assert len(r.rows) == 0


def test_device_input_matches_host_input(engine):
    import torch
    e = load_input("data_7035.bin")
    a = engine.tc(e)
    b = engine.tc(torch.from_numpy(e).cuda(), output="device")
    assert np.array_equal(a.rows, b.rows.cpu().numpy())
    assert a.deltas.tolist() == b.deltas.tolist()


def test_repeated_runs_reuse_buffers(engine):
    e = load_input("synth_dag_c0.bin")
    first = engine.tc(e)
    for _ in range(3):
        r = engine.tc(e)
        assert np.array_equal(r.rows, first.rows)


def test_release_memory_between_runs(engine):
    """The context gives its cached device memory back and the next runs
    allocate again, with the same results; a result held across the release
    stays valid."""
    import torch
    from mnmgdatalog_b200 import graphs
    e = graphs.chung_lu(n=4000, m=13000, seed=6)
    first = engine.tc(e, output="device")
    before = first.rows.clone()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    engine.release_memory()
    assert torch.cuda.mem_get_info()[0] >= free0
    assert torch.equal(first.rows, before)
    again = engine.tc(e)
    assert np.array_equal(again.rows, before.cpu().numpy())
    assert again.deltas.tolist() == first.deltas.tolist()
    sg = engine.sg(e[:3000])
    engine.release_memory()
    assert np.array_equal(engine.sg(e[:3000]).rows, sg.rows)


def test_phase_timing(engine):
    r = engine.tc(load_input("data_7035.bin"), phase_timing=True)
    assert r.seconds > 0 and set(r.phases) == {"initialization", "join", "deduplication", "merge",
                                               "finalization"}
    assert sum(r.phases.values()) > 0


TC_FILES = [f for f, e in EXP["inputs"].items() if "tc" in e]


@pytest.mark.parametrize("fname", TC_FILES)
@pytest.mark.parametrize("dedup", ["sort", "hash", "bitmap"])
def test_tc_dedup_modes(engine, fname, dedup):
    """Every way of removing known tuples gives the reference's rows, iteration
    count and per-iteration deltas."""
    e = load_input(fname)
    rec = EXP["inputs"][fname]["tc"]
    r = engine.tc(e, dedup=dedup)
    assert r.iterations == rec["iterations"]
    assert r.deltas.tolist() == rec["deltas"]
    assert sha_rows(r.rows) == rec["rows_sha256"]


@pytest.mark.parametrize("dedup", ["sort", "hash", "bitmap"])
def test_tc_dedup_modes_edge_cases(engine, dedup):
    for name, e in _edge_cases():
        got = engine.tc(e, dedup=dedup)
        want = cpu.tc(e)
        assert np.array_equal(got.rows, want.rows), name
        assert got.deltas.tolist() == list(want.deltas), name


def test_tc_dedup_modes_agree_at_scale(engine):
    """A closure of ~3e7 tuples (hash-set growth and rehash on the way)."""
    from mnmgdatalog_b200 import graphs
    import torch
    e = torch.from_numpy(graphs.chung_lu(n=40_000, m=132_500, seed=0)).cuda()
    a = engine.tc(e, dedup="sort", output="device")
    for mode in ("hash", "bitmap"):
        b = engine.tc(e, dedup=mode, output="device")
        assert a.iterations == b.iterations and a.deltas.tolist() == b.deltas.tolist(), mode
        assert a.join_rows_total == b.join_rows_total, mode
        assert torch.equal(a.rows, b.rows), mode


@pytest.mark.parametrize("unit_rows", [1, 7, 64])
def test_tc_bitmap_small_units(engine, unit_rows):
    """Work units of a few delta rows: every source's delta is split over many
    units (and CTAs) and emitted again in split units; the results must not
    change."""
    from mnmgdatalog_b200 import graphs
    before = engine.tuning()
    inputs = [graphs.chung_lu(n=3000, m=10000, seed=2), graphs.dag(n=2000, extra=700, seed=4)]
    inputs += [load_input(f) for f in TC_FILES if len(load_input(f)) <= 20000][:3]
    try:
        engine.set_tuning(bitmap_unit_rows=unit_rows)
        for k, e in enumerate(inputs):
            a = engine.tc(e, dedup="sort")
            b = engine.tc(e, dedup="bitmap")
            assert a.deltas.tolist() == b.deltas.tolist(), k
            assert a.join_rows_total == b.join_rows_total, k
            assert np.array_equal(a.rows, b.rows), k
    finally:
        engine.set_tuning(before)


def test_tc_bitmap_max_iterations_and_selection(engine):
    """The bit-matrix path stops where the sort path stops, and AUTO picks it
    only while tuning allows (bitmap_max_gib = 0 turns it off)."""
    from mnmgdatalog_b200 import graphs
    e = graphs.chung_lu(n=6000, m=20000, seed=5)
    for k in (1, 2, 5):
        a = engine.tc(e, dedup="sort", max_iterations=k)
        b = engine.tc(e, dedup="bitmap", max_iterations=k)
        assert a.deltas.tolist() == b.deltas.tolist() and np.array_equal(a.rows, b.rows), k
    before = engine.tuning()
    try:
        for gib, used in ((48, True), (0, False)):
            engine.set_tuning(bitmap_max_gib=gib)
            engine.profile(True)
            r = engine.tc(e)
            prof = engine.profile_read()
            engine.profile(False)
            assert (prof.get("bitmap_expand", {}).get("launches", 0) > 0) == used, gib
            assert (prof.get("diff_merge", {}).get("launches", 0) > 0) != used, gib
            assert np.array_equal(r.rows, engine.tc(e, dedup="sort").rows)
    finally:
        engine.set_tuning(before)


@pytest.mark.parametrize("form", [1, 2])
def test_tc_bitmap_result_forms(engine, form):
    """The bit-matrix TC result through the matrix's transpose (1) and from
    its columns with per-block offsets (2): the same rows as the sort path,
    to host and device memory, with dense and sparse id ranges, node counts
    on and off the 512 / 1024 tile edges."""
    import torch
    from mnmgdatalog_b200 import graphs
    before = engine.tuning()
    inputs = [e for _, e in EDGE_CASES]
    inputs += [graphs.chung_lu(n=n, m=3 * n, seed=n) for n in (511, 1024, 1537, 5000)]
    inputs += [load_input(f) for f in TC_FILES if len(load_input(f)) <= 40000][:4]
    try:
        engine.set_tuning(bitmap_result=form)
        for k, e in enumerate(inputs):
            a = engine.tc(e, dedup="sort")
            b = engine.tc(e, dedup="bitmap")
            assert a.deltas.tolist() == b.deltas.tolist(), k
            assert np.array_equal(a.rows, b.rows), k
            d = engine.tc(torch.from_numpy(e).cuda(), dedup="bitmap", output="device")
            assert np.array_equal(d.rows.cpu().numpy(), a.rows), k
    finally:
        engine.set_tuning(before)


@pytest.mark.parametrize("form", [1, 2])
def test_tc_bitmap_unwritten_rows_read_as_zero(engine, form):
    """Only the matrix rows of sources with out-edges are zeroed and written;
    a run after one that filled every row (same node count, so the same
    matrix buffer and layout) must not see the earlier bits in the rows of its
    sinks."""
    rng = np.random.default_rng(11)
    n = 3000
    src = np.repeat(np.arange(n), 8)  # 8 random out-edges per node, plus a cycle: every row fills up
    full = np.concatenate([np.stack([src, rng.integers(0, n, size=len(src))], 1),
                           np.stack([np.arange(n), (np.arange(n) + 1) % n], 1)]).astype(np.int32)
    half = rng.integers(0, n, size=(4000, 2)).astype(np.int32)
    half[:, 0] = half[:, 0] % (n // 2)  # sources in the lower half only
    half = np.concatenate([half, [[n - 1, n - 1]]]).astype(np.int32)  # same id range
    before = engine.tuning()
    try:
        engine.set_tuning(bitmap_result=form)
        assert engine.tc(full, dedup="bitmap").output_tuples == n * n
        a = engine.tc(half, dedup="sort")
        b = engine.tc(half, dedup="bitmap")
        assert a.deltas.tolist() == b.deltas.tolist()
        assert np.array_equal(a.rows, b.rows)
    finally:
        engine.set_tuning(before)


@pytest.mark.parametrize("unit_rows", [1, 7, 65536])
def test_sg_bitmap_agrees_with_sorted_runs(engine, unit_rows):
    """SG on the bit matrix (the base rule's units (p, {p}), one fold per
    out-edge of a unit's source) against SG on the sorted runs, with delta
    units split into 1, 7 or up to 65,536 rows: the same iterations, deltas
    and rows."""
    from mnmgdatalog_b200 import graphs
    before = engine.tuning()
    inputs = [graphs.lattice3d(side=14, p=0.3, seed=5), graphs.chung_lu(n=3000, m=8000, seed=3),
              graphs.dag(n=1500, extra=500, seed=2)]
    inputs += [load_input(f) for f in ("data_10.bin", "hipc_2019.bin", "data_7035.bin", "quiz3.bin")]
    try:
        engine.set_tuning(bitmap_unit_rows=unit_rows)
        for k, e in enumerate(inputs):
            a = engine.sg(e, dedup="sort")
            b = engine.sg(e, dedup="bitmap")
            assert a.iterations == b.iterations and a.deltas.tolist() == b.deltas.tolist(), k
            assert np.array_equal(a.rows, b.rows), k
    finally:
        engine.set_tuning(before)
