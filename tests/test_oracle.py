"""The oracle against the reference's known answers (CPU only)."""
import numpy as np
import pytest

from conftest import load_input, sha_rows
from oracle import cpu


def test_published_counts(expected):
    for key, want in expected["published"].items():
        prog, fname = key.split(":", 1)
        e = load_input(fname)
        if prog == "wcc":
            w = cpu.wcc(e, cpu.STOP_REFERENCE)
            assert (w.n_components, w.largest, w.iterations) == tuple(want), key
        else:
            r = cpu.tc(e) if prog == "tc" else cpu.sg(e)
            assert (len(r.rows), r.iterations) == tuple(want), key


def test_golden_text_closures(expected):
    # data/data_5_TC.txt and data/dummy_TC.txt of the reference, as recorded
    for fname in ("data_5.bin", "dummy.bin"):
        rec = expected["inputs"][fname]["tc"]
        r = cpu.tc(load_input(fname))
        assert r.rows.tolist() == rec["rows"]


@pytest.mark.parametrize("fname", ["data_5.bin", "data_10.bin", "data_22.bin", "hipc_2019.bin", "dummy.bin",
                                   "paper.bin", "tc_paper.bin", "quiz3.bin", "data_7035.bin",
                                   "synth_dag_c0.bin", "synth_lattice_small.bin"])
def test_oracle_matches_expected(expected, fname):
    entry = expected["inputs"][fname]
    e = load_input(fname)
    for prog in ("tc", "sg"):
        if prog in entry:
            r = cpu.tc(e) if prog == "tc" else cpu.sg(e)
            assert len(r.rows) == entry[prog]["rows_count"]
            assert r.iterations == entry[prog]["iterations"]
            assert r.deltas.tolist() == entry[prog]["deltas"]
            assert sha_rows(r.rows) == entry[prog]["rows_sha256"]
    if "wcc" in entry:
        for mode, name in ((cpu.STOP_REFERENCE, "reference"), (cpu.STOP_FIXPOINT, "fixpoint")):
            w = cpu.wcc(e, mode)
            assert w.deltas.tolist() == entry["wcc"][name]["deltas"]
            assert sha_rows(w.comp_rows) == entry["wcc"][name]["rows_sha256"]


def test_wcc_reference_stop_rule_is_early_on_sf_cedge(expected):
    # The reference stops when |delta| repeats (wcc.cu:366-383): 17 components
    # on SF.cedge instead of 1 (rough/README.md:447).
    rec = expected["inputs"]["data_223001.bin"]["wcc"]
    assert rec["reference"]["components"] == 17 and rec["reference"]["iterations"] == 306
    assert rec["fixpoint"]["components"] == 1 and rec["fixpoint"]["largest"] == 174956


def test_tc_closure_brute_force_small():
    rng = np.random.default_rng(7)
    for _ in range(20):
        n = int(rng.integers(1, 12))
        e = rng.integers(-3, n, size=(int(rng.integers(0, 30)), 2)).astype(np.int32)
        if len(e) == 0:
            continue
        nodes = sorted(set(e.ravel().tolist()))
        reach = {u: set() for u in nodes}
        for a, b in e.tolist():
            reach[a].add(b)
        changed = True
        while changed:
            changed = False
            for u in nodes:
                new = set()
                for v in reach[u]:
                    new |= reach[v]
                if not new <= reach[u]:
                    reach[u] |= new
                    changed = True
        want = sorted(((x, z) for x in nodes for z in reach[x]), key=lambda t: (t[1], t[0]))
        assert cpu.tc(e).rows.tolist() == [list(t) for t in want]


@pytest.mark.parametrize("ranks", [1, 3, 4])
@pytest.mark.parametrize("fname", ["data_7035.bin", "synth_dag_c0.bin"])
def test_reference_cpu_program_on_forked_ranks(expected, tmp_path, fname, ranks):
    """The reference's CPU program rough/tc_mpi.cpp as several MPI ranks on
    the host (oracle/_ref/tc_mpi_fork, the CPU baseline): the same closure as
    the oracle's one-rank answer. With several ranks the file holds each
    rank's partition in rank order, so the rows are compared as a set."""
    import os
    import subprocess

    from conftest import ROOT
    binary = os.path.join(ROOT, "oracle", "_ref", "tc_mpi_fork")
    if not os.path.exists(binary):
        pytest.skip("oracle/_ref/tc_mpi_fork not built (needs the reference sources)")
    inp = tmp_path / fname
    load_input(fname).astype("<i4").tofile(inp)
    r = subprocess.run([binary, str(inp)], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, MPI_FORK_RANKS=str(ranks)))
    assert r.returncode == 0, r.stderr
    row = [l for l in r.stdout.splitlines() if l.startswith("|") and l[2:3].isdigit()][-1]
    cells = [c.strip().replace(",", "").replace("'", "") for c in row.strip("|").split("|")]
    rec = expected["inputs"][fname]["tc"]
    assert (int(cells[1]), int(cells[2]), int(cells[3])) == (ranks, rec["iterations"], rec["rows_count"])
    rows = np.fromfile(str(inp) + "_tc.bin", dtype="<i4").reshape(-1, 2)
    rows = rows[np.lexsort((rows[:, 0], rows[:, 1]))]  # the one-rank file order: (x, z) by (z, x)
    assert sha_rows(rows) == rec["rows_sha256"]
