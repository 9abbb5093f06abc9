"""Drop-in checks on the GPU:
* the reference's own drivers (tc.cu, tc_nl.cu, sg.cu, sg_nl.cu, wcc.cu,
  single_join.cu), built unmodified with common/hash_table.cu and
  common/join.cu replaced by the shims over libmnmgdl (oracle/Makefile
  `compat`), write the same files and CSV counts as the engine;
* the engine's own reference-compatible CLI programs (mnmgdatalog_b200/bin)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_expected, load_input, sha_rows

EXP = load_expected()

pytestmark = pytest.mark.gpu

COMPAT = os.path.join(ROOT, "oracle", "_ref", "compat")
BIN = os.path.join(ROOT, "mnmgdatalog_b200", "bin")
FILES = ["data_5.bin", "data_10.bin", "data_22.bin", "hipc_2019.bin", "dummy.bin", "paper.bin", "data_7035.bin",
         "data_23874.bin", "synth_dag_c0.bin", "synth_lattice_small.bin"]
PROGS = [("tc", "tc", "_tc.bin"), ("tc_nl", "tc", "_tc.bin"), ("sg", "sg", "_sg.bin"), ("sg_nl", "sg", "_sg.bin"),
         ("wcc", "wcc", "_cc.bin")]


def _run(exe, args, cwd):
    r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=300, cwd=cwd)
    assert r.returncode == 0, r.stderr[-2000:]
    row = [l for l in r.stdout.splitlines() if l and l[0].isdigit()][-1]
    return row.split(",")


def _engine(engine, prog, e):
    return engine.wcc(e, wcc_stop="reference") if prog == "wcc" else engine.run(prog, e)


@pytest.mark.parametrize("fname", FILES)
@pytest.mark.parametrize("binary,prog,suffix", PROGS, ids=[p[0] for p in PROGS])
def test_reference_driver_on_library(engine, tmp_path, fname, binary, prog, suffix):
    exe = os.path.join(COMPAT, binary + ".out")
    if not os.path.exists(exe):
        pytest.skip("drop-in binaries not built (oracle/Makefile `compat` needs the reference sources)")
    if prog == "sg" and fname == "data_23874.bin":
        pytest.skip("SG of TG.cedge is large for the reference's int sizes")
    e = load_input(fname)
    inp = tmp_path / fname
    e.astype("<i4").tofile(inp)
    csv = _run(exe, [str(inp)], tmp_path)
    got = np.fromfile(str(inp) + suffix, dtype="<i4").reshape(-1, 2)
    ours = _engine(engine, prog, e)
    assert int(csv[2]) == ours.iterations
    assert int(csv[3]) == ours.output_tuples
    assert np.array_equal(got, ours.rows)


@pytest.mark.parametrize("rows,rand_range", [(1000, 100), (200000, 200000)])
def test_reference_single_join_on_library(engine, tmp_path, rows, rand_range):
    exe = os.path.join(COMPAT, "single_join.out")
    if not os.path.exists(exe):
        pytest.skip("drop-in binaries not built")
    from mnmgdatalog_b200 import generate_rows
    csv = _run(exe, [str(rows), "0", "0", str(rand_range)], tmp_path)
    assert int(csv[3]) == engine.single_join(generate_rows(rows, rand_range, 1)).output_tuples


@pytest.mark.parametrize("fname", ["data_10.bin", "dummy.bin", "data_7035.bin", "synth_lattice_small.bin"])
@pytest.mark.parametrize("prog,suffix", [("tc", "_tc.bin"), ("sg", "_sg.bin"), ("wcc", "_cc.bin")])
def test_cli_programs(engine, tmp_path, fname, prog, suffix):
    exe = os.path.join(BIN, prog)
    assert os.path.exists(exe), "python -m mnmgdatalog_b200.build builds the CLI programs"
    e = load_input(fname)
    inp = tmp_path / fname
    e.astype("<i4").tofile(inp)
    csv = _run(exe, [str(inp), "0", "0", "0"], tmp_path)
    got = np.fromfile(str(inp) + suffix, dtype="<i4").reshape(-1, 2)
    ours = _engine(engine, prog, e)
    assert int(csv[0]) == len(e) and int(csv[1]) == 1
    assert int(csv[2]) == ours.iterations and int(csv[3]) == ours.output_tuples
    assert np.array_equal(got, ours.rows)
    # and the file against the reference's own output for this input
    rec = EXP["inputs"].get(fname, {}).get(prog)
    if rec and rec.get("rows_sha256"):
        assert sha_rows(got) == rec["rows_sha256"]
    # job_run = 1 writes no file
    os.remove(str(inp) + suffix)
    _run(exe, [str(inp), "0", "0", "1"], tmp_path)
    assert not os.path.exists(str(inp) + suffix)


def test_cli_single_join(engine, tmp_path):
    from mnmgdatalog_b200 import generate_rows
    csv = _run(os.path.join(BIN, "single_join"), ["20000", "0", "0", "5000"], tmp_path)
    assert int(csv[3]) == engine.single_join(generate_rows(20000, 5000, 1)).output_tuples
