"""Engine knobs (dl_tuning) on the GPU: validation, and results that do not
depend on them; the autotuner end to end on a small sample."""
import numpy as np
import pytest

from conftest import load_expected, load_input, sha_rows
from mnmgdatalog_b200 import DatalogError, autotune, graphs

pytestmark = pytest.mark.gpu

EXP = load_expected()


def test_tuning_round_trip_and_validation(engine):
    before = engine.tuning()
    try:
        engine.set_tuning(dense_ratio=8, small_ratio=2, hash_load_factor=0.7)
        t = engine.tuning()
        assert (t["dense_ratio"], t["small_ratio"], t["hash_load_factor"]) == (8, 2, 0.7)
        for bad in ({"dense_ratio": 0}, {"small_ratio": 65}, {"sort_algorithm": 2}, {"sort_keys_per_thread": 8},
                    {"hash_load_factor": 1.0}, {"sort_input_tma": 2}, {"join_first_pass": 3},
                    {"bitmap_max_gib": -1}, {"bitmap_max_gib": 1025}, {"bitmap_unit_rows": 0}):
            with pytest.raises(DatalogError):
                engine.set_tuning(**bad)
        with pytest.raises(DatalogError):
            engine.set_tuning(tile=3)
    finally:
        engine.set_tuning(before)
    assert engine.tuning() == before


@pytest.mark.parametrize("variant", autotune.SORT_VARIANTS)
@pytest.mark.parametrize("ratios", [(1, 1), (4, 4), (64, 64)])
def test_results_do_not_depend_on_tuning(engine, variant, ratios):
    before = engine.tuning()
    try:
        engine.set_tuning(sort_algorithm=variant[0], sort_ranking=variant[1], sort_keys_per_thread=variant[2],
                          sort_input_tma=variant[3], join_first_pass=variant[4], dense_ratio=ratios[0],
                          small_ratio=ratios[1])
        for fname, rec in EXP["inputs"].items():
            e = load_input(fname)
            for prog in ("tc", "sg"):
                if prog not in rec or len(e) > 20000:
                    continue
                r = engine.run(prog, e, dedup="sort")  # TC's AUTO would take the bit matrix
                assert r.deltas.tolist() == rec[prog]["deltas"], (fname, prog)
                assert sha_rows(r.rows) == rec[prog]["rows_sha256"], (fname, prog)
    finally:
        engine.set_tuning(before)


def test_autotune_small_sample(tmp_path):
    from mnmgdatalog_b200 import Engine
    edges = graphs.chung_lu(n=6000, m=20000, seed=3)
    with Engine(0) as eng:
        res = autotune.autotune(eng, "tc", edges, repeats=1, log=lambda *_: None)
        assert eng.tuning() == res["tuning"]
        stages = {t["stage"] for t in res["trials"]}
        assert stages == {"sort", "dense_ratio", "small_ratio", "bitmap_max_gib", "hash_load_factor"}
        plain = eng.tc(edges)
    with Engine(0) as ref:
        want = ref.tc(edges)
    assert np.array_equal(plain.rows, want.rows) and plain.deltas.tolist() == want.deltas.tolist()


def test_autotune_batch_small_sample():
    from mnmgdatalog_b200 import Engine
    sets = [graphs.dag(n=n, extra=n // 3, seed=i) for i, n in enumerate((300, 900, 2000, 150))]
    with Engine(0) as eng:
        res = autotune.autotune_batch(eng, "tc", sets, repeats=1, log=lambda *_: None)
        assert eng.tuning() == res["tuning"]
        got = eng.run_batch("tc", sets)
        for e, r in zip(sets, got):
            want = eng.tc(e)
            assert np.array_equal(r.rows, want.rows) and r.deltas.tolist() == want.deltas.tolist()
