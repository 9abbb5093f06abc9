"""Autotuner host logic on CPU: the candidate settings of each stage."""
from mnmgdatalog_b200 import autotune

BASE = {"sort_algorithm": 1, "sort_ranking": 1, "sort_keys_per_thread": 16, "sort_input_tma": 1, "dense_ratio": 4,
        "small_ratio": 4, "hash_load_factor": 0.5, "join_first_pass": 1, "bitmap_max_gib": 48}


def test_sort_stage_covers_every_variant_once():
    c = autotune.candidates("sort", BASE)
    keys = [(x["sort_algorithm"], x["sort_ranking"], x["sort_keys_per_thread"], x["sort_input_tma"],
             x["join_first_pass"]) for x in c]
    assert sorted(keys) == sorted(autotune.SORT_VARIANTS)
    assert all(x["dense_ratio"] == 4 and x["hash_load_factor"] == 0.5 for x in c)


def test_ratio_and_load_factor_stages_vary_one_knob():
    for stage, values in (("dense_ratio", autotune.RATIOS), ("small_ratio", autotune.RATIOS),
                          ("hash_load_factor", autotune.LOAD_FACTORS), ("bitmap_max_gib", autotune.BITMAP_GIB)):
        c = autotune.candidates(stage, BASE)
        assert [x[stage] for x in c] == values
        for x in c:
            assert {k: v for k, v in x.items() if k != stage} == {k: v for k, v in BASE.items() if k != stage}


def test_unknown_stage():
    import pytest
    with pytest.raises(ValueError):
        autotune.candidates("tile", BASE)
