"""Autotuner host logic (no GPU): candidate generation and the committed files."""
import glob
import json
import os

from trident_b200 import tune


def test_default_is_valid_and_at_capacity():
    t = tune.default_tuning()
    assert tune.valid(t)
    assert t["sym_lim"] == tune.SYM_CAP and t["num_lim"] == tune.NUM_CAP


def test_neighbours_are_valid_and_differ_in_one_slot():
    t = tune.default_tuning()
    seen = 0
    for u in tune.neighbours(t):
        assert tune.valid(u)
        diff = sum(a != b for a, b in zip(u["sym_lim"], t["sym_lim"]))
        diff += sum(a != b for a, b in zip(u["num_lim"], t["num_lim"]))
        diff += u["hash_load"] != t["hash_load"]
        diff += u["dense_win_log2"] != t["dense_win_log2"]
        diff += u["dense_win_fill_log2"] != t["dense_win_fill_log2"]
        diff += u["dense_win_cluster"] != t["dense_win_cluster"]
        assert diff == 1
        seen += 1
    assert seen > 10


def test_validity_rule():
    t = tune.default_tuning()
    bad = dict(t, num_lim=[600, 1024, 2048, 8192])      # above the warp table
    assert not tune.valid(bad)
    bad = dict(t, sym_lim=[512, 256, 4096, 24576])     # decreasing
    assert not tune.valid(bad)
    bad = dict(t, hash_load=3)
    assert not tune.valid(bad)
    assert not tune.valid(dict(t, dense_win_log2=5))
    assert tune.valid(dict(t, dense_win_log2=0))


def test_committed_tuning_files_are_valid():
    files = glob.glob(os.path.join(tune.TUNING_DIR, "*.json"))
    for f in files:
        with open(f) as fh:
            doc = json.load(fh)
        assert tune.valid(doc["tuning"]), f
        assert doc["ms"] <= doc["default_ms"] * 1.05, f
        assert doc["workload"] == os.path.basename(f)[:-5]
