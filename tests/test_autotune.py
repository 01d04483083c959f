"""The autotuner's choice among timed launch settings (pbf_b200/autotune.py), on
the CPU with made-up timing tables: the fastest row wins, except that a
persistent launch must beat the one-block-per-tile launches by more than the
timing spread (TIE) to be chosen; the cache returns a stored result."""
import json

from pbf_b200 import autotune


def _row(cs, bs, ln, ps, ms):
    return {"cell_scale": cs, "block_size": bs, "pair_lanes": ln, "persistent": ps, "ms_per_substep": ms}


def test_fastest_row_wins():
    table = [_row(1.0, 256, 2, 0, 0.40), _row(0.5, 128, 2, 0, 0.30), _row(0.5, 256, 4, 0, 0.35)]
    assert autotune.pick(table) == table[1]


def test_persistent_needs_a_clear_margin():
    plain = _row(0.5, 128, 2, 0, 0.3034)
    pers = _row(0.5, 128, 2, 1, 0.3030)  # faster by 0.13 %: a tie
    assert autotune.pick([plain, pers]) == plain
    pers_fast = _row(0.5, 128, 2, 1, 0.3034 * (1.0 - 2.0 * autotune.TIE))  # faster by 2 %
    assert autotune.pick([plain, pers_fast]) == pers_fast


def test_among_ties_the_fastest_plain_row_wins():
    table = [_row(1.0, 64, 1, 1, 0.3000), _row(0.5, 256, 2, 0, 0.3020), _row(0.5, 128, 2, 0, 0.3010)]
    assert autotune.pick(table) == table[2]


def test_only_persistent_rows():
    table = [_row(1.0, 64, 1, 1, 0.31), _row(0.5, 128, 2, 1, 0.30)]
    assert autotune.pick(table) == table[1]


def test_cached_result_is_returned_without_timing(tmp_path, monkeypatch):
    class S:
        n = 100

        class para:
            h = 0.1

    key = autotune.signature([S()], 4)
    stored = dict(_row(0.5, 128, 2, 0, 0.3), table=[])
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({key: stored}))

    def no_timing(*a, **k):
        raise AssertionError("timed although cached")

    monkeypatch.setattr(autotune, "_time_candidate", no_timing)
    assert autotune.tune([S()], iterations=4, cache_path=str(path)) == stored


def test_dims_for_scale_covers_the_same_extent():
    assert autotune.dims_for_scale([80, 40, 40], 0.5) == [160, 80, 80]
    assert autotune.dims_for_scale([37, 21, 14], 1.0) == [37, 21, 14]
    assert autotune.dims_for_scale([10, 10, 10], 1.0 / 3.0) == [30, 30, 30]
