"""Launch tuning: the per-profile table in the library (round trip, validation, reset), the
autotuner's search and the loading of its file. Without a GPU."""
import json

import pytest

from libgail_b200 import GailError
from libgail_b200 import autotune as AT


def test_round_trip_and_rounding():
    try:
        AT.set_tuning(1, {"soloDecisions": 12000, "cmCtasPerSm": 8, "mqCtasPerSm": 24, "decCtasPerSm": 40,
                          "t1Persistent": 1, "decHeavyPct": 250, "dwtTile1": 1, "dwtTileN": 2})
        t = AT.get_tuning(1)
        assert t == {"soloDecisions": 8192, "cmCtasPerSm": 8, "mqCtasPerSm": 24, "decCtasPerSm": 40,
                     "t1Persistent": 1, "decHeavyPct": 250, "dwtTile1": 1, "dwtTileN": 2}
        assert AT.get_tuning(0) == AT.DEFAULTS  # profiles are independent
    finally:
        AT.set_tuning(1, None)
    assert AT.get_tuning(1) == AT.DEFAULTS


@pytest.mark.parametrize("bad", [{"soloDecisions": 100}, {"cmCtasPerSm": 0}, {"mqCtasPerSm": 65}, {"decCtasPerSm": -1},
                                 {"t1Persistent": 2}, {"decHeavyPct": -1}, {"dwtTile1": 3}, {"dwtTileN": -1}])
def test_invalid_values_refused(bad):
    with pytest.raises(GailError):
        AT.set_tuning(0, dict(AT.DEFAULTS, **bad))
    assert AT.get_tuning(0) == AT.DEFAULTS


def test_profile_out_of_range():
    with pytest.raises(GailError):
        AT.set_tuning(2, AT.DEFAULTS)


def test_coordinate_search_finds_the_minimum():
    target = {"a": 3, "b": 20}
    cost = lambda c: (c["a"] - target["a"]) ** 2 + (c["b"] - target["b"]) ** 2  # noqa: E731
    best, c, seen = AT.coordinate_search({"a": 0, "b": 0}, {"a": [1, 2, 3, 4], "b": [10, 20, 30]}, cost)
    assert best == target and c == 0
    assert len(seen) == 1 + 4 + 3


def test_apply_only_on_the_same_gpu(tmp_path):
    f = tmp_path / "t.json"
    f.write_text(json.dumps({"device": "NVIDIA B200", "profiles": {"4k": dict(AT.DEFAULTS, mqCtasPerSm=12)},
                             "policy": {"maxBatch": 32, "minBatchPct": 10, "maxWaitMs": 2.0}}))
    try:
        assert AT.apply(str(f), device_name="another GPU") == AT.POLICY_DEFAULT
        assert AT.get_tuning(1) == AT.DEFAULTS
        pol = AT.apply(str(f), device_name="NVIDIA B200")
        assert pol["maxBatch"] == 32 and AT.get_tuning(1)["mqCtasPerSm"] == 12
    finally:
        AT.set_tuning(1, None)
