"""CPU checks of the autotuner: the cache file format and round trip, key bucketing, the choice of
the fastest candidate, and that applied values reach the library (rbw_tuning_*), with fake
timings -- no GPU needed."""
import json

import pytest

import rapidbow_b200 as rbw
from rapidbow_b200 import autotune as at


@pytest.fixture(autouse=True)
def _clean():
    at.clear()
    yield
    at.clear()


def test_bucket_and_defaults():
    assert [at.bucket(n) for n in (0, 1, 2, 3, 4, 1023, 1024, 10_000_000)] == [0, 0, 1, 1, 2, 9, 10, 23]
    for name, value in at.DEFAULTS.items():
        assert at.get_value(name, 16, 4, 10_000_000) == value


def test_choose_fastest_smallest_on_ties():
    assert at.choose({8: 3.0, 16: 2.0, 32: 2.5}) == 16
    assert at.choose({4: 1.0, 2: 1.0, 6: 1.5}) == 2


def test_tune_records_applies_and_round_trips(tmp_path):
    path = str(tmp_path / "cache.json")
    t = at.Autotuner("NVIDIA B200", 148, path)
    fake = {2: 1.9, 3: 1.2, 4: 1.1, 5: 1.3, 6: 1.4, 7: 1.5, 8: 1.6}
    calls = []

    def measure():
        v = at.get_value("assign_ctas_per_sm", 10, 0, 10_000_000)  # the value set for this trial
        calls.append(v)
        return fake[v]

    e = t.tune("assign_ctas_per_sm", 10, 0, 10_000_000, measure)
    assert calls == [2, 3, 4, 5, 6, 7, 8]
    assert e["value"] == 4 and e["bucket"] == 23 and e["default_ms"] == 1.4
    assert at.get_value("assign_ctas_per_sm", 10, 0, 9_000_000) == 4       # same bucket
    assert at.get_value("assign_ctas_per_sm", 10, 0, 1 << 24) == 6          # next bucket: default
    assert at.get_value("assign_ctas_per_sm", 10, 6, 10_000_000) == 4       # L = 0 matches any depth
    t.record("scatter_rows", 16, 4, 10_000_000, {8: 0.05, 16: 0.04, 32: 0.06})
    t.save()
    d = json.load(open(path))
    assert d["format"] == at.FORMAT and d["version"] == 1 and d["device"] == {"name": "NVIDIA B200", "sms": 148}
    assert {e["param"] for e in d["entries"]} == {"assign_ctas_per_sm", "scatter_rows"}
    at.clear()
    assert at.get_value("assign_ctas_per_sm", 10, 0, 10_000_000) == 6
    t2 = at.Autotuner("NVIDIA B200", 148, path)
    assert t2.load() and t2.apply() == 2
    assert at.get_value("assign_ctas_per_sm", 10, 0, 10_000_000) == 4
    assert at.get_value("scatter_rows", 16, 4, 10_000_000) == 16
    # a cache written for another device is not used
    assert not at.Autotuner("NVIDIA H100", 132, path).load()
    # re-recording a key replaces its entry
    t2.record("scatter_rows", 16, 4, 10_000_000, {8: 0.01, 16: 0.04, 32: 0.06})
    assert len(t2.entries) == 2 and at.get_value("scatter_rows", 16, 4, 10_000_000) == 8


def test_library_rejects_bad_values():
    with pytest.raises(rbw.RbwError) as e:
        at.set_value("scatter_rows", 16, 4, 20, 12)
    assert e.value.status == rbw.RBW_ERR_INVALID_ARG
    with pytest.raises(rbw.RbwError):
        at.set_value("assign_ctas_per_sm", 16, 0, 20, 9)
    with pytest.raises(rbw.RbwError):
        at.set_value("assign_f32_ctas_per_sm", 1, 0, 20, 2)  # branch factor out of range
    at.set_value("scatter_rows", 16, 4, 20, 32)
    assert at.get_value("scatter_rows", 16, 4, 1 << 20) == 32
    at.set_value("scatter_rows", 16, 4, 20, 0)  # 0 removes the entry
    assert at.get_value("scatter_rows", 16, 4, 1 << 20) == 16
