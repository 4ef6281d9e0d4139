"""The mixed-serving driver's request draw (without a GPU): the kind and profile shares and
the Poisson arrivals follow the specified mix, and a seed gives the same requests."""
import numpy as np

from libgail_b200 import serve_mix as SM


def test_shares_and_determinism():
    n = 200000
    kinds, prof, picks = SM.draw(n, seed=3)
    assert abs(kinds.mean() - 0.7) < 0.01
    counts = np.bincount(prof, minlength=len(SM.PROFILES)) / n
    for share, got in zip([p[3] for p in SM.PROFILES], counts):
        assert abs(share - got) < 0.01
    assert picks.min() >= 0 and picks.max() < SM.FRAMES_PER_PROFILE
    k2, p2, c2 = SM.draw(n, seed=3)
    assert np.array_equal(kinds, k2) and np.array_equal(prof, p2) and np.array_equal(picks, c2)


def test_poisson_arrivals():
    a = SM.arrivals(100000, 250.0, seed=5)
    assert np.all(np.diff(a) > 0)
    assert abs(len(a) / a[-1] - 250.0) < 5.0  # mean rate
    gaps = np.diff(a)
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.05  # exponential gaps


def test_percentiles_empty_and_values():
    assert SM.percentiles([]) == {"requests": 0}
    r = SM.percentiles(list(range(1, 101)))
    assert r["requests"] == 100 and 50 <= r["p50_ms"] <= 51 and r["p99_ms"] >= 99
