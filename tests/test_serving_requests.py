"""The serving stream's host side on the CPU: the request generator (serve.serving_requests) and the summary of a
run (serve.summary).  The C5 stream is Poisson arrivals at a rate, sizes uniform over the mix, Re log-uniform,
half uniform and half regularised lids; the same seed gives the same stream."""
import math

import numpy as np
import pytest

from les_impulse3d_64_b200.serve import SERVING_SIZES, Result, serving_requests, summary


def test_same_seed_same_stream():
    a = serving_requests(50, 50.0, seed=3, t_end=0.2)
    b = serving_requests(50, 50.0, seed=3, t_end=0.2)
    assert [(r.arrival, r.settings, r.t_end, r.seed) for r in a] == [(r.arrival, r.settings, r.t_end, r.seed) for r in b]
    c = serving_requests(50, 50.0, seed=4, t_end=0.2)
    assert [r.arrival for r in a] != [r.arrival for r in c]


def test_stream_follows_its_distributions():
    reqs = serving_requests(4000, 50.0, seed=0, re_range=(100.0, 5000.0), t_end=5.0)
    arrivals = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arrivals) > 0)
    gaps = np.diff(np.concatenate([[0.0], arrivals]))
    assert gaps.mean() == pytest.approx(1 / 50.0, rel=0.05)           # Poisson: mean gap 1 / rate
    assert gaps.std() == pytest.approx(1 / 50.0, rel=0.1)             # exponential gaps: std = mean
    sizes = [(r.settings['nx'], r.settings['ny'], r.settings['nz']) for r in reqs]
    assert set(sizes) == set(SERVING_SIZES)
    for s in SERVING_SIZES:
        assert sizes.count(s) / len(reqs) == pytest.approx(1 / len(SERVING_SIZES), abs=0.03)
    re = np.array([1.0 / r.settings['nu'] for r in reqs])
    assert re.min() >= 100.0 * (1 - 1e-9) and re.max() <= 5000.0 * (1 + 1e-9)
    logs = (np.log(re) - math.log(100.0)) / (math.log(5000.0) - math.log(100.0))
    assert np.mean(logs < 0.5) == pytest.approx(0.5, abs=0.03)       # log-uniform: half below the geometric mean
    uniform = np.mean([r.settings['lid_shaped'] == 0 for r in reqs])
    assert uniform == pytest.approx(0.5, abs=0.03)
    assert all(r.t_end == 5.0 and r.id == k and r.seed == k for k, r in enumerate(reqs))


def test_requests_can_carry_their_noise():
    reqs = serving_requests(3, 50.0, seed=1, t_end=0.1, with_fields=True)
    for r in reqs:
        nx, ny, nz = r.settings['nx'], r.settings['ny'], r.settings['nz']
        v, w = r.fields
        assert v.shape == (nz, ny + 1, nx) and w.shape == (nz + 1, ny, nx)
        assert r.initial_fields(None) is r.fields


def test_summary():
    results = [Result(id=k, cells=1000, arrival=float(k), admitted=float(k), finished=float(k) + 1 + k, steps=10,
                      time=0.2) for k in range(5)]
    s = summary(results)
    tts = [1 + k for k in range(5)]
    assert s['requests'] == 5
    assert s['p50_s'] == pytest.approx(np.percentile(tts, 50))
    assert s['p99_s'] == pytest.approx(np.percentile(tts, 99))
    assert s['mean_s'] == pytest.approx(3.0)
    assert s['span_s'] == pytest.approx(9.0)                          # last finish (4 + 5) minus first arrival
    assert s['cell_updates_per_s'] == pytest.approx(5 * 1000 * 10 / 9.0)
