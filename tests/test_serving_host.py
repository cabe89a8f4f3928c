"""Host logic of the serving loop and the ensembles (no GPU): the seeded request stream, the FIFO sequential baseline and
the device footprint used for admission."""
import math

import numpy as np

from conftest import PKG  # noqa: F401  (puts the package on sys.path)


def test_poisson_stream_seeded_and_in_range():
    from isw.serving import poisson_requests
    a = poisson_requests(400, 50.0, seed=3)
    b = poisson_requests(400, 50.0, seed=3)
    assert [(r.arrival, r.level, r.days, r.layers) for r in a] == [(r.arrival, r.level, r.days, r.layers) for r in b]
    t = np.array([r.arrival for r in a])
    assert np.all(np.diff(t) > 0)
    assert abs(len(a) / t[-1] - 50.0) < 10.0                  # rate 50 per second
    assert {r.level for r in a} == {4, 5, 6, 7} and {r.layers for r in a} == {3, 5}
    d = np.array([r.days for r in a])
    assert d.min() >= 1.0 and d.max() <= 30.0
    assert abs(np.median(np.log(d)) - 0.5 * math.log(30.0)) < 0.4   # log-uniform


def test_sequential_baseline_fifo():
    from isw.serving import Request, sequential_baseline
    reqs = [Request(0, 0.0, 4, 1.0, 3), Request(1, 0.5, 4, 1.0, 3), Request(2, 10.0, 4, 1.0, 3)]
    out = sequential_baseline(reqs, {(4, 3): 0.01}, lambda r: (100, 1.0))   # 1 s of service each
    # completions at 1.0, 2.0 (waits for the first), 11.0 (idle until its arrival)
    lat = sorted([1.0, 1.5, 1.0])
    assert math.isclose(out['p50_s'], float(np.percentile(lat, 50)))
    assert math.isclose(out['wall_s'], 11.0)
    assert math.isclose(out['member_days_per_s'], 1.0)


def test_footprint_grows_with_level_and_layers():
    from isw.workload import stack_bytes

    class G:
        def __init__(self, n):
            self.N = 10 * 4 ** n + 2
            self.E = 3 * (self.N - 2)
            self.NV = 2 * (self.N - 2)
    f = {(n, L, m): stack_bytes(G(n), L, 2, m) for n in (4, 7) for L in (2, 3) for m in (False, True)}
    assert f[(7, 3, True)] > f[(7, 3, False)] > f[(4, 3, False)]
    assert f[(7, 3, False)] > f[(7, 2, False)]
    assert 300e6 < f[(7, 3, True)] < 600e6                     # a level-7 air stack: a few hundred MB
