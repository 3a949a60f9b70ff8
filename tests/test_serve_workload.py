"""Host side of the serving benchmark (CPU): the seeded arrival schedule follows the configured mix,
and the latency summary computes its percentiles, class and throughput as documented."""
import math

import numpy as np

from diff_envshade_b200 import serve_workload as sw


def test_schedule_is_seeded_and_follows_the_mix():
    a = sw.make_schedule(n=20000, rate=5000.0, seed=7)
    assert a == sw.make_schedule(n=20000, rate=5000.0, seed=7)
    assert a != sw.make_schedule(n=20000, rate=5000.0, seed=8)
    t = np.array([r["t"] for r in a])
    assert np.all(np.diff(t) > 0)
    assert abs(np.mean(np.diff(t)) * 5000.0 - 1.0) < 0.03           # Poisson, 5000 per second
    P = np.array([r["P"] for r in a])
    assert P.min() >= 1000 and P.max() <= sw.MAX_P
    mid = math.exp(0.5 * (math.log(1000) + math.log(sw.MAX_P)))    # log-uniform: median at the log-midpoint
    assert abs(np.median(P) / mid - 1.0) < 0.05
    for key, value, frac in (("res", (32, 64), 0.5), ("vis", True, 0.5), ("backward", True, 0.3)):
        got = np.mean([r[key] == value for r in a])
        assert abs(got - frac) < 0.02, (key, got)


def test_summary_percentiles_class_and_throughput():
    sched = [dict(P=60000, res=(16, 32), backward=False), dict(P=60000, res=(32, 64), backward=False),
             dict(P=120000, res=(16, 32), backward=True), dict(P=99999, res=(16, 32), backward=True)]
    lat_s = [0.001, 0.004, 0.002, 0.003]
    out = sw._summarize(lat_s, sched, makespan_s=0.5)
    assert out["requests"] == 4
    assert math.isclose(out["p50_ms"], 2.5) and math.isclose(out["max_ms"], 4.0)
    assert math.isclose(out["p99_ms"], np.percentile([1, 4, 2, 3], 99))
    cls = out["class_50k_100k_16x32"]                              # requests 0 and 3 only
    assert cls["n"] == 2 and math.isclose(cls["p50_ms"], 2.0)
    pairs = 60000 * 512 + 60000 * 2048 + 2 * 120000 * 512 + 2 * 99999 * 512
    assert math.isclose(out["throughput_point_texel_per_s"], pairs / 0.5)
    assert math.isclose(out["throughput_req_per_s"], 8.0)
