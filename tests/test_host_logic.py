"""Host-side logic of the served measurement (sgtsne_b200.multi), on CPU: the
plain form's latencies under an arrival stream (one FIFO server running the
requests one at a time) and the reported percentiles."""
import numpy as np


def test_fifo_latencies_queue_behind_earlier_requests():
    from sgtsne_b200 import multi as M
    arrivals = np.array([0.0, 1.0, 1.5, 10.0])
    service = np.array([2.0, 1.0, 1.0, 0.5])
    # finishes at 2, 3, 4 (queued behind the first two), then 10.5 (idle server)
    lat = M.fifo_latencies(arrivals, service)
    assert np.allclose(lat, [2.0, 2.0, 2.5, 0.5])


def test_fifo_latencies_never_below_service_time():
    from sgtsne_b200 import multi as M
    rng = np.random.default_rng(4)
    arrivals = np.cumsum(rng.exponential(0.2, 200))
    service = rng.uniform(0.05, 0.5, 200)
    lat = M.fifo_latencies(arrivals, service)
    assert np.all(lat >= service - 1e-12)
    # work conservation: the last request ends no earlier than the total work
    assert arrivals[-1] + lat[-1] >= service.sum() - 1e-9


def test_percentiles():
    from sgtsne_b200 import multi as M
    lat = np.arange(1, 101, dtype=float)
    p = M.percentiles(lat)
    assert abs(p["p50_s"] - 50.5) < 1e-12
    assert abs(p["p99_s"] - 99.01) < 1e-9
    assert abs(p["mean_s"] - 50.5) < 1e-12
