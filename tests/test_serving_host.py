"""Host-side pieces of the serving benchmark (no GPU): Poisson arrivals and latency percentiles."""
import numpy as np
import pytest

from open_source_einstar_b200.serving import latency_summary, poisson_arrivals


@pytest.mark.parametrize("rate", [120.0, 240.0, 480.0])
def test_poisson_arrivals_rate_and_order(rate):
    t = poisson_arrivals(rate, 20.0, seed=7)
    assert np.all(np.diff(t) > 0) and t[0] >= 0 and t[-1] < 20.0
    # count over 20 s is Poisson(20 * rate): within 5 standard deviations
    assert abs(len(t) - 20 * rate) < 5 * np.sqrt(20 * rate)
    gaps = np.diff(t)
    assert abs(gaps.mean() - 1 / rate) < 0.1 / rate
    # exponential gaps: coefficient of variation near 1
    assert 0.9 < gaps.std() / gaps.mean() < 1.1
    assert np.array_equal(t, poisson_arrivals(rate, 20.0, seed=7))


def test_latency_summary_percentiles():
    lat = np.arange(1, 1001, dtype=np.float64) / 100.0  # 0.01 .. 10 ms
    s = latency_summary(lat, wall_s=2.0)
    assert s["frames"] == 1000 and s["fps"] == 500.0
    assert s["p50_ms"] == pytest.approx(np.percentile(lat, 50))
    assert s["p99_ms"] == pytest.approx(np.percentile(lat, 99))
    assert s["p999_ms"] == pytest.approx(np.percentile(lat, 99.9))
    assert s["max_ms"] == 10.0
    assert latency_summary([], 1.0)["frames"] == 0
