"""The bench line's whole-step roofline arithmetic (bench.pipeline_roofline)
on fixed numbers: t_roof = max(bytes_alg / HBM, filter atomics / or-rate +
count adds / add-rate), bytes_alg = F + 64 K + 64 (K - L) + L P + R rec, the
L2-resident atomic rates as the design's ceiling, the 4 GiB random-footprint
rates reported beside them, and the host link as the end-to-end bound."""
import importlib.util
import os

import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


PEAKS = {"hbm_copy_gbs": 6000.0, "or_return_gops": 20.0, "red_add_gops": 25.0, "l2_or_return_gops": 100.0,
         "l2_red_add_gops": 200.0, "h2d_gbs": 50.0, "footprint_bytes": 4 << 30, "l2_footprint_bytes": 32 << 20}


def test_pipeline_roofline_terms(bench):
    F, K, L, R, P, rec = 6e9, 2e9, 6e8, 1e8, 8, 16
    r = bench.pipeline_roofline(PEAKS, {"hbm_gbs": 6500.0, "source": "test"}, F, K, L, R, P, rec, 80.0, 50.0)
    p = r["pipeline"]
    bytes_alg = F + 64 * K + 64 * (K - L) + L * P + R * rec
    assert p["bytes_alg"] == bytes_alg and p["atomics_alg"] == 2 * K - L
    t_hbm = bytes_alg / 6500e9 * 1e3
    t_l2 = (K / 100e9 + (K - L) / 200e9) * 1e3
    t_dram = (K / 20e9 + (K - L) / 25e9) * 1e3
    assert p["t_hbm_ms"] == pytest.approx(t_hbm) and p["t_atomic_l2_ms"] == pytest.approx(t_l2)
    assert p["t_atomic_random_4gib_ms"] == pytest.approx(t_dram)
    assert p["t_roof_ms"] == pytest.approx(max(t_hbm, t_l2)) and p["bound"] == "hbm"
    assert p["frac"] == pytest.approx(max(t_hbm, t_l2) / 80.0)
    assert p["frac_random_4gib"] == pytest.approx(max(t_hbm, t_dram) / 80.0)
    assert p["t_roof_e2e_ms"] == pytest.approx(max(t_hbm, t_l2, F / 50e9 * 1e3))
    c = r["count_routed_atomic"]
    assert c["frac"] == pytest.approx(t_l2 / 50.0)


def test_pipeline_roofline_absent_without_peaks(bench):
    assert bench.pipeline_roofline(None, {"hbm_gbs": 1.0, "source": "x"}, 1, 1, 0, 0, 8, 16, 1.0, 1.0) == {}
