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


def test_stage_rooflines(bench):
    """Per-stage algorithmic bytes: the windowed count (a subroute stage ran)
    moves keys, first occurrences and table cells; without windows the count
    is charged the workload definition's 64 B per k-mer + 64 B per repeat."""
    stats = {"total_kmers": 2_000, "low_records": 600, "root_records": 100, "table_slots": 1_000}
    ms = {"extract_scatter": 2.0, "subroute": 1.0, "count": 4.0, "pack_low": 0.5}
    r = bench.stage_rooflines(ms, stats, 6_000, 31, 1.0, 8, 16)
    assert r["extract_scatter"]["alg_bytes"] == 6_000 + 8 * 2_000
    assert r["subroute"]["alg_bytes"] == 2 * 8 * 2_000
    assert r["count"]["alg_bytes"] == 8 * 2_000 + 8 * 600 + int(2 * 16 * 1_000 * 9 / 8)
    assert r["pack_low"]["alg_bytes"] == 8 * 600 + 8 * 600
    assert r["count"]["gbs"] == pytest.approx(r["count"]["alg_bytes"] / 4e-3 / 1e9)
    r2 = bench.stage_rooflines({"count": 4.0, "init": 1.0, "export": 1.0}, dict(stats, filter_words=300), 6_000, 63,
                               1.0, 16, 24)
    assert r2["count"]["alg_bytes"] == 64 * 2_000 + 64 * 1_400 and r2["count"]["rule"].startswith("64 K")
    # 128-bit keys: 32-byte slots, and a filter of its own to initialise
    assert r2["init"]["alg_bytes"] == 32 * 1_000 + 8 * 300
    assert r2["export"]["alg_bytes"] == 32 * 1_000 + 24 * 100


def test_profiled_traffic_keyed_by_kernel_sources(bench):
    """Measured DRAM traffic is reported only for the genome-scale workload at
    full size and only while the kernel sources hash to the captured sha256;
    any other sources give null traffic with the reason."""
    class A:
        workload, scale = "genome_scale", 1.0
    stages = bench.PROFILED_TRAFFIC["genome_scale"]
    assert set(stages) == set(bench.STAGE_KERNELS)
    real = bench.kernel_sources_sha256
    try:
        bench.kernel_sources_sha256 = lambda: bench._CAPTURE_SHA
        for s, e in stages.items():
            b, note = bench.profile_traffic(A, s)
            assert b == e["bytes_per_step"] > 0 and "capture" in note
        bench.kernel_sources_sha256 = lambda: "0" * 64
        assert bench.profile_traffic(A, "count") == (None, "kernel sources changed since the last capture")
    finally:
        bench.kernel_sources_sha256 = real
    A.scale = 0.5
    assert bench.profile_traffic(A, "count")[0] is None
    A.scale, A.workload = 1.0, "large_long"
    assert bench.profile_traffic(A, "count")[0] is None

