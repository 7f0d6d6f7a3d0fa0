"""kc_measure_peaks on the GPU: every figure is measured and plausible for a
B200-class device (HBM copy in TB/s, random atomics in 10^9/s, a PCIe/C2C
link in GB/s), and the calling thread's current device is left unchanged."""
import pytest

pytestmark = pytest.mark.gpu

kc = pytest.importorskip("kmertreecounter_b200")


def test_measure_peaks_small_footprint():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    p = kc.measure_peaks(0, 512 << 20)
    assert p["footprint_bytes"] == 512 << 20 and p["ops"] == (512 << 20) // 4
    assert 1000 < p["hbm_copy_gbs"] < 20000
    assert 1 < p["red_add_gops"] < 1000 and 1 < p["or_return_gops"] < 1000
    assert 1 < p["h2d_gbs"] < 1000
    assert p["l2_footprint_bytes"] == 32 << 20 and 1 < p["l2_red_add_gops"] < 10000 and 1 < p["l2_or_return_gops"] < 10000
    assert torch.cuda.current_device() == 0
