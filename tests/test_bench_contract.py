"""Host-side pieces of bench.py's JSON line that need no GPU: the algorithmic
bytes behind roofline.achieved, the committed ncu traffic figures behind
roofline.traffic, and the peak behind roofline.peak."""
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_algorithmic_bytes():
    import bench
    n, g = 262143, 144 ** 3
    assert bench.algorithmic_bytes("gather", "mixed") == n * 16 + g * 4 + n * 24 == 22429656
    assert bench.algorithmic_bytes("spread", "mixed") == n * 16 + g * 4
    assert bench.algorithmic_bytes("gather", "fp64") == n * 32 + g * 8 + n * 24
    with pytest.raises(ValueError):
        bench.algorithmic_bytes("fft", "mixed")


def test_algorithmic_flops():
    """The spread's 13^3 points x 2 flops and the gather's 704.5 in-sphere points
    x 8 flops per atom (the gather's mean point count, checked here against the
    reference's sphere test on seeded atom offsets)."""
    import numpy as np
    import bench
    n = 262143
    assert bench.algorithmic_flops("spread") == n * 2197 * 2
    assert bench.algorithmic_flops("gather") == n * 704.5 * 8
    rng = np.random.default_rng(4)
    h, rc = 140.0 / 144, 3.0 * np.sqrt(2.0) * 2.0 * np.sqrt(0.4)
    k = np.arange(13) - 6
    cnt = []
    for _ in range(300):
        d = [(k - o) * h for o in rng.uniform(-0.5, 0.5, 3)]
        r2 = d[0][None, None, :] ** 2 + d[1][None, :, None] ** 2 + d[2][:, None, None] ** 2
        cnt.append((r2 < rc * rc).sum())
    assert abs(np.mean(cnt) - bench.GATHER_POINTS_PER_ATOM) < 5.0
    with pytest.raises(ValueError):
        bench.algorithmic_flops("fft")


def test_traffic_file_has_the_dominant_kernels():
    """bench.py reads 'kernel precision bytes' lines; the gather's cold-cache
    DRAM bytes stay below its algorithmic bytes (nothing re-read)."""
    import bench
    got = {}
    with open(os.path.join(ROOT, "profiles", "traffic_water262k.txt")) as fh:
        for ln in fh:
            parts = ln.split()
            if len(parts) == 3 and not ln.startswith("#"):
                got[(parts[0], parts[1])] = int(parts[2])
    assert set(got) >= {("gather", "mixed"), ("spread", "mixed")}
    assert 0 < got[("gather", "mixed")] <= bench.algorithmic_bytes("gather", "mixed")
    assert got[("spread", "mixed")] > 0


def test_peak_comes_from_the_measured_file_when_present():
    import bench
    peak, kind = bench.hbm_peak()
    if os.path.exists(bench.PEAKS_FILE):
        with open(bench.PEAKS_FILE) as f:
            assert peak == float(json.load(f)["hbm_gbs"]) and kind == "measured"
    else:
        assert (peak, kind) == (bench.FALLBACK_HBM_GBS, "fallback")
