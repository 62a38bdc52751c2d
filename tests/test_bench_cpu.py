"""bench.py's host-side arithmetic on CPU: the byte model behind the roofline,
the per-particle traffic the profiles supply, the peak it divides by, and the
whole-job rate of N replicas."""

import json

import pytest

import bench


def test_algorithmic_bytes_of_the_128_cubed_dam_break():
    n, cells = 56_623_104, 128 ** 3
    assert bench.algorithmic_bytes("g2p_advect", n, cells, 22) == 49 * n
    assert bench.algorithmic_bytes("p2g", n, cells, 22) == 25 * n + 32 * cells
    assert bench.algorithmic_bytes("sort", n, cells, 22) == 70 * n
    assert bench.algorithmic_bytes("solve", n, cells, 0) == bench.algorithmic_bytes("solve", n, cells, 1)
    assert bench.algorithmic_bytes("forces", n, cells, 22) is None


def test_traffic_per_unit_covers_the_roofline_stages():
    t = bench.load_traffic()
    for stage in ("g2p_advect", "p2g"):
        b = t[stage]["bytes_per_particle"]
        # at least the 16 B position stream read once; far below the gathered L1 traffic
        assert 16 <= b < 200, (stage, b)


def test_peak_is_measured_when_the_file_exists(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "REPO", str(tmp_path))
    assert bench.peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6551.4}))
    assert bench.peaks() == (6551.4, "measured")


@pytest.mark.parametrize("world", [1, 2, 8])
def test_job_rate_counts_every_replica_at_the_slowest_rank(world):
    assert bench.job_rate(world, 12.5) == pytest.approx(world * 80.0)
