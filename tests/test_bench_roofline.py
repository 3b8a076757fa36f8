"""The bench's roofline arithmetic on a synthetic per-kernel profile (no GPU): the dominant kernel
is the one with the largest summed time among those with algorithmic bytes, achieved = its
algorithmic bytes over that time, traffic = the ncu bytes per voxel times the voxels of a launch."""
import importlib.util
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


LEVELS = [("init", 1242, 375, 32, 1), ("init", 621, 187, 32, 1), ("plain", 310, 93, 64, 2)]


def test_dominant_kernel_and_achieved_bandwidth(bench):
    prof = {"hpaths_init": {"launches": 4, "ms": 12.0}, "vpaths_bt_init": {"launches": 4, "ms": 20.0},
            "vpaths_wta_init": {"launches": 4, "ms": 8.0}, "census": {"launches": 6, "ms": 4.0}}
    pairs = 512
    r = bench.roofline_of(prof, pairs, LEVELS, lambda k: "batch", 6545.3, "measured", "t")
    # the bottom-to-top pass has no counterpart in the minimal design: not a candidate
    assert r["kernel"] == "hpaths_init"
    per_pair = sum(bench.alg_bytes("hpaths_init", w, h, d, nv, 8) for (k, w, h, d, nv) in LEVELS if k == "init")
    assert per_pair == sum(2 * w * h * d * nv + 16 * w * h * nv for (k, w, h, d, nv) in LEVELS if k == "init")
    assert r["achieved"] == pytest.approx(per_pair * pairs / 12e-3 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / 6545.3)
    assert r["alg_bytes_per_launch"] == pytest.approx(per_pair * pairs / 4)
    assert r["avg_launch_us"] == pytest.approx(3000.0)
    voxels = sum(w * h * d * nv for (k, w, h, d, nv) in LEVELS if k == "init") * pairs
    assert r["traffic"] == pytest.approx(bench.NCU_DRAM_BYTES_PER_VOXEL["batch"]["hpaths_init"] * voxels / 4)


def test_plain_kernels_count_only_plain_levels_and_missing_traffic_is_null(bench):
    prof = {"hpaths_plain": {"launches": 2, "ms": 3.0}, "lr_median": {"launches": 6, "ms": 1.0}}
    r = bench.roofline_of(prof, 2, LEVELS, lambda k: "batch", 6545.3, "measured", "t")
    assert r["kernel"] == "hpaths_plain"
    assert r["alg_bytes_per_launch"] == pytest.approx(bench.alg_bytes("hpaths_plain", 310, 93, 64, 2, 8) * 2 / 2)
    assert r["traffic"] is None  # no ncu figure for this kernel in that family
    assert bench.roofline_of({"vpaths_bt_init": {"launches": 1, "ms": 1.0}}, 1, LEVELS, lambda k: "v4", 1.0, "m",
                             "t") is None
