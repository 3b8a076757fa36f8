"""Per-stage timing of the synchronous host API with print_log, the report the reference prints
from its stage timers (SgmStereoCuda/StereoCudaImpl.cpp:365-460): one line per stage with CUDA-event
times, and the same disparities as without the report."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

SCRIPT = r"""
import numpy as np
import fasterstereocuda_b200 as fsc
from fasterstereocuda_b200 import scenes
W, H = 320, 240
L, R, _ = scenes.planar_pair(5, W, H)
opt = fsc.CuSGMOption(p1=10, p2_init=150, cs_type=1, num_paths=4, do_median_filter=True, do_lr_check=True,
                      lr_threshold=1.0, unique_threshold=0.95, using_constant_p2=True, do_remove_peaks=True,
                      peaks_ratio_threshold=0.0005, post_filter_type=1)
quiet, loud = fsc.StereoCuda(), fsc.StereoCuda()
assert quiet.Init(W, H, 0, 64, opt) and loud.Init(W, H, 0, 64, opt, True)
a, b = np.empty((H, W), np.float32), np.empty((H, W), np.float32)
for _ in range(2):
    assert quiet.Match(L, R, a) and loud.Match(L, R, b)
print("SAME", bool(np.array_equal(a.view(np.uint32), b.view(np.uint32))), flush=True)
"""


@pytest.mark.gpu
def test_print_log_reports_every_stage(engine_lib):
    env = dict(os.environ, PYTHONPATH=str(ROOT))
    r = subprocess.run([sys.executable, "-c", SCRIPT], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = r.stdout
    assert "SAME True" in out
    assert out.count("Timing:") == 2
    for stage in ("input", "census", "cost + aggregation + WTA", "left-right check + median",
                  "post filter + morphology", "small-region removal", "output", "total"):
        assert f"** {stage}" in out, stage
