"""The engine against the reference's own outputs on a B200: the post filters, the morphology
steps and the depth of Match2, bit for bit. The fixtures were dumped from the reference's CUDA build
(ethan-li-coding/FasterStereoCuda compiled for sm_100a) by tests/golden/make_golden.py. Both sides
evaluate the smoothing weights with CUDA's exp on the same GPU, so the smoothed maps must agree
exactly, which the CPU oracle (C library exp) can only show within a tolerance."""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
FILTER = [n for n in ("gauss_only", "bilateral_only", "erosion_only", "open_only", "close_only", "gauss_erosion",
                      "bilateral_close") if (GOLDEN / f"ref_{n}.npz").exists()]
# even-height depth cases: the reference writes every row, so every pixel is compared
DEPTH = [n for n in ("depth_gauss_only", "depth_erosion_only", "depth_gauss_erosion")
         if (GOLDEN / f"ref_{n}.npz").exists()]


def test_fixtures_present():
    assert len(FILTER) == 7 and len(DEPTH) == 3, (FILTER, DEPTH)


def load(name):
    z = dict(np.load(GOLDEN / f"ref_{name}.npz"))
    return z, json.loads(str(z["case"]))


def option(fsc, case):
    return fsc.CuSGMOption(p1=case["p1"], p2_init=case["p2"], cs_type=case["cs_type"], num_paths=4,
                           do_median_filter=bool(case["do_median"]), do_lr_check=bool(case["do_lr_check"]),
                           lr_threshold=case["lr_threshold"], unique_threshold=case["uniqueness"],
                           using_constant_p2=True, do_remove_peaks=bool(case["do_remove_peaks"]),
                           peaks_ratio_threshold=case["peaks_ratio"], post_filter_type=case.get("post_filter", 0),
                           morphology_type=case["morphology"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", FILTER)
def test_filters_match_reference_build(engine_lib, name):
    """StereoCuda::Match with a post filter and/or morphology step (cusgm_df.cu:94-339)."""
    import fasterstereocuda_b200 as fsc
    z, case = load(name)
    W, H = case["width"], case["height"]
    s = fsc.StereoCuda()
    assert s.Init(W, H, case["min_disp"], case["disp_range"], option(fsc, case)), s.last_error()
    disp = np.empty((H, W), np.float32)
    assert s.Match(z["left"], z["right"], disp), s.last_error()
    ref = z["disp_l"]
    neq = disp.view(np.uint32) != ref.view(np.uint32)
    assert int(neq.sum()) == 0, (int(neq.sum()), np.argwhere(neq)[:5])


@pytest.mark.gpu
@pytest.mark.parametrize("name", DEPTH)
def test_match2_depth_matches_reference_build(engine_lib, name):
    """StereoCuda::Init2 / Match2 (StereoCudaImpl.cpp:263-278, :548-583): with exactly one of post
    filter / morphology the depth comes from the map before that step, with both from the final map."""
    import fasterstereocuda_b200 as fsc
    z, case = load(name)
    W, H = case["width"], case["height"]
    c = z["cam"]
    cam = fsc.CamParam(x0_left=c[0], y0_left=c[1], x0_right=c[2], y0_right=c[3], focus=c[4], baseline=c[5])
    s = fsc.StereoCuda()
    assert s.Init2(W, H, case["min_disp"], case["disp_range"], option(fsc, case), cam), s.last_error()
    depth = np.empty((H, W), np.float32)
    assert s.Match2(z["left"], z["right"], depth), s.last_error()
    neq = depth.view(np.uint32) != z["depth"].view(np.uint32)
    assert int(neq.sum()) == 0, (int(neq.sum()), np.argwhere(neq)[:5])
