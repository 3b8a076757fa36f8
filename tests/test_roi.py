"""Matching with regions of interest (StereoCuda::Match / Match2 with StereoROI_T) against the
oracle, bit for bit. A view's region is matched as its own sub-image: its paths start at the
region's edges (the reference's xoffset / xEnd / yoffset / yend, SgmStereoCuda/cusgm_ca.cu:
3991-3999), its WTA covers floor(h/2)*2 rows from the region's y (:4139-4165), everything outside
is INVALID, and small-region removal runs in strips of the region's rows
(SgmStereoCuda/StereoCudaImpl.cpp:463-498). The oracle's ROI restatement is pinned to the
reference's own ROI dumps in tests/test_golden_reference.py."""
import numpy as np
import pytest

from fasterstereocuda_b200 import scenes

INV = np.float32(-999999.0)
STRIPS = 6

CASES = {
    # name: (W, H, M, D, cs, lr, median, peaks, roi_l, roi_r, seed)
    "d64_9x7_both": (162, 120, 0, 64, 1, 1, 1, 0, (20, 16, 100, 80), (8, 10, 120, 90), 41),
    "d64_5x5_odd": (162, 120, 0, 64, 0, 1, 1, 0, (12, 5, 137, 99), (3, 7, 141, 101), 42),
    "d32_left_only": (150, 90, 0, 32, 1, 1, 1, 0, (30, 11, 90, 60), None, 43),
    "d128": (300, 96, 0, 128, 1, 1, 0, 0, (100, 20, 180, 64), (0, 0, 300, 96), 44),
    "min_disp_clip": (130, 100, 8, 64, 1, 1, 1, 0, (2, 3, 120, 90), (4, 4, 100, 80), 45),
    "peaks_in_roi": (200, 150, 0, 64, 1, 0, 1, 1, (10, 17, 180, 121), None, 46),
    "whole_image": (162, 120, 0, 64, 1, 1, 1, 0, (0, 0, 162, 120), (0, 0, 162, 120), 47),
}


def option(fsc, cs, lr, med, peaks):
    p1, p2 = (10, 150) if cs else (8, 32)
    return fsc.CuSGMOption(p1=p1, p2_init=p2, cs_type=cs, num_paths=4, do_median_filter=bool(med),
                           do_lr_check=bool(lr), lr_threshold=1.0, unique_threshold=0.95, using_constant_p2=True,
                           do_remove_peaks=bool(peaks), peaks_ratio_threshold=0.005)


def roi(fsc, r):
    return None if r is None else fsc.StereoROI(*r)


def config(O, W, H, M, D, cs, lr, med, peaks, rl, rr):
    p1, p2 = (10, 150) if cs else (8, 32)
    c = O.Config(width=W, height=H, min_disp=M, disp_range=D, cs_type=cs, p1=p1, p2=p2, do_lr_check=lr,
                 do_median=med, do_remove_peaks=peaks, peaks_ratio=0.005, peaks_strips=STRIPS)
    return c.with_roi(rl, rr if lr else None)


def same(name, a, b):
    neq = a.view(np.uint32) != b.view(np.uint32)
    assert int(neq.sum()) == 0, (name, int(neq.sum()), np.argwhere(neq)[:5])


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("lanes", [(0, 0), (1, 1), (8, 8), (2, 2)])
def test_roi_parity(engine_lib, oracle_mod, name, lanes):
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H, M, D, cs, lr, med, peaks, rl, rr, seed = CASES[name]
    if D == 128 and lanes[0] in (1, 8):
        pytest.skip("128 disparities take 2 or 4 lanes per scanline")
    L, R, _ = scenes.planar_pair(seed, W, H, dmin=2.0, dmax=min(60.0, D - 4.0))
    s = fsc.StereoCuda()
    assert s.Init(W, H, M, D, option(fsc, cs, lr, med, peaks)), s.last_error()
    assert s.set_ext_options(fsc.ExtOptions(peaks_strips=STRIPS))
    if lanes != (0, 0):
        assert s.set_tuning(fsc.Tuning(0, 0, 0, 0, 0, *lanes)), s.last_error()
    disp = np.empty((H, W), np.float32)
    disp_r = np.empty((H, W), np.float32)
    assert s.Match(L, R, disp, disp_r if lr else None, None, roi(fsc, rl), roi(fsc, rr)), s.last_error()
    want = O.match(config(O, W, H, M, D, cs, lr, med, peaks, rl, rr), L, R, dump=True, want_right=True)
    # the region's path volumes (stored compactly, the region's rows and columns only)
    x0, y0 = max(rl[0], max(0, M)), rl[1]
    w, h = rl[0] + rl[2] - x0, rl[3]
    for tag, k in (("lr", 1), ("rl", 3), ("bt", 2)):
        got = s.debug_read(tag).reshape(-1)[:h * w * D].reshape(h, w, D)
        assert np.array_equal(got, want["paths"][k][y0:y0 + h, x0:x0 + w]), tag
    same("wta left", s.debug_read("wta", 0), want["wta_l"])
    if lr:
        same("wta right", s.debug_read("wta", 1), want["wta_r"])
        same("disp right", disp_r, want["disp_r"])
    same("disp left", disp, want["disp"])
    outside = np.ones((H, W), bool)
    outside[rl[1]:rl[1] + rl[3], rl[0]:rl[0] + rl[2]] = False
    assert (disp[outside] == INV).all()
    assert (disp[~outside] != INV).mean() > 0.3


@pytest.mark.gpu
def test_roi_covering_the_image_equals_a_plain_match(engine_lib):
    """An ROI equal to the view's default region gives the match without an ROI."""
    import fasterstereocuda_b200 as fsc
    W, H = 162, 120
    L, R, _ = scenes.planar_pair(48, W, H)
    s = fsc.StereoCuda()
    assert s.Init(W, H, 0, 64, option(fsc, 1, 1, 1, 0)), s.last_error()
    a, b = np.empty((H, W), np.float32), np.empty((H, W), np.float32)
    assert s.Match(L, R, a)
    r = fsc.StereoROI(0, 0, W, H)
    assert s.Match(L, R, b, None, None, r, r), s.last_error()
    same("whole-image ROI", b, a)


@pytest.mark.gpu
def test_match2_with_roi(engine_lib, oracle_mod):
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 200, 150
    L, R, _ = scenes.planar_pair(49, W, H)
    cam = dict(x0_left=600.0, y0_left=180.0, x0_right=610.0, y0_right=180.0, focus=720.0, baseline=540.0)
    s = fsc.StereoCuda()
    assert s.Init2(W, H, 0, 64, option(fsc, 1, 1, 1, 0), fsc.CamParam(**cam)), s.last_error()
    rl, rr = (16, 20, 160, 100), (10, 20, 170, 100)
    depth = np.empty((H, W), np.float32)
    assert s.Match2(L, R, depth, None, fsc.StereoROI(*rl), fsc.StereoROI(*rr)), s.last_error()
    d = O.match(config(O, W, H, 0, 64, 1, 1, 1, 0, rl, rr), L, R)["disp"]
    same("depth", depth, O.depth_from_disp(d, cam["x0_left"], cam["x0_right"], cam["focus"], cam["baseline"]))


@pytest.mark.gpu
def test_roi_errors_on_device(engine_lib):
    import fasterstereocuda_b200 as fsc
    W, H = 64, 48
    img = np.zeros((H, W), np.uint8)
    d = np.zeros((H, W), np.float32)
    s = fsc.StereoCuda()
    assert s.Init(W, H, 8, 32, option(fsc, 1, 1, 1, 0)), s.last_error()
    for r in ((-1, 0, 10, 10), (0, 0, 65, 10), (0, 40, 10, 9), (0, 0, 0, 5), (0, 0, 8, 8)):
        assert not s.Match(img, img, d, None, None, fsc.StereoROI(*r)) and s.status == -1, r
    init = np.zeros((H, W), np.int16)
    assert not s.Match(img, img, d, None, init, fsc.StereoROI(8, 0, 20, 20)) and s.status == -4
    big = fsc.StereoCuda()
    o = option(fsc, 1, 1, 1, 0)
    o.p2_init = 20000
    assert big.Init(W, H, 0, 32, o)
    assert not big.Match(img, img, d, None, None, fsc.StereoROI(0, 0, 20, 20)) and big.status == -4
