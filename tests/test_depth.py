"""Depth output (StereoCuda::Init2 / Match2, FasterStereoCuda::Init2 / Match2) against the oracle:
the engine's depth maps are compared bit for bit with the oracle's disparity maps turned into depth
by the reference's formula (SgmStereoCuda/cusgm_util.cu:7-34), and the pyramid's coarsest disparity
range with the reference's depth-to-disparity rules (FasterStereoCuda/FasterStereoCuda.cpp:370-395)."""
import numpy as np
import pytest

from fasterstereocuda_b200 import scenes

INV = np.float32(-999999.0)
STRIPS = 6
CAM = dict(x0_left=600.0, y0_left=180.0, x0_right=610.0, y0_right=180.0, focus=720.0, baseline=540.0)


def test_depth_formula_restatement(oracle_mod):
    """CPU: the oracle's depth is (float)((baseline*focus) / ((double)d + (x0_right - x0_left)))."""
    O = oracle_mod
    d = np.array([[0.0, 1.5, 63.25], [INV, -3.0, 7.0]], np.float32)
    got = O.depth_from_disp(d, 600.0, 610.0, 720.0, 540.0)
    for (i, j), v in np.ndenumerate(d):
        want = INV if v == INV else np.float32((540.0 * 720.0) / (float(v) + (610.0 - 600.0)))
        assert got[i, j].tobytes() == np.float32(want).tobytes()
    # d = -(x0_right - x0_left): division by zero gives inf as in IEEE double
    assert np.isinf(O.depth_from_disp(np.array([-10.0], np.float32), 600.0, 610.0, 720.0, 540.0)[0])


def test_pyramid_depth_range_rules(oracle_mod):
    """CPU: coarsest-level range from a depth range (power of two >= 64 above the span, halved once
    above twice the width, minimum pulled back from the width)."""
    O = oracle_mod
    # span 17.8 at scale 4 -> 64; floor(-0.88) = -1
    assert O.pyr_init2_coarsest(1242, 3, 5000.0, 60000.0, 600.0, 610.0, 720.0, 540.0) == (-1, 64)
    # one level, near range: span ~ 388 -> 512
    assert O.pyr_init2_coarsest(1242, 1, 1000.0, 60000.0, 600.0, 610.0, 720.0, 540.0) == (-4, 512)
    # narrow image: 512 > 2 * 200 -> 256
    assert O.pyr_init2_coarsest(200, 1, 1000.0, 60000.0, 600.0, 610.0, 720.0, 540.0) == (-4, 256)
    # minimum past the width: width - range (1024 after halving), but not below -width
    assert O.pyr_init2_coarsest(100, 1, 100.0, 200.0, 600.0, 610.0, 720.0, 540.0) == (-100, 1024)


@pytest.mark.gpu
@pytest.mark.parametrize("peaks", [False, True])
def test_match2_depth_is_depth_of_the_disparity(engine_lib, oracle_mod, peaks):
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 450, 375
    L, R, _ = scenes.planar_pair(61, W, H)
    s = fsc.StereoCuda()
    opt = fsc.CuSGMOption(p1=10, p2_init=150, cs_type=1, num_paths=4, do_median_filter=True, do_lr_check=True,
                          lr_threshold=1.0, unique_threshold=0.95, using_constant_p2=True,
                          do_remove_peaks=peaks, peaks_ratio_threshold=0.0005)
    assert s.Init2(W, H, 0, 64, opt, fsc.CamParam(**CAM)), s.last_error()
    assert s.set_ext_options(fsc.ExtOptions(peaks_strips=STRIPS))
    depth = np.empty((H, W), np.float32)
    assert s.Match2(L, R, depth), s.last_error()
    disp = O.match(O.Config(width=W, height=H, disp_range=64, do_remove_peaks=int(peaks), peaks_strips=STRIPS),
                   L, R)["disp"]
    want = O.depth_from_disp(disp, CAM["x0_left"], CAM["x0_right"], CAM["focus"], CAM["baseline"])
    assert np.array_equal(depth.view(np.uint32), want.view(np.uint32)), int((depth != want).sum())
    assert (depth != INV).mean() > 0.3
    # Match2 without Init2 is refused
    t = fsc.StereoCuda()
    assert t.Init(W, H, 0, 64, opt)
    assert not t.Match2(L, R, depth) and t.status == -2


@pytest.mark.gpu
@pytest.mark.parametrize("layers", [2, 3])
def test_pyramid_init2_match2(engine_lib, oracle_mod, layers):
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 1242, 375
    L, R, _ = scenes.kitti_like(43, W, H)
    epi = fsc.EpipolarStereoParam(x0_left=CAM["x0_left"], y0_left=CAM["y0_left"], x0_right=CAM["x0_right"],
                                  y0_right=CAM["y0_right"], baseline=CAM["baseline"], focus=CAM["focus"])
    opt = fsc.StereoOption2(width=W, height=H, min_depth=5000.0, max_depth=60000.0, num_layers=layers,
                            do_lr_check=True, do_rm_peaks=True, epi=epi)
    p = fsc.FasterStereoCuda()
    assert p.Init2(opt, fsc.LevelOverride(cs_type=1, p1=10, p2=150), fsc.ExtOptions(peaks_strips=STRIPS)), \
        p.last_error()
    m0, d0 = O.pyr_init2_coarsest(W, layers, 5000.0, 60000.0, CAM["x0_left"], CAM["x0_right"], CAM["focus"],
                                  CAM["baseline"])
    assert p.level_info(layers - 1)[2:] == (m0, d0)
    # the same pyramid expressed by its full-resolution disparity range, as the oracle takes it
    scale = 2 ** (layers - 1)
    pc = O.PyrConfig(width=W, height=H, min_disp=m0 * scale, max_disp=(m0 + d0) * scale, num_layers=layers,
                     override_enable=1, cs_type=1, p1=10, p2=150, peaks_strips=STRIPS)
    for lvl in range(layers):
        c = O.pyr_level_config(pc, lvl)
        assert p.level_info(lvl) == (c.width, c.height, c.min_disp, c.disp_range)
    depth = np.empty((H, W), np.float32)
    assert p.Match2(L, R, depth), p.last_error()
    want = O.depth_from_disp(O.pyr_match(pc, L, R), CAM["x0_left"], CAM["x0_right"], CAM["focus"],
                             CAM["baseline"])
    assert np.array_equal(depth.view(np.uint32), want.view(np.uint32)), int((depth != want).sum())
    assert (depth != INV).mean() > 0.3


@pytest.mark.gpu
@pytest.mark.parametrize("pf,morph", [(1, 0), (0, 1), (2, 4)])
def test_match2_depth_source_rule(engine_lib, oracle_mod, pf, morph):
    """StereoCudaImpl::Match2 (StereoCudaImpl.cpp:548-583) reads the aggregator's buffer: with
    exactly one of post filter / morphology (and no small-region removal) that holds the map before
    the step; after both, the morphology result (cusgm_df.cu:275-339)."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 450, 376
    L, R, _ = scenes.planar_pair(62, W, H)
    opt = fsc.CuSGMOption(p1=10, p2_init=150, cs_type=1, num_paths=4, do_median_filter=True, do_lr_check=True,
                          lr_threshold=1.0, unique_threshold=0.95, using_constant_p2=True, post_filter_type=pf,
                          morphology_type=morph)
    s = fsc.StereoCuda()
    assert s.Init2(W, H, 0, 64, opt, fsc.CamParam(**CAM)), s.last_error()
    depth = np.empty((H, W), np.float32)
    assert s.Match2(L, R, depth), s.last_error()
    if pf and morph:  # the final map: the engine's own Match output, turned into depth
        disp = np.empty((H, W), np.float32)
        assert s.Match(L, R, disp), s.last_error()
    else:  # the map before the lone step, which has no smoothing in it
        cfg = O.Config(width=W, height=H, disp_range=64, post_filter=pf, morphology=morph)
        disp = O.match(O.depth_source_config(cfg), L, R)["disp"]
    want = O.depth_from_disp(disp, CAM["x0_left"], CAM["x0_right"], CAM["focus"], CAM["baseline"])
    assert np.array_equal(depth.view(np.uint32), want.view(np.uint32)), int((depth != want).sum())


@pytest.mark.gpu
def test_pyramid_match2_with_smoothing_takes_depth_before_the_gauss_filter(engine_lib, oracle_mod):
    """FasterStereoCuda::Match2 with do_smooth: the finest level runs the Gauss filter
    (SetSgmParameters, FasterStereoCuda.cpp:169-199) without small-region removal, so its depth is
    that of the map before the filter (StereoCudaImpl.cpp:548-583)."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H, layers = 1242, 375, 3
    L, R, _ = scenes.kitti_like(44, W, H)
    epi = fsc.EpipolarStereoParam(x0_left=CAM["x0_left"], y0_left=CAM["y0_left"], x0_right=CAM["x0_right"],
                                  y0_right=CAM["y0_right"], baseline=CAM["baseline"], focus=CAM["focus"])
    opt = fsc.StereoOption2(width=W, height=H, min_depth=5000.0, max_depth=60000.0, num_layers=layers,
                            do_lr_check=True, do_rm_peaks=True, do_smooth=True, epi=epi)
    p = fsc.FasterStereoCuda()
    assert p.Init2(opt, fsc.LevelOverride(cs_type=1, p1=10, p2=150), fsc.ExtOptions(peaks_strips=STRIPS)), \
        p.last_error()
    depth = np.empty((H, W), np.float32)
    assert p.Match2(L, R, depth), p.last_error()
    m0, d0 = O.pyr_init2_coarsest(W, layers, 5000.0, 60000.0, CAM["x0_left"], CAM["x0_right"], CAM["focus"],
                                  CAM["baseline"])
    scale = 2 ** (layers - 1)
    pc = O.PyrConfig(width=W, height=H, min_disp=m0 * scale, max_disp=(m0 + d0) * scale, num_layers=layers,
                     override_enable=1, cs_type=1, p1=10, p2=150, peaks_strips=STRIPS, do_smooth=0)
    want = O.depth_from_disp(O.pyr_match(pc, L, R), CAM["x0_left"], CAM["x0_right"], CAM["focus"],
                             CAM["baseline"])
    assert np.array_equal(depth.view(np.uint32), want.view(np.uint32)), int((depth != want).sum())
