"""CUDA engine vs oracle, bit-exact, stage by stage (runs on a B200).

Every case goes through the C ABI (StereoCuda.Init / Match, FasterStereoCuda.Init / Match).
Integer stages (census, cost, path volumes) and float disparities are compared bit for bit.
"""
import numpy as np
import pytest

from fasterstereocuda_b200 import scenes

pytestmark = pytest.mark.gpu

INV = np.float32(-999999.0)
STRIPS = 6


def bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


def assert_same(name, got, exp, mask=None):
    g, e = np.asarray(got), np.asarray(exp)
    assert g.shape == e.shape, (name, g.shape, e.shape)
    if g.dtype == np.float32:
        neq = g.view(np.uint32) != e.view(np.uint32)
    else:
        neq = g != e
    if neq.ndim == 3 and mask is not None and mask.ndim == 2:
        neq = neq.any(-1)
    if mask is not None:
        neq = neq & mask
    n = int(neq.sum())
    if n:
        idx = np.argwhere(neq)[:5]
        detail = [(tuple(int(v) for v in i), g[tuple(i)].tolist() if g.ndim <= 2 else None,
                   e[tuple(i)].tolist() if e.ndim <= 2 else None) for i in idx]
        pytest.fail(f"{name}: {n} mismatches, first {detail}")


def read_bt(s):
    """The bottom->top volume, or None when the vertical kernel kept it in shared memory."""
    try:
        return s.debug_read("bt")
    except RuntimeError as e:
        if "shared memory" in str(e):
            return None
        raise


def make_engine(fsc, W, H, M, D, cs, p1, p2, u, lr, med, peaks=0, ratio=0.0005, morph=0, tie=4):
    s = fsc.StereoCuda()
    opt = fsc.CuSGMOption(p1=p1, p2_init=p2, cs_type=cs, num_paths=4, do_median_filter=bool(med),
                          do_lr_check=bool(lr), lr_threshold=1.0, unique_threshold=u, using_constant_p2=True,
                          do_remove_peaks=bool(peaks), peaks_ratio_threshold=ratio, morphology_type=morph)
    assert s.Init(W, H, M, D, opt), s.last_error()
    assert s.set_ext_options(fsc.ExtOptions(tie_rule=tie, init_tie_rule=tie, peaks_strips=STRIPS, peaks_abs_mode=0))
    return s


CASES = {
    # name: (W, H, M, D, cs, p1, p2, uniq, lr, median, peaks, morph, seed)
    "d64_9x7_lr_med": (162, 120, 0, 64, 1, 10, 150, 0.95, 1, 1, 0, 0, 11),
    "d64_5x5_lr_med": (162, 120, 0, 64, 0, 8, 32, 0.95, 1, 1, 0, 0, 12),
    "d32_plain": (150, 90, 0, 32, 1, 10, 150, 0.95, 1, 1, 0, 0, 13),
    "d128": (300, 96, 0, 128, 1, 10, 150, 0.95, 1, 1, 0, 0, 14),
    "d256_generic": (400, 64, 0, 256, 1, 10, 150, 0.95, 1, 0, 0, 0, 15),
    "neg_min_disp": (130, 100, -4, 64, 1, 10, 150, 0.95, 1, 1, 0, 0, 16),
    "pos_min_disp": (130, 100, 8, 64, 1, 10, 150, 0.95, 1, 1, 0, 0, 17),
    "odd_size": (131, 77, 0, 64, 1, 10, 150, 0.9, 1, 1, 0, 0, 18),
    "no_lr_no_median": (162, 120, 0, 64, 1, 10, 150, 0.95, 0, 0, 0, 0, 19),
    "big_penalty": (162, 120, 0, 64, 1, 10, 230, 0.95, 1, 1, 0, 0, 20),
    "peaks": (200, 150, 0, 64, 1, 10, 150, 0.95, 0, 1, 1, 0, 21),
    "dilation_peaks": (200, 150, 0, 64, 0, 8, 32, 1.0, 1, 1, 1, 2, 22),
    "cfg0_450x375": (450, 375, 0, 64, 1, 10, 150, 0.95, 1, 1, 0, 0, 23),
    "tall_global_bt": (96, 1700, 0, 64, 1, 10, 150, 0.95, 1, 1, 0, 0, 24),  # B->T volume beyond shared memory
    "plain_1242x375x64": (1242, 375, 0, 64, 1, 10, 150, 0.95, 1, 1, 0, 0, 25),  # the single-level metric shape
}


SCANLINE = {"warp": (2, 0, 1, 0, 0, 0, 0), "scanline_g1": (3, 0, 3, 0, 0, 1, 1),
            "scanline_g8": (3, 0, 3, 0, 0, 8, 8), "latency": (4, 0, 4, 0, 0, 0, 0),
            "default": (0, 0, 0, 0, 0, 8, 4)}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("tie", [4, 0, 2, 1])
@pytest.mark.parametrize("variant", ["default", "warp", "scanline_g1", "scanline_g8", "latency"])
def test_plain_parity(engine_lib, oracle_mod, name, tie, variant):
    """Every stage against the oracle. 'default' runs the u16x2 scanline kernels where they are
    exact (else the warp kernels), 'warp' the lane-per-disparity kernels, 'scanline_g*' the
    scanline kernels with one and eight lanes per scanline, 'latency' the warp-per-scanline
    kernels with bulk-copied chunks (the default takes their place for D = 256 and tie rule 2)."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H, M, D, cs, p1, p2, u, lr, med, peaks, morph, seed = CASES[name]
    if tie != 4 and name not in ("d64_9x7_lr_med", "d128", "d32_plain", "d256_generic"):
        pytest.skip("tie rule variants on a subset")
    L, R, _ = scenes.planar_pair(seed, W, H, dmin=2.0, dmax=min(60.0, D - 4.0))
    ratio = 0.005 if peaks else 0.0005
    s = make_engine(fsc, W, H, M, D, cs, p1, p2, u, lr, med, peaks, ratio, morph, tie)
    if variant != "default":
        if tie != 4 and variant not in ("warp", "latency"):
            pytest.skip("tie rule variants with the default lane split only")
    # 'default': the default kernels and lane split, set explicitly (a matcher left at the default
    # tuning runs the latency kernels when its synchronous host API is called by one caller)
    assert s.set_tuning(fsc.Tuning(*SCANLINE[variant])), s.last_error()
    disp = np.empty((H, W), np.float32)
    disp_r = np.empty((H, W), np.float32)
    assert s.Match(L, R, disp, disp_r), s.last_error()
    cfg = O.Config(width=W, height=H, min_disp=M, disp_range=D, cs_type=cs, p1=p1, p2=p2, uniqueness=u,
                   do_lr_check=lr, do_median=med, do_remove_peaks=peaks, peaks_ratio=ratio,
                   morphology_dilation=int(morph == 2), peaks_strips=STRIPS, tie_rule=tie, init_tie_rule=tie)
    ref = O.match(cfg, L, R, dump=True, want_right=True)
    x0 = max(0, M)
    colmask = np.zeros((H, W), bool)
    colmask[:, x0:] = True
    assert_same("census_l", s.debug_read("census_l"), ref["census_l"])
    assert_same("census_r", s.debug_read("census_r"), ref["census_r"])
    assert_same("cost", s.debug_read("cost"), ref["cost"], colmask)
    assert_same("path L->R", s.debug_read("lr"), ref["paths"][1], colmask)
    assert_same("path R->L", s.debug_read("rl"), ref["paths"][3], colmask)
    bt = read_bt(s)
    if bt is not None:
        assert_same("path B->T", bt, ref["paths"][2], colmask)
    assert_same("wta left", s.debug_read("wta", 0), ref["wta_l"])
    if lr:
        assert_same("wta right", s.debug_read("wta", 1), ref["wta_r"])
        assert_same("disp right", disp_r, ref["disp_r"])
    assert_same("disp left", disp, ref["disp"])
    assert s.kernel_launches() >= 3
    assert engine_lib.sgm_debug_wait_timeouts() == 0


def _init_for(O, L, R, cs, p1, p2):
    h, w = L.shape
    cfg = O.Config(width=w // 2, height=h // 2, disp_range=64, cs_type=cs, p1=p1, p2=p2, uniqueness=1.0,
                   do_lr_check=1, do_median=1, morphology_dilation=1)
    coarse = O.match(cfg, O.zoom_half(L), O.zoom_half(R))["disp"]
    return O.init_next_level(coarse, w, h)


@pytest.mark.parametrize("variant", [None, (4, 0, 4, 0, 0), (4, 0, 3, 0, 0, 0, 8), (3, 0, 4, 0, 0, 8, 0)])
@pytest.mark.parametrize("tie", [4, 0])
@pytest.mark.parametrize("cs,p1,p2,lr,u", [(1, 10, 150, 0, 1.0), (0, 8, 32, 0, 0.95), (1, 10, 150, 1, 0.95),
                                           (0, 8, 32, 1, 1.0)])
def test_init_disparity_parity(engine_lib, oracle_mod, cs, p1, p2, lr, u, tie, variant):
    """Initial-disparity levels, stage by stage; `variant`: the latency kernels (variant 4) for the
    row scans, the column scans or both (None: the default kernels)."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 162, 121
    L, R, _ = scenes.planar_pair(31 + cs, W, H)
    init = _init_for(O, L, R, cs, p1, p2)
    s = make_engine(fsc, W, H, 0, 32, cs, p1, p2, u, lr, 1, tie=tie)
    if variant is not None:
        assert s.set_tuning(fsc.Tuning(*variant)), s.last_error()
    disp = np.empty((H, W), np.float32)
    assert s.Match(L, R, disp, None, init), s.last_error()
    assert engine_lib.sgm_debug_wait_timeouts() == 0
    cfg = O.Config(width=W, height=H, disp_range=32, cs_type=cs, p1=p1, p2=p2, uniqueness=u, do_lr_check=lr,
                   do_median=1, peaks_strips=STRIPS, tie_rule=tie, init_tie_rule=tie)
    ref = O.match(cfg, L, R, init, dump=True, want_right=True)
    valid = init != -32768
    assert_same("cost", s.debug_read("cost"), ref["cost"])
    assert_same("path L->R", s.debug_read("lr"), ref["paths"][1], valid)
    assert_same("path R->L", s.debug_read("rl"), ref["paths"][3], valid)
    bt = read_bt(s)
    if bt is not None:
        assert_same("path B->T", bt, ref["paths"][2], valid)
    assert_same("wta left", s.debug_read("wta", 0), ref["wta_l"])
    if lr:
        assert_same("wta right", s.debug_read("wta", 1), ref["wta_r"])
    assert_same("disp left", disp, ref["disp"])


def _blocky_pair(seed, W, H, shift=5):
    """Piecewise-constant 8x8 blocks of four grey levels: flat patches give equal costs over
    many disparities, so the WTA meets ties whose first candidate fails the uniqueness test."""
    rng = np.random.default_rng(seed)
    blocks = rng.integers(0, 4, ((H + 7) // 8, (W + 7) // 8 + 2)) * 60
    img = np.repeat(np.repeat(blocks, 8, 0), 8, 1).astype(np.uint8)
    L = np.ascontiguousarray(img[:H, 8:8 + W])
    R = np.ascontiguousarray(img[:H, 8 + shift:8 + shift + W])
    return L, R


@pytest.mark.parametrize("lanes", [(2, 2), (8, 8), "latency"])
@pytest.mark.parametrize("tie", [4, 0])
def test_init_disparity_ties_low_texture(engine_lib, oracle_mod, tie, lanes):
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 200, 96
    L, R = _blocky_pair(7, W, H)
    init = np.full((H, W), 3, np.int16)
    init[:, ::17] = 9
    s = make_engine(fsc, W, H, 0, 32, 1, 10, 150, 0.95, 1, 1, tie=tie)
    t = (4, 0, 4, 0, 0) if lanes == "latency" else (3, 0, 3, 0, 0, *lanes)
    assert s.set_tuning(fsc.Tuning(*t)), s.last_error()
    disp = np.empty((H, W), np.float32)
    assert s.Match(L, R, disp, None, init), s.last_error()
    cfg = O.Config(width=W, height=H, disp_range=32, cs_type=1, p1=10, p2=150, uniqueness=0.95, do_lr_check=1,
                   do_median=1, peaks_strips=STRIPS, tie_rule=tie, init_tie_rule=tie)
    ref = O.match(cfg, L, R, init, dump=True, want_right=True)
    assert_same("wta left", s.debug_read("wta", 0), ref["wta_l"])
    assert_same("wta right", s.debug_read("wta", 1), ref["wta_r"])
    assert_same("disp left", disp, ref["disp"])


@pytest.mark.parametrize("variant", [None, (4, 0, 4, 0, 0)])
def test_init_disparity_invalid_runs_and_jumps(engine_lib, oracle_mod, variant):
    """Initial disparities with 30 % INVALID pixels, INVALID runs longer than a 32-step chunk (whole
    chunks skipped, a scanline starting INVALID) and base jumps beyond the 32-disparity range:
    every stage against the oracle, for the default and the warp-per-scanline kernels."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 203, 97
    L, R, _ = scenes.planar_pair(57, W, H)
    rng = np.random.default_rng(5)
    init = rng.integers(0, 41, (H, W)).astype(np.int16)
    init[rng.random((H, W)) < 0.3] = -32768
    init[10:20, 30:110] = -32768   # rows with a run of 80 INVALID pixels
    init[:, 0] = -32768            # every row starts INVALID
    init[40:60, 150:190] = -32768  # columns with a run of 20
    init[5:90, 170:172] = -32768   # columns with a run of 85
    init[::7, ::5] = 0             # realignments of up to 40 between neighbours
    init[3::7, 2::5] = 40
    s = make_engine(fsc, W, H, 0, 32, 1, 10, 150, 0.95, 1, 1)
    if variant is not None:
        assert s.set_tuning(fsc.Tuning(*variant)), s.last_error()
    disp = np.empty((H, W), np.float32)
    assert s.Match(L, R, disp, None, init), s.last_error()
    assert engine_lib.sgm_debug_wait_timeouts() == 0
    cfg = O.Config(width=W, height=H, disp_range=32, do_lr_check=1, do_median=1, peaks_strips=STRIPS)
    ref = O.match(cfg, L, R, init, dump=True, want_right=True)
    valid = init != -32768
    assert_same("path L->R", s.debug_read("lr"), ref["paths"][1], valid)
    assert_same("path R->L", s.debug_read("rl"), ref["paths"][3], valid)
    bt = read_bt(s)
    if bt is not None:
        assert_same("path B->T", bt, ref["paths"][2], valid)
    assert_same("wta left", s.debug_read("wta", 0), ref["wta_l"])
    assert_same("wta right", s.debug_read("wta", 1), ref["wta_r"])
    assert_same("disp left", disp, ref["disp"])


@pytest.mark.parametrize("kind", ["plain64", "plain128", "init32"])
@pytest.mark.parametrize("p1,p2", [(10, 5_000_000), (3_000_000, 5_000_000)])
def test_latency_kernels_large_penalties(engine_lib, oracle_mod, kind, p1, p2):
    """The warp-per-scanline kernels compute in 32 bits like the reference: any penalties are exact
    (the 32-disparity row scan packs P2' into 22 bits and leaves larger penalties to the default)."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 150, 83
    L, R, _ = scenes.planar_pair(71, W, H)
    disp = np.empty((H, W), np.float32)
    if kind == "init32":
        init = _init_for(O, L, R, 1, 10, 150)
        s = make_engine(fsc, W, H, 0, 32, 1, p1, p2, 0.95, 1, 1)
        assert s.set_tuning(fsc.Tuning(4, 0, 4, 0, 0)), s.last_error()
        assert s.Match(L, R, disp, None, init), s.last_error()
        ref = O.match(O.Config(width=W, height=H, disp_range=32, p1=p1, p2=p2, do_lr_check=1, do_median=1,
                               peaks_strips=STRIPS), L, R, init)
    else:
        D = 64 if kind == "plain64" else 128
        s = make_engine(fsc, W, H, 0, D, 1, p1, p2, 0.95, 1, 1)
        assert s.set_tuning(fsc.Tuning(4, 0, 4, 0, 0)), s.last_error()
        assert s.Match(L, R, disp), s.last_error()
        ref = O.match(O.Config(width=W, height=H, disp_range=D, p1=p1, p2=p2, do_lr_check=1, do_median=1,
                               peaks_strips=STRIPS), L, R)
    assert engine_lib.sgm_debug_wait_timeouts() == 0
    assert_same(f"disp {kind}", disp, ref["disp"])


def test_init_disparity_tall_global_bt(engine_lib, oracle_mod):
    """32-disparity level taller than the shared-memory budget of the vertical kernel."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 64, 3600
    L, R, _ = scenes.planar_pair(35, W, H, dmin=2.0, dmax=30.0)
    init = _init_for(O, L, R, 1, 10, 150)
    s = make_engine(fsc, W, H, 0, 32, 1, 10, 150, 0.95, 0, 1)
    disp = np.empty((H, W), np.float32)
    assert s.Match(L, R, disp, None, init), s.last_error()
    ref = O.match(O.Config(width=W, height=H, disp_range=32, do_lr_check=0, do_median=1, peaks_strips=STRIPS), L, R,
                  init, dump=True)
    bt = read_bt(s)
    if bt is not None:
        assert_same("path B->T", bt, ref["paths"][2], init != -32768)
    assert_same("disp left", disp, ref["disp"])


@pytest.mark.parametrize("kernels", ["auto", "throughput"])
@pytest.mark.parametrize("override", [True, False])
@pytest.mark.parametrize("size,layers", [((1242, 375), 3), ((450, 375), 2), ((640, 480), 4)])
def test_pyramid_parity(engine_lib, oracle_mod, override, size, layers, kernels):
    """'auto': the default tuning, which the synchronous host API runs with the latency kernels for
    a single caller; 'throughput': the default thread-per-scanline kernels set explicitly. Three
    matches: the direct run, the graph capture and a graph replay."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = size
    L, R, _ = scenes.kitti_like(41, W, H)
    p = fsc.FasterStereoCuda()
    opt = fsc.StereoOption1(width=W, height=H, min_disp=0, max_disp=64, num_layers=layers, do_lr_check=True,
                            do_rm_peaks=True)
    ov = fsc.LevelOverride(cs_type=1, p1=10, p2=150) if override else None
    assert p.Init(opt, ov, fsc.ExtOptions(peaks_strips=STRIPS)), p.last_error()
    if kernels == "throughput":
        assert p.set_tuning(fsc.Tuning(0, 0, 0, 0, 0, 8, 4)), p.last_error()
    pc = O.PyrConfig(width=W, height=H, min_disp=0, max_disp=64, num_layers=layers, override_enable=int(override),
                     cs_type=1 if override else 0, p1=10 if override else 8, p2=150 if override else 32,
                     peaks_strips=STRIPS)
    ref = O.pyr_match(pc, L, R)
    for k in range(3):
        disp = np.empty((H, W), np.float32)
        assert p.Match(L, R, disp)
        assert_same(f"pyramid disp, match {k}", disp, ref)
    assert engine_lib.sgm_debug_wait_timeouts() == 0
    for lvl in range(layers):
        w, h, m, d = p.level_info(lvl)
        c = O.pyr_level_config(pc, lvl)
        assert (w, h, m, d) == (c.width, c.height, c.min_disp, c.disp_range)


def test_host_api_kernel_modes_under_concurrency(engine_lib, oracle_mod):
    """Default-tuned matchers called through the synchronous host API by one thread (the latency
    kernels, polled completion) and by twelve threads at once (the throughput kernels and a
    sleeping wait while more than eight calls are in flight): every match -- direct runs, captures
    and replays of both graphs -- equals the oracle."""
    import fasterstereocuda_b200 as fsc
    from concurrent.futures import ThreadPoolExecutor
    O = oracle_mod
    W, H = 450, 240
    pairs = [scenes.kitti_like(60 + i, W, H)[:2] for i in range(2)]
    pc = O.PyrConfig(width=W, height=H, min_disp=0, max_disp=64, num_layers=2, override_enable=1, cs_type=1,
                     p1=10, p2=150, peaks_strips=STRIPS)
    refs = [O.pyr_match(pc, L, R) for L, R in pairs]
    ms = []
    for _ in range(12):
        p = fsc.FasterStereoCuda()
        assert p.Init(fsc.StereoOption1(width=W, height=H, min_disp=0, max_disp=64, num_layers=2, do_lr_check=True,
                                        do_rm_peaks=True), fsc.LevelOverride(1, 10, 150),
                      fsc.ExtOptions(peaks_strips=STRIPS)), p.last_error()
        ms.append(p)

    def work(k, n):
        out = []
        for j in range(n):
            i = (k + j) % 2
            disp = np.empty((H, W), np.float32)
            assert ms[k].Match(pairs[i][0], pairs[i][1], disp), ms[k].last_error()
            out.append((i, disp))
        return out
    results = work(0, 4)  # one caller: latency kernels
    with ThreadPoolExecutor(max_workers=12) as ex:
        for r in ex.map(lambda k: work(k, 6), range(12)):
            results += r
    results += work(1, 3)  # alone again: the latency graph of a matcher that ran both
    for i, disp in results:
        assert_same("pyramid disp", disp, refs[i])
    assert engine_lib.sgm_debug_wait_timeouts() == 0


def test_device_api_matches_host_api(engine_lib, oracle_mod):
    import torch
    import fasterstereocuda_b200 as fsc
    W, H = 320, 200
    L, R, _ = scenes.planar_pair(51, W, H)
    s = make_engine(fsc, W, H, 0, 64, 1, 10, 150, 0.95, 1, 1)
    host = np.empty((H, W), np.float32)
    assert s.Match(L, R, host)
    dl, dr = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    out = torch.empty((H, W), dtype=torch.float32, device="cuda")
    out_r = torch.empty((H, W), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert s.match_device(dl, dr, out, out_r, None, stream), s.last_error()
    torch.cuda.synchronize()
    assert_same("device api", out.cpu().numpy(), host)


def test_repeated_matches_are_identical(engine_lib):
    import fasterstereocuda_b200 as fsc
    W, H = 256, 160
    L, R, _ = scenes.planar_pair(52, W, H)
    s = make_engine(fsc, W, H, 0, 64, 1, 10, 150, 0.95, 1, 1, 1, 0.001)
    a = np.empty((H, W), np.float32)
    b = np.empty((H, W), np.float32)
    assert s.Match(L, R, a) and s.Match(L, R, b)
    assert_same("repeat", a, b)


def test_errors_on_device(engine_lib):
    import fasterstereocuda_b200 as fsc
    W, H = 128, 96
    s = make_engine(fsc, W, H, 0, 64, 1, 10, 150, 0.95, 0, 1)
    img = np.zeros((H, W), np.uint8)
    out = np.empty((H, W), np.float32)
    init = np.zeros((H, W), np.int16)
    assert not s.Match(img, img, out, None, init) and s.status == -4   # init needs D=32
    roi = fsc.StereoROI(120, 0, 10, 10)  # leaves the 128-pixel-wide image
    assert not s.Match(img, img, out, None, None, roi) and s.status == -1
    s.Release()
    assert not s.Match(img, img, out) and s.status == -2


TUNINGS = [(1, 0, 1, 0, 0), (1, 2, 1, 4, 0), (2, 1, 2, 8, 1), (2, 2, 2, 2, 0), (2, 4, 2, 1, 1), (1, 4, 2, 8, 0),
           (3, 0, 3, 0, 0), (3, 0, 1, 0, 0), (2, 0, 3, 0, 0), (3, 0, 3, 0, 0, 2, 2), (3, 0, 3, 0, 0, 4, 8),
           (3, 0, 3, 0, 0, 8, 1), (4, 0, 4, 0, 0), (4, 0, 3, 0, 0, 0, 8), (3, 0, 4, 0, 0, 8, 0), (4, 0, 1, 0, 0),
           (2, 0, 4, 0, 0)]


@pytest.mark.parametrize("tuning", TUNINGS)
@pytest.mark.parametrize("kind", ["plain64", "plain128_5x5", "init32"])
def test_tuning_variants_are_bit_exact(engine_lib, oracle_mod, tuning, kind):
    """Every kernel variant / launch shape the tuner may pick gives the oracle's result."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 203, 131
    L, R, _ = scenes.planar_pair(61, W, H)
    t = fsc.Tuning(*tuning)
    disp = np.empty((H, W), np.float32)
    if kind == "init32":
        init = _init_for(O, L, R, 1, 10, 150)
        s = make_engine(fsc, W, H, 0, 32, 1, 10, 150, 0.95, 1, 1)
        assert s.set_tuning(t), s.last_error()
        assert s.Match(L, R, disp, None, init), s.last_error()
        ref = O.match(O.Config(width=W, height=H, disp_range=32, do_lr_check=1, do_median=1, peaks_strips=STRIPS),
                      L, R, init)
    else:
        D, cs, p1, p2 = (64, 1, 10, 150) if kind == "plain64" else (128, 0, 8, 32)
        s = make_engine(fsc, W, H, -2, D, cs, p1, p2, 0.95, 1, 1)
        assert s.set_tuning(t), s.last_error()
        assert s.Match(L, R, disp), s.last_error()
        ref = O.match(O.Config(width=W, height=H, min_disp=-2, disp_range=D, cs_type=cs, p1=p1, p2=p2,
                               do_lr_check=1, do_median=1, peaks_strips=STRIPS), L, R)
    assert_same(f"disp {kind} {tuning}", disp, ref["disp"])


def test_pyramid_tuning_is_bit_exact(engine_lib, oracle_mod):
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 640, 360
    L, R, _ = scenes.kitti_like(43, W, H)
    p = fsc.FasterStereoCuda()
    assert p.Init(fsc.StereoOption1(width=W, height=H, min_disp=0, max_disp=64, num_layers=3),
                  fsc.LevelOverride(1, 10, 150), fsc.ExtOptions(peaks_strips=STRIPS)), p.last_error()
    pc = O.PyrConfig(width=W, height=H, max_disp=64, num_layers=3, override_enable=1, cs_type=1, p1=10, p2=150,
                     peaks_strips=STRIPS)
    ref = O.pyr_match(pc, L, R)
    for t in TUNINGS[:3]:
        assert p.set_tuning(fsc.Tuning(*t)), p.last_error()
        disp = np.empty((H, W), np.float32)
        assert p.Match(L, R, disp)
        assert_same(f"pyramid {t}", disp, ref)


def test_large_pyramid_4800x3409_d256(engine_lib, oracle_mod):
    """The large configuration: 4800x3409, disparities 0..256, 4 levels (coarsest 600x426 at
    D=64, three 32-disparity levels), census 9x7, P1=10, P2=150, fractal texture, 40 planes."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 4800, 3409
    L, R, _ = scenes.building_like(2, W, H)
    p = fsc.FasterStereoCuda()
    assert p.Init(fsc.StereoOption1(width=W, height=H, min_disp=0, max_disp=256, num_layers=4),
                  fsc.LevelOverride(1, 10, 150), fsc.ExtOptions(peaks_strips=STRIPS)), p.last_error()
    disp = np.empty((H, W), np.float32)
    assert p.Match(L, R, disp), p.last_error()
    pc = O.PyrConfig(width=W, height=H, max_disp=256, num_layers=4, override_enable=1, cs_type=1, p1=10, p2=150,
                     peaks_strips=STRIPS)
    assert_same("large pyramid", disp, O.pyr_match(pc, L, R))
    assert (disp != INV).mean() > 0.5


def test_graph_replay_over_successive_matches(engine_lib, oracle_mod):
    """The first match runs kernel by kernel, later ones replay a captured CUDA graph (with
    copies in and out for caller buffers); a tuning change drops the graph. Every result must
    equal the oracle, for both matchers and both entry points."""
    import torch
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 320, 200
    s = make_engine(fsc, W, H, 0, 64, 1, 10, 150, 0.95, 1, 1)
    cfg = O.Config(width=W, height=H, disp_range=64, peaks_strips=STRIPS)
    p = fsc.FasterStereoCuda()
    assert p.Init(fsc.StereoOption1(width=W, height=H, min_disp=0, max_disp=64, num_layers=2),
                  fsc.LevelOverride(1, 10, 150), fsc.ExtOptions(peaks_strips=STRIPS)), p.last_error()
    pc = O.PyrConfig(width=W, height=H, max_disp=64, num_layers=2, override_enable=1, cs_type=1, p1=10, p2=150,
                     peaks_strips=STRIPS)
    stream = torch.cuda.current_stream().cuda_stream
    for k in range(5):
        L, R, _ = scenes.planar_pair(70 + k, W, H)
        if k == 3:
            assert s.set_tuning(fsc.Tuning(3, 0, 3, 0, 0, 4, 2)) and p.set_tuning(fsc.Tuning(0, 0, 0, 0, 0, 2, 4))
        out = np.empty((H, W), np.float32)
        if k % 2 == 0:
            assert s.Match(L, R, out), s.last_error()
        else:
            dout = torch.empty((H, W), dtype=torch.float32, device="cuda")
            assert s.match_device(torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda(), dout, None, None, stream)
            torch.cuda.synchronize()
            out = dout.cpu().numpy()
        assert_same(f"plain match {k}", out, O.match(cfg, L, R)["disp"])
        pout = np.empty((H, W), np.float32)
        if k % 2 == 1:
            assert p.Match(L, R, pout), p.last_error()
        else:
            dout = torch.empty((H, W), dtype=torch.float32, device="cuda")
            assert p.match_device(torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda(), dout, stream)
            torch.cuda.synchronize()
            pout = dout.cpu().numpy()
        assert_same(f"pyramid match {k}", pout, O.pyr_match(pc, L, R))
    assert s.kernel_launches() > 0 and p.kernel_launches() > 0


@pytest.mark.parametrize("pf", [0, 1, 2])
@pytest.mark.parametrize("morph", [0, 1, 2, 3, 4])
def test_post_filters_and_morphology(engine_lib, oracle_mod, pf, morph):
    """Gauss / bilateral post filters and erosion / dilation / open / close after the median
    (reference DisparityFilter::Filter). Without a post filter the maps are bit-exact; the
    filters weight by exp(), whose last bit may differ between CUDA and the host's libm, so
    there INVALID masks must be identical and values within 1e-4 px."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 220, 150
    L, R, _ = scenes.planar_pair(90 + pf + 3 * morph, W, H)
    s = fsc.StereoCuda()
    opt = fsc.CuSGMOption(p1=10, p2_init=150, cs_type=1, num_paths=4, do_median_filter=True, do_lr_check=True,
                          lr_threshold=1.0, unique_threshold=0.95, using_constant_p2=True, post_filter_type=pf,
                          morphology_type=morph)
    assert s.Init(W, H, 0, 64, opt), s.last_error()
    assert s.set_ext_options(fsc.ExtOptions(peaks_strips=STRIPS))
    disp = np.empty((H, W), np.float32)
    assert s.Match(L, R, disp), s.last_error()
    ref = O.match(O.Config(width=W, height=H, disp_range=64, post_filter=pf, morphology=morph, peaks_strips=STRIPS),
                  L, R)["disp"]
    if pf == 0:
        assert_same(f"pf0 morph{morph}", disp, ref)
    else:
        assert np.array_equal(disp == INV, ref == INV), int(((disp == INV) != (ref == INV)).sum())
        ok = disp != INV
        assert np.abs(disp[ok] - ref[ok]).max() <= 1e-4, np.abs(disp[ok] - ref[ok]).max()
    assert (disp != INV).mean() > 0.3


def test_pyramid_smoothing(engine_lib, oracle_mod):
    """do_smooth: Gauss filter at the finest pyramid level (reference SetSgmParameters)."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 450, 375
    L, R, _ = scenes.cone_like(16)
    p = fsc.FasterStereoCuda()
    assert p.Init(fsc.StereoOption1(width=W, height=H, min_disp=0, max_disp=64, num_layers=2, do_smooth=True),
                  None, fsc.ExtOptions(peaks_strips=STRIPS)), p.last_error()
    disp = np.empty((H, W), np.float32)
    assert p.Match(L, R, disp), p.last_error()
    ref = O.pyr_match(O.PyrConfig(width=W, height=H, max_disp=64, num_layers=2, do_smooth=1, override_enable=0,
                                  peaks_strips=STRIPS), L, R)
    assert np.array_equal(disp == INV, ref == INV)
    ok = disp != INV
    assert np.abs(disp[ok] - ref[ok]).max() <= 1e-4
