"""Out-of-memory paths of the initialisation calls, with a failure injected on the host side: the
engine's device allocations go through one function that can be told to fail the n-th allocation
as cudaMalloc does on an exhausted device (sgm_debug_fail_device_alloc). The reference's Init
returns false when an allocation fails (SgmStereoCuda/StereoCudaImpl.cpp:138-207); here every init
returns SGM_ERR_NOMEM at every allocation it makes and keeps nothing allocated afterwards. No GPU is
driven out of memory."""
import numpy as np
import pytest

NOMEM = -5


def _make(fsc, kind):
    """(init callable returning a status, release callable) for one kind of matcher."""
    opt = fsc.CuSGMOption(p1=10, p2_init=150, cs_type=1, num_paths=4, do_median_filter=True, do_lr_check=True,
                          lr_threshold=1.0, unique_threshold=0.95, using_constant_p2=True, do_remove_peaks=True,
                          peaks_ratio_threshold=0.0005)
    cam = fsc.CamParam(x0_left=100.0, y0_left=60.0, x0_right=104.0, y0_right=60.0, focus=300.0, baseline=200.0)
    if kind in ("single", "init2"):
        s = fsc.StereoCuda()

        def init():
            ok = s.Init(160, 96, 0, 64, opt) if kind == "single" else s.Init2(160, 96, 0, 64, opt, cam)
            return 0 if ok else s.status
        return init, s.Release
    if kind in ("pyramid", "pyramid2"):
        p = fsc.FasterStereoCuda()

        def init():
            if kind == "pyramid":
                ok = p.Init(fsc.StereoOption1(width=320, height=192, min_disp=0, max_disp=64, num_layers=3),
                            fsc.LevelOverride(1, 10, 150), fsc.ExtOptions())
            else:
                epi = fsc.EpipolarStereoParam(x0_left=100.0, y0_left=60.0, x0_right=104.0, y0_right=60.0,
                                              baseline=200.0, focus=300.0)
                ok = p.Init2(fsc.StereoOption2(width=320, height=192, min_depth=1000.0, max_depth=20000.0,
                                               num_layers=3, epi=epi), fsc.LevelOverride(1, 10, 150))
            return 0 if ok else p.status
        return init, p.Release
    pairs = [(160, 96, 0, 64), (224, 128, 0, 32)]
    if kind == "batch":
        b = fsc.StereoBatch()
        o = fsc.CuSGMOption(**{f: getattr(opt, f) for f, _ in fsc.CuSGMOption._fields_})
        o.do_remove_peaks = False

        def init():
            return 0 if b.Init(pairs, o) else b.status
        return init, lambda: None
    b = fsc.StereoBatchPyramid()

    def init():
        ok = b.Init([(320, 192, 0, 64)] * 2, fsc.StereoOption1(num_layers=2, do_lr_check=True, do_rm_peaks=True),
                    fsc.LevelOverride(1, 10, 150), fsc.ExtOptions())
        return 0 if ok else b.status
    return init, lambda: None


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["single", "init2", "pyramid", "pyramid2", "batch", "batch_pyramid"])
def test_allocation_failure_returns_nomem_and_keeps_nothing(engine_lib, kind):
    import fasterstereocuda_b200 as fsc
    lib = engine_lib
    live = lib.sgm_debug_live_device_allocations
    base = live()
    init, release = _make(fsc, kind)
    assert init() == 0
    n = live() - base
    assert n > 0
    release()
    init, release = _make(fsc, kind)  # a fresh object for every injected failure
    try:
        for k in range(n):
            lib.sgm_debug_fail_device_alloc(k)
            st = init()
            assert st == NOMEM, (k, st)
            assert live() == base, (k, live() - base)
        lib.sgm_debug_fail_device_alloc(-1)
        assert init() == 0  # and the same object initialises once memory is there again
    finally:
        lib.sgm_debug_fail_device_alloc(-1)
        release()


def test_fault_injection_is_armed_and_disarmed_without_a_device(engine_lib):
    """The hook itself needs no GPU: arming, disarming and the live count."""
    lib = engine_lib
    assert lib.sgm_debug_fail_device_alloc(3) == 0
    assert lib.sgm_debug_fail_device_alloc(-1) == 0
    assert lib.sgm_debug_live_device_allocations() >= 0
