"""The give-up path of the bounded waits in the warp-per-scanline scans, made to run without a GPU
fault: a test hook makes the plain row scans expect 16 bytes more than their first bulk copy
delivers, so that mbarrier phase never completes, and shortens every wait to a few thousand polls.
Each warp then records the timeout, waits (bounded) for its other copies in flight and stops; the
match returns, the counter read by sgm_debug_wait_timeouts shows the give-ups, and the context
stays usable: the next match, hooks off, equals the oracle."""
import numpy as np
import pytest

from fasterstereocuda_b200 import scenes

STRIPS = 8


def _matcher(fsc, W, H):
    s = fsc.StereoCuda()
    opt = fsc.CuSGMOption(p1=10, p2_init=150, cs_type=1, num_paths=4, do_median_filter=True, do_lr_check=True,
                          lr_threshold=1.0, unique_threshold=0.95, using_constant_p2=True)
    assert s.Init(W, H, 0, 64, opt), s.last_error()
    assert s.set_ext_options(fsc.ExtOptions(peaks_strips=STRIPS))
    assert s.set_tuning(fsc.Tuning(4, 0, 4, 0, 0)), s.last_error()  # the warp-per-scanline kernels
    return s


@pytest.mark.gpu
def test_wait_that_runs_out_is_recorded_and_the_context_stays_usable(engine_lib, oracle_mod):
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = 200, 96
    L, R, _ = scenes.planar_pair(83, W, H)
    assert engine_lib.sgm_debug_reset_wait_timeouts() == 0
    s = _matcher(fsc, W, H)
    disp = np.empty((H, W), np.float32)
    assert engine_lib.sgm_debug_scan_wait(4096, 1) == 0
    try:
        assert s.Match(L, R, disp), s.last_error()  # the match itself completes
        gave_up = engine_lib.sgm_debug_wait_timeouts()
    finally:
        assert engine_lib.sgm_debug_scan_wait(0, 0) == 0
    # every row scan (2 views x 2 directions x H rows) gave up on its first chunk
    assert gave_up >= 2 * 2 * H, gave_up
    assert engine_lib.sgm_debug_reset_wait_timeouts() == 0
    # hooks off: the same matcher and a new one match exactly, with no give-up
    ref = O.match(O.Config(width=W, height=H, disp_range=64, do_lr_check=1, do_median=1, peaks_strips=STRIPS),
                  L, R)["disp"]
    for m in (s, _matcher(fsc, W, H)):
        out = np.empty((H, W), np.float32)
        assert m.Match(L, R, out), m.last_error()
        assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))
    assert engine_lib.sgm_debug_wait_timeouts() == 0


def test_hooks_are_exported(engine_lib):
    """The test hooks exist without a GPU (their calls need one)."""
    for name in ("sgm_debug_scan_wait", "sgm_debug_reset_wait_timeouts", "sgm_debug_wait_timeouts"):
        assert hasattr(engine_lib, name)
