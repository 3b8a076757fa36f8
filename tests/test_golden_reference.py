"""Oracle vs the reference's own CUDA build (fixtures dumped on a B200 by tests/golden/make_golden.py).

Exact on every deterministic stage: census, cost and path volumes (digests), the WTA map on
every pixel the reference writes, the left-right check on pixels the reference's read/invalidate
race cannot change. The final filtered map agrees except where the reference's in-place median
races on block halos (checked: every such pixel can take the reference's value for some halo
ordering).
"""
import ctypes as C
import hashlib
import itertools
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem[4:] for p in GOLDEN.glob("ref_*.npz")
               if not p.stem.startswith(("ref_pyr", "ref_levels", "ref_depth", "ref_roi")))
DEPTH = sorted(p.stem[4:] for p in GOLDEN.glob("ref_depth*.npz"))
PYR = sorted(p.stem[4:] for p in GOLDEN.glob("ref_pyr*.npz"))
LEVELS = sorted(p.stem[4:] for p in GOLDEN.glob("ref_levels_*.npz"))
INV = np.float32(-999999.0)


def load(name):
    z = dict(np.load(GOLDEN / f"ref_{name}.npz"))
    return z, json.loads(str(z["case"]))


def config(O, case, strips, **kw):
    c = O.Config(width=case["width"], height=case["height"], min_disp=case["min_disp"], disp_range=case["disp_range"],
                 cs_type=case["cs_type"], p1=case["p1"], p2=case["p2"], uniqueness=case["uniqueness"],
                 peaks_strips=int(strips), tie_rule=4, init_tie_rule=4)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def written_mask(case, init):
    H, W = case["height"], case["width"]
    m = np.zeros((H, W), bool)
    m[:(H // 4) * 4 if init is not None else (H // 2) * 2, max(0, case["min_disp"]):] = True
    return m


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def halo_race_unexplained(O, pre, ref, pixels, H, W):
    """Pixels (y, x) whose reference value no ordering of the in-place 3x3 median's block halos
    produces. The reference filters 2-row x 30-column blocks in place, so a pixel outside the
    own block may be read before or after its neighbour block filtered it."""
    snap = O.median3x3(pre)
    out = []
    for y, x in pixels:
        if y >= H - 2:
            continue
        by, bx = (y - 1) // 2, (x - 1) // 30
        opts = []
        for dy, dx in itertools.product((-1, 0, 1), (-1, 0, 1)):
            yy, xx = y + dy, x + dx
            own = ((yy - 1) // 2 == by) and ((xx - 1) // 30 == bx) and 1 <= yy <= H - 2 and 1 <= xx <= W - 2
            opts.append([pre[yy, xx]] if own or (dy == 0 and dx == 0) else sorted({float(pre[yy, xx]),
                                                                                   float(snap[yy, xx])}))
        if not any(np.float32(sorted(c)[4]) == ref[y, x] for c in itertools.product(*opts)):
            out.append((int(y), int(x)))
    return out


def test_fixtures_present():
    assert len(CASES) >= 6, CASES


@pytest.mark.parametrize("name", CASES)
def test_stage_volumes_bit_exact(oracle_mod, name):
    z, case = load(name)
    if "digest_census" not in z:
        pytest.skip("volumes dumped only for the small cases")
    O = oracle_mod
    init = z.get("init")
    a = O.match(config(O, case, z["peaks_strips"], do_lr_check=0, do_median=0), z["left"], z["right"], init,
                dump=True)
    H, W = case["height"], case["width"]
    x0 = max(0, case["min_disp"])
    assert digest(np.stack([a["census_l"], a["census_r"]])) == str(z["digest_census"])
    cm = np.zeros((H, W), bool)
    cm[:, x0:] = True
    assert digest(np.where(cm[..., None], a["cost"], 0)) == str(z["digest_cost_lr"])
    from tests.golden.make_golden import path_first_pixel_mask  # noqa: E402
    valid = np.broadcast_to(cm, (4, H, W)) & ~path_first_pixel_mask(W, H, x0)
    if init is not None:
        valid = valid & np.broadcast_to(init != -32768, (4, H, W))
    assert digest(np.where(valid[..., None], a["paths"], 0)) == str(z["digest_paths_lr"])


@pytest.mark.parametrize("name", CASES)
def test_wta_bit_exact_on_written_pixels(oracle_mod, name):
    z, case = load(name)
    O = oracle_mod
    init = z.get("init")
    a = O.match(config(O, case, z["peaks_strips"], do_lr_check=0, do_median=0), z["left"], z["right"], init)
    m = written_mask(case, init)
    neq = (a["disp"].view(np.uint32) != z["wta_l"].view(np.uint32)) & m
    assert int(neq.sum()) == 0, np.argwhere(neq)[:5]


@pytest.mark.parametrize("name", CASES)
def test_lr_check_exact_on_race_free_pixels(oracle_mod, name):
    z, case = load(name)
    if z.get("init") is not None:
        pytest.skip("the pyramid checks consistency only on plain levels")
    O = oracle_mod
    cfg = config(O, case, z["peaks_strips"], do_lr_check=1, do_median=0)
    a = O.match(cfg, z["left"], z["right"], dump=True, want_right=True)
    # race-free: same result whether the right map is read before or after every invalidation
    W, H = case["width"], case["height"]
    marks = a["wta_r"].copy()
    snap = a["wta_l"].copy()
    O.lib().orc_lr_check(snap.ctypes.data, a["wta_r"].ctypes.data, marks.ctypes.data, W, H, C.c_float(1.0))
    late = a["wta_l"].copy()
    O.lib().orc_lr_check(late.ctypes.data, marks.ctypes.data, None, W, H, C.c_float(1.0))
    rf = (snap.view(np.uint32) == late.view(np.uint32)) & written_mask(case, None)
    assert np.array_equal(snap.view(np.uint32), a["disp"].view(np.uint32))
    neq = (a["disp"].view(np.uint32) != z["lr_l"].view(np.uint32)) & rf
    assert int(neq.sum()) == 0, np.argwhere(neq)[:5]
    assert rf.mean() > 0.9
    # the right map after invalidation marks matches everywhere
    assert np.array_equal(a["disp_r"][:(H // 2) * 2].view(np.uint32), z["lr_r"][:(H // 2) * 2].view(np.uint32))


@pytest.mark.parametrize("name", [c for c in CASES if c in ("c9x7", "c5x5", "negmin", "init9x7", "init5x5")])
def test_final_map_differences_are_median_halo_races(oracle_mod, name):
    z, case = load(name)
    O = oracle_mod
    H, W = case["height"], case["width"]
    init = z.get("init")
    pre = z["lr_l"] if case["do_lr_check"] else z["wta_l"]
    full = O.match(config(O, case, z["peaks_strips"], do_lr_check=case["do_lr_check"], do_median=1), z["left"],
                   z["right"], init)["disp"]
    rows = np.zeros((H, W), bool)
    rows[:H - 1 if H % 2 else H] = True
    eq = (full.view(np.uint32) == z["disp_l"].view(np.uint32))
    assert eq[rows].mean() > 0.985
    unexplained = halo_race_unexplained(O, pre, z["disp_l"], np.argwhere(~eq & rows), H, W)
    assert not unexplained, unexplained[:5]


@pytest.mark.parametrize("name", PYR)
def test_pyramid_against_reference(oracle_mod, name):
    z, case = load(name)
    O = oracle_mod
    pc = O.PyrConfig(width=case["width"], height=case["height"], min_disp=case["min_disp"], max_disp=case["max_disp"],
                     num_layers=case["num_layers"], override_enable=0, peaks_strips=int(z["peaks_strips"]),
                     do_lr_check=case.get("lr", 1), do_rm_peaks=case.get("peaks", 1))
    d = O.pyr_match(pc, z["left"], z["right"])
    eq = d.view(np.uint32) == z["disp"].view(np.uint32)
    # whole-pyramid agreement; level-by-level exactness is checked in test_pyramid_levels_against_reference
    assert eq[:case["height"] - 1].mean() > 0.9


@pytest.mark.parametrize("name", LEVELS)
def test_pyramid_levels_against_reference(oracle_mod, name):
    """Level by level: each level is matched from the reference's own initial disparities for it,
    so a race in one level does not spread to the next. On the rows the reference writes, the next
    level's initial disparities are exact, and every difference on an init level is a median halo
    race; the coarsest level (LR, small-region removal, dilation) differs on at most 0.1%."""
    z, case = load(name)
    O = oracle_mod
    W, H, layers = case["width"], case["height"], case["num_layers"]
    pc = O.PyrConfig(width=W, height=H, min_disp=case["min_disp"], max_disp=case["max_disp"], num_layers=layers,
                     override_enable=0, peaks_strips=int(z["peaks_strips"]), do_lr_check=case.get("lr", 1),
                     do_rm_peaks=case.get("peaks", 1))
    imgs = [(z["left"], z["right"])]
    for _ in range(1, layers):
        imgs.append((O.zoom_half(imgs[-1][0]), O.zoom_half(imgs[-1][1])))
    doff = ioff = 0
    init = None
    for n in range(layers - 1, -1, -1):
        c = O.pyr_level_config(pc, n)
        w, h = c.width, c.height
        ref = z["disp_levels"][doff:doff + w * h].reshape(h, w)
        doff += w * h
        ours = O.match(c, imgs[n][0], imgs[n][1], init)["disp"]
        # the WTA writes rows [0, wr); the in-place median's last row reads the unwritten row wr
        wr = (h // 4) * 4 if init is not None else (h // 2) * 2
        rows = np.zeros((h, w), bool)
        rows[:wr - 1] = True
        eq = ours.view(np.uint32) == ref.view(np.uint32)
        assert eq[rows].mean() > 0.999, (n, eq[rows].mean())
        if init is not None and not c.do_remove_peaks and not c.morphology_dilation:
            c2 = O.pyr_level_config(pc, n)
            c2.do_median = 0
            pre = O.match(c2, imgs[n][0], imgs[n][1], init)["disp"]
            bad = np.argwhere(~eq & rows)
            assert not halo_race_unexplained(O, pre, ref, bad, h, w), n
        if n > 0:
            wn, hn = W >> (n - 1), H >> (n - 1)
            ref_init = z["init_levels"][ioff:ioff + wn * hn].reshape(hn, wn)
            ioff += wn * hn
            assert np.array_equal(O.init_next_level(ref, wn, hn), ref_init), n
            init = ref_init


@pytest.mark.parametrize("name", DEPTH)
def test_depth_against_reference(oracle_mod, name):
    """Depth maps of the reference's Init2 / Match2 (both classes): the oracle's disparity turned
    into depth. Exact on the single-level cases without racy stages; the pyramid inherits the
    median races of its disparities."""
    from tests.golden.make_golden import oracle_depth
    z, case = load(name)
    want, rows = oracle_depth(z, case, int(z["peaks_strips"]))
    eq = (want.view(np.uint32) == z["depth"].view(np.uint32))[rows].mean()
    if "num_layers" in case:
        assert eq > 0.9, eq
    elif case.get("post_filter", 0) and (case["morphology"] or case["do_remove_peaks"]):
        # the depth of a smoothed map: the filter's weights come from different exp implementations
        a, b = want[rows], z["depth"][rows]
        assert np.array_equal(a == INV, b == INV)
        ok = a != INV
        np.testing.assert_allclose(a[ok], b[ok], rtol=1e-5)
    else:
        assert eq == 1.0, eq


# post filter / morphology fixtures (620x186, WTA map filtered, no LR check or median)
FILTER_TOL = 3e-5  # px: the oracle's expf/exp are the C library's, the reference's CUDA's (<= 2 ulp per weight)
MORPH = [c for c in CASES if c in ("erosion_only", "open_only", "close_only")]
FILTERED = [c for c in CASES if c in ("gauss_only", "bilateral_only", "gauss_erosion", "bilateral_close")]


def _full_options(O, z, case):
    return O.match(config(O, case, z["peaks_strips"], do_lr_check=case["do_lr_check"], do_median=case["do_median"],
                          morphology=case["morphology"], post_filter=case.get("post_filter", 0)),
                   z["left"], z["right"])["disp"]


@pytest.mark.parametrize("name", MORPH)
def test_morphology_against_reference(oracle_mod, name):
    """Erosion, OPEN, CLOSE of DisparityFilter::Filter (cusgm_df.cu:275-339): exact on every pixel
    (the reference's OPEN leaves the dilation, its CLOSE the erosion)."""
    z, case = load(name)
    full = _full_options(oracle_mod, z, case)
    assert np.array_equal(full.view(np.uint32), z["disp_l"].view(np.uint32)), int((full != z["disp_l"]).sum())


@pytest.mark.parametrize("name", FILTERED)
def test_post_filters_against_reference(oracle_mod, name):
    """Gauss / bilateral smoothing (cusgm_df.cu:94-162), alone and before a morphology step:
    the same INVALID pixels as the reference and values within FILTER_TOL. The smoothing weights
    come from the C library's exp here and from CUDA's in the reference, which differ by an ulp on
    some of the weights, so about half the smoothed values differ in their last bits; the engine,
    which uses CUDA's exp, matches the reference bit for bit (tests/test_gpu_reference_fixtures.py)."""
    z, case = load(name)
    full = _full_options(oracle_mod, z, case)
    ref = z["disp_l"]
    assert np.array_equal(full == INV, ref == INV)
    both = (full != INV) & (ref != INV)
    assert both.mean() > 0.3
    assert float(np.abs(full[both] - ref[both]).max()) <= FILTER_TOL


ROI = sorted(p.stem[4:] for p in GOLDEN.glob("ref_roi*.npz"))


@pytest.mark.parametrize("name", ROI)
def test_roi_against_reference(oracle_mod, name):
    """StereoCuda::Match with regions of interest (left and right view): the left cost (computed
    without the ROI), the right cost on its ROI (5x5: the last pixel of every D-pixel block from the
    ROI's x keeps the left cost), the four path volumes of both views on their ROIs and the WTA map
    inside the left ROI, all as the reference computed them; only the pixels where the reference
    reads path values it never stored (each path's first pixel) are left out."""
    from tests.golden.make_golden import roi_digests, roi_masks, roi_oracle
    z, case = load(name)
    a = roi_oracle(z, case)
    got = roi_digests(a, z, case)
    for k, v in got.items():
        assert v == str(z[k]), k
    _, wm = roi_masks(case["width"], case["height"], tuple(z["roi_l"]), case["min_disp"])
    neq = (a["wta_l"].view(np.uint32) != z["wta_l"].view(np.uint32)) & wm
    assert int(neq.sum()) == 0, np.argwhere(neq)[:5]
    assert wm.mean() > 0.3


def test_roi_fixtures_present():
    assert ROI == ["roi5x5", "roi9x7"], ROI
