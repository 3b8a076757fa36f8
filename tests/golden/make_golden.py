"""Generates the golden fixtures that pin the oracle to the reference itself.

The reference (ethan-li-coding/FasterStereoCuda) ships no tests or golden vectors, so the
fixtures come from running the reference's own code, built from its sources by
oracle/build_ref.sh into oracle/_ref/libsgmref.so:

  python tests/golden/make_golden.py host
      CPU only: the reference's host functions (RemovePeaks, Zoom,
      ComputeInitDispInNextLevel) on seeded inputs -> tests/golden/host_ops.npz

  python tests/golden/make_golden.py refdump --out DIR
      on a CUDA machine: the reference's stage buffers (census, cost, four path volumes,
      WTA, left-right check, filtered output) for the cases below, and its depth maps
      (Init2 / Match2 of both classes) -> DIR/<case>.npz

  python tests/golden/make_golden.py finalize DIR
      compares the dumps with the oracle, prints the agreement, and writes the compact
      fixtures tests/golden/ref_<case>.npz (inputs, reference maps, volume digests).
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from fasterstereocuda_b200 import scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402

GOLDEN = Path(__file__).resolve().parent
REF_LIB = ROOT / "oracle" / "_ref" / "libsgmref.so"
INV = np.float32(-999999.0)


class RefCase(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("min_disp", C.c_int32), ("disp_range", C.c_int32),
                ("cs_type", C.c_int32), ("p1", C.c_int32), ("p2", C.c_int32), ("uniqueness", C.c_float),
                ("do_lr_check", C.c_int32), ("lr_threshold", C.c_float), ("do_median", C.c_int32),
                ("morphology", C.c_int32), ("do_remove_peaks", C.c_int32), ("peaks_ratio", C.c_float),
                ("post_filter", C.c_int32)]


def ref_lib():
    lib = C.CDLL(str(REF_LIB))
    vp = C.c_void_p
    lib.ref_match_dump.argtypes = [C.POINTER(RefCase)] + [vp] * 14
    lib.ref_match_dump.restype = C.c_int
    lib.ref_pyr_match.argtypes = [C.c_int] * 7 + [vp, vp, vp]
    lib.ref_pyr_match.restype = C.c_int
    lib.ref_remove_peaks.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int]
    lib.ref_remove_peaks.restype = C.c_int
    lib.ref_zoom_half.argtypes = [vp, vp, C.c_int, C.c_int]
    lib.ref_init_next_level.argtypes = [vp, vp, C.c_int, C.c_int]
    lib.ref_init_next_level.restype = C.c_int
    lib.ref_hardware_threads_peaks.restype = C.c_int
    lib.ref_last_message.restype = C.c_char_p
    lib.ref_time_match.argtypes = [C.POINTER(RefCase), vp, vp, C.c_int, C.c_int]
    lib.ref_time_match.restype = C.c_double
    lib.ref_pyr_levels.argtypes = [C.c_int] * 7 + [vp, vp, vp, vp]
    lib.ref_pyr_levels.restype = C.c_int
    lib.ref_match2.argtypes = [C.POINTER(RefCase), vp, vp, vp, vp]
    lib.ref_match2.restype = C.c_int
    lib.ref_pyr_match2.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp]
    lib.ref_pyr_match2.restype = C.c_int
    lib.ref_match_roi_dump.argtypes = [C.POINTER(RefCase), vp, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.ref_match_roi_dump.restype = C.c_int
    return lib


def _p(a):
    return None if a is None else a.ctypes.data


# ----------------------------------------------------------------------------- cases
def _init_from_coarse(left, right, cs_type, p1, p2):
    """Initial disparity of a D=32 level: the oracle's matching of the half-resolution pair,
    propagated with the next-level rule (as the pyramid does)."""
    h, w = left.shape
    lh, rh = O.zoom_half(left), O.zoom_half(right)
    cfg = O.Config(width=w // 2, height=h // 2, disp_range=64, cs_type=cs_type, p1=p1, p2=p2, uniqueness=1.0,
                   do_lr_check=1, do_median=1, morphology_dilation=1)
    coarse = O.match(cfg, lh, rh)["disp"]
    return O.init_next_level(coarse, w, h)


def cases():
    """name -> (RefCase fields, left, right, init or None, dump volumes)"""
    out = {}
    base = dict(min_disp=0, disp_range=64, cs_type=1, p1=10, p2=150, uniqueness=0.95, do_lr_check=1,
                lr_threshold=1.0, do_median=1, morphology=0, do_remove_peaks=0, peaks_ratio=0.0005)
    L, R, _ = scenes.planar_pair(11, 162, 120)
    out["c9x7"] = (dict(base, width=162, height=120), L, R, None, True)
    L, R, _ = scenes.planar_pair(12, 162, 120)
    out["c5x5"] = (dict(base, width=162, height=120, cs_type=0, p1=8, p2=32), L, R, None, True)
    L, R, _ = scenes.planar_pair(13, 130, 100, dmin=0.0, dmax=50.0)
    out["negmin"] = (dict(base, width=130, height=100, min_disp=-4), L, R, None, True)
    L, R, _ = scenes.planar_pair(14, 162, 120)
    init = _init_from_coarse(L, R, 1, 10, 150)
    out["init9x7"] = (dict(base, width=162, height=120, disp_range=32, uniqueness=1.0, do_lr_check=0), L, R, init,
                      True)
    L, R, _ = scenes.planar_pair(15, 162, 120)
    init = _init_from_coarse(L, R, 0, 8, 32)
    out["init5x5"] = (dict(base, width=162, height=120, disp_range=32, cs_type=0, p1=8, p2=32, do_lr_check=0), L, R,
                      init, True)
    L, R, _ = scenes.cone_like(16)
    out["cfg0"] = (dict(base, width=450, height=375), L, R, None, False)
    out["cfg0_peaks"] = (dict(base, width=450, height=375, do_lr_check=0, do_remove_peaks=1, peaks_ratio=0.0005), L,
                         R, None, False)
    L, R, _ = scenes.kitti_like(17, 621, 187)
    out["kitti_half"] = (dict(base, width=621, height=187, morphology=2, do_remove_peaks=1, peaks_ratio=0.005), L, R,
                         None, False)
    # deterministic filter stages: no LR check, no median (their races stay out)
    out["dil_only"] = (dict(base, width=621, height=187, do_lr_check=0, do_median=0, morphology=2), L, R, None, False)
    out["peaks_only"] = (dict(base, width=621, height=187, do_lr_check=0, do_median=0, do_remove_peaks=1,
                              peaks_ratio=0.005), L, R, None, False)
    # post filters and morphology (DisparityFilter::Filter, cusgm_df.cu:275-339) on the WTA map
    # (no LR check, no median: both race in the reference); each writes a separate buffer. An even
    # height: the WTA writes every row, so no filter window reads a row the reference leaves unset
    L, R, _ = scenes.kitti_like(19, 620, 186)
    flt = dict(base, width=620, height=186, do_lr_check=0, do_median=0)
    out["gauss_only"] = (dict(flt, post_filter=1), L, R, None, False)
    out["bilateral_only"] = (dict(flt, post_filter=2), L, R, None, False)
    out["erosion_only"] = (dict(flt, morphology=1), L, R, None, False)
    out["open_only"] = (dict(flt, morphology=3), L, R, None, False)
    out["close_only"] = (dict(flt, morphology=4), L, R, None, False)
    out["gauss_erosion"] = (dict(flt, post_filter=1, morphology=1), L, R, None, False)
    out["bilateral_close"] = (dict(flt, post_filter=2, morphology=4), L, R, None, False)
    return out


# single-level cases whose final map comes from a post filter (compared within FILTER_TOL of the
# reference's map on the CPU: the oracle's expf/exp are the C library's, the reference's CUDA's)
FILTER_CASES = ("gauss_only", "bilateral_only", "gauss_erosion", "bilateral_close")


# Matches with regions of interest (StereoCuda::Match with StereoROI_T, cusgm_cc.cu:478-488,
# cusgm_ca.cu:3991-3999 / 4139-4165 / 4173-4192): name -> (seed, case fields, left ROI, right ROI),
# rectangles (x, y, w, h) inside the image with widths a multiple of 4 (see ref_match_roi_dump)
ROI_CASES = {
    "roi9x7": (31, dict(width=162, height=120, cs_type=1, p1=10, p2=150), (20, 16, 100, 80), (8, 10, 120, 90)),
    "roi5x5": (32, dict(width=162, height=120, cs_type=0, p1=8, p2=32), (12, 5, 136, 99), (4, 7, 140, 101)),
}


def roi_region(roi, min_disp):
    """Columns [x0, x1) and rows [y0, y1) of a view's region (columns start at max(0, min_disp))."""
    x, y, w, h = roi
    return max(x, max(0, min_disp)), x + w, y, y + h


def roi_masks(W, H, roi, min_disp):
    """(paths mask [4][H][W], WTA mask [H][W]) of the pixels a region's dumps are compared on: its
    path values except each path's first pixel (the reference never stores it, so the WTA reads
    what the buffer held there), and the pixels its WTA writes away from those first lines."""
    x0, x1, y0, y1 = roi_region(roi, min_disp)
    reg = np.zeros((H, W), bool)
    reg[y0:y1, x0:x1] = True
    first = np.zeros((4, H, W), bool)
    first[0, y0, x0:x1] = True        # top -> bottom
    first[1, y0:y1, x0] = True        # left -> right
    first[2, y1 - 1, x0:x1] = True    # bottom -> top
    first[3, y0:y1, x1 - 1] = True    # right -> left
    paths = np.broadcast_to(reg, (4, H, W)) & ~first
    wta = np.zeros((H, W), bool)
    wta[y0:y0 + ((y1 - y0) // 2) * 2, x0:x1] = True
    wta &= ~first.any(0)
    return paths, wta


# name: (seed, width, height, min_disp, max_disp, layers, lr check, small-region removal)
PYR_CASES = {"pyr_kitti": (17, 1242, 375, 0, 64, 3, 1, 1), "pyr_cone": (16, 450, 375, 0, 64, 2, 1, 1),
             "pyr_kitti_nolr": (18, 1242, 375, 0, 64, 3, 0, 1)}

# Depth output (Init2 / Match2). Camera: x0_left, y0_left, x0_right, y0_right, focus, baseline.
CAM = (600.0, 180.0, 610.0, 180.0, 720.0, 540.0)
# single-level cases (from cases()) whose stages have no thread races, matched to depth: with one
# of post filter / morphology and no small-region removal the reference takes the depth from the
# map before that filter (StereoCudaImpl::Match2, StereoCudaImpl.cpp:548-583)
DEPTH_CASES = ("peaks_only", "dil_only", "gauss_only", "erosion_only", "gauss_erosion")
# name: (seed, width, height, min_depth, max_depth, layers, lr check, small-region removal)
DEPTH_PYR_CASES = {"depthpyr_kitti": (43, 1242, 375, 5000.0, 60000.0, 3, 1, 1)}


# ----------------------------------------------------------------------------- host ops
def make_host():
    lib = ref_lib()
    rng = np.random.Generator(np.random.PCG64(7))
    fx = {}
    # small-region removal: piecewise-constant maps with noise, INVALID holes, one strip each
    for k, (w, h) in enumerate([(64, 32), (97, 41), (128, 16)]):
        blocks = rng.integers(0, 12, size=(h // 4 + 1, w // 4 + 1)).astype(np.float32)
        d = np.kron(blocks, np.ones((4, 4), np.float32))[:h, :w] * 1.7
        d += rng.normal(0, 0.45, size=d.shape).astype(np.float32)
        d[rng.random(d.shape) < 0.1] = INV
        for thr in (3, 11, 40):
            out = d.copy()
            seg = np.zeros(d.shape, np.int32)
            n = lib.ref_remove_peaks(_p(out), _p(seg), w, h, thr)
            fx[f"peaks_{k}_{thr}_in"] = d
            fx[f"peaks_{k}_{thr}_out"] = out
            fx[f"peaks_{k}_{thr}_n"] = np.int32(n)
    # decimation
    for k, (w, h) in enumerate([(31, 17), (64, 48), (101, 77)]):
        img = rng.integers(0, 256, size=(h, w), dtype=np.uint8)
        out = np.zeros((h // 2, w // 2), np.uint8)
        lib.ref_zoom_half(_p(img), _p(out), w, h)
        fx[f"zoom_{k}_in"], fx[f"zoom_{k}_out"] = img, out
    # next-level initial disparity (odd and even sizes); one spare INVALID after the coarse map
    # absorbs the reference's read past the end for odd widths
    for k, (w, h) in enumerate([(64, 48), (65, 48), (63, 47), (621, 187)]):
        cur = rng.uniform(0, 30, size=(h // 2, w // 2)).astype(np.float32)
        cur[rng.random(cur.shape) < 0.15] = INV
        buf = np.concatenate([cur.reshape(-1), [INV]]).astype(np.float32)
        nxt = np.zeros((h, w), np.int16)
        lib.ref_init_next_level(_p(buf), _p(nxt), w, h)
        fx[f"initnext_{k}_in"], fx[f"initnext_{k}_out"] = cur, nxt
        fx[f"initnext_{k}_size"] = np.array([w, h], np.int32)
    np.savez_compressed(GOLDEN / "host_ops.npz", **fx)
    print("wrote", GOLDEN / "host_ops.npz", len(fx), "arrays")


# ----------------------------------------------------------------------------- reference dumps
def refdump(out_dir: Path, only=None):
    lib = ref_lib()
    out_dir.mkdir(parents=True, exist_ok=True)
    meta = {"peaks_strips": lib.ref_hardware_threads_peaks()}
    for name, (f, L, R, init, vols) in cases().items():
        if only and name not in only:
            continue
        c = RefCase(**f)
        W, H, D = f["width"], f["height"], f["disp_range"]
        arr = {}
        if vols:
            arr.update(census_l=np.zeros((H, W), np.uint64), census_r=np.zeros((H, W), np.uint64),
                       cost_lr=np.zeros((H, W, D), np.uint8), paths_lr=np.zeros((4, H, W, D), np.uint8),
                       cost_rl=np.zeros((H, W, D), np.uint8), paths_rl=np.zeros((4, H, W, D), np.uint8))
        arr.update(wta_l=np.zeros((H, W), np.float32), lr_l=np.zeros((H, W), np.float32),
                   lr_r=np.zeros((H, W), np.float32), disp_l=np.zeros((H, W), np.float32),
                   disp_r=np.zeros((H, W), np.float32))
        g = arr.get
        rc = lib.ref_match_dump(C.byref(c), _p(L), _p(R), _p(init), _p(g("census_l")), _p(g("census_r")),
                                _p(g("cost_lr")), _p(g("paths_lr")), _p(g("wta_l")), _p(g("cost_rl")),
                                _p(g("paths_rl")), _p(g("lr_l")), _p(g("lr_r")), _p(g("disp_l")), _p(g("disp_r")))
        print(name, "rc", rc, lib.ref_last_message().decode(), flush=True)
        if rc != 0:
            continue
        extra = {} if init is None else {"init": init}
        np.savez_compressed(out_dir / f"{name}.npz", left=L, right=R, case=np.array(json.dumps(f)), **extra, **arr)
    for name, (seed, w, h, dmin, dmax, layers, lr, pk) in PYR_CASES.items():
        if only and name not in only:
            continue
        if name.startswith("pyr_kitti"):
            L, R, _ = scenes.kitti_like(seed, w, h)
        else:
            L, R, _ = scenes.cone_like(seed)
        assert L.shape == (h, w) and R.shape == (h, w), (name, L.shape)
        disp = np.zeros((h, w), np.float32)
        rc = lib.ref_pyr_match(w, h, dmin, dmax, layers, lr, pk, _p(L), _p(R), _p(disp))
        print(name, "rc", rc, lib.ref_last_message().decode(), flush=True)
        if rc == 0:
            np.savez_compressed(out_dir / f"{name}.npz", left=L, right=R, disp=disp,
                                case=np.array(json.dumps(dict(width=w, height=h, min_disp=dmin, max_disp=dmax,
                                                              num_layers=layers, lr=lr, peaks=pk))))
        n_d = sum((w >> i) * (h >> i) for i in range(layers))
        n_i = sum((w >> i) * (h >> i) for i in range(layers - 1))
        dl = np.zeros(n_d, np.float32)
        il = np.zeros(max(n_i, 1), np.int16)
        rc = lib.ref_pyr_levels(w, h, dmin, dmax, layers, lr, pk, _p(L), _p(R), _p(dl), _p(il))
        print(name, "levels rc", rc, lib.ref_last_message().decode(), flush=True)
        if rc == 0:
            np.savez_compressed(out_dir / f"levels_{name}.npz", left=L, right=R, disp_levels=dl, init_levels=il,
                                case=np.array(json.dumps(dict(width=w, height=h, min_disp=dmin, max_disp=dmax,
                                                              num_layers=layers, lr=lr, peaks=pk))))
    base = dict(min_disp=0, disp_range=64, uniqueness=0.95, do_lr_check=1, lr_threshold=1.0, do_median=0,
                morphology=0, do_remove_peaks=0, peaks_ratio=0.0005, post_filter=0)
    for name, (seed, f, rl, rr) in ROI_CASES.items():
        if only and name not in only:
            continue
        f = dict(base, **f)
        W, H, D = f["width"], f["height"], f["disp_range"]
        L, R, _ = scenes.planar_pair(seed, W, H)
        arr = dict(cost_lr=np.zeros((H, W, D), np.uint8), paths_lr=np.zeros((4, H, W, D), np.uint8),
                   wta_l=np.zeros((H, W), np.float32), cost_rl=np.zeros((H, W, D), np.uint8),
                   paths_rl=np.zeros((4, H, W, D), np.uint8))
        a_l, a_r = np.array(rl, np.int32), np.array(rr, np.int32)
        rc = lib.ref_match_roi_dump(C.byref(RefCase(**f)), _p(L), _p(R), _p(a_l), _p(a_r), _p(arr["cost_lr"]),
                                    _p(arr["paths_lr"]), _p(arr["wta_l"]), _p(arr["cost_rl"]), _p(arr["paths_rl"]))
        print(name, "rc", rc, lib.ref_last_message().decode(), flush=True)
        if rc == 0:
            np.savez_compressed(out_dir / f"{name}.npz", left=L, right=R, roi_l=a_l, roi_r=a_r,
                                case=np.array(json.dumps(f)), **arr)
    cam = np.array(CAM, np.float64)
    all_cases = cases()
    for base_name in DEPTH_CASES:
        name = "depth_" + base_name
        if only and name not in only:
            continue
        f, L, R, _, _ = all_cases[base_name]
        depth = np.zeros((f["height"], f["width"]), np.float32)
        rc = lib.ref_match2(C.byref(RefCase(**f)), _p(cam), _p(L), _p(R), _p(depth))
        print(name, "rc", rc, lib.ref_last_message().decode(), flush=True)
        if rc == 0:
            np.savez_compressed(out_dir / f"{name}.npz", left=L, right=R, depth=depth, cam=cam,
                                case=np.array(json.dumps(f)))
    epi = np.array([CAM[0], CAM[1], CAM[2], CAM[3], CAM[5], CAM[4]], np.float64)  # baseline before focus
    for name, (seed, w, h, zmin, zmax, layers, lr, pk) in DEPTH_PYR_CASES.items():
        if only and name not in only:
            continue
        m0, d0 = O.pyr_init2_coarsest(w, layers, zmin, zmax, CAM[0], CAM[2], CAM[4], CAM[5])
        if d0 != 64:  # the reference's 128- and 256-disparity kernels index shared memory out of range
            print(name, "skipped: coarsest range", d0, flush=True)
            continue
        L, R, _ = scenes.kitti_like(seed, w, h)
        depth = np.zeros((h, w), np.float32)
        rc = lib.ref_pyr_match2(w, h, zmin, zmax, layers, lr, pk, _p(epi), _p(L), _p(R), _p(depth))
        print(name, "rc", rc, lib.ref_last_message().decode(), flush=True)
        if rc == 0:
            np.savez_compressed(out_dir / f"{name}.npz", left=L, right=R, depth=depth, cam=cam,
                                case=np.array(json.dumps(dict(width=w, height=h, min_depth=zmin, max_depth=zmax,
                                                              num_layers=layers, lr=lr, peaks=pk))))
    (out_dir / "meta.json").write_text(json.dumps(meta))
    print("meta", meta)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _eq(a, b):
    return np.asarray(a).view(np.uint8).reshape(-1).tobytes() == np.asarray(b).view(np.uint8).reshape(-1).tobytes()


def path_first_pixel_mask(W, H, x0):
    """[4][H][W] mask of the first pixel of every path (never stored by the reference)."""
    m = np.zeros((4, H, W), bool)
    m[0, 0, x0:] = True
    m[2, H - 1, x0:] = True
    m[1, :, x0] = True
    m[3, :, W - 1] = True
    return m


def _race_free_lr(O, wta_l, wta_r, thr):
    """Pixels whose LR result is the same whether the right map is read before or after every
    invalidation (the reference reads it while other threads invalidate it)."""
    a = wta_l.copy()
    marks = wta_r.copy()
    O.lib().orc_lr_check(a.ctypes.data, wta_r.ctypes.data, marks.ctypes.data, a.shape[1], a.shape[0], C.c_float(thr))
    b = wta_l.copy()
    O.lib().orc_lr_check(b.ctypes.data, marks.ctypes.data, None, b.shape[1], b.shape[0], C.c_float(thr))
    return a.view(np.uint32) == b.view(np.uint32), a


def _race_free_median(O, inp):
    """Pixels whose median is the same when neighbouring blocks of the reference's in-place
    median (30x2 outputs per block) have already written their filtered values."""
    H, W = inp.shape
    snap = O.median3x3(inp)
    mixed = inp.copy()
    ys, xs = np.mgrid[0:H, 0:W]
    # a block writes rows 2by+1..2by+2 and columns 30bx+1..30bx+30; its halo rows/columns belong to others
    boundary_rows = (ys % 2 == 0) | (ys % 2 == 1)
    mixed[boundary_rows] = snap[boundary_rows]
    alt = O.median3x3(mixed)
    return snap.view(np.uint32) == alt.view(np.uint32), snap


def _levels_report(z, case, meta):
    """Per level: the oracle's level output given the reference's own input to that level (the
    previous level's initial disparity computed by the reference), so races do not cascade."""
    W, H, layers = case["width"], case["height"], case["num_layers"]
    pc = O.PyrConfig(width=W, height=H, min_disp=case["min_disp"], max_disp=case["max_disp"], num_layers=layers,
                     override_enable=0, peaks_strips=meta["peaks_strips"], do_lr_check=case.get("lr", 1),
                     do_rm_peaks=case.get("peaks", 1))
    imgs = [(z["left"], z["right"])]
    for i in range(1, layers):
        imgs.append((O.zoom_half(imgs[-1][0]), O.zoom_half(imgs[-1][1])))
    out, doff, ioff = {}, 0, 0
    init = None
    for n in range(layers - 1, -1, -1):
        c = O.pyr_level_config(pc, n)
        w, h = c.width, c.height
        ref_d = z["disp_levels"][doff:doff + w * h].reshape(h, w)
        doff += w * h
        ours = O.match(c, imgs[n][0], imgs[n][1], init)["disp"]
        # rows the WTA writes, minus the last one (the in-place median reads the unwritten row)
        wr = (h // 4) * 4 if init is not None else (h // 2) * 2
        out[f"level{n}"] = float((ours[:wr - 1].view(np.uint32) == ref_d[:wr - 1].view(np.uint32)).mean())
        if n > 0:
            wn, hn = W >> (n - 1), H >> (n - 1)
            ref_init = z["init_levels"][ioff:ioff + wn * hn].reshape(hn, wn)
            ioff += wn * hn
            mine = O.init_next_level(ref_d, wn, hn)
            out[f"init{n - 1}"] = float((mine == ref_init).mean())
            init = ref_init
    return out


def oracle_depth(z, case, peaks_strips):
    """The oracle's depth map for a depth dump (single level or pyramid), with the rows the
    reference writes."""
    cam = z["cam"]
    if "num_layers" in case:  # pyramid: the coarsest range from the depth range, as Init2 derives it
        layers = case["num_layers"]
        m0, d0 = O.pyr_init2_coarsest(case["width"], layers, case["min_depth"], case["max_depth"], cam[0], cam[2],
                                      cam[4], cam[5])
        s = 2 ** (layers - 1)
        pc = O.PyrConfig(width=case["width"], height=case["height"], min_disp=m0 * s, max_disp=(m0 + d0) * s,
                         num_layers=layers, override_enable=0, peaks_strips=peaks_strips,
                         do_lr_check=case["lr"], do_rm_peaks=case["peaks"])
        d = O.pyr_match(pc, z["left"], z["right"])
    else:
        cfg = O.Config(width=case["width"], height=case["height"], min_disp=case["min_disp"],
                       disp_range=case["disp_range"], cs_type=case["cs_type"], p1=case["p1"], p2=case["p2"],
                       uniqueness=case["uniqueness"], do_lr_check=case["do_lr_check"],
                       lr_threshold=case["lr_threshold"], do_median=case["do_median"],
                       morphology=case["morphology"], post_filter=case.get("post_filter", 0),
                       do_remove_peaks=case["do_remove_peaks"], peaks_ratio=case["peaks_ratio"],
                       peaks_strips=peaks_strips, tie_rule=4, init_tie_rule=4)
        d = O.match(O.depth_source_config(cfg), z["left"], z["right"])["disp"]
    rows = np.zeros(d.shape, bool)
    rows[:d.shape[0] - 1 if d.shape[0] % 2 else d.shape[0]] = True  # the reference never writes the last odd row
    return O.depth_from_disp(d, cam[0], cam[2], cam[4], cam[5]), rows


def roi_oracle(z, case):
    """The oracle's left and right views of a ROI case (LR check on, median off)."""
    cfg = O.Config(width=case["width"], height=case["height"], min_disp=case["min_disp"],
                   disp_range=case["disp_range"], cs_type=case["cs_type"], p1=case["p1"], p2=case["p2"],
                   uniqueness=case["uniqueness"], do_lr_check=1, do_median=0, tie_rule=4, init_tie_rule=4)
    a = O.match(cfg.with_roi(tuple(z["roi_l"]), tuple(z["roi_r"])), z["left"], z["right"], dump=True,
                want_right=True)
    return a


def roi_digests(a, z, case):
    """Digests of the compared parts of a ROI case's volumes (zeros elsewhere)."""
    W, H, M = case["width"], case["height"], case["min_disp"]
    pm_l, _ = roi_masks(W, H, tuple(z["roi_l"]), M)
    pm_r, _ = roi_masks(W, H, tuple(z["roi_r"]), M)
    cm_l = np.zeros((H, W), bool)
    cm_l[:, max(0, M):] = True  # the left view's cost is computed without the ROI
    x0, x1, y0, y1 = roi_region(tuple(z["roi_r"]), M)
    cm_r = np.zeros((H, W), bool)
    cm_r[y0:y1, x0:x1] = True
    cost_lr = a["cost"] if "cost" in a else a["cost_lr"]   # oracle dump keys / reference dump keys
    paths_lr = a["paths"] if "paths" in a else a["paths_lr"]
    return {"digest_cost_lr": digest(np.where(cm_l[..., None], cost_lr, 0)),
            "digest_paths_lr": digest(np.where(pm_l[..., None], paths_lr, 0)),
            "digest_cost_rl": digest(np.where(cm_r[..., None], a["cost_rl"], 0)),
            "digest_paths_rl": digest(np.where(pm_r[..., None], a["paths_rl"], 0))}


def roi_report(z, case, meta):
    a = roi_oracle(z, case)
    ours = roi_digests(a, z, case)
    ref = roi_digests(z, z, case)
    W, H, M = case["width"], case["height"], case["min_disp"]
    _, wm = roi_masks(W, H, tuple(z["roi_l"]), M)
    r = {k: ours[k] == ref[k] for k in ours}
    r["wta_compared"] = float((a["wta_l"].view(np.uint32) == z["wta_l"].view(np.uint32))[wm].mean())
    keep = {k: z[k] for k in ("left", "right", "roi_l", "roi_r", "wta_l", "case")}
    keep.update({k: np.array(v) for k, v in ref.items()})
    return r, keep


def depth_report(z, case, meta):
    want, rows = oracle_depth(z, case, meta["peaks_strips"])
    return {"depth_equal": float((want.view(np.uint32) == z["depth"].view(np.uint32))[rows].mean())}


def finalize(dump_dir: Path, write: bool = True):
    meta = json.loads((dump_dir / "meta.json").read_text())
    report = {}
    for f in sorted(dump_dir.glob("*.npz")):
        z = dict(np.load(f))
        name = f.stem
        case = json.loads(str(z["case"]))
        if name.startswith("levels_"):
            report[name] = _levels_report(z, case, meta)
            if write:
                np.savez_compressed(GOLDEN / f"ref_{name}.npz", **z, peaks_strips=np.int32(meta["peaks_strips"]))
            continue
        if name.startswith("roi"):
            report[name], keep = roi_report(z, case, meta)
            if write:
                np.savez_compressed(GOLDEN / f"ref_{name}.npz", **keep)
            continue
        if name.startswith("depth"):
            report[name] = depth_report(z, case, meta)
            if write:
                np.savez_compressed(GOLDEN / f"ref_{name}.npz", left=z["left"], right=z["right"], depth=z["depth"],
                                    cam=z["cam"], case=z["case"], peaks_strips=np.int32(meta["peaks_strips"]))
            continue
        if name.startswith("pyr_"):
            pc = O.PyrConfig(width=case["width"], height=case["height"], min_disp=case["min_disp"],
                             max_disp=case["max_disp"], num_layers=case["num_layers"], override_enable=0,
                             peaks_strips=meta["peaks_strips"], do_lr_check=case.get("lr", 1),
                             do_rm_peaks=case.get("peaks", 1))
            d = O.pyr_match(pc, z["left"], z["right"])
            same = (d.view(np.uint32) == z["disp"].view(np.uint32))
            report[name] = {"disp_equal": float(same[:case["height"] - 1].mean())}
            if write:
                np.savez_compressed(GOLDEN / f"ref_{name}.npz", left=z["left"], right=z["right"], disp=z["disp"],
                                    case=z["case"], peaks_strips=np.int32(meta["peaks_strips"]))
            continue
        W, H, D = case["width"], case["height"], case["disp_range"]
        init = z.get("init")
        x0 = max(0, case["min_disp"])
        cfg = O.Config(width=W, height=H, min_disp=case["min_disp"], disp_range=D, cs_type=case["cs_type"],
                       p1=case["p1"], p2=case["p2"], uniqueness=case["uniqueness"], do_lr_check=1, do_median=0,
                       peaks_strips=meta["peaks_strips"], tie_rule=4, init_tie_rule=4)
        r = {}
        a = O.match(cfg, z["left"], z["right"], init, dump=True, want_right=True)
        written = np.zeros((H, W), bool)
        written[:(H // 4) * 4 if init is not None else (H // 2) * 2, x0:] = True
        if "census_l" in z:
            r["census_l"] = _eq(a["census_l"], z["census_l"])
            r["census_r"] = _eq(a["census_r"], z["census_r"])
            cm = np.zeros((H, W), bool)
            cm[:, x0:] = True
            fm = path_first_pixel_mask(W, H, x0)
            valid = np.broadcast_to(cm, (4, H, W)) & ~fm
            if init is not None:
                valid = valid & np.broadcast_to(init != -32768, (4, H, W))
            for tag, ours_c, ours_p in (("lr", a["cost"], a["paths"]), ("rl", a.get("cost_rl"), a.get("paths_rl"))):
                if ours_c is None or ("cost_" + tag) not in z:
                    continue
                if tag == "rl" and init is not None:
                    continue  # right view of an init level: right initial disparities differ by design
                r["cost_" + tag] = float((ours_c == z["cost_" + tag]).all(-1)[cm].mean())
                pe = (ours_p == z["paths_" + tag]).all(-1)
                r["paths_" + tag] = [float(pe[k][valid[k]].mean()) for k in range(4)]
        r["wta_written"] = float((a["wta_l"].view(np.uint32) == z["wta_l"].view(np.uint32))[written].mean())
        # LR stage (run B: LR on, median off) -- only on plain levels (init levels have no LR in the pyramid)
        if init is None:
            rf, lr_ours = _race_free_lr(O, a["wta_l"], a["wta_r"], case["lr_threshold"])
            eq = lr_ours.view(np.uint32) == z["lr_l"].view(np.uint32)
            r["lr_all"] = float(eq[written].mean())
            r["lr_race_free"] = float(eq[written & rf].mean())
            r["lr_race_free_frac"] = float(rf[written].mean())
            r["lr_right_all"] = float((a["disp_r"].view(np.uint32) == z["lr_r"].view(np.uint32))[written].mean())
        # full options
        cf = O.Config(**{**cfg.__dict__, "do_lr_check": case["do_lr_check"], "do_median": case["do_median"],
                         "morphology": case["morphology"], "post_filter": case.get("post_filter", 0),
                         "do_remove_peaks": case["do_remove_peaks"], "peaks_ratio": case["peaks_ratio"]})
        full = O.match(cf, z["left"], z["right"], init)["disp"]
        rows = np.zeros((H, W), bool)
        rows[:H - 1 if H % 2 else H] = True  # the reference never writes the last odd row
        eq = full.view(np.uint32) == z["disp_l"].view(np.uint32)
        r["disp_all"] = float(eq[rows].mean())
        if case.get("post_filter", 0):
            a_, b_ = full[rows], z["disp_l"][rows]
            both = (a_ != INV) & (b_ != INV)
            r["disp_invalid_equal"] = bool(np.array_equal(a_ == INV, b_ == INV))
            r["disp_max_abs_diff"] = float(np.abs(a_[both] - b_[both]).max()) if both.any() else 0.0
        if case["do_median"] and not case["do_remove_peaks"] and case["morphology"] == 0:
            pre = z["lr_l"] if case["do_lr_check"] else z["wta_l"]
            mf, _ = _race_free_median(O, pre)
            mf[-2:] = False
            r["disp_median_race_free"] = float(eq[rows & mf].mean())
            r["median_race_free_frac"] = float(mf[rows].mean())
        report[name] = r
        if write:
            keep = {k: z[k] for k in ("left", "right", "wta_l", "lr_l", "lr_r", "disp_l", "case") if k in z}
            if init is not None:
                keep["init"] = init
            if "census_l" in z:
                keep["digest_census"] = np.array(digest(np.stack([z["census_l"], z["census_r"]])))
                keep["digest_cost_lr"] = np.array(digest(np.where(cm[..., None], z["cost_lr"], 0)))
                pz = np.where(valid[..., None], z["paths_lr"], 0)
                keep["digest_paths_lr"] = np.array(digest(pz))
            keep["peaks_strips"] = np.int32(meta["peaks_strips"])
            np.savez_compressed(GOLDEN / f"ref_{name}.npz", **keep)
    print(json.dumps(report, indent=1))
    if write:
        (GOLDEN / "ref_agreement.json").write_text(json.dumps(report, indent=1) + "\n")
    return report


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    sub.add_parser("host")
    d = sub.add_parser("refdump")
    d.add_argument("--out", required=True)
    d.add_argument("--only", nargs="*")
    f = sub.add_parser("finalize")
    f.add_argument("dir")
    f.add_argument("--no-write", action="store_true")
    a = ap.parse_args()
    if a.cmd == "host":
        make_host()
    elif a.cmd == "refdump":
        refdump(Path(a.out), a.only)
    else:
        finalize(Path(a.dir), not a.no_write)


if __name__ == "__main__":
    main()
