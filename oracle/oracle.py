"""ctypes binding of the C oracle (oracle/sgm_oracle.c) -- test infrastructure only.

Every function returns numpy arrays in the dense layouts described in sgm_oracle.h.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, fields
from pathlib import Path

import numpy as np

_LIB = Path(__file__).resolve().parent / "_build" / "liborc.so"
_lib = None

INVALID_FLOAT = np.float32(-999999.0)
INVALID_SHORT = np.int16(-32768)


class _Cfg(C.Structure):
    _fields_ = [(n, t) for n, t in [
        ("width", C.c_int32), ("height", C.c_int32), ("min_disp", C.c_int32), ("disp_range", C.c_int32),
        ("cs_type", C.c_int32), ("p1", C.c_int32), ("p2", C.c_int32), ("uniqueness", C.c_float),
        ("do_lr_check", C.c_int32), ("lr_threshold", C.c_float), ("do_median", C.c_int32),
        ("morphology_dilation", C.c_int32), ("do_remove_peaks", C.c_int32), ("peaks_ratio", C.c_float),
        ("peaks_strips", C.c_int32), ("peaks_abs_mode", C.c_int32), ("tie_rule", C.c_int32),
        ("init_tie_rule", C.c_int32), ("p2_div0", C.c_int32), ("threads", C.c_int32),
        ("post_filter", C.c_int32), ("morphology", C.c_int32),
        ("roi_l_enable", C.c_int32), ("roi_l_x", C.c_int32), ("roi_l_y", C.c_int32), ("roi_l_w", C.c_int32),
        ("roi_l_h", C.c_int32), ("roi_r_enable", C.c_int32), ("roi_r_x", C.c_int32), ("roi_r_y", C.c_int32),
        ("roi_r_w", C.c_int32), ("roi_r_h", C.c_int32)]]


class _PyrCfg(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "width", "height", "min_disp", "max_disp", "num_layers", "do_lr_check", "do_rm_peaks", "do_smooth",
        "override_enable", "cs_type", "p1", "p2", "peaks_strips", "peaks_abs_mode", "tie_rule", "init_tie_rule",
        "p2_div0", "threads")]


@dataclass
class Config:
    """One matching level (mirrors orc_config_t)."""
    width: int
    height: int
    min_disp: int = 0
    disp_range: int = 64
    cs_type: int = 1
    p1: int = 10
    p2: int = 150
    uniqueness: float = 0.95
    do_lr_check: int = 1
    lr_threshold: float = 1.0
    do_median: int = 1
    morphology_dilation: int = 0
    do_remove_peaks: int = 0
    peaks_ratio: float = 0.0005
    peaks_strips: int = 6
    peaks_abs_mode: int = 0
    tie_rule: int = 4
    init_tie_rule: int = 4
    p2_div0: int = -1
    threads: int = 0
    post_filter: int = 0
    morphology: int = 0
    roi_l_enable: int = 0
    roi_l_x: int = 0
    roi_l_y: int = 0
    roi_l_w: int = 0
    roi_l_h: int = 0
    roi_r_enable: int = 0
    roi_r_x: int = 0
    roi_r_y: int = 0
    roi_r_w: int = 0
    roi_r_h: int = 0

    def with_roi(self, left=None, right=None) -> "Config":
        """A copy with the regions of interest (x, y, w, h) of the left / right view."""
        kw = dict(self.__dict__)
        for tag, r in (("l", left), ("r", right)):
            if r is not None:
                kw.update({f"roi_{tag}_enable": 1, f"roi_{tag}_x": r[0], f"roi_{tag}_y": r[1], f"roi_{tag}_w": r[2],
                           f"roi_{tag}_h": r[3]})
        return Config(**kw)

    def c(self) -> _Cfg:
        s = _Cfg()
        for f in fields(self):
            setattr(s, f.name, getattr(self, f.name))
        return s


@dataclass
class PyrConfig:
    width: int
    height: int
    min_disp: int = 0
    max_disp: int = 64
    num_layers: int = 3
    do_lr_check: int = 1
    do_rm_peaks: int = 1
    do_smooth: int = 0
    override_enable: int = 1
    cs_type: int = 1
    p1: int = 10
    p2: int = 150
    peaks_strips: int = 6
    peaks_abs_mode: int = 0
    tie_rule: int = 4
    init_tie_rule: int = 4
    p2_div0: int = -1
    threads: int = 0

    def c(self) -> _PyrCfg:
        s = _PyrCfg()
        for f in fields(self):
            setattr(s, f.name, int(getattr(self, f.name)))
        return s


def lib():
    global _lib
    if _lib is None:
        if not _LIB.exists():
            from fasterstereocuda_b200.build import build_oracle
            build_oracle()
        _lib = C.CDLL(str(_LIB))
        vp, i32 = C.c_void_p, C.c_int32
        _lib.orc_match_dump.argtypes = [C.POINTER(_Cfg)] + [vp] * 13
        _lib.orc_match_dump.restype = i32
        _lib.orc_pyr_match.argtypes = [C.POINTER(_PyrCfg), vp, vp, vp]
        _lib.orc_pyr_match.restype = i32
        _lib.orc_pyr_level_config.argtypes = [C.POINTER(_PyrCfg), i32, C.POINTER(_Cfg)]
        _lib.orc_pyr_level_config.restype = i32
        _lib.orc_census.argtypes = [vp, i32, i32, i32, i32, vp]
        _lib.orc_remove_peaks.argtypes = [vp, i32, i32, i32, C.c_float, i32]
        _lib.orc_remove_peaks.restype = i32
        _lib.orc_remove_peaks_strip.argtypes = [vp, i32, i32, i32, i32]
        _lib.orc_remove_peaks_strip.restype = i32
        _lib.orc_zoom_half.argtypes = [vp, i32, i32, vp]
        _lib.orc_init_next_level.argtypes = [vp, i32, i32, vp, i32, i32]
        _lib.orc_median3x3.argtypes = [vp, vp, i32, i32]
        _lib.orc_dilation.argtypes = [vp, vp, i32, i32, i32]
        _lib.orc_lr_check.argtypes = [vp, vp, vp, i32, i32, C.c_float]
        _lib.orc_cost_adjust.argtypes = [i32]
        _lib.orc_cost_adjust.restype = C.c_uint8
        _lib.orc_set_threads.argtypes = [i32]
        _lib.orc_max_threads.restype = i32
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def match(cfg: Config, left: np.ndarray, right: np.ndarray, init: np.ndarray | None = None,
          dump: bool = False, want_right: bool = False) -> dict:
    """StereoCuda::Match restated. Returns a dict with 'disp' (and stage buffers when dump)."""
    W, H, D = cfg.width, cfg.height, cfg.disp_range
    left = np.ascontiguousarray(left, np.uint8)
    right = np.ascontiguousarray(right, np.uint8)
    out = {"disp": np.empty((H, W), np.float32)}
    if want_right:
        out["disp_r"] = np.empty((H, W), np.float32)
    if dump:
        out.update(census_l=np.empty((H, W), np.uint64), census_r=np.empty((H, W), np.uint64),
                   cost=np.empty((H, W, D), np.uint8), paths=np.empty((4, H, W, D), np.uint8),
                   wta_l=np.empty((H, W), np.float32), wta_r=np.empty((H, W), np.float32))
        if cfg.do_lr_check:
            out.update(cost_rl=np.zeros((H, W, D), np.uint8), paths_rl=np.zeros((4, H, W, D), np.uint8))
    g = out.get
    init_c = None if init is None else np.ascontiguousarray(init, np.int16)
    rc = lib().orc_match_dump(C.byref(cfg.c()), _p(left), _p(right), _p(init_c), _p(g("census_l")),
                              _p(g("census_r")), _p(g("cost")), _p(g("paths")), _p(g("wta_l")), _p(g("cost_rl")),
                              _p(g("paths_rl")), _p(g("wta_r")), _p(out["disp"]), _p(g("disp_r")))
    if rc != 0:
        raise RuntimeError(f"oracle match failed ({rc})")
    return out


def pyr_match(pc: PyrConfig, left: np.ndarray, right: np.ndarray) -> np.ndarray:
    disp = np.empty((pc.height, pc.width), np.float32)
    rc = lib().orc_pyr_match(C.byref(pc.c()), _p(np.ascontiguousarray(left, np.uint8)),
                             _p(np.ascontiguousarray(right, np.uint8)), _p(disp))
    if rc != 0:
        raise RuntimeError(f"oracle pyramid match failed ({rc})")
    return disp


def pyr_level_config(pc: PyrConfig, level: int) -> Config:
    c = _Cfg()
    if lib().orc_pyr_level_config(C.byref(pc.c()), level, C.byref(c)) != 0:
        raise IndexError(level)
    return Config(**{f.name: getattr(c, f.name) for f in fields(Config)})


def census(img: np.ndarray, cs_type: int, is_right: bool) -> np.ndarray:
    img = np.ascontiguousarray(img, np.uint8)
    out = np.empty(img.shape, np.uint64)
    lib().orc_census(_p(img), img.shape[1], img.shape[0], cs_type, int(is_right), _p(out))
    return out


def remove_peaks(disp: np.ndarray, strips: int, ratio: float, abs_mode: int = 0) -> tuple[np.ndarray, int]:
    d = np.ascontiguousarray(disp, np.float32).copy()
    n = lib().orc_remove_peaks(_p(d), d.shape[1], d.shape[0], strips, ratio, abs_mode)
    return d, n


def remove_peaks_strip(disp: np.ndarray, threshold: int, abs_mode: int = 0) -> tuple[np.ndarray, int]:
    d = np.ascontiguousarray(disp, np.float32).copy()
    n = lib().orc_remove_peaks_strip(_p(d), d.shape[1], d.shape[0], threshold, abs_mode)
    return d, n


def zoom_half(img: np.ndarray) -> np.ndarray:
    img = np.ascontiguousarray(img, np.uint8)
    h, w = img.shape
    out = np.empty((h // 2, w // 2), np.uint8)
    lib().orc_zoom_half(_p(img), w, h, _p(out))
    return out


def init_next_level(cur: np.ndarray, width: int, height: int) -> np.ndarray:
    cur = np.ascontiguousarray(cur, np.float32)
    out = np.empty((height, width), np.int16)
    lib().orc_init_next_level(_p(cur), cur.shape[1], cur.shape[0], _p(out), width, height)
    return out


def median3x3(d: np.ndarray) -> np.ndarray:
    d = np.ascontiguousarray(d, np.float32)
    out = np.empty_like(d)
    lib().orc_median3x3(_p(d), _p(out), d.shape[1], d.shape[0])
    return out


def dilation(d: np.ndarray, wnd: int) -> np.ndarray:
    d = np.ascontiguousarray(d, np.float32)
    out = np.empty_like(d)
    lib().orc_dilation(_p(d), _p(out), d.shape[1], d.shape[0], wnd)
    return out


def cost_adjust(d: int) -> int:
    return lib().orc_cost_adjust(d)


def set_threads(n: int) -> None:
    lib().orc_set_threads(n)


def max_threads() -> int:
    return lib().orc_max_threads()


def depth_from_disp(disp: np.ndarray, x0_left: float, x0_right: float, focus: float,
                    baseline: float) -> np.ndarray:
    """Depth of a disparity map, as StereoCudaImpl::Match2 (SgmStereoCuda/StereoCudaImpl.cpp:548-583)
    computes it with Kernel_ComputeDepth (SgmStereoCuda/cusgm_util.cu:7-34): in double,
    depth = (baseline * focus) / ((double)d + (x0_right - x0_left)), rounded to float; INVALID stays
    INVALID."""
    d = np.ascontiguousarray(disp, np.float32)
    f1 = float(baseline) * float(focus)
    f2 = float(x0_right) - float(x0_left)
    with np.errstate(divide="ignore", invalid="ignore"):
        depth = (f1 / (d.astype(np.float64) + f2)).astype(np.float32)
    return np.where(d == INVALID_FLOAT, INVALID_FLOAT, depth)


def depth_source_config(cfg: Config) -> Config:
    """The options whose final map StereoCudaImpl::Match2 turns into depth. Match2
    (SgmStereoCuda/StereoCudaImpl.cpp:548-583) reads the aggregator's disparity buffer unless
    small-region removal ran (then the host map after it). DisparityFilter::Filter
    (SgmStereoCuda/cusgm_df.cu:275-339) filters the median in place in that buffer, writes a post
    filter or a morphology step alone into its own buffer, and writes the morphology that follows a
    post filter back into the aggregator's buffer. So with exactly one of post filter / morphology
    and no small-region removal, the depth comes from the map before that step."""
    mp = cfg.morphology or (2 if cfg.morphology_dilation else 0)
    if cfg.do_remove_peaks or (cfg.post_filter != 0) == (mp != 0):
        return cfg
    return Config(**{**cfg.__dict__, "post_filter": 0, "morphology": 0, "morphology_dilation": 0})


def pyr_init2_coarsest(width: int, num_layers: int, min_depth: float, max_depth: float, x0_left: float,
                       x0_right: float, focus: float, baseline: float) -> tuple[int, int]:
    """(min disparity, disparity range) of the coarsest pyramid level that HierSgmCudaImpl::Init2
    (FasterStereoCuda/FasterStereoCuda.cpp:370-395) derives from a depth range, with the camera
    scaled to that level by CamParam_T::Scale (SgmStereoCuda/sgm_types.h:76-83); the range is the
    next power of two >= 64 above the span, halved once if above twice the full width, and a minimum
    at or past the width is pulled back (not below -width). min_depth/max_depth are floats there."""
    layers = max(1, int(num_layers))
    s = 2 ** (layers - 1)
    x0l, x0r, f = x0_left / s, x0_right / s, focus / s
    lo = baseline * f / float(np.float32(max_depth)) - x0r + x0l
    hi = baseline * f / float(np.float32(min_depth)) - x0r + x0l
    span = hi - lo
    k = 6
    while 2.0 ** k < span:
        k += 1
    rng = 2.0 ** k
    if rng > 2 * width:
        rng /= 2
    if lo >= width:
        lo = width - rng
        if lo < -width:
            lo = -width
    return int(np.floor(lo)), int(rng)
