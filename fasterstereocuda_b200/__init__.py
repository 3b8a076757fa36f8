"""B200 semi-global-matching stereo engine (Python host side).

The compute path is the CUDA library ``_lib/libsgmb200.so`` built from ``csrc/`` for sm_100a;
this module only binds its C ABI (``include/sgm_b200.h``) and mirrors the reference's
``StereoCuda`` / ``FasterStereoCuda`` classes (ethan-li-coding/FasterStereoCuda,
SgmStereoCuda/StereoCuda.h:14-100 and FasterStereoCuda/FasterStereoCuda.h:24-127):
same method names, argument meaning and boolean results. There is no CPU fallback: if the
library is missing, loading it raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Optional

import numpy as np

__all__ = [
    "CuSGMOption", "StereoROI", "ExtOptions", "StereoOption1", "LevelOverride",
    "StereoCuda", "FasterStereoCuda", "load_library", "INVALID_FLOAT", "INVALID_SHORT", "LEVEL_RANGE",
]

INVALID_FLOAT = np.float32(-999999.0)
INVALID_SHORT = np.int16(-32768)
LEVEL_RANGE = 32

_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libsgmb200.so"
_lib = None


class CuSGMOption(C.Structure):
    """Same fields, order and defaults as CuSGMOption (SgmStereoCuda/sgm_types.h:21-65)."""
    _fields_ = [
        ("p1", C.c_int32), ("p2_init", C.c_int32), ("p2_max", C.c_int32), ("cs_type", C.c_int32),
        ("num_paths", C.c_int32), ("do_median_filter", C.c_bool), ("do_lr_check", C.c_bool),
        ("lr_threshold", C.c_float), ("unique_threshold", C.c_float), ("using_constant_p2", C.c_bool),
        ("do_remove_peaks", C.c_bool), ("peaks_ratio_threshold", C.c_float), ("post_filter_type", C.c_int32),
        ("morphology_type", C.c_int32),
    ]
    CS_5x5, CS_9x7 = 0, 1
    PF_NONE, PF_GAUSS, PF_BILATERAL = 0, 1, 2
    MP_NONE, MP_EROSION, MP_DILATION, MP_OPEN, MP_CLOSE = 0, 1, 2, 3, 4

    def __init__(self, **kw):
        super().__init__()
        self.p1, self.p2_init, self.p2_max, self.cs_type, self.num_paths = 8, 32, 0, 0, 0
        self.do_median_filter = self.do_lr_check = False
        self.lr_threshold = self.unique_threshold = 0.0
        self.using_constant_p2 = self.do_remove_peaks = False
        self.peaks_ratio_threshold = 0.0
        self.post_filter_type = self.morphology_type = 0
        for k, v in kw.items():
            setattr(self, k, v)


class StereoROI(C.Structure):
    """StereoROI_T (SgmStereoCuda/sgm_types.h:89-92)."""
    _fields_ = [("x", C.c_int32), ("y", C.c_int32), ("w", C.c_int32), ("h", C.c_int32)]


class ExtOptions(C.Structure):
    """Rules the reference leaves to thread scheduling or its compiler (sgm_ext_options_t)."""
    _fields_ = [("tie_rule", C.c_int32), ("init_tie_rule", C.c_int32), ("peaks_strips", C.c_int32),
                ("peaks_abs_mode", C.c_int32), ("p2_div0", C.c_int32)]
    TIE_LOWEST, TIE_HIGHEST, TIE_LANE_HIGH, TIE_LANE_LOW, TIE_REF_B200 = 0, 1, 2, 3, 4
    PEAKS_ABS_INT, PEAKS_ABS_FLOAT = 0, 1

    def __init__(self, **kw):
        super().__init__()
        self.tie_rule = self.init_tie_rule = 4
        self.peaks_strips = 0
        self.peaks_abs_mode = 0
        self.p2_div0 = -1
        for k, v in kw.items():
            setattr(self, k, v)


class StereoOption1(C.Structure):
    """FasterStereoCuda::StereoOption1 (FasterStereoCuda/FasterStereoCuda.h:39-51)."""
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("min_disp", C.c_int32), ("max_disp", C.c_int32),
                ("num_layers", C.c_int32), ("do_lr_check", C.c_bool), ("do_rm_peaks", C.c_bool),
                ("do_smooth", C.c_bool)]

    def __init__(self, **kw):
        super().__init__()
        self.num_layers = 1
        self.do_lr_check = True
        self.do_rm_peaks = True
        self.do_smooth = False
        for k, v in kw.items():
            setattr(self, k, v)


class CamParam(C.Structure):
    """CamParam_T (SgmStereoCuda/sgm_types.h:70-84): principal points, focal length (pixels) and
    baseline of a rectified pair; depth = baseline * focus / (d + x0_right - x0_left)."""
    _fields_ = [("x0_left", C.c_double), ("y0_left", C.c_double), ("x0_right", C.c_double),
                ("y0_right", C.c_double), ("focus", C.c_double), ("baseline", C.c_double)]

    def __init__(self, **kw):
        super().__init__()
        for k, v in kw.items():
            setattr(self, k, v)


class EpipolarStereoParam(C.Structure):
    """FasterStereoCuda::EpipolarStereoParam (FasterStereoCuda/FasterStereoCuda.h:17-27); note the
    member order differs from CamParam_T (baseline before focus)."""
    _fields_ = [("x0_left", C.c_double), ("y0_left", C.c_double), ("x0_right", C.c_double),
                ("y0_right", C.c_double), ("baseline", C.c_double), ("focus", C.c_double)]

    def __init__(self, **kw):
        super().__init__()
        for k, v in kw.items():
            setattr(self, k, v)


class StereoOption2(C.Structure):
    """FasterStereoCuda::StereoOption2 (FasterStereoCuda/FasterStereoCuda.h:45-69): the search range
    given as a depth range seen by the camera `epi`."""
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("min_depth", C.c_float), ("max_depth", C.c_float),
                ("num_layers", C.c_int32), ("do_lr_check", C.c_bool), ("do_rm_peaks", C.c_bool),
                ("do_smooth", C.c_bool), ("epi", EpipolarStereoParam)]

    def __init__(self, **kw):
        super().__init__()
        self.num_layers = 1
        self.do_lr_check = True
        self.do_rm_peaks = True
        self.do_smooth = False
        for k, v in kw.items():
            setattr(self, k, v)


class LevelOverride(C.Structure):
    """Census type and penalties applied to every pyramid level (sgm_level_override_t)."""
    _fields_ = [("cs_type", C.c_int32), ("p1", C.c_int32), ("p2", C.c_int32)]


class Tuning(C.Structure):
    """Kernel variants and launch shapes (sgm_tuning_t); every setting gives the same result."""
    _fields_ = [("row_kernel", C.c_int32), ("rows_per_cta", C.c_int32), ("col_kernel", C.c_int32),
                ("cols_per_cta", C.c_int32), ("bt_smem", C.c_int32), ("row_lanes", C.c_int32),
                ("col_lanes", C.c_int32)]


class BatchPair(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("min_disparity", C.c_int32),
                ("disp_range", C.c_int32)]


class BatchInfo(C.Structure):
    _fields_ = [("pairs", C.c_int32), ("buckets", C.c_int32), ("arena_bytes", C.c_uint64),
                ("kernels_per_run", C.c_int64)]


class BatchBucket(C.Structure):
    _fields_ = [("disp_range", C.c_int32), ("width_class", C.c_int32), ("pairs", C.c_int32),
                ("rows_lanes", C.c_int32), ("rows_warps_per_cta", C.c_int32), ("rows_ctas", C.c_int32),
                ("cols_lanes", C.c_int32), ("cols_warps_per_cta", C.c_int32), ("cols_prefetch", C.c_int32),
                ("cols_ctas", C.c_int32)]


def load_library(path: Optional[os.PathLike] = None):
    """Loads the engine library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else _LIB_PATH
    if not p.exists():
        raise RuntimeError(f"SGM engine library not built: {p} (run python -m fasterstereocuda_b200.build)")
    lib = C.CDLL(str(p))
    vp, i32, i64, f32 = C.c_void_p, C.c_int32, C.c_int64, C.c_float
    sig = {
        "sgm_create": (i32, [C.POINTER(vp)]), "sgm_destroy": (i32, [vp]),
        "sgm_init": (i32, [vp, i32, i32, i32, i32, C.POINTER(CuSGMOption), i32]),
        "sgm_set_ext_options": (i32, [vp, C.POINTER(ExtOptions)]),
        "sgm_get_ext_options": (i32, [vp, C.POINTER(ExtOptions)]),
        "sgm_set_tuning": (i32, [vp, C.POINTER(Tuning)]), "sgm_get_tuning": (i32, [vp, C.POINTER(Tuning)]),
        "sgm_pyr_set_tuning": (i32, [vp, i32, C.POINTER(Tuning)]),
        "sgm_match": (i32, [vp, vp, vp, vp, vp, vp, C.POINTER(StereoROI), C.POINTER(StereoROI)]),
        "sgm_match_device": (i32, [vp, vp, vp, vp, vp, vp, vp]),
        "sgm_release": (i32, [vp]), "sgm_set_min_disparity": (i32, [vp, i32]),
        "sgm_get_disparity_range": (i32, [vp]),
        "sgm_roi_from_disp_map": (None, [vp, i32, i32, C.POINTER(StereoROI)]),
        "sgm_invalid_float": (f32, []), "sgm_invalid_short": (C.c_int16, []), "sgm_level_range": (C.c_int16, []),
        "sgm_malloc_page_locked": (i32, [C.POINTER(vp), C.c_size_t]), "sgm_free_page_locked": (i32, [vp]),
        "sgm_last_error": (C.c_char_p, [vp]), "sgm_kernel_launches": (i64, [vp]),
        "sgm_pyr_create": (i32, [C.POINTER(vp)]), "sgm_pyr_destroy": (i32, [vp]),
        "sgm_pyr_init": (i32, [vp, C.POINTER(StereoOption1), C.POINTER(LevelOverride), C.POINTER(ExtOptions)]),
        "sgm_pyr_init2": (i32, [vp, C.POINTER(StereoOption2), C.POINTER(LevelOverride), C.POINTER(ExtOptions)]),
        "sgm_pyr_match2": (i32, [vp, vp, vp, vp]),
        "sgm_init2": (i32, [vp, i32, i32, i32, i32, C.POINTER(CuSGMOption), C.POINTER(CamParam), i32]),
        "sgm_match2": (i32, [vp, vp, vp, vp, vp, C.POINTER(StereoROI), C.POINTER(StereoROI)]),
        "sgm_pyr_match": (i32, [vp, vp, vp, vp]), "sgm_pyr_match_device": (i32, [vp, vp, vp, vp, vp]),
        "sgm_pyr_release": (i32, [vp]),
        "sgm_pyr_level_info": (i32, [vp, i32, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]),
        "sgm_pyr_kernel_launches": (i64, [vp]),
        "sgm_debug_read": (i32, [vp, i32, i32, vp, C.c_size_t]),
        "sgm_profile_enable": (i32, [i32]), "sgm_profile_read": (i32, [C.c_char_p, C.c_size_t]),
        "sgm_debug_fail_device_alloc": (i32, [i64]), "sgm_debug_live_device_allocations": (i64, []),
        "sgm_debug_wait_timeouts": (i64, []), "sgm_debug_scan_wait": (i32, [i64, i32]),
        "sgm_debug_reset_wait_timeouts": (i32, []),
        "sgm_batch_create": (i32, [C.POINTER(vp)]), "sgm_batch_destroy": (i32, [vp]),
        "sgm_batch_last_error": (C.c_char_p, [vp]),
        "sgm_batch_init": (i32, [vp, C.POINTER(BatchPair), i32, C.POINTER(CuSGMOption), C.POINTER(ExtOptions)]),
        "sgm_batch_autotune": (i32, [vp]),
        "sgm_batch_pair_buffers": (i32, [vp, i32, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
        "sgm_batch_run": (i32, [vp, vp]),
        "sgm_batch_match": (i32, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
        "sgm_batch_info": (i32, [vp, C.POINTER(BatchInfo)]),
        "sgm_batch_bucket": (i32, [vp, i32, C.POINTER(BatchBucket)]),
        "sgm_batch_pyr_create": (i32, [C.POINTER(vp)]), "sgm_batch_pyr_destroy": (i32, [vp]),
        "sgm_batch_pyr_last_error": (C.c_char_p, [vp]),
        "sgm_batch_pyr_init": (i32, [vp, C.POINTER(BatchPair), i32, C.POINTER(StereoOption1),
                                     C.POINTER(LevelOverride), C.POINTER(ExtOptions)]),
        "sgm_batch_pyr_pair_buffers": (i32, [vp, i32, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
        "sgm_batch_pyr_run": (i32, [vp, vp]),
        "sgm_batch_pyr_match": (i32, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
        "sgm_batch_pyr_info": (i32, [vp, C.POINTER(BatchInfo)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib if path is None else _lib
    return lib


def profile_enable(on: bool = True) -> None:
    """Per-kernel CUDA-event timing of every launch in the process (resets the counters)."""
    load_library().sgm_profile_enable(int(on))


def profile_read() -> dict:
    """{kernel name: {"launches": n, "ms": total}} accumulated since profile_enable."""
    import json
    lib = load_library()
    need = lib.sgm_profile_read(None, 0)
    buf = C.create_string_buffer(max(need, 2))
    lib.sgm_profile_read(buf, len(buf))
    return json.loads(buf.value.decode() or "{}")


def _ptr(a) -> Optional[int]:
    """Address of a numpy array or a torch tensor (None passes through)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported buffer type {type(a)}")


class StereoCuda:
    """Single-level matcher; mirrors StereoCuda (SgmStereoCuda/StereoCuda.h:14-100)."""

    def __init__(self):
        self._lib = load_library()
        h = C.c_void_p()
        if self._lib.sgm_create(C.byref(h)) != 0:
            raise MemoryError("sgm_create failed")
        self._h = h
        self.width = self.height = 0
        self.status = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.sgm_destroy(h)
            self._h = None

    def last_error(self) -> str:
        return (self._lib.sgm_last_error(self._h) or b"").decode()

    def set_ext_options(self, ext: ExtOptions) -> bool:
        self.status = self._lib.sgm_set_ext_options(self._h, C.byref(ext))
        return self.status == 0

    def set_tuning(self, tuning: Tuning) -> bool:
        self.status = self._lib.sgm_set_tuning(self._h, C.byref(tuning))
        return self.status == 0

    def Init(self, width: int, height: int, min_disparity: int, disp_range: int, sgm_option: CuSGMOption,
             print_log: bool = False) -> bool:
        self.status = self._lib.sgm_init(self._h, width, height, min_disparity, disp_range, C.byref(sgm_option),
                                         int(print_log))
        if self.status == 0:
            self.width, self.height = width, height
        return self.status == 0

    def Init2(self, width: int, height: int, min_disparity: int, disp_range: int, sgm_option: CuSGMOption,
              cam_param: CamParam, print_log: bool = False) -> bool:
        """StereoCuda::Init2 (SgmStereoCuda/StereoCuda.h:57): Init plus the camera used by Match2."""
        self.status = self._lib.sgm_init2(self._h, width, height, min_disparity, disp_range, C.byref(sgm_option),
                                          C.byref(cam_param), int(print_log))
        if self.status == 0:
            self.width, self.height = width, height
        return self.status == 0

    def Match2(self, img_left, img_right, depth_left, init_disp_left=None,
               ste_roi_left: Optional[StereoROI] = None, ste_roi_right: Optional[StereoROI] = None) -> bool:
        """StereoCuda::Match2 (SgmStereoCuda/StereoCuda.h:69): the left disparity map of Match turned
        into depth (INVALID kept), written into the host array depth_left."""
        for a, t, n in ((img_left, np.uint8, "img_left"), (img_right, np.uint8, "img_right"),
                        (depth_left, np.float32, "depth_left"), (init_disp_left, np.int16, "init_disp_left")):
            self._check_host(a, t, n)
        self.status = self._lib.sgm_match2(
            self._h, _ptr(img_left), _ptr(img_right), _ptr(depth_left), _ptr(init_disp_left),
            C.byref(ste_roi_left) if ste_roi_left is not None else None,
            C.byref(ste_roi_right) if ste_roi_right is not None else None)
        return self.status == 0

    def _check_host(self, a, dtype, name):
        if a is None:
            return
        if not isinstance(a, np.ndarray) or a.dtype != dtype or a.size != self.width * self.height:
            raise ValueError(f"{name}: expected a {dtype} array of {self.width}x{self.height}")

    def Match(self, img_left, img_right, disp_left, disp_right=None, init_disp_left=None,
              ste_roi_left: Optional[StereoROI] = None, ste_roi_right: Optional[StereoROI] = None) -> bool:
        """Host arrays in, host arrays out (disp_* are written in place), like StereoCuda::Match."""
        for a, t, n in ((img_left, np.uint8, "img_left"), (img_right, np.uint8, "img_right"),
                        (disp_left, np.float32, "disp_left"), (disp_right, np.float32, "disp_right"),
                        (init_disp_left, np.int16, "init_disp_left")):
            self._check_host(a, t, n)
        self.status = self._lib.sgm_match(
            self._h, _ptr(img_left), _ptr(img_right), _ptr(disp_left), _ptr(disp_right), _ptr(init_disp_left),
            C.byref(ste_roi_left) if ste_roi_left is not None else None,
            C.byref(ste_roi_right) if ste_roi_right is not None else None)
        return self.status == 0

    def match_device(self, d_left, d_right, d_disp_left, d_disp_right=None, d_init=None, stream: int = 0) -> bool:
        """Device buffers (torch CUDA tensors or raw addresses); enqueued on `stream`, not synchronised."""
        self.status = self._lib.sgm_match_device(self._h, _ptr(d_left), _ptr(d_right), _ptr(d_disp_left),
                                                 _ptr(d_disp_right), _ptr(d_init), stream or None)
        return self.status == 0

    def Release(self) -> None:
        self._lib.sgm_release(self._h)

    def SetMinDisparity(self, min_disparity: int) -> None:
        self._lib.sgm_set_min_disparity(self._h, min_disparity)

    def GetDispartyRange(self) -> int:
        return self._lib.sgm_get_disparity_range(self._h)

    def kernel_launches(self) -> int:
        return self._lib.sgm_kernel_launches(self._h)

    def debug_read(self, which: str, view: int = 0, disp_range: int = 0) -> np.ndarray:
        """Internal stage buffer of the last match: census_l, census_r, cost, lr, rl, bt, wta."""
        code = {"census_l": 0, "census_r": 1, "cost": 2, "lr": 3, "rl": 4, "bt": 5, "wta": 6}[which]
        H, W = self.height, self.width
        D = disp_range or self.GetDispartyRange()
        shape, dt = ((H, W), np.uint64) if code < 2 else (((H, W, D), np.uint8) if code < 6 else ((H, W), np.float32))
        out = np.empty(shape, dt)
        st = self._lib.sgm_debug_read(self._h, code, view, out.ctypes.data, out.nbytes)
        if st != 0:
            raise RuntimeError(f"sgm_debug_read({which}) failed: {st} {self.last_error()}")
        return out

    @staticmethod
    def GetRoiFromDispMap(disp, width: int, height: int, ste_roi: StereoROI) -> None:
        load_library().sgm_roi_from_disp_map(_ptr(disp), width, height, C.byref(ste_roi))

    @staticmethod
    def get_invad_float() -> float:
        return load_library().sgm_invalid_float()

    @staticmethod
    def get_invad_short() -> int:
        return load_library().sgm_invalid_short()

    @staticmethod
    def get_level_range() -> int:
        return load_library().sgm_level_range()


class FasterStereoCuda:
    """Pyramid matcher; mirrors FasterStereoCuda (FasterStereoCuda/FasterStereoCuda.h:24-127).

    `override` replaces the census type and penalties the reference hard-codes per level."""

    def __init__(self):
        self._lib = load_library()
        h = C.c_void_p()
        if self._lib.sgm_pyr_create(C.byref(h)) != 0:
            raise MemoryError("sgm_pyr_create failed")
        self._h = h
        self.width = self.height = 0
        self.status = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.sgm_pyr_destroy(h)
            self._h = None

    def last_error(self) -> str:
        return (self._lib.sgm_last_error(None) or b"").decode()

    def Init(self, option: StereoOption1, override: Optional[LevelOverride] = None,
             ext: Optional[ExtOptions] = None) -> bool:
        self.status = self._lib.sgm_pyr_init(self._h, C.byref(option),
                                             C.byref(override) if override is not None else None,
                                             C.byref(ext) if ext is not None else None)
        if self.status == 0:
            self.width, self.height = option.width, option.height
        return self.status == 0

    def Init2(self, option: StereoOption2, override: Optional[LevelOverride] = None,
              ext: Optional[ExtOptions] = None) -> bool:
        """FasterStereoCuda::Init2 (FasterStereoCuda/FasterStereoCuda.h:102): the coarsest level's
        disparity range from the depth range and the camera scaled to that level."""
        self.status = self._lib.sgm_pyr_init2(self._h, C.byref(option),
                                              C.byref(override) if override is not None else None,
                                              C.byref(ext) if ext is not None else None)
        if self.status == 0:
            self.width, self.height = option.width, option.height
        return self.status == 0

    def Match2(self, bytes_left, bytes_right, depth_data) -> bool:
        """FasterStereoCuda::Match2 (FasterStereoCuda/FasterStereoCuda.h:123): depth of the finest level."""
        n = self.width * self.height
        for a, t in ((bytes_left, np.uint8), (bytes_right, np.uint8), (depth_data, np.float32)):
            if not isinstance(a, np.ndarray) or a.dtype != t or a.size != n:
                raise ValueError("expected host arrays of width*height elements")
        self.status = self._lib.sgm_pyr_match2(self._h, _ptr(bytes_left), _ptr(bytes_right), _ptr(depth_data))
        return self.status == 0

    def set_tuning(self, tuning: Tuning, level: int = -1) -> bool:
        """After Init: tuning of one level, or of every level (-1)."""
        self.status = self._lib.sgm_pyr_set_tuning(self._h, level, C.byref(tuning))
        return self.status == 0

    def Match(self, bytes_left, bytes_right, disparity_data) -> bool:
        n = self.width * self.height
        for a, t in ((bytes_left, np.uint8), (bytes_right, np.uint8), (disparity_data, np.float32)):
            if not isinstance(a, np.ndarray) or a.dtype != t or a.size != n:
                raise ValueError("expected host arrays of width*height elements")
        self.status = self._lib.sgm_pyr_match(self._h, _ptr(bytes_left), _ptr(bytes_right), _ptr(disparity_data))
        return self.status == 0

    def match_device(self, d_left, d_right, d_disp, stream: int = 0) -> bool:
        self.status = self._lib.sgm_pyr_match_device(self._h, _ptr(d_left), _ptr(d_right), _ptr(d_disp),
                                                     stream or None)
        return self.status == 0

    def Release(self) -> None:
        self._lib.sgm_pyr_release(self._h)

    def level_info(self, level: int):
        w, h, m, d = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        if self._lib.sgm_pyr_level_info(self._h, level, C.byref(w), C.byref(h), C.byref(m), C.byref(d)) != 0:
            raise IndexError(level)
        return w.value, h.value, m.value, d.value

    def kernel_launches(self) -> int:
        return self._lib.sgm_pyr_kernel_launches(self._h)

    @staticmethod
    def MallocPageLockedPtr(size: int) -> int:
        p = C.c_void_p()
        if load_library().sgm_malloc_page_locked(C.byref(p), size) != 0:
            raise MemoryError(size)
        return p.value

    @staticmethod
    def FreePageLockedPtr(ptr: int) -> bool:
        return load_library().sgm_free_page_locked(C.c_void_p(ptr)) == 0


class StereoBatch:
    """Many pairs of different sizes / disparity ranges matched by one CUDA graph launch
    (sgm_batch_*). Each pair's disparity equals StereoCuda's for the same pair and options."""

    def __init__(self):
        self._lib = load_library()
        h = C.c_void_p()
        st = self._lib.sgm_batch_create(C.byref(h))
        if st != 0:
            raise RuntimeError(f"sgm_batch_create failed ({st})")
        self._h = h
        self.status = 0
        self.shapes = []

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._lib.sgm_batch_destroy(h)

    def last_error(self) -> str:
        return (self._lib.sgm_batch_last_error(self._h) or b"").decode()

    def Init(self, pairs, sgm_option: CuSGMOption, ext: Optional[ExtOptions] = None) -> bool:
        """pairs: sequence of (width, height, min_disparity, disp_range)."""
        arr = (BatchPair * len(pairs))(*[BatchPair(*p) for p in pairs])
        self.status = self._lib.sgm_batch_init(self._h, arr, len(pairs), C.byref(sgm_option),
                                               C.byref(ext) if ext is not None else None)
        if self.status == 0:
            self.shapes = [(p[1], p[0]) for p in pairs]
        return self.status == 0

    def autotune(self) -> bool:
        self.status = self._lib.sgm_batch_autotune(self._h)
        return self.status == 0

    def buffers(self, i: int):
        """(d_left, d_right, d_disp) device addresses of pair i inside the batch arena."""
        a, b, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
        self.status = self._lib.sgm_batch_pair_buffers(self._h, i, C.byref(a), C.byref(b), C.byref(c))
        if self.status != 0:
            raise RuntimeError(self.last_error())
        return a.value, b.value, c.value

    def run(self, stream: int = 0) -> bool:
        self.status = self._lib.sgm_batch_run(self._h, C.c_void_p(stream) if stream else None)
        return self.status == 0

    def Match(self, lefts, rights, disps) -> bool:
        n = len(self.shapes)
        for i, (L, R, O) in enumerate(zip(lefts, rights, disps)):
            h, w = self.shapes[i]
            for a, dt in ((L, np.uint8), (R, np.uint8), (O, np.float32)):
                if a.dtype != dt or a.shape != (h, w) or not a.flags["C_CONTIGUOUS"]:
                    raise ValueError(f"pair {i}: expected C-contiguous {dt.__name__} array of shape {(h, w)}")
        pl = (C.c_void_p * n)(*[L.ctypes.data for L in lefts])
        pr = (C.c_void_p * n)(*[R.ctypes.data for R in rights])
        po = (C.c_void_p * n)(*[O.ctypes.data for O in disps])
        self.status = self._lib.sgm_batch_match(self._h, pl, pr, po)
        return self.status == 0

    def info(self) -> dict:
        i = BatchInfo()
        if self._lib.sgm_batch_info(self._h, C.byref(i)) != 0:
            raise RuntimeError(self.last_error())
        return {f: getattr(i, f) for f, _ in BatchInfo._fields_}

    def buckets(self) -> list:
        out = []
        for k in range(self.info()["buckets"]):
            b = BatchBucket()
            if self._lib.sgm_batch_bucket(self._h, k, C.byref(b)) != 0:
                raise RuntimeError(self.last_error())
            out.append({f: getattr(b, f) for f, _ in BatchBucket._fields_})
        return out


class StereoBatchPyramid:
    """Many pyramid pairs (FasterStereoCuda semantics) of different sizes in one CUDA graph
    launch (sgm_batch_pyr_*). Each pair's disparity equals FasterStereoCuda's for that pair."""

    def __init__(self):
        self._lib = load_library()
        h = C.c_void_p()
        st = self._lib.sgm_batch_pyr_create(C.byref(h))
        if st != 0:
            raise RuntimeError(f"sgm_batch_pyr_create failed ({st})")
        self._h = h
        self.status = 0
        self.shapes = []

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._lib.sgm_batch_pyr_destroy(h)

    def last_error(self) -> str:
        return (self._lib.sgm_batch_pyr_last_error(self._h) or b"").decode()

    def Init(self, pairs, option: StereoOption1, override: Optional[LevelOverride] = None,
             ext: Optional[ExtOptions] = None) -> bool:
        """pairs: sequence of (width, height, min_disp, max_disp); option: layers, LR, removal."""
        arr = (BatchPair * len(pairs))(*[BatchPair(w, h, mn, mx - mn) for (w, h, mn, mx) in pairs])
        self.status = self._lib.sgm_batch_pyr_init(self._h, arr, len(pairs), C.byref(option),
                                                   C.byref(override) if override is not None else None,
                                                   C.byref(ext) if ext is not None else None)
        if self.status == 0:
            self.shapes = [(p[1], p[0]) for p in pairs]
        return self.status == 0

    def buffers(self, i: int):
        a, b, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
        self.status = self._lib.sgm_batch_pyr_pair_buffers(self._h, i, C.byref(a), C.byref(b), C.byref(c))
        if self.status != 0:
            raise RuntimeError(self.last_error())
        return a.value, b.value, c.value

    def run(self, stream: int = 0) -> bool:
        self.status = self._lib.sgm_batch_pyr_run(self._h, C.c_void_p(stream) if stream else None)
        return self.status == 0

    def Match(self, lefts, rights, disps) -> bool:
        n = len(self.shapes)
        for i, (L, R, O) in enumerate(zip(lefts, rights, disps)):
            h, w = self.shapes[i]
            for a, dt in ((L, np.uint8), (R, np.uint8), (O, np.float32)):
                if a.dtype != dt or a.shape != (h, w) or not a.flags["C_CONTIGUOUS"]:
                    raise ValueError(f"pair {i}: expected C-contiguous {dt.__name__} array of shape {(h, w)}")
        pl = (C.c_void_p * n)(*[L.ctypes.data for L in lefts])
        pr = (C.c_void_p * n)(*[R.ctypes.data for R in rights])
        po = (C.c_void_p * n)(*[O.ctypes.data for O in disps])
        self.status = self._lib.sgm_batch_pyr_match(self._h, pl, pr, po)
        return self.status == 0

    def info(self) -> dict:
        i = BatchInfo()
        if self._lib.sgm_batch_pyr_info(self._h, C.byref(i)) != 0:
            raise RuntimeError(self.last_error())
        return {f: getattr(i, f) for f, _ in BatchInfo._fields_}
