"""The C ABI library loads and exports every entry point include/*.h declares (no GPU needed)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        for m in re.finditer(r"SGM_API\s+[\w\s\*]+?\b(sgm_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_all_declared_symbols(engine_lib):
    lib_path = ROOT / "fasterstereocuda_b200" / "_lib" / "libsgmb200.so"
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    declared = declared_symbols()
    assert len(declared) >= 25
    missing = sorted(declared - exported)
    assert not missing, f"declared but not exported: {missing}"
    # only the C ABI and the C++ drop-in classes are visible
    extra = sorted(s for s in exported if s.startswith("sgm_") and s not in declared)
    assert not extra, f"exported but not declared: {extra}"


def test_struct_layouts_match_reference(engine_lib):
    import fasterstereocuda_b200 as fsc
    # CuSGMOption (sgm_types.h:21-65): 5 ints, 2 bools, 2 floats, 2 bools, float, 2 enums
    assert C.sizeof(fsc.CuSGMOption) == 48
    assert fsc.CuSGMOption.lr_threshold.offset == 24
    assert fsc.CuSGMOption.using_constant_p2.offset == 32
    assert fsc.CuSGMOption.peaks_ratio_threshold.offset == 36
    assert fsc.CuSGMOption.morphology_type.offset == 44
    assert C.sizeof(fsc.StereoROI) == 16
    assert C.sizeof(fsc.StereoOption1) == 24


def test_reference_defaults():
    import fasterstereocuda_b200 as fsc
    o = fsc.CuSGMOption()
    assert (o.p1, o.p2_init, o.cs_type, o.do_lr_check, o.unique_threshold) == (8, 32, 0, False, 0.0)
    s = fsc.StereoOption1()
    assert (s.num_layers, s.do_lr_check, s.do_rm_peaks, s.do_smooth) == (1, True, True, False)


def test_constants(engine_lib):
    import fasterstereocuda_b200 as fsc
    assert fsc.StereoCuda.get_invad_float() == -999999.0
    assert fsc.StereoCuda.get_invad_short() == -32768
    assert fsc.StereoCuda.get_level_range() == 32


def test_argument_errors_without_device(engine_lib):
    """Validation happens before any CUDA call, so these run without a GPU."""
    import fasterstereocuda_b200 as fsc
    s = fsc.StereoCuda()
    opt = fsc.CuSGMOption(cs_type=1, p1=10, p2_init=150)
    assert not s.Init(0, 10, 0, 64, opt) and s.status == -1
    assert not s.Init(10, 10, 0, 0, opt) and s.status == -1
    assert not s.Init(100, 100, 0, 96, opt) and s.status == -4      # not 32/64/128/256
    assert not s.Init(100, 100, 0, 64, fsc.CuSGMOption(p1=-1)) and s.status == -1
    assert not s.Init(100, 100, 0, 64, fsc.CuSGMOption(post_filter_type=3)) and s.status == -1
    assert not s.Init(100, 100, 0, 64, fsc.CuSGMOption(morphology_type=5)) and s.status == -1
    # a minimum disparity at or past the width leaves nothing to match: refused
    assert not s.Init(100, 100, 100, 64, opt) and s.status == -1
    assert "minimum disparity" in s.last_error()
    img = np.zeros((10, 10), np.uint8)
    d = np.zeros((10, 10), np.float32)
    s.width = s.height = 10
    assert not s.Match(img, img, d) and s.status == -2                 # not initialised
    assert "not initialised" in s.last_error()


def test_float_sgm_sizes_and_argument_errors_without_device(engine_lib):
    """Float-SGM buffer sizes, and argument checks that return before any CUDA call."""
    from fasterstereocuda_b200.float_sgm import _lib
    lib = _lib()
    B, H, W, D = 2, 29, 37, 64
    assert lib.sgm_float_workspace_elems(B, H, W, D) == 3 * B * H * W * D + 8 * B * H * W
    seg = 8  # checkpoint interval of the scans
    per_dir = max(B * H * ((W + seg - 1) // seg), B * W * ((H + seg - 1) // seg)) * D
    assert lib.sgm_float_checkpoint_elems(B, H, W, D) == 4 * per_dir
    a16 = 1 << 20  # 16-byte aligned addresses; never dereferenced on these paths
    st = lib.sgm_float_forward(a16, a16, a16, B, H, W, 48, 1.0, a16, a16, a16, a16, None)
    assert st == -1 and b"D in {32, 64}" in lib.sgm_last_error(None)
    st = lib.sgm_float_forward(a16 + 4, a16, a16, B, H, W, D, 1.0, a16, a16, a16, a16, None)
    assert st == -1 and b"16-byte aligned" in lib.sgm_last_error(None)
    st = lib.sgm_float_backward(a16, a16, a16, B, H, W, D, 1.0, a16, a16, a16, a16 + 8, a16, a16, a16, a16, None)
    assert st == -1 and b"16-byte aligned" in lib.sgm_last_error(None)
    st = lib.sgm_float_forward(a16, a16, a16, B, H, W, D, 1.0, a16, a16, a16, None, None)
    assert st == -1 and b"null device pointer" in lib.sgm_last_error(None)
    big = (1 << 31) - 1  # B*H*W*D would wrap a 64-bit product
    st = lib.sgm_float_forward(a16, a16, a16, big, big, big, D, 1.0, a16, a16, a16, a16, None)
    assert st == -1 and b"too large" in lib.sgm_last_error(None)
    for t in (0.0, -1.0, float("nan"), 1e-40):
        st = lib.sgm_float_forward(a16, a16, a16, B, H, W, D, t, a16, a16, a16, a16, None)
        assert st == -1 and b"temperature" in lib.sgm_last_error(None), t


def test_roi_from_disp_map(engine_lib):
    import fasterstereocuda_b200 as fsc
    d = np.full((20, 30), -999999.0, np.float32)
    d[5:12, 7:19] = 3.0
    roi = fsc.StereoROI()
    fsc.StereoCuda.GetRoiFromDispMap(d, 30, 20, roi)
    assert (roi.x, roi.y, roi.w, roi.h) == (7, 5, 12, 7)


def test_cxx_classes_export_the_reference_symbols(engine_lib):
    """StereoCuda / FasterStereoCuda export exactly the mangled names of the reference's classes
    (list taken from the reference built from its sources), so reference-linked code relinks."""
    want = set((ROOT / "tests" / "golden" / "reference_cxx_symbols.txt").read_text().split())
    lib_path = ROOT / "fasterstereocuda_b200" / "_lib" / "libsgmb200.so"
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], capture_output=True, text=True, check=True)
    have = {l.split()[-1] for l in out.stdout.splitlines() if "10StereoCuda" in l or "16FasterStereoCuda" in l}
    assert len(want) == 28
    assert want == have, (sorted(want - have), sorted(have - want))


C_CALLER = r"""
#include <stdio.h>
#include "sgm_b200.h"
int main(void) {
  float disp[6] = {-999999.0f, 2.0f, 3.0f, -999999.0f, 4.0f, -999999.0f};
  sgm_roi_t roi;
  sgm_handle_t h;
  sgm_option_t o = {10, 150, 0, 1, 4, true, true, 1.0f, 0.95f, true, false, 0.0f, 0, 0};
  int st;
  sgm_roi_from_disp_map(disp, 3, 2, &roi);
  if (sgm_create(&h) != SGM_OK) return 1;
  st = sgm_init(h, 0, 10, 0, 64, &o, 0);
  printf("%g %d %d %d %d %d\n", sgm_invalid_float(), roi.x, roi.y, roi.w, roi.h, st);
  sgm_destroy(h);
  return 0;
}
"""

CXX_CALLER = r"""
#include <cstdio>
#include "FasterStereoCuda.h"
#include "StereoCuda.h"
int main() {
  FasterStereoCuda stereo;  // the reference console's use
  FasterStereoCuda::StereoOption1 opt;
  opt.width = 0; opt.height = 375; opt.max_disp = 64; opt.num_layers = 3;
  const bool ok = stereo.Init(opt);
  StereoROI_T roi;
  float disp[4] = {StereoCuda::get_invad_float(), 1.0f, 2.0f, StereoCuda::get_invad_float()};
  StereoCuda::GetRoiFromDispMap(disp, 2, 2, roi);
  std::printf("%d %g %d %d %d %d %d\n", ok, StereoCuda::get_invad_float(), StereoCuda::get_level_range(),
              roi.x, roi.y, roi.w, roi.h);
  return 0;
}
"""


@pytest.mark.parametrize("lang", ["c", "c++"])
def test_c_and_cxx_callers_build_against_the_headers(engine_lib, tmp_path, lang):
    """A C caller of include/sgm_b200.h and a C++ caller of the reference's classes compile with
    warnings as errors, link against the library and run the calls that need no GPU."""
    libdir = ROOT / "fasterstereocuda_b200" / "_lib"
    src = tmp_path / ("caller.c" if lang == "c" else "caller.cpp")
    src.write_text(C_CALLER if lang == "c" else CXX_CALLER)
    exe = tmp_path / "caller"
    cc = ["gcc", "-std=c99"] if lang == "c" else ["g++", "-std=c++17"]
    subprocess.run(cc + ["-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-L", str(libdir), "-lsgmb200",
                         f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    if lang == "c":
        assert out == ["-999999", "1", "0", "2", "2", "-1"]   # ROI of the valid pixels; w = 0 rejected
    else:
        assert out == ["0", "-999999", "32", "0", "0", "2", "2"]
