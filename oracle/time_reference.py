"""Times the reference's own CUDA build (oracle/_ref/libsgmref.so) through its public API on
the GPU, host buffers in and out, as the reference's console measures itself.
TEST INFRASTRUCTURE: gives the reference-build numbers the engine is compared against.

    python oracle/time_reference.py [--n 50]

Only configurations whose kernels stay inside their shared-memory allocations are run
(disparity range 64 at the plain level, 32 at pyramid levels).
"""
import argparse
import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
from fasterstereocuda_b200 import scenes  # noqa: E402
from tests.golden.make_golden import RefCase, ref_lib  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    a = ap.parse_args()
    lib = ref_lib()
    lib.ref_time_pyr.argtypes = [C.c_int] * 7 + [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
    lib.ref_time_pyr.restype = C.c_double
    L, R, _ = scenes.kitti_like(100, 1242, 375)
    out = {}
    plain = RefCase(width=1242, height=375, min_disp=0, disp_range=64, cs_type=1, p1=10, p2=150, uniqueness=0.95,
                    do_lr_check=1, lr_threshold=1.0, do_median=1, morphology=0, do_remove_peaks=0, peaks_ratio=0.0)
    ms = lib.ref_time_match(C.byref(plain), L.ctypes.data, R.ctypes.data, a.warmup, a.n)
    out["plain_1242x375x64_9x7_lr_median"] = {"ms_per_pair": ms, "pairs_per_s": 1e3 / ms if ms > 0 else None}
    ms = lib.ref_time_pyr(1242, 375, 0, 64, 3, 1, 1, L.ctypes.data, R.ctypes.data, a.warmup, a.n)
    out["pyramid_1242x375_3layers_reference_params"] = {"ms_per_pair": ms, "pairs_per_s": 1e3 / ms if ms > 0 else None,
                                                         "note": "census 5x5, P1 8, P2 32 (hard-coded per level)"}
    L0, R0, _ = scenes.cone_like(100)
    cone = RefCase(width=450, height=375, min_disp=0, disp_range=64, cs_type=1, p1=10, p2=150, uniqueness=0.95,
                   do_lr_check=1, lr_threshold=1.0, do_median=1, morphology=0, do_remove_peaks=0, peaks_ratio=0.0)
    ms = lib.ref_time_match(C.byref(cone), L0.ctypes.data, R0.ctypes.data, a.warmup, a.n)
    out["plain_450x375x64_9x7_lr_median"] = {"ms_per_pair": ms, "pairs_per_s": 1e3 / ms if ms > 0 else None}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
