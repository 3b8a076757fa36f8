"""Oracle vs the reference's own host functions (RemovePeaks, Zoom, ComputeInitDispInNextLevel).

Golden fixture tests/golden/host_ops.npz was produced by tests/golden/make_golden.py from the
reference built from its sources; when that build is present the live reference is compared too.
"""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
REF_SO = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "libsgmref.so"


@pytest.fixture(scope="module")
def host_ops():
    return dict(np.load(GOLDEN / "host_ops.npz"))


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


def test_remove_peaks_strip_matches_reference(oracle_mod, host_ops):
    n = 0
    for k in host_ops:
        if k.startswith("peaks_") and k.endswith("_in"):
            base = k[:-3]
            thr = int(base.split("_")[2])
            out, cnt = oracle_mod.remove_peaks_strip(host_ops[k], thr, 0)
            assert np.array_equal(_bits(out), _bits(host_ops[base + "_out"])), base
            assert cnt == int(host_ops[base + "_n"]), base
            n += 1
    assert n == 9


def test_remove_peaks_float_mode_differs(oracle_mod, host_ops):
    """The g++ build merges |d| < 2 (int abs); the float rule (MSVC build) must give other results."""
    d = host_ops["peaks_1_11_in"]
    a, _ = oracle_mod.remove_peaks_strip(d, 11, 0)
    b, _ = oracle_mod.remove_peaks_strip(d, 11, 1)
    assert not np.array_equal(a, b)


def test_zoom_matches_reference(oracle_mod, host_ops):
    for k in ("zoom_0", "zoom_1", "zoom_2"):
        assert np.array_equal(oracle_mod.zoom_half(host_ops[k + "_in"]), host_ops[k + "_out"]), k


def test_init_next_level_matches_reference(oracle_mod, host_ops):
    for k in ("initnext_0", "initnext_1", "initnext_2", "initnext_3"):
        w, h = (int(v) for v in host_ops[k + "_size"])
        assert np.array_equal(oracle_mod.init_next_level(host_ops[k + "_in"], w, h), host_ops[k + "_out"]), k


@pytest.mark.skipif(not REF_SO.exists(), reason="reference not built here (oracle/build_ref.sh)")
def test_live_reference_remove_peaks_random(oracle_mod):
    import ctypes as C
    lib = C.CDLL(str(REF_SO))
    lib.ref_remove_peaks.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
    rng = np.random.Generator(np.random.PCG64(99))
    for trial in range(20):
        w, h = int(rng.integers(8, 90)), int(rng.integers(4, 40))
        d = (rng.integers(0, 6, size=(h, w)) * 0.9 + rng.normal(0, 0.3, size=(h, w))).astype(np.float32)
        d[rng.random((h, w)) < 0.2] = -999999.0
        thr = int(rng.integers(1, 30))
        ref = d.copy()
        seg = np.zeros((h, w), np.int32)
        lib.ref_remove_peaks(ref.ctypes.data, seg.ctypes.data, w, h, thr)
        out, _ = oracle_mod.remove_peaks_strip(d, thr, 0)
        assert np.array_equal(_bits(out), _bits(ref)), trial
