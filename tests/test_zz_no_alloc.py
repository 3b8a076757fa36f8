"""sgm_match_noalloc: matching for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc while they run (graph capture, real-time loops, plugin hosts
that own the memory budget). sgm_match_noalloc serves them from a fixed 64 MiB working array
inside the library. These tests call it through the C ABI and compare it, bit for bit (the
tolerance every parity test here uses), with the allocating entry point on two calls in a row.
This file is collected last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from fasterstereocuda_b200 import scenes


def _noalloc(lib):
    fn = lib.sgm_match_noalloc
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                   C.c_void_p]
    fn.restype = C.c_int32
    return fn


def _option(fsc, lr=True):
    return fsc.CuSGMOption(p1=10, p2_init=150, cs_type=1, num_paths=4, do_median_filter=True, do_lr_check=lr,
                           lr_threshold=1.0, unique_threshold=0.95, using_constant_p2=True)


def test_noalloc_rejects_sizes_beyond_its_working_memory(engine_lib):
    """Argument checks happen before any CUDA call, so this runs without a GPU."""
    import fasterstereocuda_b200 as fsc
    fn = _noalloc(engine_lib)
    opt = _option(fsc)
    dummy = C.c_void_p(16)  # never dereferenced: the size check fails first
    st = fn(dummy, dummy, dummy, 1920, 1080, 0, 64, C.byref(opt), None)
    assert st == -1
    msg = engine_lib.sgm_last_error(None).decode()
    assert "working memory" in msg and "67108864" in msg, msg
    assert fn(dummy, dummy, dummy, 320, 240, 0, 96, C.byref(opt), None) == -4   # unsupported range
    peaks = _option(fsc)
    peaks.do_remove_peaks = True
    assert fn(dummy, dummy, dummy, 320, 240, 0, 64, C.byref(peaks), None) == -4


@pytest.mark.gpu
@pytest.mark.parametrize("lr", [True, False])
def test_noalloc_matches_allocating_entry_point_twice(engine_lib, lr):
    import torch
    import fasterstereocuda_b200 as fsc
    fn = _noalloc(engine_lib)
    W, H, D = 320, 240, 64
    opt = _option(fsc, lr)
    ref = fsc.StereoCuda()
    assert ref.Init(W, H, 0, D, opt), ref.last_error()
    stream = torch.cuda.current_stream().cuda_stream
    for seed in (61, 62):  # two calls in a row, different inputs, shared working memory
        L, R, _ = scenes.planar_pair(seed, W, H)
        dl, dr = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
        want = torch.empty((H, W), dtype=torch.float32, device="cuda")
        got = torch.full((H, W), 7.0, dtype=torch.float32, device="cuda")
        assert ref.match_device(dl, dr, want, None, None, stream), ref.last_error()
        st = fn(dl.data_ptr(), dr.data_ptr(), got.data_ptr(), W, H, 0, D, C.byref(opt), C.c_void_p(stream))
        assert st == 0, engine_lib.sgm_last_error(None).decode()
        torch.cuda.synchronize()
        a, b = got.cpu().numpy(), want.cpu().numpy()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), int((a != b).sum())
        assert (a != -999999.0).mean() > 0.5
