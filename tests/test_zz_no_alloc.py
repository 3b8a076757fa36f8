"""sgm_match_noalloc: matching for callers that cannot allocate device memory.

Some callers may not call cudaMalloc once they are running: real-time loops that forbid
allocation after start-up, and plugin hosts that own the GPU memory budget and hand a plugin only
its input and output buffers. sgm_match_noalloc serves them from a fixed 64 MiB working array
inside the library. These tests call it through the C ABI and compare it, bit for bit (the
tolerance every parity test here uses), with the allocating entry point on two calls in a row,
and with the oracle across disparity ranges, census sizes and minimum disparities.
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
    # sizes whose byte counts would wrap, grids beyond the launch limit, empty disparity search
    assert fn(dummy, dummy, dummy, 1 << 30, 1 << 30, 0, 32, C.byref(opt), None) == -1
    assert "too large" in engine_lib.sgm_last_error(None).decode()
    assert fn(dummy, dummy, dummy, 16, 70000, 0, 32, C.byref(opt), None) == -1
    assert "65535" in engine_lib.sgm_last_error(None).decode()
    assert fn(dummy, dummy, dummy, 320, 240, 320, 64, C.byref(opt), None) == -1
    assert "minimum disparity" in engine_lib.sgm_last_error(None).decode()


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


@pytest.mark.gpu
@pytest.mark.parametrize("D,cs,M", [(32, 1, 0), (128, 1, 0), (64, 0, 0), (64, 1, 6), (64, 1, -5), (32, 0, 3)])
def test_noalloc_matches_the_oracle(engine_lib, oracle_mod, D, cs, M):
    """Other template instantiations of the entry point: 32/128 disparities, census 5x5 (whose
    right view keeps the left cost in the last pixel of every D-pixel block), non-zero minimum
    disparities; bit for bit against the oracle and against sgm_match_device."""
    import torch
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    fn = _noalloc(engine_lib)
    W, H = 200, 120
    p1, p2 = (10, 150) if cs else (8, 32)
    opt = fsc.CuSGMOption(p1=p1, p2_init=p2, cs_type=cs, num_paths=4, do_median_filter=True, do_lr_check=True,
                          lr_threshold=1.0, unique_threshold=0.95, using_constant_p2=True)
    L, R, _ = scenes.planar_pair(70 + D + cs + M, W, H, dmin=2.0, dmax=min(60.0, D - 4.0))
    dl, dr = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    got = torch.full((H, W), 7.0, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = fn(dl.data_ptr(), dr.data_ptr(), got.data_ptr(), W, H, M, D, C.byref(opt), C.c_void_p(stream))
    assert st == 0, engine_lib.sgm_last_error(None).decode()
    ref = fsc.StereoCuda()
    assert ref.Init(W, H, M, D, opt), ref.last_error()
    want = torch.empty((H, W), dtype=torch.float32, device="cuda")
    assert ref.match_device(dl, dr, want, None, None, stream), ref.last_error()
    torch.cuda.synchronize()
    a = got.cpu().numpy()
    cfg = O.Config(width=W, height=H, min_disp=M, disp_range=D, cs_type=cs, p1=p1, p2=p2)
    exp = O.match(cfg, L, R)["disp"]
    assert np.array_equal(a.view(np.uint32), exp.view(np.uint32)), int((a != exp).sum())
    assert np.array_equal(a.view(np.uint32), want.cpu().numpy().view(np.uint32))
