"""Batched matching (sgm_batch_*): many pairs of different sizes and disparity ranges in one CUDA
graph launch, each pair bit-identical to the oracle and to the single-pair engine."""
import numpy as np
import pytest

from fasterstereocuda_b200 import scenes

STRIPS = 6


def option(fsc, cs=1, lr=True, med=True, p1=10, p2=150, u=0.95):
    return fsc.CuSGMOption(p1=p1, p2_init=p2, cs_type=cs, num_paths=4, do_median_filter=med, do_lr_check=lr,
                           lr_threshold=1.0, unique_threshold=u, using_constant_p2=True)


def test_batch_rejects_unsupported_before_any_device_call(engine_lib):
    import fasterstereocuda_b200 as fsc
    b = fsc.StereoBatch()
    assert not b.Init([(320, 240, 0, 96)], option(fsc)) and b.status == -4
    assert "disparity range 96" in b.last_error()
    assert not b.Init([(0, 240, 0, 64)], option(fsc)) and b.status == -1
    o = option(fsc)
    o.do_remove_peaks = True
    assert not b.Init([(320, 240, 0, 64)], o) and b.status == -4
    o = option(fsc)
    o.cs_type = 3
    assert not b.Init([(320, 240, 0, 64)], o) and b.status == -1
    assert not b.Init([], option(fsc)) and b.status == -1
    with pytest.raises(RuntimeError):
        b.buffers(0)


SMALL = [  # (W, H, min_disp, D)
    (203, 131, 0, 64), (96, 64, 0, 32), (320, 200, -3, 128), (150, 240, 5, 64), (257, 97, 0, 64),
    (131, 77, 0, 128), (400, 120, 0, 32), (64, 300, 0, 64),
]


def _pairs(specs, seed0):
    out = []
    for i, (W, H, M, D) in enumerate(specs):
        L, R, _ = scenes.planar_pair(seed0 + i, W, H, dmin=2.0, dmax=min(60.0, D - 4.0))
        out.append((L, R))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("cs,lr,med", [(1, True, True), (0, True, True), (1, False, True), (1, True, False)])
def test_batch_matches_oracle_bit_exact(engine_lib, oracle_mod, cs, lr, med):
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    p1, p2 = (10, 150) if cs == 1 else (8, 32)
    b = fsc.StereoBatch()
    assert b.Init(SMALL, option(fsc, cs, lr, med, p1, p2)), b.last_error()
    imgs = _pairs(SMALL, 300)
    outs = [np.full((H, W), 7.0, np.float32) for (W, H, _, _) in SMALL]
    assert b.Match([L for L, _ in imgs], [R for _, R in imgs], outs), b.last_error()
    for (W, H, M, D), (L, R), got in zip(SMALL, imgs, outs):
        cfg = O.Config(width=W, height=H, min_disp=M, disp_range=D, cs_type=cs, p1=p1, p2=p2, uniqueness=0.95,
                       do_lr_check=int(lr), do_median=int(med), peaks_strips=STRIPS)
        exp = O.match(cfg, L, R)["disp"]
        neq = got.view(np.uint32) != exp.view(np.uint32)
        assert not neq.any(), ((W, H, M, D), int(neq.sum()), np.argwhere(neq)[:3].tolist())
    info = b.info()
    assert info["pairs"] == len(SMALL) and 2 + 2 * info["buckets"] <= info["kernels_per_run"] <= 2 + 3 * info["buckets"]


@pytest.mark.gpu
def test_batch_graph_replays_with_new_inputs_and_device_buffers(engine_lib):
    """Runs in a row with different images written into the arena's device buffers and launched
    on a caller stream, against one StereoCuda per pair; re-tuning changes nothing."""
    import torch
    import fasterstereocuda_b200 as fsc
    b = fsc.StereoBatch()
    o = option(fsc)
    assert b.Init(SMALL, o), b.last_error()
    stream = torch.cuda.current_stream()
    for rnd in range(3):
        if rnd == 2:
            assert b.autotune(), b.last_error()
        imgs = _pairs(SMALL, 400 + 50 * (rnd % 2))
        staged = [(torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()) for L, R in imgs]
        for i, (tl, tr) in enumerate(staged):
            dl, dr, _ = b.buffers(i)
            _memcpy(dl, tl.data_ptr(), tl.numel())
            _memcpy(dr, tr.data_ptr(), tr.numel())
        assert b.run(stream.cuda_stream), b.last_error()
        torch.cuda.synchronize()
        for i, ((W, H, M, D), (L, R)) in enumerate(zip(SMALL, imgs)):
            _, _, dd = b.buffers(i)
            got = torch.empty((H, W), dtype=torch.float32, device="cuda")
            _memcpy(got.data_ptr(), dd, H * W * 4)
            got = got.cpu().numpy()
            s = fsc.StereoCuda()
            assert s.Init(W, H, M, D, o), s.last_error()
            exp = np.empty((H, W), np.float32)
            assert s.Match(L, R, exp), s.last_error()
            assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), (rnd, i)


def _memcpy(dst, src, n):
    """Synchronous device-to-device copy between raw addresses (CUDA runtime binding)."""
    import torch
    from cuda.bindings import runtime as rt
    torch.cuda.synchronize()
    (err,) = rt.cudaMemcpy(dst, src, n, rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
    assert err == rt.cudaError_t.cudaSuccess, err


@pytest.mark.gpu
def test_batch_of_uneven_full_size_pairs_equals_per_pair_engine(engine_lib):
    """The first 12 pairs of the 64-pair uneven batch (widths 320..1920, heights 240..1080,
    D in {64, 128}) at full size, batch vs StereoCuda per pair, bit for bit."""
    import fasterstereocuda_b200 as fsc
    specs = scenes.batch_specs()[:12]
    pairs = [(w, h, 0, d) for (w, h, d, _) in specs]
    o = option(fsc)
    b = fsc.StereoBatch()
    assert b.Init(pairs, o), b.last_error()
    imgs = [scenes.planar_pair(seed, w, h)[:2] for (w, h, d, seed) in specs]
    outs = [np.empty((h, w), np.float32) for (w, h, _, _) in pairs]
    assert b.Match([L for L, _ in imgs], [R for _, R in imgs], outs), b.last_error()
    for (w, h, m, d), (L, R), got in zip(pairs, imgs, outs):
        s = fsc.StereoCuda()
        assert s.Init(w, h, m, d, o), s.last_error()
        exp = np.empty((h, w), np.float32)
        assert s.Match(L, R, exp), s.last_error()
        assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), (w, h, d)
        assert (got != -999999.0).mean() > 0.5
    buckets = b.buckets()
    assert sum(k["pairs"] for k in buckets) == 12
    assert all(k["rows_ctas"] > 0 and k["cols_ctas"] > 0 for k in buckets)


PYR_PAIRS = [(640, 360, 0, 64), (450, 375, 0, 64), (1242, 375, 0, 64), (800, 600, 0, 64), (320, 256, 0, 64)]


def test_batch_pyramid_rejects_before_any_device_call(engine_lib):
    import fasterstereocuda_b200 as fsc
    b = fsc.StereoBatchPyramid()
    opt = fsc.StereoOption1(num_layers=3, do_lr_check=True, do_rm_peaks=True)
    assert not b.Init([(64, 24, 0, 64)], opt) and b.status == -1 and "too many layers" in b.last_error()
    assert not b.Init([], fsc.StereoOption1(num_layers=3)) and b.status == -1


@pytest.mark.gpu
@pytest.mark.parametrize("layers,override,smooth", [(3, True, False), (3, False, False), (2, True, False),
                                                    (1, True, False), (3, True, True), (1, False, True)])
def test_batch_pyramid_equals_per_pair_pyramid(engine_lib, oracle_mod, layers, override, smooth):
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    opt = fsc.StereoOption1(num_layers=layers, do_lr_check=True, do_rm_peaks=True, do_smooth=smooth)
    ov = fsc.LevelOverride(1, 10, 150) if override else None
    ext = fsc.ExtOptions(peaks_strips=STRIPS)
    b = fsc.StereoBatchPyramid()
    assert b.Init(PYR_PAIRS, opt, ov, ext), b.last_error()
    imgs = [scenes.kitti_like(500 + i, w, h)[:2] for i, (w, h, _, _) in enumerate(PYR_PAIRS)]
    outs = [np.full((h, w), 7.0, np.float32) for (w, h, _, _) in PYR_PAIRS]
    for rnd in range(2):  # two graph launches in a row
        assert b.Match([L for L, _ in imgs], [R for _, R in imgs], outs), b.last_error()
        for i, ((w, h, mn, mx), (L, R)) in enumerate(zip(PYR_PAIRS, imgs)):
            p = fsc.FasterStereoCuda()
            assert p.Init(fsc.StereoOption1(width=w, height=h, min_disp=mn, max_disp=mx, num_layers=layers,
                                            do_lr_check=True, do_rm_peaks=True, do_smooth=smooth), ov, ext), \
                p.last_error()
            exp = np.empty((h, w), np.float32)
            assert p.Match(L, R, exp)
            assert np.array_equal(outs[i].view(np.uint32), exp.view(np.uint32)), (rnd, i, int((outs[i] != exp).sum()))
    # one pair against the oracle as well
    w, h, mn, mx = PYR_PAIRS[1]
    pc = O.PyrConfig(width=w, height=h, min_disp=mn, max_disp=mx, num_layers=layers, override_enable=int(override),
                     cs_type=1 if override else 0, p1=10 if override else 8, p2=150 if override else 32,
                     peaks_strips=STRIPS, do_smooth=int(smooth))
    ref = O.pyr_match(pc, *imgs[1])
    if smooth:  # exp() of CUDA vs the host's libm: masks equal, values within 1e-4 px
        assert np.array_equal(outs[1] == -999999.0, ref == -999999.0)
        ok = ref != -999999.0
        assert np.abs(outs[1][ok] - ref[ok]).max() <= 1e-4
    else:
        assert np.array_equal(outs[1].view(np.uint32), ref.view(np.uint32))
    assert b.info()["pairs"] == len(PYR_PAIRS)


@pytest.mark.gpu
@pytest.mark.parametrize("pyramid", [True, False])
def test_profiled_batch_run_equals_graph_run(engine_lib, pyramid):
    """With the per-launch profiler on, a batch run enqueues its kernels one at a time on the
    caller's stream instead of launching its graph: the same bits, and every kernel timed."""
    import torch
    import fasterstereocuda_b200 as fsc
    if pyramid:
        b = fsc.StereoBatchPyramid()
        pairs = PYR_PAIRS
        assert b.Init(pairs, fsc.StereoOption1(num_layers=3, do_lr_check=True, do_rm_peaks=True),
                      fsc.LevelOverride(1, 10, 150), fsc.ExtOptions(peaks_strips=STRIPS)), b.last_error()
        imgs = [scenes.kitti_like(520 + i, w, h)[:2] for i, (w, h, _, _) in enumerate(pairs)]
    else:
        b = fsc.StereoBatch()
        pairs = SMALL
        assert b.Init(pairs, option(fsc)), b.last_error()
        imgs = _pairs(pairs, 470)
    for i, (L, R) in enumerate(imgs):
        tl, tr = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
        dl, dr, _ = b.buffers(i)
        _memcpy(dl, tl.data_ptr(), tl.numel())
        _memcpy(dr, tr.data_ptr(), tr.numel())

    def outputs():
        res = []
        for i, p in enumerate(pairs):
            w, h = p[0], p[1]
            got = torch.empty((h, w), dtype=torch.float32, device="cuda")
            _memcpy(got.data_ptr(), b.buffers(i)[2], h * w * 4)
            res.append(got.cpu().numpy())
        return res

    stream = torch.cuda.current_stream().cuda_stream
    assert b.run(stream), b.last_error()
    torch.cuda.synchronize()
    want = outputs()
    try:
        fsc.profile_enable(True)
        for i, p in enumerate(pairs):  # stale outputs must not pass
            torch.cuda.synchronize()
            fill = torch.full((p[1], p[0]), 3.0, dtype=torch.float32, device="cuda")
            _memcpy(b.buffers(i)[2], fill.data_ptr(), p[0] * p[1] * 4)
        assert b.run(stream), b.last_error()
        torch.cuda.synchronize()
        prof = fsc.profile_read()
    finally:
        fsc.profile_enable(False)
    got = outputs()
    for i in range(len(pairs)):
        assert np.array_equal(got[i].view(np.uint32), want[i].view(np.uint32)), i
    names = set(prof)
    assert {"census", "lr_median"} <= names, names
    assert any(k.startswith("hpaths") for k in names) and any(k.startswith("vpaths") for k in names), names
    if pyramid:
        assert {"decimate", "init_next_level", "hpaths_init", "vpaths_wta_init", "cc_rows"} <= names, names
    assert all(v["launches"] >= 1 and v["ms"] > 0 for v in prof.values()), prof
