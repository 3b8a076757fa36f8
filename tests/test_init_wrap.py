"""32-disparity levels where the reference's uint32 recurrence wraps.

After a realignment beyond the disparity range every neighbour candidate is 127, so when the
previous minimum m exceeds 127 + C all new path costs wrap below zero; alternating such pixels
with invalid-cost (255) pixels grows |m| by up to 255 every two steps. The CUDA kernels run the
recurrence in 16 bits while |m| <= 8192 at the end of every block of up to 8 steps and continue
a scanline in 32 bits beyond that; these cases drive |m| far past 2^15, so a 16-bit-only form
would differ from the oracle.
"""
import numpy as np
import pytest

from fasterstereocuda_b200 import scenes

STRIPS = 6
M32 = 1 << 32


def adversarial_init(kind, W, H, seed=0):
    """Initial disparities: 'cols' alternates base 0 / 2000 along each row (every pixel a
    realignment beyond the range, the 2000 pixels all invalid cost), 'rows' along each column,
    'random' draws bases in [-40, 80) with 10 % INVALID."""
    if kind == "cols":
        row = np.where(np.arange(W) % 2 == 0, 0, 2000)
        return np.ascontiguousarray(np.broadcast_to(row, (H, W))).astype(np.int16)
    if kind == "rows":
        col = np.where(np.arange(H) % 2 == 0, 0, 2000)[:, None]
        return np.ascontiguousarray(np.broadcast_to(col, (H, W))).astype(np.int16)
    rng = np.random.default_rng(seed)
    init = rng.integers(-40, 80, (H, W)).astype(np.int16)
    init[rng.random((H, W)) < 0.1] = -32768
    return init


def scanline_minima(cost, bases, p1, p2, p2_div0=-1):
    """The path recurrence of one left-to-right scanline at a 32-disparity level (as the oracle's
    orc_path_init), in exact integers modulo 2^32. Returns (stored u8 path costs, signed m per
    step)."""
    D = cost.shape[1]
    Lq = [int(c) for c in cost[0]]
    m = min(Lq)
    last = int(bases[0])
    out = [np.array(Lq, np.int64) & 0xFF]
    ms = [m]
    for s in range(1, cost.shape[0]):
        base = int(bases[s])
        if base == -32768:
            m = 127
            out.append(None)
            ms.append(m)
            continue
        div = abs(last - base + 1)
        q = int(p2 / div) if div else p2_div0
        l4 = (m + max(p1, q)) % M32
        Lp = []
        for d in range(D):
            i1, i2 = d + base - 1 - last, d + base + 1 - last
            a = (Lq[i1] + p1) % M32 if 0 <= i1 < D else 127
            b = (Lq[i2] + p1) % M32 if 0 <= i2 < D else 127
            Lp.append((int(cost[s][d]) + min(Lq[d], a, b, l4) - m) % M32)
        Lq, m, last = Lp, min(Lp), base
        out.append(np.array(Lp, np.int64) & 0xFF)
        ms.append(m)
    return out, [v - M32 if v >= 1 << 31 else v for v in ms]


def test_alternating_realignment_drives_minimum_past_16_bits(oracle_mod):
    """The 'cols' case really leaves the 16-bit range: an exact-integer model of the recurrence
    agrees with the oracle's stored path costs and its |m| passes 2^15."""
    O = oracle_mod
    W, H = 720, 4
    L, R, _ = scenes.planar_pair(71, W, H)
    init = adversarial_init("cols", W, H)
    cfg = O.Config(width=W, height=H, disp_range=32, cs_type=1, p1=10, p2=150, uniqueness=0.95, do_lr_check=0,
                   do_median=1, peaks_strips=STRIPS)
    ref = O.match(cfg, L, R, init, dump=True)
    y = 2
    out, ms = scanline_minima(ref["cost"][y], init[y], 10, 150)
    for x, v in enumerate(out):
        if v is not None:
            assert np.array_equal(v, ref["paths"][1][y, x]), x
    assert max(abs(v) for v in ms) > 1 << 15
    assert min(ms) < -(1 << 15)


def test_minimum_grows_at_most_382_plus_p2_per_step():
    """The bound behind the 16-bit form: per step |m| and every |L| grow by at most 382 + P2'
    over the |m| the step started from, on random scanlines with random realignments, INVALID
    bases and cost 255 pixels."""
    rng = np.random.default_rng(11)
    for trial in range(40):
        n = 60
        p1 = int(rng.integers(0, 40))
        p2 = int(rng.integers(p1, 2048))
        cost = rng.integers(0, 118, (n, 32))
        cost[rng.random(n) < 0.3] = 255
        bases = rng.choice([0, 1, -1, 3, 40, -40, 2000], size=n).astype(np.int64)
        bases[rng.random(n) < 0.1] = -32768
        bases[0] = 0
        Lq = [int(c) for c in cost[0]]
        m, last = min(Lq), 0
        for s in range(1, n):
            base = int(bases[s])
            if base == -32768:
                m = 127
                continue
            div = abs(last - base + 1)
            q = int(p2 / div) if div else -1
            p2p = max(p1, q)
            ms = m - M32 if m >= 1 << 31 else m
            Lp = []
            for d in range(32):
                i1, i2 = d + base - 1 - last, d + base + 1 - last
                a = (Lq[i1] + p1) % M32 if 0 <= i1 < 32 else 127
                b = (Lq[i2] + p1) % M32 if 0 <= i2 < 32 else 127
                Lp.append((int(cost[s][d]) + min(Lq[d], a, b, (m + p2p) % M32) - m) % M32)
            signed = [v - M32 if v >= 1 << 31 else v for v in Lp]
            assert max(abs(v) for v in signed) <= abs(ms) + 382 + p2p, (trial, s)
            Lq, m, last = Lp, min(Lp), base
            m_new = m - M32 if m >= 1 << 31 else m
            assert abs(m_new) <= abs(ms) + 382 + p2p, (trial, s)


@pytest.mark.gpu
@pytest.mark.parametrize("lanes", [(2, 2), (4, 4), (8, 8)])
@pytest.mark.parametrize("p1,p2", [(10, 150), (10, 2047), (10, 9000)])
@pytest.mark.parametrize("kind", ["cols", "rows", "random"])
def test_wrapping_paths_match_oracle(engine_lib, oracle_mod, kind, p1, p2, lanes):
    """Path volumes and disparities bit-exact on the wrapping cases, for every lane split of the
    scanline kernels; P2 = 2047 is the largest penalty of the 16-bit form, P2 = 9000 runs them in
    32 bits from the first pixel."""
    import fasterstereocuda_b200 as fsc
    O = oracle_mod
    W, H = {"cols": (720, 40), "rows": (48, 600), "random": (300, 200)}[kind]
    L, R, _ = scenes.planar_pair(73, W, H)
    init = adversarial_init(kind, W, H, seed=5)
    s = fsc.StereoCuda()
    opt = fsc.CuSGMOption(p1=p1, p2_init=p2, cs_type=1, num_paths=4, do_median_filter=True, do_lr_check=True,
                          lr_threshold=1.0, unique_threshold=0.95, using_constant_p2=True)
    assert s.Init(W, H, 0, 32, opt), s.last_error()
    assert s.set_ext_options(fsc.ExtOptions(peaks_strips=STRIPS))
    assert s.set_tuning(fsc.Tuning(3, 0, 3, 0, 0, *lanes)), s.last_error()
    disp = np.empty((H, W), np.float32)
    assert s.Match(L, R, disp, None, init), s.last_error()
    cfg = O.Config(width=W, height=H, disp_range=32, cs_type=1, p1=p1, p2=p2, uniqueness=0.95, do_lr_check=1,
                   do_median=1, peaks_strips=STRIPS)
    ref = O.match(cfg, L, R, init, dump=True, want_right=True)
    valid = init != -32768
    for name, got, exp in [("L->R", s.debug_read("lr"), ref["paths"][1]),
                           ("R->L", s.debug_read("rl"), ref["paths"][3])]:
        neq = (got != exp).any(-1) & valid
        assert not neq.any(), (name, int(neq.sum()), np.argwhere(neq)[:3].tolist())
    bt = s.debug_read("bt")
    neq = (bt != ref["paths"][2]).any(-1) & valid
    assert not neq.any(), ("B->T", int(neq.sum()), np.argwhere(neq)[:3].tolist())
    assert np.array_equal(s.debug_read("wta", 0).view(np.uint32), ref["wta_l"].view(np.uint32))
    assert np.array_equal(s.debug_read("wta", 1).view(np.uint32), ref["wta_r"].view(np.uint32))
    assert np.array_equal(disp.view(np.uint32), ref["disp"].view(np.uint32))
