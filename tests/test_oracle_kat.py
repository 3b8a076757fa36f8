"""Known-answer tests of the oracle on hand-computed tiny cases."""
import numpy as np
import pytest

INV = np.float32(-999999.0)


def test_census_9x7_bits(oracle_mod):
    img = np.zeros((7, 9), np.uint8)
    img[3, 4] = 100                      # centre
    img[0, 0] = 50                       # first window element: MSB of 63 bits (bit 62)
    img[6, 8] = 50                       # last element: bit 0
    img[3, 3] = 200                      # not smaller -> 0
    c = oracle_mod.census(img, 1, False)
    # every other neighbour is 0 < 100 -> 1, except (3,3) (200) and the centre itself
    expect = (1 << 63) - 1
    expect &= ~(1 << (63 - 1 - (3 * 9 + 3)))      # (3,3)
    expect &= ~(1 << (63 - 1 - (3 * 9 + 4)))      # centre compares with itself: 0
    assert int(c[3, 4]) == expect
    # border pixels: left view 0, right view 0xFFFFFFFF
    assert int(c[0, 0]) == 0
    assert int(oracle_mod.census(img, 1, True)[0, 0]) == 0xFFFFFFFF


def test_census_5x5_is_24_bits(oracle_mod):
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, size=(20, 20), dtype=np.uint8)
    c = oracle_mod.census(img, 0, False)
    assert int(c[2:-2, 2:-2].max()) < (1 << 25)
    assert np.all((c[2:-2, 2:-2] >> np.uint64(12)) & np.uint64(1) == 0)   # centre bit (position 12) is 0


def test_cost_adjust_table(oracle_mod):
    assert [oracle_mod.cost_adjust(d) for d in (16, 13, 12, 8, 4, 0, 31)] == [1, 1, 2, 7, 20, 54, 20]


def test_median_and_dilation(oracle_mod):
    d = np.arange(25, dtype=np.float32).reshape(5, 5)
    d[2, 2] = 100.0
    m = oracle_mod.median3x3(d)
    assert m[2, 2] == 13.0                       # median of 6,7,8,11,100,13,16,17,18
    assert m[0, 0] == d[0, 0]                    # border untouched
    e = np.full((7, 7), INV, np.float32)
    e[1, 1] = 5.0
    e[3, 5] = 9.0
    out = oracle_mod.dilation(e, 3)
    assert out[2, 2] == 5.0 and out[3, 4] == 9.0 and out[0, 0] == INV   # interior only


def test_lr_rounding_half_away(oracle_mod):
    # one row: dL(x=5) = 2.5 -> xr = round(2.5) = 3 ; dR[3] = 2.0 -> |0.5| <= 1 -> (2.5+2)/2
    W = 8
    dl = np.full((1, W), INV, np.float32)
    dr = np.full((1, W), 9.0, np.float32)
    dl[0, 5] = 2.5
    dr[0, 3] = 2.0
    dl[0, 1] = 3.5          # x - d = -2.5 -> -3 -> out of range -> INVALID
    import ctypes as C
    lib = oracle_mod.lib()
    out_r = dr.copy()
    lib.orc_lr_check(dl.ctypes.data, dr.ctypes.data, out_r.ctypes.data, W, 1, C.c_float(1.0))
    assert dl[0, 5] == np.float32(2.25) and dl[0, 1] == INV


def _recurrence(C, P1, P2):
    """Direct restatement on python ints for a single scanline (for the KAT below)."""
    D = C.shape[1]
    L = [int(v) for v in C[0]]
    out = [list(L)]
    m = min(L)
    for p in range(1, C.shape[0]):
        nl = []
        for d in range(D):
            a = L[d - 1] + P1 if d > 0 else 127
            b = L[d + 1] + P1 if d < D - 1 else 127
            t = min(L[d], a, b, m + P2)
            nl.append((int(C[p, d]) + t - m) & 0xFFFFFFFF)
        L = nl
        m = min(L)
        out.append(list(L))
    return np.array(out) & 0xFF


def test_path_recurrence_d4(oracle_mod):
    """4 pixels x D=4 by hand: row 0 = C; then min(L(d), L(d±1)+P1, m+P2) - m."""
    C = np.array([[5, 1, 4, 9], [2, 8, 8, 3], [7, 0, 6, 6], [1, 1, 1, 1]], np.uint8)
    exp = _recurrence(C, 2, 6)
    # hand check of the second row: m=1; d0: min(5, 127, 1+2, 7)=3 -> 2+3-1 = 4
    assert exp[1, 0] == 4
    # the oracle's left->right path on a 1-row image whose cost volume is C
    import ctypes as Cc
    lib = oracle_mod.lib()
    lib.orc_path_plain.argtypes = [Cc.c_void_p, Cc.c_int, Cc.c_int, Cc.c_int, Cc.c_int, Cc.c_int32, Cc.c_int32,
                                   Cc.c_int, Cc.c_void_p]
    cost = np.ascontiguousarray(C.reshape(1, 4, 4))
    out = np.zeros_like(cost)
    lib.orc_path_plain(cost.ctypes.data, 4, 1, 0, 4, 2, 6, 1, out.ctypes.data)
    assert np.array_equal(out[0], exp.astype(np.uint8))


def test_subpixel_formula(oracle_mod):
    """WTA at one pixel: S = (.., 20, 10, 14, ..) at d*=3 -> 3 + (20-14+14)/(2*14)."""
    W, H, D = 16, 16, 32
    paths = np.zeros((4, H, W, D), np.uint8)
    S = np.full(D, 60, np.uint8)
    S[2], S[3], S[4] = 20, 10, 14
    paths[0, 8, 8] = S
    import ctypes as Cc
    lib = oracle_mod.lib()
    lib.orc_wta_plain.argtypes = [Cc.c_void_p * 4, Cc.c_int, Cc.c_int, Cc.c_int, Cc.c_int, Cc.c_int, Cc.c_float,
                                  Cc.c_int, Cc.c_void_p]
    arr = (Cc.c_void_p * 4)(*[paths[k].ctypes.data for k in range(4)])
    disp = np.zeros((H, W), np.float32)
    lib.orc_wta_plain(arr, W, H, 0, 0, D, Cc.c_float(0.95), 0, disp.ctypes.data)
    den = np.float32(20 + 14 - 2 * 10)
    assert disp[8, 8] == np.float32(3) + (np.float32(20 - 14) + den) / (np.float32(2) * den)
    assert disp[0, 0] == INV
