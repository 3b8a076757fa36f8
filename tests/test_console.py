"""The headless console (python -m fasterstereocuda_b200.console), the reference's
FasterStereoConsole (FasterStereoConsole/FasterStereoConsole.cpp:80-337) without display windows:
argument modes, option files, the per-frame timing line and the written maps."""
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from fasterstereocuda_b200 import scenes

ROOT = Path(__file__).resolve().parent.parent


def run(args, cwd):
    env = dict(os.environ, PYTHONPATH=str(ROOT))
    return subprocess.run([sys.executable, "-m", "fasterstereocuda_b200.console", *args], cwd=cwd, env=env,
                          capture_output=True, text=True, timeout=600)


def write_pair(dirpath, name, L, R):
    import cv2
    os.makedirs(dirpath / "l", exist_ok=True)
    os.makedirs(dirpath / "r", exist_ok=True)
    cv2.imwrite(str(dirpath / "l" / f"{name}.png"), L)
    cv2.imwrite(str(dirpath / "r" / f"{name}.png"), R)


def test_console_modes_without_a_device(tmp_path, engine_lib):
    """Argument errors, the option-file mode and unreadable data need no GPU."""
    r = run(["a.png", "b.png"], tmp_path)
    assert r.returncode == 1 and "insufficient parameters!" in r.stdout
    r = run(["opt"], tmp_path)
    assert r.returncode == 0 and "initialize parameter file of algorithm done!" in r.stdout
    assert (tmp_path / "option.xml").exists() and (tmp_path / "option2.xml").exists()
    assert "<Option1>" in (tmp_path / "option.xml").read_text()
    assert "<Option2>" in (tmp_path / "option2.xml").read_text()
    r = run(["missing_l.png", "missing_r.png", "option.xml"], tmp_path)
    assert r.returncode == 1 and "data error!" in r.stdout
    (tmp_path / "bad.xml").write_text("<Nothing/>")
    r = run(["a.png", "b.png", "bad.xml"], tmp_path)
    assert r.returncode == 1 and "loading parameters of algorithm failed!" in r.stdout


@pytest.mark.gpu
def test_console_matches_a_pair_and_prints_the_timing_line(tmp_path, engine_lib, oracle_mod):
    """Mode 1 on a synthetic 450x375 pair with a one-layer option file (the reference's Cone
    set-up: disparities 0..64, LR check and small-region removal); the written float map is the
    oracle's map of FasterStereoCuda::Match with the reference's per-level parameters."""
    import fasterstereocuda_b200 as fsc
    from fasterstereocuda_b200.console import read_pfm
    from fasterstereocuda_b200.options import OptionManager
    O = oracle_mod
    W, H = 450, 375
    L, R, _ = scenes.cone_like(81)
    write_pair(tmp_path, "cone", L, R)
    opt = fsc.StereoOption1(width=W, height=H, min_disp=0, max_disp=64, num_layers=1, do_lr_check=True,
                            do_rm_peaks=True)
    OptionManager()._save(str(tmp_path / "option.xml"), opt)
    r = run([str(tmp_path / "l" / "cone.png"), str(tmp_path / "r" / "cone.png"), str(tmp_path / "option.xml"),
             "--frames", "4", "--out", str(tmp_path / "out")], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("frame")]
    assert len(lines) == 4
    for l in lines:
        m = re.fullmatch(r"frame 0, timing: +([0-9.]+) ms fps = +([0-9.]+)", l)
        assert m and float(m.group(1)) > 0 and float(m.group(2)) > 0, l
    d = read_pfm(str(tmp_path / "out" / "cone.pfm"))
    strips = max(1, (os.cpu_count() or 1) * 3 // 4)
    want = O.pyr_match(O.PyrConfig(width=W, height=H, min_disp=0, max_disp=64, num_layers=1, override_enable=0,
                                   peaks_strips=strips), L, R)
    assert np.array_equal(d.view(np.uint32), want.view(np.uint32)), int((d != want).sum())
    assert (tmp_path / "out" / "cone.png").exists()


@pytest.mark.gpu
def test_console_folder_mode_and_depth_options(tmp_path, engine_lib, oracle_mod):
    """Mode 2 over two folders of pairs with an <Option2> file (depth through Init2 / Match2)."""
    import fasterstereocuda_b200 as fsc
    from fasterstereocuda_b200.console import read_pfm
    from fasterstereocuda_b200.options import OptionManager
    O = oracle_mod
    W, H, layers = 640, 376, 2
    pairs = {f"p{k}": scenes.kitti_like(90 + k, W, H)[:2] for k in range(2)}
    for name, (L, R) in pairs.items():
        write_pair(tmp_path, name, L, R)
    epi = fsc.EpipolarStereoParam(x0_left=320.0, y0_left=188.0, x0_right=330.0, y0_right=188.0, baseline=540.0,
                                  focus=720.0)
    opt = fsc.StereoOption2(width=W, height=H, min_depth=5000.0, max_depth=60000.0, num_layers=layers,
                            do_lr_check=True, do_rm_peaks=True, epi=epi)
    OptionManager()._save(str(tmp_path / "option2.xml"), opt)
    r = run([str(tmp_path / "l"), str(tmp_path / "r"), "png", str(tmp_path / "option2.xml"), "--out",
             str(tmp_path / "out")], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert len([l for l in r.stdout.splitlines() if l.startswith("frame")]) == 2
    strips = max(1, (os.cpu_count() or 1) * 3 // 4)
    m0, d0 = O.pyr_init2_coarsest(W, layers, 5000.0, 60000.0, 320.0, 330.0, 720.0, 540.0)
    s = 2 ** (layers - 1)
    pc = O.PyrConfig(width=W, height=H, min_disp=m0 * s, max_disp=(m0 + d0) * s, num_layers=layers,
                     override_enable=0, peaks_strips=strips)
    for name, (L, R) in pairs.items():
        want = O.depth_from_disp(O.pyr_match(pc, L, R), 320.0, 330.0, 720.0, 540.0)
        got = read_pfm(str(tmp_path / "out" / f"{name}.pfm"))
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (name, int((got != want).sum()))
