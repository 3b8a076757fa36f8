"""Headless stereo console: the reference's FasterStereoConsole (FasterStereoConsole/
FasterStereoConsole.cpp:80-337) without its display windows.

    python -m fasterstereocuda_b200.console LEFT RIGHT OPTION.xml [--frames N] [--out DIR]
    python -m fasterstereocuda_b200.console LEFT_DIR RIGHT_DIR EXT OPTION.xml [--frames N] [--out DIR]
    python -m fasterstereocuda_b200.console opt

Mode 1 matches one pair, mode 2 every pair of two folders (files *.EXT, paired in name order),
mode 3 writes default option files (option.xml, option2.xml) into the working directory. The
option file chooses the interface as in the reference (OptionManager::GaussType): an <Option1> file
gives disparity maps through FasterStereoCuda::Init / Match, an <Option2> file depth maps through
Init2 / Match2. Images are read as 8-bit grey (cv2.IMREAD_GRAYSCALE, as the reference's imread).

The reference matches the pairs in an endless loop and shows each result in a window; here the loop
runs --frames matches (default: each pair once) and, with --out, writes each pair's last map as
<name>.pfm (the float map as matched, INVALID = -999999) and <name>.png (the reference's 8-bit view
of it: (d - min) / (max - min) * 255 over the valid pixels, 0 where the map is INVALID or the left
image is 0). Every frame prints the reference's timing line: the frame's wall time and the frames
per second over all frames but the first (:251-294). Errors print the reference's messages and exit
with status 1 (the reference exits with 0).
"""
from __future__ import annotations

import argparse
import ctypes as C
import glob
import os
import sys
import time

import numpy as np

from . import FasterStereoCuda, StereoOption1, StereoOption2, load_library
from .options import OptionManager

INVALID = np.float32(-999999.0)


def read_grey(path: str) -> np.ndarray | None:
    """8-bit grey image (None when it cannot be read), as imread(path, IMREAD_GRAYSCALE)."""
    try:
        import cv2
        img = cv2.imread(path, cv2.IMREAD_GRAYSCALE)
        return None if img is None else np.ascontiguousarray(img, np.uint8)
    except ImportError:
        from PIL import Image
        try:
            return np.ascontiguousarray(np.asarray(Image.open(path).convert("L")), np.uint8)
        except OSError:
            return None


def disparity_view(d: np.ndarray, left: np.ndarray) -> np.ndarray:
    """The reference console's 8-bit view of a map (FasterStereoConsole.cpp:259-281)."""
    valid = d != INVALID
    out = np.zeros(d.shape, np.uint8)
    if valid.any():
        lo, hi = np.float32(d[valid].min()), np.float32(d[valid].max())
        scale = (d - lo) / (hi - lo) * np.float32(255) if hi > lo else np.zeros(d.shape, np.float32)
        out = np.where(valid & (left != 0), scale.astype(np.uint8, casting="unsafe"), 0).astype(np.uint8)
    return out


def write_pfm(path: str, d: np.ndarray) -> None:
    """Portable float map, grey, little endian, rows stored bottom to top."""
    with open(path, "wb") as f:
        f.write(b"Pf\n%d %d\n-1.0\n" % (d.shape[1], d.shape[0]))
        f.write(np.ascontiguousarray(d[::-1], "<f4").tobytes())


def read_pfm(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        assert f.readline().strip() == b"Pf"
        w, h = (int(v) for v in f.readline().split())
        scale = float(f.readline())
        d = np.frombuffer(f.read(), "<f4" if scale < 0 else ">f4").reshape(h, w)
    return np.ascontiguousarray(d[::-1], np.float32)


def write_png(path: str, img: np.ndarray) -> None:
    try:
        import cv2
        cv2.imwrite(path, img)
    except ImportError:
        from PIL import Image
        Image.fromarray(img).save(path)


class _Pinned:
    """A page-locked host array (FasterStereoCuda::MallocPageLockedPtr, as the console uses them)."""

    def __init__(self, shape, dtype):
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        self.ptr = FasterStereoCuda.MallocPageLockedPtr(n)
        self.array = np.ctypeslib.as_array((C.c_uint8 * n).from_address(self.ptr)).view(dtype).reshape(shape)

    def free(self):
        if self.ptr:
            FasterStereoCuda.FreePageLockedPtr(self.ptr)
            self.ptr = 0


def load_pairs(a) -> tuple[list, list, list]:
    if a.mode == "S":
        names = [os.path.splitext(os.path.basename(a.left))[0]]
        return [read_grey(a.left)], [read_grey(a.right)], names
    lefts = sorted(glob.glob(os.path.join(a.left, "*." + a.ext)))
    rights = sorted(glob.glob(os.path.join(a.right, "*." + a.ext)))
    names = [os.path.splitext(os.path.basename(p))[0] for p in lefts]
    return [read_grey(p) for p in lefts], [read_grey(p) for p in rights], names


def parse(argv):
    if len(argv) == 1 and argv[0] == "opt":
        return argparse.Namespace(mode="opt")
    ap = argparse.ArgumentParser(prog="python -m fasterstereocuda_b200.console", description=__doc__.split("\n\n")[0])
    ap.add_argument("paths", nargs="+", help="LEFT RIGHT OPTION.xml | LEFT_DIR RIGHT_DIR EXT OPTION.xml")
    ap.add_argument("--frames", type=int, default=0, help="matches to run (default: every pair once)")
    ap.add_argument("--out", default="", help="folder for the maps of the pairs (.pfm float map, .png 8-bit view)")
    a = ap.parse_args(argv)
    if len(a.paths) == 3:
        a.left, a.right, a.option = a.paths
        a.mode = "S"
    elif len(a.paths) == 4:
        a.left, a.right, a.ext, a.option = a.paths
        a.mode = "M"
    else:
        print("insufficient parameters!" if len(a.paths) < 3 else "parameter type error!")
        return None
    return a


def main(argv=None) -> int:
    a = parse(sys.argv[1:] if argv is None else argv)
    if a is None:
        return 1
    om = OptionManager()
    if a.mode == "opt":  # mode 3: default option files (FasterStereoConsole.cpp:121-129)
        om.Load("option.xml", StereoOption1())
        om.Load("option2.xml", StereoOption2())
        print("initialize parameter file of algorithm done!")
        return 0
    kind = om.GaussType(a.option)
    if kind == OptionManager.OPTION_1:
        opt = StereoOption1()
    elif kind == OptionManager.OPTION_2:
        opt = StereoOption2()
    else:
        print("loading parameters of algorithm failed!")
        return 1
    if not om.Load(a.option, opt):
        print("loading parameters of algorithm failed!")
        return 1
    lefts, rights, names = load_pairs(a)
    if not lefts or len(lefts) != len(rights) or any(x is None for x in lefts + rights):
        print("data error!")
        return 1
    height, width = lefts[0].shape
    if any(x.shape != (height, width) for x in lefts + rights):
        print("data error!")
        return 1
    # the images decide the size, as in the reference (width = cols, height = rows)
    opt.width, opt.height = width, height
    load_library()
    stereo = FasterStereoCuda()
    ok = stereo.Init(opt) if kind == OptionManager.OPTION_1 else stereo.Init2(opt)
    if not ok:
        print(f"initialize algorithm failed! {stereo.last_error()}")
        return 1
    print("initialize algorithm done!")
    img_l, img_r, d_data = (_Pinned((height, width), np.uint8), _Pinned((height, width), np.uint8),
                            _Pinned((height, width), np.float32))
    frames = a.frames if a.frames > 0 else len(lefts)
    if a.out:
        os.makedirs(a.out, exist_ok=True)
    time_all = time_first = 0.0
    try:
        for count in range(frames):
            i = count % len(lefts)
            img_l.array[:] = lefts[i]
            img_r.array[:] = rights[i]
            t = time.perf_counter()
            if kind == OptionManager.OPTION_1:
                ok = stereo.Match(img_l.array, img_r.array, d_data.array)
            else:
                ok = stereo.Match2(img_l.array, img_r.array, d_data.array)
            ms = (time.perf_counter() - t) * 1e3
            if not ok:
                print(f"matching failed! {stereo.last_error()}")
                return 1
            time_all += ms
            if count == 0:
                time_first = ms
            avg = (time_all - time_first) / count if count > 0 else ms
            fps = int(1000.0 / avg * 100 + 0.5) / 100.0
            print("frame %d, timing: %6.4f ms fps = %6.4f" % (i, ms, fps), flush=True)
            if a.out and count >= frames - len(lefts):  # the last match of each pair
                d = d_data.array.copy()
                write_pfm(os.path.join(a.out, names[i] + ".pfm"), d)
                write_png(os.path.join(a.out, names[i] + ".png"), disparity_view(d, lefts[i]))
    finally:
        stereo.Release()
        for p in (img_l, img_r, d_data):
            p.free()
    return 0


if __name__ == "__main__":
    sys.exit(main())
