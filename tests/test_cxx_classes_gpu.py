"""The C++ drop-in classes on a GPU: a program compiled against include/StereoCuda.h and
include/FasterStereoCuda.h (the reference's class interfaces, SgmStereoCuda/StereoCuda.h:14-100 and
FasterStereoCuda/FasterStereoCuda.h:24-127) and linked with libsgmb200.so runs Init / Match /
Init2 / Match2 / Release of both classes on host buffers, the way the reference's console calls
them. Every map it writes is compared bit for bit with the oracle."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from fasterstereocuda_b200 import scenes

ROOT = Path(__file__).resolve().parent.parent
CAM = (600.0, 180.0, 610.0, 180.0, 720.0, 540.0)  # x0_left, y0_left, x0_right, y0_right, focus, baseline

CALLER = r"""
#include <cstdio>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>
#include "FasterStereoCuda.h"
#include "StereoCuda.h"

static std::vector<unsigned char> read_bytes(const char* path, size_t n) {
  std::vector<unsigned char> v(n);
  FILE* f = std::fopen(path, "rb");
  if (!f || std::fread(v.data(), 1, n, f) != n) std::exit(10);
  std::fclose(f);
  return v;
}
static void write_floats(const char* path, const std::vector<float>& v) {
  FILE* f = std::fopen(path, "wb");
  if (!f || std::fwrite(v.data(), sizeof(float), v.size(), f) != v.size()) std::exit(11);
  std::fclose(f);
}

int main(int argc, char** argv) {
  if (argc != 5) return 2;
  const int w = std::atoi(argv[1]), h = std::atoi(argv[2]);
  const std::string dir = argv[3];
  const int layers = std::atoi(argv[4]);
  const size_t n = (size_t)w * h;
  std::vector<unsigned char> L = read_bytes((dir + "/left.bin").c_str(), n);
  std::vector<unsigned char> R = read_bytes((dir + "/right.bin").c_str(), n);
  std::vector<float> a(n), b(n);

  // single level: census 9x7, P1 10, P2 150, LR check, median, small-region removal
  CuSGMOption opt;
  opt.p1 = 10; opt.p2_init = 150; opt.cs_type = CuSGMOption::CS_9x7; opt.num_paths = 4;
  opt.do_median_filter = true; opt.do_lr_check = true; opt.lr_threshold = 1.0f; opt.unique_threshold = 0.95f;
  opt.using_constant_p2 = true; opt.do_remove_peaks = true; opt.peaks_ratio_threshold = 0.0005f;
  {
    StereoCuda s;
    if (!s.Init(w, h, 0, 64, opt)) return 3;
    if (s.GetDispartyRange() != 64) return 4;
    if (!s.Match(L.data(), R.data(), a.data(), b.data())) return 5;
    write_floats((dir + "/disp_l.bin").c_str(), a);
    write_floats((dir + "/disp_r.bin").c_str(), b);
    s.Release();
    CamParam_T cam;
    cam.x0_left = %(x0l)r; cam.y0_left = %(y0l)r; cam.x0_right = %(x0r)r; cam.y0_right = %(y0r)r;
    cam.focus = %(f)r; cam.baseline = %(b)r;
    if (!s.Init2(w, h, 0, 64, opt, cam)) return 6;
    if (!s.Match2(L.data(), R.data(), a.data())) return 7;
    write_floats((dir + "/depth.bin").c_str(), a);
    s.Release();
    if (s.Match(L.data(), R.data(), a.data())) return 8;  // released: refused
  }
  // pyramid with the reference's own per-level parameters
  {
    FasterStereoCuda p;
    FasterStereoCuda::StereoOption1 o1;
    o1.width = w; o1.height = h; o1.min_disp = 0; o1.max_disp = 64; o1.num_layers = layers;
    if (!p.Init(o1)) return 9;
    if (!p.Match(L.data(), R.data(), a.data())) return 12;
    write_floats((dir + "/pyr.bin").c_str(), a);
    p.Release();
    FasterStereoCuda::StereoOption2 o2;
    o2.width = w; o2.height = h; o2.min_depth = 5000.0f; o2.max_depth = 60000.0f; o2.num_layers = layers;
    o2.epi.x0_left = %(x0l)r; o2.epi.y0_left = %(y0l)r; o2.epi.x0_right = %(x0r)r; o2.epi.y0_right = %(y0r)r;
    o2.epi.baseline = %(b)r; o2.epi.focus = %(f)r;
    if (!p.Init2(o2)) return 13;
    if (!p.Match2(L.data(), R.data(), a.data())) return 14;
    write_floats((dir + "/pyr_depth.bin").c_str(), a);
  }
  std::printf("%%u\n", std::thread::hardware_concurrency());
  return 0;
}
""" % dict(x0l=CAM[0], y0l=CAM[1], x0r=CAM[2], y0r=CAM[3], f=CAM[4], b=CAM[5])


@pytest.mark.gpu
def test_cxx_classes_match_the_oracle(engine_lib, oracle_mod, tmp_path):
    O = oracle_mod
    W, H, layers = 640, 376, 3
    L, R, _ = scenes.kitti_like(71, W, H)
    L.tofile(tmp_path / "left.bin")
    R.tofile(tmp_path / "right.bin")
    libdir = ROOT / "fasterstereocuda_b200" / "_lib"
    src = tmp_path / "caller.cpp"
    src.write_text(CALLER)
    exe = tmp_path / "caller"
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-L", str(libdir),
                    "-lsgmb200", f"-Wl,-rpath,{libdir}", "-pthread", "-o", str(exe)], check=True, capture_output=True,
                   text=True)
    run = subprocess.run([str(exe), str(W), str(H), str(tmp_path), str(layers)], capture_output=True, text=True)
    assert run.returncode == 0, (run.returncode, run.stderr[-2000:])
    strips = max(1, int(run.stdout.split()[-1]) * 3 // 4)  # the classes' default strip count

    def load(name):
        return np.fromfile(tmp_path / name, np.float32).reshape(H, W)

    def same(a, b):
        neq = int((a.view(np.uint32) != b.view(np.uint32)).sum())
        assert neq == 0, neq
        return True

    cfg = O.Config(width=W, height=H, disp_range=64, do_remove_peaks=1, peaks_ratio=0.0005, peaks_strips=strips)
    want = O.match(cfg, L, R, want_right=True)
    assert same(load("disp_l.bin"), want["disp"])
    assert same(load("disp_r.bin"), want["disp_r"])
    x0l, _, x0r, _, f, b = CAM
    assert same(load("depth.bin"), O.depth_from_disp(want["disp"], x0l, x0r, f, b))
    pc = O.PyrConfig(width=W, height=H, min_disp=0, max_disp=64, num_layers=layers, override_enable=0,
                     peaks_strips=strips)
    assert same(load("pyr.bin"), O.pyr_match(pc, L, R))
    m0, d0 = O.pyr_init2_coarsest(W, layers, 5000.0, 60000.0, x0l, x0r, f, b)
    s = 2 ** (layers - 1)
    pc2 = O.PyrConfig(width=W, height=H, min_disp=m0 * s, max_disp=(m0 + d0) * s, num_layers=layers,
                      override_enable=0, peaks_strips=strips)
    assert same(load("pyr_depth.bin"), O.depth_from_disp(O.pyr_match(pc2, L, R), x0l, x0r, f, b))
    assert (load("disp_l.bin") != -999999.0).mean() > 0.3
