"""Builds the engine's shared library for sm_100a (and the oracle, for the tests).

    python -m fasterstereocuda_b200.build            # engine + oracle
    python -m fasterstereocuda_b200.build --engine   # engine only

The engine library lands in fasterstereocuda_b200/_lib/libsgmb200.so (in-tree, so it ships
with the repository snapshot). The oracle (test infrastructure) lands in oracle/_build/.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "_lib"
ENGINE_LIB = LIB_DIR / "libsgmb200.so"
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "_build" / "liborc.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
ENGINE_SOURCES = ["sgm_engine.cu", "stereo_cuda.cpp", "sgm_noalloc.cu", "float_sgm.cu", "sgm_batch.cu"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def build_engine(force: bool = False, verbose: bool = False) -> Path:
    sources = [CSRC / s for s in ENGINE_SOURCES if (CSRC / s).exists()]
    deps = sources + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    if not force and not _stale(ENGINE_LIB, deps):
        return ENGINE_LIB
    LIB_DIR.mkdir(exist_ok=True)
    objs, cmds = [], []
    for src in sources:
        obj = LIB_DIR / (src.stem + ".o")
        cmd = [_nvcc(), "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
               "-I", str(ROOT / "include"), "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cpp":
            cmd[1:1] = ["-x", "cu"]
        if verbose:
            cmd.append("-Xptxas=-v")
        cmds.append(cmd)
        objs.append(str(obj))
    # the translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c), cmds)):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    tmp = ENGINE_LIB.with_suffix(".so.tmp")
    subprocess.run([_nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"], check=True)
    os.replace(tmp, ENGINE_LIB)
    for o in objs:
        os.remove(o)
    return ENGINE_LIB


def build_oracle(force: bool = False) -> Path:
    src = ORACLE_DIR / "sgm_oracle.c"
    deps = [src, ORACLE_DIR / "sgm_oracle.h"]
    if not force and not _stale(ORACLE_LIB, deps):
        return ORACLE_LIB
    ORACLE_LIB.parent.mkdir(exist_ok=True)
    tmp = ORACLE_LIB.with_suffix(".so.tmp")
    subprocess.run(["gcc", "-std=c11", "-O3", "-march=x86-64-v3", "-mtune=generic", "-fopenmp", "-ffp-contract=off",
                    "-fPIC", "-shared", "-Wall", "-o", str(tmp), str(src), "-lm"], check=True)
    os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--engine", action="store_true")
    ap.add_argument("--oracle", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    both = not (a.engine or a.oracle)
    if a.engine or both:
        print(build_engine(a.force, a.verbose))
    if a.oracle or both:
        print(build_oracle(a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
