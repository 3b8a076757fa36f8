#!/usr/bin/env python
"""Throughput benchmark of the B200 SGM stereo engine.

Metric: stereo pairs per second at 1242x375 with a 64-disparity search, the headline
configuration (3-level pyramid with per-pixel range propagation, census 9x7, P1=10, P2=150,
left-right check, median, small-region removal). Inputs are seeded synthetic KITTI-like pairs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload pyramid|plain]

`value` is timed on the device with CUDA events over exactly K steps whose inputs already sit in
HBM, in two execution modes of the same workload, the faster one giving `value` (`config.mode`;
both are in `modes`): "streams", --streams matchers on as many CUDA streams, one step = --batch
pairs from a rotating pool of distinct pairs larger than L2; "batched_graph", one CUDA graph
launch of the batched engine per step, one step = --graph-pairs resident pairs (more than L2
holds). `e2e` is the same metric through the host-buffer API (pinned host memory, copies inside
the timed region). Under torchrun every rank runs its own matchers on its own GPU (weak scaling).
`--impl reference` times the CPU restatement of the reference's algorithm (oracle/) on the
host cores, on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
# one hardware work queue per matcher stream (the runtime's default of 8 serialises streams
# beyond the eighth); must be set before CUDA initialises
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

W_, H_, DMAX = 1242, 375, 64
LAYERS = 3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["pyramid", "plain"], default="pyramid")
    ap.add_argument("--batch", type=int, default=64, help="pairs per step")
    ap.add_argument("--streams", type=int, default=32, help="matchers (one CUDA stream each) per GPU")
    ap.add_argument("--pool", type=int, default=160, help="distinct input pairs resident in HBM")
    ap.add_argument("--graph-pairs", type=int, default=256,
                    help="pairs per launch of the batched-graph mode (0: streams only); value = the faster mode")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-extras", action="store_true", help="skip the CPU baseline and extra workloads")
    ap.add_argument("--tuning", default="", help="kernel variants row_kernel,rows_per_cta,col_kernel,cols_per_cta,"
                                                 "bt_smem,row_lanes,col_lanes (default: autotuned lane split)")
    ap.add_argument("--profile-pairs", type=int, default=16, help="pairs of the serialised per-kernel timing pass")
    ap.add_argument("--e2e-threads", type=int, default=96, help="host threads (one matcher each) of the e2e pass")
    ap.add_argument("--extra", choices=["batch_pyramid", "batch", "batch_uneven", "float_sgm", "large_pyramid"],
                    default="", help="run one extra workload alone and print its JSON (e.g. for a profiler)")
    ap.add_argument("--extra-pairs", type=int, default=64, help="pairs of the --extra batch workloads")
    ap.add_argument("--float-batch", type=int, default=4, help="pairs of the --extra float_sgm workload")
    ap.add_argument("--dry-run", action="store_true",
                    help="launch, shard and time the ranks without CUDA (gloo); for testing the launcher")
    return ap.parse_args()


# ------------------------------------------------------------------------------------ helpers
def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_pool(n_distinct, seed=100, indices=None):
    """Distinct pairs of a global pool: pair i is one of 8 scenes (i % 8), rolled by a shift drawn
    from i and flipped on every other group of 8. `indices` picks pairs of the global pool (a
    rank's shard); by default the first n_distinct."""
    from fasterstereocuda_b200 import scenes
    idx = list(range(n_distinct)) if indices is None else list(indices)
    base = {k: scenes.kitti_like(seed + k, W_, H_)[:2] for k in sorted({i % 8 for i in idx})}
    pool = []
    for i in idx:
        L, R = base[i % 8]
        dy = int(np.random.Generator(np.random.PCG64([seed, i])).integers(0, 40))
        L2, R2 = np.roll(L, dy, 0), np.roll(R, dy, 0)
        if (i // 8) % 2:
            L2, R2 = L2[::-1].copy(), R2[::-1].copy()
        pool.append((np.ascontiguousarray(L2), np.ascontiguousarray(R2)))
    return pool


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms while the timed region runs (the
    region starts once the sampler has written its first line)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            t = time.perf_counter()
            while time.perf_counter() - t < 5.0 and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.skip = os.path.getsize(self.path)  # lines written before the timed region
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        with open(self.path) as f:
            data = f.read()
        os.remove(self.path)
        timed = data[getattr(self, "skip", 0):]
        rows = [l.split(",") for l in (timed if timed.strip() else data).splitlines() if l.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i] and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def alg_bytes(kernel, W, H, D, nviews, census_bytes):
    """Algorithmic HBM bytes of one launch (minimal two-pass design: row pass writes the 16-bit
    sum of the two horizontal paths, column pass reads it once and writes the disparity)."""
    V = W * H * D
    n = W * H
    if kernel.startswith("hpaths"):
        return nviews * (2 * V + 2 * census_bytes * n)
    if kernel.startswith(("vpaths_bt", "vpaths_tb")):  # a column pass launched on its own that
        return 0                                         # stores its paths: no counterpart
    if kernel.startswith(("vpaths", "wta")):  # the pass that ends in the disparity
        return nviews * (2 * V + 4 * n)
    if kernel == "census":
        return 2 * n + 2 * census_bytes * n
    if kernel == "cost":
        return nviews * (V + 2 * census_bytes * n)
    if kernel == "lr_median":
        return 12 * n
    return 0


# DRAM bytes per voxel (W*H*D*views of the launch) measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum) at 1242x375x64, one pair per launch: the plain kernels on the
# single-level workload, the 32-disparity kernels on the pyramid's finest level; per kernel
# family: "v3" the thread-per-scanline kernels, "v4" the warp-per-scanline kernels; "batch" the
# batched pyramid's persistent kernels as its graph runs them, 32 pairs per launch, over the
# launches at both 32-disparity levels (1242x375 and 621x187).
NCU_DRAM_BYTES_PER_VOXEL = {
    "v3": {"hpaths_plain": 2.83, "vpaths_bt_plain": 1.25, "vpaths_wta_plain": 4.04, "hpaths_init": 1.07,
           "vpaths_wta_init": 3.29},
    "v4": {"hpaths_plain": 2.76, "vpaths_bt_plain": 1.22, "vpaths_wta_plain": 4.04, "hpaths_init": 1.07,
           "vpaths_bt_init": 1.06, "vpaths_tb_init": 1.06, "wta_init": 3.42},
    "batch": {"hpaths_init": 3.90, "vpaths_bt_init": 1.80, "vpaths_wta_init": 4.43},
}


def roofline_of(kprof, pairs, levels, family, hbm_peak, peak_kind, timing):
    """Roofline of the dominant kernel of a profiled pass over `pairs` pairs.

    kprof: {kernel: {"launches": n, "ms": total}} (sgm_profile_read); levels: (kind, w, h, D,
    views) of each level a pair goes through. achieved = the kernel's algorithmic bytes (per pair,
    over every level it runs at, x pairs) over its summed launch durations. The dominant kernel is
    taken among those with a counterpart in the minimal design (the bottom-to-top pass launched on
    its own has none); family(kernel) names the row of NCU_DRAM_BYTES_PER_VOXEL that gives its
    measured traffic (bytes per voxel x voxels per launch)."""
    pb, pv = {}, {}
    for k in kprof:
        mine = [(w, h, d, nv) for (kind, w, h, d, nv) in levels
                if not k.startswith(("hpaths", "vpaths", "wta")) or k.endswith(kind)]
        pb[k] = sum(alg_bytes(k, w, h, d, nv, 8) for (w, h, d, nv) in mine)
        pv[k] = sum(w * h * d * nv for (w, h, d, nv) in mine)
    cand = [k for k in kprof if pb.get(k, 0) > 0 and kprof[k]["ms"] > 0]
    if not cand:
        return None
    dom = max(cand, key=lambda k: kprof[k]["ms"])
    total_ms, nl = kprof[dom]["ms"], max(1, kprof[dom]["launches"])
    byts = pb[dom] * pairs
    ach = byts / (total_ms / 1e3) / 1e9
    bpv = NCU_DRAM_BYTES_PER_VOXEL[family(dom)].get(dom)
    return {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
            "frac": ach / hbm_peak, "traffic": bpv * pv[dom] * pairs / nl if bpv else None,
            "peak_kind": peak_kind,
            "traffic_source": "ncu DRAM bytes per voxel of this kernel x voxels per launch",
            "kernel_family": family(dom), "avg_launch_us": total_ms / nl * 1e3,
            "alg_bytes_per_launch": byts / nl, "timing": timing}


# ------------------------------------------------------------------------------------ reference arm
def run_reference(a, rank, world):
    if rank != 0:
        return 0
    from oracle import oracle as O
    O.lib()
    cores = O.max_threads()
    pool = make_pool(8)
    if a.workload == "pyramid":
        pc = O.PyrConfig(width=W_, height=H_, min_disp=0, max_disp=DMAX, num_layers=LAYERS)
        one = lambda L, R: O.pyr_match(pc, L, R)  # noqa: E731
    else:
        cfg = O.Config(width=W_, height=H_, disp_range=DMAX)
        one = lambda L, R: O.match(cfg, L, R)["disp"]  # noqa: E731
    t = time.perf_counter()
    one(*pool[0])
    per = time.perf_counter() - t
    sample = max(1, min(a.batch, int(round(1.0 / max(per, 1e-3)))))  # ~1 s of CPU work per step
    for i in range(a.warmup):
        for j in range(sample):
            one(*pool[(i * sample + j) % len(pool)])
    t = time.perf_counter()
    for i in range(a.steps):
        for j in range(sample):
            one(*pool[(i * sample + j) % len(pool)])
    dt = time.perf_counter() - t
    v = a.steps * sample / dt
    line = {"impl": "reference", "metric": metric_name(a.workload), "value": v, "unit": "pairs/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": dt / a.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8/u32", "data": "synthetic",
            "config": workload_config(a, sample),
            "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": cores, "kind": "port",
                             "sample": f"{sample} pairs per step, oracle/ C restatement, OpenMP {cores} threads"},
            "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not a.no_extras:
        line["ref_cuda_build"] = ref_cuda_build(a)
    print(json.dumps(line), flush=True)
    return 0


def ref_cuda_build(a):
    """The reference's own CUDA build (its sources compiled for sm_100a into oracle/_ref/ by
    oracle/build_ref.sh) timed through its public API with host buffers in and out, as its console
    measures itself: StereoCuda::Match on the plain workload (census 9x7, P1 10, P2 150, LR check,
    median) and FasterStereoCuda::Match on the 3-level pyramid with the reference's own per-level
    parameters, each with 1 host thread and with --streams host threads (one instance each, the
    concurrency the engine's throughput figure uses). Only 64- and 32-disparity levels run: the
    reference's 128-disparity row kernel indexes shared memory past its allocation."""
    import ctypes as C
    lib_path = ROOT / "oracle" / "_ref" / "libsgmref.so"
    if not lib_path.exists():
        return {"unavailable": "oracle/_ref/libsgmref.so not built (needs the reference sources)"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
        from tests.golden.make_golden import RefCase
        lib = C.CDLL(str(lib_path))
        vp = C.c_void_p
        lib.ref_throughput_match.argtypes = [C.POINTER(RefCase), vp, vp, C.c_int, C.c_int, C.c_int]
        lib.ref_throughput_match.restype = C.c_double
        lib.ref_throughput_pyr.argtypes = [C.c_int] * 7 + [vp, vp, C.c_int, C.c_int, C.c_int]
        lib.ref_throughput_pyr.restype = C.c_double
        L, R = make_pool(1)[0]
        plain = RefCase(width=W_, height=H_, min_disp=0, disp_range=DMAX, cs_type=1, p1=10, p2=150, uniqueness=0.95,
                        do_lr_check=1, lr_threshold=1.0, do_median=1, morphology=0, do_remove_peaks=0,
                        peaks_ratio=0.0, post_filter=0)
        T = max(1, a.streams)
        out = {"api": "StereoCuda::Match / FasterStereoCuda::Match, host buffers, one instance per host thread",
               "threads": [1, T]}
        res = {}
        for th, n in ((1, 200), (T, max(4, 400 // T))):
            res[f"plain_{th}"] = lib.ref_throughput_match(C.byref(plain), L.ctypes.data, R.ctypes.data, 3, n, th)
        for th, n in ((1, 150), (T, max(4, 300 // T))):
            res[f"pyramid_{th}"] = lib.ref_throughput_pyr(W_, H_, 0, DMAX, LAYERS, 1, 1, L.ctypes.data, R.ctypes.data,
                                                          3, n, th)
        out["plain_1242x375x64_census9x7_p10_p150_lr_median_pairs_per_s"] = {str(k.split("_")[1]): v
                                                                             for k, v in res.items()
                                                                             if k.startswith("plain")}
        out["pyramid_1242x375_3layers_reference_params_pairs_per_s"] = {str(k.split("_")[1]): v
                                                                        for k, v in res.items()
                                                                        if k.startswith("pyramid")}
        out["pyramid_params"] = "census 5x5, P1 8, P2 32 per level (SetSgmParameters, FasterStereoCuda.cpp:169-199)"
        return out
    except Exception as e:  # the CPU arm's line stands without it
        return {"unavailable": f"{type(e).__name__}: {e}"}


def metric_name(workload):
    if workload == "pyramid":
        return "pairs/s at 1242x375x64 (3-level pyramid, census 9x7, P1=10 P2=150, LR + median + peaks)"
    return "pairs/s at 1242x375x64 (single level, census 9x7, P1=10 P2=150, LR + median)"


def workload_config(a, batch):
    c = {"workload": f"{W_}x{H_} D={DMAX} " + ("3-level pyramid, slanted ground plane + 12 boxes scene" if a.workload == "pyramid"
                                                 else "single-level plain SGM"),
         "width": W_, "height": H_, "disparities": DMAX, "census": "9x7", "p1": 10, "p2": 150,
         "batch_pairs": batch}
    if a.workload == "pyramid":
        c["layers"] = LAYERS
    return c


# ------------------------------------------------------------------------------------ our arm
def run_ours(a, rank, world, local_rank):
    import torch
    import fasterstereocuda_b200 as fsc
    from fasterstereocuda_b200 import replicas

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = fsc.load_library()

    def plain_option():
        return fsc.CuSGMOption(p1=10, p2_init=150, cs_type=1, num_paths=4, do_median_filter=True, do_lr_check=True,
                               lr_threshold=1.0, unique_threshold=0.95, using_constant_p2=True)

    def make_matcher():
        if a.workload == "pyramid":
            m = fsc.FasterStereoCuda()
            ok = m.Init(fsc.StereoOption1(width=W_, height=H_, min_disp=0, max_disp=DMAX, num_layers=LAYERS,
                                          do_lr_check=True, do_rm_peaks=True), fsc.LevelOverride(1, 10, 150),
                        fsc.ExtOptions())
        else:
            m = fsc.StereoCuda()
            ok = m.Init(W_, H_, 0, DMAX, plain_option())
        if not ok:
            raise RuntimeError(f"matcher init failed: {m.last_error()}")
        if a.tuning and not m.set_tuning(fsc.Tuning(*[int(v) for v in a.tuning.split(",")])):
            raise RuntimeError(f"tuning rejected: {m.last_error()}")
        return m

    def apply_tuning(t, init_t=None, ms=None):
        """t for every level; init_t (pyramid) for the 32-disparity levels below the coarsest."""
        for m in (matchers if ms is None else ms):
            if not m.set_tuning(fsc.Tuning(*t)):
                raise RuntimeError(f"tuning rejected: {m.last_error()}")
            if init_t is not None:
                for lv in range(LAYERS - 1):
                    if not m.set_tuning(fsc.Tuning(*init_t), lv):
                        raise RuntimeError(f"tuning rejected: {m.last_error()}")

    def run_one(m, L, R, out, stream):
        if a.workload == "pyramid":
            ok = m.match_device(L, R, out, stream)
        else:
            ok = m.match_device(L, R, out, None, None, stream)
        if not ok:
            raise RuntimeError(f"match failed: {m.last_error()}")
        return m.kernel_launches()

    S = max(1, a.streams)
    matchers = [make_matcher() for _ in range(S)]
    streams = [torch.cuda.Stream(device=dev) for _ in range(S)]
    # weak scaling: the pairs of a step and the pool of distinct pairs are split over the ranks
    # (replicas.shard), every rank matching a.batch pairs per step from its own share of the pool
    pool = make_pool(0, indices=replicas.shard(a.pool * world, rank, world))
    dL = [torch.from_numpy(L).to(dev) for L, _ in pool]
    dR = [torch.from_numpy(R).to(dev) for _, R in pool]
    outs = [torch.empty((H_, W_), dtype=torch.float32, device=dev) for _ in range(a.batch)]
    pool_bytes = sum(x.numel() for x in dL) * 2
    main = torch.cuda.current_stream(dev)
    cursor = [0]

    def step():
        ev0 = torch.cuda.Event()
        ev0.record(main)
        launches = 0
        for s in streams:
            s.wait_event(ev0)
        for b in range(a.batch):
            i = cursor[0] % len(dL)
            cursor[0] += 1
            k = b % S
            launches += run_one(matchers[k], dL[i], dR[i], outs[b], streams[k].cuda_stream)
        for s in streams:
            e = torch.cuda.Event()
            e.record(s)
            main.wait_event(e)
        return launches

    def barrier():
        replicas.barrier(world)

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, world, dev)

    def graph_mode(n):
        """The same workload as one batched graph launch of n pairs per step (sgm_batch_pyr_* for the
        pyramid, sgm_batch_* for the single level), inputs resident in HBM (n pairs of the rank's
        pool, more than L2 holds), W untimed and K timed launches; pair 0 checked bit for bit
        against the per-pair matcher."""
        if a.workload == "pyramid":
            b = fsc.StereoBatchPyramid()
            ok = b.Init([(W_, H_, 0, DMAX)] * n, fsc.StereoOption1(num_layers=LAYERS, do_lr_check=True,
                                                                   do_rm_peaks=True),
                        fsc.LevelOverride(1, 10, 150), fsc.ExtOptions())
        else:
            b = fsc.StereoBatch()
            ok = b.Init([(W_, H_, 0, DMAX)] * n, plain_option())
        if not ok:
            raise RuntimeError(f"batch init failed: {b.last_error()}")
        for i in range(n):
            al, ar, _ = b.buffers(i)
            _dev_copy(al, dL[i % len(dL)])
            _dev_copy(ar, dR[i % len(dR)])
        gs = torch.cuda.Stream(device=dev)
        for _ in range(a.warmup):
            if not b.run(gs.cuda_stream):
                raise RuntimeError(f"batch run failed: {b.last_error()}")
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local_rank) as gclk:
            e0.record(gs)
            for _ in range(a.steps):
                b.run(gs.cuda_stream)
            e1.record(gs)
            torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        gms = max_over_ranks(e0.elapsed_time(e1))
        ref = torch.empty((H_, W_), dtype=torch.float32, device=dev)
        run_one(matchers[0], dL[0], dR[0], ref, main.cuda_stream)
        torch.cuda.synchronize()
        same = torch.equal(_read_dev(b.buffers(0)[2], H_, W_).view(torch.int32), ref.view(torch.int32))
        # per-kernel CUDA events of two more runs of the same batch on the same stream, its kernels
        # enqueued one after another instead of as the graph (no side branches), so that each
        # launch's duration is its own; the roofline of this mode's dominant kernel comes from here
        fsc.profile_enable(True)
        for _ in range(2):
            if not b.run(gs.cuda_stream):
                raise RuntimeError(f"batch run failed: {b.last_error()}")
        torch.cuda.synchronize()
        gprof = fsc.profile_read()
        fsc.profile_enable(False)
        info = b.info()
        del b
        torch.cuda.synchronize()
        inputs = min(n, len(dL)) * 2 * W_ * H_
        return {"value": a.steps * n * world / (gms / 1e3), "ms_per_step": gms / a.steps, "pairs_per_step": n,
                "how": f"one CUDA graph launch of {n} pairs per step ("
                       + ("sgm_batch_pyr_run" if a.workload == "pyramid" else "sgm_batch_run") + ")",
                "gpu_launches": info["kernels_per_run"] * a.steps, "kernels_per_graph": info["kernels_per_run"],
                "arena_gib": info["arena_bytes"] / 2**30, "bit_exact_vs_per_pair": bool(same),
                "l2": f"inputs larger than L2: {n} pairs ({inputs / 2**20:.0f} MiB of distinct input buffers)",
                "clocks": gclk.summary(), "profile": {"runs": 2, "pairs_per_run": n, "kernels": gprof}}

    # parity: first output vs the oracle (outside every timed region)
    bit_exact = None
    if rank == 0 and not a.no_extras:
        from oracle import oracle as O
        run_one(matchers[0], dL[0], dR[0], outs[0], main.cuda_stream)
        torch.cuda.synchronize()
        if a.workload == "pyramid":
            exp = O.pyr_match(O.PyrConfig(width=W_, height=H_, max_disp=DMAX, num_layers=LAYERS,
                                          peaks_strips=max(1, (os.cpu_count() or 1) * 3 // 4)), *pool[0])
        else:
            exp = O.match(O.Config(width=W_, height=H_, disp_range=DMAX), *pool[0])["disp"]
        bit_exact = bool(np.array_equal(outs[0].cpu().numpy().view(np.uint32), exp.view(np.uint32)))

    # autotune: the lane split of the scanline kernels that is fastest at this concurrency
    # (every split gives the same disparities); one untimed and six timed steps per candidate
    tuning = a.tuning or None
    chosen, chosen_init = None, None  # tunings applied to matchers made later
    if not a.tuning:
        def timed(t, init_t=None):
            apply_tuning(t, init_t)
            step()
            torch.cuda.synchronize()
            t0c = time.perf_counter()
            for _ in range(6):
                step()
            torch.cuda.synchronize()
            return max_over_ranks(time.perf_counter() - t0c)
        # the thread-per-scanline kernels with each lane split, and the warp-per-scanline kernels
        cands = [(0, 0, 0, 0, 0) + lanes for lanes in ((8, 8), (8, 4), (4, 4), (4, 2), (2, 2))]
        cands.append((4, 0, 4, 0, 0, 0, 0))
        best = min(((timed(t), t) for t in cands), key=lambda r: r[0])
        chosen = best[1]
        tuning = "autotuned " + ",".join(str(v) for v in chosen)
        if a.workload == "pyramid":  # then the 32-disparity levels on their own
            best_i = min(((timed(chosen, t), t) for t in ((0, 0, 0, 0, 0, 8, 8), (0, 0, 0, 0, 0, 4, 4),
                                                            (0, 0, 0, 0, 0, 2, 2), (4, 0, 4, 0, 0, 0, 0))),
                         key=lambda r: r[0])
            if best_i[0] < best[0]:
                chosen_init = best_i[1]
                tuning += "; 32-disparity levels " + ",".join(str(v) for v in best_i[1])
        apply_tuning(chosen, chosen_init)
    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    with ClockSampler(local_rank) as clk:
        t0.record(main)
        for _ in range(a.steps):
            launches += step()
        t1.record(main)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(t0.elapsed_time(t1))
    value = a.steps * a.batch * world / (ms / 1e3)
    clk_summary = clk.summary()
    modes = {"streams": {"value": value, "ms_per_step": ms / a.steps, "pairs_per_step": a.batch,
                         "how": f"{S} matchers on {S} streams, {a.batch} pairs per step", "tuning": tuning,
                         "gpu_launches": launches, "clocks": clk_summary}}
    mode = "streams"
    if a.graph_pairs > 0:
        g = graph_mode(a.graph_pairs)
        modes["batched_graph"] = g
        if g["value"] > value:  # the faster execution mode of the same workload gives `value`
            mode = "batched_graph"
            value, ms, launches, clk_summary = g["value"], g["ms_per_step"] * a.steps, g["gpu_launches"], g["clocks"]

    # single-pair latency: one matcher alone on the GPU, one pair at a time, CUDA events around
    # each pair. Few scanlines in flight favour more lanes per scanline, so the lane split is tuned
    # for this case on its own (every split gives the same disparities).
    lat_m = make_matcher()
    lat_s = torch.cuda.Stream(device=dev)  # a stream of its own: the events must see the matcher's work

    def pair_ms(n):
        ts = []
        for j in range(n):
            i = j % len(dL)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(lat_s)
            run_one(lat_m, dL[i], dR[i], outs[0], lat_s.cuda_stream)
            e1.record(lat_s)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)
    lat_tuning = a.tuning or None
    if not a.tuning:
        # kernel variants (row_kernel, rows_per_cta, col_kernel, cols_per_cta, bt_smem, row_lanes,
        # col_lanes); variant 4 (one warp per scanline, bulk-copied chunks) runs at the 32-disparity
        # levels, the default elsewhere
        cands = {}
        for t in ((0, 0, 0, 0, 0, 8, 8), (0, 0, 0, 0, 0, 8, 4), (4, 0, 4, 0, 0, 8, 8), (4, 0, 3, 0, 0, 8, 8),
                  (3, 0, 4, 0, 0, 8, 8), (2, 1, 2, 1, 0, 8, 8)):
            apply_tuning(t, ms=[lat_m])
            pair_ms(3)
            cands[t] = pair_ms(8)
        best_t = min(cands, key=cands.get)
        apply_tuning(best_t, ms=[lat_m])
        lat_tuning = "tuning " + ",".join(str(v) for v in best_t)
    pair_ms(3)
    latency = {"ms_per_pair": pair_ms(20), "tuning": lat_tuning,
               "how": "one matcher, one stream, one pair at a time, inputs in HBM, CUDA events around each "
                      "match_device call (median of 20)"}

    # per-kernel CUDA events over a serialised pass (the latency matcher, one stream, one pair at a
    # time), so each launch's duration is its own: the roofline of the dominant kernel comes from here
    fsc.profile_enable(True)
    for j in range(a.profile_pairs):
        i = j % len(dL)
        run_one(lat_m, dL[i], dR[i], outs[0], lat_s.cuda_stream)
    torch.cuda.synchronize()
    prof = fsc.profile_read()
    fsc.profile_enable(False)
    latency["kernel_ms_per_pair"] = sum(v["ms"] for v in prof.values()) / max(1, a.profile_pairs)

    # e2e: the host-buffer API (synchronous Match, like the reference's), pinned host memory, one
    # host thread per matcher (the reference API is per object; ctypes releases the GIL)
    # each host thread matches its share of e2e_steps * batch pairs in one loop
    from concurrent.futures import ThreadPoolExecutor
    e2e_steps = max(1, min(a.steps, 5))
    E = max(S, a.e2e_threads)
    e2e_matchers = matchers + [make_matcher() for _ in range(E - S)]
    if chosen is not None:
        apply_tuning(chosen, chosen_init, e2e_matchers[S:])
    hostL = [torch.from_numpy(L).pin_memory().numpy() for L, _ in pool[:a.batch]]
    hostR = [torch.from_numpy(R).pin_memory().numpy() for _, R in pool[:a.batch]]
    hostO = [[torch.empty((H_, W_), dtype=torch.float32).pin_memory().numpy() for _ in range(2)] for _ in range(E)]
    total_pairs = e2e_steps * a.batch

    def host_worker(k, count):
        m = e2e_matchers[k]
        for j, b in enumerate(range(k, count, E)):
            i = b % len(hostL)
            if not m.Match(hostL[i], hostR[i], hostO[k][j % 2]):
                raise RuntimeError(m.last_error())

    with ThreadPoolExecutor(max_workers=E) as ex:
        list(ex.map(lambda k: host_worker(k, 2 * E), range(E)))  # warm-up (direct run, graph capture)
        barrier()
        te = time.perf_counter()
        list(ex.map(lambda k: host_worker(k, total_pairs), range(E)))
        te = max_over_ranks(time.perf_counter() - te)
    e2e_value = total_pairs * world / te

    if rank != 0:
        return 0
    hbm_peak, peak_kind = peaks()
    # (kind, w, h, D, views) of each level a pair goes through
    levels = []
    if a.workload == "pyramid":
        for lv in range(LAYERS):
            w, h, mn, d = matchers[0].level_info(lv)
            levels.append(("plain", w, h, d, 2) if lv == LAYERS - 1 else ("init", w, h, d, 1))
    else:
        levels.append(("plain", W_, H_, DMAX, 2))

    # kernel family of the latency matcher's row / column scans
    lat_t = [int(v) for v in lat_tuning.split()[-1].split(",")] if lat_tuning else [0, 0, 0]
    fam = lambda k: "v4" if (lat_t[0] if k.startswith("hpaths") else lat_t[2]) == 4 else "v3"  # noqa: E731
    calls = a.profile_pairs
    roofline_single = roofline_of(prof, calls, levels, fam, hbm_peak, peak_kind,
                                  f"CUDA events around each launch, serialised pass of {calls} pairs on one "
                                  f"stream (the single-pair latency matcher)")
    latency["roofline"] = roofline_single
    roofline = roofline_single
    if mode == "batched_graph":
        gp = modes["batched_graph"]["profile"]
        roofline = roofline_of(gp["kernels"], gp["runs"] * gp["pairs_per_run"], levels, lambda k: "batch",
                               hbm_peak, peak_kind,
                               f"CUDA events around each launch of {gp['runs']} runs of the timed batch "
                               f"({gp['pairs_per_run']} pairs per launch), its kernels enqueued one after "
                               f"another on the timed stream")
    if roofline is not None:
        # the path is integer-ALU bound: algorithmic int ops per view 34*W*H*D + 248*W*H (xor+popc,
        # 7 per path step x 4 paths, 3 adds, 1 min per voxel; census per pixel), over all levels,
        # against the nominal INT32 rate of the measured SM clock (148 SMs x 128 lanes)
        ops = sum(nv * (34 * w * h * d + 248 * w * h) for (kind, w, h, d, nv) in levels)
        clk = (clk_summary or {}).get("sm_mhz") or 1965.0
        peak = 148 * 128 * clk * 1e6
        # the scans execute their recurrence on packed 16x2 words (two disparities per
        # instruction): frac_packed16x2 is against twice the INT32 rate
        roofline["alu"] = {"ops_alg_per_pair": ops, "achieved_tops": ops * value / 1e12 / world,
                           "int32_peak_tops": peak / 1e12, "frac": ops * value / world / peak,
                           "frac_packed16x2": ops * value / world / (2 * peak),
                           "peak_kind": "nominal: 148 SMs x 128 INT32 lanes x median SM clock under load",
                           "per": "GPU"}
    def shares(kprof):
        tot = sum(x["ms"] for x in kprof.values()) or 1.0
        return {k: {"launches": v["launches"], "avg_us": round(v["ms"] / max(1, v["launches"]) * 1e3, 2),
                    "share": round(v["ms"] / tot, 4)} for k, v in kprof.items()}
    # per-kernel launches, average duration and share of the profiled pass of value's mode
    latency["kernels"] = shares(prof)
    kernels = shares(modes["batched_graph"]["profile"]["kernels"]) if mode == "batched_graph" else latency["kernels"]

    cpu = None
    extras = None
    if not a.no_extras:
        cpu = cpu_baseline(a, pool)
        extras = {"equal_concurrency": equal_concurrency(pool[:8], max(1, a.streams))}
        extras.update(extra_batches(pool))
        extras["float_sgm"] = extra_float_sgm()
        extras["large_pyramid"] = extra_large_pyramid()
    clocks = clk_summary
    line = {"metric": metric_name(a.workload), "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8/u32 (f32 subpixel)",
            "data": "synthetic seeded KITTI-like pairs",
            "config": (dict(workload_config(a, a.batch), mode="streams", streams=S, tuning=tuning,
                            l2=f"inputs larger than L2: rotating pool of {len(dL)} distinct pairs "
                               f"({pool_bytes / 2**20:.0f} MiB) per GPU")
                       if mode == "streams" else
                       dict(workload_config(a, a.graph_pairs), mode="batched_graph", l2=modes[mode]["l2"])),
            "modes": modes,
            "e2e": {"value": e2e_value, "unit": "pairs/s",
                    "h2d_bytes_per_step": a.batch * 2 * W_ * H_, "d2h_bytes_per_step": a.batch * 4 * W_ * H_,
                    "api": ("FasterStereoCuda.Match" if a.workload == "pyramid" else "StereoCuda.Match")
                    + f" (host buffers, synchronous), {E} host threads with one matcher each"},
            "latency": latency, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
            "gpu_launches": launches,
            "bit_exact_vs_oracle": bit_exact, "kernels": kernels, "extras": extras}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------ extras
def equal_concurrency(pairs, T):
    """The engine through the same host-buffer calls and at the same concurrency as the reference
    arm's timing of the reference CUDA build: StereoCuda.Match on the plain workload (census 9x7,
    P1 10, P2 150, LR check, median) and FasterStereoCuda.Match on the 3-level pyramid with the
    reference's own per-level parameters (no override), with 1 host thread and with T host threads,
    one matcher each, pinned host buffers."""
    import torch
    import fasterstereocuda_b200 as fsc
    from concurrent.futures import ThreadPoolExecutor

    def make(kind):
        if kind == "plain":
            m = fsc.StereoCuda()
            ok = m.Init(W_, H_, 0, DMAX, fsc.CuSGMOption(p1=10, p2_init=150, cs_type=1, num_paths=4,
                                                          do_median_filter=True, do_lr_check=True,
                                                          lr_threshold=1.0, unique_threshold=0.95,
                                                          using_constant_p2=True))
        else:
            m = fsc.FasterStereoCuda()
            ok = m.Init(fsc.StereoOption1(width=W_, height=H_, min_disp=0, max_disp=DMAX, num_layers=LAYERS,
                                          do_lr_check=True, do_rm_peaks=True))
        if not ok:
            raise RuntimeError(m.last_error())
        return m

    hl = [torch.from_numpy(L).pin_memory().numpy() for L, _ in pairs]
    hr = [torch.from_numpy(R).pin_memory().numpy() for _, R in pairs]
    out = {"api": "StereoCuda.Match / FasterStereoCuda.Match, host buffers, one matcher per host thread",
           "threads": [1, T]}
    for kind, key in (("plain", "plain_1242x375x64_census9x7_p10_p150_lr_median_pairs_per_s"),
                      ("pyramid", "pyramid_1242x375_3layers_reference_params_pairs_per_s")):
        rates = {}
        for th in (1, T):
            ms = [make(kind) for _ in range(th)]
            outs = [torch.empty((H_, W_), dtype=torch.float32).pin_memory().numpy() for _ in range(th)]
            n = max(8, (400 if kind == "plain" else 300) // th)

            def work(k, count):
                for j in range(count):
                    i = (k + j) % len(hl)
                    if not ms[k].Match(hl[i], hr[i], outs[k]):
                        raise RuntimeError(ms[k].last_error())
            with ThreadPoolExecutor(max_workers=th) as ex:
                list(ex.map(lambda k: work(k, 3), range(th)))
                t = time.perf_counter()
                list(ex.map(lambda k: work(k, n), range(th)))
                rates[str(th)] = th * n / (time.perf_counter() - t)
            del ms
        out[key] = rates
    return out


def _dev_copy(dst_addr, src_tensor):
    from cuda.bindings import runtime as rt
    (err,) = rt.cudaMemcpy(dst_addr, src_tensor.data_ptr(), src_tensor.numel() * src_tensor.element_size(),
                           rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
    if err != rt.cudaError_t.cudaSuccess:
        raise RuntimeError(f"cudaMemcpy failed: {err}")


def _read_dev(addr, h, w):
    import torch
    from cuda.bindings import runtime as rt
    out = torch.empty((h, w), dtype=torch.float32, device="cuda")
    (err,) = rt.cudaMemcpy(out.data_ptr(), addr, h * w * 4, rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
    if err != rt.cudaError_t.cudaSuccess:
        raise RuntimeError(f"cudaMemcpy failed: {err}")
    return out


def batch_vs_loop(pairs, images, runs, warmup):
    """One batch graph over `pairs` vs a loop of per-pair StereoCuda.match_device calls on one
    stream (the plain path), same inputs resident in HBM, device-timed; outputs compared bit for bit."""
    import torch
    import fasterstereocuda_b200 as fsc
    opt = fsc.CuSGMOption(p1=10, p2_init=150, cs_type=1, num_paths=4, do_median_filter=True, do_lr_check=True,
                          lr_threshold=1.0, unique_threshold=0.95, using_constant_p2=True)
    b = fsc.StereoBatch()
    t = time.perf_counter()
    if not b.Init(pairs, opt):
        raise RuntimeError(b.last_error())
    init_s = time.perf_counter() - t
    dev = [(torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()) for L, R in images]
    for i, (dl, dr) in enumerate(dev):
        al, ar, _ = b.buffers(i)
        _dev_copy(al, dl)
        _dev_copy(ar, dr)
    torch.cuda.synchronize()
    main = torch.cuda.Stream()  # a real stream handle: NULL would mean the batch's own stream
    for _ in range(warmup):
        b.run(main.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(main)
    for _ in range(runs):
        b.run(main.cuda_stream)
    e1.record(main)
    torch.cuda.synchronize()
    batch_ms = e0.elapsed_time(e1) / runs
    # plain per-pair loop: one matcher per distinct shape, pairs matched one after another
    engines, outs = {}, []
    for (w, h, m, d) in pairs:
        if (w, h, m, d) not in engines:
            s = fsc.StereoCuda()
            if not s.Init(w, h, m, d, opt):
                raise RuntimeError(s.last_error())
            engines[(w, h, m, d)] = s
        outs.append(torch.empty((h, w), dtype=torch.float32, device="cuda"))

    def loop():
        for i, p in enumerate(pairs):
            if not engines[p].match_device(dev[i][0], dev[i][1], outs[i], None, None, main.cuda_stream):
                raise RuntimeError(engines[p].last_error())
    for _ in range(warmup):
        loop()
    torch.cuda.synchronize()
    e0.record(main)
    for _ in range(runs):
        loop()
    e1.record(main)
    torch.cuda.synchronize()
    loop_ms = e0.elapsed_time(e1) / runs
    same = all(torch.equal(_read_dev(b.buffers(i)[2], p[1], p[0]).view(torch.int32), outs[i].view(torch.int32))
               for i, p in enumerate(pairs))
    info = b.info()
    return {"pairs": len(pairs), "batch_pairs_per_s": len(pairs) / (batch_ms / 1e3),
            "loop_pairs_per_s": len(pairs) / (loop_ms / 1e3), "speedup": loop_ms / batch_ms,
            "batch_ms": batch_ms, "loop_ms": loop_ms, "bit_exact_vs_per_pair": bool(same),
            "kernels_per_graph": info["kernels_per_run"], "arena_gib": info["arena_bytes"] / 2**30,
            "init_s": init_s, "buckets": b.buckets()}


def batch_pyramid_vs_loop(images, runs, warmup, streams=None):
    """64 pyramid pairs (1242x375, disparities 0..64, 3 layers, census 9x7, P1=10, P2=150, LR +
    median + removal) as one graph launch vs a loop of FasterStereoCuda.match_device on one
    stream; outputs compared bit for bit."""
    import torch
    import fasterstereocuda_b200 as fsc
    n = len(images)
    opt = fsc.StereoOption1(num_layers=LAYERS, do_lr_check=True, do_rm_peaks=True)
    ov = fsc.LevelOverride(1, 10, 150)
    b = fsc.StereoBatchPyramid()
    t = time.perf_counter()
    if not b.Init([(W_, H_, 0, DMAX)] * n, opt, ov, fsc.ExtOptions()):
        raise RuntimeError(b.last_error())
    init_s = time.perf_counter() - t
    dev = [(torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()) for L, R in images]
    for i, (dl, dr) in enumerate(dev):
        al, ar, _ = b.buffers(i)
        _dev_copy(al, dl)
        _dev_copy(ar, dr)
    torch.cuda.synchronize()
    main = torch.cuda.Stream()
    for _ in range(warmup):
        b.run(main.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(main)
    for _ in range(runs):
        b.run(main.cuda_stream)
    e1.record(main)
    torch.cuda.synchronize()
    batch_ms = e0.elapsed_time(e1) / runs
    m = fsc.FasterStereoCuda()
    if not m.Init(fsc.StereoOption1(width=W_, height=H_, min_disp=0, max_disp=DMAX, num_layers=LAYERS,
                                    do_lr_check=True, do_rm_peaks=True), ov, fsc.ExtOptions()):
        raise RuntimeError(m.last_error())
    outs = [torch.empty((H_, W_), dtype=torch.float32, device="cuda") for _ in range(n)]

    def loop():
        for i in range(n):
            if not m.match_device(dev[i][0], dev[i][1], outs[i], main.cuda_stream):
                raise RuntimeError(m.last_error())
    for _ in range(warmup):
        loop()
    torch.cuda.synchronize()
    e0.record(main)
    for _ in range(runs):
        loop()
    e1.record(main)
    torch.cuda.synchronize()
    loop_ms = e0.elapsed_time(e1) / runs
    same = all(torch.equal(_read_dev(b.buffers(i)[2], H_, W_).view(torch.int32), outs[i].view(torch.int32))
               for i in range(n))
    info = b.info()
    return {"pairs": n, "batch_pairs_per_s": n / (batch_ms / 1e3), "loop_pairs_per_s": n / (loop_ms / 1e3),
            "speedup": loop_ms / batch_ms, "batch_ms": batch_ms, "loop_ms": loop_ms, "bit_exact_vs_per_pair": bool(same),
            "kernels_per_graph": info["kernels_per_run"], "arena_gib": info["arena_bytes"] / 2**30, "init_s": init_s}


def extra_batches(pool):
    from fasterstereocuda_b200 import scenes
    out = {}
    n = 32
    out["batch_1242x375x64"] = batch_vs_loop([(W_, H_, 0, DMAX)] * n, [pool[i % len(pool)] for i in range(n)],
                                             runs=5, warmup=2)
    specs = scenes.batch_specs()
    imgs = [scenes.planar_pair(seed, w, h, dmin=2.0, dmax=60.0)[:2] for (w, h, d, seed) in specs]
    out["batch64_uneven"] = batch_vs_loop([(w, h, 0, d) for (w, h, d, _) in specs], imgs, runs=3, warmup=1)
    out["batch_pyramid_1242x375x64"] = batch_pyramid_vs_loop([pool[i % len(pool)] for i in range(64)], runs=5,
                                                             warmup=2)
    out["batch64_uneven"]["workload"] = ("64 pairs, widths 320..1920, heights 240..1080 (multiples of 32), "
                                         "D in {64,128}, seeded planar scenes, census 9x7, LR + median")
    return out


def extra_float_sgm(B=4):
    """Differentiable float32 SGM: forward + backward of B x 1242x375 x 64 (device-timed)."""
    import torch
    from fasterstereocuda_b200.float_sgm import float_sgm
    H, W, D = H_, W_, DMAX
    g = torch.Generator(device="cuda").manual_seed(0)
    cost = (torch.randint(0, 64, (B, H, W, D), generator=g, device="cuda").float()
            + torch.rand((B, H, W, D), generator=g, device="cuda") * 0.5).requires_grad_()
    p1 = torch.full((B, H, W), 10.0, device="cuda", requires_grad=True)
    p2 = torch.full((B, H, W), 150.0, device="cuda", requires_grad=True)
    w = torch.randn((B, H, W), generator=g, device="cuda")

    def step():
        cost.grad = p1.grad = p2.grad = None
        (float_sgm(cost, p1, p2) * w).sum().backward()
    for _ in range(3):
        step()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    torch.cuda.synchronize()
    n = 5
    e0.record()
    for _ in range(n):
        step()
    e1.record()
    torch.cuda.synchronize()
    fwd = []
    with torch.no_grad():
        for _ in range(n):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            float_sgm(cost, p1, p2)
            b.record()
            torch.cuda.synchronize()
            fwd.append(a.elapsed_time(b))
    ms = e0.elapsed_time(e1) / n
    # algorithmic bytes of one forward + backward: the cost volume read and its gradient written
    # (4 B per voxel each), the penalty maps read and their gradients written, disparity and its
    # gradient (4 B per pixel each)
    vox, pix = B * H * W * D, B * H * W
    alg = 8 * vox + 4 * 6 * pix
    peak, src = peaks()
    return {"workload": f"float32 SGM {B} x 1242x375, D=64, 4 paths + soft-argmin", "fwd_bwd_ms": ms,
            "fwd_ms": statistics.median(fwd),
            "roofline": {"bound": "latency: each row scan is a chain of 1242 dependent steps",
                         "alg_bytes": alg, "achieved_gbs": alg / (ms * 1e6), "peak_gbs": peak,
                         "frac": alg / (ms * 1e6) / peak, "peak_source": src}}


def extra_large_pyramid():
    """4800x3409, disparities 0..256, 4-level pyramid, census 9x7, P1=10, P2=150 (fractal scene), one
    pair alone: device time per pair and device memory, with the warp-per-scanline (latency)
    kernels -- what a single caller of the host API gets -- and with the default kernels."""
    import torch
    import fasterstereocuda_b200 as fsc
    from fasterstereocuda_b200 import scenes
    from cuda.bindings import runtime as rt
    W, H = 4800, 3409
    L, R, _ = scenes.building_like(2, W, H)
    dl, dr = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    out = torch.empty((H, W), dtype=torch.float32, device="cuda")

    def run(tuning):
        torch.cuda.synchronize()
        free0 = rt.cudaMemGetInfo()[1]
        p = fsc.FasterStereoCuda()
        if not p.Init(fsc.StereoOption1(width=W, height=H, min_disp=0, max_disp=256, num_layers=4),
                      fsc.LevelOverride(1, 10, 150), fsc.ExtOptions()):
            raise RuntimeError(p.last_error())
        if tuning and not p.set_tuning(fsc.Tuning(*tuning)):
            raise RuntimeError(p.last_error())
        torch.cuda.synchronize()
        used = free0 - rt.cudaMemGetInfo()[1]
        s = torch.cuda.Stream()
        for _ in range(2):
            p.match_device(dl, dr, out, s.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n = 5
        e0.record(s)
        for _ in range(n):
            if not p.match_device(dl, dr, out, s.cuda_stream):
                raise RuntimeError(p.last_error())
        e1.record(s)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / n
        peak = free0 - rt.cudaMemGetInfo()[1]  # after the first matches (the latency kernels' extra volume)
        levels = [p.level_info(i) for i in range(4)]
        p.Release()
        torch.cuda.synchronize()
        return ms, used, peak, levels

    ms, used, peak, levels = run((4, 0, 4, 0, 0, 8, 8))
    ms_d, used_d, peak_d, _ = run(None)
    # algorithmic bytes of a pair: 4*W*H*D + 6*W*H per view and level (the two-pass design's cost
    # and path traffic plus images and maps); the coarsest level matches both views (LR check)
    alg = sum((2 if i == len(levels) - 1 else 1) * (4 * w * h * d + 6 * w * h) for i, (w, h, _, d) in enumerate(levels))
    hbm, src = peaks()
    extra = (dl.numel() * 2 + out.numel() * 4) / 2**30
    return {"workload": "4800x3409, D=256, 4-level pyramid, census 9x7, P1=10 P2=150, fractal scene, one pair alone",
            "ms_per_pair": ms, "pairs_per_s": 1e3 / ms, "kernels": "warp per scanline (row_kernel = col_kernel = 4)",
            "matcher_device_gib": used / 2**30, "peak_device_gib": peak / 2**30 + extra,
            "default_kernels": {"ms_per_pair": ms_d, "matcher_device_gib": used_d / 2**30,
                                "peak_device_gib": peak_d / 2**30 + extra},
            "roofline": {"bound": "hbm", "alg_bytes_per_pair": alg, "achieved_gbs": alg / (ms * 1e6), "peak_gbs": hbm,
                         "frac": alg / (ms * 1e6) / hbm, "peak_source": src},
            "levels": levels}


def cpu_baseline(a, pool):
    from oracle import oracle as O
    O.lib()
    cores = O.max_threads()
    if a.workload == "pyramid":
        pc = O.PyrConfig(width=W_, height=H_, max_disp=DMAX, num_layers=LAYERS)
        one = lambda L, R: O.pyr_match(pc, L, R)  # noqa: E731
    else:
        cfg = O.Config(width=W_, height=H_, disp_range=DMAX)
        one = lambda L, R: O.match(cfg, L, R)  # noqa: E731
    one(*pool[0])
    n, t = 0, time.perf_counter()
    while n < 3 or time.perf_counter() - t < a.cpu_seconds:
        one(*pool[n % len(pool)])
        n += 1
    dt = time.perf_counter() - t
    return {"value": n / dt, "unit": "pairs/s", "cores": cores, "kind": "port",
            "sample": f"{n} pairs of the same workload in {dt:.1f} s (oracle/ C restatement, OpenMP)"}


def run_extra(a):
    """One extra workload on its own (single GPU), with a small pool of distinct pairs."""
    from fasterstereocuda_b200 import scenes
    n = a.extra_pairs
    if a.extra == "float_sgm":
        out = extra_float_sgm(a.float_batch)
    elif a.extra == "large_pyramid":
        out = extra_large_pyramid()
    elif a.extra == "batch_uneven":
        specs = scenes.batch_specs()[:n]
        imgs = [scenes.planar_pair(seed, w, h, dmin=2.0, dmax=60.0)[:2] for (w, h, d, seed) in specs]
        out = batch_vs_loop([(w, h, 0, d) for (w, h, d, _) in specs], imgs, runs=3, warmup=1)
    else:
        pool = make_pool(min(n, 16))
        imgs = [pool[i % len(pool)] for i in range(n)]
        if a.extra == "batch":
            out = batch_vs_loop([(W_, H_, 0, DMAX)] * n, imgs, runs=5, warmup=2)
        else:
            out = batch_pyramid_vs_loop(imgs, runs=5, warmup=2)
    print(json.dumps({"extra": a.extra, **out}), flush=True)
    return 0


def relaunch(a):
    """--gpus N without a launcher: one process per GPU under torch.distributed.run (which sets
    RANK / LOCAL_RANK / WORLD_SIZE), this script's arguments passed through."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={a.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve()), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def run_dry(a, rank, world):
    """The launcher's plumbing without CUDA: each rank takes its shard of a step's pairs, the ranks
    meet at the barriers of a timed region whose length differs per rank, and rank 0 prints the
    maximum over ranks and every rank's shard."""
    from fasterstereocuda_b200 import replicas
    mine = replicas.shard(a.batch * world, rank, world)
    replicas.barrier(world)
    t = time.perf_counter()
    time.sleep(0.02 * (rank + 1))
    replicas.barrier(world)
    ms = replicas.max_over_ranks((time.perf_counter() - t) * 1e3, world)
    shards = replicas.gather_to_rank0([mine.start, mine.stop], world, rank)
    if rank == 0:
        print(json.dumps({"dry_run": True, "n_gpus": world, "pairs_per_step": a.batch * world, "shards": shards,
                          "ms_per_step": ms}), flush=True)
    return 0


def main():
    a = parse()
    if "WORLD_SIZE" not in os.environ and a.gpus > 1:
        return relaunch(a)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != a.gpus:
        print(f"bench.py: --gpus {a.gpus} but {world} ranks were launched", file=sys.stderr)
        return 2
    if a.impl == "reference":
        return run_reference(a, rank, world)
    if a.extra:
        return run_extra(a)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if a.dry_run:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        else:
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local_rank))
    try:
        return run_dry(a, rank, world) if a.dry_run else run_ours(a, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
