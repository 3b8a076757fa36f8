#!/usr/bin/env python
"""Throughput benchmark of the B200 SGM stereo engine.

Metric: stereo pairs per second at 1242x375 with a 64-disparity search, the headline
configuration (3-level pyramid with per-pixel range propagation, census 9x7, P1=10, P2=150,
left-right check, median, small-region removal). Inputs are seeded synthetic KITTI-like pairs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload pyramid|plain]

One step = one batch of --batch pairs. `value` is timed on the device with CUDA events over
exactly K steps whose inputs already sit in HBM (a rotating pool of distinct pairs larger than
L2); `e2e` is the same metric through the host-buffer API (pinned host memory, copies inside the
timed region). Under torchrun every rank runs its own matchers on its own GPU (weak scaling).
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

W_, H_, DMAX = 1242, 375, 64
LAYERS = 3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["pyramid", "plain"], default="pyramid")
    ap.add_argument("--batch", type=int, default=32, help="pairs per step")
    ap.add_argument("--streams", type=int, default=8, help="matchers (one CUDA stream each) per GPU")
    ap.add_argument("--pool", type=int, default=160, help="distinct input pairs resident in HBM")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-extras", action="store_true", help="skip the CPU baseline and extra workloads")
    return ap.parse_args()


# ------------------------------------------------------------------------------------ helpers
def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_pool(n_distinct, seed=100):
    """n_distinct different pairs: 8 scenes, each shifted/flipped into many variants."""
    from fasterstereocuda_b200 import scenes
    base = [scenes.kitti_like(seed + i, W_, H_)[:2] for i in range(8)]
    pool = []
    rng = np.random.Generator(np.random.PCG64(seed))
    for i in range(n_distinct):
        L, R = base[i % 8]
        dy = int(rng.integers(0, 40))
        L2, R2 = np.roll(L, dy, 0), np.roll(R, dy, 0)
        if (i // 8) % 2:
            L2, R2 = L2[::-1].copy(), R2[::-1].copy()
        pool.append((np.ascontiguousarray(L2), np.ascontiguousarray(R2)))
    return pool


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""
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
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
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
        rows = [l.split(",") for l in open(self.path).read().splitlines() if l.count(",") >= 8]
        os.remove(self.path)
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
    if kernel.startswith("vpaths"):
        return nviews * (2 * V + 4 * n)
    if kernel == "census":
        return 2 * n + 2 * census_bytes * n
    if kernel == "lr_median":
        return 12 * n
    return 0


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
    print(json.dumps(line), flush=True)
    return 0


def metric_name(workload):
    if workload == "pyramid":
        return "pairs/s at 1242x375x64 (3-level pyramid, census 9x7, P1=10 P2=150, LR + median + peaks)"
    return "pairs/s at 1242x375x64 (single level, census 9x7, P1=10 P2=150, LR + median)"


def workload_config(a, batch):
    c = {"workload": f"{W_}x{H_} D={DMAX} " + ("3-level pyramid (configs[1] scene)" if a.workload == "pyramid"
                                                 else "single-level plain SGM"),
         "width": W_, "height": H_, "disparities": DMAX, "census": "9x7", "p1": 10, "p2": 150,
         "batch_pairs": batch}
    if a.workload == "pyramid":
        c["layers"] = LAYERS
    return c


# ------------------------------------------------------------------------------------ our arm
def run_ours(a, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import fasterstereocuda_b200 as fsc

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = fsc.load_library()

    def make_matcher():
        if a.workload == "pyramid":
            m = fsc.FasterStereoCuda()
            ok = m.Init(fsc.StereoOption1(width=W_, height=H_, min_disp=0, max_disp=DMAX, num_layers=LAYERS,
                                          do_lr_check=True, do_rm_peaks=True), fsc.LevelOverride(1, 10, 150),
                        fsc.ExtOptions())
        else:
            m = fsc.StereoCuda()
            ok = m.Init(W_, H_, 0, DMAX, fsc.CuSGMOption(p1=10, p2_init=150, cs_type=1, num_paths=4,
                                                          do_median_filter=True, do_lr_check=True, lr_threshold=1.0,
                                                          unique_threshold=0.95, using_constant_p2=True))
        if not ok:
            raise RuntimeError(f"matcher init failed: {m.last_error()}")
        return m

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
    pool = make_pool(a.pool, seed=100 + 17 * rank)
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
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

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

    # second pass of the same steps with per-kernel CUDA events (roofline of the dominant kernel)
    fsc.profile_enable(True)
    for _ in range(a.steps):
        step()
    torch.cuda.synchronize()
    prof = fsc.profile_read()
    fsc.profile_enable(False)

    # e2e: the host-buffer API (synchronous, like the reference's Match), pinned host memory
    e2e_steps = max(1, min(a.steps, 5))
    hostL = [torch.from_numpy(L).pin_memory().numpy() for L, _ in pool[:a.batch]]
    hostR = [torch.from_numpy(R).pin_memory().numpy() for _, R in pool[:a.batch]]
    hostO = [torch.empty((H_, W_), dtype=torch.float32).pin_memory().numpy() for _ in range(a.batch)]
    m0 = matchers[0]

    def host_call(i):
        if a.workload == "pyramid":
            ok = m0.Match(hostL[i], hostR[i], hostO[i])
        else:
            ok = m0.Match(hostL[i], hostR[i], hostO[i])
        if not ok:
            raise RuntimeError(m0.last_error())

    host_call(0)
    barrier()
    te = time.perf_counter()
    for _ in range(e2e_steps):
        for b in range(a.batch):
            host_call(b)
    te = max_over_ranks(time.perf_counter() - te)
    e2e_value = e2e_steps * a.batch * world / te

    if rank != 0:
        return 0
    hbm_peak, peak_kind = peaks()
    # per-kernel algorithmic bytes over the profiled pass
    levels = []
    if a.workload == "pyramid":
        for lv in range(LAYERS):
            w, h, mn, d = matchers[0].level_info(lv)
            levels.append((w, h, d, 2 if lv == LAYERS - 1 else 1))
    else:
        levels.append((W_, H_, DMAX, 2))
    per_call_bytes = {}
    for k in prof:
        per_call_bytes[k] = sum(alg_bytes(k, w, h, d, nv, 8) for (w, h, d, nv) in levels)
    dom = max(prof, key=lambda k: prof[k]["ms"]) if prof else None
    calls = a.steps * a.batch
    roofline = None
    if dom:
        total_ms = prof[dom]["ms"]
        byts = per_call_bytes.get(dom, 0) * calls
        ach = byts / (total_ms / 1e3) / 1e9 if total_ms > 0 else 0.0
        roofline = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
                    "frac": ach / hbm_peak, "traffic": None, "peak_kind": peak_kind,
                    "avg_launch_us": total_ms / prof[dom]["launches"] * 1e3,
                    "alg_bytes_per_launch": per_call_bytes.get(dom, 0) / max(1, prof[dom]["launches"] // calls)}
    kernels = {k: {"launches": v["launches"], "ms": round(v["ms"], 4),
                   "share": round(v["ms"] / sum(x["ms"] for x in prof.values()), 4)} for k, v in prof.items()}

    cpu = None
    if not a.no_extras:
        cpu = cpu_baseline(a, pool)
    clocks = clk.summary()
    line = {"metric": metric_name(a.workload), "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8/u32 (f32 subpixel)",
            "data": "synthetic seeded KITTI-like pairs",
            "config": dict(workload_config(a, a.batch), streams=S,
                           l2=f"inputs larger than L2: rotating pool of {len(dL)} distinct pairs "
                              f"({pool_bytes / 2**20:.0f} MiB) per GPU"),
            "e2e": {"value": e2e_value, "unit": "pairs/s",
                    "h2d_bytes_per_step": a.batch * 2 * W_ * H_, "d2h_bytes_per_step": a.batch * 4 * W_ * H_,
                    "api": "FasterStereoCuda.Match (host buffers, synchronous)" if a.workload == "pyramid"
                    else "StereoCuda.Match (host buffers, synchronous)"},
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches,
            "bit_exact_vs_oracle": bit_exact, "kernels": kernels}
    print(json.dumps(line), flush=True)
    return 0


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


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return run_reference(a, rank, world)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        return run_ours(a, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
