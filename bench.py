"""Benchmark of the path-guiding hot path on B200.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workload "sdtree" (SD-tree standalone): 2^20 seeded radiance records (uniform positions,
4-lobe vMF directions kappa 50, lognormal(0,1) radiance) are recorded, the trees are built and
refined at 12000*sqrt(2), then 2^22 guided sample+pdf queries run at uniform positions.  One
step = clear + record + build + refine + sample/pdf.  Inputs are resident in HBM when the
timed region starts (value); "e2e" repeats the step through the C ABI from pinned host
buffers with the host<->device copies inside the timed region.  L2 is flushed (a 256 MiB
write) before every timed step.  N GPUs run independent replicas (no collective): value is
the work of all ranks over the slowest rank's time.

--impl reference runs RTLib's own SD-tree code (oracle/_ref, built from the reference sources)
on this machine's host cores with the same workload and metric.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_REC = 1 << 20
N_Q = 1 << 22
# algorithmic bytes of one sample+pdf query: position in (12 B), direction (12 B) and pdf
# (4 B) out; the Xorshift32 seed is derived from the query index
Q_BYTES = 28
LAUNCHES_PER_STEP = 21  # clear 1, record 1, build 1, refine 17, sample 1


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML every ~2 ms while the timed region
    runs (reading only; no setting of the GPU is touched)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "hw_power_brake_slowdown": 0x80, "sw_power_cap": 0x4}

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self.run = False
        self.th = None
        self.nv = None

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv = nv
            self.h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
        except Exception as e:  # noqa: BLE001
            self.err = str(e)
            return
        self.run = True

        def loop():
            while self.run:
                try:
                    self.samples.append((self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM),
                                         self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)))
                except Exception:  # noqa: BLE001
                    pass
                time.sleep(0.002)

        self.th = threading.Thread(target=loop, daemon=True)
        self.th.start()

    def stop(self):
        if self.nv is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [f"nvml unavailable: {getattr(self, 'err', '')}"]}
        self.run = False
        self.th.join()
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["no samples"]}
        mhz = [m for m, _ in self.samples]
        reasons = sorted({k for _, r in self.samples for k, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.samples), "source": "nvml, ~2 ms period"}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------- SD-tree workload
def _sdtree_inputs():
    from rtlib_b200 import workloads as W
    rec = W.sdtree_records(N_REC, 0)
    q = W.sdtree_queries(N_Q, 1)
    return rec, q, W.spatial_threshold(1)


def _traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get(kernel)
    return None


def bench_sdtree_ours(args, rank, world):
    import torch
    from rtlib_b200.sdtree import SDTree

    dev = torch.device("cuda", rank % max(1, torch.cuda.device_count()))
    torch.cuda.set_device(dev)
    rec, q, th = _sdtree_inputs()
    T = lambda a: torch.from_numpy(a).to(dev)
    pos, uv, rad = T(rec["pos"]), T(rec["uv"]), T(rec["radiance"])
    qpos = T(q["pos"])
    out_dir = torch.empty((N_Q, 3), dtype=torch.float32, device=dev)
    out_pdf = torch.empty(N_Q, dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    tree = SDTree((0, 0, 0), (1, 1, 1))

    def build_part(p, u, r):
        tree.clear()
        tree.record(p, u, r)
        tree.build()
        tree.refine(th)

    def sample_part(qp):
        # guided direction + pdf of the sampled point (DTreeT::Sample + DTreeT::Pdf)
        tree.sample_pdf(qp, None, seed_base=0, out_dir=out_dir, out_pdf_uv=out_pdf)

    # one CUDA graph per half of the step (the split lets the sample kernel be timed alone)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(2):
            build_part(pos, uv, rad)
            sample_part(qpos)
    torch.cuda.current_stream().wait_stream(side)
    g_build, g_sample = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
    with torch.cuda.graph(g_build):
        build_part(pos, uv, rad)
    with torch.cuda.graph(g_sample):
        sample_part(qpos)
    stream = torch.cuda.current_stream()
    t0 = time.perf_counter()
    k = 0
    while k < args.warmup or time.perf_counter() - t0 < 0.5:  # also lets the clocks ramp up
        g_build.replay()
        g_sample.replay()
        k += 1
    torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = ClockSampler(dev.index)
    _barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    for k in range(args.steps):
        flush.fill_(k & 0xff)
        a, b, c = ev[k]
        a.record(stream)
        g_build.replay()
        b.record(stream)
        g_sample.replay()
        c.record(stream)
    torch.cuda.synchronize()
    _barrier(world)
    clk = clocks.stop()
    step_ms = [a.elapsed_time(c) for a, b, c in ev]
    sample_ms = [b.elapsed_time(c) for a, b, c in ev]
    ms = sum(step_ms) / len(step_ms)
    ms = _max_over_ranks(ms, world, dev)
    st = tree.stats()
    assert tree.status() == 0

    # e2e: pinned host buffers through the same C-ABI calls, copies inside the timed region
    hp = {k: torch.from_numpy(v).pin_memory() for k, v in (("pos", rec["pos"]), ("uv", rec["uv"]),
                                                          ("rad", rec["radiance"]), ("qpos", q["pos"]))}
    h_dir = torch.empty((N_Q, 3), dtype=torch.float32).pin_memory()
    h_pdf = torch.empty(N_Q, dtype=torch.float32).pin_memory()
    dpos, duv, drad, dq = (torch.empty_like(x, device=dev) for x in (hp["pos"], hp["uv"], hp["rad"], hp["qpos"]))
    h2d = sum(x.numel() * x.element_size() for x in hp.values())
    d2h = h_dir.numel() * 4 + h_pdf.numel() * 4
    e2e_ms = []
    for k in range(args.warmup + args.steps):
        flush.fill_(k & 0xff)
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        dpos.copy_(hp["pos"], non_blocking=True)
        duv.copy_(hp["uv"], non_blocking=True)
        drad.copy_(hp["rad"], non_blocking=True)
        dq.copy_(hp["qpos"], non_blocking=True)
        build_part(dpos, duv, drad)
        sample_part(dq)
        h_dir.copy_(out_dir, non_blocking=True)
        h_pdf.copy_(out_pdf, non_blocking=True)
        c.record(stream)
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e_ms.append(a.elapsed_time(c))
    e2e = _max_over_ranks(sum(e2e_ms) / len(e2e_ms), world, dev)
    ops = (N_REC + N_Q) * world
    peak, peak_kind = _peaks()
    s_ms = sum(sample_ms) / len(sample_ms)
    achieved = Q_BYTES * N_Q / (s_ms * 1e-3) / 1e9
    return {
        "metric": "SD-tree record+refine+sample throughput (config 1)",
        "value": ops / (ms * 1e-3) / 1e6,
        "unit": "Mops/s",
        "ms_per_step": ms,
        "e2e": {"value": ops / (e2e * 1e-3) / 1e6, "unit": "Mops/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": {"kernel": "k_sample_pdf", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs (burst copy)",
                     "traffic": _traffic("k_sample_pdf"), "algorithmic_bytes_per_launch": Q_BYTES * N_Q,
                     "launch_ms": s_ms},
        "clocks": clk,
        "gpu_launches": LAUNCHES_PER_STEP * args.steps,
        "sdtree": st,
    }


def _ref_workload(lib_kind, threads, reps=1):
    """One config-1 pass on the host: record (single thread), build + refine (single
    thread), sample+pdf over `threads` threads.  Returns seconds per pass."""
    from oracle.oracle import Oracle, Reference
    rec, q, th = _sdtree_inputs()
    times = []
    for _ in range(reps):
        if lib_kind == "reference":
            t = Reference().sdtree((0, 0, 0), (1, 1, 1))
        else:
            t = Oracle().sdtree((0, 0, 0), (1, 1, 1))
        t0 = time.perf_counter()
        t.record(rec["pos"], rec["uv"], rec["radiance"])
        t.build()
        t.refine(th)
        if lib_kind == "reference":
            t.sample_pdf(q["pos"], q["seeds"], threads=threads, with_dir=True)
        else:
            t.sample_pdf(q["pos"], q["seeds"], with_dir=True)
        times.append(time.perf_counter() - t0)
    return times


def _ref_kind():
    from oracle.oracle import REF_SO
    return "reference" if os.path.exists(REF_SO) else "port"


def cpu_baseline_sdtree():
    kind = _ref_kind()
    cores = os.cpu_count() or 1
    threads = cores if kind == "reference" else 1
    times = []
    t_start = time.perf_counter()
    while time.perf_counter() - t_start < 10.0 and len(times) < 30:
        times += _ref_workload(kind, threads)
    s = statistics.median(times)
    return {"value": (N_REC + N_Q) / s / 1e6, "unit": "Mops/s", "cores": threads, "kind": kind,
            "sample": f"{len(times)} full config-1 passes (2^20 records, refine, 2^22 queries); record/build/"
                      f"refine single-threaded as in RTLib, sample+pdf on {threads} thread(s)",
            "seconds_per_pass": s}


# ---------------------------------------------------------------------------- plumbing
def _barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _max_over_ranks(x, world, dev):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sdtree", choices=["sdtree"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)

    if args.impl == "reference":
        if rank != 0:
            return 0
        kind = _ref_kind()
        cores = os.cpu_count() or 1
        threads = cores if kind == "reference" else 1
        _ref_workload(kind, threads, reps=args.warmup)
        times = _ref_workload(kind, threads, reps=args.steps)
        s = sum(times) / len(times)
        v = (N_REC + N_Q) / s / 1e6
        line = {"impl": "reference", "metric": "SD-tree record+refine+sample throughput (config 1)", "value": v,
                "unit": "Mops/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": s * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": "sdtree-standalone: 2^20 records, refine at 12000*sqrt(2), 2^22 sample+pdf",
                           "records": N_REC, "queries": N_Q},
                "cpu_baseline": {"value": v, "unit": "Mops/s", "cores": threads, "kind": kind,
                                 "sample": "full config-1 passes on the host"},
                "e2e": {"value": v, "unit": "Mops/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(_env_int("LOCAL_RANK", rank))
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    res = bench_sdtree_ours(args, rank, world)
    line = {"metric": res["metric"], "value": res["value"], "unit": res["unit"], "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "sdtree-standalone: 2^20 records, refine at 12000*sqrt(2), 2^22 sample+pdf",
                       "records": N_REC, "queries": N_Q, "l2": "flushed (256 MiB write) before every timed step",
                       "parallelism": f"replicas x{world}"},
            "e2e": res["e2e"], "roofline": res["roofline"], "clocks": res["clocks"],
            "gpu_launches": res["gpu_launches"], "sdtree": res["sdtree"]}
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sdtree()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
