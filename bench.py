"""Benchmark of the path-guiding hot path on B200.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workload "cornell" (default; the guided path-tracing configuration): the procedural
Cornell-style box (5 walls, 2 boxes rotated -18/+18 degrees, 0.25 x 0.25 light of radiance
(17,12,4)) at 512 x 512, max depth 8, NEE, SD-tree guiding with 50% BSDF/guide mixing, passes
doubling from 1 to 1024 spp (2047 spp in total) under the pass controller, with record ->
build -> refine between passes.  One step = one complete guided render.  Metric: Mpaths/s
(camera paths = pixels x spp).  "e2e" repeats the step through the C ABI from host arrays:
the scene goes host->device, the image comes back device->host, both inside the timed region.

Workload "occluded": the occluded-light scene (1280 x 720, ~1M triangles in a 10 x 4 x 10 room lit
only through a 1 x 2 doorway by 4096 emitters) with NEE + RIS (32 candidates), max depth 16 and
the hash-grid guide (2^20 slots, Morton keys, Morton quadtrees) under its pass controller.

Workload "learned": equal-time relMSE of the learned guide against plain SD-tree guiding on the
occluded scene (budgets --budgets, reference --ref-seconds of SD-tree rendering).

Workload "sdtree" (SD-tree standalone): 2^20 seeded radiance records (uniform positions,
4-lobe vMF directions kappa 50, lognormal(0,1) radiance) are recorded, the trees are built and
refined at 12000*sqrt(2), then 2^22 guided sample+pdf queries run at uniform positions.

Workload "hashgrid": the hash-grid guide's batched routines on the occluded scene's grid
(256 x 64 x 192 cells, 2^20 slots, 63-bit Morton keys, level-4 Morton quadtrees): insert 2^19
surface points, look up 2^22 surface points, record 2^22 Morton-leaf values, build every cell's
sampling pyramid, 2^22 guided sample+pdf queries.  The CPU baseline is RTLib's own per-point
routines (oracle/_ref), single-threaded, on the workload scaled down 64x.

Inputs are resident in HBM when the timed region starts (value).  L2 is flushed (a 256 MiB
write) before every timed step.  N GPUs run independent replicas (no collective): value is
the work of all ranks over the slowest rank's time.

--impl reference runs the CPU implementation of the same workload on this machine's host
cores: RTLib's own SD-tree code (oracle/_ref) for "sdtree"; for "cornell", where RTLib's
integrator exists only as OptiX programs, the CPU restatement of that integrator (oracle/)
rendering the same 512 x 512 image into one shared SD-tree over all host threads, each step
the pass schedule truncated at 15 spp (a bounded sample of the 2047-spp step).
"""
from __future__ import annotations

import argparse
import gc
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
# algorithmic bytes of one record: position 12 B, canonical direction 8 B, radiance 4 B
REC_BYTES = 24
LAUNCHES_PER_STEP = 23  # clear 2, record 1, build 1, refine 18, sample 1 (three CUDA graphs)


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
    from rtlib_b200.workloads import spatial_threshold as W_th
    T = lambda a: torch.from_numpy(a).to(dev)
    pos, uv, rad = T(rec["pos"]), T(rec["uv"]), T(rec["radiance"])
    qpos = T(q["pos"])
    out_dir = torch.empty((N_Q, 3), dtype=torch.float32, device=dev)
    out_pdf = torch.empty(N_Q, dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    tree = SDTree((0, 0, 0), (1, 1, 1))

    def record_part(p, u, r):
        tree.clear()
        tree.record(p, u, r)

    def refine_part(p, u, r):
        tree.build()
        tree.refine(th)
        for it in range(2, args.passes + 1):
            # the same records again into the refined topology (deeper quadtrees to sample)
            tree.record(p, u, r)
            tree.build()
            tree.refine(W_th(it))

    def build_part(p, u, r):
        record_part(p, u, r)
        refine_part(p, u, r)

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
    # one CUDA graph per phase of the step (record, build + refine, sample) so that each is
    # timed alone
    g_record, g_refine, g_sample = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
    with torch.cuda.graph(g_record):
        record_part(pos, uv, rad)
    with torch.cuda.graph(g_refine):
        refine_part(pos, uv, rad)
    with torch.cuda.graph(g_sample):
        sample_part(qpos)
    stream = torch.cuda.current_stream()
    t0 = time.perf_counter()
    k = 0
    while k < args.warmup or time.perf_counter() - t0 < 0.5:  # also lets the clocks ramp up
        g_record.replay()
        g_refine.replay()
        g_sample.replay()
        k += 1
    torch.cuda.synchronize()

    ev = [tuple(torch.cuda.Event(enable_timing=True) for _ in range(4)) for _ in range(args.steps)]
    clocks = ClockSampler(dev.index)
    _barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    for k in range(args.steps):
        flush.fill_(k & 0xff)
        a, r, b, c = ev[k]
        a.record(stream)
        g_record.replay()
        r.record(stream)
        g_refine.replay()
        b.record(stream)
        g_sample.replay()
        c.record(stream)
    torch.cuda.synchronize()
    _barrier(world)
    clk = clocks.stop()
    step_ms = [a.elapsed_time(c) for a, r, b, c in ev]
    sample_ms = [b.elapsed_time(c) for a, r, b, c in ev]
    record_ms = [a.elapsed_time(r) for a, r, b, c in ev]
    refine_ms = [r.elapsed_time(b) for a, r, b, c in ev]
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
    e2e_steps = getattr(args, "e2e_steps", None) or args.steps
    for k in range(args.warmup + e2e_steps):
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
    ops = (args.passes * N_REC + N_Q) * world  # every pass records the 2^20 records once
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
        "gpu_launches": (LAUNCHES_PER_STEP + (args.passes - 1) * 21) * args.steps,
        "sdtree": st,
        "roofline_issue": _issue_roofline_sample(s_ms, clk),
        "roofline_record": {"kernel": "k_record (with clear)", "bound": "L2 atomics", "unit": "GB/s",
                            "achieved": REC_BYTES * N_REC / (statistics.mean(record_ms) * 1e-3) / 1e9,
                            "peak": peak, "frac": REC_BYTES * N_REC / (statistics.mean(record_ms) * 1e-3) / 1e9 / peak,
                            "algorithmic_bytes_per_record": REC_BYTES,
                            "atomics_per_s": 2 * N_REC / (statistics.mean(record_ms) * 1e-3),
                            "note": "2 int64 atomics per record before warp / CTA aggregation"},
        "phases": {"record_Mrec_s": N_REC / (statistics.mean(record_ms) * 1e-3) / 1e6,
                   "build_refine_ms": statistics.mean(refine_ms),
                   "sample_pdf_Mq_s": N_Q / (s_ms * 1e-3) / 1e6},
    }


def _ref_workload(lib_kind, threads, reps=1, phases=None):
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
        t1 = time.perf_counter()
        t.build()
        t.refine(th)
        t2 = time.perf_counter()
        if lib_kind == "reference":
            t.sample_pdf(q["pos"], q["seeds"], threads=threads, with_dir=True)
        else:
            t.sample_pdf(q["pos"], q["seeds"], with_dir=True)
        t3 = time.perf_counter()
        times.append(t3 - t0)
        if phases is not None:
            phases.append((t1 - t0, t2 - t1, t3 - t2))
    return times


def _ref_kind():
    from oracle.oracle import REF_SO
    return "reference" if os.path.exists(REF_SO) else "port"


def cpu_baseline_sdtree():
    kind = _ref_kind()
    cores = os.cpu_count() or 1
    threads = cores if kind == "reference" else 1
    times, ph = [], []
    t_start = time.perf_counter()
    while time.perf_counter() - t_start < 10.0 and len(times) < 30:
        times += _ref_workload(kind, threads, phases=ph)
    s = statistics.median(times)
    return {"value": (N_REC + N_Q) / s / 1e6, "unit": "Mops/s", "cores": threads, "kind": kind,
            "sample": f"{len(times)} full config-1 passes (2^20 records, refine, 2^22 queries); record/build/"
                      f"refine single-threaded as in RTLib, sample+pdf on {threads} thread(s)",
            "seconds_per_pass": s,
            "phases": {"record_Mrec_s": N_REC / statistics.median(p[0] for p in ph) / 1e6,
                       "build_refine_ms": 1e3 * statistics.median(p[1] for p in ph),
                       "sample_pdf_Mq_s": N_Q / statistics.median(p[2] for p in ph) / 1e6,
                       "sample_pdf_1thread_Mq_s": _ref_sample_1thread(kind)}}


# steps of the config-1 SD-tree sub-record of the default line: ~0.15 ms each, so that the
# timed region spans a few hundred milliseconds of clock samples
SUB_SDTREE_STEPS = 2000


def sdtree_subrecord(args, rank, world):
    """Config 1 (SD-tree standalone) measured inside the default workload's run: the same
    record -> build -> refine -> sample+pdf step as --workload sdtree, with its own clocks,
    rooflines and the host-side rate of RTLib's own SD-tree code as its CPU baseline."""
    sub = argparse.Namespace(**vars(args))
    sub.steps, sub.warmup, sub.passes, sub.e2e_steps = SUB_SDTREE_STEPS, 20, 1, 20
    r = bench_sdtree_ours(sub, rank, world)
    out = {"metric": r["metric"], "value": r["value"], "unit": r["unit"], "steps": sub.steps, "warmup": sub.warmup,
           "ms_per_step": r["ms_per_step"],
           "config": {"workload": "sdtree-standalone: 2^20 records, refine at 12000*sqrt(2), 2^22 sample+pdf",
                      "records": N_REC, "queries": N_Q, "l2": "flushed (256 MiB write) before every timed step"},
           "e2e": dict(r["e2e"], steps=sub.e2e_steps), "roofline": r["roofline"], "roofline_issue": r["roofline_issue"],
           "roofline_record": r["roofline_record"],
           "phases": r["phases"], "clocks": r["clocks"], "gpu_launches": r["gpu_launches"], "sdtree": r["sdtree"]}
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_sdtree()
    return out


def _ref_sample_1thread(kind, n=1 << 18):
    """Single-threaded sample+pdf rate of the host implementation on the first n queries."""
    from oracle.oracle import Oracle, Reference
    rec, q, th = _sdtree_inputs()
    t = Reference().sdtree((0, 0, 0), (1, 1, 1)) if kind == "reference" else Oracle().sdtree((0, 0, 0), (1, 1, 1))
    t.record(rec["pos"], rec["uv"], rec["radiance"])
    t.build()
    t.refine(th)
    t0 = time.perf_counter()
    if kind == "reference":
        t.sample_pdf(q["pos"][:n], q["seeds"][:n], threads=1, with_dir=True)
    else:
        t.sample_pdf(q["pos"][:n], q["seeds"][:n], with_dir=True)
    return n / (time.perf_counter() - t0) / 1e6


# ---------------------------------------------------------------------------- Cornell workload
C_W = C_H = 512
C_BUDGET = 2047          # passes of 1, 2, 4, ..., 512, 1024 spp
C_MAX_DEPTH = 8
C_FRACTION = 0.5
C_AABB = ((-0.005,) * 3, (1.005,) * 3)  # world AABB padded by 0.005 as the application does
# compulsory SoA bytes of one bounce visit (one path-bounce): reads queue index, origin,
# direction, throughput, depth, flags, rng, color (64 B); writes origin, direction,
# throughput, flags, rng, color, depth and the next-queue index (64 B).  Scene, material and
# tree reads are L2-resident and not counted; per-bounce radiance and trace-vertex writes
# (recording passes only) are excluded.
BOUNCE_BYTES = 128


def _issue_roofline(path_bounces, bounce_ms, clk):
    """k_bounce against the issue limit: its warp-instructions per path-bounce (ncu, see
    profiles/traffic.json) times the step's path-bounces over its CUDA-event time, against one
    warp-instruction per cycle on each of the 4 schedulers of the 148 SMs at the sampled clock."""
    ipb = _traffic("k_bounce_warp_inst_per_path_bounce")
    if ipb is None:
        return None
    mhz = clk.get("sm_mhz") or 1965.0
    achieved = ipb * path_bounces / (bounce_ms * 1e-3) / 1e9
    peak = 4 * 148 * mhz * 1e6 / 1e9
    return {"kernel": "k_bounce", "bound": "issue", "achieved": achieved, "peak": peak,
            "unit": "G warp-instructions/s", "frac": achieved / peak,
            "warp_inst_per_path_bounce": ipb, "thread_inst_per_inst": _traffic("k_bounce_thread_inst_per_inst"),
            "peak_source": f"4 schedulers x 148 SMs x {mhz:.0f} MHz (sampled SM clock)",
            "note": "instructions per path-bounce from ncu on the 7-spp case (profiles/k_bounce_commit_cornell_512.md)"}


def _issue_roofline_sample(launch_ms, clk):
    """k_sample_pdf against the issue limit: its warp-instructions per query (ncu, see
    profiles/traffic.json) times the 2^22 queries over the launch's CUDA-event time."""
    ipq = _traffic("k_sample_pdf_warp_inst_per_query")
    if ipq is None:
        return None
    mhz = clk.get("sm_mhz") or 1965.0
    achieved = ipq * N_Q / (launch_ms * 1e-3) / 1e9
    peak = 4 * 148 * mhz * 1e6 / 1e9
    return {"kernel": "k_sample_pdf", "bound": "issue", "achieved": achieved, "peak": peak,
            "unit": "G warp-instructions/s", "frac": achieved / peak, "warp_inst_per_query": ipq,
            "peak_source": f"4 schedulers x 148 SMs x {mhz:.0f} MHz (sampled SM clock)",
            "note": "instructions per query from ncu (profiles/k_sample_pdf_record_sdtree_cfg1.md)"}


def _recording_launches(budget, iteration_for_built=0):
    """Launches of the SD-tree pass schedule (RTSTreeControllerT::BegTrace / EndTrace, one
    sample per launch) that record, i.e. whose waves end with the trace-vertex commit."""
    remain, pas, per_all, per_tmp, it, rec = budget, 0, 0, 0, 0, 0
    while True:
        if per_tmp == 0:
            remain -= pas
            pas = min(remain, 1 << it)
            if remain - pas < 2 * pas or per_all >= budget:
                pas = remain
        rec += 0 if (it > iteration_for_built and remain <= pas) else 1
        per_all += 1
        per_tmp += 1
        if per_tmp >= pas:
            it += 1
            per_tmp = 0
        if per_all > budget:
            return rec


def set_budget(b):
    global C_BUDGET
    C_BUDGET = int(b)


def bench_cornell_ours(args, rank, world):
    import torch
    from rtlib_b200 import scenes
    from rtlib_b200.sdtree import SDTree, SDTreeController
    from rtlib_b200.tracer import FLAG_NEE, Tracer

    dev = torch.device("cuda", rank % max(1, torch.cuda.device_count()))
    torch.cuda.set_device(dev)
    sc = scenes.cornell_box(C_W, C_H)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    tr = Tracer(sc, dev, max_depth=C_MAX_DEPTH, seed=1)
    tree = SDTree(*C_AABB, fraction=C_FRACTION)
    ctrl = SDTreeController(tree, C_BUDGET, iteration_for_built=0, ratio_for_budget=1.0, samples_per_launch=1)
    img = torch.empty((C_H, C_W, 3), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def step():
        tr.clear()
        ctrl.start()
        tr.render_guided(tree, ctrl, FLAG_NEE, samples_per_launch=1)
        tr.image(img)

    t0 = time.perf_counter()
    k = 0
    while k < args.warmup or time.perf_counter() - t0 < 0.5:
        step()
        k += 1
    torch.cuda.synchronize()
    paths_per_step = C_W * C_H * (C_BUDGET + 1)  # the controller runs one extra launch after the last pass
    clocks = ClockSampler(dev.index)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    _barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    for k in range(args.steps):
        flush.fill_(k & 0xff)
        a, c = ev[k]
        a.record(stream)
        step()
        c.record(stream)
    torch.cuda.synchronize()
    _barrier(world)
    clk = clocks.stop()
    ms = sum(a.elapsed_time(c) for a, c in ev) / len(ev)
    ms = _max_over_ranks(ms, world, dev)
    cnt = tr.counters()
    st = tree.stats()
    assert tree.status() == 0
    assert tr.stats()["samples"] == C_BUDGET + 1

    # kernel times: one more step in measurement mode (events around every kernel, no graph)
    tr.set_timing(True)
    torch.cuda.synchronize()
    step()
    torch.cuda.synchronize()
    tk = tr.timings()
    tr.set_timing(False)
    ext_ms = tk["bounce"][0]
    peak, peak_kind = _peaks()
    achieved = cnt["path_bounces"] * BOUNCE_BYTES / (ext_ms * 1e-3) / 1e9

    # e2e: scene from host memory through the C ABI, image back to host
    e2e_ms, e2e_setup_ms = [], []
    h_img = torch.empty((C_H, C_W, 3), dtype=torch.float32).pin_memory()
    h2d = sum(np.asarray(sc[k]).nbytes for k in ("tri_v", "tri_mat", "tri_uv", "light_tris"))
    # one untimed run first; the objects of each run are released (and collected) outside the
    # timed region, so that no destructor's cudaFree stalls a later run's issue
    for k in range(1 + max(1, args.steps // 2)):
        flush.fill_(k & 0xff)
        torch.cuda.synchronize()
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        tr2 = Tracer(sc, dev, max_depth=C_MAX_DEPTH, seed=1)
        tree2 = SDTree(*C_AABB, fraction=C_FRACTION)
        ctrl2 = SDTreeController(tree2, C_BUDGET, iteration_for_built=0, ratio_for_budget=1.0, samples_per_launch=1)
        ctrl2.start()
        b = torch.cuda.Event(enable_timing=True)
        b.record(stream)
        tr2.render_guided(tree2, ctrl2, FLAG_NEE, samples_per_launch=1)
        h_img.copy_(tr2.image(), non_blocking=True)
        c.record(stream)
        torch.cuda.synchronize()
        if k > 0:
            e2e_ms.append(a.elapsed_time(c))
            e2e_setup_ms.append(a.elapsed_time(b))
        del tr2, tree2, ctrl2
        gc.collect()
        torch.cuda.synchronize()
    e2e = _max_over_ranks(sum(e2e_ms) / len(e2e_ms), world, dev)
    paths = paths_per_step * world
    return {
        "metric": "Mpaths/s",
        "value": paths / (ms * 1e-3) / 1e6,
        "unit": "Mpaths/s",
        "ms_per_step": ms,
        "e2e": {"value": paths / (e2e * 1e-3) / 1e6, "unit": "Mpaths/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(h_img.numel() * 4), "ms_per_step": e2e,
                "setup_ms": sum(e2e_setup_ms) / len(e2e_setup_ms),
                "note": "setup = scene upload, BVH build, tracer and SD-tree creation; the rest is the render "
                        "and the image read-back"},
        "roofline": {"kernel": "k_bounce", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs (burst copy)",
                     "traffic": (None if _traffic("k_bounce_bytes_per_path_bounce") is None else
                                 _traffic("k_bounce_bytes_per_path_bounce") * cnt["path_bounces"]
                                 / max(1, C_MAX_DEPTH * (C_BUDGET + 1))),
                     "traffic_bytes_per_path_bounce": _traffic("k_bounce_bytes_per_path_bounce"),
                     "algorithmic_bytes_per_path_bounce": BOUNCE_BYTES,
                     "path_bounces_per_step": cnt["path_bounces"],
                     "launch_ms": ext_ms / max(1, tk["bounce"][1]),
                     "kernel_ms_per_step": {kk: v[0] for kk, v in tk.items()},
                     "note": "bounce = BVH closest hit + shading + shadow ray; its bound is instruction "
                             "issue and traversal latency, the HBM figure is the SoA state traffic"},
        "roofline_issue": _issue_roofline(cnt["path_bounces"], ext_ms, clk),
        "clocks": clk,
        # raygen, max_depth bounces and the accumulation per launch, plus the commit of every
        # recording launch
        "gpu_launches": ((1 + C_MAX_DEPTH + 1) * (C_BUDGET + 1) + _recording_launches(C_BUDGET)) * args.steps,
        "counters_per_step": cnt,
        "sdtree": st,
    }


# budget of the host-side sample of the Cornell workload: passes of 1, 2, 4 and 8 spp (16
# launches) of the same 512 x 512 render; the full 2047-spp schedule would take many minutes
C_REF_BUDGET = 15


def _cornell_cpu_step(threads, budget=C_REF_BUDGET):
    """One host-side step: the guided 512 x 512 render of the pass schedule truncated at
    `budget` spp on the CPU restatement of the integrator, every frame split into pixel bands
    over `threads` host threads that record into one shared SD-tree (exact fixed-point merge
    after each frame).  Returns (paths, seconds)."""
    from oracle.oracle import Oracle, OracleRenderer
    from rtlib_b200 import scenes
    o = Oracle()
    sc = scenes.cornell_box(C_W, C_H)
    t = o.sdtree(*C_AABB)
    r = OracleRenderer(o, sc, max_depth=C_MAX_DEPTH, fraction=C_FRACTION, width=C_W, height=C_H)
    t0 = time.perf_counter()
    r.render_guided(t, budget, ratio_for_budget=1.0, threads=threads)
    dt = time.perf_counter() - t0
    return r.samples * C_W * C_H, dt


def _cornell_cpu(threads, seconds):
    """Host-side Mpaths/s: repeated steps (at least one) for about `seconds`."""
    paths, dt, n = 0, 0.0, 0
    while n == 0 or dt < seconds:
        p, d = _cornell_cpu_step(threads)
        paths += p
        dt += d
        n += 1
    return paths / dt / 1e6, dt, paths, n


# ---------------------------------------------------------------------------- occluded workload
O_W, O_H, O_DEPTH = 1280, 720, 16
O_AABB = ((-0.005,) * 3, (14.005, 4.005, 10.005))
O_GRID_BOUNDS, O_SLOTS, O_LEVEL = (256, 64, 192), 1 << 20, 4
O_BUDGET = 15  # passes of 1 (locate), 2 (record), 4 and 8 spp (record + sample)


def bench_occluded_ours(args, rank, world):
    """The occluded-light scene with NEE + RIS (32 candidates) and the hash-grid guide (Morton
    keys, 2^20 slots): one step = one HT-guided render of O_BUDGET spp under the Morton pass
    controller (locate, record, record + sample)."""
    import torch
    from rtlib_b200 import scenes
    from rtlib_b200.hashgrid import KEY_MORTON, HashGrid, MortonQuadTreeController, MortonQuadTrees
    from rtlib_b200.tracer import FLAG_NEE, FLAG_RIS, Tracer

    dev = torch.device("cuda", rank % max(1, torch.cuda.device_count()))
    torch.cuda.set_device(dev)
    sc = scenes.occluded_rooms(O_W, O_H)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    flags = FLAG_NEE | FLAG_RIS
    tr = Tracer(sc, dev, max_depth=O_DEPTH, num_candidates=32, seed=1)
    grid = HashGrid(*O_AABB, O_GRID_BOUNDS, O_SLOTS, keying=KEY_MORTON)
    trees = MortonQuadTrees(O_SLOTS, level=O_LEVEL, fraction=0.3)
    ctrl = MortonQuadTreeController(trees, O_BUDGET, iteration_for_built=1, ratio_for_budget=0.5)
    stream = torch.cuda.current_stream()

    def step(t=tr, g=grid, q=trees, c=ctrl):
        t.clear()
        g.clear()
        c.start()
        t.render_grid_guided(g, q, c, flags, samples_per_launch=1)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    samples = tr.stats()["samples"]
    clocks = ClockSampler(dev.index)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    _barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    for k in range(args.steps):
        flush.fill_(k & 0xff)
        a, c = ev[k]
        a.record(stream)
        step()
        c.record(stream)
    torch.cuda.synchronize()
    _barrier(world)
    clk = clocks.stop()
    ms = _max_over_ranks(sum(a.elapsed_time(c) for a, c in ev) / len(ev), world, dev)
    cnt = tr.counters()
    grid_status = grid.status()  # RTPG_STATUS_HASH_FULL if a bucket of 32 overflowed
    assert trees.status() == 0
    cells = int((grid.export() != 0).sum())
    # unguided NEE + RIS on the same tracer, and kernel times of one guided step
    a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tr.clear()
    a.record(stream)
    tr.render(samples, flags)
    c.record(stream)
    torch.cuda.synchronize()
    plain_ms = a.elapsed_time(c)
    tr.set_timing(True)
    step()
    tk = tr.timings()
    tr.set_timing(False)
    peak, peak_kind = _peaks()
    bpb = _traffic("k_bounce_bytes_per_path_bounce")
    achieved = cnt["path_bounces"] * BOUNCE_BYTES / (tk["bounce"][0] * 1e-3) / 1e9
    # e2e: scene and structures from host arrays, image back to host
    h_img = torch.empty((O_H, O_W, 3), dtype=torch.float32).pin_memory()
    h2d = sum(np.asarray(sc[k]).nbytes for k in ("tri_v", "tri_mat", "tri_uv", "light_tris"))
    e2e_ms, e2e_setup_ms = [], []
    # one untimed run first; each run's objects are released (and collected) outside the timed region
    for k in range(1 + max(1, args.steps // 2)):
        flush.fill_(k & 0xff)
        torch.cuda.synchronize()
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record(stream)
        tr2 = Tracer(sc, dev, max_depth=O_DEPTH, num_candidates=32, seed=1)
        g2 = HashGrid(*O_AABB, O_GRID_BOUNDS, O_SLOTS, keying=KEY_MORTON)
        q2 = MortonQuadTrees(O_SLOTS, level=O_LEVEL, fraction=0.3)
        c2 = MortonQuadTreeController(q2, O_BUDGET, iteration_for_built=1, ratio_for_budget=0.5)
        b.record(stream)
        step(tr2, g2, q2, c2)
        h_img.copy_(tr2.image(), non_blocking=True)
        c.record(stream)
        torch.cuda.synchronize()
        if k > 0:
            e2e_ms.append(a.elapsed_time(c))
            e2e_setup_ms.append(a.elapsed_time(b))
        del tr2, g2, q2, c2
        gc.collect()
        torch.cuda.synchronize()
    e2e = _max_over_ranks(sum(e2e_ms) / len(e2e_ms), world, dev)
    paths = O_W * O_H * samples * world
    return {
        "metric": "Mpaths/s", "value": paths / (ms * 1e-3) / 1e6, "unit": "Mpaths/s", "ms_per_step": ms,
        "e2e": {"value": paths / (e2e * 1e-3) / 1e6, "unit": "Mpaths/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(h_img.numel() * 4), "ms_per_step": e2e,
                "setup_ms": sum(e2e_setup_ms) / len(e2e_setup_ms),
                "note": "setup = scene upload, BVH build over the 1M triangles, tracer, hash grid and Morton "
                        "quadtree creation; the rest is the render and the image read-back"},
        "roofline": {"kernel": "k_bounce", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs (burst copy)",
                     "traffic": None if bpb is None else bpb * cnt["path_bounces"] / max(1, O_DEPTH * samples),
                     "algorithmic_bytes_per_path_bounce": BOUNCE_BYTES,
                     "kernel_ms_per_step": {kk: v[0] for kk, v in tk.items()},
                     "note": "bounce = BVH closest hit over 1M triangles + shading + RIS over 32 light samples + "
                             "one shadow ray; bound by traversal latency and issue"},
        "clocks": clk,
        "gpu_launches": ((1 + O_DEPTH + 1) * samples + _recording_launches(O_BUDGET, 1)) * args.steps,
        "counters_per_step": cnt,
        "unguided_nee_ris_Mpaths_s": O_W * O_H * samples / (plain_ms * 1e-3) / 1e6,
        "grid_cells": cells, "spp_per_step": samples,
    }


# ---------------------------------------------------------------------------- hash-grid workload
HG_POINTS = _HG_POINTS = 1 << 19    # surface points inserted into the grid (~380k distinct cells)
HG_QUERIES = _HG_QUERIES = 1 << 22  # lookups, Morton-leaf records and sample+pdf queries
HG_SLOTS = _HG_SLOTS = 1 << 20
HG_LEVEL = 4
HG_BOUNDS = (256, 64, 192)
HG_AABB = ((-0.005,) * 3, (14.005, 4.005, 10.005))
# algorithmic bytes per unit: lookup position 12 in + slot 4 out; record cell 4 + canonical
# direction 8 + value 4; sample cell 4 + seed 4 in, direction 12 + pdf 4 out
HG_LOOKUP_BYTES, HG_RECORD_BYTES, HG_SAMPLE_BYTES = 16, 16, 24


def _hg_cell_bytes(level=HG_LEVEL):
    """Algorithmic bytes of one cell's pyramid build: every int64 leaf read and zeroed (16 B)
    and every float of the (4^(L+1)-1)/3-entry pyramid written (4 B)."""
    return (1 << (2 * level)) * 16 + (((1 << (2 * (level + 1))) - 1) // 3) * 4


def bench_hashgrid_ours(args, rank, world):
    """The hash-grid guide's batched routines on the occluded-light scene's grid (2^20 slots,
    63-bit Morton keys, 256x64x192 cells): insert 2^19 surface points into the current table,
    snapshot it, look up 2^22 surface points, record 2^22 Morton-leaf values into the found
    cells, build the level-4 sampling pyramids of all 2^20 cells, and 2^22 guided
    sample+pdf queries.  One CUDA graph per phase."""
    import torch
    from rtlib_b200 import workloads as W
    from rtlib_b200.hashgrid import KEY_MORTON, HashGrid, MortonQuadTrees

    dev = torch.device("cuda", rank % max(1, torch.cuda.device_count()))
    torch.cuda.set_device(dev)
    # --scale-log2 k divides points, queries and slots by 2^k (small cases for profiling)
    HG_POINTS, HG_QUERIES, HG_SLOTS = (x >> args.scale_log2 for x in (_HG_POINTS, _HG_QUERIES, _HG_SLOTS))
    d = W.hashgrid_inputs(HG_POINTS, HG_QUERIES, 0)
    T = lambda a: torch.from_numpy(a).to(dev)
    pts, qpos, quv, qval, qseed = T(d["points"]), T(d["queries"]), T(d["uv"]), T(d["value"]), T(d["seeds"])
    slot_p = torch.empty(HG_POINTS, dtype=torch.int32, device=dev)
    slot_q = torch.empty(HG_QUERIES, dtype=torch.int32, device=dev)
    out_dir = torch.empty((HG_QUERIES, 3), dtype=torch.float32, device=dev)
    out_pdf = torch.empty(HG_QUERIES, dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    grid = HashGrid(*HG_AABB, HG_BOUNDS, HG_SLOTS, keying=KEY_MORTON)
    trees = MortonQuadTrees(HG_SLOTS, level=HG_LEVEL, fraction=0.3)

    def insert_part(p):
        grid.clear()
        grid.insert(p, slot_p)
        grid.swap()

    parts = [lambda: insert_part(pts), lambda: grid.lookup(qpos, slot_q),
             lambda: trees.record(slot_q, quv, qval, canonical=True), lambda: trees.update(),
             lambda: trees.sample_pdf(slot_q, qseed, out_dir=out_dir, out_pdf=out_pdf)]
    names = ["insert", "lookup", "record", "build", "sample_pdf"]
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(2):
            for f in parts:
                f()
    torch.cuda.current_stream().wait_stream(side)
    graphs = []
    for f in parts:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            f()
        graphs.append(g)
    stream = torch.cuda.current_stream()
    t0 = time.perf_counter()
    k = 0
    while k < args.warmup or time.perf_counter() - t0 < 0.5:
        for g in graphs:
            g.replay()
        k += 1
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(graphs) + 1)] for _ in range(args.steps)]
    clocks = ClockSampler(dev.index)
    _barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    for k in range(args.steps):
        flush.fill_(k & 0xff)
        ev[k][0].record(stream)
        for j, g in enumerate(graphs):
            g.replay()
            ev[k][j + 1].record(stream)
    torch.cuda.synchronize()
    _barrier(world)
    clk = clocks.stop()
    ph = {nm: statistics.mean(e[j].elapsed_time(e[j + 1]) for e in ev) for j, nm in enumerate(names)}
    ms = _max_over_ranks(statistics.mean(e[0].elapsed_time(e[-1]) for e in ev), world, dev)
    found = int((slot_q >= 0).sum().item())
    cells = int(torch.unique(slot_p).numel())
    grid_status = grid.status()  # RTPG_STATUS_HASH_FULL if a bucket of 32 overflowed
    assert trees.status() == 0

    # e2e: pinned host inputs through the same C-ABI calls, results read back, all timed
    hp = [torch.from_numpy(d[k]).pin_memory() for k in ("points", "queries", "uv", "value", "seeds")]
    dv = [pts, qpos, quv, qval, qseed]
    h_dir = torch.empty((HG_QUERIES, 3), dtype=torch.float32).pin_memory()
    h_pdf = torch.empty(HG_QUERIES, dtype=torch.float32).pin_memory()
    h2d = sum(x.numel() * x.element_size() for x in hp)
    d2h = (h_dir.numel() + h_pdf.numel()) * 4
    e2e_ms = []
    for k in range(args.warmup + args.steps):
        flush.fill_(k & 0xff)
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for x, y in zip(dv, hp):
            x.copy_(y, non_blocking=True)
        for f in parts:
            f()
        h_dir.copy_(out_dir, non_blocking=True)
        h_pdf.copy_(out_pdf, non_blocking=True)
        c.record(stream)
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e_ms.append(a.elapsed_time(c))
    e2e = _max_over_ranks(statistics.mean(e2e_ms), world, dev)
    ops = (HG_POINTS + 3 * HG_QUERIES) * world
    peak, peak_kind = _peaks()
    gbs = lambda b, t: b / (t * 1e-3) / 1e9
    build_bytes = HG_SLOTS * _hg_cell_bytes()
    achieved = gbs(build_bytes, ph["build"])
    return {
        "metric": "hash-grid guide insert+lookup+record+build+sample throughput (config-3 grid)",
        "value": ops / (ms * 1e-3) / 1e6, "unit": "Mops/s", "ms_per_step": ms,
        "e2e": {"value": ops / (e2e * 1e-3) / 1e6, "unit": "Mops/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {"kernel": "k_mqt_build", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs (burst copy)",
                     "traffic": _traffic("k_mqt_build"), "algorithmic_bytes_per_launch": build_bytes,
                     "launch_ms": ph["build"]},
        "clocks": clk,
        # clear 1 + insert (prepare, 2 sorts, heads, assign, scatter) + swap 1; lookup 1; record 1;
        # build 1; sample 1 (cub sorts counted as one launch each)
        "gpu_launches": 12 * args.steps,
        "phases": {"insert_Mpts_s": HG_POINTS / (ph["insert"] * 1e-3) / 1e6,
                   "lookup_Mq_s": HG_QUERIES / (ph["lookup"] * 1e-3) / 1e6,
                   "lookup_GBs": gbs(HG_LOOKUP_BYTES * HG_QUERIES, ph["lookup"]),
                   "record_Mrec_s": HG_QUERIES / (ph["record"] * 1e-3) / 1e6,
                   "record_GBs": gbs(HG_RECORD_BYTES * HG_QUERIES, ph["record"]),
                   "build_ms": ph["build"], "build_GBs": achieved,
                   "sample_pdf_Mq_s": HG_QUERIES / (ph["sample_pdf"] * 1e-3) / 1e6,
                   "sample_pdf_GBs": gbs(HG_SAMPLE_BYTES * HG_QUERIES, ph["sample_pdf"]),
                   "ms": ph},
        "grid_cells": cells, "queries_found": found, "grid_status": grid_status,
    }


def cpu_baseline_hashgrid(seconds=10.0, scale_log2=6):
    """RTLib's own hash grid and Morton quadtree code on the host, single thread (its routines
    are per-point device functions; the reference has no batched host path), on the workload
    scaled down by 2^scale_log2 with the table alike (the full workload's 2^19 points fall into
    373k distinct cells of 2^20 slots, load 0.36; scaled down nearly every point has a cell of
    its own, load 0.5), and RTLib's keying (its checksum covers this 256x64x192 grid).
    Returns the line's cpu_baseline."""
    from oracle.oracle import Reference
    from rtlib_b200 import workloads as W
    r = Reference()
    npts, nq, slots = HG_POINTS >> scale_log2, HG_QUERIES >> scale_log2, HG_SLOTS >> scale_log2
    d = W.hashgrid_inputs(npts, nq, 0)
    mn, mx = np.array(HG_AABB[0], np.float32), np.array(HG_AABB[1], np.float32)
    size = mx - mn
    per = ((1 << (2 * (6 + 1))) - 1) // 3  # RTLib's quadtree storage is sized for level 6
    times = []
    t_start = time.perf_counter()
    while not times or (time.perf_counter() - t_start < seconds and len(times) < 200):
        cur = np.zeros(slots, np.uint32)
        weights = np.zeros(slots * per, np.float32)
        t0 = time.perf_counter()
        r.hashgrid_insert(d["points"], mn, size, HG_BOUNDS, slots, cur)
        prv = cur.copy()
        cell = r.hashgrid_lookup(d["queries"], mn, size, HG_BOUNDS, slots, prv)
        r.mqt_record(HG_LEVEL, weights, cell, d["uv"], d["value"])
        r.mqt_build(slots, HG_LEVEL, weights)
        ok = cell != np.uint32(0xFFFFFFFF)
        r.mqt_sample_pdf(HG_LEVEL, weights, cell[ok], d["seeds"][ok])
        times.append(time.perf_counter() - t0)
    s = statistics.median(times)
    return {"value": (npts + 3 * nq) / s / 1e6, "unit": "Mops/s", "cores": 1, "kind": "reference",
            "sample": f"{len(times)} runs of the workload scaled by 1/{1 << scale_log2} ({npts} inserts, {nq} lookups, "
                      f"records and samples, {slots} slots), RTLib's own routines single-threaded",
            "seconds_per_run": s}


# ---------------------------------------------------------------------------- learned-guide workload
def _timed_render(fn, seconds):
    import torch
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < seconds:
        fn()
        torch.cuda.synchronize()
        n += 1
    return n


def bench_learned(args):
    """Equal-time comparison on the occluded-light scene (NEE + RIS, 32 candidates, max depth 16):
    plain SD-tree guiding against the learned guide with the SD-tree as its fallback (the same
    pass schedule; guide density half network, half SD-tree; network trained on the tracer's
    records after every pass) and against the network alone, relMSE against a long SD-tree
    render.  Wall-clock budgets include every training step; each method synchronises per
    launch."""
    import torch
    from rtlib_b200 import metrics, scenes
    from rtlib_b200.learned import render_learned, render_learned_with_fallback
    from rtlib_b200.mlp import MLPGuide
    from rtlib_b200.sdtree import SDTree, SDTreeController
    from rtlib_b200.tracer import FLAG_NEE, FLAG_RIS, Tracer

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    w, h = args.size
    sc = scenes.occluded_rooms(w, h)
    flags = FLAG_NEE | FLAG_RIS

    def sdtree_run(tr, seconds, fraction=0.5):
        tree = SDTree(*O_AABB, fraction=fraction)
        ctrl = SDTreeController(tree, 1 << 20, iteration_for_built=0, ratio_for_budget=0.5, samples_per_launch=1)
        ctrl.start()
        return _timed_render(lambda: tr.render_guided(tree, ctrl, flags, max_launches=1), seconds)

    warm = Tracer(sc, dev, max_depth=O_DEPTH, seed=5)
    sdtree_run(warm, 2.0)
    del warm
    # two independent reference renders (own seeds, own SD-trees) of half the reference time
    # each: their mean is the reference, their difference estimates its remaining variance
    refs, ref_spps = [], []
    for seed in (99, 98):
        ref_tr = Tracer(sc, dev, max_depth=O_DEPTH, seed=seed)
        ref_spps.append(sdtree_run(ref_tr, 0.5 * args.ref_seconds))
        refs.append(ref_tr.image().cpu().numpy())
        del ref_tr
    ref_spp = sum(ref_spps)

    def err(img):
        return metrics.relmse_denoised(img, refs[0], refs[1], ref_spps[0], ref_spps[1], normalize=True)

    out = []
    for budget in args.budgets:
        tr = Tracer(sc, dev, max_depth=O_DEPTH, seed=3)
        n_sd = sdtree_run(tr, budget)
        e_sd, d_sd = err(tr.image().cpu().numpy())
        del tr
        # the SD-tree with the learned arm's guide probability, for a like-for-like reading
        tr = Tracer(sc, dev, max_depth=O_DEPTH, seed=3)
        n_sd2 = sdtree_run(tr, budget, args.guide_fraction)
        e_sd2, d_sd2 = err(tr.image().cpu().numpy())
        del tr
        # the learned guide with the SD-tree as its fallback (the configuration the line reports)
        tr = Tracer(sc, dev, max_depth=O_DEPTH, seed=3)
        g = MLPGuide((-0.1, -0.1, -0.1), (14.1, 4.1, 10.1), seed=1, learning_rate=1e-3, record_capacity=1 << 18)
        tree = SDTree(*O_AABB, fraction=0.5)
        log, crit = [], []
        n_ml = render_learned_with_fallback(tr, g, tree, time_budget_s=budget, base_flags=flags,
                                            fraction=args.guide_fraction, mlp_share=0.5, epochs=args.epochs,
                                            batch=4096, log=log, criteria=crit)
        e_ml, d_ml = err(tr.image().cpu().numpy())
        st_ml = g.status()
        del tr, g, tree
        # the network alone (its own doubling schedule, no SD-tree)
        tr = Tracer(sc, dev, max_depth=O_DEPTH, seed=3)
        g = MLPGuide((-0.1, -0.1, -0.1), (14.1, 4.1, 10.1), seed=1, learning_rate=1e-3, record_capacity=1 << 18)
        n_mo = render_learned(tr, g, time_budget_s=budget, base_flags=flags, fraction=args.guide_fraction, ratio=0.5,
                              epochs=args.epochs, batch=4096)
        e_mo, d_mo = err(tr.image().cpu().numpy())
        del tr, g
        out.append({"budget_s": budget, "relmse_sdtree": e_sd, "relmse_learned": e_ml, "ratio": e_ml / e_sd,
                    "relmse_network_only": e_mo,
                    "denoised": {"relmse_sdtree": d_sd, "relmse_learned": d_ml, "relmse_network_only": d_mo,
                                 "ratio": d_ml / d_sd if d_sd > 0 else None,
                                 "relmse_sdtree_at_guide_fraction": d_sd2},
                    "relmse_sdtree_at_guide_fraction": e_sd2, "spp_sdtree_at_guide_fraction": n_sd2,
                    "spp_sdtree": n_sd, "spp_learned": n_ml, "spp_network_only": n_mo,
                    "train_log": log[-3:], "mlp_status": st_ml,
                    # per recording pass, on that pass's records before either guide is fitted to
                    # them: second moment of f / p with p = (1 - f_g) cos/pi + f_g q for each guide q
                    "second_moment_per_pass": crit})
    return {"budgets": out, "ref_spp": ref_spp, "ref_seconds": args.ref_seconds}


# ---------------------------------------------------------------------------- learned-guide kernels
# tensor-core FLOPs executed per sample (padding included): forward 2*(80*64 + 2*64*64 + 64*48);
# training adds dX of layers 3..1 (2*(48*64 + 2*64*64)) and dW^T of layers 3..0 at M = 64
# (2*(3*64*64 + 64*80))
MLP_FWD_FLOP = 2 * (80 * 64 + 2 * 64 * 64 + 64 * 48)
MLP_TRAIN_FLOP = MLP_FWD_FLOP + 2 * (48 * 64 + 2 * 64 * 64) + 2 * (3 * 64 * 64 + 64 * 80)
MLP_N_TRAIN, MLP_BATCH, MLP_N_EVAL = 1 << 18, 1 << 14, 1 << 20


def bench_mlp_ours(args, rank, world):
    """The learned guide's tcgen05 kernels: one training epoch over 2^18 records (16 Adam steps
    of 16384) and inference of 2^20 samples.  Metric: training records per second."""
    import torch
    from rtlib_b200.mlp import MLPGuide

    dev = torch.device("cuda", rank % max(1, torch.cuda.device_count()))
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(1)

    def unit(n):
        v = rng.normal(size=(n, 3)).astype(np.float32)
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    def T(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    n = MLP_N_TRAIN
    rec = (T(rng.uniform(0, 10, (n, 3)).astype(np.float32)), T(unit(n)), T(unit(n)), T(unit(n)),
           T(rng.lognormal(0, 1, n).astype(np.float32)))
    q = (T(rng.uniform(0, 10, (MLP_N_EVAL, 3)).astype(np.float32)), T(unit(MLP_N_EVAL)), T(unit(MLP_N_EVAL)))
    g = MLPGuide((0, 0, 0), (10, 10, 10), seed=1)
    out = torch.empty((MLP_N_EVAL, 40), dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        g.train(rec, batch=MLP_BATCH, epochs=1)
        g.eval(*q, raw=False)
    torch.cuda.synchronize()
    clocks = ClockSampler(dev.index)
    tr_ms, ev_ms = [], []
    _barrier(world)
    clocks.start()
    for k in range(args.steps):
        flush.fill_(k & 0xff)
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record(stream)
        g.train(rec, batch=MLP_BATCH, epochs=1)
        b.record(stream)
        g.eval(*q, raw=False)
        c.record(stream)
        torch.cuda.synchronize()
        tr_ms.append(a.elapsed_time(b))
        ev_ms.append(b.elapsed_time(c))
    _barrier(world)
    clk = clocks.stop()
    assert g.status() == 0
    t_ms = _max_over_ranks(sum(tr_ms) / len(tr_ms), world, dev)
    e_ms = sum(ev_ms) / len(ev_ms)
    # e2e: records from pinned host memory, the mixture of the queries back to host
    hrec = [x.cpu().pin_memory() for x in rec]
    hq = [x.cpu().pin_memory() for x in q]
    hout = torch.empty((MLP_N_EVAL, 40), dtype=torch.float32).pin_memory()
    e2e = []
    for k in range(max(1, args.steps // 2)):
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        drec = tuple(x.to(dev, non_blocking=True) for x in hrec)
        g.train(drec, batch=MLP_BATCH, epochs=1)
        dq = tuple(x.to(dev, non_blocking=True) for x in hq)
        hout.copy_(g.eval(*dq, raw=False), non_blocking=True)
        c.record(stream)
        torch.cuda.synchronize()
        e2e.append(a.elapsed_time(c))
    e2e_ms = _max_over_ranks(sum(e2e) / len(e2e), world, dev)
    peak = _peaks_tensor()
    achieved = MLP_TRAIN_FLOP * n / (t_ms * 1e-3) / 1e12
    steps = n // MLP_BATCH
    return {
        "metric": "learned-guide training throughput (records/s, 2^18 records, Adam steps of 16384)",
        "value": n * world / (t_ms * 1e-3) / 1e6, "unit": "Mrecords/s", "ms_per_step": t_ms,
        "e2e": {"value": n * world / (e2e_ms * 1e-3) / 1e6, "unit": "Mrecords/s",
                "h2d_bytes_per_step": int(sum(x.numel() * 4 for x in hrec + hq)),
                "d2h_bytes_per_step": int(hout.numel() * 4)},
        "roofline": {"kernel": "k_mlp_train", "bound": "tensor", "achieved": achieved, "peak": peak[0],
                     "unit": "TFLOP/s", "frac": achieved / peak[0], "peak_source": peak[1],
                     "traffic": None, "flop_per_record": MLP_TRAIN_FLOP,
                     "note": "64-wide layers: 128-row tiles of dependent tcgen05 MMAs, latency bound; the "
                             "step time includes the weight-sum and Adam kernels"},
        "inference": {"Msamples_s": MLP_N_EVAL / (e_ms * 1e-3) / 1e6, "ms": e_ms,
                      "tflops": MLP_FWD_FLOP * MLP_N_EVAL / (e_ms * 1e-3) / 1e12},
        "clocks": clk,
        "gpu_launches": (3 * steps + 1) * args.steps,
    }


def _peaks_tensor():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("bf16_tflops", 1590.0), "measured bf16_tflops (cuBLAS burst)"
    return 1590.0, "fallback bf16 TFLOP/s"


# ---------------------------------------------------------------------------- adjoint workload
def bench_adjoint(args):
    """Config 4: path-replay gradients of an L2 image loss w.r.t. a 256 x 256 albedo texture and
    16 emitter radiances at 512 x 512, 64 spp, against common-random-number central differences
    (eps 1e-3) on 512 texels and all emitters.  The value is the largest relative error of the
    checked gradients (those above 1 % of the largest, below which the difference itself is
    float noise); the line also carries the median, the relative error of the whole vector and
    the render rates."""
    import torch
    from rtlib_b200 import diff
    dev = torch.device("cuda", 0)
    clocks = ClockSampler(0)
    clocks.start()
    t0 = time.perf_counter()
    r = diff.config4_gradients(dev)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    adj = np.concatenate([r["adj_texels"], r["adj_lights"]]).astype(np.float64)
    fd = np.concatenate([r["fd_texels"], r["fd_lights"]])
    rel_all = []
    for a, f in ((r["adj_texels"], r["fd_texels"]), (r["adj_lights"], r["fd_lights"])):
        a, f = np.asarray(a, np.float64), np.asarray(f, np.float64)
        big = np.abs(f) > 1e-2 * np.abs(f).max()
        rel_all.append(np.abs(a[big] - f[big]) / np.abs(f[big]))
    rel = np.concatenate(rel_all)
    paths = r["paths_per_render"]
    return {"metric": "adjoint-vs-FD gradient relative error (max over checked gradients)", "value": float(rel.max()),
            "unit": "ratio", "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": wall * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "config 4: Cornell box 512x512, back-wall albedo texture 256x256 RGB, ceiling light "
                                   "as 4x4 emitters, L2 loss to a target with the texture perturbed N(0,0.05); "
                                   "forward and adjoint 64 spp, depth 8, NEE; CRN central differences eps 1e-3 on "
                                   "512 random texels (x3 channels) and all 16 emitters (x3)"},
            "median_rel_err": float(np.median(rel)), "checked": int(rel.size), "gradients": int(adj.size),
            "texel_rel_err_max": float(rel_all[0].max()), "emitter_rel_err_max": float(rel_all[1].max()),
            "vector_rel_err": float(np.linalg.norm(adj - fd) / np.linalg.norm(fd)),
            "forward_Mpaths_s": paths / (r["forward_ms"] * 1e-3) / 1e6,
            "adjoint_Mpaths_s": paths / (r["adjoint_ms"] * 1e-3) / 1e6,
            "note": "adjoint = one primal and one adjoint replay wave per sample", "clocks": clk}


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
    ap.add_argument("--workload", default="cornell", choices=["cornell", "sdtree", "hashgrid", "occluded", "learned",
                                                               "mlp", "adjoint"])
    ap.add_argument("--budgets", default="30,120", help="learned: equal-time budgets in seconds")
    ap.add_argument("--ref-seconds", type=float, default=300.0, help="learned: reference render time")
    ap.add_argument("--epochs", type=int, default=8, help="learned: Adam epochs over each pass's records")
    ap.add_argument("--guide-fraction", type=float, default=0.7,
                    help="learned: probability of sampling the guide (network / SD-tree mixture) at a vertex")
    ap.add_argument("--size", default="1280x720", help="learned: image size")
    ap.add_argument("--passes", type=int, default=1,
                    help="sdtree: record+build+refine passes before the queries (1 = the literal config; 2 = "
                         "the same records again into the refined topology)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sdtree-subrecord", action="store_true",
                    help="cornell: skip the config-1 SD-tree sub-record of the line")
    ap.add_argument("--scale-log2", type=int, default=0,
                    help="hashgrid: divide points, queries and slots by 2^k (small cases for profiling)")
    ap.add_argument("--budget", type=int, default=2047,
                    help="cornell: total spp of the pass schedule (2047 = passes 1..1024); smaller values "
                         "give the short case used for profiling")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    if args.workload == "learned":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the learned guide has no counterpart in RTLib; "
                              "it is compared with the SD-tree arm of the same run"}), flush=True)
            return 0
        if rank != 0:
            return 0
        args.budgets = [float(x) for x in args.budgets.split(",")]
        args.size = tuple(int(x) for x in args.size.split("x"))
        r = bench_learned(args)
        last = r["budgets"][-1]
        line = {"metric": "equal-time relMSE, learned guide (SD-tree fallback) / plain SD-tree guide (occluded scene)",
                "value": last["ratio"], "value_denoised": last["denoised"]["ratio"],
                "unit": "ratio", "n_gpus": 1, "steps": len(r["budgets"]), "warmup": args.warmup,
                "ms_per_step": last["budget_s"] * 1e3, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16 network / f32 tracer", "data": "synthetic",
                "config": {"workload": f"occluded-rooms {args.size[0]}x{args.size[1]}, NEE+RIS 32, depth 16; "
                                       f"equal wall-clock budgets {args.budgets} s; reference: two independent "
                                       f"SD-tree renders of {r['ref_seconds'] / 2} s each ({r['ref_spp']} spp in "
                                       f"all)", "relmse": "normalised by the reference mean, eps 1e-2; 'value' "
                                       "against the reference's mean, 'value_denoised' with the reference's own "
                                       "variance (from the difference of the two renders) removed",
                           "learned_arm": f"guide sampled with probability {args.guide_fraction}, density half network "
                                          f"half SD-tree, {args.epochs} Adam epochs per pass",
                           "sdtree_arm": "plain SD-tree guiding, BSDF/guide mixing 0.5"},
                "budgets": r["budgets"]}
        print(json.dumps(line), flush=True)
        return 0
    if args.workload == "adjoint":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "RTLib has no adjoint / differentiable renderer"}),
                      flush=True)
            return 0
        if rank != 0:
            return 0
        print(json.dumps(bench_adjoint(args)), flush=True)
        return 0
    if args.workload == "mlp" and args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the learned guide has no counterpart in RTLib"}),
                  flush=True)
        return 0
    if args.workload == "occluded" and args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "RTLib's integrator exists only as OptiX "
                              "programs and the CPU restatement intersects by brute force, which is not a "
                              "meaningful baseline over 1M triangles; see the cornell workload"}), flush=True)
        return 0
    cornell = args.workload == "cornell"
    occluded = args.workload == "occluded"
    mlp = args.workload == "mlp"
    hashgrid = args.workload == "hashgrid"
    set_budget(args.budget)
    if mlp:
        cfg = {"workload": "learned-guide kernels: 3x64 ReLU MLP -> 8 vMF lobes, BF16 tcgen05 / FP32 TMEM; "
                           "train 2^18 records (batch 16384, Adam), infer 2^20 samples"}
        metric, unit = "learned-guide training throughput", "Mrecords/s"
    elif occluded:
        cfg = {"workload": f"occluded-rooms HTRIS: {O_W}x{O_H}, ~1M triangles, 4096 emitters, NEE + RIS 32 "
                           f"candidates, max depth 16, hash grid 2^20 slots (Morton keys) + level-{O_LEVEL} "
                           f"Morton quadtrees, {O_BUDGET} spp budget", "width": O_W, "height": O_H, "max_depth": O_DEPTH}
        metric, unit = "Mpaths/s", "Mpaths/s"
    elif hashgrid:
        cfg = {"workload": "hashgrid-guide: occluded-scene grid 256x64x192, 2^20 slots, 63-bit Morton keys, "
                           "level-4 Morton quadtrees; insert 2^19 surface points, 2^22 lookups, records and "
                           "sample+pdf queries", "points": HG_POINTS >> args.scale_log2,
               "queries": HG_QUERIES >> args.scale_log2, "slots": HG_SLOTS >> args.scale_log2, "level": HG_LEVEL}
        if args.scale_log2:
            cfg["workload"] += f" (scaled down by 2^{args.scale_log2})"
        metric, unit = "hash-grid guide insert+lookup+record+build+sample throughput (config-3 grid)", "Mops/s"
    elif cornell:
        cfg = {"workload": f"cornell-guided: 512x512, {C_BUDGET} spp budget in doubling passes, max depth 8, NEE, "
                           "SD-tree guiding fraction 0.5", "width": C_W, "height": C_H, "spp": C_BUDGET + 1,
               "max_depth": C_MAX_DEPTH}
        metric, unit = "Mpaths/s", "Mpaths/s"
    else:
        cfg = {"workload": "sdtree-standalone: 2^20 records, refine at 12000*sqrt(2), 2^22 sample+pdf"
                           + (f" ({args.passes} record+refine passes)" if args.passes > 1 else ""),
               "records": N_REC, "queries": N_Q, "passes": args.passes}
        metric, unit = "SD-tree record+refine+sample throughput (config 1)", "Mops/s"

    if args.impl == "reference":
        if rank != 0:
            return 0
        cores = os.cpu_count() or 1
        if cornell:
            for _ in range(args.warmup):
                _cornell_cpu_step(cores)
            step_s, paths = [], 0
            for _ in range(args.steps):
                p, d = _cornell_cpu_step(cores)
                paths += p
                step_s.append(d)
            dt = sum(step_s)
            v = paths / dt / 1e6
            kind, threads = "port", cores
            sample = (f"each step: the same 512x512 guided render (NEE, depth 8, SD-tree fraction 0.5) over the pass "
                      f"schedule truncated at {C_REF_BUDGET} spp ({C_REF_BUDGET + 1} launches of passes 1, 2, 4, 8), "
                      f"every frame split into pixel bands over {cores} host threads recording into one shared "
                      f"SD-tree; CPU restatement of RTLib's integrator (its own exists only as OptiX programs); "
                      f"{paths} paths in {dt:.1f} s over {args.steps} steps")
            ms = dt * 1e3 / args.steps
            # the config-1 SD-tree sub-record of the default line, on RTLib's own code
            kind_s = _ref_kind()
            thr_s = cores if kind_s == "reference" else 1
            _ref_workload(kind_s, thr_s, reps=1)
            ph = []
            times_s = _ref_workload(kind_s, thr_s, reps=5, phases=ph)
            sec_s = sum(times_s) / len(times_s)
            sdtree_sub = {"metric": "SD-tree record+refine+sample throughput (config 1)",
                          "value": (N_REC + N_Q) / sec_s / 1e6, "unit": "Mops/s", "steps": len(times_s),
                          "ms_per_step": sec_s * 1e3,
                          "cpu_baseline": {"value": (N_REC + N_Q) / sec_s / 1e6, "unit": "Mops/s", "cores": thr_s,
                                           "kind": kind_s,
                                           "sample": "full config-1 passes (2^20 records, refine, 2^22 queries); "
                                                     "record/build/refine single-threaded as in RTLib, sample+pdf on "
                                                     f"{thr_s} thread(s)"},
                          "phases": {"record_Mrec_s": N_REC / statistics.median(p[0] for p in ph) / 1e6,
                                     "build_refine_ms": 1e3 * statistics.median(p[1] for p in ph),
                                     "sample_pdf_Mq_s": N_Q / statistics.median(p[2] for p in ph) / 1e6}}
        elif hashgrid:
            cpu_baseline_hashgrid(seconds=0.0)  # warm-up (pages in)
            cb = cpu_baseline_hashgrid(seconds=20.0)
            v, kind, threads, sample, ms = cb["value"], cb["kind"], cb["cores"], cb["sample"], cb["seconds_per_run"] * 1e3
        else:
            kind = _ref_kind()
            threads = cores if kind == "reference" else 1
            _ref_workload(kind, threads, reps=args.warmup)
            times = _ref_workload(kind, threads, reps=args.steps)
            sec = sum(times) / len(times)
            v = (N_REC + N_Q) / sec / 1e6
            ms = sec * 1e3
            sample = "full config-1 passes on the host"
        line = {"impl": "reference", "metric": metric, "value": v, "unit": unit, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
                "cpu_baseline": {"value": v, "unit": unit, "cores": threads, "kind": kind, "sample": sample},
                "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        if cornell and not args.no_sdtree_subrecord:
            line["sdtree_config1"] = sdtree_sub
        print(json.dumps(line), flush=True)
        return 0

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(_env_int("LOCAL_RANK", rank))
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    res = (bench_mlp_ours if mlp else bench_occluded_ours if occluded else bench_cornell_ours if cornell
           else bench_hashgrid_ours if hashgrid else bench_sdtree_ours)(args, rank, world)
    cfg["l2"] = "flushed (256 MiB write) before every timed step"
    cfg["parallelism"] = f"replicas x{world}"
    line = {"metric": res["metric"], "value": res["value"], "unit": res["unit"], "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": ("bf16" if mlp else "f32"),
            "data": "synthetic", "config": cfg, "e2e": res["e2e"], "roofline": res["roofline"],
            "clocks": res["clocks"], "gpu_launches": res["gpu_launches"]}
    for k in ("roofline_issue", "sdtree", "phases", "roofline_record", "counters_per_step", "unguided_nee_ris_Mpaths_s", "grid_cells", "spp_per_step",
              "inference", "queries_found", "grid_status"):
        if k in res:
            line[k] = res[k]
    if cornell and not args.no_sdtree_subrecord:
        # the north star's SD-tree target (config 1) measured in the same run
        line["sdtree_config1"] = sdtree_subrecord(args, rank, world)
    if rank == 0 and not args.no_cpu_baseline and not occluded and not mlp:
        if cornell:
            cores = os.cpu_count() or 1
            v, dt, paths, n = _cornell_cpu(cores, 10.0)
            line["cpu_baseline"] = {"value": v, "unit": "Mpaths/s", "cores": cores, "kind": "port",
                                    "sample": f"{n} x the same 512x512 guided render over the pass schedule truncated "
                                              f"at {C_REF_BUDGET} spp, pixel bands over {cores} host threads into one "
                                              f"shared SD-tree, CPU restatement of the integrator; {paths} paths in "
                                              f"{dt:.1f} s"}
        elif hashgrid:
            line["cpu_baseline"] = cpu_baseline_hashgrid()
        else:
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
