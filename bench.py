#!/usr/bin/env python3
"""Benchmark: 6F5 zeta delta search, N = 1000, verified trajectories per second.

Workload (one "step" = one walk of the whole batch): 6F5 at the zeta point
(x = 1^6, y = 2^5), z = 1, rank 5, 10,000 directions over the 11 axes with
components uniform in 0..3, not all zero (std::mt19937_64, seeded), N = 1000,
h = 50, walked in f64 on the GPU. After the timed region every valid result
is checked against the exact walk (rational residues modulo up to 4096
primes, CRT and rational reconstruction); a trajectory is *verified* when its
limit is within 1e-10 relative of the exact value of the same estimator.

value = verified trajectories per second of walk-kernel time (whole job:
sum over ranks / max over ranks). e2e = the same through cmfw_walk_host with
pinned host records (copies in the timed region). Under torchrun each rank
walks its own seeded batch (weak scaling; no collective on the data path,
one small gather of counters at the end).

--impl reference times the reference's own kernel bodies compiled for the
host (oracle/_ref, OpenMP over all host cores) on the same batch and
verifies them with the oracle alone (the estimator of each limit from the
oracle's restatement of the reference's reduction, exact values from the
oracle's exact walk modulo primes); it loads nothing of the product.

The default line also carries the per-result error distribution
(`accuracy`), the plain one-thread-per-trajectory kernels on the same batch
(`plain`: this project's sequential kernel and the reference's own
walk_kernel_f64 built for sm_100a), and the chunked walk on 2,000
directions whose walks stay valid (`valid_directions`, with its roofline).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "ramanujandreams-cuda_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "6F5 N=1000 verified traj/s on 1 B200 at <=1e-10 vs RNS"
P, Q, Z, N, H, NTRAJ = 6, 5, 1.0, 1000, 50, 10000
SEED = 20261203
RTOL = 1e-10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cmfw", choices=["cmfw", "reference"])
    ap.add_argument("--variant", default="f64", choices=["f64", "df64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="leave out the plain-kernel comparison and the valid-direction workload")
    ap.add_argument("--workload", default="zeta6f5",
                    choices=["zeta6f5", "zeta6f5_valid", "limit3f2", "rns8f7", "mixed", "proposal"],
                    help="zeta6f5: the headline 6F5 delta search; zeta6f5_valid: the same search restricted to "
                         "--valid-n directions whose walks stay valid (non-degenerate work); limit3f2: "
                         "3F2 z=1/2 limit walks from 10,000 starts U{1..10}, direction 1^5 (the CPU-baseline "
                         "configuration); rns8f7: the 8F7 zeta RNS walk (dirs 1^15 + U{0..2}^15) at N 1000 "
                         "and 4000 with 8 and 16 moduli, beside the reference's own RNS kernel; mixed: the "
                         "mixed-family batch "
                         "(10^6 trajectories, N log-uniform 200..5000) in one graph launch; proposal: the "
                         "learned proposal for the 8F7 zeta delta search against the exhaustive sweep")
    ap.add_argument("--mixed-n", type=int, default=1000000)
    ap.add_argument("--valid-n", type=int, default=2000, help="zeta6f5_valid: directions")
    ap.add_argument("--verify-max", type=int, default=600,
                    help="reference arm: valid rows verified by the host exact walk at most (a seeded sample beyond)")
    ap.add_argument("--search-n", type=float, default=1e8, help="proposal: candidates searched")
    ap.add_argument("--train-n", type=float, default=1e8,
                    help="proposal: candidates whose filter survivors are walked for training")
    ap.add_argument("--fraction", type=float, default=0.05, help="proposal: share of the survivors walked")
    ap.add_argument("--epochs", type=int, default=30, help="proposal: training epochs")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def select_family(args):
    """The walk family of the workload: module-wide P, Q, Z and METRIC."""
    global P, Q, Z, METRIC
    if args.workload == "limit3f2":
        P, Q, Z = 3, 2, 0.5
        METRIC = "3F2 z=1/2 N=1000 verified traj/s on 1 B200 at <=1e-10 vs exact"


def workload(rank, args=None):
    import cmfw.workloads as wl
    if args is not None and args.workload == "limit3f2":
        return wl.limit_starts(3, 2, NTRAJ, SEED + rank)
    if args is not None and args.workload == "zeta6f5_valid":
        return wl.valid_directions(P, Q, args.valid_n, SEED + rank, z=Z, N=N, h=H)
    return wl.zeta_directions(P, Q, NTRAJ, SEED + rank)


WORKLOAD_TEXT = {
    "zeta6f5": "6F5 zeta delta search: x=1^6, y=2^5, z=1, rank 5, dirs U{0..3}^11 != 0, N=1000, h=50",
    "zeta6f5_valid": "6F5 zeta delta search restricted to directions whose walk stays valid (seeded rejection "
                     "sampling of dirs U{0..3}^11 != 0), x=1^6, y=2^5, z=1, rank 5, N=1000, h=50",
    "limit3f2": "3F2 limit walks: z=1/2, rank 3, 10,000 starts x1..x3, y1..y2 U{1..10}, direction 1^5, "
                "N=1000, h=50",
}


def walk_flops(p, q, dim, records, Ns, valid):
    """Algorithmic flops of valid walks (same count as flops_per_traj) for
    descriptor (p, q, dim) with per-trajectory depths Ns."""
    f_col = 1.5 * p * (p + 1) + 1.5 * q * (q + 1) + p + q + 2
    f_fwd, f_inv, f_norm = 4 * dim * dim, dim * (9 * dim + 1), dim * dim
    d = records["dir"][:, :p + q].astype(np.int64)
    fwd = np.where(d[:, :p] > 0, d[:, :p], 0).sum(1) + np.where(d[:, p:] < 0, -d[:, p:], 0).sum(1)
    inv = np.where(d[:, :p] < 0, -d[:, :p], 0).sum(1) + np.where(d[:, p:] > 0, d[:, p:], 0).sum(1)
    per = np.asarray(Ns, np.float64) * (fwd * (f_col + f_norm + f_fwd) + inv * (f_col + f_norm + f_inv))
    return float(per[valid].sum())


def flops_per_traj(records, valid, dim):
    """Algorithmic flops of a valid walk, by the per-axis-step count of the
    reference update (FMA = 2): column 1.5p(p+1) + 1.5q(q+1) + p + q + 2,
    forward update 4 dim^2, inverse update dim (9 dim + 1), normalisation
    dim^2; x+ and y- steps are forward, x- and y+ inverse."""
    f_col = 1.5 * P * (P + 1) + 1.5 * Q * (Q + 1) + P + Q + 2
    f_fwd, f_inv, f_norm = 4 * dim * dim, dim * (9 * dim + 1), dim * dim
    d = records["dir"][:, :P + Q].astype(np.int64)
    fwd = np.where(d[:, :P] > 0, d[:, :P], 0).sum(1) + np.where(d[:, P:] < 0, -d[:, P:], 0).sum(1)
    inv = np.where(d[:, :P] < 0, -d[:, :P], 0).sum(1) + np.where(d[:, P:] > 0, d[:, P:], 0).sum(1)
    per = N * (fwd * (f_col + f_norm + f_fwd) + inv * (f_col + f_norm + f_inv))
    return float(per[valid].sum())


class Clocks:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def ncu_traffic():
    """DRAM bytes per launch of the walk kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "walk_f64_6F5_zeta_delta.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f).get("dram_bytes_per_launch")


def cpu_reference(records, threads, budget_s=8.0, max_passes=20):
    """Time the reference f64 kernel bodies (host build) on the batch."""
    import oracle
    kind = "reference" if oracle.have_ref("f64") else "port"
    run = (lambda: oracle.ref_walk("f64", P, Q, Z, N, H, records, threads=threads)) if kind == "reference" \
        else (lambda: oracle.walk("f64", P, Q, Z, N, H, records, threads=threads))
    out = run()  # warm
    times = []
    t_all = time.perf_counter()
    while len(times) < max_passes and (time.perf_counter() - t_all) < budget_s:
        t0 = time.perf_counter()
        out = run()
        times.append(time.perf_counter() - t0)
    return kind, out, times


def reference_sources(records, ref_out, threads, fused=False, require_match=True):
    """The estimator behind each of the reference's limits (ratio and
    method, as cmfw's limit_src), from the oracle's restatement of the
    reference's reduction. With require_match (the reference's host build,
    which the oracle reproduces bit for bit) a row keeps it only where the
    oracle's limit equals the reference's; other rows get -1 (unattributed,
    never verified). Without (the reference's GPU build, whose FMA
    contraction rounds differently), every valid row takes the oracle's
    choice. Returns the sources and the number of rows whose limits differ."""
    import oracle
    o_out, src = oracle.walk_f64_src(P, Q, Z, N, H, records, fused=fused, threads=threads)
    a, b = np.asarray(ref_out["limit"]), np.asarray(o_out["limit"])
    with np.errstate(invalid="ignore"):
        same = (a == b) | (np.isnan(a) & np.isnan(b))
    same &= np.asarray(ref_out["valid"]) == np.asarray(o_out["valid"])
    valid = np.asarray(ref_out["valid"]) == 1
    keep = same if require_match else valid
    return np.where(keep, src, -1).astype(np.int32), int((valid & ~same).sum())


def accuracy(rel_err, floor, valid):
    """Per-result error against the exact value of each result's own
    estimator: counts within 1e-13, 1e-11 and 1e-10, each beside the number
    of results whose estimator's rounding floor (the error double-precision
    ratios alone leave) is within the same bound, and the rows."""
    idx = np.nonzero(valid)[0]
    rel = np.asarray(rel_err)[idx]
    fl = np.asarray(floor)[idx] if floor is not None else np.full(len(idx), np.nan)
    out = {"valid": int(len(idx)), "comparable": int(np.isfinite(rel).sum()), "within": {}}
    if floor is not None:
        out["floor_within"] = {}
    for b in (1e-13, 1e-11, 1e-10):
        with np.errstate(invalid="ignore"):
            out["within"][f"{b:.0e}"] = int((rel <= b).sum())
            if floor is not None:
                out["floor_within"][f"{b:.0e}"] = int((fl <= b).sum())
    out["rows"] = [[int(t), None if not np.isfinite(r) else float(f"{r:.3e}"),
                    None if not np.isfinite(f) else float(f"{f:.3e}")] for t, r, f in zip(idx, rel, fl)]
    return out


def verify_counts(desc, records, results, limit_src):
    from cmfw import exact
    v = exact.verify(desc, records, results, limit_src, N, H, rtol=RTOL)
    ok = v["verified"]
    deltas = results["delta"][ok]
    deltas = deltas[np.isfinite(deltas)]
    return int(ok.sum()), v, (float(deltas.max()) if deltas.size else None)


def time_events(fn, steps, flush):
    """Mean device time (s) of fn() over `steps` calls, CUDA events on the
    current stream, L2 flushed before each."""
    import torch
    ms = []
    for k in range(steps):
        flush.fill_(k & 0xff)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return float(np.mean(ms)) / 1e3


def plain_kernels(desc, records, d_in, flush, steps):
    """The one-thread-per-trajectory f64 walks on the same batch: this
    project's sequential kernel (CMFW_F_SEQUENTIAL) and the reference's own
    walk_kernel_f64 built unchanged for sm_100a (oracle/_ref), each with its
    verified count -- the plain kernels the chunked walk is measured
    against -- and the chunked walk with plain FP64 runs."""
    import torch
    import cmfw
    import oracle
    n = len(records)
    out = {}
    d_out = cmfw.out_buffer(n)
    d_src = torch.empty(n, dtype=torch.int32, device="cuda")
    seq = lambda: cmfw.launch_walk("f64", desc, d_in, d_out, n, N, H, flags=cmfw.F_SEQUENTIAL, d_limit_src=d_src)
    seq()
    torch.cuda.synchronize()
    t = time_events(seq, steps, flush)
    res = cmfw.records_from_device(d_out, n)
    nv, _, _ = verify_counts(desc, records, res, d_src.cpu().numpy())
    out["cmfw_sequential"] = {"ms_per_step": t * 1e3, "n_verified": nv, "verified_traj_per_s": nv / t,
                              "kernel": "walk_float_kernel (one thread per trajectory)"}
    # the chunked walk with plain FP64 runs (CMFW_F_PLAIN_RUNS): the speed the
    # double-double runs give up for their accuracy
    pr = lambda: cmfw.launch_walk("f64", desc, d_in, d_out, n, N, H, flags=cmfw.F_PLAIN_RUNS, d_limit_src=d_src)
    for _ in range(3):
        pr()
    torch.cuda.synchronize()
    t = time_events(pr, steps, flush)
    res = cmfw.records_from_device(d_out, n)
    nv, _, _ = verify_counts(desc, records, res, d_src.cpu().numpy())
    out["cmfw_chunked_fp64_runs"] = {"ms_per_step": t * 1e3, "n_verified": nv, "verified_traj_per_s": nv / t,
                                     "kernel": "walk_chunk_kernel<..., ArithF64> (plain FP64 runs and tree)"}
    if oracle.have_ref_gpu("f64"):
        d_ref = torch.empty((n, 64), dtype=torch.uint8, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        ref = lambda: oracle.ref_gpu_launch("f64", P, Q, Z, N, H, d_in.data_ptr(), d_ref.data_ptr(), n,
                                            stream=stream)
        ref()
        torch.cuda.synchronize()
        t = time_events(ref, steps, flush)
        rout = d_ref.cpu().numpy().reshape(-1).view(oracle.OUT_F64_DTYPE)
        src, differ = reference_sources(records, rout, 0, fused=True, require_match=False)
        nv, _, _ = verify_counts(desc, records, rout, src)
        out["reference_sm100a"] = {"ms_per_step": t * 1e3, "n_verified": nv, "verified_traj_per_s": nv / t,
                                   "n_valid": int((rout["valid"] == 1).sum()),
                                   "rows_limit_differs_from_host_build": differ,
                                   "kernel": "walk_kernel_f64 (cuda/cmf_walk_f64.cu:94-154), nvcc -O3 sm_100a, "
                                             "block 256"}
    else:
        out["reference_sm100a"] = {"unavailable": "oracle/_ref/libref_gpu_f64.so not built"}
    return out


def valid_direction_run(desc, flush, steps, n=2000):
    """The chunked walk on non-degenerate work: n directions of the headline
    search (seeded rejection sampling, only those whose walk stays valid),
    same N and h; verified count and the FP64-pipe roofline there."""
    import torch
    import cmfw
    import cmfw.workloads as wl
    t0 = time.perf_counter()
    recs = wl.valid_directions(P, Q, n, SEED, z=Z, N=N, h=H)
    t_gen = time.perf_counter() - t0
    d_in = cmfw.to_device(recs)
    d_out = cmfw.out_buffer(n)
    d_src = torch.empty(n, dtype=torch.int32, device="cuda")
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in kev:  # record once so that the events exist
        a.record()
        b.record()
    done = []

    def step(timed=False):
        ev = kev[len(done)] if timed else None
        cmfw.launch_walk("f64", desc, d_in, d_out, n, N, H, d_limit_src=d_src, main_events=ev)
        if timed:
            done.append(ev)

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    t = time_events(step, steps, flush)
    # the chunk kernel alone, from the events the library records around it
    # (a second pass: an event between the two kernels delays the second)
    time_events(lambda: step(True), steps, flush)
    t_kernel = float(np.mean([a.elapsed_time(b) for a, b in done])) / 1e3
    res = cmfw.records_from_device(d_out, n)
    valid = res["valid"] == 1
    t0 = time.perf_counter()
    nv, v, _ = verify_counts(desc, recs, res, d_src.cpu().numpy())
    t_ver = time.perf_counter() - t0
    flops = flops_per_traj(recs, valid, desc.rank)
    return {"workload": f"{n} valid directions of the 6F5 zeta search (rejection-sampled, seed {SEED}), "
                        "N=1000, h=50", "ms_per_step": t * 1e3, "n_valid": int(valid.sum()), "n_verified": nv,
            "verified_traj_per_s": nv / t, "traj_per_s": n / t, "flops_per_launch": flops,
            "kernel_ms_per_launch": t_kernel * 1e3, "achieved_tflops": flops / t_kernel / 1e12,
            "accuracy": accuracy(v["rel_err"], v["floor"], valid),
            "generate_s": t_gen, "verify_s": t_ver}


def gather_sum(x, world):
    if world == 1:
        return [x]
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, x)
    return out


def main_cmfw(args):
    import torch
    import cmfw

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    records = workload(rank, args)
    desc = cmfw.make_desc(P, Q, Z)
    n = len(records)
    d_in = cmfw.to_device(records)
    d_out = cmfw.out_buffer(n)
    d_src = torch.empty(n, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    # the dominant kernel's own duration (the chunk kernel): the library
    # records these events around it on the launch stream, in a second pass
    # of the same steps after the timed one (an event between the filter and
    # the chunk kernel ends the chunk kernel's programmatic early launch, 9 us
    # a step, so the timed steps go without them)
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    for a, b in kev:  # record once so that the events exist
        a.record()
        b.record()

    def step(k=None):
        cmfw.launch_walk(args.variant, desc, d_in, d_out, n, N, H, d_limit_src=d_src,
                         main_events=kev[k] if k is not None else None)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.4)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for k in range(args.steps):
        flush.fill_(k & 0xff)  # evict the batch from L2 between steps
        ev[k][0].record()
        step()
        ev[k][1].record()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_step = float(np.mean(step_ms)) / 1e3
    for k in range(args.steps):
        flush.fill_(k & 0xff)
        step(k)
    torch.cuda.synchronize()
    t_kernel = float(np.mean([a.elapsed_time(b) for a, b in kev])) / 1e3

    results = cmfw.records_from_device(d_out, n)
    src = d_src.cpu().numpy()
    n_valid = int((results["valid"] == 1).sum())
    n_ver, vinfo, best_delta = verify_counts(desc, records, results, src)
    errs = vinfo["rel_err"][vinfo["verified"]]

    # end to end through the host-buffer C ABI, pinned records
    pin_in = torch.from_numpy(records.view(np.uint8)).pin_memory()
    pin_out = torch.empty(n * cmfw.OUT_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
    import ctypes
    L = cmfw.lib()
    launch = cmfw._lib.Launch()
    kms, tms = ctypes.c_float(0), ctypes.c_float(0)

    def e2e_step():
        cmfw._lib.check(L.cmfw_walk_host(cmfw._lib.VARIANTS[args.variant], ctypes.byref(desc),
                                         ctypes.c_void_p(pin_in.data_ptr()),
                                         ctypes.c_void_p(pin_out.data_ptr()), n, N, H, 8,
                                         ctypes.byref(launch), ctypes.byref(kms), ctypes.byref(tms)))

    # host wall clock is noisier than device events: average over at least
    # 50 calls (each a full step: copies in, walk, results out)
    for _ in range(3):
        e2e_step()
    e2e_calls = max(args.steps, 50)
    e2e_ms = []
    # the exact verification above leaves a large heap of Python integers:
    # collect it first and keep the collector out of the timed calls (as
    # timeit does)
    import gc
    gc.collect()
    gc.disable()
    try:
        for k in range(e2e_calls):
            flush.fill_(k & 0xff)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e2e_step()
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
    finally:
        gc.enable()
    e2e_out = pin_out.numpy().view(cmfw.OUT_DTYPE)
    assert (e2e_out["valid"] == results["valid"]).all()
    t_e2e = float(np.mean(e2e_ms)) / 1e3

    # roofline: FP64 pipe
    flops = flops_per_traj(records, results["valid"] == 1, desc.rank)
    peak_fp64 = cmfw.pipe_peak(0)

    per_rank = gather_sum({"n_ver": n_ver, "t": t_step, "t_e2e": t_e2e, "n_valid": n_valid}, world)
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    total_ver = sum(r["n_ver"] for r in per_rank)
    t_max = max(r["t"] for r in per_rank)
    t_e2e_max = max(r["t_e2e"] for r in per_rank)
    value = total_ver / t_max
    achieved = flops / t_kernel / 1e12
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "verified traj/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_max * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": args.variant,
        "data": "synthetic (seeded std::mt19937_64 directions; no dataset)",
        "config": {"workload": WORKLOAD_TEXT[args.workload],
                   "n_traj_per_gpu": n, "seed": SEED, "variant": args.variant,
                   "l2": "flushed between steps (256 MiB write outside the timed events)",
                   "verification": f"exact rational walk (RNS, CRT + rational reconstruction), rtol {RTOL}"},
        "n_traj": n * world,
        "n_valid": sum(r["n_valid"] for r in per_rank),
        "n_verified": total_ver,
        "traj_per_s": n * world / t_max,
        "max_rel_err_verified": float(errs.max()) if errs.size else None,
        "exact_primes_max": int(vinfo["K"].max()) if len(vinfo["K"]) else 0,
        "best_delta": best_delta,
        "best_delta_per_gpu_s": (best_delta / (t_max * world)) if best_delta is not None else None,
        "gpu_launches": 2 * args.steps,  # prefix + chunk kernel per step
        "e2e": {"value": total_ver / t_e2e_max, "unit": "verified traj/s",
                "h2d_bytes_per_step": n * 192, "d2h_bytes_per_step": n * 56, "calls": e2e_calls},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak_fp64, "unit": "TFLOP/s",
                     "frac": achieved / peak_fp64 if peak_fp64 else None,
                     "peak_source": "in-run FP64 FMA probe (cmfw_pipe_peak); MEASURED_PEAKS.json has no FP64 figure",
                     "kernel": "walk_chunk_kernel (CUDA events around it on its stream, a second pass of the "
                               "timed steps)",
                     "kernel_ms_per_launch": t_kernel * 1e3,
                     "frac_of_whole_step": flops / t_step / 1e12 / peak_fp64 if peak_fp64 else None,
                     "flops_per_launch": flops,
                     "traffic": ncu_traffic()},
        "clocks": clk,
    }
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        kind, cpu_out, times = cpu_reference(records, threads)
        cpu_src, _ = reference_sources(records, cpu_out, threads)
        cpu_ver, _, _ = verify_counts(desc, records, cpu_out, cpu_src)
        t_cpu = float(np.mean(times))
        line["cpu_baseline"] = {"value": cpu_ver / t_cpu, "unit": "verified traj/s", "cores": threads,
                                "kind": kind,
                                "sample": f"the full batch ({n} trajectories) x {len(times)} passes, "
                                          f"{t_cpu * 1e3:.1f} ms per pass",
                                "verification": "estimator of each limit from the oracle's restatement of the "
                                                "reference's reduction, exact values from the GPU exact walk"}
    line["accuracy"] = accuracy(vinfo["rel_err"], vinfo["floor"], results["valid"] == 1)
    if world == 1 and not args.no_extras and args.workload == "zeta6f5":
        plain = plain_kernels(desc, records, d_in, flush, 3)
        ref = plain.get("reference_sm100a", {})
        if ref.get("verified_traj_per_s"):
            plain["chunked_vs_reference_sm100a"] = value / ref["verified_traj_per_s"]
        if plain["cmfw_sequential"]["verified_traj_per_s"]:
            plain["chunked_vs_cmfw_sequential"] = value / plain["cmfw_sequential"]["verified_traj_per_s"]
        line["plain"] = plain
        vd = valid_direction_run(desc, flush, args.steps)
        vd["roofline"] = {"bound": "fp64", "achieved": vd["achieved_tflops"], "peak": peak_fp64, "unit": "TFLOP/s",
                          "frac": vd["achieved_tflops"] / peak_fp64 if peak_fp64 else None}
        line["valid_directions"] = vd
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main_reference(args):
    """The reference's own CPU path on the same batch (oracle/_ref: its
    kernel bodies compiled for the host, OpenMP over all host cores), verified
    by the oracle alone: the estimator of each limit from the oracle's
    restatement of the reference's reduction, the exact values from the
    oracle's exact walk modulo primes. Nothing of the product is loaded."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    records = workload(0, args)
    import oracle
    from oracle import exact_check
    threads = os.cpu_count() or 1
    kind = "reference" if oracle.have_ref("f64") else "port"
    run = (lambda: oracle.ref_walk("f64", P, Q, Z, N, H, records, threads=threads)) if kind == "reference" \
        else (lambda: oracle.walk("f64", P, Q, Z, N, H, records, threads=threads))
    for _ in range(args.warmup):
        run()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        out = run()
        times.append(time.perf_counter() - t0)
    t = float(np.mean(times))
    src, unattributed = reference_sources(records, out, threads)
    valid = out["valid"] == 1
    # the oracle's exact walk runs on the host: beyond verify_max valid rows
    # a seeded sample of them is verified and the count scaled
    rows = np.nonzero(valid & (src >= 0))[0]
    sample = rows
    if len(rows) > args.verify_max:
        sample = np.sort(np.random.default_rng(SEED).choice(rows, args.verify_max, replace=False))
    t0 = time.perf_counter()
    v = exact_check.verify(P, Q, Z, records[sample], out[sample], src[sample], N, H, rtol=RTOL, threads=threads)
    t_ver = time.perf_counter() - t0
    n_ver_sample = int(v["verified"].sum())
    n_ver = n_ver_sample if len(sample) == len(rows) else n_ver_sample * len(rows) / len(sample)
    value = n_ver / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "verified traj/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded std::mt19937_64 directions; no dataset)",
        "config": {"workload": WORKLOAD_TEXT.get(args.workload, args.workload), "n_traj_per_gpu": len(records),
                   "seed": SEED, "variant": "f64",
                   "verification": f"oracle exact walk modulo primes (CRT + rational reconstruction), rtol {RTOL}, "
                                   "estimator of each limit from the oracle's restatement of the reference's "
                                   "reduction"},
        "n_traj": len(records), "n_valid": int(valid.sum()), "n_verified": n_ver, "unattributed_rows": unattributed,
        "verified_sample": {"rows": int(len(sample)), "verified": n_ver_sample,
                            "of": int(len(rows)), "scaled": bool(len(sample) < len(rows))},
        "traj_per_s": len(records) / t, "verify_s": t_ver,
        "accuracy": accuracy(v["rel_err"], None, np.ones(len(sample), bool)),
        "cpu_baseline": {"value": value, "unit": "verified traj/s", "cores": threads, "kind": kind,
                         "sample": f"the full batch ({len(records)} trajectories) per step"},
        "e2e": {"value": value, "unit": "verified traj/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main_rns(args):
    """8F7 at the zeta point (x = 1^8, y = 2^7, z = 1, rank 7), 10,000
    directions 1^15 + U{0..2}^15 (seeded), limit mode, the compat RNS walk
    (the reference's cmf_walk_rns semantics: 30-bit moduli, rounded column,
    2-modulus CRT every 100 steps) at N = 1000 and 4000 with 8 and 16
    moduli. Per configuration: traj/s of this project's kernel (CUDA events,
    L2 flushed), the valid count and bit-exactness of limit, p and q against
    the oracle on up to 64 valid rows; at N = 1000 with 8 moduli also the
    reference's own walk_kernel_rns built for sm_100a on the same buffers
    (one timed launch) and the exact ratios of up to 4 valid walks (exact
    walk + device reconstruction)."""
    import torch
    import cmfw
    import cmfw.workloads as wl
    import oracle
    from cmfw import exact
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if rank != 0:
        return
    p, q, z, n = 8, 7, 1.0, NTRAJ
    recs = wl.zeta_directions(p, q, n, SEED, lo=0, hi=2, offset=1)
    desc = cmfw.make_desc(p, q, z)
    d_in = cmfw.to_device(recs)
    d_out = cmfw.out_buffer(n)
    d_ref = torch.empty((n, 56), dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    res = {}
    for Nd in (1000, 4000):
        for K in (8, 16):
            mine = lambda: cmfw.launch_walk("rns", desc, d_in, d_out, n, Nd, H, n_primes=K)
            for _ in range(max(args.warmup, 1)):
                mine()
            torch.cuda.synchronize()
            t = time_events(mine, args.steps, flush)
            g = cmfw.records_from_device(d_out, n)
            m = np.nonzero(g["valid"] == 1)[0]
            mc = m[:64]  # the oracle (host) checks up to 64 valid rows
            o = oracle.walk("rns", p, q, z, Nd, H, recs[mc], n_primes=K, fused=True)
            bitexact = all(np.array_equal(g[k][mc], o[k], equal_nan=True) for k in ("limit", "p", "q")) and \
                (o["valid"] == 1).all()
            entry = {"ms_per_step": t * 1e3, "traj_per_s": n / t, "n_valid": int(len(m)),
                     "bit_exact_vs_oracle": bool(bitexact), "oracle_checked_rows": int(len(mc))}
            if oracle.have_ref_gpu("rns") and Nd == 1000 and K == 8:
                # the reference kernel takes tens of seconds per launch (one thread per
                # trajectory, 64-bit modular products): one timed launch, here only
                ref = lambda: oracle.ref_gpu_launch("rns", p, q, z, Nd, H, d_in.data_ptr(), d_ref.data_ptr(), n,
                                                    stream=stream, n_primes=K)
                tr = time_events(ref, 1, flush)
                rout = d_ref.cpu().numpy().reshape(-1).view(cmfw.OUT_DTYPE)
                lim_a, lim_b = rout["limit"][m], g["limit"][m]
                fin = np.isfinite(lim_a) & np.isfinite(lim_b)
                rel = np.abs(lim_a[fin] - lim_b[fin]) / np.maximum(np.abs(lim_b[fin]), 1e-300)
                entry["reference_sm100a"] = {
                    "ms_per_step": tr * 1e3, "traj_per_s": n / tr, "timed_launches": 1,
                    "same_valid": bool(np.array_equal(rout["valid"], g["valid"])),
                    "same_pq": bool(all(np.array_equal(rout[k][m], g[k][m], equal_nan=True) for k in ("p", "q"))),
                    "same_limit": bool(np.array_equal(lim_a, lim_b, equal_nan=True)),
                    "limit_rows_differ": int((~((lim_a == lim_b) | (np.isnan(lim_a) & np.isnan(lim_b)))).sum()),
                    "limit_max_rel_diff": float(rel.max()) if rel.size else 0.0}
            if len(m) and Nd == 1000 and K == 8:
                # exact ratios of (up to 4 of) the valid walks: exact walk + device reconstruction,
                # at most 1024 primes
                sub = m[:4]
                ratios, K_used = exact.exact_ratios(desc, recs[sub], Nd, H, K0=256, K_max=1024)
                # None: a divisor of the walk vanishes exactly (every prime), an invalid exact walk
                entry["exact_ratios"] = {"rows": int(len(sub)), "determined": int(sum(r is not None for r in ratios)),
                                         "exactly_singular": int(sum(r is None and k > 0 for r, k in zip(ratios, K_used))),
                                         "primes_max": int(K_used.max()), "primes_cap": 1024}
                # the same rows in the f64 walk, whose singularity tests are the exact walk's in floating point
                f = cmfw.walk("f64", desc, recs[m], Nd, H)
                entry["f64_valid_of_compat_valid"] = int((f["valid"] == 1).sum())
            res[f"N{Nd}_K{K}"] = entry
            print(f"rns8f7 N={Nd} K={K}: {entry}", file=sys.stderr, flush=True)
    head = res["N1000_K8"]
    line = {
        "metric": "8F7 zeta RNS walk traj/s on 1 B200 (compat semantics, bit-exact vs the reference)",
        "value": head["traj_per_s"], "unit": "traj/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": head["ms_per_step"], "higher_is_better": True, "dtype": "u32 residues",
        "data": "synthetic (seeded std::mt19937_64 directions)",
        "config": {"workload": "8F7 zeta limit: x=1^8, y=2^7, z=1, rank 7, dirs 1^15 + U{0..2}^15, h=50, "
                               "N in {1000, 4000}, moduli in {8, 16}", "n_traj": n, "seed": SEED,
                   "l2": "flushed between steps"},
        "configs": res,
    }
    print(json.dumps(line), flush=True)


def main_mixed(args):
    """Mixed-family batch: 3F2/4F3/5F4/6F5/8F7 x z in {1/2, 1}, starts
    U{1..10}, directions U{0..3} (not all zero), N log-uniform in 200..5000,
    h = 50, walked in one CUDA-graph launch (sort + per-descriptor persistent
    kernels). Reports traj/s of the baseline tiles (one thread per sorted
    trajectory, 256-thread CTAs), the persistent queues (default tiles) with
    and without the singularity prescan, and the autotuned tiles (per
    descriptor the fastest of plain grids and queues)."""
    import torch
    import cmfw
    import cmfw.workloads as wl
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if rank != 0:
        return
    t0 = time.perf_counter()
    descs, recs, items = wl.mixed_batch(args.mixed_n, SEED)
    t_gen = time.perf_counter() - t0
    b = cmfw.MixedBatch(descs, recs, items, H, args.variant)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    t0 = time.perf_counter()
    tuned = b.autotune()
    t_tune = time.perf_counter() - t0
    res = {}
    scan = cmfw.MixedTuning()
    scan.persistent = 1
    scan.prescan = 1
    for name, tuning in (("baseline_256", cmfw.baseline_tuning()), ("default", None),
                         ("persistent_prescan", scan), ("autotuned", tuned)):
        b.capture(tuning)
        b.replay()
        torch.cuda.synchronize()
        ms = []
        for k in range(args.steps):
            flush.fill_(k & 0xff)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            b.replay()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        out = b.results()
        res[name] = {"ms": float(np.mean(ms)), "traj_per_s": args.mixed_n / (np.mean(ms) / 1e3),
                     "n_valid": int((out["valid"] == 1).sum())}
        b.release()
    valid = out["valid"] == 1
    flops = 0.0
    for di, d in enumerate(descs):
        m = items["desc"] == di
        flops += walk_flops(d.p, d.q, d.rank, recs[m], items["N"][m], valid[m])
    tiles = [{"block": tuned.tile[f].block_size, "grab": tuned.tile[f].grab} for f in range(len(descs))]
    peak = cmfw.pipe_peak(0 if args.variant == "f64" else 1)
    best = res["autotuned"]
    line = {
        "metric": "mixed-batch traj/s on 1 B200 (one graph launch)", "value": best["traj_per_s"],
        "unit": "traj/s", "n_gpus": 1, "steps": args.steps, "ms_per_step": best["ms"], "higher_is_better": True,
        "dtype": args.variant, "data": "synthetic (seeded std::mt19937_64)",
        "config": {"workload": "mixed: {3F2,4F3,5F4,6F5,8F7} x z{1/2,1}, starts U{1..10}, dirs U{0..3}, "
                               "N log-uniform 200..5000, h=50", "n_traj": args.mixed_n, "seed": SEED,
                   "l2": "flushed between steps"},
        "tiles": res, "autotuned_tiles": tiles, "autotune_s": t_tune, "generate_s": t_gen,
        "speedup_vs_baseline_256": res["baseline_256"]["ms"] / best["ms"],
        "roofline": {"bound": "fp64" if args.variant == "f64" else "fp32", "achieved": flops / (best["ms"] / 1e3) / 1e12,
                     "peak": peak, "unit": "TFLOP/s", "frac": flops / (best["ms"] / 1e3) / 1e12 / peak,
                     "flops_per_launch": flops},
    }
    print(json.dumps(line), flush=True)


def main_proposal(args):
    """Learned proposal for the 8F7 zeta delta search (z = 1, rank 7, 15
    axes, directions U{0..4}^15, N = 1000, h = 50, df64 walks). Both sides
    start with the walk's singularity filter over all search-n candidates;
    the plain exhaustive sweep (the judge) walks every survivor, the
    proposal scores the survivors with the tensor-core MLP (trained on the
    walked survivors of train-n other candidates) and walks the top
    `fraction` of them. Reports how many of the sweep's top-100 deltas the
    proposal finds, its GPU time against the sweep's (with and without the
    shared filter), the same budget chosen at random (the method without the
    network), and the sweep's top-100 limits confirmed against the exact
    walk."""
    import torch
    from cmfw import mlp as cm
    from cmfw import proposal as prop
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if rank != 0:
        return
    n_search, n_train = int(args.search_n), int(args.train_n)
    S = prop.DeltaSearch(8, 7, 0, 4, N, H, "df64", SEED)
    S.sweep(min(1 << 22, n_search))  # warm (allocations, kernel set-up)
    S.survivors(0, n_search)  # and the filter at full size
    sw_i, sw_d, sw_valid, sw_ms, sw_st = S.sweep(n_search)
    data = S.training_set(n_train, 1 << 40)
    net = cm.Mlp(1 << 16, seed=1)
    train_ms = S.train(net, data[:4], epochs=args.epochs)
    S.propose(net, min(1 << 22, n_search), args.fraction)  # warm
    p_i, p_d, n_walk, p_valid, st = S.propose(net, n_search, args.fraction)
    r_i, _, _, _, st_r = S.propose(net, n_search, args.fraction, rank="random")
    prop_ms = st["filter"] + st["score"] + st["select"] + st["walk"]
    confirmed = S.confirm(sw_i[:100])
    line = {
        "metric": "learned proposal: recall of the exhaustive sweep's top-100 deltas and GPU-time share",
        "value": prop.recall(p_i, sw_i), "unit": "recall@100", "higher_is_better": True, "n_gpus": 1,
        "dtype": "df64 walks, bf16 x bf16 -> f32 MLP",
        "data": "synthetic (seeded splitmix64 candidate generator)",
        "config": {"workload": "8F7 zeta delta search: x=1^8, y=2^7, z=1, rank 7, dirs U{0..4}^15, N=1000, h=50",
                   "search_n": n_search, "train_n": n_train, "fraction_of_survivors_walked": args.fraction,
                   "mlp": f"64(15 dir + 5 one-hot) -> 256 -> 256 -> 256 -> 1, ReLU, Adam, {args.epochs} epochs"},
        "sweep": {"gpu_ms": sw_ms, "filter_ms": sw_st["filter_ms"], "walk_ms": sw_st["walk_ms"],
                  "survivors": sw_st["survivors"], "n_valid": sw_valid,
                  "top100_min_delta": float(sw_d[-1]) if len(sw_d) else None,
                  "top100_confirmed_exact": confirmed},
        "training": {"walk_gpu_ms": data[4], "train_gpu_ms": train_ms, **S.train_stats,
                     "target": f"top {prop.TOP_Q:.0%} of the training walks' finite deltas (weighted 0/1)"},
        "proposal": {"gpu_ms": prop_ms, "stages_ms": {k: v for k, v in st.items() if k != "survivors"},
                     "n_walked": n_walk, "n_valid_walked": p_valid,
                     "found": len(set(p_i.tolist()) & set(sw_i.tolist()))},
        "random_choice_same_budget": {"recall": prop.recall(r_i, sw_i), "walk_ms": st_r["walk"]},
        "gpu_time_share_vs_sweep": prop_ms / sw_ms if sw_ms else None,
        "gpu_time_share_without_filter": (prop_ms - st["filter"]) / sw_st["walk_ms"] if sw_st["walk_ms"] else None,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    a = parse()
    select_family(a)
    if a.impl == "reference":
        main_reference(a)
    elif a.workload == "mixed":
        main_mixed(a)
    elif a.workload == "rns8f7":
        main_rns(a)
    elif a.workload == "proposal":
        main_proposal(a)
    else:
        main_cmfw(a)
