#!/usr/bin/env python
"""Benchmark of the box-image path: Lorenz, depth 27, on B200.

One step = one whole Lorenz job of the reference's subdivision driver
(subdivision.m:18-45): 27 subdivision steps (sigma=10, rho=28, beta=8/3, RK4 h=0.01 x 20,
5x5x5 inner grid, domain centre (0,0,27) radius (30,30,40)), the CSR transition matrix
on the final boxes, and 200 FP64 power iterations for the invariant measure.

The headline uses the explicit-FMA integrator (the same fused multiply-adds in the
kernel, the oracle and the reference harness's plug-in map); its box sets and transition
matrix equal the reference's strict (-fmad=false) run at every step on this workload.
The strict integrator - one rounding per operation, the reference's own Map_Lorenz.h
order - is measured in the same run and reported under "strict".

metric = box-images per second of whole-job time (a box-image is one box's 125 test
points sampled, integrated and located): the subdivision steps image 2*n(k-1) boxes each.
The transition matrix is assembled from the targets the last step stored, so its
n(27) boxes are not imaged again and are not counted (the job's time includes it).
Inputs are synthetic: the workload is defined entirely by its parameters.

The reference arm (--impl reference) runs the reference's own Thrust code (OMP backend,
all host cores) on a bounded sample of the same job: subdivision step 25 from the
depth-24 tree the reference itself saved, then transitionMatrixForLeaves on the
depth-25 tree, timed per round; its value is that step's box-images over the step's and
the matrix's time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs its own job (weak scaling, no collective on the
data path); value = all ranks' box-images / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

DEPTH = 27
MEASURE_ITERS = 200
P = 125
FLOP_PER_POINT = 20 * 78          # RK4 step: 4 right-hand sides (9 FLOP) + 42 update FLOP
METRIC = "Lorenz box-images/s"
UNIT = "box-images/s"
CONFIG = {"workload": "lorenz-rk4-depth27", "sigma": 10.0, "rho": 28.0, "beta": 8.0 / 3.0, "h": 0.01,
          "rk4_steps": 20, "grid": "inner 5x5x5", "depth": DEPTH, "tm": "csr", "measure_iters": MEASURE_ITERS,
          "l2": "flushed between timed steps (256 MiB write)", "arith": "fma"}
NOMINAL_FP64_TFLOPS = 37.0
IMAGE_DRAM_BYTES_PER_BOX = 2.346752e6 / 47304   # ncu: DRAM bytes of one image launch / its boxes


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout: float = 5.0):
        """block until nvidia-smi has produced its first sample (it starts slowly)"""
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.02)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
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
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------ CPU arms
def ref_exe(name: str):
    exe = os.path.join(REPO, "oracle", "_ref", name)
    return exe if os.path.exists(exe) else None


def cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_ref(name: str, args, threads: int) -> dict:
    """One run of a reference harness binary; its JSON line (the harness times itself,
    so process start-up and file writes are outside every figure)."""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    res = subprocess.run([ref_exe(name)] + [str(x) for x in args], env=env, check=True, capture_output=True,
                         text=True)
    return json.loads(res.stdout.strip().splitlines()[-1])


REF_FROM_DEPTH = 24              # the reference arm's rounds start from the saved depth-24 tree
REF_BUF = 1 << 30                # nHostBufferBytes for Lorenz (the reference's default is 4 GiB)
REF_SMALL_BUF = 64 << 20         # for Henon and forced Duffing


class ReferenceLorenz:
    """The reference's Lorenz job on a bounded sample: the reference saves its own
    depth-24 tree once (untimed); a round loads it, runs subdivision step 25 and
    transitionMatrixForLeaves of the depth-25 tree."""

    def __init__(self, threads: int):
        import tempfile
        self.threads = threads
        self.dir = tempfile.mkdtemp(prefix="b12_ref_")
        base = os.path.join(self.dir, "d24")
        run_ref("ref_lorenz", ["--steps", REF_FROM_DEPTH, "--tm", 0, "--buf", REF_BUF, "--save", base], threads)
        self.tree = base + "_tree.json"

    def rounds(self, n: int) -> list:
        rec = run_ref("ref_lorenz", ["--load", self.tree, "--steps", 1, "--tm", 1, "--buf", REF_BUF,
                                     "--repeat", n], self.threads)
        return rec["rounds"]          # [subdivision s, matrix s, box-images, leaves, nonzeros]

    def close(self):
        import shutil
        shutil.rmtree(self.dir, ignore_errors=True)

    def sample_text(self, r) -> str:
        return (f"Lorenz subdivision step {REF_FROM_DEPTH + 1} from the depth-{REF_FROM_DEPTH} tree the reference "
                f"saved ({r[2]} box-images, {r[0]:.2f} s) + transitionMatrixForLeaves on its {r[3]} boxes "
                f"({r[4]} nonzeros, {r[1]:.2f} s); strict arithmetic (the reference's own Map_Lorenz.h); "
                f"nHostBufferBytes {REF_BUF >> 20} MiB; Thrust OMP backend; the reference has no invariant measure")


def run_port_sample():
    """The oracle restatement (OpenMP C) on the same sample, when the reference build is absent:
    step 25 from its own depth-24 tree, then the transition matrix."""
    from oracle import oracle as O
    o = O.Oracle(O.lorenz_spec())
    o.subdivision(REF_FROM_DEPTH)
    t0 = time.perf_counter()
    _, bi = o.subdivision(1)
    t1 = time.perf_counter()
    rowptr, _, _, _ = o.transition_matrix()
    t2 = time.perf_counter()
    return [t1 - t0, t2 - t1, bi, len(rowptr) - 1, int(rowptr[-1])]


def cpu_baseline(threads: int):
    if ref_exe("ref_lorenz"):
        ref = ReferenceLorenz(threads)
        try:
            r = ref.rounds(2)[-1]
            text = ref.sample_text(r)
        finally:
            ref.close()
        kind = "reference"
    else:
        from oracle import oracle as O
        threads = O.lib().orc_num_threads()
        r = run_port_sample()
        kind = "port"
        text = f"Lorenz step {REF_FROM_DEPTH + 1} + transition matrix, OpenMP C restatement"
    return {"value": r[2] / (r[0] + r[1]), "unit": UNIT, "cores": threads, "kind": kind, "sample": text}


def reference_arm(args, rank: int, world: int):
    if rank != 0:
        return 0
    threads = cpu_cores()
    if ref_exe("ref_lorenz"):
        kind = "reference"
        ref = ReferenceLorenz(threads)
        try:
            rounds = ref.rounds(args.warmup + args.steps)[args.warmup:]
            text = ref.sample_text(rounds[0])
        finally:
            ref.close()
    else:
        kind = "port"
        rounds = [run_port_sample() for _ in range(args.warmup + args.steps)][args.warmup:]
        text = f"Lorenz step {REF_FROM_DEPTH + 1} + transition matrix, OpenMP C restatement"
    tot_bi = sum(r[2] for r in rounds)
    tot_s = sum(r[0] + r[1] for r in rounds)
    value = tot_bi / tot_s
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / len(rounds), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": dict(CONFIG, arith="strict", measure_iters=0,
                           sample=f"per step: subdivision step {REF_FROM_DEPTH + 1} + transition matrix "
                                  f"(the job's most expensive regime; steps 25-27 and the matrix are most of "
                                  f"the reference's whole job)"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": text},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------ GPU arm
def box_images_of(counts) -> tuple[int, int]:
    prev = np.concatenate([[1], counts[:-1]]).astype(np.int64)
    return int(2 * prev.sum()), int(counts[-1])


def measure_mode(args, rank, world, dist, fma: bool, peak_tflops: float):
    """Time args.steps whole jobs with the given integrator arithmetic."""
    import torch
    import b12_b200 as B
    from b12_b200 import tree as T
    from b12_b200.ranks import throughput

    dev = torch.cuda.current_device()
    sc = B.Scheme(B.lorenz(rho=28.0, fma=fma), B.inner_grid(5))
    tree = B.ImplicitBoxTree([0.0, 0.0, 27.0], [30.0, 30.0, 40.0])
    tree.reserve(1 << 20)
    stream = torch.cuda.ExternalStream(tree.stream_handle(), device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    state = {"csr": None}

    def job():
        tree.delete_depth(0)
        counts = tree.subdivision_run(sc, DEPTH)
        state["csr"] = tree.transition_matrix(sc, into=state["csr"])
        state["csr"].invariant_measure(MEASURE_ITERS, keep_on_device=True)
        return counts

    counts = None
    for _ in range(args.warmup):
        counts = job()
    bi_sub, n_final = box_images_of(counts)
    box_images = bi_sub          # imaged boxes only: the matrix's rows come from stored targets

    # phase breakdown of a job (host clock around the synchronous API calls): the median
    # of three jobs per phase, so that one host stall does not make the breakdown
    samples = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tree.delete_depth(0)
        t1 = time.perf_counter()
        tree.subdivision_run(sc, DEPTH)
        t2 = time.perf_counter()
        state["csr"] = tree.transition_matrix(sc, into=state["csr"])
        t3 = time.perf_counter()
        state["csr"].invariant_measure(MEASURE_ITERS, keep_on_device=True)
        t4 = time.perf_counter()
        samples.append((t1 - t0, t2 - t1, t3 - t2, t4 - t3))
    med = [1e3 * sorted(x[i] for x in samples)[1] for i in range(4)]
    phases = {"reset_ms": med[0], "subdivision_ms": med[1], "transition_matrix_ms": med[2],
              "invariant_measure_ms": med[3], "jobs": len(samples)}

    tree.profile(True)
    tree.profile_read(0)
    tree.profile_read(1)
    launches0 = T.launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clocks:
        clocks.wait_first()
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                ev[i][0].record(stream)
            c = job()
            with torch.cuda.stream(stream):
                ev[i][1].record(stream)
            if list(c) != list(counts):
                raise RuntimeError("box counts changed between steps")
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = T.launch_count() - launches0
    total_ms = sum(a.elapsed_time(b) for a, b in ev)
    img_ms, img_n = tree.profile_read(0)
    row_ms, row_n = tree.profile_read(1)
    tree.profile(False)
    # all ranks' box-images over the slowest rank's device time
    value, _, slowest_s = throughput(dist, args.steps * box_images, total_ms * 1e-3, dev)
    total_ms = 1e3 * slowest_s
    flops_img = args.steps * bi_sub * P * FLOP_PER_POINT
    achieved = flops_img / (img_ms * 1e-3) / 1e12 if img_ms > 0 else None
    # the rows come from the targets the last subdivision step stored (no map evaluation):
    # every survivor's P targets, two ranks per child, a row count and its (column, count) runs
    n_children = 2 * int(counts[-2]) if len(counts) > 1 else 2
    rows_bytes = n_final * P * 4 + n_children * 4 * 2 + n_final * 4 + state["csr"].nnz * 8
    rows_gbs = args.steps * rows_bytes / (row_ms * 1e-3) / 1e9 if row_ms > 0 else None
    rows_info = {"kernel": "stored_rows_kernel", "ms_per_step": row_ms / args.steps, "bytes_per_launch": rows_bytes,
                 "achieved_gbs": rows_gbs,
                 "note": "rows from the image targets the last subdivision step stored (the same points), "
                         "so the matrix re-evaluates no map"}

    # end to end through the public API: results copied to pinned host memory each step
    csr = state["csr"]
    codes = torch.empty(n_final, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    depth = torch.empty(n_final, dtype=torch.uint8, pin_memory=True).numpy()
    flags = torch.empty(n_final, dtype=torch.uint8, pin_memory=True).numpy()
    rowptr = torch.empty(n_final + 1, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    cols = torch.empty(max(csr.nnz, 1), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    vals = torch.empty(max(csr.nnz, 1), dtype=torch.float64, pin_memory=True).numpy()
    meas = torch.empty(n_final, dtype=torch.float64, pin_memory=True).numpy()
    root = (np.zeros(1, np.uint64), np.zeros(1, np.uint8), np.zeros(1, np.uint8))
    h2d = 8 + 1 + 1
    d2h = codes.nbytes + depth.nbytes + flags.nbytes + rowptr.nbytes + cols.nbytes + vals.nbytes + meas.nbytes
    e2e_steps = max(1, min(args.steps, 5))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        tree.load_leaves(*root)                       # the job's input: the surrounding box
        tree.subdivision_run(sc, DEPTH)
        csr = tree.transition_matrix(sc, into=csr)
        csr.invariant_measure(MEASURE_ITERS, out=meas)
        lib_leaves(tree, codes, depth, flags)
        csr.to_host_into(rowptr, cols, vals)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_value, _, e2e_s = throughput(dist, e2e_steps * box_images, e2e_s, dev)
    e2e = {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": int(d2h), "steps": e2e_steps, "timer": "host wall clock, synchronous API"}
    roofline = {"bound": "fp64", "kernel": "image_points_kernel (fused sample/RK4/locate)", "achieved": achieved,
                "peak": peak_tflops, "unit": "TFLOP/s", "frac": (achieved / peak_tflops) if achieved else None,
                "traffic": (IMAGE_DRAM_BYTES_PER_BOX * bi_sub + n_children * P * 4) / img_n * args.steps
                if img_n else None,
                "traffic_source": "ncu (profiles/image_points_kernel_lorenz_depth23.md): 2.35 MB of DRAM reads "
                                  "and writes in one launch over 47,304 boxes, scaled to this job's boxes per launch, "
                                  "plus the 4-byte target of every point the last step stores",
                "peak_source": "measured: FP64 FMA-chain probe kernel on this device "
                               f"(nominal {NOMINAL_FP64_TFLOPS} TFLOP/s)",
                "flop_per_box_image": P * FLOP_PER_POINT, "launches": img_n,
                "kernel_ms_per_step": img_ms / args.steps, "transition_rows": rows_info}
    out = dict(value=value, total_ms=total_ms, e2e=e2e, launches=launches, roofline=roofline,
               clocks=clocks.summary(), phases=phases, counts=[int(c) for c in counts], box_images=box_images,
               n_final=n_final, nnz=csr.nnz)
    state["csr"] = None
    csr.close()
    tree.close()
    return out


def gpu_arm(args, rank: int, world: int, dist):
    import torch
    from b12_b200 import tree as T

    dev = int(os.environ.get("LOCAL_RANK", "0")) % torch.cuda.device_count()
    torch.cuda.set_device(dev)
    # FP64 roofline denominator, measured on this device
    peak_tflops, _ = T.probe_fp64_fma(0.25)
    main = measure_mode(args, rank, world, dist, fma=not args.strict, peak_tflops=peak_tflops)
    other = None if args.single else measure_mode(args, rank, world, dist, fma=args.strict, peak_tflops=peak_tflops)
    cpu = cpu_baseline(cpu_cores()) if (rank == 0 and world == 1 and not args.no_cpu) else None
    configs = configs_mode(args, peak_tflops) if (rank == 0 and world == 1 and not args.no_configs) else None
    serving = serve_mode(args) if (rank == 0 and world == 1 and args.serve_jobs > 0) else None
    # with several ranks, the workloads that shard by themselves (independent instances and
    # jobs) are split over the ranks: every rank takes every world-th instance / job
    sharded = sharded_mode(args, rank, world, dist, peak_tflops) if (world > 1 and not args.no_configs) else None
    if rank == 0:
        arith = "strict" if args.strict else "fma"
        line = {"metric": METRIC, "value": main["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": main["total_ms"] / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(CONFIG, arith=arith,
                               parallelism=f"{world} independent jobs" if world > 1 else "1 job",
                               box_images_per_step=main["box_images"], final_boxes=main["n_final"],
                               matrix_boxes_not_counted=main["n_final"], nnz=main["nnz"]),
                "e2e": main["e2e"], "gpu_launches": int(main["launches"]), "roofline": main["roofline"],
                "clocks": main["clocks"], "cpu_baseline": cpu, "phases_ms": main["phases"],
                "counts": main["counts"]}
        if other is not None:
            line["strict" if not args.strict else "fma"] = {
                "value": other["value"], "ms_per_step": other["total_ms"] / args.steps, "e2e": other["e2e"]["value"],
                "roofline_achieved": other["roofline"]["achieved"], "roofline_frac": other["roofline"]["frac"],
                "transition_rows_ms": other["roofline"]["transition_rows"]["ms_per_step"], "phases_ms": other["phases"],
                "counts_identical": other["counts"] == main["counts"], "clocks": other["clocks"]}
        if configs is not None:
            line["configs"] = configs
        if serving is not None:
            line["serving"] = serving
        if sharded is not None:
            line["sharded"] = sharded
        print(json.dumps(line), flush=True)
    return 0


def sharded_mode(args, rank: int, world: int, dist, peak_tflops: float):
    """The 512-instance Lorenz scan and the served stream split over the ranks (no
    collective on the data path: each rank runs its own instances / jobs on its own GPU);
    whole-job throughput = all ranks' units over the slowest rank's time.  Every rank
    takes the same collective steps."""
    import torch
    import b12_b200 as B
    from b12_b200.ranks import shard, throughput
    from b12_b200.server import JobServer, replay
    from b12_b200.workloads import LORENZ_CENTER, LORENZ_RADIUS, job_stream, lorenz_scan

    dev = torch.cuda.current_device()
    out = {}
    rho, depth = lorenz_scan(512, 0)
    mine = shard(range(512), world, rank)
    b = B.Batch(LORENZ_CENTER, LORENZ_RADIUS, B.Scheme(B.lorenz(fma=True), B.inner_grid(5)),
                [(10.0, rho[i], 8.0 / 3.0) for i in mine], [depth[i] for i in mine])
    b.run()                                   # autotunes the launch shape
    b.transition_matrices()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.run()
    b.transition_matrices()
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    info = b.info()
    b.close()
    units = info["box_images"] + info["final_boxes"]
    rate, total, slowest = throughput(dist, units, sec, dev)
    out["lorenz_batch_512"] = {"instances_per_rank": len(mine), "box_images_per_s": rate, "box_images": total,
                               "slowest_rank_s": slowest, "split": "instance i on rank i mod world",
                               "scaling": "strong (the 512 instances are split)"}
    if args.serve_jobs > 0:
        jobs = [dict(j, arrival=0.0) for j in shard(job_stream(args.serve_jobs, 1.0, 0), world, rank)]
        with JobServer(SERVE_CAP // world) as srv:
            warm = [dict(j, arrival=0.0) for j in job_stream(min(len(jobs), 500), 1.0, 1)]
            replay(srv, warm, lambda job, jid: srv.release(jid), timeout=SERVE_TIMEOUT)
            if dist:
                dist.barrier()
            res = replay(srv, jobs, lambda job, jid: srv.release(jid), timeout=SERVE_TIMEOUT)
        rate, total, slowest = throughput(dist, len(jobs), res["span"], dev)
        out["served_stream"] = {"jobs_per_rank": len(jobs), "jobs_per_s": rate, "jobs": total,
                                "slowest_rank_s": slowest, "split": "job j on rank j mod world, all submitted at once",
                                "scaling": "strong (the stream is split)"}
    return out


# ------------------------------------------------------------------------------ other configurations
def _timed(fn, reps: int):
    """Best-of-`reps` host wall time of a synchronous call (after one untimed call)."""
    fn()
    best = float("inf")
    out = None
    for _ in range(reps):
        t0 = time.perf_counter()
        out = fn()
        best = min(best, time.perf_counter() - t0)
    return best, out


def configs_mode(args, peak_tflops: float):
    """The Henon validity workload, the coupled-Duffing continuation and the 512-instance
    Lorenz scan, each timed on its own after a warm-up call, each beside the reference's
    own code on a stated sample (all host cores)."""
    import b12_b200 as B
    from b12_b200.workloads import LORENZ_CENTER, LORENZ_RADIUS, lorenz_scan

    threads = cpu_cores()
    cpu = not args.no_cpu and all(ref_exe(x) for x in ("ref_henon", "ref_lorenz", "ref_duffing"))
    out = {}
    # Henon a=1.4 b=0.3, 20 steps, 4x4 inner grid, CSR
    sc = B.Scheme(B.henon(1.4, 0.3), B.inner_grid(4))
    t = B.ImplicitBoxTree((0.0, 0.0), (1.5, 0.45))

    def henon():
        t.delete_depth(0)
        c = t.subdivision_run(sc, 20)
        m = t.transition_matrix(sc)
        nnz = m.nnz
        m.close()
        return c, nnz

    sec, (c, nnz) = _timed(henon, 5)
    bi, nf = box_images_of(c)
    out["henon_d20"] = {"boxes": nf, "nnz": nnz, "ms_per_job": 1e3 * sec, "box_images_per_s": bi / sec,
                        "note": "imaged boxes of the 20 steps per second of job time (the matrix comes from "
                                "the last step's stored targets)"}
    if cpu:
        rec = run_ref("ref_henon", ["--steps", 20, "--tm", 1, "--buf", REF_SMALL_BUF], threads)
        job_s = rec["subdivision_s"] + rec["tm_s"]
        out["henon_d20"]["cpu_baseline"] = {
            "value": rec["box_images"] / job_s, "unit": UNIT, "cores": threads, "kind": "reference",
            "ms_per_job": 1e3 * job_s, "boxes": rec["steps"][-1][1], "nnz": rec["nnz"],
            "sample": f"the whole job: 20 steps + transitionMatrixForLeaves, nHostBufferBytes {REF_SMALL_BUF >> 20} "
                      "MiB, Thrust OMP backend"}
    t.close()

    # coupled Duffing, unstable-manifold continuation at depth 24 from the box of the origin,
    # 64 Philox points per box (seed 0), Stormer-Verlet h=0.05 x 10
    sc = B.Scheme(B.coupled_duffing(), B.philox_grid(64, 0))
    t = B.ImplicitBoxTree((0.0,) * 4, (2.0,) * 4)
    t.reserve(16 << 20)
    sec, sweeps = _timed(lambda: t.continuation_run(sc, np.zeros(4), 24), 2)
    n = int(sweeps[-1])
    flop = 64 * 280
    # one more run with CUDA events around every image launch (the insert-mode kernel)
    t.profile(True)
    t.profile_read(0)
    t.continuation_run(sc, np.zeros(4), 24)
    img_ms, img_n = t.profile_read(0)
    t.profile(False)
    img_tflops = n * flop / (img_ms * 1e-3) / 1e12 if img_ms > 0 else None
    out["coupled_duffing_continuation_d24"] = {
        "boxes": n, "sweeps": len(sweeps), "seconds": sec, "box_images": n,
        "box_images_per_s": n / sec, "tflops": n * flop / sec / 1e12, "flop_per_box_image": flop,
        "roofline": {"bound": "fp64", "kernel": "image_points_kernel (insert mode, Stormer-Verlet, Philox grid)",
                     "achieved": img_tflops, "peak": peak_tflops, "unit": "TFLOP/s",
                     "frac": img_tflops / peak_tflops if img_tflops else None,
                     "strict_cap": 0.5, "kernel_ms": img_ms, "launches": img_n,
                     "note": "strict arithmetic (one rounding per operation, the reference's own "
                             "SymplecticIntegratorAuto order): at most half the FMA peak; the rest of the run is "
                             "the candidate sort, unique, merge and flag updates (launch list in profiles/)"},
        "note": "every box is imaged once, in the sweep after it was inserted"}
    if cpu:
        sweeps_ref = 20
        rec = run_ref("ref_duffing", ["--steps", 24, "--buf", REF_BUF, "--max-sweeps", sweeps_ref], threads)
        out["coupled_duffing_continuation_d24"]["cpu_baseline"] = {
            "value": rec["box_images"] / rec["continuation_s"], "unit": UNIT, "cores": threads, "kind": "reference",
            "seconds": rec["continuation_s"], "box_images": rec["box_images"],
            "boxes_after_sample": rec["sweeps"][-1][1],
            "sample": f"sweeps 1-{sweeps_ref} of the same depth-24 continuation (of 49), nHostBufferBytes "
                      f"{REF_BUF >> 20} MiB, Thrust OMP backend"}
    t.close()

    # selective refinement (leaves of several depths): Lorenz (explicit FMA) refined to
    # depth 21, SD kept on the leaves of the lower half in x, then 6 steps that subdivide
    # and select only those, and the CSR of the final tree (depths 21-27)
    sc = B.Scheme(B.lorenz(fma=True), B.inner_grid(5))
    t = B.ImplicitBoxTree(LORENZ_CENTER, LORENZ_RADIUS)
    t.subdivision_run(sc, 21)
    codes, depth, flags = t.leaves()
    lower = (codes >> np.uint64(20)) == 0
    start = (codes, depth, ((flags & ~np.uint8(B.SD)) | np.where(lower, B.SD, 0)).astype(np.uint8))

    def selective():
        t.load_leaves(*start)
        imaged = 0
        for _ in range(6):
            t.subdivide(B.SD)
            imaged += t.count()
            t.set_flags_by_image(sc, B.HIT)
            t.remove(B.HIT)
            t.unset_flags(B.HIT)
        m = t.transition_matrix(sc)
        nnz = m.nnz
        m.close()
        d = t.leaves()[1]
        return imaged, t.count(), nnz, int(d.min()), int(d.max())

    sec, (imaged, nf, nnz, dmin, dmax) = _timed(selective, 3)
    flop = P * FLOP_PER_POINT
    out["lorenz_selective_d21_plus6"] = {
        "start_boxes": int(len(codes)), "final_boxes": nf, "depths": [dmin, dmax], "nnz": nnz,
        "box_images": imaged + nf, "seconds": sec, "box_images_per_s": (imaged + nf) / sec,
        "tflops": (imaged + nf) * flop / sec / 1e12,
        "frac_of_fp64_peak": (imaged + nf) * flop / sec / 1e12 / peak_tflops,
        "note": "per-leaf-depth kernels (binary search over comparable patterns); includes the "
                "reload of the depth-21 start leaves from the host and every host round trip"}
    t.close()

    # 512 Lorenz instances, rho ~ U[15,35], depth 18-27 (SplitMix64 seed 0): batched
    rho, depth = lorenz_scan(512, 0)
    params = [(10.0, r, 8.0 / 3.0) for r in rho]
    b = B.Batch(LORENZ_CENTER, LORENZ_RADIUS, B.Scheme(B.lorenz(fma=True), B.inner_grid(5)), params, depth)
    b.run()                       # first run: autotunes the launch shape
    b.transition_matrices()
    run_s, _ = _timed(b.run, 2)
    tm_s, _ = _timed(b.transition_matrices, 2)
    info = b.info()
    bi, nf = info["box_images"], info["final_boxes"]
    flop = P * FLOP_PER_POINT
    out["lorenz_batch_512"] = {
        "instances": 512, "box_images": bi, "final_boxes": nf, "nnz": info["nnz"],
        "subdivision_s": run_s, "transition_matrices_s": tm_s,
        "box_images_per_s": (bi + nf) / (run_s + tm_s),
        "subdivision_tflops": bi * flop / run_s / 1e12, "subdivision_frac_of_fp64_peak": bi * flop / run_s / 1e12 /
        peak_tflops, "launch_shape": {k: info[k] for k in ("threads", "points_per_thread", "chunk")},
        "frac_note": "whole batched run (every kernel of the 27 steps) against the measured FP64 peak"}
    b.close()
    if cpu:
        # the reference runs one instance after another; sample: the first instances in
        # scan order of depth <= 22 (deeper ones skipped, which favours the reference)
        picked = [i for i in range(512) if depth[i] <= 22][:3]
        bi_ref, sec_ref = 0, 0.0
        for i in picked:
            rec = run_ref("ref_lorenz", ["--steps", depth[i], "--tm", 1, "--rho", repr(rho[i]), "--buf", REF_BUF],
                          threads)
            bi_ref += rec["box_images"] + rec["tm_box_images"]
            sec_ref += rec["subdivision_s"] + rec["tm_s"]
        out["lorenz_batch_512"]["cpu_baseline"] = {
            "value": bi_ref / sec_ref, "unit": UNIT, "cores": threads, "kind": "reference",
            "seconds": sec_ref, "box_images": bi_ref,
            "sample": f"instances {picked} of the scan (depths {[depth[i] for i in picked]}) run one at a time, "
                      f"27-step loop to each depth + transitionMatrixForLeaves, strict arithmetic (the reference's "
                      f"Map_Lorenz.h), nHostBufferBytes {REF_BUF >> 20} MiB, Thrust OMP backend"}
    return out


# ------------------------------------------------------------------------------ serving
SERVE_RATES = (500.0, 1000.0, 2000.0)
SERVE_TIMEOUT = 300.0            # seconds per replayed stream before the bench gives up
SERVE_DIGEST_EVERY = 10          # full-result digests on every 10th job; counts and nnz on all
SERVE_CAP = 150 * 10**9
SERVE_FRESH_JOBS = 2000          # jobs of the fresh-tree plain path (a prefix of the stream)
SERVE_CPU_SECONDS = 8.0          # reference sample: jobs in arrival order until this much CPU time


def serve_cpu_baseline(base):
    """The reference running served-stream jobs one at a time (its only way): jobs in
    arrival order, Lorenz jobs deeper than 22 skipped (which favours the reference), until
    SERVE_CPU_SECONDS of job time; each job is the subdivision loop + transitionMatrixForLeaves."""
    threads = cpu_cores()
    done, sec, fams = 0, 0.0, {}
    for job in base:
        fam, p, d = job["family"], job["params"], job["depth"]
        if fam == "henon":
            rec = run_ref("ref_henon", ["--steps", d, "--tm", 1, "--a", repr(p[0]), "--b", repr(p[1]),
                                        "--buf", REF_SMALL_BUF], threads)
        elif fam == "lorenz":
            if d > 22:
                continue
            rec = run_ref("ref_lorenz", ["--steps", d, "--tm", 1, "--rho", repr(p[1]), "--buf", REF_BUF], threads)
        else:
            rec = run_ref("ref_forced", ["--steps", d, "--tm", 1, "--buf", REF_SMALL_BUF], threads)
        sec += rec["subdivision_s"] + rec["tm_s"]
        done += 1
        fams[fam] = fams.get(fam, 0) + 1
        if sec >= SERVE_CPU_SECONDS:
            break
    return {"value": done / sec, "unit": "jobs/s", "cores": threads, "kind": "reference", "jobs": done,
            "seconds": sec, "sample": f"the first {done} jobs of the stream in arrival order ({fams}), Lorenz "
                                      "jobs deeper than 22 skipped; one job at a time; Lorenz in strict arithmetic "
                                      f"(the reference's Map_Lorenz.h); nHostBufferBytes {REF_SMALL_BUF >> 20} MiB "
                                      f"(Henon, forced Duffing) / {REF_BUF >> 20} MiB (Lorenz); Thrust OMP backend"}


def _job_digest(codes, counts, rowptr, cols, vals) -> str:
    import hashlib
    h = hashlib.sha256()
    for a in (codes, counts, rowptr, cols, vals):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def fifo_latencies(arrivals, service):
    """Latencies of a single server taking jobs one at a time in arrival order."""
    t, out = 0.0, []
    for a, s in zip(arrivals, service):
        t = max(t, a) + s
        out.append(t - a)
    return out


def _pct(x, q):
    return float(np.percentile(np.asarray(x), q)) * 1e3


def serve_mode(args):
    """The served stream (Henon / Lorenz / forced Duffing jobs, Poisson arrivals) through the
    job server against the plain path: one ImplicitBoxTree per job, one job at a time
    (subdivision_run, then transition_matrix), on the same GPU and the same jobs."""
    from b12_b200 import tree as T
    from b12_b200.server import JobServer, replay, stream_job_args
    from b12_b200.workloads import job_stream

    n = args.serve_jobs
    base = job_stream(n, 1.0, 0)          # family, parameters, depth of every job (seed 0)
    fams = [j["family"] for j in base]

    # the plain path: one job at a time through the single-tree API, one tree handle
    # per family reused across jobs (delete_depth(0) resets it; the matrix is refilled in
    # place), as the integration notes recommend
    trees = {}

    def plain_job(job):
        c, r, mp, g, d = stream_job_args(job)
        ent = trees.get(job["family"])
        if ent is None:
            ent = trees[job["family"]] = [T.ImplicitBoxTree(c, r), None]
        t = ent[0]
        t.delete_depth(0)
        sc = T.Scheme(mp, g)
        counts = t.subdivision_run(sc, d)
        ent[1] = t.transition_matrix(sc, into=ent[1])
        return t, counts, ent[1]

    def fresh_job(job):
        c, r, mp, g, d = stream_job_args(job)
        t = T.ImplicitBoxTree(c, r)
        sc = T.Scheme(mp, g)
        t.subdivision_run(sc, d)
        m = t.transition_matrix(sc)
        m.close()
        t.close()

    # warm-up on other jobs, then every job timed on its own
    for job in job_stream(6, 1.0, 1):
        plain_job(job)
        fresh_job(job)
    service, plain_digest, plain_shape = [], {}, []
    for k, job in enumerate(base):
        t0 = time.perf_counter()
        t, counts, m = plain_job(job)
        service.append(time.perf_counter() - t0)
        plain_shape.append((tuple(int(c) for c in counts), int(m.nnz)))
        if k % SERVE_DIGEST_EVERY == 0:
            rowptr, cols, vals = m.to_host()
            plain_digest[k] = _job_digest(t.leaves()[0], np.asarray(counts, np.uint32), rowptr, cols, vals)
    for t, m in trees.values():
        if m is not None:
            m.close()
        t.close()
    plain_rate = n / sum(service)
    # the same path with a new tree per job (allocations, graph instantiation), on a prefix
    n_fresh = min(n, SERVE_FRESH_JOBS)
    t0 = time.perf_counter()
    for job in base[:n_fresh]:
        fresh_job(job)
    fresh_s = time.perf_counter() - t0

    out = {"workload": f"served stream of {n} jobs (seed 0): Henon a~U[1.0,1.4] depth 14-22, Lorenz "
                       "rho~U[15,35] depth 18-27, forced Duffing depth 16-22, uniform family mix",
           "jobs": n, "hbm_cap_bytes": SERVE_CAP,
           "plain": {"jobs_per_s": plain_rate, "service_ms_mean": 1e3 * sum(service) / n,
                     "per_family_ms": {f: 1e3 * float(np.mean([s for s, g in zip(service, fams) if g == f]))
                                       for f in sorted(set(fams))},
                     "path": "one job at a time, one reused tree handle per family (delete_depth(0) between "
                             "jobs, matrix refilled in place)"},
           "plain_fresh_tree": {"jobs_per_s": n_fresh / fresh_s, "jobs": n_fresh,
                                "reused_handle_jobs_per_s_same_jobs": n_fresh / sum(service[:n_fresh]),
                                "path": "a new ImplicitBoxTree per job (first jobs of the stream)"}}
    if args.no_cpu or not all(ref_exe(x) for x in ("ref_henon", "ref_lorenz", "ref_forced")):
        pass
    else:
        out["cpu_baseline"] = serve_cpu_baseline(base)
    with JobServer(SERVE_CAP) as srv:
        # warm-up on a burst of other jobs: engines created, buffers and the result pool grown
        warm = [dict(j, arrival=0.0) for j in job_stream(min(n, 1000), 1.0, 1)]
        replay(srv, warm, lambda job, jid: srv.release(jid), timeout=SERVE_TIMEOUT)
        # saturated: every job submitted at once and released as it finishes (a resident
        # result counts against the admission cap), as the plain path frees each tree; the
        # results stay on the device in both, so neither timing reads them back
        sat = [dict(j, arrival=0.0) for j in base]
        res = replay(srv, sat, lambda job, jid: srv.release(jid), timeout=SERVE_TIMEOUT)
        out["served_saturated"] = {"jobs_per_s": n / res["span"], "span_s": res["span"],
                                   "p50_ms": _pct(res["latency"], 50), "p99_ms": _pct(res["latency"], 99)}
        # the same burst again, untimed: every result read and checked against the plain path
        check = {"shape": 0, "digest": 0}

        def check_and_release(job, jid):
            k = job["id"]
            inf = srv.info(jid)
            if k in plain_digest:
                r = srv.result(jid)
                check["digest"] += _job_digest(r["codes"], r["counts"], r["rowptr"], r["cols"],
                                               r["vals"]) == plain_digest[k]
                counts = r["counts"]
            else:
                counts = srv.counts(jid)
            check["shape"] += (tuple(int(c) for c in counts), int(inf["nnz"])) == plain_shape[k]
            srv.release(jid)

        replay(srv, sat, check_and_release, timeout=SERVE_TIMEOUT)
        same_shape, same = check["shape"], check["digest"]
        out["identical_to_plain"] = {"step_counts_and_nnz": f"{same_shape}/{n}",
                                     "full_result_sha256": f"{same}/{len(plain_digest)}",
                                     "pass": "a second, untimed saturated burst whose results are read back"}
        out["jobs_per_s_vs_plain"] = out["served_saturated"]["jobs_per_s"] / plain_rate
        out["jobs_per_s_vs_plain_fresh_tree"] = out["served_saturated"]["jobs_per_s"] / out["plain_fresh_tree"][
            "jobs_per_s"]
        sweep = []
        for rate in SERVE_RATES:
            st = job_stream(n, rate, 0)
            res = replay(srv, st, lambda job, jid: srv.release(jid), timeout=SERVE_TIMEOUT)
            arr = [j["arrival"] for j in st]
            pl = fifo_latencies(arr, service)
            plain_span = max(a + x for a, x in zip(arr, pl)) - arr[0]
            sweep.append({"offered_jobs_per_s": rate,
                          "served": {"jobs_per_s": n / res["span"],
                                     "p50_ms": _pct(res["latency"], 50), "p99_ms": _pct(res["latency"], 99),
                                     "submit_lag_ms": 1e3 * res["submit_lag"]},
                          "plain": {"jobs_per_s": n / plain_span, "p50_ms": _pct(pl, 50), "p99_ms": _pct(pl, 99)}})
        out["rate_sweep"] = sweep
        out["ticks"] = srv.stats()["ticks"]
    out["latency"] = ("finish minus scheduled arrival; plain-path latencies are its measured per-job times "
                      "queued first come, first served at the same arrivals")
    return out


def lib_leaves(tree, codes, depth, flags):
    from b12_b200._lib import check, lib
    check(lib().b12g_leaves(tree._h, codes.ctypes.data, depth.ctypes.data, flags.ctypes.data), "leaves")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--strict", action="store_true",
                    help="headline with the strict (one rounding per operation) integrator instead of explicit FMA")
    ap.add_argument("--single", action="store_true", help="measure only the headline arithmetic")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the Henon, coupled-Duffing continuation and 512-instance batch measurements")
    ap.add_argument("--serve-jobs", type=int, default=10000,
                    help="jobs of the served stream measured against the plain path at 1 GPU (0: skip)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as D
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")) % torch.cuda.device_count())
        # B12_BENCH_BACKEND=gloo runs the ranks' timing collectives on the host (a check of
        # the multi-rank steps on fewer GPUs than ranks; nothing on the data path waits)
        D.init_process_group(os.environ.get("B12_BENCH_BACKEND", "nccl"), timeout=datetime.timedelta(seconds=120))
        dist = D
    try:
        return gpu_arm(args, rank, world, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
