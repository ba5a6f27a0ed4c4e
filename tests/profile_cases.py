"""Single workloads sized for an ncu capture of one kernel family on one GPU (profiling
infrastructure, not part of the library).

    python tests/profile_cases.py <case> [options]

image     a Lorenz tree subdivided to --depth - 1 (default 23), then one subdivide and
          one set_flags_by_image with the strict and one with the explicit-FMA integrator:
          two launches of the fused box-image kernel over the same 2n boxes.
compact   64 Lorenz instances (rho = 28, explicit FMA) batched to depth 27: the last
          steps compact ~20 M children (code 8 B + flags 1 B + hit 1 B each), well
          beyond the 126 MB L2, so the compaction's DRAM traffic is meaningful.
continuation
          the coupled-Duffing continuation at depth 24 (64 Philox points per box) over
          the bitmap of the depth's boxes.
sort      --points uniform random 4-D points inserted at depth 24 into the boxes of 12
          sweeps of that continuation: the candidate codes of the points in no leaf
          are radix-sorted (one histogram pass, three digit passes), made unique and
          merged into the leaves.
measure   one Lorenz job to --depth (default 27), its transition matrix and 200 power
          iterations; depth 32 gives ~2.6 M boxes, a matrix of ~0.25 GB (HBM-bound SpMV).
serve     a burst of --jobs served-stream jobs through the job server.
mixed     a Lorenz tree (explicit FMA) refined to --depth (default 21), SD kept on the
          lower half in x, four selective steps (leaves of depths d..d+4), then one more
          subdivide and set_flags_by_image: the per-leaf-depth image kernel over the tree.
partition one Lorenz job to --depth (default 27) over --world ranks emulated in one
          process, against the fused single-tree loop (times of both, same results).

Every case prints one line of sizes; none writes files.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np


def case_image(args):
    import b12_b200 as B
    from b12_b200.workloads import LORENZ_CENTER, LORENZ_RADIUS
    t = B.ImplicitBoxTree(LORENZ_CENTER, LORENZ_RADIUS)
    strict = B.Scheme(B.lorenz(), B.inner_grid(5))
    fma = B.Scheme(B.lorenz(fma=True), B.inner_grid(5))
    t.subdivision_run(strict, args.depth - 1)
    t.subdivide(B.SD)
    n = t.count()
    a = t.set_flags_by_image(strict, B.HIT)
    t.unset_flags(B.HIT)
    b = t.set_flags_by_image(fma, B.HIT)
    print(f"image: {n} boxes at depth {args.depth}, {n * 125} points per launch, hits {a} / {b}")
    t.close()


def case_compact(args):
    import b12_b200 as B
    from b12_b200.workloads import LORENZ_CENTER, LORENZ_RADIUS
    n = args.instances
    b = B.Batch(LORENZ_CENTER, LORENZ_RADIUS, B.Scheme(B.lorenz(fma=True), B.inner_grid(5)),
                [(10.0, 28.0, 8.0 / 3.0)] * n, [args.depth] * n)
    b.run()                       # first run: autotunes the launch shape
    # the second run (one CUDA graph, 27 steps) inside a profiler range: capture it with
    # ncu --profile-from-start off
    import torch
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    t0 = time.perf_counter()
    b.run()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    info = b.info()
    print(f"compact: {n} instances depth {args.depth}: {info['final_boxes']} final boxes, "
          f"{info['box_images']} box-images, {time.perf_counter() - t0:.3f} s (second run)")
    b.close()


def case_continuation(args):
    import b12_b200 as B
    t = B.ImplicitBoxTree((0.0,) * 4, (2.0,) * 4)
    t.reserve(16 << 20)
    sc = B.Scheme(B.coupled_duffing(), B.philox_grid(64, 0))
    t0 = time.perf_counter()
    sweeps = t.continuation_run(sc, np.zeros(4), args.depth)
    print(f"continuation: depth {args.depth}: {int(sweeps[-1])} boxes in {len(sweeps)} sweeps, "
          f"{time.perf_counter() - t0:.3f} s")
    t.close()


def case_sort(args):
    import b12_b200 as B
    t = B.ImplicitBoxTree((0.0,) * 4, (2.0,) * 4)
    sc = B.Scheme(B.coupled_duffing(), B.philox_grid(64, 0))
    sweeps = t.continuation_run(sc, np.zeros(4), args.depth, max_sweeps=12)
    rng = np.random.default_rng(0)
    pts = rng.uniform(-2.0, 2.0, size=(args.points, 4))
    t0 = time.perf_counter()
    new = t.insert_points(pts, args.depth, B.INS, B.NONE)
    print(f"sort: {args.points} random points into {int(sweeps[-1])} boxes of depth {args.depth} "
          f"(12 continuation sweeps): {new} new boxes, {time.perf_counter() - t0:.3f} s")
    t.close()


def case_measure(args):
    import b12_b200 as B
    from b12_b200.workloads import LORENZ_CENTER, LORENZ_RADIUS
    t = B.ImplicitBoxTree(LORENZ_CENTER, LORENZ_RADIUS)
    sc = B.Scheme(B.lorenz(fma=True), B.inner_grid(5))
    counts = t.subdivision_run(sc, args.depth)
    m = t.transition_matrix(sc)
    t.close()                     # the matrix owns its memory; only it stays on the device
    v = m.invariant_measure(200)          # first call: builds P^T
    t0 = time.perf_counter()
    for _ in range(args.repeat):
        m.invariant_measure(200, keep_on_device=True)
    m.measure(v)
    print(f"measure: depth {args.depth}: {int(counts[-1])} boxes, {m.nnz} nonzeros, sum {v.sum():.15f}, "
          f"{1e3 * (time.perf_counter() - t0) / max(args.repeat, 1):.3f} ms per 200 iterations")
    m.close()


def case_serve(args):
    from b12_b200.server import JobServer, replay
    from b12_b200.workloads import job_stream
    with JobServer(150 * 10**9) as srv:
        warm = [dict(j, arrival=0.0) for j in job_stream(60, 1.0, 1)]
        replay(srv, warm, lambda job, jid: srv.release(jid))
        burst = [dict(j, arrival=0.0) for j in job_stream(args.jobs, 1.0, 0)]
        res = replay(srv, burst, lambda job, jid: srv.release(jid))
        print(f"serve: {args.jobs} jobs in {res['span']:.3f} s, {srv.stats()['ticks']} ticks")


def case_mixed(args):
    import b12_b200 as B
    from b12_b200.workloads import LORENZ_CENTER, LORENZ_RADIUS
    t = B.ImplicitBoxTree(LORENZ_CENTER, LORENZ_RADIUS)
    sc = B.Scheme(B.lorenz(fma=True), B.inner_grid(5))
    t.subdivision_run(sc, args.depth)
    codes, depth, flags = t.leaves()
    lower = (codes >> np.uint64(args.depth - 1)) == 0
    t.load_leaves(codes, depth, ((flags & ~np.uint8(B.SD)) | np.where(lower, B.SD, 0)).astype(np.uint8))
    for _ in range(5):
        t.subdivide(B.SD)
        n = t.count()
        hits = t.set_flags_by_image(sc, B.HIT)
        t.remove(B.HIT)
        t.unset_flags(B.HIT)
    d = t.leaves()[1]
    print(f"mixed: last image launch over {n} boxes ({n * 125} points), {hits} hit; depths {d.min()}-{d.max()}")
    t.close()


def case_partition(args):
    """One Lorenz job (explicit FMA) to --depth split over --world ranks emulated in this
    process (their collectives answered on the host between launches), against the fused
    single-tree loop: the same leaves and matrix, and the time of each."""
    import torch
    import b12_b200 as B
    from b12_b200.partition import DeviceRun, PartitionedTree, drive_lockstep
    from b12_b200.workloads import LORENZ_CENTER, LORENZ_RADIUS
    sc = B.Scheme(B.lorenz(fma=True), B.inner_grid(5))
    res = {}
    for rep in range(2):                   # the second repetition is timed
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        t = B.ImplicitBoxTree(LORENZ_CENTER, LORENZ_RADIUS)
        counts = t.subdivision_run(sc, args.depth)
        m = t.transition_matrix(sc)
        fused = time.perf_counter() - t0
        nnz_fused = m.nnz
        m.close()
        runs = [DeviceRun(B.ImplicitBoxTree(LORENZ_CENTER, LORENZ_RADIUS), "cuda") for _ in range(args.world)]
        for r in runs[1:]:
            r.empty = True
        parts = [PartitionedTree(r, i, args.world) for i, r in enumerate(runs)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pc = drive_lockstep([p.subdivision(sc, args.depth) for p in parts])
        blocks = drive_lockstep([p.transition_matrix(sc) for p in parts])
        torch.cuda.synchronize()
        split = time.perf_counter() - t0
        nnz = sum(b.rows.nnz for b in blocks if b.rows is not None)
        assert list(pc[0]) == [int(c) for c in counts] and nnz == nnz_fused
        res = dict(fused=fused, split=split, boxes=int(counts[-1]), nnz=nnz)
        for b in blocks:
            if b.rows is not None:
                b.rows.close()
        for r in runs:
            r.tree.close()
        t.close()
    print(f"partition: Lorenz depth {args.depth}, {res['boxes']} boxes, {res['nnz']} nonzeros: fused single tree "
          f"{1e3 * res['fused']:.1f} ms (fresh tree), {args.world} emulated ranks {1e3 * res['split']:.1f} ms")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["image", "compact", "continuation", "sort", "measure", "serve", "mixed",
                                     "partition"])
    ap.add_argument("--points", type=int, default=8 << 20, help="sort: random points inserted")
    ap.add_argument("--depth", type=int, default=None)
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--jobs", type=int, default=300)
    ap.add_argument("--repeat", type=int, default=1, help="measure: timed calls after the first")
    ap.add_argument("--world", type=int, default=2, help="partition: emulated ranks")
    args = ap.parse_args()
    if args.depth is None:
        args.depth = {"image": 23, "compact": 27, "continuation": 24, "sort": 24, "measure": 27, "serve": 0,
                      "mixed": 21, "partition": 27}[args.case]
    {"image": case_image, "compact": case_compact, "continuation": case_continuation, "sort": case_sort, "measure": case_measure,
     "serve": case_serve, "mixed": case_mixed, "partition": case_partition}[args.case](args)


if __name__ == "__main__":
    main()
