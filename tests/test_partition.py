"""CPU: one tree range-partitioned over ranks (b12_b200.partition) against one oracle tree.

The ranks' runs are held by the oracle (tests/partition_runs.py), either emulated in one
process (drive_lockstep) or as two gloo processes (drive over a process group).  After
every subdivision step the runs, concatenated in rank order, must be the single tree's
leaves (codes, depths, flags), and the rows of the partitioned transition matrix must be
the single tree's matrix, bit for bit."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from b12_b200.partition import PartitionedTree, drive_lockstep, split_leaves
from oracle import oracle as O
from partition_runs import OracleRun, concat_leaves, concat_rows
from workloads import oracle_spec

ROOT = (np.zeros(1, np.uint64), np.zeros(1, np.uint8), np.zeros(1, np.uint8))


class _Scheme:
    """The fields of a scheme the partitioned steps read (the oracle runs hold the map)."""
    flags_to_check = 0
    depth = 255


def _runs(spec, world, leaves=ROOT):
    parts = split_leaves(*leaves, world)
    return [OracleRun(spec, *p) for p in parts]


def _single(spec, steps):
    o = O.Oracle(spec)
    counts, _ = o.subdivision(steps)
    return o, list(counts)


@pytest.mark.parametrize("world,balance", [(1, 1.05), (2, 1.05), (3, 1.0), (4, 1.5)])
def test_subdivision_matches_one_tree(world, balance):
    spec = O.henon_spec()
    steps = 14
    runs = _runs(spec, world)
    trees = [PartitionedTree(r, i, world, balance) for i, r in enumerate(runs)]
    counts = drive_lockstep([t.subdivision(_Scheme(), steps) for t in trees])
    o, want = _single(spec, steps)
    for c in counts:
        assert c == want
    for x, y in zip(concat_leaves(runs), o.leaves()):
        np.testing.assert_array_equal(x, y)
    if balance == 1.0:
        assert max(r.n for r in runs) <= -(-int(want[-1]) // world)


@pytest.mark.parametrize("name,absolute,invalid", [
    ("henon_d12_abs", True, False), ("henon_d12_lost", False, True),
    ("lorenz_rho15_d4_invalid_column_unused", False, True)])
def test_transition_matrix_matches_one_tree(golden, name, absolute, invalid):
    meta, _ = golden(name)
    spec = oracle_spec(meta["spec"])
    steps = len(meta["steps"])
    o, _ = _single(spec, steps)
    for world in (2, 3):
        runs = _runs(spec, world, o.leaves())
        trees = [PartitionedTree(r, i, world) for i, r in enumerate(runs)]
        blocks = drive_lockstep([t.transition_matrix(_Scheme(), absolute, invalid) for t in trees])
        rowptr, cols, vals, n_cols = concat_rows(blocks)
        want = o.transition_matrix(absolute=absolute, invalid=invalid)
        np.testing.assert_array_equal(rowptr, want[0])
        np.testing.assert_array_equal(cols, want[1])
        np.testing.assert_array_equal(vals, want[2])
        assert n_cols == want[3] == meta["tm"]["n_cols"]
        assert [b.row_offset for b in blocks] == list(np.cumsum([0] + [b.n_rows for b in blocks[:-1]]))


def test_runs_of_a_tree_of_several_depths():
    """Leaves of two depths split over three ranks; the steps keep them bit-exact."""
    spec = O.henon_spec()
    o = O.Oracle(spec)
    o.subdivision(10)
    codes, depth, flags = o.leaves()
    mask = np.zeros(len(codes), np.uint8)
    mask[: len(codes) // 3] = 1
    o.unset_flags(0xFF)
    o.set_flags_mask(mask, 0x08)
    o.subdivide(0x08)
    leaves = o.leaves()
    assert len(set(leaves[1].tolist())) == 2
    runs = _runs(spec, 3, leaves)
    trees = [PartitionedTree(r, i, 3) for i, r in enumerate(runs)]
    counts = drive_lockstep([t.subdivision(_Scheme(), 3) for t in trees])
    ref = O.Oracle(spec)
    ref.load(*leaves)
    want, _ = ref.subdivision(3)
    assert counts[0] == list(want)
    for x, y in zip(concat_leaves(runs), ref.leaves()):
        np.testing.assert_array_equal(x, y)


def test_surrounding_box_comes_back_when_every_leaf_is_lost():
    """Every image leaves the domain: the tree becomes its surrounding box, on rank 0."""
    spec = O.henon_spec()
    spec["center"] = [10.0, 0.0]
    spec["radius"] = [1.0, 1.0]
    runs = _runs(spec, 3)
    trees = [PartitionedTree(r, i, 3) for i, r in enumerate(runs)]
    counts = drive_lockstep([t.subdivision(_Scheme(), 3) for t in trees])
    o, want = _single(spec, 3)
    assert counts[0] == want == [1, 1, 1]
    assert sorted(r.n for r in runs) == [0, 0, 1]
    for x, y in zip(concat_leaves(runs), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_ranks_must_take_the_same_steps():
    spec = O.henon_spec()
    runs = _runs(spec, 2)
    trees = [PartitionedTree(r, i, 2) for i, r in enumerate(runs)]
    with pytest.raises(RuntimeError):
        drive_lockstep([trees[0].subdivision(_Scheme(), 2), trees[1].subdivision(_Scheme(), 3)])


# ----------------------------------------------------------------------------- two gloo ranks
def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    from b12_b200.partition import ProcessGroupExchange, drive
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        spec = O.lorenz_spec()
        run = _runs(spec, world)[rank]
        t = PartitionedTree(run, rank, world)
        ex = ProcessGroupExchange(dist, "cpu")
        counts = drive(t.subdivision(_Scheme(), 12), ex)
        block = drive(t.transition_matrix(_Scheme(), False, True), ex)
        codes, depth, flags = run.host_leaves()
        out[rank] = dict(counts=counts, codes=codes.tobytes(), depth=depth.tobytes(), flags=flags.tobytes(),
                         rows=[np.asarray(x).tobytes() for x in block.rows[:3]] if block.rows else None,
                         n_cols=block.n_cols, row_offset=block.row_offset, n_rows=block.n_rows)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_one_tree():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    o, want = _single(O.lorenz_spec(), 12)
    assert res[0]["counts"] == res[1]["counts"] == want
    codes = np.concatenate([np.frombuffer(res[r]["codes"], np.uint64) for r in range(world)])
    depth = np.concatenate([np.frombuffer(res[r]["depth"], np.uint8) for r in range(world)])
    flags = np.concatenate([np.frombuffer(res[r]["flags"], np.uint8) for r in range(world)])
    for x, y in zip((codes, depth, flags), o.leaves()):
        np.testing.assert_array_equal(x, y)
    rp, cols, vals, nc = o.transition_matrix(invalid=True)
    got_cols = np.concatenate([np.frombuffer(res[r]["rows"][1], np.uint32) for r in range(world) if res[r]["rows"]])
    got_vals = np.concatenate([np.frombuffer(res[r]["rows"][2], np.float64) for r in range(world) if res[r]["rows"]])
    np.testing.assert_array_equal(got_cols, cols)
    np.testing.assert_array_equal(got_vals, vals)
    assert res[0]["n_cols"] == res[1]["n_cols"] == nc
    assert res[1]["row_offset"] == res[0]["n_rows"]
