"""GPU: the entry points of a range-partitioned tree through the C ABI against the oracle,
and the partitioned subdivision and transition matrix (ranks emulated in one process on
one GPU, their collectives answered on the host between launches) against one tree.

Point boxes, leaf indices, flags, rows, leaf counts and matrices must be bit-exact."""
import numpy as np
import pytest

from oracle import oracle as O
from workloads import domain, oracle_spec, scheme, sha

pytestmark = pytest.mark.gpu

B = pytest.importorskip("b12_b200")


@pytest.fixture(scope="module", autouse=True)
def _device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _tree(spec):
    c, r = domain(spec)
    return B.ImplicitBoxTree(c, r)


def _grown(name, golden, steps=None):
    meta, _ = golden(name)
    spec = meta["spec"]
    t = _tree(spec)
    sc = scheme(spec)
    k = len(meta["steps"]) if steps is None else steps
    t.subdivision_run(sc, k)
    o = O.Oracle(oracle_spec(spec))
    o.load(*t.leaves())
    return meta, spec, t, sc, o


@pytest.mark.parametrize("name", ["henon_d12_lost", "lorenz_d15"])
def test_point_box_entries_match_oracle(golden, name):
    import torch
    _, spec, t, sc, o = _grown(name, golden)
    codes, valid = t.image_point_boxes(sc, "cuda")
    oc, ov = o.image_point_boxes()
    np.testing.assert_array_equal(codes.cpu().numpy().view(np.uint64), oc)
    np.testing.assert_array_equal(valid.cpu().numpy(), ov)
    assert (ov == 0).any() or name == "lorenz_d15"
    # search and flags over the same point boxes
    idx = t.search_point_boxes(codes, valid).cpu().numpy()
    want = o.search_point_boxes(oc, ov).astype(np.int64)
    want[want == 0xFFFFFFFF] = -1
    np.testing.assert_array_equal(idx, want)
    half = codes.numel() // 2
    assert t.set_flags_by_point_boxes(codes[:half], valid[:half], B.EQU) == \
        o.set_flags_by_point_boxes(oc[:half], ov[:half], 0x10)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)
    # rows from the targets equal the tree's own matrix
    P = sc.grid.points_per_box(t.dim)
    for invalid in (False, True):
        m = t.transition_rows(torch.from_numpy(want).cuda(), P, t.count(), False, invalid)
        ref = t.transition_matrix(sc, invalid_column=invalid)
        for x, y in zip(m.to_host(), ref.to_host()):
            np.testing.assert_array_equal(x, y)
        assert m.n_cols == ref.n_cols
        m.close()
        ref.close()


@pytest.mark.parametrize("name", ["henon_d12_lost", "lorenz_d15"])
def test_distinct_point_boxes_are_the_set_of_the_point_boxes(golden, name):
    """The image boxes as a set (each warp's distinct boxes once): the same set of
    (code, validity) pairs as every point's box, each at most once per 32 points, and the
    same flags set from them."""
    _, spec, t, sc, o = _grown(name, golden)
    oc, ov = o.image_point_boxes()
    codes, valid = t.image_distinct_point_boxes(sc, "cuda")
    dc, dv = codes.cpu().numpy().view(np.uint64), valid.cpu().numpy()
    assert set(zip(dc.tolist(), dv.tolist())) == set(zip(oc.tolist(), ov.tolist()))
    assert len(dc) <= len(oc)
    # no pair twice within one group of 32 consecutive points: at most as many entries
    # as the groups' distinct pairs summed
    groups = sum(len(set(zip(oc[i:i + 32].tolist(), ov[i:i + 32].tolist()))) for i in range(0, len(oc), 32))
    assert len(dc) <= groups
    assert t.set_flags_by_point_boxes(codes, valid, B.EQU) == o.set_flags_by_point_boxes(oc, ov, 0x10)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)
    # cut to the leaves' depth: far fewer boxes, the same leaves hit
    d = t.depth()
    keep = ~np.uint64(0) if d >= 64 else ~np.uint64((1 << (64 - d)) - 1)
    cc, cv = t.image_distinct_point_boxes(sc, "cuda", d)
    hc, hv = cc.cpu().numpy().view(np.uint64), cv.cpu().numpy()
    want = set(zip(np.where(ov != 0, oc & keep, oc).tolist(), ov.tolist()))
    assert set(zip(hc.tolist(), hv.tolist())) == want
    assert len(hc) < len(oc) // 4
    t.unset_flags(B.EQU)
    o.unset_flags(0x10)
    assert t.set_flags_by_point_boxes(cc, cv, B.EQU) == o.set_flags_by_point_boxes(oc, ov, 0x10)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_point_boxes_of_a_tree_of_several_depths(golden):
    meta, arrays = golden("henon_d14_mixed8")
    spec = meta["spec"]
    t = _tree(spec)
    t.load_leaves(arrays["mixed_codes_00"], arrays["mixed_depth_00"], arrays["mixed_flags_00"])
    t.subdivide(B.SD)
    o = O.Oracle(oracle_spec(spec))
    o.load(*t.leaves())
    assert len(set(t.leaves()[1].tolist())) == 2
    sc = scheme(spec)
    codes, valid = t.image_point_boxes(sc, "cuda")
    oc, ov = o.image_point_boxes()
    np.testing.assert_array_equal(codes.cpu().numpy().view(np.uint64), oc)
    idx = t.search_point_boxes(codes, valid).cpu().numpy()
    want = o.search_point_boxes(oc, ov).astype(np.int64)
    want[want == 0xFFFFFFFF] = -1
    np.testing.assert_array_equal(idx, want)
    assert len(set(t.leaves()[1].tolist())) == 2      # still a tree of two depths


def test_leaves_through_device_buffers(golden):
    import torch
    _, spec, t, sc, o = _grown("henon_d12_lost", golden)
    c, d, f = t.leaves_device("cuda")
    u = _tree(spec)
    u.load_leaves_device(c, d, f)
    for x, y in zip(u.leaves(), t.leaves()):
        np.testing.assert_array_equal(x, y)
    # out of order: refused on the device, the tree is its surrounding box
    with pytest.raises(B.B12gError):
        u.load_leaves_device(torch.flip(c, [0]).contiguous(), d, f)
    assert u.count() == 1 and u.depth() == 0
    # a run of two depths keeps them
    codes, depth, flags = t.leaves()
    depth = depth.copy()
    codes = codes.copy()
    codes[0] >>= np.uint64(1)
    depth[0] -= 1
    ok = codes[0] != codes[1] >> np.uint64(1)
    if ok:
        u.load_leaves_device(torch.from_numpy(codes.view(np.int64)).cuda(), torch.from_numpy(depth).cuda(),
                             torch.from_numpy(flags).cuda())
        for x, y in zip(u.leaves(), (codes, depth, flags)):
            np.testing.assert_array_equal(x, y)


def _partitioned(spec, world, leaves=None):
    from b12_b200.partition import DeviceRun, PartitionedTree, split_leaves
    if leaves is None:
        leaves = (np.zeros(1, np.uint64), np.zeros(1, np.uint8), np.zeros(1, np.uint8))
    runs = []
    for part in split_leaves(*leaves, world):
        r = DeviceRun(_tree(spec), "cuda")
        if len(part[0]):
            r.tree.load_leaves(*part)
        else:
            r.empty = True
        runs.append(r)
    return runs, [PartitionedTree(r, i, world) for i, r in enumerate(runs)]


def _concat(runs):
    parts = [r.host_leaves() for r in runs]
    return tuple(np.concatenate([p[k] for p in parts]) for k in range(3))


@pytest.mark.parametrize("name,world", [("henon_d20", 2), ("lorenz_d15", 3), ("forced_duffing_d16", 4)])
def test_partitioned_subdivision_matches_reference(golden, name, world):
    from b12_b200.partition import drive_lockstep
    meta, _ = golden(name)
    spec = meta["spec"]
    steps = len(meta["steps"])
    runs, trees = _partitioned(spec, world)
    counts = drive_lockstep([t.subdivision(scheme(spec), steps) for t in trees])
    assert counts[0] == [s["n"] for s in meta["steps"]]
    codes, depth, flags = _concat(runs)
    assert sha(codes) == meta["steps"][-1]["codes_sha256"]
    assert sha(flags) == meta["steps"][-1]["flags_sha256"]
    assert max(r.n for r in runs) <= 1.05 * len(codes) / world + 1


@pytest.mark.parametrize("name,absolute,invalid", [
    ("henon_d20", False, False), ("henon_d12_lost", False, True), ("lorenz_d15", False, False),
    ("lorenz_rho15_d4_invalid_column_unused", False, True)])
def test_partitioned_transition_matrix_matches_reference(golden, name, absolute, invalid):
    from b12_b200.partition import drive_lockstep
    from workloads import csr_digests
    meta, _ = golden(name)
    spec = meta["spec"]
    t = _tree(spec)
    t.subdivision_run(scheme(spec), len(meta["steps"]))
    for world in (2, 3):
        runs, trees = _partitioned(spec, world, t.leaves())
        blocks = drive_lockstep([p.transition_matrix(scheme(spec), absolute, invalid) for p in trees])
        rowptr, cols, vals, base = [np.zeros(1, np.uint64)], [], [], 0
        for b in blocks:
            rp, c, v = b.rows.to_host()
            rowptr.append(rp[1:].astype(np.uint64) + base)
            base += int(rp[-1])
            cols.append(c)
            vals.append(v)
            b.rows.close()
        d = csr_digests(np.concatenate(rowptr).astype(np.uint32), np.concatenate(cols), np.concatenate(vals))
        for k in ("nnz", "rowptr_sha256", "cols_sha256", "vals_sha256"):
            assert d[k] == meta["tm"][k], k
        assert blocks[0].n_cols == meta["tm"]["n_cols"]


def test_partitioned_run_over_an_nccl_group_of_one(golden):
    """The process-group driver with NCCL collectives (one rank on this GPU): the same
    steps as the emulated ranks, through torch.distributed."""
    import socket
    import datetime
    import torch.distributed as dist
    from b12_b200.partition import ProcessGroupExchange, drive
    from workloads import csr_digests
    meta, _ = golden("lorenz_d15")
    spec = meta["spec"]
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        runs, trees = _partitioned(spec, 1)
        ex = ProcessGroupExchange(dist, "cuda")
        counts = drive(trees[0].subdivision(scheme(spec), len(meta["steps"])), ex)
        assert counts == [s["n"] for s in meta["steps"]]
        assert sha(runs[0].host_leaves()[0]) == meta["steps"][-1]["codes_sha256"]
        block = drive(trees[0].transition_matrix(scheme(spec)), ex)
        d = csr_digests(*block.rows.to_host())
        for k in ("nnz", "rowptr_sha256", "cols_sha256", "vals_sha256"):
            assert d[k] == meta["tm"][k], k
        block.rows.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n_runs", [(2, 2), (4, 3), (300, 17)])
def test_route_point_boxes_matches_a_stable_partition(world, n_runs):
    """b12g_route_point_boxes against the definition: owner = the last run whose first
    code is at or below the box (unsigned order), the last run for a box outside the
    domain; the boxes grouped by owner, stable within each owner."""
    import torch
    rng = np.random.default_rng(world)
    n = 100_003
    codes = rng.integers(0, 2**63, n, dtype=np.int64).view(np.uint64) * np.uint64(2) + rng.integers(
        0, 2, n).astype(np.uint64)
    valid = (rng.random(n) > 0.05).astype(np.uint8)
    ranks = np.sort(rng.choice(world, n_runs, replace=False)).astype(np.uint32)
    starts = np.sort(rng.integers(1, 2**63, n_runs - 1, dtype=np.int64).view(np.uint64) * np.uint64(2))
    starts = np.concatenate([[np.uint64(0)], starts]).astype(np.uint64)
    pos = np.searchsorted(starts, codes, side="right") - 1
    owner = np.where(valid != 0, ranks[pos], ranks[-1])
    order = np.argsort(owner, kind="stable")
    t = B.ImplicitBoxTree([0.0, 0.0], [1.0, 1.0])
    d_codes = torch.from_numpy(codes.view(np.int64)).cuda()
    d_valid = torch.from_numpy(valid).cuda()
    slot, c_parts, v_parts = t.route_point_boxes(d_codes, d_valid, starts, ranks, world)
    assert [p.numel() for p in c_parts] == np.bincount(owner, minlength=world).tolist()
    got_c = torch.cat(c_parts).cpu().numpy().view(np.uint64)
    got_v = torch.cat(v_parts).cpu().numpy()
    np.testing.assert_array_equal(got_c, codes[order])
    np.testing.assert_array_equal(got_v, valid[order])
    inv = np.empty(n, dtype=np.int64)
    inv[order] = np.arange(n)
    np.testing.assert_array_equal(slot.cpu().numpy(), inv)
