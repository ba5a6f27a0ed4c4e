"""GPU: the batched subdivision (many instances, one persistent launch per step) gives
every instance exactly the single-tree result - leaf codes, flags, per-step counts and
transition matrices bit-exact - and the reference's golden runs."""
import numpy as np
import pytest

from workloads import csr_digests, sha

pytestmark = pytest.mark.gpu

B = pytest.importorskip("b12_b200")
from b12_b200.workloads import LORENZ_CENTER, LORENZ_RADIUS, lorenz_scan  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def single(center, radius, mp, grid, depth):
    t = B.ImplicitBoxTree(center, radius)
    sc = B.Scheme(mp, grid)
    counts = t.subdivision_run(sc, depth)
    m = t.transition_matrix(sc)
    return counts, t.leaves(), m.to_host()


@pytest.mark.parametrize("fma", [False, True])
def test_lorenz_batch_matches_single_trees(fma):
    rho, _ = lorenz_scan(12, 0)
    depths = [8, 14, 11, 9, 12, 14, 10, 13, 9, 12, 8, 11]
    params = [(10.0, r, 8.0 / 3.0) for r in rho]
    grid = B.inner_grid(5)
    b = B.Batch(LORENZ_CENTER, LORENZ_RADIUS, B.Scheme(B.lorenz(fma=fma), grid), params, depths)
    b.run()
    b.transition_matrices()
    for i in range(12):
        counts, leaves, csr = single(LORENZ_CENTER, LORENZ_RADIUS, B.lorenz(rho=rho[i], fma=fma), grid, depths[i])
        np.testing.assert_array_equal(b.counts(i), counts)
        for x, y in zip(b.leaves(i), leaves):
            np.testing.assert_array_equal(x, y)
        for x, y in zip(b.csr(i), csr):
            np.testing.assert_array_equal(x, y)


def test_batch_replays_identically_and_reports_tuning():
    rho, depth = lorenz_scan(40, 3)
    depth = [min(d, 16) for d in depth]
    b = B.Batch(LORENZ_CENTER, LORENZ_RADIUS, B.Scheme(B.lorenz(fma=True), B.inner_grid(5)),
                [(10.0, r, 8.0 / 3.0) for r in rho], depth)
    b.run()
    first = [b.leaves(i)[0].copy() for i in range(40)]
    b.run()
    for i in range(40):
        np.testing.assert_array_equal(b.leaves(i)[0], first[i])
    info = b.info()
    assert info["threads"] in (128, 256, 512) and info["points_per_thread"] in (1, 2)
    assert info["final_boxes"] == sum(len(f) for f in first)


def test_batch_members_match_reference_goldens(golden):
    metas = [golden("lorenz_rho15_d18")[0], golden("lorenz_rho35_d18")[0], golden("lorenz_d15")[0]]
    params = [(10.0, m["spec"]["rho"], 8.0 / 3.0) for m in metas]
    depths = [len(m["steps"]) for m in metas]
    b = B.Batch(LORENZ_CENTER, LORENZ_RADIUS, B.Scheme(B.lorenz(), B.inner_grid(5)), params, depths)
    b.run()
    b.transition_matrices()
    for i, m in enumerate(metas):
        assert list(b.counts(i)) == [s["n"] for s in m["steps"]]
        codes, _, flags = b.leaves(i)
        assert sha(codes) == m["steps"][-1]["codes_sha256"] and sha(flags) == m["steps"][-1]["flags_sha256"]
        d = csr_digests(*b.csr(i))
        for k in ("nnz", "rowptr_sha256", "cols_sha256", "vals_sha256"):
            assert d[k] == m["tm"][k], (i, k)


def test_henon_batch_matches_single_trees():
    a_vals = [1.0, 1.1, 1.2, 1.3, 1.4, 1.05]
    depths = [14, 12, 16, 10, 15, 13]
    grid = B.inner_grid(4)
    b = B.Batch((0.0, 0.0), (1.5, 0.45), B.Scheme(B.henon(), grid), [(a, 0.3) for a in a_vals], depths)
    b.run()
    b.transition_matrices()
    for i, a in enumerate(a_vals):
        counts, leaves, csr = single((0.0, 0.0), (1.5, 0.45), B.henon(a, 0.3), grid, depths[i])
        np.testing.assert_array_equal(b.counts(i), counts)
        np.testing.assert_array_equal(b.leaves(i)[0], leaves[0])
        for x, y in zip(b.csr(i), csr):
            np.testing.assert_array_equal(x, y)


def test_forced_duffing_batch_matches_single_trees_and_reference(golden):
    # the two-dimensional maps run several points per thread, interleaved: every point's
    # operations stay those of the single-point integrator
    from b12_b200.workloads import FORCED_CENTER, FORCED_RADIUS
    meta = golden("forced_duffing_d16")[0]
    params = [(0.25, -1.0, 1.0, 0.3), (0.2, -1.0, 1.0, 0.3), (0.25, -1.0, 1.0, 0.35), (0.3, -1.0, 1.0, 0.25)]
    depths = [len(meta["steps"]), 12, 14, 11]
    grid = B.inner_grid(4)
    b = B.Batch(FORCED_CENTER, FORCED_RADIUS, B.Scheme(B.forced_duffing(), grid), params, depths)
    b.run()
    b.transition_matrices()
    assert list(b.counts(0)) == [s["n"] for s in meta["steps"]]
    codes, _, flags = b.leaves(0)
    assert sha(codes) == meta["steps"][-1]["codes_sha256"] and sha(flags) == meta["steps"][-1]["flags_sha256"]
    d = csr_digests(*b.csr(0))
    for k in ("nnz", "rowptr_sha256", "cols_sha256", "vals_sha256"):
        assert d[k] == meta["tm"][k], k
    for i in range(1, 4):
        counts, leaves, csr = single(FORCED_CENTER, FORCED_RADIUS, B.forced_duffing(200, *params[i]), grid, depths[i])
        np.testing.assert_array_equal(b.counts(i), counts)
        np.testing.assert_array_equal(b.leaves(i)[0], leaves[0])
        for x, y in zip(b.csr(i), csr):
            np.testing.assert_array_equal(x, y)


def test_full_lorenz_scan_512_matches_single_trees_and_reference(golden):
    """The configured batch: 512 Lorenz instances (rho ~ U[15,35], depth 18-27 from
    SplitMix64 seed 0, explicit-FMA map, 125-point grid), one persistent launch per step.
    Every instance equals its own single-tree run (per-step counts, leaf codes and flags,
    CSR bit for bit), and four instances run one at a time by the reference (two of
    depth 27, one of 24, one of 21) give the reference's digests."""
    rho, depth = lorenz_scan(512, 0)
    grid = B.inner_grid(5)
    b = B.Batch(LORENZ_CENTER, LORENZ_RADIUS, B.Scheme(B.lorenz(fma=True), grid),
                [(10.0, r, 8.0 / 3.0) for r in rho], depth)
    b.run()
    b.transition_matrices()
    total = 0
    tree = B.ImplicitBoxTree(LORENZ_CENTER, LORENZ_RADIUS)
    for i in range(512):
        sc = B.Scheme(B.lorenz(rho=rho[i], fma=True), grid)
        tree.delete_depth(0)
        counts = tree.subdivision_run(sc, depth[i])
        np.testing.assert_array_equal(b.counts(i), counts, err_msg=str(i))
        codes, _, flags = b.leaves(i)
        scodes, _, sflags = tree.leaves()
        assert sha(codes) == sha(scodes) and sha(flags) == sha(sflags), i
        m = tree.transition_matrix(sc)
        assert csr_digests(*b.csr(i)) == csr_digests(*m.to_host()), i
        m.close()
        total += len(codes)
    assert total == b.info()["final_boxes"]
    for name in ("lorenz_scan0_i1_d27_fma", "lorenz_scan0_i14_d27_fma", "lorenz_scan0_i10_d24_fma",
                 "lorenz_scan0_i2_d21_fma"):
        meta = golden(name)[0]
        i = meta["spec"]["scan_index"]
        assert meta["spec"]["rho"] == rho[i] and meta["spec"]["steps"] == depth[i]
        assert list(b.counts(i)) == [s["n"] for s in meta["steps"]], name
        codes, _, flags = b.leaves(i)
        assert sha(codes) == meta["steps"][-1]["codes_sha256"], name
        assert sha(flags) == meta["steps"][-1]["flags_sha256"], name
        d = csr_digests(*b.csr(i))
        for k in ("nnz", "rowptr_sha256", "cols_sha256", "vals_sha256"):
            assert d[k] == meta["tm"][k], (name, k)
