"""GPU parity of the unstable-manifold continuation (continuation.m:13-44) and of box
insertion (insertByPoints / insertByIterators) against the reference's golden runs
and the oracle: leaf codes, flags and per-sweep counts bit-exact."""
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


def make_tree(spec):
    c, r = domain(spec)
    return B.ImplicitBoxTree(c, r)


@pytest.mark.parametrize("name", ["coupled_duffing_cont_d8", "coupled_duffing_cont_d12", "coupled_duffing_cont_d24"])
def test_continuation_run_matches_reference(golden, name):
    meta, _ = golden(name)
    spec = meta["spec"]
    t = make_tree(spec)
    counts = t.continuation_run(scheme(spec), np.zeros(4), spec["depth"])
    ref = [s for s in meta["steps"] if s["step"] > 0]
    assert list(counts) == [s["n"] for s in ref]
    codes, depth, flags = t.leaves()
    assert sha(codes) == ref[-1]["codes_sha256"]
    assert sha(flags) == ref[-1]["flags_sha256"]
    assert (depth == spec["depth"]).all()


@pytest.mark.parametrize("name", ["coupled_duffing_cont_d8", "coupled_duffing_cont_d24"])
def test_continuation_step_api_matches_reference_each_sweep(golden, name):
    """Every sweep's leaf codes and flags, through the step-by-step API (at depth 24: 49
    sweeps up to 9,910,846 boxes, the configured continuation)."""
    meta, _ = golden(name)
    spec = meta["spec"]
    d = spec["depth"]
    t = make_tree(spec)
    sc = scheme(spec, depth=d, flags_to_check=B.EXPD)
    assert t.delete_depth(0) == 1
    assert t.insert_points(np.zeros(4), d, B.INS, B.NONE) == 1
    for st in meta["steps"]:
        if st["step"] > 0:
            t.change_flags(B.INS, B.EXPD, d)
            t.insert_by_image(sc, d, B.INS, B.NONE)
            t.unset_flags(B.EXPD)
        codes, _, flags = t.leaves()
        assert len(codes) == st["n"], st["step"]
        assert sha(codes) == st["codes_sha256"] and sha(flags) == st["flags_sha256"], st["step"]


@pytest.mark.parametrize("sweeps", [1, 7, 30])
def test_continuation_cut_short_matches_reference_at_that_sweep(golden, sweeps):
    """max_sweeps ends the run while boxes are still being added: the leaves and flags
    (INS on the last sweep's new boxes) of that sweep of the reference's run."""
    meta, _ = golden("coupled_duffing_cont_d24")
    spec = meta["spec"]
    t = make_tree(spec)
    counts = t.continuation_run(scheme(spec), np.zeros(4), spec["depth"], max_sweeps=sweeps)
    ref = [s for s in meta["steps"] if 0 < s["step"] <= sweeps]
    assert list(counts) == [s["n"] for s in ref]
    codes, _, flags = t.leaves()
    assert sha(codes) == ref[-1]["codes_sha256"] and sha(flags) == ref[-1]["flags_sha256"]
    assert (flags == B.INS).sum() == ref[-1]["n"] - (ref[-2]["n"] if len(ref) > 1 else 1)


@pytest.mark.parametrize("depth", [31, 40])
def test_continuation_deeper_than_the_bitmap_matches_oracle(depth):
    """Depths above the box bitmap's (30) take the lookup-table sweeps."""
    spec = dict(map="coupled_duffing", points=64, seed=0)
    t = make_tree(spec)
    counts = t.continuation_run(scheme(spec), np.zeros(4), depth, max_sweeps=6)
    o, oc = O.continuation(oracle_spec(spec), depth, np.zeros(4), max_sweeps=6)
    assert list(counts) == oc
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_henon_continuation_matches_oracle():
    """A two-dimensional continuation (the Henon map from its fixed point) to the end."""
    spec = dict(map="henon", a=1.4, b=0.3, grid=4)
    x0 = np.array([0.6313544770895048, 0.18940634312685142])
    t = make_tree(spec)
    counts = t.continuation_run(scheme(spec), x0, 16)
    o, oc = O.continuation(oracle_spec(spec), 16, x0)
    assert list(counts) == oc and len(oc) > 3
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("fma", [False, True])
def test_lorenz_continuation_matches_oracle(fma):
    """A three-dimensional continuation (Lorenz, inner grid 3^3) from a point near the
    attractor: the box bitmap's 3-D code assembly and the leaves it writes."""
    spec = dict(map="lorenz", rho=28.0, fma=fma, grid=3)
    x0 = np.array([[-8.5, -8.5, 27.0]])
    t = make_tree(spec)
    counts = t.continuation_run(scheme(spec), x0, 18, max_sweeps=40)
    o, oc = O.continuation(oracle_spec(spec), 18, x0, max_sweeps=40)
    assert list(counts) == oc and len(oc) > 10
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_continuation_depth16_matches_oracle():
    spec = dict(map="coupled_duffing", points=64, seed=0)
    t = make_tree(spec)
    counts = t.continuation_run(scheme(spec), np.zeros(4), 16)
    o, oc = O.continuation(oracle_spec(spec), 16, np.zeros(4))
    assert list(counts) == oc
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_insert_by_image_with_hit_flags_matches_oracle():
    spec = dict(map="henon", a=1.4, b=0.3, grid=4)
    t = make_tree(spec)
    o = O.Oracle(oracle_spec(spec))
    t.subdivision_run(scheme(spec), 12)
    o.subdivision(12)
    # keep a sparse subset of the attractor, flag a part of it, and insert its images
    codes, depth, _ = o.leaves()
    keep = np.arange(len(codes)) % 3 == 0
    flags = np.where(np.arange(keep.sum()) % 2 == 0, B.EXPD, B.NONE).astype(np.uint8)
    t.load_leaves(codes[keep], depth[keep], flags)
    o.load(codes[keep], depth[keep], flags)
    sc = scheme(spec, depth=12, flags_to_check=B.EXPD)
    n_new = t.insert_by_image(sc, 12, B.INS, B.HIT)
    assert n_new == o.insert_by_image(B.EXPD, B.INS, B.HIT)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_insert_points_into_a_tree_of_one_depth():
    spec = dict(map="lorenz", rho=28.0, grid=3)
    t = make_tree(spec)
    o = O.Oracle(oracle_spec(spec))
    t.subdivision_run(scheme(spec), 9)
    o.subdivision(9)
    rng = np.random.default_rng(5)
    pts = rng.uniform([-35, -35, -15], [35, 35, 70], size=(2000, 3))   # some outside the domain
    assert t.insert_points(pts, 9, B.INS, B.HIT) == o.insert_points(pts, 9, 2, 1)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_insert_many_distinct_boxes_into_root_merges_like_the_reference():
    # the surrounding box shares every path: it merges with the new boxes next to it in
    # tree order (the reference's two HasSamePath scans), so its flags reach some of them
    t = B.ImplicitBoxTree([0.0, 0.0], [1.0, 1.0])
    t.set_flags(B.SD, 0)
    pts = np.array([[0.5, 0.5], [-0.5, -0.5], [0.5, -0.5], [-0.9, 0.9]])
    assert t.insert_points(pts, 4, B.INS) == 4
    o = O.Oracle(dict(O.henon_spec(), center=np.zeros(2), radius=np.ones(2)))
    o.set_flags(8)
    assert o.insert_points_general(pts, 4, 2, 0) == 4
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)
    assert t.count() == 4 and t.depth() == 4
