"""GPU: trees whose leaves have different depths, through the C ABI, against the
reference's selective-refinement runs (tests/golden, `--mixed K`) and the oracle.

The start state is the reference's uniform tree with SD kept on the leaves in the lower
half of the first coordinate; subdivide(SD) then gives the tree two depths, and every
further step deepens the flagged part only.  Leaves (codes, depths, flags), counts and
transition matrices must be bit-exact."""
import numpy as np
import pytest

from oracle import oracle as O
from workloads import csr_digests, domain, oracle_spec, scheme, sha

pytestmark = pytest.mark.gpu

B = pytest.importorskip("b12_b200")

CASES = ["henon_d14_mixed8", "lorenz_d15_mixed6_lost", "forced_duffing_d12_mixed5", "henon_d8_mixed4_files"]


@pytest.fixture(scope="module", autouse=True)
def _device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def start(meta, arrays):
    spec = meta["spec"]
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    t.load_leaves(arrays["mixed_codes_00"], arrays["mixed_depth_00"], arrays["mixed_flags_00"])
    return t


def step(t, sc):
    k = t.subdivide(B.SD)
    t.set_flags_by_image(sc, B.HIT)
    t.remove(B.HIT)
    t.unset_flags(B.HIT)
    return k


def check_leaves(t, st, arrays):
    codes, depth, flags = t.leaves()
    k = st["step"]
    assert t.count() == st["n"], f"step {k}"
    assert t.depth() == st["max_depth"], f"step {k}"
    assert sha(codes) == st["codes_sha256"], f"step {k} codes"
    assert sha(depth) == st["depth_sha256"], f"step {k} depths"
    assert sha(flags) == st["flags_sha256"], f"step {k} flags"
    if f"mixed_codes_{k:02d}" in arrays:
        np.testing.assert_array_equal(depth, arrays[f"mixed_depth_{k:02d}"])


@pytest.mark.parametrize("name", CASES)
def test_selective_refinement_matches_reference(golden, name):
    meta, arrays = golden(name)
    spec = meta["spec"]
    t = start(meta, arrays)
    o = O.Oracle(oracle_spec(spec))
    o.load(arrays["mixed_codes_00"], arrays["mixed_depth_00"], arrays["mixed_flags_00"])
    sc = scheme(spec)
    for st in meta["mixed"][1:]:
        assert step(t, sc) == o.subdivide(8)
        o.set_flags_by_image(1)
        o.remove(1)
        o.unset_flags(1)
        check_leaves(t, st, arrays)
    m = t.transition_matrix(sc, absolute=spec.get("absolute", False), invalid_column=spec.get("invalid", False))
    rowptr, cols, vals = m.to_host()
    d = csr_digests(rowptr, cols, vals)
    tm = meta["tm"]
    assert m.n_cols == tm["n_cols"]
    for key in ("nnz", "rowptr_sha256", "cols_sha256", "vals_sha256"):
        assert d[key] == tm[key], key


def test_return_values_of_each_call_match_oracle(golden):
    meta, arrays = golden("henon_d14_mixed8")
    spec = meta["spec"]
    t = start(meta, arrays)
    o = O.Oracle(oracle_spec(spec))
    o.load(arrays["mixed_codes_00"], arrays["mixed_depth_00"], arrays["mixed_flags_00"])
    sc = scheme(spec)
    for _ in range(4):
        assert t.subdivide(B.SD) == o.subdivide(8)
        assert t.set_flags_by_image(sc, B.HIT) == o.set_flags_by_image(1)
        assert t.remove(B.HIT) == o.remove(1)
        assert t.unset_flags(B.HIT) == o.unset_flags(1)
        assert t.set_flags(B.EXPD) == o.set_flags(4)
        assert t.change_flags(B.EXPD, B.INS) == o.change_flags(4, 2)
        assert t.unset_flags(B.INS) == o.unset_flags(2)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("name", ["henon_d14_mixed8", "lorenz_d15_mixed6_lost"])
def test_search_by_image_matches_oracle(golden, name):
    meta, arrays = golden(name)
    spec = meta["spec"]
    t = start(meta, arrays)
    sc = scheme(spec)
    for _ in range(3):
        step(t, sc)
    codes, depth, flags = t.leaves()
    o = O.Oracle(oracle_spec(spec))
    o.load(codes, depth, flags)
    np.testing.assert_array_equal(t.search_by_image(sc), o.search_by_image())
    # sources filtered by flags: every third leaf carries EXPD
    mask = np.zeros(len(codes), dtype=np.uint8)
    mask[::3] = 1
    o.set_flags_mask(mask, 4)
    t.load_leaves(codes, depth, flags | (mask * 4).astype(np.uint8))
    src = np.nonzero(mask)[0].astype(np.uint32)
    np.testing.assert_array_equal(t.search_by_image(B.Scheme(sc.map, sc.grid, 255, B.EXPD)), o.search_by_image(src))


def count_reference(codes, depth, d):
    """count(d) (ImplicitBoxTree.hpp:1061-1095): leaves that start a new depth-d box."""
    keep = depth >= d
    pre = np.where(keep, codes >> (depth.astype(np.uint64) - np.uint64(d)) * keep, 0)
    fresh = keep.copy()
    fresh[1:] &= ~(keep[:-1] & (pre[1:] == pre[:-1]))
    return int(fresh.sum())


def test_count_at_inner_depths(golden):
    meta, arrays = golden("henon_d14_mixed8")
    t = start(meta, arrays)
    sc = scheme(meta["spec"])
    for _ in range(5):
        step(t, sc)
    codes, depth, flags = t.leaves()
    assert t.count(0) == 1 and t.count() == len(codes)
    for d in range(1, int(depth.max()) + 3):
        assert t.count(d) == count_reference(codes, depth, d), d


def test_subdivision_run_on_a_mixed_tree_matches_oracle(golden):
    meta, arrays = golden("forced_duffing_d12_mixed5")
    spec = meta["spec"]
    t = start(meta, arrays)
    sc = scheme(spec)
    step(t, sc)
    codes, depth, flags = t.leaves()
    assert depth.min() != depth.max()
    o = O.Oracle(oracle_spec(spec))
    o.load(codes, depth, flags)
    want, _ = o.subdivision(3)
    np.testing.assert_array_equal(t.subdivision_run(sc, 3), want)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_self_hit_selection_on_a_mixed_tree(golden):
    meta, arrays = golden("henon_d14_mixed8")
    spec = meta["spec"]
    t = start(meta, arrays)
    sc = scheme(spec)
    for _ in range(2):
        step(t, sc)
    codes, depth, flags = t.leaves()
    o = O.Oracle(oracle_spec(spec))
    o.load(codes, depth, flags)
    tgt = o.search_by_image().reshape(len(codes), -1)
    want = (tgt == np.arange(len(codes))[:, None]).any(axis=1)
    assert t.set_flags_by_self_hit(sc, B.HIT) == int(want.sum())
    np.testing.assert_array_equal(t.leaves()[2] & B.HIT != 0, want)


def test_mixed_tree_returns_to_one_depth(golden):
    meta, arrays = golden("henon_d8_mixed4_files")
    t = start(meta, arrays)
    sc = scheme(meta["spec"])
    step(t, sc)
    codes, depth, flags = t.leaves()
    assert depth.min() == 8 and depth.max() == 9
    # subdividing every leaf but the depth-8 ones joins the depths again
    t.unset_flags(B.SD)
    t.load_leaves(codes, depth, (flags & ~np.uint8(B.SD)) | np.where(depth == 8, B.SD, 0).astype(np.uint8))
    assert t.subdivide(B.SD) == int((depth == 8).sum())
    c2, d2, _ = t.leaves()
    assert (d2 == 9).all() and t.depth() == 9
    o = O.Oracle(oracle_spec(meta["spec"]))
    o.load(codes, depth, (flags & ~np.uint8(8)) | np.where(depth == 8, 8, 0).astype(np.uint8))
    o.subdivide(8)
    np.testing.assert_array_equal(c2, o.leaves()[0])
    # a uniform tree again: the fused loop takes over and matches the oracle
    want, _ = o.subdivision(2)
    np.testing.assert_array_equal(t.subdivision_run(sc, 2), want)
    np.testing.assert_array_equal(t.leaves()[0], o.leaves()[0])


def test_removing_every_leaf_leaves_the_surrounding_box(golden):
    meta, arrays = golden("henon_d8_mixed4_files")
    t = start(meta, arrays)
    step(t, scheme(meta["spec"]))
    t.unset_flags(B.HIT)
    assert t.remove(B.HIT) == meta["mixed"][1]["n"]
    codes, depth, flags = t.leaves()
    assert list(codes) == [0] and list(depth) == [0] and t.depth() == 0


def test_unsupported_calls_refuse_and_leave_the_tree(golden):
    meta, arrays = golden("henon_d8_mixed4_files")
    t = start(meta, arrays)
    sc = scheme(meta["spec"])
    step(t, sc)
    before = [a.copy() for a in t.leaves()]
    for call in (lambda: t.set_flags(B.EXPD, 254), lambda: t.set_flags_by_image(sc, B.HIT, 0),
                 lambda: t.insert_by_image(B.Scheme(sc.map, sc.grid, 0, B.INS), 9)):
        with pytest.raises(B.B12gError) as e:
            call()
        assert e.value.status == B._lib.ERR_MIXED_DEPTH
    for x, y in zip(t.leaves(), before):
        np.testing.assert_array_equal(x, y)


# ---------------------------------------------------------------- unsubdivide and insertion
EDIT_CASES = ["henon_d12_mixed6_edits", "lorenz_d12_mixed4_edits", "forced_duffing_d10_mixed3_edits"]


def check_edit(t, e, key):
    codes, depth, flags = t.leaves()
    assert t.count() == e["n"], key
    assert sha(codes) == e["codes_sha256"], f"{key} codes"
    assert sha(depth) == e["depth_sha256"], f"{key} depths"
    assert sha(flags) == e["flags_sha256"], f"{key} flags"
    assert t.depth() == int(depth.max())


@pytest.mark.parametrize("name", EDIT_CASES)
def test_unsubdivide_and_insert_match_reference(golden, name):
    """The reference run's edits of a mixed tree (oracle/ref/runner.h, runEdits) call by
    call, leaves after each against the reference, return values against the oracle."""
    meta, arrays = golden(name)
    spec = meta["spec"]
    last = meta["mixed"][-1]["step"]
    start_leaves = (arrays[f"mixed_codes_{last:02d}"], arrays[f"mixed_depth_{last:02d}"],
                    arrays[f"mixed_flags_{last:02d}"])
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    t.load_leaves(*start_leaves)
    o = O.Oracle(oracle_spec(spec))
    o.load(*start_leaves)
    sc = scheme(spec)
    want = {e["step"]: e for e in meta["edits"]}
    maxd = meta["timing"]["edit_max_depth"]
    assert t.unsubdivide(B.SD) == o.unsubdivide(8) == meta["timing"]["edits"][0]
    check_edit(t, want["01"], "01")
    assert t.unsubdivide(B.SD) == o.unsubdivide(8) == meta["timing"]["edits"][1]
    check_edit(t, want["02"], "02")
    assert t.depth() == maxd
    assert t.insert_points(arrays["points_3"], 255, B.INS, B.HIT) == o.insert_points_general(arrays["points_3"], 255, 2, 1)
    check_edit(t, want["03"], "03")
    assert t.insert_points(arrays["points_4"], maxd + 2, B.INS) == o.insert_points_general(arrays["points_4"], maxd + 2, 2)
    check_edit(t, want["04"], "04")
    assert t.insert_points(arrays["points_5"], maxd - 1, B.EXPD) == o.insert_points_general(arrays["points_5"], maxd - 1, 4)
    check_edit(t, want["05"], "05")
    src = B.Scheme(sc.map, sc.grid, 255, B.INS)
    assert t.insert_by_image(src, 255, B.EXPD) == o.insert_by_image_general(2, 255, 4)
    check_edit(t, want["06"], "06")
    t.set_flags_by_image(sc, B.HIT)
    t.remove(B.HIT)
    t.unset_flags(B.HIT)
    check_edit(t, want["07"], "07")
    # flags of the boxes at inner depths: every leaf of such a box changes
    md = meta["timing"]["edit_flag_depth"]
    counts = meta["timing"]["edits"]
    assert t.depth() == md
    assert t.set_flags(B.EXPD, md - 2) == counts[7]
    check_edit(t, want["08"], "08")
    assert t.change_flags(B.EXPD, B.INS, md - 3) == counts[8]
    check_edit(t, want["09"], "09")
    assert t.unset_flags(B.INS, md - 1) == counts[9]
    check_edit(t, want["10"], "10")
    # images located at inner depths: flags on the boxes hit, box indices, insertion hits
    assert t.set_flags_by_image(sc, B.HIT, md - 2) == counts[10]
    check_edit(t, want["11"], "11")
    np.testing.assert_array_equal(t.search_by_image(sc, md - 3), arrays["search_12"])
    t.insert_points(arrays["points_13"], md - 1, B.INS, B.EXPD)
    check_edit(t, want["13"], "13")
    # images of the boxes of an inner depth (sources: boxes whose leaves all carry EXPD)
    assert t.set_flags_by_image(B.Scheme(sc.map, sc.grid, md - 3, B.EXPD), B.ENTR) == counts[13]
    check_edit(t, want["14"], "14")
    np.testing.assert_array_equal(t.search_by_image(B.Scheme(sc.map, sc.grid, md - 2, 0)), arrays["search_15"])
    m = t.transition_matrix(sc, invalid_column=spec.get("invalid", False))
    d = csr_digests(*m.to_host())
    for key in ("nnz", "rowptr_sha256", "cols_sha256", "vals_sha256"):
        assert d[key] == meta["tm"][key], key


@pytest.mark.parametrize("name", EDIT_CASES)
def test_points_into_the_surrounding_box_alone(golden, name):
    meta, arrays = golden(name)
    c, r = domain(meta["spec"])
    t = B.ImplicitBoxTree(c, r)
    t.set_flags(B.SD, 0)
    t.insert_points(arrays["points_root"], 6, B.INS, B.HIT)
    check_edit(t, {x["step"]: x for x in meta["edits"]}["root"], "root")


@pytest.mark.parametrize("depth_of", [lambda d: 255, lambda d: d + 3, lambda d: d - 2])
def test_insert_into_a_one_depth_tree_at_another_depth(golden, depth_of):
    meta, arrays = golden("henon_d12_mixed6_edits")
    spec = meta["spec"]
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    t.subdivision_run(scheme(spec), 10)
    o = O.Oracle(oracle_spec(spec))
    o.subdivision(10)
    depth = depth_of(10)
    hit = B.HIT if depth == 255 else 0
    assert t.insert_points(arrays["points_3"], depth, B.INS, hit) == o.insert_points_general(arrays["points_3"], depth,
                                                                                           2, hit)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)
    # and then a step of the image selection on whatever depths resulted
    step(t, scheme(spec))
    o.subdivide(8)
    o.set_flags_by_image(1)
    o.remove(1)
    o.unset_flags(1)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_unsubdivide_of_a_one_depth_tree(golden):
    meta, arrays = golden("henon_d12_mixed6_edits")
    spec = meta["spec"]
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    t.subdivision_run(scheme(spec), 12)
    o = O.Oracle(oracle_spec(spec))
    o.subdivision(12)
    codes, depth, flags = t.leaves()
    mask = (np.arange(len(codes)) % 3 == 0).astype(np.uint8)
    t.load_leaves(codes, depth, (flags & ~np.uint8(B.SD)) | (mask * B.SD).astype(np.uint8))
    o.load(codes, depth, (flags & ~np.uint8(8)) | (mask * 8).astype(np.uint8))
    for _ in range(3):
        assert t.unsubdivide(B.SD) == o.unsubdivide(8)
        for x, y in zip(t.leaves(), o.leaves()):
            np.testing.assert_array_equal(x, y)


def test_insertion_hits_at_an_inner_depth_match_oracle(golden):
    meta, arrays = golden("henon_d12_mixed6_edits")
    spec = meta["spec"]
    last = meta["mixed"][-1]["step"]
    leaves = (arrays[f"mixed_codes_{last:02d}"], arrays[f"mixed_depth_{last:02d}"], arrays[f"mixed_flags_{last:02d}"])
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    t.load_leaves(*leaves)
    o = O.Oracle(oracle_spec(spec))
    o.load(*leaves)
    for d, pts in ((14, arrays["points_3"]), (17, arrays["points_4"]), (12, arrays["points_5"])):
        assert t.insert_points(pts, d, B.INS, B.HIT) == o.insert_points_general(pts, d, 2, 1)
        for x, y in zip(t.leaves(), o.leaves()):
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("op", [0, 1, 2])
def test_flags_at_an_inner_depth_of_a_one_depth_tree(golden, op):
    meta, arrays = golden("henon_d12_mixed6_edits")
    spec = meta["spec"]
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    t.subdivision_run(scheme(spec), 12)
    o = O.Oracle(oracle_spec(spec))
    o.subdivision(12)
    codes, depth, flags = t.leaves()
    mask = ((codes * np.uint64(2654435761)) >> np.uint64(7)) % np.uint64(3) == 0   # some leaves carry EXPD
    f2 = (flags | np.where(mask, B.EXPD, 0)).astype(np.uint8)
    t.load_leaves(codes, depth, f2)
    o.load(codes, depth, f2)
    for d in (3, 9, 11, 13):
        if op == 0:
            got, want = t.set_flags(B.INS, d), o.flags_at_depth(0, 0, 2, d)
        elif op == 1:
            got, want = t.unset_flags(B.EXPD, d), o.flags_at_depth(1, 0, 4, d)
        else:
            got, want = t.change_flags(B.EXPD, B.HIT, d), o.flags_at_depth(2, 4, 1, d)
        assert got == want, d
        for x, y in zip(t.leaves(), o.leaves()):
            np.testing.assert_array_equal(x, y)
        assert t.depth() == 12


@pytest.mark.parametrize("src_depth,depth", [(13, 255), (15, 17), (12, 14)])
def test_insertion_of_images_of_inner_boxes_matches_oracle(golden, src_depth, depth):
    meta, arrays = golden("henon_d12_mixed6_edits")
    spec = meta["spec"]
    last = meta["mixed"][-1]["step"]
    leaves = (arrays[f"mixed_codes_{last:02d}"], arrays[f"mixed_depth_{last:02d}"], arrays[f"mixed_flags_{last:02d}"])
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    t.load_leaves(*leaves)
    o = O.Oracle(oracle_spec(spec))
    o.load(*leaves)
    sc = scheme(spec)
    got = t.insert_by_image(B.Scheme(sc.map, sc.grid, src_depth, B.SD), depth, B.INS, B.HIT)
    assert got == o.insert_by_image_src(src_depth, 8, depth, 2, 1)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def comparable(code, depth):
    """getComparableBitPattern (Box.hpp:67-73) of a depth <= 64 box"""
    s = 64 - depth
    high = (code << s) & ((1 << 64) - 1) if s < 64 else 0
    return high | (((1 << (s - 1)) - 1) if s >= 2 else 0)


def deepest_leaves(o, points, depths):
    """leaves around the given points at the given depths (<= 64), in tree order"""
    boxes = []
    for p, d in zip(points, depths):
        c, ok = o.point_code64(np.asarray(p, dtype=np.float64))
        assert ok
        boxes.append((c >> (64 - d) if d < 64 else c, d))
    boxes.sort(key=lambda b: (comparable(*b), -b[1]))
    codes = np.array([b[0] for b in boxes], dtype=np.uint64)
    depth = np.array([b[1] for b in boxes], dtype=np.uint8)
    return codes, depth


def test_leaves_at_the_maximal_depth():
    """Depth-64 leaves stay whole under subdivide (which still counts them), and a point
    inside one at the leaf depth is not inserted but flags it as hit."""
    o = O.Oracle(O.henon_spec())
    codes, depth = deepest_leaves(o, [(-1.0, 0.1), (0.5, -0.2), (1.2, 0.3)], [64, 63, 64])
    flags = np.full(len(codes), 8, dtype=np.uint8)
    t = B.ImplicitBoxTree([0.0, 0.0], [1.5, 0.45])
    t.load_leaves(codes, depth, flags)
    o.load(codes, depth, flags)
    assert t.subdivide(B.SD) == o.subdivide(8) == 3
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)
    assert t.count() == 4 and t.depth() == 64
    # one point inside the first depth-64 leaf, one elsewhere
    pts = np.array([[-1.0, 0.1], [0.0, 0.0]])
    assert t.insert_points(pts, 255, B.INS, B.HIT) == o.insert_points_general(pts, 255, 2, 1)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)
    # a uniform tree at depth 64: subdivide counts the flagged leaves and splits none
    u_codes, u_depth = deepest_leaves(o, [(-1.0, 0.1), (1.2, 0.3)], [64, 64])
    t.load_leaves(u_codes, u_depth, np.full(2, 8, dtype=np.uint8))
    assert t.subdivide(B.SD) == 2
    np.testing.assert_array_equal(t.leaves()[0], u_codes)
    assert t.depth() == 64
