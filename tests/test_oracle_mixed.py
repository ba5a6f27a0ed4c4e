"""CPU: the oracle on trees whose leaves have different depths, against the reference.

The reference run (tests/golden/make_golden.py, `--mixed K`) refines uniformly to depth
d, keeps SD only on the leaves in the lower half of the first coordinate, and then runs
K steps of subdivide(SD) + image selection, so that the leaves span depths d..d+K.  Each
step's leaves (codes, depths, flags) and the final transition matrix pin the oracle's
ordering (isStrictlyPreceding), search (lower_bound + ComputeSearchIndexFunctor) and
subdivision on mixed trees.
"""
import numpy as np
import pytest

from oracle import oracle as O
from workloads import csr_digests, oracle_spec, sha

MIXED_CASES = ["henon_d14_mixed8", "lorenz_d15_mixed6_lost", "forced_duffing_d12_mixed5", "henon_d8_mixed4_files"]


def mixed_start(meta, arrays):
    return arrays["mixed_codes_00"], arrays["mixed_depth_00"], arrays["mixed_flags_00"]


@pytest.mark.parametrize("name", MIXED_CASES)
def test_start_state_is_the_uniform_run_with_a_lower_half_stencil(golden, name):
    meta, arrays = golden(name)
    codes, depth, flags = mixed_start(meta, arrays)
    d = meta["steps"][-1]["depth"]
    assert (depth == d).all() and len(codes) == meta["steps"][-1]["n"]
    assert sha(codes) == meta["steps"][-1]["codes_sha256"]
    lower = (codes >> np.uint64(d - 1)) == 0
    assert np.array_equal(flags & 8 != 0, lower)


@pytest.mark.parametrize("name", MIXED_CASES)
def test_mixed_steps_match_reference(golden, name):
    meta, arrays = golden(name)
    o = O.Oracle(oracle_spec(meta["spec"]))
    o.load(*mixed_start(meta, arrays))
    for st in meta["mixed"][1:]:
        o.subdivide(8)
        o.set_flags_by_image(1)
        o.remove(1)
        o.unset_flags(1)
        codes, depth, flags = o.leaves()
        k = st["step"]
        assert len(codes) == st["n"], f"step {k}"
        assert sha(codes) == st["codes_sha256"], f"step {k} codes"
        assert sha(depth) == st["depth_sha256"], f"step {k} depths"
        assert sha(flags) == st["flags_sha256"], f"step {k} flags"
        assert int(depth.min()) == st["min_depth"] and int(depth.max()) == st["max_depth"]
    spec = meta["spec"]
    rowptr, cols, vals, ncols = o.transition_matrix(absolute=spec.get("absolute", False),
                                                    invalid=spec.get("invalid", False))
    d = csr_digests(rowptr, cols, vals)
    tm = meta["tm"]
    assert ncols == tm["n_cols"]
    for key in ("nnz", "rowptr_sha256", "cols_sha256", "vals_sha256"):
        assert d[key] == tm[key], key


def test_mixed_search_candidates_follow_the_reference_rule():
    # a point on the path of the leaf before the lower bound, at the lower bound, or of neither
    spec = O.henon_spec()
    o = O.Oracle(spec)
    # leaves: 0 (depth 1), 10 (depth 2), 11 (depth 2) - the left half and the right quarters
    o.load(np.array([0, 2, 3], dtype=np.uint64), np.array([1, 2, 2], dtype=np.uint8), np.zeros(3, np.uint8))
    for x, want in (((-1.0, 0.0), 0), ((0.2, -0.2), 1), ((0.2, 0.2), 2), ((1.4, 0.44), 2)):
        c, ok = o.point_code64(np.array(x))
        assert ok
        assert o.L.orc_search(O.C.byref(o.tree), c, 1) == want, x
    assert o.L.orc_search(O.C.byref(o.tree), 0, 0) == 0xFFFFFFFF  # invalid point: the last code is not 0


EDIT_CASES = ["henon_d12_mixed6_edits", "lorenz_d12_mixed4_edits", "forced_duffing_d10_mixed3_edits"]


def edit_sequence(o, meta, arrays):
    """The reference run's edits (oracle/ref/runner.h, runEdits), yielding after each."""
    maxd = meta["timing"]["edit_max_depth"]
    yield "01", o.unsubdivide(8)
    yield "02", o.unsubdivide(8)
    yield "03", o.insert_points_general(arrays["points_3"], 255, 2, 1)
    yield "04", o.insert_points_general(arrays["points_4"], maxd + 2, 2, 0)
    yield "05", o.insert_points_general(arrays["points_5"], maxd - 1, 4, 0)
    yield "06", o.insert_by_image_general(2, 255, 4, 0)
    o.set_flags_by_image(1)
    o.remove(1)
    o.unset_flags(1)
    yield "07", None
    md = meta["timing"]["edit_flag_depth"]
    yield "08", o.flags_at_depth(0, 0, 4, md - 2)        # setFlags(EXPD, md - 2)
    yield "09", o.flags_at_depth(2, 4, 2, md - 3)        # changeFlags(EXPD, INS, md - 3)
    yield "10", o.flags_at_depth(1, 0, 2, md - 1)        # unsetFlags(INS, md - 1)
    yield "11", o.image_flags_at_depth(md - 2, 1)       # setFlagsByIterators(leaves, HIT, md - 2)
    yield "search", o.image_search_at_depth(md - 3)     # searchByIterators(leaves, md - 3)
    yield "13", o.insert_points_general(arrays["points_13"], md - 1, 2, 4)   # insert(pts, md - 1, INS, EXPD)
    yield "14", o.image_flags(md - 3, 4, 255, 0x20)      # setFlagsByIterators(ByFlags(md - 3, EXPD), ENTR)
    yield "search15", o.image_search(md - 2, 0, 255)    # searchByIterators(OverDepth(md - 2), leaves)


@pytest.mark.parametrize("name", EDIT_CASES)
def test_unsubdivide_and_insert_match_reference(golden, name):
    meta, arrays = golden(name)
    spec = meta["spec"]
    last = meta["mixed"][-1]["step"]
    o = O.Oracle(oracle_spec(spec))
    o.load(arrays[f"mixed_codes_{last:02d}"], arrays[f"mixed_depth_{last:02d}"], arrays[f"mixed_flags_{last:02d}"])
    want = {e["step"]: e for e in meta["edits"]}
    counts = meta["timing"]["edits"]
    for k, (key, ret) in enumerate(edit_sequence(o, meta, arrays)):
        if key in ("search", "search15"):
            np.testing.assert_array_equal(ret, arrays["search_12" if key == "search" else "search_15"])
            assert len(ret) == counts[k]
            continue
        codes, depth, flags = o.leaves()
        e = want[key]
        assert len(codes) == e["n"], key
        assert sha(codes) == e["codes_sha256"], f"{key} codes"
        assert sha(depth) == e["depth_sha256"], f"{key} depths"
        assert sha(flags) == e["flags_sha256"], f"{key} flags"
        if key in ("01", "02", "08", "09", "10", "11", "14"):
            assert ret == counts[k], key          # the call's own return value
        else:
            assert len(codes) == counts[k], key   # the run records the leaf count


@pytest.mark.parametrize("name", EDIT_CASES)
def test_insert_into_the_surrounding_box_alone(golden, name):
    # several new boxes merge with the surrounding box, which shares every path
    meta, arrays = golden(name)
    o = O.Oracle(oracle_spec(meta["spec"]))
    o.set_flags(8)
    o.insert_points_general(arrays["points_root"], 6, 2, 1)
    codes, depth, flags = o.leaves()
    e = {x["step"]: x for x in meta["edits"]}["root"]
    assert sha(codes) == e["codes_sha256"] and sha(depth) == e["depth_sha256"] and sha(flags) == e["flags_sha256"]
