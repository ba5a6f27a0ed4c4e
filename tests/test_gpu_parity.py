"""GPU parity: the CUDA library (through its C ABI) against the reference's golden
fixtures and the oracle.  Leaf sets, flags, counts and sparsity patterns must be
bit-exact; transition probabilities are bit-exact too (count / P is one IEEE
division on both sides; the stated tolerance is 1e-13 relative); the invariant
measure is compared to the oracle's FP64 power iteration in L1."""
import numpy as np
import pytest

from oracle import oracle as O
from workloads import csr_digests, domain, oracle_spec, scheme, sha

pytestmark = pytest.mark.gpu

B = pytest.importorskip("b12_b200")

TM_RTOL = 1e-13
MEASURE_L1 = 1e-12


@pytest.fixture(scope="module", autouse=True)
def _device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def make_tree(spec):
    c, r = domain(spec)
    return B.ImplicitBoxTree(c, r)


# ------------------------------------------------------------------ subdivision
def test_henon_step_by_step_api_matches_reference(golden):
    """The reference's loop (B12_doc.tex:269-290) call by call, with return values."""
    meta, arrays = golden("henon_d20")
    spec = meta["spec"]
    t = make_tree(spec)
    o = O.Oracle(oracle_spec(spec))
    sc = scheme(spec)
    assert t.set_flags(B.SD, 0) == o.set_flags(8) == 1
    for st in meta["steps"]:
        assert t.subdivide(B.SD) == o.subdivide(8)
        assert t.set_flags_by_image(sc, B.HIT) == o.set_flags_by_image(1)
        assert t.remove(B.HIT) == o.remove(1)
        assert t.unset_flags(B.HIT) == o.unset_flags(1)
        codes, depth, flags = t.leaves()
        assert t.count() == st["n"] and t.depth() == st["step"]
        assert sha(codes) == st["codes_sha256"], f"step {st['step']}"
        assert sha(flags) == st["flags_sha256"], f"step {st['step']}"
        if f"codes_{st['step']:02d}" in arrays:
            np.testing.assert_array_equal(codes, arrays[f"codes_{st['step']:02d}"])


@pytest.mark.parametrize("name", ["henon_d20", "henon_a1.0_d16", "lorenz_d15", "forced_duffing_d16",
                                  "lorenz_rho15_d18", "lorenz_rho35_d18"])
def test_fused_subdivision_matches_reference(golden, name):
    meta, arrays = golden(name)
    spec = meta["spec"]
    t = make_tree(spec)
    counts = t.subdivision_run(scheme(spec), len(meta["steps"]))
    assert list(counts) == [s["n"] for s in meta["steps"]]
    codes, depth, flags = t.leaves()
    last = meta["steps"][-1]
    assert sha(codes) == last["codes_sha256"]
    assert sha(flags) == last["flags_sha256"]
    assert (depth == last["step"]).all()


@pytest.mark.parametrize("name", ["lorenz_d27", "lorenz_fma_d27"])
def test_lorenz_depth27_box_sets_bit_identical(golden, name):
    try:
        meta, _ = golden(name)
    except FileNotFoundError:
        pytest.skip(f"{name} fixture not generated")
    spec = meta["spec"]
    t = make_tree(spec)
    steps = len(meta["steps"])
    # run the steps one fused call at a time so that every intermediate leaf set is checked
    for st in meta["steps"]:
        t.subdivision_run(scheme(spec), 1)
        codes, _, flags = t.leaves()
        assert len(codes) == st["n"], f"step {st['step']}"
        assert sha(codes) == st["codes_sha256"], f"step {st['step']}"
    assert t.depth() == steps
    m = t.transition_matrix(scheme(spec))
    d = csr_digests(*m.to_host())
    for k in ("nnz", "rowptr_sha256", "cols_sha256", "vals_sha256"):
        assert d[k] == meta["tm"][k], k


def test_fused_and_step_api_agree():
    spec = dict(map="lorenz", rho=28.0, grid=3, steps=12)
    a, b = make_tree(spec), make_tree(spec)
    sc = scheme(spec)
    counts = a.subdivision_run(sc, 12)
    b.set_flags(B.SD)
    for k in range(12):
        b.subdivide(B.SD)
        b.set_flags_by_image(sc, B.HIT)
        b.remove(B.HIT)
        b.unset_flags(B.HIT)
        assert b.count() == counts[k]
    for x, y in zip(a.leaves(), b.leaves()):
        np.testing.assert_array_equal(x, y)


# ------------------------------------------------------------------ transition matrix
@pytest.mark.parametrize("name,absolute,invalid", [
    ("henon_d20", False, False), ("henon_d12_abs", True, False), ("henon_d12_lost", False, True),
    ("lorenz_d15", False, False), ("forced_duffing_d16", False, False), ("lorenz_rho15_d18", False, False),
    ("lorenz_rho15_d4_invalid_column_unused", False, True)])
def test_transition_matrix_matches_reference(golden, name, absolute, invalid):
    meta, arrays = golden(name)
    spec = meta["spec"]
    t = make_tree(spec)
    sc = scheme(spec)
    t.subdivision_run(sc, len(meta["steps"]))
    m = t.transition_matrix(sc, absolute=absolute, invalid_column=invalid)
    assert m.n_rows == meta["tm"]["n_rows"] and m.n_cols == meta["tm"]["n_cols"]
    rowptr, cols, vals = m.to_host()
    d = csr_digests(rowptr, cols, vals)
    for k in ("nnz", "rowptr_sha256", "cols_sha256"):
        assert d[k] == meta["tm"][k], k
    if "tm_vals" in arrays:
        np.testing.assert_allclose(vals, arrays["tm_vals"], rtol=TM_RTOL, atol=0)
        np.testing.assert_array_equal(cols, arrays["tm_cols"])
    assert d["vals_sha256"] == meta["tm"]["vals_sha256"]


def test_matrix_from_stored_targets_and_after_changes(golden):
    """From a tree's second fused run on, the matrix right after subdivision_run is
    assembled from the targets its last step stored; once the leaves or the scheme differ
    it is recomputed.  Every matrix must be the oracle's."""
    meta, _ = golden("henon_d12_lost")
    spec = meta["spec"]
    t = make_tree(spec)
    sc = scheme(spec)
    t.subdivision_run(sc, len(meta["steps"]))       # first run: nothing stored
    t.transition_matrix(sc).close()
    t.delete_depth(0)
    t.subdivision_run(sc, len(meta["steps"]))       # second run: targets stored
    o = O.Oracle(oracle_spec(spec))

    def check(m, sc_spec, absolute=False, invalid=False):
        o = O.Oracle(oracle_spec(sc_spec))
        o.load(*t.leaves())
        want = o.transition_matrix(absolute=absolute, invalid=invalid)
        got = m.to_host()
        for x, y in zip(got, want[:3]):
            np.testing.assert_array_equal(x, y)
        assert m.n_cols == want[3]
        m.close()

    for absolute, invalid in ((False, False), (True, False), (False, True)):
        check(t.transition_matrix(sc, absolute=absolute, invalid_column=invalid), spec, absolute, invalid)
    t.set_flags(B.EQU)                                # flags only: the same leaves
    check(t.transition_matrix(sc, invalid_column=True), spec, invalid=True)
    other = dict(spec, grid=3)                        # another scheme over the same leaves
    check(t.transition_matrix(scheme(other)), other)
    check(t.transition_matrix(sc), spec)              # and back to the stored one
    t.subdivide(B.SD)                                 # new leaves
    check(t.transition_matrix(sc, invalid_column=True), spec, invalid=True)
    # one step: the stored children are the children of the loaded leaves
    t2 = make_tree(spec)
    t2.subdivision_run(sc, 9)
    codes, depth, flags = t2.leaves()
    t.load_leaves(codes, depth, flags)
    t.subdivision_run(sc, 1)
    o.load(codes, depth, flags)
    o.subdivision(1)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)
    check(t.transition_matrix(sc, invalid_column=True), spec, invalid=True)


def test_stored_targets_find_outside_points_in_a_last_leaf_of_code_0():
    """A run that ends with the single leaf of code 0 while 12 of its 16 image points leave
    the domain: those points are found in that leaf (hasSamePath of the invalid box), in
    the recomputed matrix and in the one built from stored targets alike."""
    a, b, center, radius = 5.8223, -0.912, [1.5308, 0.2375], [1.4846, 0.5467]
    spec = O.henon_spec(a, b, 4)
    spec["center"], spec["radius"] = center, radius
    o = O.Oracle(spec)
    o.subdivision(2)
    codes, depth, _ = o.leaves()
    assert list(codes) == [0] and list(depth) == [2]
    assert (o.image_point_boxes()[1] == 0).sum() == 12
    want = o.transition_matrix(invalid=True)
    t = B.ImplicitBoxTree(center, radius)
    sc = B.Scheme(B.henon(a, b), B.inner_grid(4))
    for run in range(2):                       # the second run stores its targets
        t.delete_depth(0)
        assert list(t.subdivision_run(sc, 2)) == [1, 1]
        m = t.transition_matrix(sc, invalid_column=True)
        for x, y in zip(m.to_host(), want[:3]):
            np.testing.assert_array_equal(x, y)
        assert m.n_cols == want[3] == 1
        m.close()


def test_invariant_measure_against_oracle():
    spec = dict(map="henon", a=1.4, b=0.3, grid=4)
    t = make_tree(spec)
    sc = scheme(spec)
    t.subdivision_run(sc, 16)
    m = t.transition_matrix(sc)
    rowptr, cols, vals = m.to_host()
    v = m.invariant_measure(200)
    ref = O.invariant_measure(rowptr, cols, vals, 200)
    l1 = np.abs(v - ref).sum()
    assert l1 < MEASURE_L1, l1
    assert abs(v.sum() - 1.0) < 1e-12
    # a second call reuses the transposed matrix and gives the same vector
    np.testing.assert_array_equal(v, m.invariant_measure(200))


def test_invariant_measure_on_a_second_device_after_the_first():
    """The power iteration's launch set-up (shared-memory opt-in, occupancy) is made per
    device: a measure on device 1 after one on device 0 runs and matches the oracle."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two CUDA devices")
    spec = dict(map="lorenz", rho=28.0, grid=5)
    results = []
    try:
        for dev in (0, 1):
            torch.cuda.set_device(dev)
            t = make_tree(spec)
            sc = scheme(spec)
            t.subdivision_run(sc, 18)
            m = t.transition_matrix(sc)
            rowptr, cols, vals = m.to_host()
            results.append((m.invariant_measure(200), O.invariant_measure(rowptr, cols, vals, 200)))
    finally:
        torch.cuda.set_device(0)
    for v, ref in results:
        assert np.abs(v - ref).sum() < MEASURE_L1
    np.testing.assert_array_equal(results[0][0], results[1][0])


# ------------------------------------------------------------------ search and flags
@pytest.mark.parametrize("spec", [dict(map="henon", a=1.4, b=0.3, grid=4),
                                  dict(map="lorenz", rho=28.0, grid=3),
                                  dict(map="forced_duffing", grid=3)])
def test_search_by_image_matches_oracle(spec):
    t = make_tree(spec)
    o = O.Oracle(oracle_spec(spec))
    sc = scheme(spec)
    t.subdivision_run(sc, 10)
    o.subdivision(10)
    np.testing.assert_array_equal(t.leaves()[0], o.leaves()[0])
    np.testing.assert_array_equal(t.search_by_image(sc), o.search_by_image())


def test_search_on_root_matches_reference_quirk():
    """On the root-only tree every mapped point, inside the domain or not, is found in
    leaf 0 (the reference's hasSamePath of an invalid box with code 0)."""
    spec = dict(map="henon", a=1.4, b=0.3, grid=4)
    t = make_tree(spec)
    o = O.Oracle(oracle_spec(spec))
    got = t.search_by_image(scheme(spec))
    np.testing.assert_array_equal(got, o.search_by_image())
    assert (got == 0).all()


def test_flag_operations_match_oracle():
    spec = dict(map="henon", a=1.4, b=0.3, grid=4)
    t = make_tree(spec)
    o = O.Oracle(oracle_spec(spec))
    t.subdivision_run(scheme(spec), 8)
    o.subdivision(8)
    rng = np.random.default_rng(1)
    codes, depth, _ = o.leaves()
    flags = rng.integers(0, 256, size=len(codes)).astype(np.uint8)
    t.load_leaves(codes, depth, flags)
    o.load(codes, depth, flags)
    for op, args in [("set", (B.INS,)), ("unset", (B.HIT | B.EXPD,)), ("change", (B.INS, B.EXPD)),
                     ("set", (B.SD | B.EQU,)), ("change", (B.SD | B.HIT, B.NONE))]:
        if op == "set":
            assert t.set_flags(*args) == o.set_flags(*args)
        elif op == "unset":
            assert t.unset_flags(*args) == o.unset_flags(*args)
        else:
            assert t.change_flags(*args) == o.change_flags(*args)
        np.testing.assert_array_equal(t.leaves()[2], o.leaves()[2])
    assert t.remove(B.EQU) == o.remove(0x10)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_remove_everything_leaves_the_root():
    spec = dict(map="henon", a=1.4, b=0.3, grid=4)
    t = make_tree(spec)
    t.subdivision_run(scheme(spec), 6)
    n = t.count()
    assert t.remove(B.EXPD) == n
    codes, depth, flags = t.leaves()
    assert list(codes) == [0] and list(depth) == [0] and list(flags) == [0]
    assert t.depth() == 0


def test_subdividing_one_leaf_gives_two_depths():
    spec = dict(map="henon", a=1.4, b=0.3, grid=4)
    t = make_tree(spec)
    t.subdivision_run(scheme(spec), 4)
    codes, depth, flags = t.leaves()
    flags = flags.copy()
    flags[0] |= B.INS
    t.load_leaves(codes, depth, flags)
    o = O.Oracle(oracle_spec(spec))
    o.load(codes, depth, flags)
    assert t.subdivide(B.INS) == o.subdivide(2) == 1
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)
    assert t.count() == len(codes) + 1 and t.depth() == depth[0] + 1 and t.count(int(depth[0])) == len(codes)
    # the shallower depth is now an inner depth for the split box: its two halves are one box
    assert t.set_flags(B.EXPD, int(depth[0])) == o.flags_at_depth(0, 0, 4, int(depth[0]))
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)
    # the unsubdividable depth 254 stays refused and changes nothing
    before = [a.copy() for a in t.leaves()]
    with pytest.raises(B.B12gError) as e:
        t.set_flags(B.HIT, 254)
    assert e.value.status == 5
    for x, y in zip(t.leaves(), before):
        np.testing.assert_array_equal(x, y)


def test_capacity_retry_in_fused_run():
    """The fused loop starts with a small buffer and must grow it transparently."""
    spec = dict(map="lorenz", rho=28.0, grid=5, steps=21)
    t = make_tree(spec)
    counts = t.subdivision_run(scheme(spec), 21)
    o = O.Oracle(oracle_spec(spec))
    oc, _ = o.subdivision(21)
    np.testing.assert_array_equal(counts, oc)
    np.testing.assert_array_equal(t.leaves()[0], o.leaves()[0])


def test_invariant_measure_lorenz_depth27_against_oracle(capsys):
    # the benchmark's job: Lorenz depth 27 (explicit-FMA integrator), its transition
    # matrix and 200 power iterations; L1 distance to the oracle's FP64 power iteration
    spec = dict(map="lorenz", rho=28.0, fma=True, grid=5)
    t = make_tree(spec)
    sc = scheme(spec)
    counts = t.subdivision_run(sc, 27)
    assert counts[-1] == 249450
    m = t.transition_matrix(sc)
    rowptr, cols, vals = m.to_host()
    assert len(vals) == 1615474
    v = m.invariant_measure(200)
    ref = O.invariant_measure(rowptr, cols, vals, 200)
    l1 = float(np.abs(v - ref).sum())
    with capsys.disabled():
        print(f"\nLorenz d27 invariant measure: L1 to the oracle = {l1:.3e} (n = {len(v)})")
    assert l1 < MEASURE_L1, l1
