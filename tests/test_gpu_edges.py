"""GPU: edge cases of the insertion, continuation, routing and measure entry points
against the oracle - empty inputs, points outside the domain, many duplicates, a tree of
one box, runs shorter than a convergence check."""
import numpy as np
import pytest

from oracle import oracle as O
from workloads import domain, oracle_spec, scheme

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


@pytest.mark.parametrize("x0", [np.array([[5.0, 0.0, 0.0, 0.0]]),                       # outside the domain
                                np.array([[0.0, 0.0, 0.0, 0.0], [0.0, 0.0, 0.0, 0.0],
                                          [0.3, -0.2, 0.1, 0.05]])])                     # a duplicate, two boxes
def test_continuation_from_unusual_start_points_matches_oracle(x0):
    spec = dict(map="coupled_duffing", points=64, seed=0)
    t = make_tree(spec)
    counts = t.continuation_run(scheme(spec), x0, 10)
    o, oc = O.continuation(oracle_spec(spec), 10, x0)
    assert list(counts) == oc
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_insert_of_no_points_and_of_many_duplicates_matches_oracle():
    spec = dict(map="henon", a=1.4, b=0.3, grid=4)
    t = make_tree(spec)
    o = O.Oracle(oracle_spec(spec))
    t.subdivision_run(scheme(spec), 10)
    o.subdivision(10)
    assert t.insert_points(np.zeros((0, 2)), 10, B.INS, B.HIT) == o.insert_points(np.zeros((0, 2)), 10, 2, 1)
    rng = np.random.default_rng(3)
    centres = rng.uniform([-1.4, -0.4], [1.4, 0.4], size=(7, 2))
    pts = centres[rng.integers(0, 7, 20000)]                 # 20,000 points in at most 7 boxes
    assert t.insert_points(pts, 10, B.INS, B.HIT) == o.insert_points(pts, 10, 2, 1)
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_transition_matrix_of_the_surrounding_box_matches_oracle():
    spec = dict(map="lorenz", rho=28.0, grid=5)
    t = make_tree(spec)
    o = O.Oracle(oracle_spec(spec))
    for invalid in (False, True):
        m = t.transition_matrix(scheme(spec), invalid_column=invalid)
        want = o.transition_matrix(invalid=invalid)
        for x, y in zip(m.to_host(), want[:3]):
            np.testing.assert_array_equal(x, y)
        assert m.n_cols == want[3]
        m.close()


def test_route_point_boxes_with_no_boxes_and_with_boxes_outside():
    import torch
    t = B.ImplicitBoxTree([0.0, 0.0], [1.0, 1.0])
    starts = np.array([0, 1 << 62, 1 << 63], dtype=np.uint64)
    ranks = np.array([0, 2, 3], dtype=np.uint32)
    empty = torch.empty(0, dtype=torch.int64, device="cuda")
    slot, c_parts, v_parts = t.route_point_boxes(empty, empty.to(torch.uint8), starts, ranks, 4)
    assert slot.numel() == 0 and [p.numel() for p in c_parts] == [0, 0, 0, 0]
    codes = torch.arange(1000, dtype=torch.int64, device="cuda")
    invalid = torch.zeros(1000, dtype=torch.uint8, device="cuda")
    slot, c_parts, _ = t.route_point_boxes(codes, invalid, starts, ranks, 4)
    assert [p.numel() for p in c_parts] == [0, 0, 0, 1000]        # every box outside: the last run
    np.testing.assert_array_equal(slot.cpu().numpy(), np.arange(1000))


def test_measure_to_tolerance_shorter_than_a_check_equals_the_fixed_count():
    """A tolerance run capped at k iterations is the fixed k-iteration run: the same launch
    when k fits one check (bit for bit), two launches otherwise (each normalises its last
    two iterates, so the vectors agree to rounding)."""
    spec = dict(map="henon", a=1.4, b=0.3, grid=4)
    t = make_tree(spec)
    sc = scheme(spec)
    t.subdivision_run(sc, 14)
    m = t.transition_matrix(sc)
    for k in (1, 7, 20, 33):
        v, done, _ = m.invariant_measure_tol(0.0, k, 20)
        assert done == k
        fixed = m.invariant_measure(k)
        if k <= 20:
            np.testing.assert_array_equal(v, fixed)
        else:
            assert np.abs(v - fixed).sum() < 1e-14
    m.close()


@pytest.mark.parametrize("mixed", [False, True])
def test_flag_updates_without_a_count_change_the_same_leaves(mixed):
    """set_flags / unset_flags with count=False (no read-back of the changed leaves) leave
    the same flags as the counting calls, on a tree of one depth and one of mixed depths."""
    spec = dict(map="lorenz", grid=3)
    trees = []
    for _ in range(2):
        t = make_tree(spec)
        t.subdivision_run(scheme(spec), 9)
        if mixed:
            t.set_flags(B.SD)
            codes, depth, flags = t.leaves()
            half = np.zeros_like(flags)
            half[: len(half) // 2] = B.SD
            t.load_leaves(codes, depth, half)
            t.subdivide(B.SD)
        trees.append(t)
    a, b = trees
    assert a.set_flags(B.HIT) > 0
    assert b.set_flags(B.HIT, count=False) is None
    assert a.unset_flags(B.HIT | B.SD) > 0
    assert b.unset_flags(B.HIT | B.SD, count=False) is None
    assert a.set_flags(B.INS) > 0
    assert b.set_flags(B.INS, count=False) is None
    for x, y in zip(a.leaves(), b.leaves()):
        np.testing.assert_array_equal(x, y)


def _write_coo_json(path, n, rows, cols, vals):
    """A transition matrix in the reference's CooMatrix file layout (row-major entries)."""
    def block(name, xs):
        body = ",\n".join(f"    {x!r}" for x in xs)
        return f'  "{name}": [\n{body}\n  ],'      # the reference's writer ends every list with a comma
    text = "{\n" + f'  "nRows": {n},\n  "nColumns": {n},\n  "nnz": {len(vals)},\n'
    text += block("rowIndices", rows) + "\n" + block("columnIndices", cols) + "\n" + block("values", vals)
    with open(path, "w") as f:
        f.write(text + "\n}")


def test_measure_of_a_matrix_with_long_rows_matches_oracle(tmp_path):
    """A matrix whose transpose has a row of 300 entries and one of 30 is iterated by the
    kernel that lists its rows by length class (the matrix-on-chip kernel takes rows of
    up to 64 entries only); its measure equals the oracle's."""
    n = 300
    rows, cols, vals = [], [], []
    for i in range(n):
        entry = {0: 0.5}
        other = 2 + (7 * i) % (n - 2)
        if i % 10 == 0:
            entry[1] = 0.25
            entry[other] = 0.25
        else:
            entry[other] = 0.5
        for c in sorted(entry):
            rows.append(i)
            cols.append(c)
            vals.append(entry[c])
    path = tmp_path / "long_rows_tm.json"
    _write_coo_json(path, n, rows, cols, vals)
    m = B.CsrMatrix.load(str(path))
    rowptr, c, v = m.to_host()
    np.testing.assert_array_equal(c, np.array(cols, dtype=c.dtype))
    np.testing.assert_array_equal(v, np.array(vals))
    got = m.invariant_measure(200)
    want = O.invariant_measure(rowptr, c, v, 200)
    assert np.abs(got - want).sum() < 1e-12
    np.testing.assert_array_equal(got, m.invariant_measure(200))
    m.close()
