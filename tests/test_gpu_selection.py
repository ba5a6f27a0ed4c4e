"""GPU: strongly connected components of transition graphs, the two selection drivers
that use a transition matrix (chain recurrent set, natural invariant measure) and the
fixed-box driver, against the oracle: Tarjan's algorithm and the same loops on the CPU."""
import numpy as np
import pytest

from oracle import oracle as O
from workloads import domain, oracle_spec, scheme

pytestmark = pytest.mark.gpu

B = pytest.importorskip("b12_b200")
from b12_b200 import tree as T  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def device_matrix(tmp_path, n, edges):
    """A CSR on the device for a synthetic graph (through the JSON reader)."""
    edges = sorted(set(edges))
    rowptr = np.zeros(n + 1, dtype=np.uint32)
    for u, _ in edges:
        rowptr[u + 1] += 1
    rowptr = np.cumsum(rowptr).astype(np.uint32)
    cols = np.array([v for _, v in edges], dtype=np.uint32)
    vals = np.ones(len(edges))
    T.json_write_coo(tmp_path / "g.json", n, n, rowptr, cols, vals)
    return B.CsrMatrix.load(tmp_path / "g.json"), rowptr, cols


def test_components_of_a_synthetic_graph(tmp_path):
    rng = np.random.default_rng(7)
    n = 3000
    edges = [(i, (i + 1) % 40) for i in range(40)]                       # a 40-cycle
    edges += [(100 + i, 100 + i + 1) for i in range(500)]                 # a long chain into ...
    edges += [(600, 601), (601, 600), (600, 600), (2000, 2000)]           # a 2-cycle, self-loops
    edges += [(int(a), int(b)) for a, b in rng.integers(700, n, size=(4000, 2))]   # a random tangle
    m, rowptr, cols = device_matrix(tmp_path, n, edges)
    comp, k = m.strong_components()
    want = O.strong_components(rowptr, cols)
    np.testing.assert_array_equal(comp, want)
    assert k == len(np.unique(want))


@pytest.mark.parametrize("spec,steps", [(dict(map="henon"), 16), (dict(map="lorenz", rho=28.0, grid=5), 15),
                                        (dict(map="forced_duffing", grid=4), 12)])
def test_components_of_transition_matrices(spec, steps):
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    sc = scheme(spec)
    t.subdivision_run(sc, steps)
    m = t.transition_matrix(sc)
    rowptr, cols, _ = m.to_host()
    comp, _ = m.strong_components()
    np.testing.assert_array_equal(comp, O.strong_components(rowptr, cols))


@pytest.mark.parametrize("spec,steps", [(dict(map="henon"), 14), (dict(map="lorenz", rho=28.0, grid=5), 12)])
def test_chain_recurrent_run_matches_oracle(spec, steps):
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    counts = t.chain_recurrent_run(scheme(spec), steps)
    o, ocounts = O.chain_recurrent(oracle_spec(spec), steps)
    assert list(counts) == ocounts
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def test_nim_run_matches_oracle():
    spec = dict(map="henon")
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    counts = t.nim_run(scheme(spec), 14, 200)
    o, ocounts = O.nim_selection(oracle_spec(spec), 14, 200)
    assert list(counts) == ocounts
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


def checkpoint_changes(rowptr, cols, vals, tol, max_iters, every):
    """The oracle's stopping point and the changes at its last two checks."""
    v, k, ch = O.invariant_measure_tol(rowptr, cols, vals, tol, max_iters, every)
    prev = O.invariant_measure_tol(rowptr, cols, vals, 0.0, k - every, every)[2] if k > every else np.inf
    return v, k, ch, prev


@pytest.mark.parametrize("spec,steps,tol", [(dict(map="henon"), 12, 1e-10), (dict(map="lorenz", rho=28.0, grid=5), 14,
                                                                             1e-12)])
def test_invariant_measure_to_tolerance_matches_oracle(spec, steps, tol):
    """The tolerance-driven power iteration stops at the oracle's check (the changes at the
    last two checks straddle tol by at least 10 % here) with the same vector, within the
    measure tolerance of the other tests."""
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    sc = scheme(spec)
    t.subdivision_run(sc, steps)
    m = t.transition_matrix(sc)
    rowptr, cols, vals = m.to_host()
    want, k, ch, prev = checkpoint_changes(rowptr, cols, vals, tol, 100000, 20)
    assert ch <= 0.9 * tol and prev >= 1.1 * tol, (ch, prev)      # a decision no rounding can flip
    v, k_gpu, ch_gpu = m.invariant_measure_tol(tol, 100000, 20)
    assert k_gpu == k
    assert abs(ch_gpu - ch) <= 1e-3 * tol + 1e-15
    assert np.abs(v - want).sum() < 1e-12
    # a cap below the stopping point ends the run there
    v2, k2, _ = m.invariant_measure_tol(0.0, 50, 20)
    assert k2 == 50
    np.testing.assert_allclose(v2, O.invariant_measure(rowptr, cols, vals, 50), rtol=0, atol=1e-13)


def test_nim_run_to_tolerance_matches_oracle():
    spec = dict(map="henon")
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    counts = t.nim_run_tol(scheme(spec), 12, 1e-12, 100000)
    o, ocounts = O.nim_selection(oracle_spec(spec), 12, 100000, tol=1e-12)
    assert list(counts) == ocounts
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("spec,steps", [(dict(map="henon"), 16), (dict(map="lorenz", rho=28.0, grid=5), 14),
                                        (dict(map="forced_duffing", grid=4), 12)])
def test_fixed_boxes_run_matches_oracle(spec, steps):
    c, r = domain(spec)
    t = B.ImplicitBoxTree(c, r)
    counts = t.fixed_boxes_run(scheme(spec), steps)
    o, ocounts = O.fixed_boxes(oracle_spec(spec), steps)
    assert list(counts) == ocounts
    for x, y in zip(t.leaves(), o.leaves()):
        np.testing.assert_array_equal(x, y)
