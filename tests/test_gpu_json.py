"""GPU: trees and transition matrices saved from and loaded into device objects, in the
reference's JSON format (fixtures written by the reference's own save functions)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

B = pytest.importorskip("b12_b200")
from b12_b200.workloads import HENON_CENTER, HENON_RADIUS  # noqa: E402

FILES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "files")


@pytest.fixture(scope="module", autouse=True)
def _device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def henon_d8():
    t = B.ImplicitBoxTree(HENON_CENTER, HENON_RADIUS)
    sc = B.Scheme(B.henon(), B.inner_grid(4))
    t.subdivision_run(sc, 8)
    return t, sc


def test_saved_tree_and_matrix_equal_the_reference_files(tmp_path):
    t, sc = henon_d8()
    t.save(tmp_path / "tree")
    t.transition_matrix(sc).save(tmp_path / "tm.json")
    for part in ("tree", "tm"):
        with open(os.path.join(FILES, f"henon_d8_files_{part}.json"), "rb") as f:
            want = f.read()
        with open(tmp_path / f"{part}.json", "rb") as f:
            assert f.read() == want, part


def test_loaded_tree_continues_like_the_original(tmp_path):
    # a tree read from the reference's file subdivides and images like the tree it came from
    t = B.ImplicitBoxTree.load(os.path.join(FILES, "henon_d8_files_tree.json"))
    ref, sc = henon_d8()
    for x, y in zip(t.leaves(), ref.leaves()):
        np.testing.assert_array_equal(x, y)
    a = t.subdivision_run(sc, 4)
    b = ref.subdivision_run(sc, 4)
    np.testing.assert_array_equal(a, b)
    for x, y in zip(t.transition_matrix(sc).to_host(), ref.transition_matrix(sc).to_host()):
        np.testing.assert_array_equal(x, y)


def test_loaded_matrix_gives_the_same_measure():
    t, sc = henon_d8()
    m = t.transition_matrix(sc)
    loaded = B.CsrMatrix.load(os.path.join(FILES, "henon_d8_files_tm.json"))
    for x, y in zip(loaded.to_host(), m.to_host()):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(loaded.invariant_measure(200), m.invariant_measure(200))


def test_mixed_depth_files_round_trip_byte_for_byte(tmp_path):
    """A tree whose leaves have different depths (written by the reference's save) loads,
    saves back to the same bytes, and gives the reference's transition-matrix file."""
    t = B.ImplicitBoxTree.load(os.path.join(FILES, "henon_d8_mixed4_files_tree.json"))
    codes, depths, flags = t.leaves()
    assert depths.min() == 8 and depths.max() == 12 and t.depth() == 12
    t.save(tmp_path / "tree")
    t.transition_matrix(B.Scheme(B.henon(), B.inner_grid(4))).save(tmp_path / "tm.json")
    for part in ("tree", "tm"):
        with open(os.path.join(FILES, f"henon_d8_mixed4_files_{part}.json"), "rb") as f:
            want = f.read()
        with open(tmp_path / f"{part}.json", "rb") as f:
            assert f.read() == want, part


def test_nested_leaves_are_refused(tmp_path):
    from b12_b200 import tree as T
    c, r, codes, depths, flags = T.json_read_leaves(os.path.join(FILES, "henon_d8_files_tree.json"))
    # a depth-7 box in front of its own depth-8 half: the leaves overlap
    parent = codes[0] >> np.uint64(1)
    codes = np.concatenate([[parent], codes]).astype(np.uint64)
    depths = np.concatenate([[7], depths]).astype(np.uint8)
    flags = np.concatenate([[flags[0]], flags]).astype(np.uint8)
    T.json_write_leaves(tmp_path / "nested.json", c, r, codes, depths, flags)
    with pytest.raises(B.B12gError) as e:
        B.ImplicitBoxTree.load(tmp_path / "nested.json")
    assert e.value.status == B._lib.ERR_INVALID
