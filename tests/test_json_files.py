"""CPU: tree and transition-matrix files in the reference's JSON format.

The fixtures under tests/golden/files/ were written by the reference's own
ImplicitBoxTree::save and CooMatrix::save (tests/golden/make_golden.py).  The library's
writer must reproduce them byte for byte from the oracle's leaves and matrix, its reader
must recover exactly those arrays, and the reference's own loaders must read the
library's files (when the reference harness has been built here)."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

B = pytest.importorskip("b12_b200")
from b12_b200 import tree as T  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = os.path.join(HERE, "golden", "files")
REF_LOAD = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ref_load")

CASES = [("henon_d8_files", O.henon_spec, 8, False), ("henon_d10_lost_files", O.henon_spec, 10, True),
         ("lorenz_d9_files", O.lorenz_spec, 9, False)]


def oracle_run(spec_fn, steps, invalid):
    spec = spec_fn()
    o = O.Oracle(spec)
    o.subdivision(steps)
    return spec, o.leaves(), o.transition_matrix(invalid=invalid)


@pytest.mark.parametrize("name,spec_fn,steps,invalid", CASES)
def test_writer_reproduces_the_reference_files(tmp_path, name, spec_fn, steps, invalid):
    spec, (codes, depths, flags), (rowptr, cols, vals, ncols) = oracle_run(spec_fn, steps, invalid)
    T.json_write_leaves(tmp_path / "tree", spec["center"], spec["radius"], codes, depths, flags)
    T.json_write_coo(tmp_path / "tm", len(rowptr) - 1, ncols, rowptr, cols, vals)
    for part in ("tree", "tm"):
        with open(os.path.join(FILES, f"{name}_{part}.json"), "rb") as f:
            want = f.read()
        with open(tmp_path / f"{part}.json", "rb") as f:   # ".json" appended like the reference
            got = f.read()
        assert got == want, part


@pytest.mark.parametrize("name,spec_fn,steps,invalid", CASES)
def test_reader_recovers_the_reference_files(name, spec_fn, steps, invalid):
    spec, (codes, depths, flags), (rowptr, cols, vals, ncols) = oracle_run(spec_fn, steps, invalid)
    c, r, fc, fd, ff = T.json_read_leaves(os.path.join(FILES, f"{name}_tree.json"))
    assert c == list(spec["center"]) and r == list(spec["radius"])
    for x, y in ((fc, codes), (fd, depths), (ff, flags)):
        np.testing.assert_array_equal(x, y)
    nr, nc, rp, cl, vl = T.json_read_coo(os.path.join(FILES, f"{name}_tm.json"))
    assert (nr, nc) == (len(rowptr) - 1, ncols)
    for x, y in ((rp, rowptr), (cl, cols), (vl, vals)):
        np.testing.assert_array_equal(x, y)


@pytest.mark.skipif(not os.path.exists(REF_LOAD), reason="reference harness not built here")
def test_reference_loaders_read_the_library_files(tmp_path):
    spec, (codes, depths, flags), (rowptr, cols, vals, ncols) = oracle_run(O.lorenz_spec, 9, False)
    T.json_write_leaves(tmp_path / "t.json", spec["center"], spec["radius"], codes, depths, flags)
    T.json_write_coo(tmp_path / "m.json", len(rowptr) - 1, ncols, rowptr, cols, vals)
    subprocess.run([REF_LOAD, "--dim", "3", "--tree", str(tmp_path / "t.json"), "--leaves",
                    str(tmp_path / "leaves.bin")], check=True, capture_output=True)
    subprocess.run([REF_LOAD, "--coo", str(tmp_path / "m.json"), "--out", str(tmp_path / "coo.bin")],
                   check=True, capture_output=True)
    with open(tmp_path / "leaves.bin", "rb") as f:
        n = int(np.frombuffer(f.read(8), "<u8")[0])
        np.testing.assert_array_equal(np.frombuffer(f.read(8 * n), "<u8"), codes)
        np.testing.assert_array_equal(np.frombuffer(f.read(n), np.uint8), depths)
        np.testing.assert_array_equal(np.frombuffer(f.read(n), np.uint8), flags)
    with open(tmp_path / "coo.bin", "rb") as f:
        nnz = int(np.frombuffer(f.read(8), "<u8")[0])
        nr, nc = np.frombuffer(f.read(8), "<u4")
        rows = np.frombuffer(f.read(4 * nnz), "<u4")
        np.testing.assert_array_equal(np.frombuffer(f.read(4 * nnz), "<u4"), cols)
        np.testing.assert_array_equal(np.frombuffer(f.read(8 * nnz), "<f8"), vals)
    assert (int(nr), int(nc)) == (len(rowptr) - 1, ncols)
    np.testing.assert_array_equal(np.repeat(np.arange(len(rowptr) - 1), np.diff(rowptr)), rows)


def test_unsupported_files_are_refused(tmp_path):
    with pytest.raises(B.B12gError):
        T.json_read_leaves(tmp_path / "missing.json")
    text = open(os.path.join(FILES, "henon_d8_files_tree.json")).read()
    # a subdivision scheme other than the default one
    bad = text.replace('"sdScheme": [\n    0,\n    1,', '"sdScheme": [\n    1,\n    0,', 1)
    (tmp_path / "sd.json").write_text(bad)
    with pytest.raises(B.B12gError):
        T.json_read_leaves(tmp_path / "sd.json")
    (tmp_path / "short.json").write_text(text.replace('"nLeaves": 81', '"nLeaves": 80'))
    with pytest.raises(B.B12gError):
        T.json_read_leaves(tmp_path / "short.json")
