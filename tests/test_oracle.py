"""CPU: the oracle (plain-C restatement) against the reference's own outputs.

The golden fixtures were produced by the reference's ImplicitBoxTree compiled from its
headers (tests/golden/make_golden.py); these tests pin the oracle to them before the
oracle is trusted as the checker of the CUDA library.
"""
import numpy as np
import pytest

from oracle import oracle as O
from workloads import csr_digests, oracle_spec, sha

SUBDIVISION_CASES = ["henon_d20", "henon_a1.0_d16", "lorenz_d15", "forced_duffing_d16", "lorenz_rho15_d18",
                     "lorenz_scan0_i2_d21_fma"]


@pytest.mark.parametrize("name", SUBDIVISION_CASES)
def test_subdivision_matches_reference(golden, name):
    meta, arrays = golden(name)
    o = O.Oracle(oracle_spec(meta["spec"]))
    o.set_flags(8)
    for st in meta["steps"]:
        o.subdivide(8)
        o.set_flags_by_image(1)
        o.remove(1)
        o.unset_flags(1)
        codes, depth, flags = o.leaves()
        assert len(codes) == st["n"], f"step {st['step']}"
        assert sha(codes) == st["codes_sha256"], f"step {st['step']} codes"
        assert sha(flags) == st["flags_sha256"], f"step {st['step']} flags"


@pytest.mark.parametrize("name,absolute,invalid", [
    ("henon_d20", False, False), ("henon_d12_abs", True, False), ("henon_d12_lost", False, True),
    ("lorenz_d15", False, False), ("forced_duffing_d16", False, False),
    ("lorenz_rho15_d4_invalid_column_unused", False, True), ("lorenz_scan0_i2_d21_fma", False, False)])
def test_transition_matrix_matches_reference(golden, name, absolute, invalid):
    meta, arrays = golden(name)
    o = O.Oracle(oracle_spec(meta["spec"]))
    counts, _ = o.subdivision(len(meta["steps"]))
    assert counts[-1] == meta["steps"][-1]["n"]
    rowptr, cols, vals, ncols = o.transition_matrix(absolute=absolute, invalid=invalid)
    d = csr_digests(rowptr, cols, vals)
    tm = meta["tm"]
    assert ncols == tm["n_cols"]
    for k in ("nnz", "rowptr_sha256", "cols_sha256", "vals_sha256"):
        assert d[k] == tm[k], k


def test_oracle_counts_henon_known_answer():
    # the reference's documented Henon example gives 14,733 boxes and 37,023 nonzeros
    o = O.Oracle(O.henon_spec())
    counts, box_images = o.subdivision(20)
    assert counts[-1] == 14733
    assert box_images == 2 * int(np.sum(np.concatenate([[1], counts[:-1]])))
    rowptr, cols, vals, _ = o.transition_matrix()
    assert len(cols) == 37023
    # rows are stochastic up to points that leave the domain
    sums = np.add.reduceat(vals, rowptr[:-1][np.diff(rowptr) > 0])
    assert np.all(sums <= 1.0 + 1e-12)


def test_point_code_edge_wraps_like_reference():
    # ((p - c) / r + 1) / 2 rounds to 1.0 just below c + r: the reference drops the
    # overflow bit, so the point lands in box index 0 of that dimension
    o = O.Oracle(O.lorenz_spec())
    p = np.array([np.nextafter(30.0, 0.0), 0.0, 27.0])
    code, ok = o.point_code64(p)
    assert ok
    # dimension 0 occupies bit positions 0, 3, ..., 63 of the depth-64 code
    dim0 = sum(((code >> (3 * i)) & 1) << i for i in range(22))
    u = ((p[0] - 0.0) / 30.0 + 1.0) / 2.0
    if u == 1.0:
        assert dim0 == 0
    outside, ok2 = o.point_code64(np.array([30.0, 0.0, 27.0]))
    assert not ok2 and outside == 2**64 - 1


def test_invariant_measure_is_fixed_point():
    o = O.Oracle(O.henon_spec())
    o.subdivision(12)
    rowptr, cols, vals, _ = o.transition_matrix()
    v = O.invariant_measure(rowptr, cols, vals, 400)
    assert abs(v.sum() - 1.0) < 1e-12 and (v >= 0).all()
    w = np.zeros_like(v)
    for i in range(len(v)):
        for e in range(rowptr[i], rowptr[i + 1]):
            w[cols[e]] += vals[e] * v[i]
    w /= np.abs(w).sum()
    assert np.abs(w - v).sum() < 1e-3


def test_philox_known_answer():
    # Random123's published known-answer vectors for philox4x32_10
    import ctypes as C
    L = O.lib()
    for ctr, key, expect in [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]:
        c = (C.c_uint32 * 4)(*ctr)
        L.orc_philox4x32_10(c, key[0], key[1])
        assert tuple(c) == expect


@pytest.mark.parametrize("name", ["coupled_duffing_cont_d8", "coupled_duffing_cont_d12"])
def test_continuation_matches_reference(golden, name):
    meta, arrays = golden(name)
    spec = meta["spec"]
    o, counts = O.continuation(oracle_spec(spec), spec["depth"], np.zeros(4))
    ref = [s for s in meta["steps"] if s["step"] > 0]
    assert counts == [s["n"] for s in ref]
    codes, depth, flags = o.leaves()
    assert sha(codes) == ref[-1]["codes_sha256"] and sha(flags) == ref[-1]["flags_sha256"]


def test_continuation_each_sweep_matches_reference(golden):
    meta, arrays = golden("coupled_duffing_cont_d8")
    o = O.Oracle(oracle_spec(meta["spec"]))
    o.delete_depth0()
    o.insert_points(np.zeros(4), 8, 2)
    for st in meta["steps"]:
        if st["step"] > 0:
            o.change_flags(2, 4)
            o.insert_by_image(4, 2, 0)
            o.unset_flags(4)
        codes, depth, flags = o.leaves()
        assert len(codes) == st["n"] and sha(codes) == st["codes_sha256"] and sha(flags) == st["flags_sha256"]
