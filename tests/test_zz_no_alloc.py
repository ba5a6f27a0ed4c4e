"""GPU: the allocation-free invariant measure against the allocating entry point.

b12g_invariant_measure_noalloc serves callers that cannot let the library allocate
device memory (their own memory pool owns the free HBM, or cudaMalloc/cudaFree would
synchronize the device inside a latency-critical loop).  Its scratch lives in one fixed
__device__ array, so two calls in a row must each give the same measure as
b12g_invariant_measure, within the tolerance the other measure tests use.  The file is
named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

B = pytest.importorskip("b12_b200")
from b12_b200 import _lib  # noqa: E402

MEASURE_L1 = 1e-12
MAX_ROWS = 1 << 18


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def transpose(rowptr, cols, vals, n):
    """CSR of P^T with the sources ascending in every row."""
    rows = np.repeat(np.arange(n, dtype=np.uint32), np.diff(rowptr).astype(np.int64))
    keep = cols < n
    rows, c, v = rows[keep], cols[keep], vals[keep]
    order = np.lexsort((rows, c))
    tptr = np.zeros(n + 1, dtype=np.uint32)
    tptr[1:] = np.cumsum(np.bincount(c, minlength=n))
    return tptr, rows[order], v[order]


def device_u32(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()


def test_noalloc_measure_matches_allocating_entry_point(torch):
    sc = B.Scheme(B.lorenz(rho=28.0), B.inner_grid(5))
    tree = B.ImplicitBoxTree([0.0, 0.0, 27.0], [30.0, 30.0, 40.0])
    tree.subdivision_run(sc, 18)
    P = tree.transition_matrix(sc)
    rowptr, cols, vals = P.to_host()
    n = P.n_rows
    expect = P.invariant_measure(200)

    tptr, trows, tvals = transpose(rowptr, cols, vals, n)
    d_tptr, d_trows = device_u32(torch, tptr), device_u32(torch, trows)
    d_tvals = torch.from_numpy(np.ascontiguousarray(tvals)).cuda()
    d_v = torch.empty(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    L = _lib.lib()
    for call in range(2):
        d_v.fill_(float("nan"))
        st = L.b12g_invariant_measure_noalloc(d_tptr.data_ptr(), d_trows.data_ptr(), d_tvals.data_ptr(), n, 200,
                                              d_v.data_ptr(), ctypes.c_void_p(stream))
        assert st == _lib.OK, L.b12g_last_error()
        torch.cuda.synchronize()
        got = d_v.cpu().numpy()
        l1 = np.abs(got - expect).sum()
        assert l1 < MEASURE_L1, (call, l1)


def test_noalloc_measure_after_a_larger_call_and_on_a_bad_matrix(torch):
    """The scratch keeps the last call's iterates and barrier words: a smaller matrix
    after a larger one must still match the allocating entry point, and a matrix with a
    source index >= n is refused before the iteration reads anything."""
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for depth, mp, center, radius, grid in ((18, B.lorenz(rho=28.0), [0.0, 0.0, 27.0], [30.0, 30.0, 40.0], 5),
                                            (8, B.henon(1.4, 0.3), [0.0, 0.0], [1.5, 0.45], 4)):
        sc = B.Scheme(mp, B.inner_grid(grid))
        tree = B.ImplicitBoxTree(center, radius)
        tree.subdivision_run(sc, depth)
        P = tree.transition_matrix(sc)
        rowptr, cols, vals = P.to_host()
        n = P.n_rows
        expect = P.invariant_measure(200)
        tptr, trows, tvals = transpose(rowptr, cols, vals, n)
        d_tptr, d_trows = device_u32(torch, tptr), device_u32(torch, trows)
        d_tvals = torch.from_numpy(np.ascontiguousarray(tvals)).cuda()
        d_v = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        st = L.b12g_invariant_measure_noalloc(d_tptr.data_ptr(), d_trows.data_ptr(), d_tvals.data_ptr(), n, 200,
                                              d_v.data_ptr(), ctypes.c_void_p(stream))
        assert st == _lib.OK, L.b12g_last_error()
        torch.cuda.synchronize()
        l1 = np.abs(d_v.cpu().numpy() - expect).sum()
        assert l1 < MEASURE_L1, (depth, l1)
    bad = trows.copy()
    bad[len(bad) // 2] = n
    d_bad = device_u32(torch, bad)
    st = L.b12g_invariant_measure_noalloc(d_tptr.data_ptr(), d_bad.data_ptr(), d_tvals.data_ptr(), n, 200,
                                          d_v.data_ptr(), ctypes.c_void_p(stream))
    assert st == _lib.ERR_INVALID, st
    assert b"trows" in L.b12g_last_error()


def test_noalloc_rejects_more_boxes_than_its_scratch(torch):
    L = _lib.lib()
    one = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = one.data_ptr()
    st = L.b12g_invariant_measure_noalloc(p, p, p, MAX_ROWS + 1, 10, p, None)
    assert st == _lib.ERR_CAPACITY
    assert b"262144" in L.b12g_last_error()
