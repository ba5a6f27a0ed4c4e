"""Python mirror of the reference's ImplicitBoxTree for the box-image path.

Method names follow the reference (B12c/src/include/ImplicitBoxTree.h:72-603) in
snake_case; the reference's camelCase names are provided as aliases.  Every call goes
through the C ABI of libb12g.so (include/b12g.h) and runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from ._lib import check, lib

LEAF = L.LEAF_DEPTH


# ----------------------------------------------------------------------------- schemes
@dataclass
class MapSpec:
    kind: int
    steps: int = 1
    h: float = 0.0
    p: tuple = ()
    arith: int = L.ARITH_STRICT

    def to_c(self) -> L.Map:
        m = L.Map()
        m.kind, m.arith, m.steps, m.h = self.kind, self.arith, self.steps, self.h
        for i, v in enumerate(self.p):
            m.p[i] = v
        return m


@dataclass
class GridSpec:
    kind: int
    n: int = 1
    points: int = 1
    seed: int = 0
    eps: float = 0.0

    def to_c(self) -> L.Grid:
        g = L.Grid()
        g.kind, g.n, g.points, g.seed, g.eps = self.kind, self.n, self.points, self.seed, self.eps
        return g

    def points_per_box(self, dim: int) -> int:
        return self.points if self.kind == L.GRID_PHILOX else self.n ** dim


def henon(a: float = 1.4, b: float = 0.3, steps: int = 1) -> MapSpec:
    """Henon<2,double>(a, b, steps) (Map_Henon.h:27-40)."""
    return MapSpec(L.MAP_HENON, steps=steps, p=(a, b))


def lorenz(sigma: float = 10.0, rho: float = 28.0, beta: float = 8.0 / 3.0, h: float = 0.01, steps: int = 20,
           fma: bool = False) -> MapSpec:
    """Lorenz<3,double>(sigma, rho, beta, h, steps) (Map_Lorenz.h:27-44); fma=True uses
    explicit fused multiply-adds in the integrator."""
    return MapSpec(L.MAP_LORENZ, steps=steps, h=h, p=(sigma, rho, beta), arith=L.ARITH_FMA if fma else L.ARITH_STRICT)


def coupled_duffing(h: float = 0.05, steps: int = 10) -> MapSpec:
    """Stormer-Verlet map of H = |p|^2/2 - q1^2/2 + q1^4/4 + 1.69 q2^2/2 + 0.1 q1^2 q2^2."""
    return MapSpec(L.MAP_COUPLED_DUFFING, steps=steps, h=h)


FORCED_PERIOD = 2.0 * 3.14159265358979323846


def forced_duffing(steps: int = 200, delta: float = 0.25, alpha: float = -1.0, beta: float = 1.0,
                   gamma: float = 0.3) -> MapSpec:
    """Period-2pi map of x'' + delta x' + alpha x + beta x^3 = gamma cos t, `steps` RK4 steps."""
    return MapSpec(L.MAP_FORCED_DUFFING, steps=steps, h=FORCED_PERIOD / steps, p=(delta, alpha, beta, gamma))


def inner_grid(n: int) -> GridSpec:
    """InnerGrid<DIM,double>(n) (Grids.hpp:103-134)."""
    return GridSpec(L.GRID_INNER, n=n)


def full_grid(n: int, eps: float = 0.0) -> GridSpec:
    """FullGrid<DIM,double>(n, eps) (Grids.hpp:60-95)."""
    return GridSpec(L.GRID_FULL, n=n, eps=eps)


def philox_grid(points: int, seed: int = 0) -> GridSpec:
    """`points` uniform points per box from Philox4x32-10 keyed by (seed, point index)."""
    return GridSpec(L.GRID_PHILOX, points=points, seed=seed)


@dataclass
class Scheme:
    """The Matlab driver's {grid, map, depth, flags} point-iterator description."""
    map: MapSpec
    grid: GridSpec
    depth: int = LEAF
    flags_to_check: int = 0

    def to_c(self) -> L.Scheme:
        s = L.Scheme()
        s.map = self.map.to_c()
        s.grid = self.grid.to_c()
        s.depth = self.depth
        s.flags_to_check = self.flags_to_check
        return s


# ----------------------------------------------------------------------------- matrices
class CsrMatrix:
    """Row-major transition matrix resident on the GPU (row = source leaf)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        r, c, z = C.c_uint32(), C.c_uint32(), C.c_uint64()
        check(lib().b12g_csr_shape(self._h, C.byref(r), C.byref(c), C.byref(z)), "csr_shape")
        self.n_rows, self.n_cols, self.nnz = r.value, c.value, z.value

    def to_host(self):
        rowptr = np.zeros(self.n_rows + 1, dtype=np.uint32)
        cols = np.zeros(max(self.nnz, 1), dtype=np.uint32)
        vals = np.zeros(max(self.nnz, 1), dtype=np.float64)
        check(lib().b12g_csr_copy(self._h, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data), "csr_copy")
        return rowptr, cols[: self.nnz], vals[: self.nnz]

    def invariant_measure(self, iters: int = 200, out=None, keep_on_device: bool = False):
        """FP64 power iteration; returns the measure (into `out` if given), or None with
        keep_on_device=True (fetch it later with measure())."""
        if keep_on_device:
            check(lib().b12g_invariant_measure(self._h, iters, None), "invariant_measure")
            return None
        v = np.zeros(self.n_rows, dtype=np.float64) if out is None else out
        check(lib().b12g_invariant_measure(self._h, iters, v.ctypes.data), "invariant_measure")
        return v

    def invariant_measure_tol(self, tol: float = 1e-14, max_iters: int = 1_000_000, check_every: int = 20,
                              out=None):
        """The power iteration until one iteration changes the measure by at most `tol` in
        L1 (checked every `check_every` iterations); returns (measure, iterations, change)."""
        v = np.zeros(self.n_rows, dtype=np.float64) if out is None else out
        k = C.c_uint32()
        ch = C.c_double()
        check(lib().b12g_invariant_measure_tol(self._h, float(tol), int(max_iters), int(check_every), v.ctypes.data,
                                               C.byref(k), C.byref(ch)), "invariant_measure_tol")
        return v, k.value, ch.value

    def measure(self, out=None) -> np.ndarray:
        v = np.zeros(self.n_rows, dtype=np.float64) if out is None else out
        check(lib().b12g_csr_measure(self._h, v.ctypes.data), "csr_measure")
        return v

    def to_host_into(self, rowptr, cols, vals):
        check(lib().b12g_csr_copy(self._h, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data), "csr_copy")

    def strong_components(self):
        """(labels, count): every row's strongly connected component, labelled by its largest row."""
        comp = np.zeros(self.n_rows, dtype=np.uint32)
        k = C.c_uint32()
        check(lib().b12g_csr_strong_components(self._h, comp.ctypes.data, C.byref(k)), "csr_strong_components")
        return comp, k.value

    def save(self, path: str) -> None:
        """CooMatrix::save (CooMatrix.hpp:473-525): the reference's JSON file."""
        check(lib().b12g_csr_save_json(self._h, str(path).encode()), "csr_save_json")

    @classmethod
    def load(cls, path: str) -> "CsrMatrix":
        """CooMatrix(fileName) (CooMatrix.hpp:236-291): a matrix from the reference's JSON file."""
        h = C.c_void_p()
        check(lib().b12g_csr_load_json(str(path).encode(), C.byref(h)), "csr_load_json")
        return cls(h)

    def close(self):
        if self._h:
            lib().b12g_csr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------------------- JSON files (host arrays)
def json_write_leaves(path, center, radius, codes, depths, flags) -> None:
    """Write leaves in the reference's tree JSON format (no device involved)."""
    d = L.Domain()
    d.dim = len(center)
    for j in range(d.dim):
        d.center[j], d.radius[j] = float(center[j]), float(radius[j])
    codes = np.ascontiguousarray(codes, dtype=np.uint64)
    depths = np.ascontiguousarray(depths, dtype=np.uint8)
    flags = np.ascontiguousarray(flags, dtype=np.uint8)
    check(lib().b12g_json_write_leaves(str(path).encode(), C.byref(d), codes.ctypes.data, depths.ctypes.data,
                                       flags.ctypes.data, len(codes)), "json_write_leaves")


def json_read_leaves(path):
    """(center, radius, codes, depths, flags) of a tree JSON file (no device involved)."""
    d = L.Domain()
    n = C.c_uint64(0)
    check(lib().b12g_json_read_leaves(str(path).encode(), C.byref(d), None, None, None, C.byref(n)), "json_read_leaves")
    codes = np.zeros(n.value, dtype=np.uint64)
    depths = np.zeros(n.value, dtype=np.uint8)
    flags = np.zeros(n.value, dtype=np.uint8)
    check(lib().b12g_json_read_leaves(str(path).encode(), C.byref(d), codes.ctypes.data, depths.ctypes.data,
                                      flags.ctypes.data, C.byref(n)), "json_read_leaves")
    return list(d.center[: d.dim]), list(d.radius[: d.dim]), codes, depths, flags


def json_write_coo(path, n_rows, n_cols, rowptr, cols, vals) -> None:
    """Write CSR arrays in the reference's CooMatrix JSON format (no device involved)."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    check(lib().b12g_json_write_coo(str(path).encode(), n_rows, n_cols, rowptr.ctypes.data, cols.ctypes.data,
                                    vals.ctypes.data), "json_write_coo")


def json_read_coo(path):
    """(n_rows, n_cols, rowptr, cols, vals) of a CooMatrix JSON file (no device involved)."""
    r, c, z = C.c_uint32(), C.c_uint32(), C.c_uint64()
    check(lib().b12g_json_read_coo(str(path).encode(), C.byref(r), C.byref(c), None, None, None, C.byref(z)),
          "json_read_coo")
    rowptr = np.zeros(r.value + 1, dtype=np.uint32)
    cols = np.zeros(max(z.value, 1), dtype=np.uint32)
    vals = np.zeros(max(z.value, 1), dtype=np.float64)
    check(lib().b12g_json_read_coo(str(path).encode(), C.byref(r), C.byref(c), rowptr.ctypes.data, cols.ctypes.data,
                                   vals.ctypes.data, C.byref(z)), "json_read_coo")
    return r.value, c.value, rowptr, cols[: z.value], vals[: z.value]


def launch_count() -> int:
    n = C.c_uint64()
    check(lib().b12g_launch_count(C.byref(n)), "launch_count")
    return n.value


def probe_fp64_fma(seconds: float = 0.2):
    """FP64 FMA throughput of the current device in TFLOP/s (and the probe's seconds)."""
    tf, sec = C.c_double(), C.c_double()
    check(lib().b12g_probe_fp64_fma(seconds, C.byref(tf), C.byref(sec)), "probe_fp64_fma")
    return tf.value, sec.value


# ----------------------------------------------------------------------------- tree
class ImplicitBoxTree:
    """ImplicitBoxTree<CUDA, DIM, double, 64> on one B200 (uniform leaf depth)."""

    def __init__(self, center, radius):
        center = list(map(float, center))
        radius = list(map(float, radius))
        if len(center) != len(radius) or not 1 <= len(center) <= L.MAX_DIM:
            raise ValueError("center and radius must have the same length 1..4")
        d = L.Domain()
        d.dim = len(center)
        for j in range(d.dim):
            d.center[j] = center[j]
            d.radius[j] = radius[j]
        self.dim = d.dim
        self._h = C.c_void_p()
        check(lib().b12g_tree_create(C.byref(d), C.byref(self._h)), "tree_create")

    def close(self):
        if self._h:
            lib().b12g_tree_destroy(self._h)
            self._h = None

    def save(self, path: str) -> None:
        """ImplicitBoxTree::save (ImplicitBoxTree.hpp:435-528): the reference's JSON file."""
        check(lib().b12g_tree_save_json(self._h, str(path).encode()), "tree_save_json")

    @classmethod
    def load(cls, path: str) -> "ImplicitBoxTree":
        """ImplicitBoxTree(fileName) (ImplicitBoxTree.hpp:144-359): a tree from the reference's JSON file."""
        h = C.c_void_p()
        check(lib().b12g_tree_load_json(str(path).encode(), C.byref(h)), "tree_load_json")
        t = cls.__new__(cls)
        d = L.Domain()
        n = C.c_uint64(0)
        check(lib().b12g_json_read_leaves(str(path).encode(), C.byref(d), None, None, None, C.byref(n)),
              "json_read_leaves")
        t.dim = d.dim
        t._h = h
        return t

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- queries
    def count(self, depth: int = LEAF) -> int:
        c = C.c_uint32()
        check(lib().b12g_count(self._h, depth, C.byref(c)), "count")
        return c.value

    def depth(self) -> int:
        d = C.c_uint8()
        check(lib().b12g_depth(self._h, C.byref(d)), "depth")
        return d.value

    def leaves(self):
        n = self.count()
        codes = np.zeros(n, dtype=np.uint64)
        depth = np.zeros(n, dtype=np.uint8)
        flags = np.zeros(n, dtype=np.uint8)
        check(lib().b12g_leaves(self._h, codes.ctypes.data, depth.ctypes.data, flags.ctypes.data), "leaves")
        return codes, depth, flags

    def load_leaves(self, codes, depth, flags):
        codes = np.ascontiguousarray(codes, dtype=np.uint64)
        depth = np.ascontiguousarray(depth, dtype=np.uint8)
        flags = np.ascontiguousarray(flags, dtype=np.uint8)
        check(lib().b12g_load_leaves(self._h, codes.ctypes.data, depth.ctypes.data, flags.ctypes.data, len(codes)),
              "load_leaves")

    def reserve(self, n_boxes: int):
        check(lib().b12g_tree_reserve(self._h, n_boxes), "reserve")

    # ---- flags
    def _n(self, fn, *args):
        c = C.c_uint32()
        check(getattr(lib(), fn)(self._h, *args, C.byref(c)), fn)
        return c.value

    def set_flags(self, flags: int, depth: int = LEAF, count: bool = True):
        """Returns the leaves that changed, or None with count=False (no device read-back)."""
        if not count:
            check(lib().b12g_set_flags(self._h, flags, depth, None), "b12g_set_flags")
            return None
        return self._n("b12g_set_flags", flags, depth)

    def unset_flags(self, flags: int, depth: int = LEAF, count: bool = True):
        """Returns the leaves that changed, or None with count=False (no device read-back)."""
        if not count:
            check(lib().b12g_unset_flags(self._h, flags, depth, None), "b12g_unset_flags")
            return None
        return self._n("b12g_unset_flags", flags, depth)

    def change_flags(self, to_unset: int, to_set: int, depth: int = LEAF) -> int:
        return self._n("b12g_change_flags", to_unset, to_set, depth)

    # ---- structure
    def subdivide(self, flags: int = L.SD) -> int:
        return self._n("b12g_subdivide", flags)

    def remove(self, flags: int) -> int:
        return self._n("b12g_remove", flags)

    def delete_depth(self, depth: int) -> int:
        return self._n("b12g_delete_depth", depth)

    def unsubdivide(self, flags: int = L.SD) -> int:
        return self._n("b12g_unsubdivide", flags)

    # ---- box images
    def set_flags_by_image(self, scheme: Scheme, flags: int, depth: int = LEAF) -> int:
        s = scheme.to_c()
        return self._n("b12g_set_flags_by_image", C.byref(s), flags, depth)

    def search_by_image(self, scheme: Scheme, depth: int = LEAF) -> np.ndarray:
        s = scheme.to_c()
        n = C.c_uint64()
        check(lib().b12g_search_by_image(self._h, C.byref(s), depth, None, 0, C.byref(n)), "search_by_image")
        out = np.zeros(max(n.value, 1), dtype=np.uint32)
        check(lib().b12g_search_by_image(self._h, C.byref(s), depth, out.ctypes.data, len(out), C.byref(n)),
              "search_by_image")
        return out[: n.value]

    def insert_points(self, points, depth: int, flags_for_inserted: int = L.INS, flags_for_hit: int = L.NONE) -> int:
        pts = np.ascontiguousarray(points, dtype=np.float64)
        return self._n("b12g_insert_points", pts.ctypes.data, pts.size // self.dim, depth, flags_for_inserted,
                       flags_for_hit)

    def insert_by_image(self, scheme: Scheme, depth: int, flags_for_inserted: int = L.INS,
                        flags_for_hit: int = L.NONE) -> int:
        s = scheme.to_c()
        return self._n("b12g_insert_by_image", C.byref(s), depth, flags_for_inserted, flags_for_hit)

    def transition_matrix(self, scheme: Scheme, absolute: bool = False, invalid_column: bool = False,
                          into: "CsrMatrix | None" = None) -> CsrMatrix:
        """Build the matrix; `into` refills an existing matrix in place (no new device memory)."""
        s = scheme.to_c()
        h = C.c_void_p(into._h.value if into is not None else None)
        check(lib().b12g_transition_matrix(self._h, C.byref(s), int(absolute), int(invalid_column), C.byref(h)),
              "transition_matrix")
        if into is not None:
            into.__init__(h)
            return into
        return CsrMatrix(h)

    # ---- device buffers of a range-partitioned tree (torch tensors on this tree's GPU)
    # Every call waits for torch's current stream first (the tensors, or the memory torch
    # just handed out for them, may still be in use by work queued there, a collective
    # among it) and returns after its own work, queued on the tree's stream, has finished.
    @staticmethod
    def _ready(*tensors):
        import torch
        for x in tensors:
            if x is not None and x.is_cuda:
                torch.cuda.current_stream(x.device).synchronize()
                return

    def image_point_boxes(self, scheme: Scheme, device):
        """(codes, valid): the depth-64 point boxes of the images of the scheme's sources,
        source-major, as int64 (the code's bits) and uint8 tensors on `device`."""
        import torch
        room = self.count() * scheme.grid.points_per_box(self.dim)
        codes = torch.empty(max(room, 1), dtype=torch.int64, device=device)
        valid = torch.empty(max(room, 1), dtype=torch.uint8, device=device)
        n = C.c_uint64()
        s = scheme.to_c()
        self._ready(codes)
        check(lib().b12g_image_point_boxes(self._h, C.byref(s), codes.data_ptr(), valid.data_ptr(), room,
                                           C.byref(n)), "image_point_boxes")
        return codes[: n.value], valid[: n.value]

    def image_distinct_point_boxes(self, scheme: Scheme, device, depth: int = 64):
        """(codes, valid): the point boxes of image_point_boxes cut to their first `depth`
        bisections, as a set (each distinct box of 32 consecutive points once, in no fixed
        order), for the flags of a step over leaves no deeper than `depth`."""
        import torch
        room = self.count() * scheme.grid.points_per_box(self.dim)
        codes = torch.empty(max(room, 1), dtype=torch.int64, device=device)
        valid = torch.empty(max(room, 1), dtype=torch.uint8, device=device)
        n = C.c_uint64()
        s = scheme.to_c()
        self._ready(codes)
        check(lib().b12g_image_distinct_point_boxes(self._h, C.byref(s), depth, codes.data_ptr(), valid.data_ptr(),
                                                    room, C.byref(n)), "image_distinct_point_boxes")
        return codes[: n.value], valid[: n.value]

    def search_point_boxes(self, codes, valid):
        """searchByIterators over point boxes: an int64 tensor of leaf indices (-1: none)."""
        import torch
        n = codes.numel()
        out = torch.empty(max(n, 1), dtype=torch.int32, device=codes.device)
        self._ready(codes, valid)
        check(lib().b12g_search_point_boxes(self._h, codes.data_ptr(), valid.data_ptr(), n, out.data_ptr()),
              "search_point_boxes")
        return out[:n].to(torch.int64)   # B12G_INVALID_INDEX reads as -1 in int32

    def set_flags_by_point_boxes(self, codes, valid, flags: int) -> int:
        self._ready(codes, valid)
        return self._n("b12g_set_flags_by_point_boxes", codes.data_ptr(), valid.data_ptr(), codes.numel(), flags)

    def transition_rows(self, targets, points_per_row: int, n_columns: int, absolute: bool = False,
                        invalid_column: bool = False) -> CsrMatrix:
        """Rows of this tree's leaves from global targets (int32/int64 tensor, -1 for lost points)."""
        import torch
        t = targets.to(torch.int32).contiguous()
        self._ready(t)
        h = C.c_void_p()
        check(lib().b12g_transition_rows(self._h, t.data_ptr(), points_per_row, n_columns, int(absolute),
                                         int(invalid_column), C.byref(h)), "transition_rows")
        return CsrMatrix(h)

    def route_point_boxes(self, codes, valid, starts, ranks, world: int, want_slot: bool = True):
        """The point boxes grouped by the rank that owns them (b12g_route_point_boxes):
        (slot int64 tensor: position of box i in the output, or None when not wanted,
        per-rank code tensors, per-rank validity tensors).  starts: unsigned depth-64 first
        codes of the non-empty runs, ranks: their ranks (both ascending)."""
        import torch
        n = codes.numel()
        out_c = torch.empty(max(n, 1), dtype=torch.int64, device=codes.device)
        out_v = torch.empty(max(n, 1), dtype=torch.uint8, device=codes.device)
        slot = torch.empty(max(n, 1), dtype=torch.int32, device=codes.device) if want_slot else None
        st = np.ascontiguousarray(starts, dtype=np.uint64)
        rk = np.ascontiguousarray(ranks, dtype=np.uint32)
        cnt = np.zeros(world, dtype=np.uint64)
        c, v = codes.contiguous(), valid.contiguous()
        self._ready(c, v)
        check(lib().b12g_route_point_boxes(self._h, c.data_ptr(), v.data_ptr(), n, st.ctypes.data, rk.ctypes.data,
                                           len(st), world, out_c.data_ptr(), out_v.data_ptr(),
                                           slot.data_ptr() if slot is not None else None, cnt.ctypes.data),
              "route_point_boxes")
        sizes = [int(x) for x in cnt]
        return (slot[:n].to(torch.int64) if slot is not None else None, list(out_c[:n].split(sizes)),
                list(out_v[:n].split(sizes)))

    def leaf_at(self, index: int):
        """(code, depth, flags) of leaf `index` in tree order."""
        c, d, f = C.c_uint64(), C.c_uint8(), C.c_uint8()
        check(lib().b12g_leaf_at(self._h, index, C.byref(c), C.byref(d), C.byref(f)), "leaf_at")
        return c.value, d.value, f.value

    def leaves_device(self, device):
        """(codes int64, depths uint8, flags uint8) tensors of the leaves on `device`."""
        import torch
        n = self.count()
        codes = torch.empty(n, dtype=torch.int64, device=device)
        depth = torch.empty(n, dtype=torch.uint8, device=device)
        flags = torch.empty(n, dtype=torch.uint8, device=device)
        self._ready(codes)
        check(lib().b12g_leaves(self._h, codes.data_ptr(), depth.data_ptr(), flags.data_ptr()), "leaves")
        return codes, depth, flags

    def load_leaves_device(self, codes, depth, flags):
        """b12g_load_leaves from device tensors (checked on the device)."""
        c, d, f = codes.contiguous(), depth.contiguous(), flags.contiguous()
        self._ready(c, d, f)
        check(lib().b12g_load_leaves_device(self._h, c.data_ptr(), d.data_ptr(), f.data_ptr(), c.numel()),
              "load_leaves_device")

    # ---- measurement hooks
    def stream_handle(self) -> int:
        p = C.c_void_p()
        check(lib().b12g_tree_stream(self._h, C.byref(p)), "tree_stream")
        return p.value or 0

    def profile(self, enable: bool = True) -> None:
        check(lib().b12g_profile_enable(self._h, int(enable)), "profile_enable")

    def profile_read(self, kind: int, reset: bool = True):
        ms, n = C.c_double(), C.c_uint64()
        check(lib().b12g_profile_read(self._h, kind, C.byref(ms), C.byref(n), int(reset)), "profile_read")
        return ms.value, n.value

    # ---- fused drivers
    def set_flags_by_components(self, matrix: "CsrMatrix", flags: int, min_size: int = 2) -> int:
        """chainRecurrentSet.m:29-37: flag the leaves in strongly connected components of at least min_size."""
        k = C.c_uint32()
        check(lib().b12g_set_flags_by_components(self._h, matrix._h, min_size, flags, C.byref(k)),
              "set_flags_by_components")
        return k.value

    def set_flags_by_measure(self, matrix: "CsrMatrix", threshold: float, flags: int) -> int:
        """subdivisionByNim.m:56-62: flag the leaves whose invariant measure is at least `threshold`."""
        k = C.c_uint32()
        check(lib().b12g_set_flags_by_measure(self._h, matrix._h, float(threshold), flags, C.byref(k)),
              "set_flags_by_measure")
        return k.value

    def chain_recurrent_run(self, scheme: Scheme, steps: int) -> np.ndarray:
        """chainRecurrentSet.m:18-44 on the GPU; leaf counts after each step."""
        counts = np.zeros(max(steps, 1), dtype=np.uint32)
        s = scheme.to_c()
        check(lib().b12g_chain_recurrent_run(self._h, C.byref(s), steps, counts.ctypes.data), "chain_recurrent_run")
        return counts[:steps]

    def nim_run(self, scheme: Scheme, steps: int, power_iterations: int = 200) -> np.ndarray:
        """subdivisionByNim.m:22-66 with the FP64 power iteration; leaf counts after each step."""
        counts = np.zeros(max(steps, 1), dtype=np.uint32)
        s = scheme.to_c()
        check(lib().b12g_nim_run(self._h, C.byref(s), steps, power_iterations, counts.ctypes.data), "nim_run")
        return counts[:steps]

    def nim_run_tol(self, scheme: Scheme, steps: int, tol: float = 1e-14, max_iters: int = 1_000_000) -> np.ndarray:
        """The NIM driver with every step's measure run to `tol` (checked every 20 iterations)."""
        counts = np.zeros(max(steps, 1), dtype=np.uint32)
        s = scheme.to_c()
        check(lib().b12g_nim_run_tol(self._h, C.byref(s), steps, float(tol), int(max_iters), counts.ctypes.data),
              "nim_run_tol")
        return counts[:steps]

    def set_flags_by_self_hit(self, scheme: Scheme, flags: int) -> int:
        """fixedBoxes.m:15-17: flag the leaves one of whose own test points lands in them again."""
        k = C.c_uint32()
        s = scheme.to_c()
        check(lib().b12g_set_flags_by_self_hit(self._h, C.byref(s), flags, C.byref(k)), "set_flags_by_self_hit")
        return k.value

    def fixed_boxes_run(self, scheme: Scheme, steps: int) -> np.ndarray:
        """fixedBoxes.m:10-22 on the GPU; leaf counts after each step."""
        counts = np.zeros(max(steps, 1), dtype=np.uint32)
        s = scheme.to_c()
        check(lib().b12g_fixed_boxes_run(self._h, C.byref(s), steps, counts.ctypes.data), "fixed_boxes_run")
        return counts[:steps]

    def subdivision_run(self, scheme: Scheme, steps: int) -> np.ndarray:
        counts = np.zeros(max(steps, 1), dtype=np.uint32)
        s = scheme.to_c()
        check(lib().b12g_subdivision_run(self._h, C.byref(s), steps, counts.ctypes.data), "subdivision_run")
        return counts[:steps]

    def continuation_run(self, scheme: Scheme, x0, depth: int, max_sweeps: int = 100000) -> np.ndarray:
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        counts = np.zeros(max_sweeps, dtype=np.uint32)
        k = C.c_uint32()
        s = scheme.to_c()
        check(lib().b12g_continuation_run(self._h, C.byref(s), x0.ctypes.data, x0.size // self.dim, depth,
                                          max_sweeps, counts.ctypes.data, C.byref(k)), "continuation_run")
        return counts[: k.value]

    # ---- the reference's member names
    setFlags = set_flags
    unsetFlags = unset_flags
    changeFlags = change_flags
    deleteDepth = delete_depth
    insertByPoints = insert_points

    def setFlagsByIterators(self, scheme: Scheme, flags: int, depth: int = LEAF) -> int:
        return self.set_flags_by_image(scheme, flags, depth)

    def searchByIterators(self, scheme: Scheme, depth: int = LEAF) -> np.ndarray:
        return self.search_by_image(scheme, depth)

    def insertByIterators(self, scheme: Scheme, depth: int, flags_for_inserted: int = L.INS,
                          flags_for_hit: int = L.NONE) -> int:
        return self.insert_by_image(scheme, depth, flags_for_inserted, flags_for_hit)

    def transitionMatrixForLeaves(self, grid: GridSpec, map_: MapSpec, use_absolute_values: bool = False,
                                  use_invalid_nr_boxes: bool = False) -> CsrMatrix:
        return self.transition_matrix(Scheme(map_, grid), use_absolute_values, use_invalid_nr_boxes)


# ----------------------------------------------------------------------------- batches
class Batch:
    """Many independent subdivision jobs (same domain, map kind, grid) advanced together."""

    def __init__(self, center, radius, scheme: Scheme, params, depths):
        params = np.asarray(params, dtype=np.float64)
        if params.ndim != 2:
            raise ValueError("params must be n x k")
        n = params.shape[0]
        p6 = np.zeros((n, 6), dtype=np.float64)
        p6[:, : params.shape[1]] = params
        self._params = np.ascontiguousarray(p6)
        self._depths = np.ascontiguousarray(np.asarray(depths, dtype=np.uint8))
        if len(self._depths) != n:
            raise ValueError("one depth per instance")
        d = L.Domain()
        d.dim = len(center)
        for j in range(d.dim):
            d.center[j] = float(center[j])
            d.radius[j] = float(radius[j])
        self.n = n
        self.dim = d.dim
        s = scheme.to_c()
        self._h = C.c_void_p()
        check(lib().b12g_batch_create(C.byref(d), C.byref(s), n, self._params.ctypes.data, self._depths.ctypes.data,
                                      C.byref(self._h)), "batch_create")

    def close(self):
        if self._h:
            lib().b12g_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self) -> None:
        check(lib().b12g_batch_run(self._h), "batch_run")

    def counts(self, i: int) -> np.ndarray:
        c = np.zeros(int(self._depths[i]), dtype=np.uint32)
        check(lib().b12g_batch_counts(self._h, i, c.ctypes.data), "batch_counts")
        return c

    def leaves(self, i: int):
        n, d = C.c_uint32(), C.c_uint8()
        check(lib().b12g_batch_leaves(self._h, i, None, None, C.byref(n), C.byref(d)), "batch_leaves")
        codes = np.zeros(n.value, dtype=np.uint64)
        flags = np.zeros(n.value, dtype=np.uint8)
        check(lib().b12g_batch_leaves(self._h, i, codes.ctypes.data, flags.ctypes.data, C.byref(n), C.byref(d)),
              "batch_leaves")
        return codes, np.full(n.value, d.value, dtype=np.uint8), flags

    def transition_matrices(self, absolute: bool = False, invalid_column: bool = False) -> None:
        check(lib().b12g_batch_transition_matrices(self._h, int(absolute), int(invalid_column)),
              "batch_transition_matrices")

    def csr(self, i: int):
        rows, nnz = C.c_uint32(), C.c_uint64()
        check(lib().b12g_batch_csr(self._h, i, None, None, None, C.byref(rows), C.byref(nnz)), "batch_csr")
        rowptr = np.zeros(rows.value + 1, dtype=np.uint32)
        cols = np.zeros(max(nnz.value, 1), dtype=np.uint32)
        vals = np.zeros(max(nnz.value, 1), dtype=np.float64)
        check(lib().b12g_batch_csr(self._h, i, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data,
                                   C.byref(rows), C.byref(nnz)), "batch_csr")
        return rowptr, cols[: nnz.value], vals[: nnz.value]

    def info(self) -> dict:
        bi, fb, nnz = C.c_uint64(), C.c_uint64(), C.c_uint64()
        th, ppt, ch = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib().b12g_batch_info(self._h, C.byref(bi), C.byref(fb), C.byref(nnz), C.byref(th), C.byref(ppt),
                                    C.byref(ch)), "batch_info")
        return dict(box_images=bi.value, final_boxes=fb.value, nnz=nnz.value, threads=th.value,
                    points_per_thread=ppt.value, chunk=ch.value)

    def stream_handle(self) -> int:
        p = C.c_void_p()
        check(lib().b12g_batch_stream(self._h, C.byref(p)), "batch_stream")
        return p.value or 0
