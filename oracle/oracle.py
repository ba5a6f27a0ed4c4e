"""ORACLE - test infrastructure only.

ctypes binding of ``oracle/liboracle.so``, the plain-C restatement of the
reference's box-image path (``oracle/b12_oracle.c``).  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this
module; the library in ``b12_b200`` never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

MAP_HENON, MAP_LORENZ, MAP_COUPLED_DUFFING, MAP_FORCED_DUFFING = 1, 2, 3, 4
GRID_INNER, GRID_FULL, GRID_PHILOX = 1, 2, 3
INVALID = 0xFFFFFFFF


class OrcMap(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("fma", C.c_uint32), ("steps", C.c_uint32), ("pad", C.c_uint32),
                ("h", C.c_double), ("p", C.c_double * 6), ("table", C.POINTER(C.c_double))]


class OrcGrid(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("n", C.c_uint32), ("points", C.c_uint64), ("seed", C.c_uint64),
                ("eps", C.c_double)]


class OrcDomain(C.Structure):
    _fields_ = [("dim", C.c_uint32), ("center", C.c_double * 4), ("radius", C.c_double * 4)]


class OrcTree(C.Structure):
    _fields_ = [("dom", OrcDomain), ("n", C.c_uint64), ("cap", C.c_uint64),
                ("code", C.POINTER(C.c_uint64)), ("depth", C.POINTER(C.c_uint8)),
                ("flags", C.POINTER(C.c_uint8))]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        u8, u32, u64, dbl = C.c_uint8, C.c_uint32, C.c_uint64, C.c_double
        sig = {
            "orc_grid_points_per_box": (u64, [P(OrcGrid), u32]),
            "orc_grid_point": (None, [P(OrcGrid), u32, u64, P(dbl)]),
            "orc_map_apply": (None, [P(OrcMap), P(dbl), P(dbl)]),
            "orc_box_coordinates": (None, [P(OrcDomain), u64, u32, P(dbl), P(dbl)]),
            "orc_point_code64": (C.c_int, [P(OrcDomain), P(dbl), P(u64)]),
            "orc_forced_duffing_table": (None, [u32, dbl, P(dbl)]),
            "orc_philox4x32_10": (None, [P(u32), u32, u32]),
            "orc_tree_init": (None, [P(OrcTree), P(OrcDomain)]),
            "orc_tree_free": (None, [P(OrcTree)]),
            "orc_tree_load": (None, [P(OrcTree), P(u64), P(u8), P(u8), u64]),
            "orc_set_flags": (u32, [P(OrcTree), u8]),
            "orc_set_flags_mask": (u32, [P(OrcTree), P(u8), u8]),
            "orc_strong_components": (None, [u32, P(u32), P(u32), P(u32)]),
            "orc_unset_flags": (u32, [P(OrcTree), u8]),
            "orc_change_flags": (u32, [P(OrcTree), u8, u8]),
            "orc_subdivide": (u32, [P(OrcTree), u8]),
            "orc_remove": (u32, [P(OrcTree), u8]),
            "orc_search": (u32, [P(OrcTree), u64, C.c_int]),
            "orc_search_by_image": (None, [P(OrcTree), P(OrcMap), P(OrcGrid), P(u32), u64, P(u32)]),
            "orc_set_flags_by_image": (u32, [P(OrcTree), P(OrcMap), P(OrcGrid), u8]),
            "orc_insert_by_image": (u32, [P(OrcTree), P(OrcMap), P(OrcGrid), u8, u8, u8]),
            "orc_insert_points": (u32, [P(OrcTree), P(dbl), u64, u32, u8, u8]),
            "orc_delete_depth0": (None, [P(OrcTree)]),
            "orc_unsubdivide": (u32, [P(OrcTree), u8]),
            "orc_flags_at_depth": (u32, [P(OrcTree), C.c_int, u8, u8, u32]),
            "orc_image_at_depth": (u32, [P(OrcTree), P(OrcMap), P(OrcGrid), u32, u8, P(u32)]),
            "orc_insert_by_image_src": (u32, [P(OrcTree), P(OrcMap), P(OrcGrid), u32, u8, u32, u8, u8, P(C.c_int)]),
            "orc_image_search": (u32, [P(OrcTree), P(OrcMap), P(OrcGrid), u32, u8, u32, u8, P(u32), P(u64)]),
            "orc_insert_points_general": (u32, [P(OrcTree), P(dbl), u64, u32, u8, u8, P(C.c_int)]),
            "orc_insert_by_image_general": (u32, [P(OrcTree), P(OrcMap), P(OrcGrid), u8, u32, u8, u8,
                                                  P(C.c_int)]),
            "orc_transition_matrix": (u64, [P(OrcTree), P(OrcMap), P(OrcGrid), C.c_int, C.c_int,
                                            P(u32), P(u32), P(dbl), P(u32)]),
            "orc_invariant_measure": (None, [u32, P(u32), P(u32), P(dbl), u32, P(dbl)]),
            "orc_invariant_measure_tol": (None, [u32, P(u32), P(u32), P(dbl), dbl, u32, u32, P(dbl), P(u32),
                                                 P(dbl)]),
            "orc_image_point_boxes": (None, [P(OrcTree), P(OrcMap), P(OrcGrid), P(u64), P(u8)]),
            "orc_search_point_boxes": (None, [P(OrcTree), P(u64), P(u8), u64, P(u32)]),
            "orc_set_flags_by_point_boxes": (u32, [P(OrcTree), P(u64), P(u8), u64, u8]),
            "orc_transition_rows": (u64, [P(u32), u64, u64, u32, C.c_int, C.c_int, P(u32), P(u32), P(dbl), P(u32)]),
            "orc_subdivision": (u64, [P(OrcTree), P(OrcMap), P(OrcGrid), u32, P(u32)]),
            "orc_num_threads": (C.c_int, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


# ------------------------------------------------------------------ workload specs
def henon_spec(a=1.4, b=0.3, n=4):
    return dict(dim=2, center=[0.0, 0.0], radius=[1.5, 0.45],
                map=dict(kind=MAP_HENON, steps=1, p=[a, b]), grid=dict(kind=GRID_INNER, n=n))


def lorenz_spec(rho=28.0, fma=False, n=5):
    return dict(dim=3, center=[0.0, 0.0, 27.0], radius=[30.0, 30.0, 40.0],
                map=dict(kind=MAP_LORENZ, steps=20, h=0.01, fma=int(fma), p=[10.0, rho, 8.0 / 3.0]),
                grid=dict(kind=GRID_INNER, n=n))


def coupled_duffing_spec(points=64, seed=0):
    return dict(dim=4, center=[0.0] * 4, radius=[2.0] * 4,
                map=dict(kind=MAP_COUPLED_DUFFING, steps=10, h=0.05),
                grid=dict(kind=GRID_PHILOX, points=points, seed=seed))


FORCED_PERIOD = 2.0 * 3.14159265358979323846


def forced_duffing_spec(n=4, steps=200):
    return dict(dim=2, center=[0.0, 0.0], radius=[2.0, 2.0],
                map=dict(kind=MAP_FORCED_DUFFING, steps=steps, h=FORCED_PERIOD / steps,
                         p=[0.25, -1.0, 1.0, 0.3]),
                grid=dict(kind=GRID_INNER, n=n))


class Oracle:
    """One oracle tree plus its map and grid (mirrors one reference ImplicitBoxTree)."""

    def __init__(self, spec: dict):
        self.L = lib()
        self.spec = spec
        d = OrcDomain()
        d.dim = spec["dim"]
        for j in range(spec["dim"]):
            d.center[j] = spec["center"][j]
            d.radius[j] = spec["radius"][j]
        self.dom = d
        m = OrcMap()
        ms = spec["map"]
        m.kind = ms["kind"]
        m.fma = ms.get("fma", 0)
        m.steps = ms.get("steps", 1)
        m.h = ms.get("h", 0.0)
        for i, v in enumerate(ms.get("p", [])):
            m.p[i] = v
        self._table = None
        if m.kind == MAP_FORCED_DUFFING:
            self._table = np.zeros(2 * m.steps + 1)
            self.L.orc_forced_duffing_table(m.steps, FORCED_PERIOD, _ptr(self._table, C.c_double))
            m.table = _ptr(self._table, C.c_double)
        self.map = m
        g = OrcGrid()
        gs = spec["grid"]
        g.kind = gs["kind"]
        g.n = gs.get("n", 1)
        g.points = gs.get("points", 1)
        g.seed = gs.get("seed", 0)
        g.eps = gs.get("eps", 0.0)
        self.grid = g
        self.tree = OrcTree()
        self.L.orc_tree_init(C.byref(self.tree), C.byref(self.dom))

    def __del__(self):
        try:
            self.L.orc_tree_free(C.byref(self.tree))
        except Exception:
            pass

    # -- state
    @property
    def n(self) -> int:
        return int(self.tree.n)

    def leaves(self):
        n = self.n
        codes = np.ctypeslib.as_array(self.tree.code, shape=(n,)).copy()
        depth = np.ctypeslib.as_array(self.tree.depth, shape=(n,)).copy()
        flags = np.ctypeslib.as_array(self.tree.flags, shape=(n,)).copy()
        return codes, depth, flags

    def load(self, codes, depth, flags):
        codes = np.ascontiguousarray(codes, dtype=np.uint64)
        depth = np.ascontiguousarray(depth, dtype=np.uint8)
        flags = np.ascontiguousarray(flags, dtype=np.uint8)
        self.L.orc_tree_load(C.byref(self.tree), _ptr(codes, C.c_uint64), _ptr(depth, C.c_uint8),
                             _ptr(flags, C.c_uint8), len(codes))

    # -- reference operations
    def set_flags(self, f): return self.L.orc_set_flags(C.byref(self.tree), f)
    def unset_flags(self, f): return self.L.orc_unset_flags(C.byref(self.tree), f)

    def set_flags_mask(self, mask, f):
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        assert len(m) == self.n
        return self.L.orc_set_flags_mask(C.byref(self.tree), _ptr(m, C.c_uint8), f)
    def change_flags(self, u, s): return self.L.orc_change_flags(C.byref(self.tree), u, s)
    def subdivide(self, f=8): return self.L.orc_subdivide(C.byref(self.tree), f)
    def remove(self, f): return self.L.orc_remove(C.byref(self.tree), f)

    def set_flags_by_image(self, f=1):
        return self.L.orc_set_flags_by_image(C.byref(self.tree), C.byref(self.map), C.byref(self.grid), f)

    def insert_by_image(self, check=4, ins=2, hit=0):
        return self.L.orc_insert_by_image(C.byref(self.tree), C.byref(self.map), C.byref(self.grid),
                                          check, ins, hit)

    def insert_points(self, pts, depth, ins=2, hit=0):
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        return self.L.orc_insert_points(C.byref(self.tree), _ptr(pts, C.c_double),
                                        pts.size // self.spec["dim"], depth, ins, hit)

    def delete_depth0(self): self.L.orc_delete_depth0(C.byref(self.tree))

    def unsubdivide(self, f): return self.L.orc_unsubdivide(C.byref(self.tree), f)

    def image_flags_at_depth(self, depth, f):
        """flags on the boxes at an inner depth hit by the images of every leaf"""
        return self.L.orc_image_at_depth(C.byref(self.tree), C.byref(self.map), C.byref(self.grid), depth, f, None)

    def image_search_at_depth(self, depth):
        """each image point's box index at an inner depth (0xFFFFFFFF: none)"""
        out = np.zeros(self.n * self.points_per_box(), dtype=np.uint32)
        self.L.orc_image_at_depth(C.byref(self.tree), C.byref(self.map), C.byref(self.grid), depth, 0,
                                  _ptr(out, C.c_uint32))
        return out

    def image_flags(self, src_depth, check, target, f):
        """flags on what the images of a scheme's sources hit (sources at src_depth with
        all of `check`; target 255 = leaves, else an inner depth); returns the count"""
        return self.L.orc_image_search(C.byref(self.tree), C.byref(self.map), C.byref(self.grid), src_depth, check,
                                       target, f, None, None)

    def image_search(self, src_depth, check, target):
        """each image point's leaf (target 255) or box index at an inner target depth"""
        npts = C.c_uint64()
        self.L.orc_image_search(C.byref(self.tree), C.byref(self.map), C.byref(self.grid), src_depth, check, target, 0,
                                None, C.byref(npts))
        out = np.zeros(max(npts.value, 1), dtype=np.uint32)
        self.L.orc_image_search(C.byref(self.tree), C.byref(self.map), C.byref(self.grid), src_depth, check, target, 0,
                                _ptr(out, C.c_uint32), None)
        return out[:npts.value]

    def flags_at_depth(self, op, u, f, depth):
        """set (0) / unset (1) / change (2, u -> f) flags of the boxes at an inner depth"""
        return self.L.orc_flags_at_depth(C.byref(self.tree), op, u, f, depth)

    def insert_points_general(self, pts, depth, ins=2, hit=0):
        """insertByPoints for any tree and depth (255: leaf depth); None if not restated"""
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        uns = C.c_int()
        r = self.L.orc_insert_points_general(C.byref(self.tree), _ptr(pts, C.c_double), pts.size // self.spec["dim"],
                                             depth, ins, hit, C.byref(uns))
        return None if uns.value else r

    def insert_by_image_src(self, src_depth, check, depth, ins=2, hit=0):
        uns = C.c_int()
        return self.L.orc_insert_by_image_src(C.byref(self.tree), C.byref(self.map), C.byref(self.grid), src_depth,
                                              check, depth, ins, hit, C.byref(uns))

    def insert_by_image_general(self, check, depth, ins=2, hit=0):
        uns = C.c_int()
        r = self.L.orc_insert_by_image_general(C.byref(self.tree), C.byref(self.map), C.byref(self.grid), check,
                                               depth, ins, hit, C.byref(uns))
        return None if uns.value else r

    def points_per_box(self) -> int:
        return int(self.L.orc_grid_points_per_box(C.byref(self.grid), self.spec["dim"]))

    def search_by_image(self, src=None):
        if src is None:
            src = np.arange(self.n, dtype=np.uint32)
        src = np.ascontiguousarray(src, dtype=np.uint32)
        out = np.zeros(len(src) * self.points_per_box(), dtype=np.uint32)
        self.L.orc_search_by_image(C.byref(self.tree), C.byref(self.map), C.byref(self.grid),
                                   _ptr(src, C.c_uint32), len(src), _ptr(out, C.c_uint32))
        return out

    def subdivision(self, steps: int):
        counts = np.zeros(max(steps, 1), dtype=np.uint32)
        bi = self.L.orc_subdivision(C.byref(self.tree), C.byref(self.map), C.byref(self.grid), steps,
                                    _ptr(counts, C.c_uint32))
        return counts[:steps], int(bi)

    def transition_matrix(self, absolute=False, invalid=False):
        t, m, g = C.byref(self.tree), C.byref(self.map), C.byref(self.grid)
        nnz = self.L.orc_transition_matrix(t, m, g, int(absolute), int(invalid), None, None, None, None)
        rowptr = np.zeros(self.n + 1, dtype=np.uint32)
        cols = np.zeros(max(nnz, 1), dtype=np.uint32)
        vals = np.zeros(max(nnz, 1), dtype=np.float64)
        ncols = C.c_uint32()
        self.L.orc_transition_matrix(t, m, g, int(absolute), int(invalid), _ptr(rowptr, C.c_uint32),
                                     _ptr(cols, C.c_uint32), _ptr(vals, C.c_double), C.byref(ncols))
        return rowptr, cols[:nnz], vals[:nnz], int(ncols.value)

    # -- point boxes of a range-partitioned tree
    def image_point_boxes(self):
        """the point boxes (depth-64 codes, validity) of the images of every leaf, leaf-major"""
        total = self.n * self.points_per_box()
        codes = np.zeros(max(total, 1), dtype=np.uint64)
        valid = np.zeros(max(total, 1), dtype=np.uint8)
        self.L.orc_image_point_boxes(C.byref(self.tree), C.byref(self.map), C.byref(self.grid),
                                     _ptr(codes, C.c_uint64), _ptr(valid, C.c_uint8))
        return codes[:total], valid[:total]

    def search_point_boxes(self, codes, valid):
        codes = np.ascontiguousarray(codes, dtype=np.uint64)
        valid = np.ascontiguousarray(valid, dtype=np.uint8)
        out = np.zeros(max(len(codes), 1), dtype=np.uint32)
        self.L.orc_search_point_boxes(C.byref(self.tree), _ptr(codes, C.c_uint64), _ptr(valid, C.c_uint8),
                                      len(codes), _ptr(out, C.c_uint32))
        return out[:len(codes)]

    def set_flags_by_point_boxes(self, codes, valid, flags):
        codes = np.ascontiguousarray(codes, dtype=np.uint64)
        valid = np.ascontiguousarray(valid, dtype=np.uint8)
        return self.L.orc_set_flags_by_point_boxes(C.byref(self.tree), _ptr(codes, C.c_uint64),
                                                   _ptr(valid, C.c_uint8), len(codes), flags)

    @staticmethod
    def transition_rows(targets, P, n_cols, absolute=False, invalid=False):
        """(rowptr, cols, vals, n_cols) of rows of P targets each (ORC_INVALID: lost)"""
        tgt = np.array(targets, dtype=np.uint32).reshape(-1)
        n = len(tgt) // P
        L = lib()
        nnz = L.orc_transition_rows(_ptr(tgt.copy(), C.c_uint32), n, P, n_cols, int(absolute), int(invalid),
                                    None, None, None, None)
        rowptr = np.zeros(n + 1, dtype=np.uint32)
        cols = np.zeros(max(nnz, 1), dtype=np.uint32)
        vals = np.zeros(max(nnz, 1), dtype=np.float64)
        nc = C.c_uint32()
        L.orc_transition_rows(_ptr(tgt, C.c_uint32), n, P, n_cols, int(absolute), int(invalid),
                              _ptr(rowptr, C.c_uint32), _ptr(cols, C.c_uint32), _ptr(vals, C.c_double), C.byref(nc))
        return rowptr, cols[:nnz], vals[:nnz], int(nc.value)

    # -- geometry
    def point_code64(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        c = C.c_uint64()
        ok = self.L.orc_point_code64(C.byref(self.dom), _ptr(p, C.c_double), C.byref(c))
        return int(c.value), bool(ok)

    def map_apply(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        self.L.orc_map_apply(C.byref(self.map), _ptr(x, C.c_double), _ptr(y, C.c_double))
        return y

    def grid_point(self, i):
        r = np.zeros(self.spec["dim"])
        self.L.orc_grid_point(C.byref(self.grid), self.spec["dim"], i, _ptr(r, C.c_double))
        return r


def invariant_measure(rowptr, cols, vals, iters=200):
    n = len(rowptr) - 1
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    v = np.zeros(n)
    lib().orc_invariant_measure(n, _ptr(rowptr, C.c_uint32), _ptr(cols, C.c_uint32), _ptr(vals, C.c_double),
                                iters, _ptr(v, C.c_double))
    return v


def invariant_measure_tol(rowptr, cols, vals, tol, max_iters, check_every=20):
    """The power iteration until the L1 change of one iteration, checked every
    `check_every` iterations, is at most `tol`: (v, iterations run, last change)."""
    n = len(rowptr) - 1
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    v = np.zeros(n)
    k = C.c_uint32()
    ch = C.c_double()
    lib().orc_invariant_measure_tol(n, _ptr(rowptr, C.c_uint32), _ptr(cols, C.c_uint32), _ptr(vals, C.c_double),
                                    float(tol), int(max_iters), int(check_every), _ptr(v, C.c_double), C.byref(k),
                                    C.byref(ch))
    return v, k.value, ch.value


def strong_components(rowptr, cols):
    """Component label (largest vertex of the component) of every row's box."""
    n = len(rowptr) - 1
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    comp = np.zeros(n, dtype=np.uint32)
    lib().orc_strong_components(n, _ptr(rowptr, C.c_uint32), _ptr(cols, C.c_uint32), _ptr(comp, C.c_uint32))
    return comp


def chain_recurrent(spec: dict, steps: int):
    """chainRecurrentSet.m:18-44: subdivide, transition matrix, keep the boxes of strongly
    connected components with more than one box; returns the oracle and per-step counts."""
    o = Oracle(spec)
    o.set_flags(8)
    counts = []
    for _ in range(steps):
        o.subdivide(8)
        rowptr, cols, _, _ = o.transition_matrix()
        comp = strong_components(rowptr, cols)
        sizes = np.bincount(comp, minlength=len(comp))
        o.set_flags_mask(sizes[comp] > 1, 1)
        o.remove(1)
        o.unset_flags(1)
        counts.append(o.n)
    return o, counts


def nim_selection(spec: dict, steps: int, iters: int = 200, tol: float | None = None):
    """subdivisionByNim.m:22-66 with the FP64 power iteration for the eigenvector: keep the
    boxes whose measure is at least 1e-9 / n; returns the oracle and per-step counts.
    With `tol` the iteration runs to that tolerance (checked every 20, at most `iters`)."""
    o = Oracle(spec)
    o.set_flags(8)
    counts = []
    for _ in range(steps):
        o.subdivide(8)
        rowptr, cols, vals, _ = o.transition_matrix()
        if tol is None:
            v = invariant_measure(rowptr, cols, vals, iters)
        else:
            v = invariant_measure_tol(rowptr, cols, vals, tol, iters, 20)[0]
        o.set_flags_mask(v >= 1e-9 / len(v), 1)
        o.remove(1)
        o.unset_flags(1)
        counts.append(o.n)
    return o, counts


def fixed_boxes(spec: dict, steps: int):
    """fixedBoxes.m:10-22: keep the boxes one of whose own test points lands in them
    again; returns the oracle and per-step counts."""
    o = Oracle(spec)
    o.delete_depth0()
    o.set_flags(8)
    counts = []
    P = o.points_per_box()
    for _ in range(steps):
        o.subdivide(8)
        s = o.search_by_image().reshape(-1, P)
        o.set_flags_mask((s == np.arange(len(s), dtype=s.dtype)[:, None]).any(axis=1), 1)
        o.remove(1)
        o.unset_flags(1)
        counts.append(o.n)
    return o, counts


def count_at_depth(o: "Oracle", depth: int) -> int:
    """ImplicitBoxTree::count(depth) (ImplicitBoxTree.hpp:1061-1095) for the trees the
    continuation makes: 1 at depth 0, every leaf when all leaves have that depth, 0 for a
    depth below every leaf (the remaining branch, boxes of an inner depth, is not needed)."""
    if depth == 0:
        return 1
    d = o.leaves()[1]
    if len(d) and (d == depth).all():
        return o.n
    if len(d) == 0 or depth > int(d.max()):
        return 0
    raise NotImplementedError("count at an inner depth of a tree of several depths")


def continuation(spec: dict, depth: int, x0, max_sweeps: int = 10_000):
    """continuation.m:13-44 at one depth (its counts are count(d)); returns the oracle and
    per-sweep counts."""
    o = Oracle(spec)
    o.delete_depth0()
    o.insert_points(np.asarray(x0, dtype=np.float64), depth, 2)
    counts = []
    nb0, nb1 = 0, count_at_depth(o, depth)
    while nb1 > nb0 and len(counts) < max_sweeps:
        o.change_flags(2, 4)          # INS -> EXPD
        o.insert_by_image(4, 2, 0)    # insert images of EXPD boxes with INS
        o.unset_flags(4)              # drop EXPD
        nb0, nb1 = nb1, count_at_depth(o, depth)
        counts.append(nb1)
    return o, counts
