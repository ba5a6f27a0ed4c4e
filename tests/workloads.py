"""Workload specs shared by the tests: golden-fixture spec -> oracle spec / library scheme."""
from __future__ import annotations

import hashlib

import numpy as np

from oracle import oracle as O


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def oracle_spec(spec: dict) -> dict:
    m = spec["map"]
    if m == "henon":
        return O.henon_spec(spec.get("a", 1.4), spec.get("b", 0.3), spec.get("grid", 4))
    if m == "lorenz":
        return O.lorenz_spec(spec.get("rho", 28.0), spec.get("fma", False), spec.get("grid", 5))
    if m == "forced_duffing":
        return O.forced_duffing_spec(spec.get("grid", 4))
    if m == "coupled_duffing":
        return O.coupled_duffing_spec(spec.get("points", 64), spec.get("seed", 0))
    raise ValueError(m)


def domain(spec: dict):
    o = oracle_spec(spec)
    return o["center"], o["radius"]


def scheme(spec: dict, depth: int = 255, flags_to_check: int = 0):
    import b12_b200 as B
    m = spec["map"]
    if m == "henon":
        mp = B.henon(spec.get("a", 1.4), spec.get("b", 0.3))
        g = B.inner_grid(spec.get("grid", 4))
    elif m == "lorenz":
        mp = B.lorenz(rho=spec.get("rho", 28.0), fma=spec.get("fma", False))
        g = B.inner_grid(spec.get("grid", 5))
    elif m == "forced_duffing":
        mp = B.forced_duffing()
        g = B.inner_grid(spec.get("grid", 4))
    elif m == "coupled_duffing":
        mp = B.coupled_duffing()
        g = B.philox_grid(spec.get("points", 64), spec.get("seed", 0))
    else:
        raise ValueError(m)
    return B.Scheme(mp, g, depth, flags_to_check)


def csr_digests(rowptr, cols, vals) -> dict:
    return dict(n_rows=len(rowptr) - 1, nnz=int(len(vals)), rowptr_sha256=sha(rowptr.astype(np.uint32)),
                cols_sha256=sha(cols.astype(np.uint32)), vals_sha256=sha(vals.astype(np.float64)))
