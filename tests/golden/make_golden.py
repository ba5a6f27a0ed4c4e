"""Generate the golden fixtures from the reference itself.

Runs the reference's own ImplicitBoxTree (compiled from its headers with the Thrust
OMP backend into oracle/_ref by oracle/ref/Makefile) on the workloads below and
stores, per subdivision step, the leaf count and SHA-256 digests of the leaf codes and
flags, plus the transition matrix as CSR digests; small cases are also stored in full
(<name>.npz).  The GPU tests compare the CUDA library against these files, which is
why they are committed: the reference is not available where the GPU tests run.

    python tests/golden/make_golden.py [name ...]
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(REPO, "oracle", "_ref")

# name -> (binary, args, spec for the library/oracle, full-array limit)
WORKLOADS = {
    "henon_d20": ("ref_henon", ["--steps", "20", "--tm", "1"], dict(map="henon", a=1.4, b=0.3, grid=4, steps=20)),
    "henon_d12_abs": ("ref_henon", ["--steps", "12", "--tm", "2"],
                      dict(map="henon", a=1.4, b=0.3, grid=4, steps=12, absolute=True)),
    "lorenz_rho15_d4_invalid_column_unused": ("ref_lorenz", ["--steps", "4", "--tm", "3", "--rho", "15"],
                                               dict(map="lorenz", rho=15.0, grid=5, steps=4, invalid=True)),
    "henon_d12_lost": ("ref_henon", ["--steps", "12", "--tm", "3", "--grid", "6"],
                       dict(map="henon", a=1.4, b=0.3, grid=6, steps=12, invalid=True)),
    "henon_a1.0_d16": ("ref_henon", ["--steps", "16", "--tm", "1", "--a", "1.0"],
                       dict(map="henon", a=1.0, b=0.3, grid=4, steps=16)),
    "lorenz_d15": ("ref_lorenz", ["--steps", "15", "--tm", "1"], dict(map="lorenz", rho=28.0, grid=5, steps=15)),
    "lorenz_d27": ("ref_lorenz", ["--steps", "27", "--tm", "1", "--buf", "1073741824"],
                   dict(map="lorenz", rho=28.0, grid=5, steps=27)),
    "lorenz_fma_d27": ("ref_lorenz", ["--steps", "27", "--tm", "1", "--fma", "1", "--buf", "1073741824"],
                       dict(map="lorenz", rho=28.0, grid=5, steps=27, fma=True)),
    "lorenz_rho15_d18": ("ref_lorenz", ["--steps", "18", "--tm", "1", "--rho", "15"],
                         dict(map="lorenz", rho=15.0, grid=5, steps=18)),
    "lorenz_rho35_d18": ("ref_lorenz", ["--steps", "18", "--tm", "1", "--rho", "35"],
                         dict(map="lorenz", rho=35.0, grid=5, steps=18)),
    "forced_duffing_d16": ("ref_forced", ["--steps", "16", "--tm", "1"],
                           dict(map="forced_duffing", grid=4, steps=16)),
    # files written by the reference's ImplicitBoxTree::save and CooMatrix::save (JSON)
    "henon_d8_files": ("ref_henon", ["--steps", "8", "--tm", "1", "--buf", "4294967296"],
                       dict(map="henon", a=1.4, b=0.3, grid=4, steps=8, save=True)),
    "henon_d10_lost_files": ("ref_henon", ["--steps", "10", "--tm", "3", "--buf", "4294967296"],
                             dict(map="henon", a=1.4, b=0.3, grid=4, steps=10, invalid=True, save=True)),
    "lorenz_d9_files": ("ref_lorenz", ["--steps", "9", "--tm", "1", "--buf", "4294967296"],
                        dict(map="lorenz", rho=28.0, grid=5, steps=9, save=True)),
    # selective refinement after uniform steps: trees whose leaves have different depths
    "henon_d14_mixed8": ("ref_henon", ["--steps", "14", "--mixed", "8", "--tm", "1"],
                         dict(map="henon", a=1.4, b=0.3, grid=4, steps=14, mixed=8)),
    "lorenz_d15_mixed6_lost": ("ref_lorenz", ["--steps", "15", "--mixed", "6", "--tm", "3"],
                               dict(map="lorenz", rho=28.0, grid=5, steps=15, mixed=6, invalid=True)),
    "forced_duffing_d12_mixed5": ("ref_forced", ["--steps", "12", "--mixed", "5", "--tm", "2"],
                                  dict(map="forced_duffing", grid=4, steps=12, mixed=5, absolute=True)),
    "henon_d8_mixed4_files": ("ref_henon", ["--steps", "8", "--mixed", "4", "--tm", "1", "--buf", "4294967296"],
                              dict(map="henon", a=1.4, b=0.3, grid=4, steps=8, mixed=4, save=True)),
    # then unsubdivide twice, insert points at the leaf depth, deeper and at an inner
    # depth, insert the images of the inserted leaves at the leaf depth, select once
    "henon_d12_mixed6_edits": ("ref_henon", ["--steps", "12", "--mixed", "6", "--edits", "1", "--tm", "1"],
                               dict(map="henon", a=1.4, b=0.3, grid=4, steps=12, mixed=6, edits=True)),
    "lorenz_d12_mixed4_edits": ("ref_lorenz", ["--steps", "12", "--mixed", "4", "--edits", "1", "--tm", "3"],
                                dict(map="lorenz", rho=28.0, grid=5, steps=12, mixed=4, edits=True, invalid=True)),
    "forced_duffing_d10_mixed3_edits": ("ref_forced", ["--steps", "10", "--mixed", "3", "--edits", "1", "--tm", "1"],
                                        dict(map="forced_duffing", grid=4, steps=10, mixed=3, edits=True)),
    "coupled_duffing_cont_d8": ("ref_duffing", ["--steps", "8"], dict(map="coupled_duffing", points=64, seed=0,
                                                                          depth=8)),
    "coupled_duffing_cont_d12": ("ref_duffing", ["--steps", "12"], dict(map="coupled_duffing", points=64, seed=0,
                                                                            depth=12)),
    # the configured continuation: depth 24, about 10^7 boxes (digests only)
    "coupled_duffing_cont_d24": ("ref_duffing", ["--steps", "24", "--buf", "1073741824"],
                                 dict(map="coupled_duffing", points=64, seed=0, depth=24)),
}

# members of the 512-instance Lorenz parameter scan (SplitMix64 seed 0, explicit-FMA map),
# run one at a time by the reference: two of depth 27, one of depth 24 and one of depth 21
for _i, _rho, _d in ((1, "15.528675431851955", 27), (14, "27.729680145646142", 27),
                     (10, "32.109794817225435", 24), (2, "17.12693383134425", 21)):
    WORKLOADS[f"lorenz_scan0_i{_i}_d{_d}_fma"] = (
        "ref_lorenz", ["--steps", str(_d), "--tm", "1", "--fma", "1", "--rho", _rho, "--buf", "1073741824"],
        dict(map="lorenz", rho=float(_rho), grid=5, steps=_d, fma=True, scan_seed=0, scan_index=_i))

FULL_LIMIT = 20000  # store leaf arrays of steps with at most this many leaves


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def read_leaves(path):
    with open(path, "rb") as f:
        n = int(np.frombuffer(f.read(8), dtype="<u8")[0])
        codes = np.frombuffer(f.read(8 * n), dtype="<u8").copy()
        depth = np.frombuffer(f.read(n), dtype=np.uint8).copy()
        flags = np.frombuffer(f.read(n), dtype=np.uint8).copy()
    return codes, depth, flags


def read_points(path):
    with open(path, "rb") as f:
        n = int(np.frombuffer(f.read(8), dtype="<u8")[0])
        dim = int(np.frombuffer(f.read(4), dtype="<u4")[0])
        return np.frombuffer(f.read(8 * n * dim), dtype="<f8").reshape(n, dim).copy()


def read_coo(path):
    with open(path, "rb") as f:
        nnz = int(np.frombuffer(f.read(8), dtype="<u8")[0])
        nr, nc = np.frombuffer(f.read(8), dtype="<u4")
        rows = np.frombuffer(f.read(4 * nnz), dtype="<u4").copy()
        cols = np.frombuffer(f.read(4 * nnz), dtype="<u4").copy()
        vals = np.frombuffer(f.read(8 * nnz), dtype="<f8").copy()
    return int(nr), int(nc), rows, cols, vals


def coo_to_csr(nr, rows):
    counts = np.bincount(rows, minlength=nr).astype(np.uint64)
    rowptr = np.zeros(nr + 1, dtype=np.uint32)
    rowptr[1:] = np.cumsum(counts).astype(np.uint32)
    return rowptr


def generate(name: str) -> None:
    binary, args, spec = WORKLOADS[name]
    exe = os.path.join(REF, binary)
    if not os.path.exists(exe):
        raise SystemExit(f"{exe} missing: build it with `make -C oracle/ref`")
    with tempfile.TemporaryDirectory() as tmp:
        cmd = [exe, "--out", tmp] + args
        if "--buf" not in args:
            cmd += ["--buf", str(64 << 20)]
        if spec.get("save"):
            cmd += ["--save", os.path.join(tmp, "saved")]
        res = subprocess.run(cmd, check=True, capture_output=True, text=True)
        timing = json.loads(res.stdout.strip().splitlines()[-1])
        out = dict(workload=name, spec=spec, reference_cmd=" ".join([binary] + args), timing=timing, steps=[])
        arrays = {}
        is_cont = binary == "ref_duffing"
        prefix = "cont_" if is_cont else "leaves_"
        files = sorted(f for f in os.listdir(tmp) if f.startswith(prefix))
        # selective refinement (--mixed K): mixed_00 is the flagged start, mixed_KK step KK
        for fn in sorted(f for f in os.listdir(tmp) if f.startswith("mixed_")):
            k = int(fn[len("mixed_"):-4])
            codes, depth, flags = read_leaves(os.path.join(tmp, fn))
            out.setdefault("mixed", []).append(dict(step=k, n=int(len(codes)), max_depth=int(depth.max()),
                                                    min_depth=int(depth.min()), codes_sha256=sha(codes),
                                                    depth_sha256=sha(depth), flags_sha256=sha(flags)))
            if k == 0 or len(codes) <= FULL_LIMIT:
                arrays[f"mixed_codes_{k:02d}"] = codes
                arrays[f"mixed_depth_{k:02d}"] = depth
                arrays[f"mixed_flags_{k:02d}"] = flags
        # edits (--edits 1): unsubdivide and inserts on the mixed tree, and the points used
        for fn in sorted(f for f in os.listdir(tmp) if f.startswith("edit_") or f == "root_insert.bin"):
            key = "root" if fn == "root_insert.bin" else f"{int(fn[len('edit_'):-4]):02d}"
            codes, depth, flags = read_leaves(os.path.join(tmp, fn))
            out.setdefault("edits", []).append(dict(step=key, n=int(len(codes)), codes_sha256=sha(codes),
                                                    depth_sha256=sha(depth), flags_sha256=sha(flags)))
            arrays[f"edit_codes_{key}"] = codes
            arrays[f"edit_depth_{key}"] = depth
            arrays[f"edit_flags_{key}"] = flags
        for fn in sorted(f for f in os.listdir(tmp) if f.startswith("points_")):
            arrays[fn[:-4]] = read_points(os.path.join(tmp, fn))
        # box indices of a search at an inner depth (u64 n, then u32 indices)
        for fn in sorted(f for f in os.listdir(tmp) if f.startswith("search_")):
            with open(os.path.join(tmp, fn), "rb") as f:
                ns = int(np.frombuffer(f.read(8), dtype="<u8")[0])
                idx = np.frombuffer(f.read(4 * ns), dtype="<u4").copy()
            out.setdefault("searches", {})[fn[:-4]] = dict(n=ns, sha256=sha(idx))
            arrays[fn[:-4]] = idx
        for fn in files:
            k = int(fn[len(prefix):-4])
            codes, depth, flags = read_leaves(os.path.join(tmp, fn))
            out["steps"].append(dict(step=k, n=int(len(codes)), depth=int(depth[0]) if len(depth) else 0,
                                     uniform_depth=bool((depth == depth[0]).all()) if len(depth) else True,
                                     codes_sha256=sha(codes), flags_sha256=sha(flags)))
            if len(codes) <= FULL_LIMIT:
                arrays[f"codes_{k:02d}"] = codes
                arrays[f"flags_{k:02d}"] = flags
        tm_path = os.path.join(tmp, "tm.bin")
        if os.path.exists(tm_path):
            nr, nc, rows, cols, vals = read_coo(tm_path)
            rowptr = coo_to_csr(nr, rows)
            out["tm"] = dict(n_rows=nr, n_cols=nc, nnz=int(len(vals)), rowptr_sha256=sha(rowptr),
                             cols_sha256=sha(cols), vals_sha256=sha(vals))
            if len(vals) <= 60000:
                arrays["tm_rowptr"] = rowptr
                arrays["tm_cols"] = cols
                arrays["tm_vals"] = vals
        if spec.get("save"):
            # the reference's own JSON files, byte for byte
            os.makedirs(os.path.join(HERE, "files"), exist_ok=True)
            for part in ("tree", "tm"):
                src = os.path.join(tmp, f"saved_{part}.json")
                with open(src, "rb") as fi, open(os.path.join(HERE, "files", f"{name}_{part}.json"), "wb") as fo:
                    fo.write(fi.read())
    with open(os.path.join(HERE, f"{name}.json"), "w") as f:
        json.dump(out, f, indent=1)
    if arrays:
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
    print(name, "steps", len(out["steps"]), "tm", out.get("tm", {}).get("nnz"), flush=True)


if __name__ == "__main__":
    for name in sys.argv[1:] or list(WORKLOADS):
        generate(name)
