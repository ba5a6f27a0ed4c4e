"""Test helper: a rank's run of leaves held by the oracle (CPU), with the methods of
b12_b200.partition.DeviceRun, so that the partitioned steps can be checked against one
oracle tree on the CPU (emulated ranks, or gloo ranks)."""
from __future__ import annotations

import numpy as np
import torch

from oracle import oracle as O

SD, HIT = 0x08, 0x01


def _u64(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().astype(np.int64).view(np.uint64)


class OracleRun:
    def __init__(self, spec: dict, codes=None, depth=None, flags=None):
        self.o = O.Oracle(spec)
        self.device = "cpu"
        self.empty = codes is not None and len(codes) == 0
        if codes is not None and len(codes):
            self.o.load(codes, depth, flags)

    @property
    def n(self) -> int:
        return 0 if self.empty else self.o.n

    def start(self) -> int:
        codes, depth, _ = self.o.leaves()
        d = int(depth[0])
        return 0 if d == 0 else (int(codes[0]) << (64 - d)) & ((1 << 64) - 1)

    def set_flags(self, flags):
        if not self.empty:
            self.o.set_flags(flags)

    def unset_flags(self, flags):
        if not self.empty:
            self.o.unset_flags(flags)

    def subdivide(self, flags):
        if not self.empty:
            self.o.subdivide(flags)

    def remove(self, flags):
        if self.empty:
            return
        before = self.o.n
        if self.o.remove(flags) == before:
            self.empty = True

    def points_per_box(self, scheme) -> int:
        return self.o.points_per_box()

    def image_point_boxes(self, scheme):
        if self.empty:
            return torch.empty(0, dtype=torch.int64), torch.empty(0, dtype=torch.uint8)
        c, v = self.o.image_point_boxes()
        return torch.from_numpy(c.view(np.int64).copy()), torch.from_numpy(v.copy())

    def set_flags_by_point_boxes(self, codes, valid, flags) -> int:
        if self.empty:
            return 0
        return self.o.set_flags_by_point_boxes(_u64(codes), valid.cpu().numpy(), flags)

    def search_point_boxes(self, codes, valid):
        if self.empty:
            return torch.full((codes.numel(),), -1, dtype=torch.int64)
        idx = self.o.search_point_boxes(_u64(codes), valid.cpu().numpy()).astype(np.int64)
        idx[idx == 0xFFFFFFFF] = -1
        return torch.from_numpy(idx)

    def leaves(self):
        if self.empty:
            return torch.empty(0, dtype=torch.int64), torch.empty(0, dtype=torch.uint8), \
                torch.empty(0, dtype=torch.uint8)
        c, d, f = self.o.leaves()
        return torch.from_numpy(c.view(np.int64).copy()), torch.from_numpy(d.copy()), torch.from_numpy(f.copy())

    def load(self, codes, depth, flags):
        if codes.numel() == 0:
            self.empty = True
            return
        self.o.load(_u64(codes), depth.numpy(), flags.numpy())
        self.empty = False

    def transition_rows(self, targets, points_per_row, n_columns, absolute, invalid_column):
        if self.empty:
            return None
        t = targets.cpu().numpy().astype(np.int64)
        t = np.where(t < 0, 0xFFFFFFFF, t).astype(np.uint32)
        return O.Oracle.transition_rows(t, points_per_row, n_columns, absolute, invalid_column)

    def host_leaves(self):
        if self.empty:
            return np.zeros(0, np.uint64), np.zeros(0, np.uint8), np.zeros(0, np.uint8)
        return self.o.leaves()


def concat_leaves(runs):
    parts = [r.host_leaves() for r in runs]
    return tuple(np.concatenate([p[k] for p in parts]) for k in range(3))


def concat_rows(blocks):
    """(rowptr, cols, vals, n_cols) of the whole matrix from the ranks' RowBlocks
    (rows given as (rowptr, cols, vals, ...) host arrays)."""
    rowptr, cols, vals, base = [np.zeros(1, np.uint64)], [], [], 0
    for b in blocks:
        if b.rows is None:
            continue
        rp, c, v = b.rows[0], b.rows[1], b.rows[2]
        rowptr.append(rp[1:].astype(np.uint64) + base)
        base += int(rp[-1])
        cols.append(c)
        vals.append(v)
    n_cols = blocks[0].n_cols
    return (np.concatenate(rowptr).astype(np.uint32), np.concatenate(cols) if cols else np.zeros(0, np.uint32),
            np.concatenate(vals) if vals else np.zeros(0), n_cols)
