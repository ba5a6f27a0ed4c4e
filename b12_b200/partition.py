"""One box tree range-partitioned over the ranks of a process group.

Every rank holds a contiguous run of the leaves in the reference's order
(isStrictlyPreceding, Box.hpp:124-135): all of rank r's leaves precede rank r+1's.  A
non-empty run owns the codes from the start of its first leaf up to the start of the
next non-empty run, so every depth-64 point box has one owner, and the leaf that holds
it, if any, lies in the owner's run: the reference's search (ImplicitBoxTree.hpp:
2394-2432) looks only at the leaves on either side of the point's lower bound, and the
leaf that contains a point starts at or below it and ends above it.  A point box that
left the domain goes to the last non-empty run, whose last leaf is the tree's last leaf
(the only leaf such a box can be found in).

One step of the subdivision loop (subdivision.m:18-45: subdivide, setFlagsByImage(HIT),
remove(HIT), unsetFlags(HIT)) therefore needs one exchange: every rank images its own
leaves, sends each point box to its owner (an all-to-all), and the owners flag the
leaves hit.  Then the runs' sizes are gathered; when they drift apart, leaves move to
even the runs out, keeping the order.  The transition matrix adds the way back: the
owners return the global column of each point box and every rank assembles the rows of
its own leaves.  When no leaf is left anywhere the surrounding box comes back on rank 0,
as insertSurroundingBoxIfEmpty does for one tree.

The ranks' work is written as generators that yield their collective requests, so the
same code runs over a torch.distributed group (NCCL between GPUs, gloo on CPU), with
`drive`, or as several ranks emulated in one process, with `drive_lockstep`.  A request
is ("allgather", 1-D int64 tensor), answered with a (world, k) tensor, or ("alltoall",
list of world 1-D tensors of one dtype), answered with the list of what every rank sent
this one.  Every rank yields the same requests in the same order.

A run is any object with the methods of `DeviceRun` (one `ImplicitBoxTree` on a GPU);
an empty run is one that holds no leaves.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib as L

_SIGN = -(1 << 63)   # xor with the sign bit: unsigned order of int64 bit patterns


def _ordered(u: int) -> int:
    """The int64 whose signed order is the unsigned order of the 64-bit value u."""
    v = (u & ((1 << 64) - 1)) ^ (1 << 63)
    return v - (1 << 64) if v >= (1 << 63) else v


def box_start(code: int, depth: int) -> int:
    """The first depth-64 code inside the box (code, depth)."""
    return 0 if depth == 0 else (int(code) << (64 - depth)) & ((1 << 64) - 1)


# ----------------------------------------------------------------------------- a run on a GPU
class DeviceRun:
    """A rank's run of leaves: an ImplicitBoxTree on this rank's GPU, or nothing."""

    def __init__(self, tree, device):
        self.tree = tree
        self.device = device
        self.empty = False

    @property
    def n(self) -> int:
        return 0 if self.empty else self.tree.count()

    def start(self) -> int:
        c, d, _ = self.tree.leaf_at(0)
        return box_start(c, d)

    def route_point_boxes(self, codes, valid, starts, ranks, world: int, want_slot: bool = True):
        """The point boxes grouped by owner rank, on this GPU (b12g_route_point_boxes)."""
        return self.tree.route_point_boxes(codes, valid, starts, ranks, world, want_slot)

    def set_flags(self, flags: int) -> None:
        if not self.empty:
            self.tree.set_flags(flags, count=False)

    def unset_flags(self, flags: int) -> None:
        if not self.empty:
            self.tree.unset_flags(flags, count=False)   # the count is not needed: no round trip

    def subdivide(self, flags: int) -> None:
        if not self.empty:
            self.tree.subdivide(flags)

    def remove(self, flags: int) -> None:
        if self.empty:
            return
        before = self.tree.count()
        if self.tree.remove(flags) == before:
            self.empty = True         # the tree put the surrounding box back; this run holds nothing

    def points_per_box(self, scheme) -> int:
        return scheme.grid.points_per_box(self.tree.dim)

    def image_point_boxes(self, scheme):
        import torch
        if self.empty:
            return (torch.empty(0, dtype=torch.int64, device=self.device),
                    torch.empty(0, dtype=torch.uint8, device=self.device))
        return self.tree.image_point_boxes(scheme, self.device)

    def max_depth(self) -> int:
        return 0 if self.empty else self.tree.depth()

    def image_hit_boxes(self, scheme, depth: int):
        """The point boxes of image_point_boxes cut to `depth` (at least every leaf's depth,
        on every rank) as a set (each warp's distinct boxes once): all that setting the
        flags of the leaves they hit needs, in fewer boxes to send."""
        import torch
        if self.empty:
            return (torch.empty(0, dtype=torch.int64, device=self.device),
                    torch.empty(0, dtype=torch.uint8, device=self.device))
        return self.tree.image_distinct_point_boxes(scheme, self.device, depth)

    def set_flags_by_point_boxes(self, codes, valid, flags: int) -> int:
        return 0 if self.empty else self.tree.set_flags_by_point_boxes(codes, valid, flags)

    def search_point_boxes(self, codes, valid):
        import torch
        if self.empty:
            return torch.full((codes.numel(),), -1, dtype=torch.int64, device=self.device)
        return self.tree.search_point_boxes(codes, valid)

    def leaves(self):
        import torch
        if self.empty:
            z = torch.empty(0, dtype=torch.uint8, device=self.device)
            return torch.empty(0, dtype=torch.int64, device=self.device), z, z.clone()
        return self.tree.leaves_device(self.device)

    def load(self, codes, depth, flags) -> None:
        if codes.numel() == 0:
            self.empty = True
            return
        self.tree.load_leaves_device(codes, depth, flags)
        self.empty = False

    def transition_rows(self, targets, points_per_row, n_columns, absolute, invalid_column):
        if self.empty:
            return None
        return self.tree.transition_rows(targets, points_per_row, n_columns, absolute, invalid_column)

    def host_leaves(self):
        if self.empty:
            return np.zeros(0, np.uint64), np.zeros(0, np.uint8), np.zeros(0, np.uint8)
        return self.tree.leaves()


# ----------------------------------------------------------------------------- the ranks' steps
@dataclass
class RowBlock:
    """A rank's rows of the partitioned transition matrix: rows row_offset .. + n_rows of
    the whole matrix, global columns; n_cols is the whole matrix's column count."""
    rows: object
    row_offset: int
    n_rows: int
    n_cols: int


class PartitionedTree:
    """Rank `rank` of `world` of one range-partitioned tree (see the module docstring).

    `balance`: the runs are evened out when the largest exceeds the mean by this factor.
    """

    def __init__(self, run, rank: int, world: int, balance: float = 1.05):
        if world < 1 or not 0 <= rank < world:
            raise ValueError(f"rank {rank} of {world}")
        self.run, self.rank, self.world, self.balance = run, rank, world, float(balance)
        self.table = None          # (world, 2): leaves and ordered start of every run

    # -- layout
    def _layout(self):
        import torch
        n = self.run.n
        start = _ordered(self.run.start()) if n else 0
        depth = self.run.max_depth() if hasattr(self.run, "max_depth") else 64
        row = torch.tensor([n, start, depth], dtype=torch.int64, device=self.run.device)
        self.table = (yield ("allgather", row)).to("cpu")
        return self.table

    def _owned_runs(self):
        """(ranks, unsigned first codes) of the non-empty runs, ascending."""
        ranks = [r for r in range(self.world) if int(self.table[r, 0]) > 0]
        starts = [(int(self.table[r, 1]) & ((1 << 64) - 1)) ^ (1 << 63) for r in ranks]
        return ranks, starts

    def _owners(self, codes, valid):
        """The rank that owns each point box (int16 tensor), or an int when one rank owns all
        (runs held on the host; a run on a GPU routes with its own kernels, _route_boxes)."""
        import torch
        n = self.table[:, 0]
        ranks = torch.nonzero(n > 0).flatten()
        if ranks.numel() == 1:
            return int(ranks[0])
        starts = self.table[ranks, 1].to(codes.device)
        ranks = ranks.to(device=codes.device, dtype=torch.int16)
        pos = torch.searchsorted(starts, codes ^ _SIGN, right=True) - 1
        owner = ranks[pos.clamp_(min=0)]
        return torch.where(valid != 0, owner, ranks[-1])

    def _route(self, owner, *fields):
        """Per destination rank, the fields of the point boxes it owns (in their order)."""
        import torch
        if isinstance(owner, int):
            # one rank owns every point box: no permutation
            empty = [f[:0] for f in fields]
            parts = [[f if d == owner else e for d in range(self.world)] for f, e in zip(fields, empty)]
            return None, parts
        # a stable partition by owner: each point box's slot is its owner's offset plus
        # the number of earlier point boxes with the same owner
        splits = torch.bincount(owner.to(torch.int32), minlength=self.world).tolist()
        slot = torch.empty(owner.shape, dtype=torch.int64, device=owner.device)
        base = 0
        for d in range(self.world):
            if splits[d] == 0:
                continue
            mine = owner == d
            slot = torch.where(mine, torch.cumsum(mine, 0) - 1 + base, slot)
            base += splits[d]
        parts = []
        for f in fields:
            g = torch.empty_like(f)
            g[slot] = f
            parts.append(list(g.split(splits)))
        return slot, parts

    def _route_boxes(self, codes, valid, want_slot=True):
        """(slot or None, per-rank codes, per-rank validity) of this rank's point boxes."""
        ranks, starts = self._owned_runs()
        route = getattr(self.run, "route_point_boxes", None)
        if len(ranks) > 1 and route is not None:
            slot, c_parts, v_parts = route(codes, valid, starts, ranks, self.world, want_slot)
            return slot, (c_parts, v_parts)
        return self._route(self._owners(codes, valid), codes, valid)

    def _exchange_point_boxes(self, codes, valid, want_slot=True):
        import torch
        slot, (c_parts, v_parts) = self._route_boxes(codes, valid, want_slot)
        rc = yield ("alltoall", c_parts)
        rv = yield ("alltoall", v_parts)
        return slot, [x.numel() for x in rc], torch.cat(rc), torch.cat(rv)

    def _rebalance(self):
        """Even the runs out when the largest exceeds `balance` times the mean and the
        share of an even split (rank r gets leaves r*n//world .. (r+1)*n//world - 1)."""
        import torch
        n = self.table[:, 0].tolist()
        total = sum(n)
        if total == 0 or max(n) <= max(self.balance * total / self.world, -(-total // self.world)):
            return False
        off = np.concatenate([[0], np.cumsum(n)])
        lo, hi = int(off[self.rank]), int(off[self.rank + 1])
        codes, depth, flags = self.run.leaves()
        packed = depth.to(torch.int32) << 8 | flags.to(torch.int32)
        c_parts, p_parts = [], []
        for d in range(self.world):
            a, b = max(lo, d * total // self.world), min(hi, (d + 1) * total // self.world)
            a, b = a - lo, max(b - lo, a - lo)
            c_parts.append(codes[a:b])
            p_parts.append(packed[a:b])
        rc = yield ("alltoall", c_parts)
        rp = yield ("alltoall", p_parts)
        c, p = torch.cat(rc), torch.cat(rp)
        self.run.load(c, (p >> 8).to(torch.uint8), (p & 0xFF).to(torch.uint8))
        return True

    def _settle(self):
        """After leaves were removed: the surrounding box when none is left, then even out."""
        import torch
        yield from self._layout()
        if int(self.table[:, 0].sum()) == 0:
            if self.rank == 0:
                z = torch.zeros(1, dtype=torch.int64, device=self.run.device)
                u = torch.zeros(1, dtype=torch.uint8, device=self.run.device)
                self.run.load(z, u, u.clone())      # insertSurroundingBoxIfEmpty
            yield from self._layout()
        if (yield from self._rebalance()):
            yield from self._layout()

    # -- the operations (generators; run them with drive or drive_lockstep)
    def start(self):
        """Gathers the layout; the first request of every rank."""
        yield from self._layout()
        if (yield from self._rebalance()):
            yield from self._layout()

    def subdivision(self, scheme, steps: int):
        """setFlags(SD), then `steps` steps of subdivision.m:18-45; returns the whole
        tree's leaf count after each step (the same list on every rank)."""
        if scheme.flags_to_check != 0 or scheme.depth != L.LEAF_DEPTH:
            raise ValueError("the subdivision loop maps every leaf (depth 255, no flag filter)")
        if self.table is None:
            yield from self.start()
        self.run.set_flags(L.SD)
        counts = []
        # a run that can send its image boxes as a set does, cut to the depth of the
        # deepest leaf on any rank after the subdivision (the flags need no more)
        hit_boxes = getattr(self.run, "image_hit_boxes", None)
        for _ in range(steps):
            self.run.subdivide(L.SD)
            if hit_boxes is not None:
                codes, valid = hit_boxes(scheme, min(64, int(self.table[:, 2].max()) + 1))
            else:
                codes, valid = self.run.image_point_boxes(scheme)
            _, _, rc, rv = yield from self._exchange_point_boxes(codes, valid, want_slot=False)
            self.run.set_flags_by_point_boxes(rc, rv, L.HIT)
            self.run.remove(L.HIT)
            self.run.unset_flags(L.HIT)
            yield from self._settle()
            counts.append(int(self.table[:, 0].sum()))
        return counts

    def transition_matrix(self, scheme, absolute: bool = False, invalid_column: bool = False):
        """transitionMatrixForLeaves over the whole tree: this rank's rows (a RowBlock)."""
        import torch
        if scheme.flags_to_check != 0 or scheme.depth != L.LEAF_DEPTH:
            raise ValueError("transitionMatrixForLeaves maps every leaf")
        if self.table is None:
            yield from self.start()
        n = self.table[:, 0].tolist()
        total, offset = sum(n), sum(n[: self.rank])
        P = self.run.points_per_box(scheme)
        codes, valid = self.run.image_point_boxes(scheme)
        slot, sizes, rc, rv = yield from self._exchange_point_boxes(codes, valid)
        idx = self.run.search_point_boxes(rc, rv)
        glob = torch.where(idx >= 0, idx + offset, torch.full_like(idx, -1))
        back = yield ("alltoall", list(glob.split(sizes)))
        targets = torch.cat(back)
        if slot is not None:
            targets = targets[slot]
        lost = torch.tensor([int(bool((targets < 0).any().item())) if targets.numel() else 0],
                            dtype=torch.int64, device=self.run.device)
        any_lost = bool((yield ("allgather", lost)).sum().item())
        rows = self.run.transition_rows(targets, P, total, absolute, invalid_column)
        n_cols = total + 1 if invalid_column and any_lost else total
        return RowBlock(rows, offset, n[self.rank], n_cols)


# ----------------------------------------------------------------------------- drivers
class ProcessGroupExchange:
    """Serves the requests of one rank over a torch.distributed process group."""

    def __init__(self, dist, device, group=None):
        self.dist, self.device, self.group = dist, device, group
        self.world = dist.get_world_size(group)

    def allgather(self, x):
        import torch
        parts = [torch.empty_like(x) for _ in range(self.world)]
        self.dist.all_gather(parts, x.contiguous(), group=self.group)
        return torch.stack(parts)

    def alltoall(self, sends):
        import torch
        sizes = [s.numel() for s in sends]
        cnt = torch.tensor(sizes, dtype=torch.int64, device=self.device)
        rcnt = torch.empty_like(cnt)
        self.dist.all_to_all_single(rcnt, cnt, group=self.group)
        rsizes = rcnt.tolist()
        inp = torch.cat(sends).contiguous()
        out = torch.empty(sum(rsizes), dtype=inp.dtype, device=self.device)
        self.dist.all_to_all_single(out, inp, output_split_sizes=rsizes, input_split_sizes=sizes, group=self.group)
        return list(out.split(rsizes))

    def serve(self, request):
        kind, payload = request
        if kind == "allgather":
            return self.allgather(payload)
        if kind == "alltoall":
            return self.alltoall(payload)
        raise ValueError(f"unknown request {kind}")


def drive(gen, exchange):
    """Runs one rank's generator against a ProcessGroupExchange; returns its result."""
    try:
        request = next(gen)
        while True:
            request = gen.send(exchange.serve(request))
    except StopIteration as stop:
        return stop.value


def drive_lockstep(gens):
    """Runs the generators of `world` ranks emulated in one process, answering their
    collective requests among themselves; returns their results.  Their kernels never
    wait on one another: each request is answered on the host between launches."""
    import torch
    world = len(gens)
    results = [None] * world
    pending = []
    for i, g in enumerate(gens):
        try:
            pending.append(next(g))
        except StopIteration as stop:
            pending.append(None)
            results[i] = stop.value
    while any(p is not None for p in pending):
        if any(p is None for p in pending):
            raise RuntimeError("ranks took different collective steps")
        kinds = {p[0] for p in pending}
        if len(kinds) != 1:
            raise RuntimeError(f"ranks took different collective steps: {sorted(kinds)}")
        kind = kinds.pop()
        if kind == "allgather":
            table = torch.stack([p[1].to(pending[0][1].device) for p in pending])
            replies = [table.to(p[1].device) for p in pending]
        elif kind == "alltoall":
            replies = [[pending[s][1][d].to(pending[d][1][d].device) for s in range(world)] for d in range(world)]
        else:
            raise ValueError(f"unknown request {kind}")
        for i, g in enumerate(gens):
            try:
                pending[i] = g.send(replies[i])
            except StopIteration as stop:
                pending[i] = None
                results[i] = stop.value
    return results


def split_leaves(codes, depth, flags, world: int):
    """Contiguous runs of about the same size: rank r gets leaves r*n//world ..
    (r+1)*n//world - 1 of the tree's order."""
    n = len(codes)
    cuts = [r * n // world for r in range(world + 1)]
    return [(codes[a:b], depth[a:b], flags[a:b]) for a, b in zip(cuts[:-1], cuts[1:])]
