"""Job server over libb12g's continuous-batching engines (include/b12g.h, b12g_server_*).

A job is `depth` steps of the subdivision loop of the reference's subdivision.m:18-45
from the surrounding box, followed by transitionMatrixForLeaves
(B12c/src/include/ImplicitBoxTree.h:468-603) with relative probabilities and lost
points dropped.  Its result - per-step leaf counts, final leaf codes and CSR - equals
what one ImplicitBoxTree gives for the same job, whatever else the server runs.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib as L
from ._lib import check, lib
from .tree import GridSpec, MapSpec


def job_spec(center, radius, mp: MapSpec, grid: GridSpec, depth: int) -> L.Job:
    j = L.Job()
    j.domain.dim = len(center)
    for k in range(len(center)):
        j.domain.center[k] = float(center[k])
        j.domain.radius[k] = float(radius[k])
    j.map = mp.to_c()
    j.grid = grid.to_c()
    j.depth = int(depth)
    return j


class JobServer:
    """Submit subdivision jobs; poll for finished ones; read and release their results."""

    def __init__(self, hbm_cap_bytes: int = 0):
        self._h = C.c_void_p()
        check(lib().b12g_server_create(int(hbm_cap_bytes), C.byref(self._h)), "server_create")

    def close(self) -> None:
        if self._h:
            lib().b12g_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, center, radius, mp: MapSpec, grid: GridSpec, depth: int) -> int:
        j = job_spec(center, radius, mp, grid, depth)
        jid = C.c_uint64()
        check(lib().b12g_server_submit(self._h, C.byref(j), C.byref(jid)), "server_submit")
        return jid.value

    def poll(self, wait: float = 0.0, max_ids: int = 4096) -> list[int]:
        ids = np.zeros(max_ids, dtype=np.uint64)
        n = C.c_uint32()
        check(lib().b12g_server_poll(self._h, ids.ctypes.data, max_ids, C.byref(n), float(wait)), "server_poll")
        return [int(x) for x in ids[: n.value]]

    def info(self, jid: int) -> dict:
        i = L.JobInfo()
        check(lib().b12g_server_job(self._h, jid, C.byref(i)), "server_job")
        return dict(state=i.state, depth=i.depth, n_boxes=i.n_boxes, nnz=i.nnz, t_submit=i.t_submit,
                    t_start=i.t_start, t_done=i.t_done)

    def result(self, jid: int) -> dict:
        """counts after each step, final leaf codes, CSR (rowptr, cols, vals) of a done job."""
        inf = self.info(jid)
        n, z = inf["n_boxes"], inf["nnz"]
        codes = np.zeros(max(n, 1), dtype=np.uint64)
        counts = np.zeros(inf["depth"], dtype=np.uint32)
        rowptr = np.zeros(max(n, 1) + 1, dtype=np.uint32)
        cols = np.zeros(max(z, 1), dtype=np.uint32)
        vals = np.zeros(max(z, 1), dtype=np.float64)
        check(lib().b12g_server_result(self._h, jid, codes.ctypes.data, counts.ctypes.data, rowptr.ctypes.data,
                                       cols.ctypes.data, vals.ctypes.data), "server_result")
        return dict(codes=codes[:n], counts=counts, rowptr=rowptr[: n + 1], cols=cols[:z], vals=vals[:z])

    def counts(self, jid: int) -> np.ndarray:
        """Leaf counts after each step of a done job."""
        counts = np.zeros(self.info(jid)["depth"], dtype=np.uint32)
        check(lib().b12g_server_result(self._h, jid, None, counts.ctypes.data, None, None, None), "server_result")
        return counts

    def release(self, jid: int) -> None:
        check(lib().b12g_server_release(self._h, jid), "server_release")

    def stats(self) -> dict:
        t, b, u, c = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        w, r = C.c_uint32(), C.c_uint32()
        check(lib().b12g_server_stats(self._h, C.byref(t), C.byref(b), C.byref(u), C.byref(c), C.byref(w),
                                      C.byref(r)), "server_stats")
        return dict(ticks=t.value, box_images=b.value, in_use_bytes=u.value, cap_bytes=c.value, waiting=w.value,
                    running=r.value)

    def engine_stats(self) -> list[dict]:
        """Per engine (family): map kind, ticks, finished jobs, host seconds in ticks and in finishing."""
        out = []
        while True:
            k, t, d = C.c_uint32(), C.c_uint64(), C.c_uint64()
            ts, fs = C.c_double(), C.c_double()
            st = lib().b12g_server_engine_stats(self._h, len(out), C.byref(k), C.byref(t), C.byref(d), C.byref(ts),
                                                C.byref(fs))
            if st != L.OK:
                return out
            out.append(dict(map_kind=k.value, ticks=t.value, jobs_done=d.value, tick_seconds=ts.value,
                            finish_seconds=fs.value))

    def wait_all(self, ids, timeout: float = 600.0) -> list[int]:
        """Block until every job in `ids` has finished (done or failed); returns them in finish order."""
        left = set(ids)
        order = []
        t_end = time.monotonic() + timeout
        while left:
            if time.monotonic() > t_end:
                raise TimeoutError(f"{len(left)} jobs still unfinished")
            for jid in self.poll(wait=0.05):
                if jid in left:
                    left.discard(jid)
                    order.append(jid)
        return order


def stream_job_args(job: dict):
    """(center, radius, map, grid, depth) of a served-stream job (b12_b200.workloads.job_stream):
    Henon and forced Duffing with 4x4 inner grids, Lorenz (explicit FMA integrator) with a
    5x5x5 inner grid."""
    from . import tree as T
    from . import workloads as W
    fam, p, d = job["family"], job["params"], job["depth"]
    if fam == "henon":
        return W.HENON_CENTER, W.HENON_RADIUS, T.henon(p[0], p[1]), T.inner_grid(4), d
    if fam == "lorenz":
        return W.LORENZ_CENTER, W.LORENZ_RADIUS, T.lorenz(p[0], p[1], p[2], fma=True), T.inner_grid(5), d
    if fam == "forced_duffing":
        return W.FORCED_CENTER, W.FORCED_RADIUS, T.forced_duffing(200, *p), T.inner_grid(4), d
    raise ValueError(fam)


def replay(server: JobServer, stream: list, on_done=None, timeout: float = 3600.0) -> dict:
    """Submit every job of `stream` at its arrival time (seconds after the start) and wait
    for all of them.  Returns per-job latency (finish minus scheduled arrival, seconds),
    the time from the first arrival to the last finish, and the largest submission lag.
    `on_done(job, jid)` is called for every finished job (e.g. to read and release it)."""
    n = len(stream)
    t0 = time.monotonic()
    ids = {}
    latency = [0.0] * n
    lag = 0.0
    i = 0
    finished = 0
    t_first = None
    t_last = 0.0
    while finished < n:
        now = time.monotonic() - t0
        if now > timeout:
            raise TimeoutError(f"{n - finished} jobs unfinished")
        while i < n and stream[i]["arrival"] <= now:
            jid = server.submit(*stream_job_args(stream[i]))
            ids[jid] = i
            lag = max(lag, time.monotonic() - t0 - stream[i]["arrival"])
            if t_first is None:
                t_first = stream[i]["arrival"]
            i += 1
        wait = min(0.01, stream[i]["arrival"] - now) if i < n else 0.01
        for jid in server.poll(wait=max(wait, 0.0)):
            k = ids[jid]
            inf = server.info(jid)
            if inf["state"] != L.JOB_DONE:
                server.result(jid)  # raises with the job's error
            latency[k] = inf["t_done"] - (t0 + stream[k]["arrival"])
            t_last = max(t_last, inf["t_done"] - t0)
            finished += 1
            if on_done is not None:
                on_done(stream[k], jid)
    return dict(latency=latency, span=t_last - (t_first or 0.0), submit_lag=lag)
