"""GPU: the job server (continuous batching of subdivision jobs across families) gives
every job exactly what one ImplicitBoxTree gives for it - per-step counts, final leaf
codes and transition matrix bit-exact - whether it runs alone or joins a mix of jobs
already in flight, and matches the reference's golden runs."""
import numpy as np
import pytest

from workloads import csr_digests, sha

pytestmark = pytest.mark.gpu

B = pytest.importorskip("b12_b200")
from b12_b200.workloads import (FORCED_CENTER, FORCED_RADIUS, HENON_CENTER, HENON_RADIUS,  # noqa: E402
                                LORENZ_CENTER, LORENZ_RADIUS, lorenz_scan)

HENON = (HENON_CENTER, HENON_RADIUS)
DUFFING = (FORCED_CENTER, FORCED_RADIUS)


@pytest.fixture(scope="module", autouse=True)
def _device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def single(center, radius, mp, grid, depth):
    t = B.ImplicitBoxTree(center, radius)
    sc = B.Scheme(mp, grid)
    counts = t.subdivision_run(sc, depth)
    rowptr, cols, vals = t.transition_matrix(sc).to_host()
    return dict(counts=np.asarray(counts, dtype=np.uint32), codes=t.leaves()[0], rowptr=rowptr, cols=cols, vals=vals)


def done_result(srv, jid):
    inf = srv.info(jid)
    if inf["state"] != B._lib.JOB_DONE:
        srv.result(jid)  # raises with the job's error
    assert inf["t_submit"] <= inf["t_start"] <= inf["t_done"]
    return srv.result(jid)


def assert_same(got, want, what):
    for k in ("counts", "codes", "rowptr", "cols", "vals"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=f"{what}: {k}")


def mixed_jobs():
    rho, _ = lorenz_scan(6, 1)
    jobs = []
    for a, d in [(1.4, 14), (1.2, 12), (1.0, 16), (1.3, 10), (1.1, 13)]:
        jobs.append((*HENON, B.henon(a, 0.3), B.inner_grid(4), d))
    for r, d in zip(rho, [12, 10, 14, 11, 13, 9]):
        jobs.append((LORENZ_CENTER, LORENZ_RADIUS, B.lorenz(rho=float(r), fma=True), B.inner_grid(5), d))
    jobs.append((*DUFFING, B.forced_duffing(), B.inner_grid(4), 12))
    return jobs


def test_jobs_in_a_staggered_mix_match_single_trees():
    jobs = mixed_jobs()
    with B.JobServer() as srv:
        # first wave; the second wave joins while the first is in flight
        first = [srv.submit(*j) for j in jobs[::2]]
        done = srv.poll(wait=60.0)
        assert done, "no job finished"
        second = [srv.submit(*j) for j in jobs[1::2]]
        srv.wait_all(set(first + second) - set(done))
        ids = dict(zip(range(0, len(jobs), 2), first)) | dict(zip(range(1, len(jobs), 2), second))
        for k, jid in sorted(ids.items()):
            assert_same(done_result(srv, jid), single(*jobs[k]), f"job {k}")
        st = srv.stats()
        assert st["running"] == 0 and st["waiting"] == 0 and st["ticks"] > 0
        for jid in ids.values():
            srv.release(jid)
        assert srv.stats()["in_use_bytes"] == 0


def test_a_job_gives_the_same_result_alone_and_in_the_mix():
    jobs = mixed_jobs()
    with B.JobServer() as srv:
        jid = srv.submit(*jobs[2])
        srv.wait_all([jid])
        alone = done_result(srv, jid)
    with B.JobServer() as srv:
        ids = [srv.submit(*j) for j in jobs]
        srv.wait_all(ids)
        mixed = done_result(srv, ids[2])
    assert_same(mixed, alone, "alone vs mix")


def test_served_jobs_match_reference_goldens(golden):
    cases = [("henon_d20", (*HENON, B.henon(), B.inner_grid(4))),
             ("lorenz_d15", (LORENZ_CENTER, LORENZ_RADIUS, B.lorenz(), B.inner_grid(5))),
             ("forced_duffing_d16", (*DUFFING, B.forced_duffing(), B.inner_grid(4)))]
    with B.JobServer() as srv:
        ids = [srv.submit(*spec, len(golden(name)[0]["steps"])) for name, spec in cases]
        srv.wait_all(ids)
        for jid, (name, _) in zip(ids, cases):
            meta = golden(name)[0]
            r = done_result(srv, jid)
            assert list(r["counts"]) == [s["n"] for s in meta["steps"]], name
            assert sha(r["codes"]) == meta["steps"][-1]["codes_sha256"], name
            d = csr_digests(r["rowptr"], r["cols"], r["vals"])
            for k in ("nnz", "rowptr_sha256", "cols_sha256", "vals_sha256"):
                assert d[k] == meta["tm"][k], (name, k)


def test_admission_holds_jobs_until_memory_is_released():
    # a cap that holds one of these jobs at a time (each is projected at about 2 MB):
    # the rest wait until the previous result is released
    rho, _ = lorenz_scan(4, 2)
    with B.JobServer(hbm_cap_bytes=3 << 20) as srv:
        ids = [srv.submit(LORENZ_CENTER, LORENZ_RADIUS, B.lorenz(rho=float(r), fma=True), B.inner_grid(5), 15)
               for r in rho]
        seen_waiting = False
        done = []
        while len(done) < len(ids):
            st = srv.stats()
            seen_waiting |= st["waiting"] > 0
            assert st["running"] <= 1
            for jid in srv.poll(wait=0.05):
                assert srv.info(jid)["state"] == B._lib.JOB_DONE
                done.append(jid)
                srv.release(jid)
        assert seen_waiting and done == ids
        assert srv.stats()["in_use_bytes"] == 0


def test_invalid_jobs_are_refused():
    with B.JobServer() as srv:
        with pytest.raises(B.B12gError):
            srv.submit(*HENON, B.henon(), B.inner_grid(4), 0)
        with pytest.raises(B.B12gError):
            srv.submit(*HENON, B.henon(), B.philox_grid(16, 1), 8)
