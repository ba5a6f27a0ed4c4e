"""CPU: the seeded workload generators of the batched and served benchmarks."""
import math

from b12_b200.workloads import SplitMix64, job_stream, lorenz_scan


def test_splitmix64_known_answers():
    g = SplitMix64(0)
    # published first outputs of splitmix64 seeded with 0
    assert g.next_u64() == 0xE220A8397B1DCDAF
    assert g.next_u64() == 0x6E789E6AA1B965F4
    assert g.next_u64() == 0x06C45D188009454F


def test_lorenz_scan_ranges_and_determinism():
    rho, depth = lorenz_scan(512, 0)
    assert len(rho) == len(depth) == 512
    assert all(15.0 <= r < 35.0 for r in rho) and all(18 <= d <= 27 for d in depth)
    assert (rho, depth) == lorenz_scan(512, 0)
    g = SplitMix64(0)
    assert rho[0] == 15.0 + 20.0 * g.uniform() and depth[0] == 18 + math.floor(10.0 * g.uniform())


def test_job_stream_is_poisson_and_seeded():
    jobs = job_stream(4000, 50.0, 7)
    gaps = [b["arrival"] - a["arrival"] for a, b in zip(jobs, jobs[1:])]
    assert all(g > 0 for g in gaps)
    assert abs(sum(gaps) / len(gaps) - 1 / 50.0) < 0.1 / 50.0
    fam = {f: sum(j["family"] == f for j in jobs) for f in ("henon", "lorenz", "forced_duffing")}
    assert all(1100 < c < 1600 for c in fam.values())
    for j in jobs:
        lo, hi = {"henon": (14, 22), "lorenz": (18, 27), "forced_duffing": (16, 22)}[j["family"]]
        assert lo <= j["depth"] <= hi
    assert job_stream(50, 50.0, 7) == jobs[:50]
