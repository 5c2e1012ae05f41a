"""Continuous-batching server (topx_server_* in include/topx.h).

CPU tests cover argument checks and the admission refusal; the GPU tests check that a job's
result is the same alone and among others, that the HBM budget bounds how many jobs are
admitted at once, and that the footprint estimate used for admission covers what an engine
holds.
"""
import numpy as np
import pytest

from top3d_xl_b200 import Server, TopxError

JOBS = [  # (shape, consType, V0, nLoop, rHat)
    ((12, 24, 12), "GLOBAL", 0.12, 6, 0.0),
    ((16, 32, 16), "GLOBAL", 0.2, 5, 0.0),
    ((12, 24, 12), "LOCAL", 0.5, 5, 6.0),
    ((20, 40, 20), "GLOBAL", 0.1, 4, 0.0),
]


def test_submit_rejects_bad_jobs():
    with Server(slots=1, hbm_budget_bytes=1.0) as s:
        with pytest.raises(TopxError):
            s.submit((2, 24, 12))
        with pytest.raises(TopxError):
            s.submit((12, 24, 12), consType="BOTH")


def test_job_larger_than_the_budget_is_refused_not_run():
    with Server(slots=2, hbm_budget_bytes=1.0) as s:  # 1 byte: nothing fits
        jid = s.submit((12, 24, 12), "GLOBAL", 0.12, 3)
        r = s.wait(jid)
        assert r["status"] == -1 and r["loops"] == 0
        assert "budget" in s.last_error()
        assert s.stats()["failed"] == 1 and s.stats()["max_running"] == 0


def _run_all(slots, budget=0.0, keep=True):
    out = []
    with Server(slots=slots, hbm_budget_bytes=budget) as s:
        ids = [s.submit(sh, ct, V0, nl, np.sqrt(3), rh, keep_density=keep) for sh, ct, V0, nl, rh in JOBS]
        for jid in ids:
            r = s.wait(jid)
            assert r["status"] == 0, s.last_error()
            out.append((r, s.history(jid), s.density(jid, r["numElements"]) if keep else None))
        stats = s.stats()
    return out, stats


@pytest.mark.gpu
def test_each_result_is_the_same_alone_and_in_the_mix():
    alone, st1 = _run_all(slots=1)
    mixed, st4 = _run_all(slots=4)
    assert st1["max_running"] == 1
    assert st4["max_running"] >= 2  # jobs did share the device
    for (ra, ha, xa), (rm, hm, xm) in zip(alone, mixed):
        assert ra["loops"] == rm["loops"] and ra["pcg_its"] == rm["pcg_its"]
        assert [h["c"] for h in ha] == [h["c"] for h in hm]  # bit for bit
        assert np.array_equal(xa, xm)


@pytest.mark.gpu
def test_budget_bounds_the_jobs_on_the_device_and_estimates_cover_footprints():
    # learn one footprint estimate, then allow just one job's worth of memory
    with Server(slots=1) as s:
        r = s.wait(s.submit(JOBS[3][0], "GLOBAL", 0.1, 1))
    assert r["status"] == 0
    assert 0 < r["footprint_bytes"] <= r["footprint_estimate"]
    res, st = _run_all(slots=4, budget=1.2 * r["footprint_estimate"], keep=False)
    assert st["max_running"] == 1
    for rr, _, _ in res:
        assert 0 < rr["footprint_bytes"] <= rr["footprint_estimate"]
