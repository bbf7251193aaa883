"""The request loop (svmb_server_*): continuous batching of independent
binary solves.  Requests submitted while others run are admitted next to
them (concurrent launches); every result must equal the same request solved
alone (the exact form is bit-reproducible, so the check is equality)."""
import time

import numpy as np
import pytest

from svmb200 import datagen
from svmb200.lib import EngineError, Server, make_params

pytestmark = pytest.mark.gpu


def _params(job, form=0):
    return make_params(svm_type=job.svm_type, kernel_type=job.kernel_type, gamma=job.gamma, degree=job.degree,
                       C_pos=job.C, nu=job.nu, cache_mb=40.0, form=form)


def test_results_equal_alone_and_in_the_mix(engine):
    jobs = datagen.serving_mix(n_jobs=14, rate=400.0, n_lo=300, n_hi=6000, seed=11)
    big, _ = datagen.dense_gauss(n=12000, n_test=0, d=64, seed=12, flip=0.05)
    big_prm = make_params(svm_type=0, kernel_type=2, gamma=1.0 / 64, C_pos=10.0, cache_mb=40.0)
    srv = Server(engine, max_inflight=4)
    try:
        t_big = srv.submit(big, big_prm)
        time.sleep(0.02)
        tickets = []
        t0 = time.perf_counter()
        for j in jobs:
            while time.perf_counter() - t0 < j.arrival:
                time.sleep(0.0005)
            tickets.append(srv.submit(j.problem, _params(j)))
        got = [srv.wait(t) for t in tickets]
        got_big = srv.wait(t_big)
        st = srv.stats()
    finally:
        srv.close()
    assert st["completed"] == len(jobs) + 1 and st["failed"] == 0, st
    assert st["max_concurrent_waves"] >= 2, st          # later requests ran next to the large one
    assert 0 < st["p50_s"] <= st["p99_s"] <= st["max_s"]
    for j, (alpha, stats, lat) in zip(jobs, got):
        want, st_want = engine.solve_binary(j.problem, _params(j))
        assert np.array_equal(alpha, want)
        assert stats["iters"] == st_want["iters"] and stats["rho"] == st_want["rho"]
        assert lat > 0
    want_big, _ = engine.solve_binary(big, big_prm)
    assert np.array_equal(got_big[0], want_big)


def test_rejects_a_request_larger_than_the_budget(engine):
    p, _ = datagen.dense_gauss(n=2000, n_test=0, d=16, seed=3)
    srv = Server(engine, mem_bytes=1 << 20)
    try:
        t = srv.submit(p, make_params(svm_type=0, kernel_type=2, gamma=1.0 / 16, C_pos=1.0))
        with pytest.raises(EngineError, match="budget"):
            srv.wait(t)
    finally:
        srv.close()
