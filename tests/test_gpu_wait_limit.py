"""The bounded waits of the solver, made to run out without faulting anything.

A solver group's blocks meet at two exchanges per iteration; every wait of a
block for the others is bounded (the host sets the bound with the
"wait_limit_ms" option).  The "test_drop_block" hook launches the next wave
without its last thread block, so the other blocks of that group wait for a
record that never comes: the wait runs out, the group sets its error flag and
returns, and the call reports the failure.  The device stays usable: the
next ordinary solve must succeed and give the usual result."""
import time

import numpy as np
import pytest

from svmb200 import cabi, datagen
from svmb200.lib import EngineError, Server, make_params

pytestmark = pytest.mark.gpu


@pytest.fixture
def short_waits(engine):
    engine.set_option("wait_limit_ms", 500)
    engine.set_option("graphs", 0)
    yield engine
    engine.set_option("wait_limit_ms", 0)
    engine.set_option("graphs", 1)


def test_solve_reports_a_group_that_never_completes(short_waits):
    eng = short_waits
    tr, _ = datagen.dense_gauss(n=2000, n_test=0, d=16, seed=5)
    params = make_params(svm_type=0, kernel_type=2, gamma=1.0 / 16, blocks=2)
    want, st_want = eng.solve_binary(tr, params)
    eng.set_option("test_drop_block", 1)
    t0 = time.perf_counter()
    with pytest.raises(EngineError, match="timed out"):
        eng.solve_binary(tr, params)
    assert time.perf_counter() - t0 < 20.0
    got, st = eng.solve_binary(tr, params)
    np.testing.assert_array_equal(got, want)
    assert st["iters"] == st_want["iters"]


def test_svm_train_returns_null_and_recovers(short_waits):
    eng = short_waits
    tr, _ = datagen.dense_gauss(n=2000, n_test=0, d=16, seed=6)
    prm = cabi.make_param(svm_type=0, kernel_type=2, gamma=1.0 / 16, C_=1.0)
    eng.set_option("blocks", 2)
    try:
        eng.set_option("test_drop_block", 1)
        with pytest.raises(EngineError, match="svm_train failed"):
            eng.train(tr, prm)
        model = eng.train(tr, prm)
        assert model.contents.l > 0
        model.free()
    finally:
        eng.set_option("blocks", 0)


def test_request_loop_fails_only_the_broken_request(short_waits):
    """Two requests of three blocks each; the next launch loses its last
    block.  Exactly one request (the last one of that launch) fails; the
    other's result equals its solve alone."""
    eng = short_waits
    a, _ = datagen.dense_gauss(n=3000, n_test=0, d=16, seed=7)
    b, _ = datagen.dense_gauss(n=3000, n_test=0, d=16, seed=8)
    params = make_params(svm_type=0, kernel_type=2, gamma=1.0 / 16)
    alone = [eng.solve_binary(p, params)[0] for p in (a, b)]
    srv = Server(eng, rows_per_block=1000)
    try:
        eng.set_option("test_drop_block", 1)
        tickets = [srv.submit(a, params), srv.submit(b, params)]
        outcome = []
        for t, want in zip(tickets, alone):
            try:
                got, _, _ = srv.wait(t)
                np.testing.assert_array_equal(got, want)
                outcome.append(True)
            except EngineError:
                outcome.append(False)
        assert sorted(outcome) == [False, True], outcome
        # the loop keeps serving
        got, _, _ = srv.wait(srv.submit(a, params))
        np.testing.assert_array_equal(got, alone[0])
        st = srv.stats()
        assert st["failed"] == 1
    finally:
        srv.close()
