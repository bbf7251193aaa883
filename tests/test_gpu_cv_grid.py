"""svmb_cross_validation_grid: the stratified k-fold cross-validation of the
reference (svm.cpp:2407-2525) over a (C, gamma) grid in one call, every
point's and fold's one-vs-one subproblems solved in batched launches.  Each
point's predictions must equal svm_cross_validation run alone with that
point's parameters and the same rand() state (same folds)."""
import ctypes as C

import numpy as np
import pytest

import cases
from helpers import load_golden, max_index, param_from_opts

pytestmark = pytest.mark.gpu


def test_grid_equals_one_point_at_a_time(engine):
    build, opts, mode = cases.CASES["cv_multiclass"]
    tr, _ = build()
    prm = param_from_opts(opts, max_index(tr))
    Cs = [0.5, 2.0, 8.0]
    gs = [0.0625, 0.25, 0.0625]
    libc = C.CDLL(None)
    libc.srand(7)
    grid = engine.cross_validation_grid(tr, prm, 5, Cs, gs)
    for q, (c, g) in enumerate(zip(Cs, gs)):
        p2 = param_from_opts(opts, max_index(tr))
        p2.C, p2.gamma = c, g
        libc.srand(7)
        one = engine.cross_validation(tr, p2, 5)
        assert np.array_equal(grid[q], one), q


def test_grid_point_matches_reference_cv(engine):
    """A one-point grid is svm_cross_validation: the reference's golden CV targets."""
    build, opts, mode = cases.CASES["cv_multiclass"]
    tr, _ = build()
    prm = param_from_opts(opts, max_index(tr))
    C.CDLL(None).srand(1)
    grid = engine.cross_validation_grid(tr, prm, int(mode[3:]), [prm.C], [prm.gamma])
    assert np.array_equal(grid[0], np.array(load_golden("cv_multiclass")["cv"]))
