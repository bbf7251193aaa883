"""Repeated batched solves replay a captured CUDA graph of the launch's stream
work; the autotuner varies only speed knobs.  Results must be identical with
graphs on or off and whatever the tuner tries."""
import numpy as np
import pytest

from svmb200 import datagen
from svmb200.lib import ResidentRows, make_params

pytestmark = pytest.mark.gpu


def test_graph_replays_give_identical_results(engine):
    tr, _, _ = datagen.multiclass_geo(n_classes=4, largest=1500, d=32, seed=8)
    rows = ResidentRows(engine, tr)
    labels = np.unique(tr.y)
    inst_rows, inst_y = [], []
    for a in range(len(labels)):
        for b in range(a + 1, len(labels)):
            sel = np.where((tr.y == labels[a]) | (tr.y == labels[b]))[0].astype(np.int32)
            inst_rows.append(sel)
            inst_y.append(np.where(tr.y[sel] == labels[a], 1.0, -1.0))
    prm = [make_params(svm_type=0, kernel_type=2, gamma=1 / 32, C_pos=1.0) for _ in inst_rows]
    engine.set_option("graphs", 0)
    try:
        ref, st_ref = rows.solve_many(inst_rows, inst_y, prm)
    finally:
        engine.set_option("graphs", 1)
    g0 = engine.graph_counts()
    outs = [rows.solve_many(inst_rows, inst_y, prm) for _ in range(10)]   # tuner explores, then settles
    g1 = engine.graph_counts()
    assert g1["replayed"] > g0["replayed"]
    for al, st in outs:
        for a, b in zip(al, ref):
            assert np.array_equal(a, b)
        assert [s["iters"] for s in st] == [s["iters"] for s in st_ref]
    assert not engine.autotune_last()["exploring"]


def test_fill_depths_give_identical_results(engine):
    """The ring of column slices per warp in the CUDA-core row fills (1 to 4
    deep) changes only how much of a fill is in flight: alphas and iteration
    counts are bit-identical at every depth, in the exact and fp32 forms, with
    a width (d=100) whose last slice is partial."""
    tr, _, _ = datagen.multiclass_geo(n_classes=3, largest=1200, d=100, seed=11)
    rows = ResidentRows(engine, tr, layout=1)
    sel = np.where(tr.y != tr.y[0])[0]
    inst_rows = [np.arange(tr.n, dtype=np.int32), sel.astype(np.int32)]
    inst_y = [np.where(tr.y == tr.y[0], 1.0, -1.0), np.where(tr.y[sel] == tr.y[sel][0], 1.0, -1.0)]
    for bad in (0, 5):
        with pytest.raises(Exception):
            engine.set_option("fill_depth", bad)
    try:
        for form in (0, 1):
            prm = [make_params(svm_type=0, kernel_type=2, gamma=1 / 100, C_pos=2.0, form=form) for _ in inst_rows]
            out = {}
            for depth in (1, 2, 3, 4):
                engine.set_option("fill_depth", depth)
                out[depth] = rows.solve_many(inst_rows, inst_y, prm)
            for depth in (1, 2, 3):
                for a, b in zip(out[depth][0], out[4][0]):
                    assert np.array_equal(a, b), (form, depth)
                assert [s["iters"] for s in out[depth][1]] == [s["iters"] for s in out[4][1]]
    finally:
        engine.set_option("fill_depth", 2)
