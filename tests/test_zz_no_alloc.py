"""svmb_solve_dense_noalloc: the entry point for callers that cannot allocate
device memory (everything it needs lives in a fixed workspace inside the
library; the caller only owns the rows, labels and output, already on the
device).

Its result must equal the allocating entry point's (svmb_solve_binary_csr) on
the same problem, on two calls in a row (the second call reuses a workspace
that still holds the first call's state).  This file is collected last so that
a run that stops at the first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from svmb200 import datagen
from svmb200.lib import SolveStats, SvmbParams, make_params

pytestmark = pytest.mark.gpu


def _noalloc_fn(eng):
    fn = eng.lib.svmb_solve_dense_noalloc
    fn.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(SvmbParams), C.c_void_p,
                   C.POINTER(SolveStats), C.c_void_p]
    fn.restype = C.c_int
    return fn


@pytest.mark.parametrize("kernel,gamma,C_", [(2, 1.0 / 32, 1.0), (0, 0.0, 0.5)])
def test_noalloc_matches_allocating_entry_point(engine, kernel, gamma, C_):
    import torch
    tr, _ = datagen.dense_gauss(n=3000, n_test=0, d=32, seed=21)
    params = make_params(svm_type=0, kernel_type=kernel, gamma=gamma, C_pos=C_)
    want, st_want = engine.solve_binary(tr, params)

    X = torch.from_numpy(tr.to_dense()).cuda().contiguous()          # [n][32] float32, ld = 32
    y = torch.from_numpy(np.ascontiguousarray(tr.y)).cuda()
    out = torch.zeros(tr.n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    fn = _noalloc_fn(engine)
    free_after = []
    for call in range(2):
        out.fill_(float("nan"))
        st = SolveStats()
        rc = fn(tr.n, X.shape[1], X.data_ptr(), y.data_ptr(), C.byref(params), out.data_ptr(), C.byref(st), None)
        assert rc == 0, engine.error()
        torch.cuda.synchronize()
        free_after.append(torch.cuda.mem_get_info()[0])
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-9, err_msg=f"call {call}")
        assert st.iters == st_want["iters"]
        assert abs(st.rho - st_want["rho"]) <= 1e-9
        assert abs(st.obj - st_want["obj"]) <= 1e-9 * abs(st_want["obj"])
    # the property the entry point exists for: a call takes no device memory
    # (the first call may still load the module; the second must not allocate)
    assert abs(free_after[1] - free_after[0]) <= 2 << 20, free_after


def test_noalloc_rejects_sizes_beyond_the_workspace(engine):
    import torch
    n = 16385
    X = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    y = torch.ones(n, dtype=torch.float64, device="cuda")
    out = torch.zeros(n, dtype=torch.float64, device="cuda")
    fn = _noalloc_fn(engine)
    rc = fn(n, 4, X.data_ptr(), y.data_ptr(), C.byref(make_params()), out.data_ptr(), None, None)
    assert rc != 0
    assert "16384" in engine.error()


def test_noalloc_rejects_a_misaligned_row_pointer(engine):
    """Rows are read in 16-byte pieces; a view 4 bytes into a buffer is refused
    before anything is launched, so the caller's context stays usable."""
    import torch
    n, ld = 64, 8
    X = torch.zeros((n + 1) * ld, dtype=torch.float32, device="cuda")
    y = torch.ones(n, dtype=torch.float64, device="cuda")
    y[::2] = -1
    out = torch.zeros(n, dtype=torch.float64, device="cuda")
    fn = _noalloc_fn(engine)
    rc = fn(n, ld, X.data_ptr() + 4, y.data_ptr(), C.byref(make_params()), out.data_ptr(), None, None)
    assert rc != 0
    assert "aligned" in engine.error()
    torch.cuda.synchronize()
