"""ctypes bindings of libsvm_b200.so."""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import cabi
from .cabi import NodeRows, svm_model, svm_parameter, svm_problem
from .datagen import CSR

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libsvm_b200.so")
CLI_PATH = os.path.join(PKG_DIR, "svm-train")

FORM_EXACT, FORM_FP32, FORM_BF16X3, FORM_FP16X3, FORM_TF32 = 0, 1, 2, 3, 4


class EngineError(RuntimeError):
    pass


class SolveStats(C.Structure):
    _fields_ = [("iters", C.c_longlong), ("obj", C.c_double), ("rho", C.c_double), ("r", C.c_double),
                ("l", C.c_int), ("nr_sv", C.c_int), ("nr_bsv", C.c_int), ("status", C.c_int),
                ("active_size", C.c_int), ("launch", C.c_int), ("seconds", C.c_double),
                ("sum_active", C.c_longlong), ("q_evals", C.c_longlong), ("lookups", C.c_longlong),
                ("hits", C.c_longlong), ("fills", C.c_longlong), ("prefetched", C.c_longlong),
                ("prefetch_used", C.c_longlong), ("prof_cycles", C.c_longlong * 8),
                ("fill_targets", C.c_longlong), ("fill_path", C.c_int),
                ("reserved", C.c_int)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "prof_cycles"}
        d["prof_cycles"] = list(self.prof_cycles)
        return d


class SvmbParams(C.Structure):
    _fields_ = [("svm_type", C.c_int), ("kernel_type", C.c_int), ("degree", C.c_int), ("shrinking", C.c_int),
                ("gamma", C.c_double), ("coef0", C.c_double), ("C_pos", C.c_double), ("C_neg", C.c_double),
                ("nu", C.c_double), ("eps", C.c_double), ("cache_mb", C.c_double), ("form", C.c_int),
                ("blocks", C.c_int), ("prefetch", C.c_int), ("gbar_mode", C.c_int), ("p", C.c_double)]


class ServerConfig(C.Structure):
    _fields_ = [("mem_bytes", C.c_longlong), ("max_inflight", C.c_int), ("max_batch", C.c_int), ("form", C.c_int),
                ("policy", C.c_int), ("rows_per_block", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_longlong), ("failed", C.c_longlong), ("waves", C.c_longlong),
                ("max_concurrent_waves", C.c_longlong), ("peak_mem_bytes", C.c_longlong), ("pending", C.c_longlong),
                ("p50_s", C.c_double), ("p99_s", C.c_double), ("max_s", C.c_double), ("solves_per_s", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def make_params(svm_type=0, kernel_type=2, degree=3, gamma=0.0, coef0=0.0, C_pos=1.0, C_neg=None, nu=0.5,
                eps=1e-3, cache_mb=100.0, shrinking=1, form=FORM_EXACT, blocks=0, prefetch=0,
                gbar_mode=0, eps_tube=0.1) -> SvmbParams:
    p = SvmbParams()
    p.svm_type, p.kernel_type, p.degree, p.shrinking = svm_type, kernel_type, degree, shrinking
    p.gamma, p.coef0, p.C_pos = gamma, coef0, C_pos
    p.C_neg = C_pos if C_neg is None else C_neg
    p.nu, p.eps, p.cache_mb, p.form, p.blocks, p.prefetch = nu, eps, cache_mb, form, blocks, prefetch
    p.gbar_mode = gbar_mode
    p.p = eps_tube
    return p


_P = C.POINTER


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise EngineError(f"{path} is not built (run `make -C libsvm-cuda_b200`)")
    lib = C.CDLL(path)
    lib.svm_train.restype = _P(svm_model)
    lib.svm_train.argtypes = [_P(svm_problem), _P(svm_parameter)]
    lib.svm_cross_validation.argtypes = [_P(svm_problem), _P(svm_parameter), C.c_int, _P(C.c_double)]
    lib.svm_predict_values.restype = C.c_double
    lib.svm_predict_values.argtypes = [_P(svm_model), _P(cabi.svm_node), _P(C.c_double)]
    lib.svm_predict.restype = C.c_double
    lib.svm_predict.argtypes = [_P(svm_model), _P(cabi.svm_node)]
    lib.svm_save_model.argtypes = [C.c_char_p, _P(svm_model)]
    lib.svm_load_model.restype = _P(svm_model)
    lib.svm_load_model.argtypes = [C.c_char_p]
    lib.svm_free_and_destroy_model.argtypes = [_P(_P(svm_model))]
    lib.svm_check_parameter.restype = C.c_char_p
    lib.svm_check_parameter.argtypes = [_P(svm_problem), _P(svm_parameter)]
    lib.svm_set_print_string_function.argtypes = [cabi.PRINT_FUNC]
    lib.svmb_last_error.restype = C.c_char_p
    lib.svmb_kernel_launches.restype = C.c_longlong
    lib.svmb_set_option.argtypes = [C.c_char_p, C.c_longlong]
    lib.svmb_last_train_stats.argtypes = [_P(SolveStats), C.c_int]
    lib.svmb_predict_batch.argtypes = [_P(svm_model), C.c_void_p, C.c_int, _P(C.c_double), _P(C.c_double)]
    lib.svmb_predict_probability_batch.argtypes = [_P(svm_model), C.c_void_p, C.c_int, _P(C.c_double),
                                                   _P(C.c_double)]
    lib.svm_predict_probability.restype = C.c_double
    lib.svm_predict_probability.argtypes = [_P(svm_model), _P(cabi.svm_node), _P(C.c_double)]
    lib.svmb_solve_binary_csr.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          _P(SvmbParams), C.c_void_p, _P(SolveStats)]
    lib.svmb_solve_many_csr.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                        C.c_void_p, C.c_void_p, _P(SvmbParams), C.c_void_p, _P(SolveStats)]
    lib.svmb_rows_upload_csr.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                         _P(C.c_void_p)]
    lib.svmb_rows_info.argtypes = [C.c_void_p, _P(C.c_int), _P(C.c_int), _P(C.c_int), _P(C.c_longlong)]
    lib.svmb_rows_solve_many.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, _P(SvmbParams),
                                         C.c_void_p, _P(SolveStats)]
    lib.svmb_rows_free.argtypes = [C.c_void_p]
    lib.svmb_rows_kernel_block.argtypes = [C.c_void_p, _P(SvmbParams), C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                           C.c_void_p]
    lib.svmb_cross_validation_grid.argtypes = [_P(svm_problem), _P(svm_parameter), C.c_int, C.c_int, C.c_void_p,
                                               C.c_void_p, C.c_void_p]
    lib.svmb_autotune_last.argtypes = [_P(C.c_int), _P(C.c_int), _P(C.c_int)]
    lib.svmb_graph_counts.argtypes = [_P(C.c_longlong), _P(C.c_longlong)]
    lib.svmb_server_create.argtypes = [_P(ServerConfig), _P(C.c_void_p)]
    lib.svmb_server_submit.restype = C.c_longlong
    lib.svmb_server_submit.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       _P(SvmbParams)]
    lib.svmb_server_poll.argtypes = [C.c_void_p, C.c_longlong]
    lib.svmb_server_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, _P(SolveStats), _P(C.c_double)]
    lib.svmb_server_get_stats.argtypes = [C.c_void_p, _P(ServerStats)]
    lib.svmb_server_destroy.argtypes = [C.c_void_p]
    return lib


def csr_arrays(p: CSR) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """0-based int32 columns, float32 values, int64 row pointer."""
    return (np.ascontiguousarray(p.indptr, dtype=np.int64), np.ascontiguousarray(p.indices - 1, dtype=np.int32),
            np.ascontiguousarray(p.values, dtype=np.float32))


class Model:
    """An svm_model* owned by the engine (freed with svm_free_and_destroy_model)."""

    def __init__(self, eng: "Engine", ptr, keep=None):
        self.eng, self.ptr, self.keep = eng, ptr, keep

    @property
    def contents(self) -> svm_model:
        return self.ptr.contents

    def arrays(self) -> dict:
        return cabi.model_arrays(self.contents)

    def free(self):
        if self.ptr:
            self.eng.lib.svm_free_and_destroy_model(C.byref(self.ptr))
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Engine:
    def __init__(self, path: str = LIB_PATH, quiet: bool = True):
        self.lib = _load(path)
        self.path = path
        self._log: List[str] = []
        self._cb = cabi.PRINT_FUNC(lambda s: self._log.append(s.decode("utf-8", "replace")))
        if quiet:
            self.lib.svm_set_print_string_function(self._cb)

    # -- errors -------------------------------------------------------
    def error(self) -> str:
        return (self.lib.svmb_last_error() or b"").decode()

    def _ok(self, rc: int, what: str):
        if rc != 0:
            raise EngineError(f"{what}: {self.error()}")

    def launches(self) -> int:
        return int(self.lib.svmb_kernel_launches())

    def available(self) -> bool:
        return bool(self.lib.svmb_device_available())

    def set_option(self, name: str, value: int):
        self._ok(self.lib.svmb_set_option(name.encode(), value), f"option {name}")

    def take_log(self) -> str:
        s = "".join(self._log)
        self._log.clear()
        return s

    # -- svm.h ----------------------------------------------------------
    def train(self, p: CSR, param: svm_parameter) -> Model:
        rows = NodeRows(p)
        m = self.lib.svm_train(C.byref(rows.prob), C.byref(param))
        if not m:
            raise EngineError(f"svm_train failed: {self.error()}")
        return Model(self, m, keep=rows)

    def check_parameter(self, p: CSR, param: svm_parameter) -> Optional[str]:
        rows = NodeRows(p)
        r = self.lib.svm_check_parameter(C.byref(rows.prob), C.byref(param))
        return r.decode() if r else None

    def cross_validation(self, p: CSR, param: svm_parameter, nfold: int) -> np.ndarray:
        rows = NodeRows(p)
        out = np.zeros(max(p.n, 1))
        self.lib.svm_cross_validation(C.byref(rows.prob), C.byref(param), nfold, out.ctypes.data_as(_P(C.c_double)))
        return out[:p.n]

    def graph_counts(self) -> dict:
        a, b = C.c_longlong(), C.c_longlong()
        self.lib.svmb_graph_counts(C.byref(a), C.byref(b))
        return {"captured": a.value, "replayed": b.value}

    def autotune_last(self) -> dict:
        pf, rpb, ex = C.c_int(), C.c_int(), C.c_int()
        self.lib.svmb_autotune_last(C.byref(pf), C.byref(rpb), C.byref(ex))
        return {"prefetch": pf.value, "rows_per_block": rpb.value, "exploring": bool(ex.value)}

    def cross_validation_grid(self, p: CSR, param: svm_parameter, nfold: int, Cs, gammas) -> np.ndarray:
        """svmb_cross_validation_grid: predictions [npoints][n] of every (C, gamma) point."""
        rows = NodeRows(p)
        Cs = np.ascontiguousarray(Cs, dtype=np.float64)
        gs = np.ascontiguousarray(gammas, dtype=np.float64)
        out = np.zeros((len(Cs), max(p.n, 1)))
        rc = self.lib.svmb_cross_validation_grid(C.byref(rows.prob), C.byref(param), nfold, len(Cs), Cs.ctypes.data,
                                                 gs.ctypes.data, out.ctypes.data)
        self._ok(rc, "svmb_cross_validation_grid")
        return out[:, :p.n]

    def predict(self, model: Model, p: CSR) -> Tuple[np.ndarray, np.ndarray]:
        rows = NodeRows(p)
        k = model.contents.nr_class
        npair = max(k * (k - 1) // 2, 1)
        lab = np.zeros(max(p.n, 1))
        dec = np.zeros((max(p.n, 1), npair))
        rc = self.lib.svmb_predict_batch(model.ptr, C.c_void_p(int(rows.addrs.ctypes.data)) if p.n else None, p.n,
                                         lab.ctypes.data_as(_P(C.c_double)), dec.ctypes.data_as(_P(C.c_double)))
        self._ok(rc, "svmb_predict_batch")
        return lab[:p.n], dec[:p.n, :k * (k - 1) // 2]

    def predict_probability(self, model: Model, p: CSR) -> Tuple[np.ndarray, np.ndarray]:
        """svmb_predict_probability_batch: labels and [n][nr_class] probabilities."""
        rows = NodeRows(p)
        k = model.contents.nr_class
        lab = np.zeros(max(p.n, 1))
        prob = np.zeros((max(p.n, 1), max(k, 1)))
        rc = self.lib.svmb_predict_probability_batch(model.ptr, C.c_void_p(int(rows.addrs.ctypes.data)) if p.n else None,
                                                     p.n, lab.ctypes.data_as(_P(C.c_double)),
                                                     prob.ctypes.data_as(_P(C.c_double)))
        self._ok(rc, "svmb_predict_probability_batch")
        return lab[:p.n], prob[:p.n, :k]

    def predict_probability_one(self, model: Model, p: CSR, i: int) -> Tuple[float, np.ndarray]:
        rows = NodeRows(p)
        k = model.contents.nr_class
        prob = np.zeros(max(k, 1))
        lab = self.lib.svm_predict_probability(model.ptr, rows.row(i), prob.ctypes.data_as(_P(C.c_double)))
        return lab, prob[:k]

    def predict_one(self, model: Model, p: CSR, i: int) -> Tuple[float, np.ndarray]:
        rows = NodeRows(p)
        k = model.contents.nr_class
        dec = np.zeros(max(k * (k - 1) // 2, 1))
        lab = self.lib.svm_predict_values(model.ptr, rows.row(i), dec.ctypes.data_as(_P(C.c_double)))
        return lab, dec[:k * (k - 1) // 2]

    def last_stats(self) -> List[dict]:
        buf = (SolveStats * 4096)()
        n = self.lib.svmb_last_train_stats(buf, 4096)
        return [buf[i].as_dict() for i in range(min(n, 4096))]

    # -- svmb C-ABI -------------------------------------------------------
    def solve_binary(self, p: CSR, params: SvmbParams, y: Optional[np.ndarray] = None):
        rp, col, val = csr_arrays(p)
        yy = np.ascontiguousarray(p.y if y is None else y, dtype=np.float64)
        alpha = np.zeros(max(p.n, 1))
        st = SolveStats()
        rc = self.lib.svmb_solve_binary_csr(p.n, p.d, rp.ctypes.data, col.ctypes.data, val.ctypes.data, yy.ctypes.data,
                                            C.byref(params), alpha.ctypes.data, C.byref(st))
        self._ok(rc, "svmb_solve_binary_csr")
        return alpha[:p.n], st.as_dict()

    def solve_many(self, p: CSR, inst_rows: Sequence[np.ndarray], inst_y: Sequence[np.ndarray],
                   params: Sequence[SvmbParams]):
        rp, col, val = csr_arrays(p)
        ptr = np.zeros(len(inst_rows) + 1, dtype=np.int32)
        ptr[1:] = np.cumsum([len(r) for r in inst_rows])
        rows = np.ascontiguousarray(np.concatenate(inst_rows) if inst_rows else np.zeros(0), dtype=np.int32)
        ys = np.ascontiguousarray(np.concatenate(inst_y) if inst_y else np.zeros(0), dtype=np.float64)
        prm = (SvmbParams * len(params))(*params)
        alpha = np.zeros(max(int(ptr[-1]), 1))
        st = (SolveStats * len(params))()
        rc = self.lib.svmb_solve_many_csr(p.n, p.d, rp.ctypes.data, col.ctypes.data, val.ctypes.data, len(params),
                                          ptr.ctypes.data, rows.ctypes.data, ys.ctypes.data, prm, alpha.ctypes.data, st)
        self._ok(rc, "svmb_solve_many_csr")
        return [alpha[ptr[k]:ptr[k + 1]] for k in range(len(params))], [s.as_dict() for s in st]


class ResidentRows:
    """Rows uploaded to HBM once (svmb_rows_upload_csr); solves reuse them."""

    def __init__(self, eng: Engine, p: CSR, layout: int = -1):
        self.eng = eng
        rp, col, val = csr_arrays(p)
        h = C.c_void_p()
        eng._ok(eng.lib.svmb_rows_upload_csr(p.n, p.d, rp.ctypes.data, col.ctypes.data, val.ctypes.data, layout,
                                             C.byref(h)), "svmb_rows_upload_csr")
        self.h = h
        n, d, dense, nbytes = C.c_int(), C.c_int(), C.c_int(), C.c_longlong()
        eng.lib.svmb_rows_info(h, C.byref(n), C.byref(d), C.byref(dense), C.byref(nbytes))
        self.n, self.d, self.dense, self.bytes = n.value, d.value, bool(dense.value), nbytes.value

    def solve_many(self, inst_rows, inst_y, params):
        ptr = np.zeros(len(inst_rows) + 1, dtype=np.int32)
        ptr[1:] = np.cumsum([len(r) for r in inst_rows])
        rows = np.ascontiguousarray(np.concatenate(inst_rows), dtype=np.int32)
        ys = np.ascontiguousarray(np.concatenate(inst_y), dtype=np.float64)
        prm = (SvmbParams * len(params))(*params)
        alpha = np.zeros(max(int(ptr[-1]), 1))
        st = (SolveStats * len(params))()
        rc = self.eng.lib.svmb_rows_solve_many(self.h, len(params), ptr.ctypes.data, rows.ctypes.data, ys.ctypes.data,
                                               prm, alpha.ctypes.data, st)
        self.eng._ok(rc, "svmb_rows_solve_many")
        return [alpha[ptr[k]:ptr[k + 1]] for k in range(len(params))], [s.as_dict() for s in st]

    def kernel_block(self, ia, ib, params: SvmbParams) -> np.ndarray:
        """K(x_ia[i], x_ib[j]) as a float64 [len(ia)][len(ib)] array (svmb_rows_kernel_block)."""
        ia = np.ascontiguousarray(ia, dtype=np.int32)
        ib = np.ascontiguousarray(ib, dtype=np.int32)
        out = np.zeros((len(ia), len(ib)))
        rc = self.eng.lib.svmb_rows_kernel_block(self.h, C.byref(params), len(ia), ia.ctypes.data, len(ib),
                                                 ib.ctypes.data, out.ctypes.data)
        self.eng._ok(rc, "svmb_rows_kernel_block")
        return out

    def free(self):
        if self.h:
            self.eng.lib.svmb_rows_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """Request loop (svmb_server_*): submitted binary solves are batched
    continuously onto the GPU; wait(ticket) returns (signed alpha, stats, latency)."""

    def __init__(self, eng: Engine, mem_bytes: int = 0, max_inflight: int = 0, max_batch: int = 0, form: int = 0,
                 policy: int = 0, rows_per_block: int = 0):
        self.eng = eng
        self.h = None
        cfg = ServerConfig(mem_bytes, max_inflight, max_batch, form, policy, rows_per_block)
        h = C.c_void_p()
        eng._ok(eng.lib.svmb_server_create(C.byref(cfg), C.byref(h)), "svmb_server_create")
        self.h = h
        self._n = {}

    def submit(self, p: CSR, params: SvmbParams, y: Optional[np.ndarray] = None) -> int:
        rp, col, val = csr_arrays(p)
        yy = np.ascontiguousarray(p.y if y is None else y, dtype=np.float64)
        t = self.eng.lib.svmb_server_submit(self.h, p.n, p.d, rp.ctypes.data, col.ctypes.data, val.ctypes.data,
                                            yy.ctypes.data, C.byref(params))
        if t < 0:
            raise EngineError(f"svmb_server_submit: {self.eng.error()}")
        self._n[t] = p.n
        return t

    def done(self, ticket: int) -> bool:
        return self.eng.lib.svmb_server_poll(self.h, ticket) == 1

    def wait(self, ticket: int):
        n = self._n.pop(ticket)
        alpha = np.zeros(n)
        st = SolveStats()
        lat = C.c_double()
        self.eng._ok(self.eng.lib.svmb_server_wait(self.h, ticket, alpha.ctypes.data, C.byref(st), C.byref(lat)),
                     "svmb_server_wait")
        return alpha, st.as_dict(), lat.value

    def stats(self) -> dict:
        s = ServerStats()
        self.eng._ok(self.eng.lib.svmb_server_get_stats(self.h, C.byref(s)), "svmb_server_get_stats")
        return s.as_dict()

    def close(self):
        if self.h:
            self.eng.lib.svmb_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
