"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the oracle restatement
(oracle/_build/libsvm_oracle*.so, see svm_oracle.h) and of the reference's own
CPU build (oracle/_ref/libsvm_ref.so).  Only tests/, __graft_entry__.smoke()
and bench.py's cpu_baseline leg may import this module."""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "libsvm-cuda_b200"))

from svmb200 import cabi  # noqa: E402
from svmb200.cabi import NodeRows, svm_model, svm_parameter, svm_problem  # noqa: E402

_P = C.POINTER


class SolveInfo(C.Structure):
    _fields_ = [("iters", C.c_longlong), ("obj", C.c_double), ("rho", C.c_double), ("r", C.c_double),
                ("l", C.c_int), ("nr_free", C.c_int), ("nr_sv", C.c_int)]


class Oracle:
    """The C restatement; fp64=True loads the double-Q build (the FP64 oracle)."""

    def __init__(self, fp64: bool = False):
        name = "libsvm_oracle_fp64.so" if fp64 else "libsvm_oracle.so"
        path = os.path.join(HERE, "_build", name)
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle oracle`")
        lib = C.CDLL(path)
        lib.oracle_svm_train.restype = _P(svm_model)
        lib.oracle_svm_train.argtypes = [_P(svm_problem), _P(svm_parameter)]
        lib.oracle_cross_validation.argtypes = [_P(svm_problem), _P(svm_parameter), C.c_int, _P(C.c_double)]
        lib.oracle_predict_values.restype = C.c_double
        lib.oracle_predict_values.argtypes = [_P(svm_model), _P(cabi.svm_node), _P(C.c_double)]
        lib.oracle_free_model.argtypes = [_P(svm_model)]
        lib.oracle_solve_binary.argtypes = [_P(svm_problem), _P(svm_parameter), C.c_double, C.c_double,
                                            _P(C.c_double), _P(SolveInfo)]
        lib.oracle_solve_get.argtypes = [C.c_int, _P(SolveInfo)]
        lib.oracle_srand.argtypes = [C.c_uint]
        self.lib = lib

    def train(self, p, param):
        rows = NodeRows(p)
        m = self.lib.oracle_svm_train(C.byref(rows.prob), C.byref(param))
        arrays = cabi.model_arrays(m.contents)
        infos = self.infos()
        return m, rows, arrays, infos

    def infos(self):
        out = []
        for k in range(self.lib.oracle_solve_count()):
            s = SolveInfo()
            self.lib.oracle_solve_get(k, C.byref(s))
            out.append({f: getattr(s, f) for f, _ in SolveInfo._fields_})
        return out

    def predict(self, m, p):
        rows = NodeRows(p)
        k = m.contents.nr_class
        npair = max(k * (k - 1) // 2, 1)
        lab = np.zeros(p.n)
        dec = np.zeros((p.n, npair))
        for i in range(p.n):
            lab[i] = self.lib.oracle_predict_values(m, rows.row(i), dec[i].ctypes.data_as(_P(C.c_double)))
        return lab, dec[:, :k * (k - 1) // 2]

    def solve_binary(self, p, param, Cp, Cn):
        rows = NodeRows(p)
        alpha = np.zeros(max(p.n, 1))
        s = SolveInfo()
        self.lib.oracle_solve_binary(C.byref(rows.prob), C.byref(param), Cp, Cn,
                                     alpha.ctypes.data_as(_P(C.c_double)), C.byref(s))
        return alpha[:p.n], {f: getattr(s, f) for f, _ in SolveInfo._fields_}

    def cross_validation(self, p, param, nfold, seed=1):
        rows = NodeRows(p)
        self.lib.oracle_srand(seed)
        out = np.zeros(max(p.n, 1))
        self.lib.oracle_cross_validation(C.byref(rows.prob), C.byref(param), nfold, out.ctypes.data_as(_P(C.c_double)))
        return out[:p.n], self.infos()

    def free(self, m):
        self.lib.oracle_free_model(m)


def reference_lib():
    """The reference's own CPU solver as a shared library (oracle/_ref/libsvm_ref.so)."""
    path = os.path.join(HERE, "_ref", "libsvm_ref.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.svm_train.restype = _P(svm_model)
    lib.svm_train.argtypes = [_P(svm_problem), _P(svm_parameter)]
    lib.svm_check_parameter.restype = C.c_char_p
    lib.svm_check_parameter.argtypes = [_P(svm_problem), _P(svm_parameter)]
    lib.svm_save_model.argtypes = [C.c_char_p, _P(svm_model)]
    lib.svm_load_model.restype = _P(svm_model)
    lib.svm_load_model.argtypes = [C.c_char_p]
    lib.svm_set_print_string_function.argtypes = [cabi.PRINT_FUNC]
    lib.svm_free_and_destroy_model.argtypes = [_P(_P(svm_model))]
    return lib


def parse_dump(text: str) -> dict:
    """Parse ref_dump / oracle_dump output into arrays."""
    out = {"iter": [], "obj": [], "dec": [], "cv": [], "sv_coef": [], "prob": []}
    for line in text.splitlines():
        parts = line.split()
        if not parts:
            continue
        key = parts[0]
        if key in ("nr_class", "total_sv"):
            out[key] = int(parts[1])
        elif key in ("labels", "nsv", "sv_indices"):
            out[key] = np.array([int(v) for v in parts[1:]], dtype=np.int64)
        elif key in ("rho", "probA", "probB"):
            out[key] = np.array([float(v) for v in parts[1:]])
        elif key == "prob":
            out["prob"].append([float(v) for v in parts[2:]])
        elif key == "sv_coef":
            out["sv_coef"].append(np.array([float(v) for v in parts[2:]]))
        elif key == "iter":
            out["iter"].append(int(parts[2]))
        elif key == "obj":
            out["obj"].append(float(parts[2]))
        elif key == "dec":
            out["dec"].append([float(v) for v in parts[2:]])
        elif key == "cv":
            out["cv"].append(float(parts[2]))
        elif key == "error":
            out["error"] = " ".join(parts[1:])
    out["sv_coef"] = np.array(out["sv_coef"]) if out["sv_coef"] else np.zeros((0, 0))
    if out["prob"]:
        pr = np.array(out["prob"])
        out["prob_pred"] = pr[:, 0]
        out["prob"] = pr[:, 1:]
    if out["dec"]:
        d = np.array(out["dec"])
        out["pred"] = d[:, 0]
        out["dec"] = d[:, 1:]
    return out
