"""ctypes mirrors of the svm.h structures (include/svm.h) and helpers that
turn CSR arrays into svm_problem / svm_node rows without copying per element.

The layouts must match include/svm.h exactly (they are the reference's ABI,
reference libsvm/svm.h:31-92); test_cabi.py checks the sizes and offsets
against the compiled library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .datagen import CSR

NODE_DTYPE = np.dtype([("index", "<i4"), ("pad", "<i4"), ("value", "<f8")])
assert NODE_DTYPE.itemsize == 16

C_SVC, NU_SVC, ONE_CLASS, EPSILON_SVR, NU_SVR = range(5)
LINEAR, POLY, RBF, SIGMOID, PRECOMPUTED = range(5)


class svm_node(C.Structure):
    _fields_ = [("index", C.c_int), ("value", C.c_double)]


class svm_problem(C.Structure):
    _fields_ = [("l", C.c_int), ("y", C.POINTER(C.c_double)), ("x", C.POINTER(C.POINTER(svm_node)))]


class svm_parameter(C.Structure):
    _fields_ = [
        ("cuda_flag", C.c_int), ("svm_type", C.c_int), ("kernel_type", C.c_int), ("degree", C.c_int),
        ("gamma", C.c_double), ("coef0", C.c_double), ("cache_size", C.c_double), ("eps", C.c_double),
        ("C", C.c_double), ("nr_weight", C.c_int), ("weight_label", C.POINTER(C.c_int)),
        ("weight", C.POINTER(C.c_double)), ("nu", C.c_double), ("p", C.c_double),
        ("shrinking", C.c_int), ("probability", C.c_int),
    ]


class svm_model(C.Structure):
    _fields_ = [
        ("param", svm_parameter), ("nr_class", C.c_int), ("l", C.c_int),
        ("SV", C.POINTER(C.POINTER(svm_node))), ("sv_coef", C.POINTER(C.POINTER(C.c_double))),
        ("rho", C.POINTER(C.c_double)), ("probA", C.POINTER(C.c_double)), ("probB", C.POINTER(C.c_double)),
        ("sv_indices", C.POINTER(C.c_int)), ("label", C.POINTER(C.c_int)), ("nSV", C.POINTER(C.c_int)),
        ("free_sv", C.c_int),
    ]


PRINT_FUNC = C.CFUNCTYPE(None, C.c_char_p)


def make_param(svm_type=C_SVC, kernel_type=RBF, degree=3, gamma=0.0, coef0=0.0, cache_size=100.0,
               eps=1e-3, C_=1.0, nu=0.5, p=0.1, shrinking=1, probability=0, weights=None,
               cuda_flag=1) -> svm_parameter:
    """svm_parameter with the svm-train defaults (reference svm-train.c:167-181)."""
    prm = svm_parameter()
    prm.cuda_flag = cuda_flag
    prm.svm_type = svm_type
    prm.kernel_type = kernel_type
    prm.degree = degree
    prm.gamma = gamma
    prm.coef0 = coef0
    prm.cache_size = cache_size
    prm.eps = eps
    prm.C = C_
    prm.nu = nu
    prm.p = p
    prm.shrinking = shrinking
    prm.probability = probability
    if weights:
        labs = (C.c_int * len(weights))(*[int(k) for k in weights])
        vals = (C.c_double * len(weights))(*[float(v) for v in weights.values()])
        prm.nr_weight = len(weights)
        prm.weight_label = C.cast(labs, C.POINTER(C.c_int))
        prm.weight = C.cast(vals, C.POINTER(C.c_double))
        prm._keep = (labs, vals)
    else:
        prm.nr_weight = 0
    return prm


class NodeRows:
    """svm_node rows of a CSR problem, each terminated by index -1.

    `ptrs` is a (svm_node*)[n] array pointing into one contiguous buffer; the
    object owns every buffer, so keep it alive while C code holds pointers."""

    def __init__(self, p: CSR):
        n = p.n
        lens = np.diff(p.indptr)
        total = int(p.nnz + n)
        buf = np.zeros(total, dtype=NODE_DTYPE)
        starts = (p.indptr[:-1] + np.arange(n)).astype(np.int64)
        ends = starts + lens
        # position of each nonzero in the node buffer
        rows = np.repeat(np.arange(n), lens)
        pos = np.arange(p.nnz) + rows
        buf["index"][pos] = p.indices
        buf["value"][pos] = p.values
        buf["index"][ends] = -1
        self.buf = buf
        self.n = n
        base = buf.ctypes.data
        addrs = (base + starts * 16).astype(np.uint64)
        self.addrs = addrs
        self.ptrs = (C.POINTER(svm_node) * max(n, 1)).from_address(addrs.ctypes.data) if n else None
        self.y = np.ascontiguousarray(p.y, dtype=np.float64)
        self.prob = svm_problem()
        self.prob.l = n
        self.prob.y = self.y.ctypes.data_as(C.POINTER(C.c_double))
        self.prob.x = C.cast(addrs.ctypes.data, C.POINTER(C.POINTER(svm_node))) if n else None

    def row(self, i: int):
        return C.cast(C.c_void_p(int(self.addrs[i])), C.POINTER(svm_node))


def model_arrays(m: svm_model) -> dict:
    """Copy the numeric content of an svm_model into numpy arrays."""
    k = m.nr_class
    npair = k * (k - 1) // 2
    out = {
        "nr_class": k,
        "total_sv": m.l,
        "rho": np.array([m.rho[i] for i in range(npair)], dtype=np.float64),
        "labels": np.array([m.label[i] for i in range(k)], dtype=np.int64) if m.label else None,
        "nsv": np.array([m.nSV[i] for i in range(k)], dtype=np.int64) if m.nSV else None,
        "sv_indices": np.array([m.sv_indices[i] for i in range(m.l)], dtype=np.int64) if m.sv_indices else None,
        "probA": np.array([m.probA[i] for i in range(max(npair, 1) if m.probA else 0)], dtype=np.float64)
        if m.probA else None,
        "probB": np.array([m.probB[i] for i in range(max(npair, 1) if m.probB else 0)], dtype=np.float64)
        if m.probB else None,
    }
    coef = np.zeros((max(k - 1, 0), m.l), dtype=np.float64)
    for j in range(k - 1):
        coef[j] = np.ctypeslib.as_array(m.sv_coef[j], shape=(m.l,)) if m.l else 0
    out["sv_coef"] = coef
    return out
