"""Shared test helpers: svm-train option strings -> svm_parameter, golden loading."""
import os

import numpy as np

from svmb200 import cabi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def param_from_opts(opts: str, d: int, cuda_flag: int = 1) -> cabi.svm_parameter:
    """Parse svm-train options (reference svm-train.c:162-284) into svm_parameter."""
    kw = dict(svm_type=0, kernel_type=2, degree=3, gamma=0.0, coef0=0.0, cache_size=100.0, eps=1e-3, C_=1.0,
              nu=0.5, p=0.1, shrinking=1, probability=0)
    weights = {}
    toks = opts.split()
    i = 0
    names = {"s": "svm_type", "t": "kernel_type", "d": "degree", "g": "gamma", "r": "coef0", "m": "cache_size",
             "e": "eps", "c": "C_", "n": "nu", "p": "p", "h": "shrinking", "b": "probability"}
    while i < len(toks):
        t = toks[i]
        if t[1] == "w":
            weights[int(t[2:])] = float(toks[i + 1])
        else:
            k = names[t[1]]
            kw[k] = type(kw[k])(float(toks[i + 1])) if isinstance(kw[k], float) else int(toks[i + 1])
        i += 2
    if kw["gamma"] == 0 and d > 0:
        kw["gamma"] = 1.0 / d
    return cabi.make_param(weights=weights or None, cuda_flag=cuda_flag, **kw)


def load_golden(name: str, suffix: str = "ref") -> dict:
    import oracle_py
    with open(os.path.join(GOLDEN, f"{name}.{suffix}.txt")) as f:
        return oracle_py.parse_dump(f.read())


def max_index(p) -> int:
    return int(p.indices.max()) if p.nnz else 0
