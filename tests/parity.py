"""Comparison of an engine model with a reference dump (shared by GPU tests, smoke and bench)."""
import numpy as np


def coef_matrix(sv_indices, sv_coef, l):
    """Per-training-row coefficients (l x (k-1)), zero for non-SVs."""
    k1 = sv_coef.shape[0]
    out = np.zeros((l, max(k1, 1)))
    if len(sv_indices):
        out[np.asarray(sv_indices) - 1, :k1] = np.asarray(sv_coef).T
    return out


def compare_models(ours: dict, gold: dict, l: int) -> dict:
    """Differences between an engine model (cabi.model_arrays) and a parsed reference dump."""
    a = coef_matrix(ours["sv_indices"], ours["sv_coef"], l)
    b = coef_matrix(gold["sv_indices"], gold["sv_coef"], l)
    sv_a, sv_b = set(ours["sv_indices"].tolist()), set(gold["sv_indices"].tolist())
    return {
        "same_classes": ours["nr_class"] == gold["nr_class"] and (
            np.array_equal(ours["labels"], gold["labels"]) if "labels" in gold else ours["labels"] is None),
        "sv_sym_diff": sorted(sv_a ^ sv_b),
        "max_coef_diff": float(np.max(np.abs(a - b))) if a.size else 0.0,
        "coef_bit_equal": bool(np.array_equal(a, b)),
        "max_rho_diff": float(np.max(np.abs(ours["rho"] - gold["rho"]))) if len(gold["rho"]) else 0.0,
        "rho_bit_equal": bool(np.array_equal(ours["rho"], gold["rho"])),
    }
