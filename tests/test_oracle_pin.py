"""The oracle restatement (oracle/svm_oracle.c) against the reference's own
CPU solver: the committed golden outputs were produced by oracle/_ref/ref_dump
(built from the reference sources); the restatement must reproduce them
exactly, for the stock float-Q build and for the FP64-Q build."""
import os
import subprocess
import tempfile

import pytest

import cases

ORACLE = os.path.join(cases.ROOT, "oracle", "_build")


def run_dump(binary, trp, tep, opts, mode):
    args = [os.path.join(ORACLE, binary)]
    if mode.startswith("cv:"):
        args += ["-v", mode[3:]]
    args += opts.split() + [trp] + ([tep] if tep else [])
    return subprocess.run(args, check=True, capture_output=True, text=True, timeout=120).stdout


@pytest.mark.parametrize("name", [k for k in cases.FAST if k not in cases.REFERENCE_ONLY] + ["rbf_dense_c1"])
def test_restatement_matches_reference(name):
    with tempfile.TemporaryDirectory() as td:
        trp, tep, opts, mode, sha = cases.materialise(name, td)
        with open(os.path.join(cases.HERE, f"{name}.sha256")) as f:
            assert f.read().strip() == sha, "generated input drifted from the golden input"
        for binary, suffix in (("oracle_dump", "ref"), ("oracle_dump_fp64", "fp64")):
            out = run_dump(binary, trp, tep, opts, mode)
            with open(os.path.join(cases.HERE, f"{name}.{suffix}.txt")) as f:
                gold = f.read()
            assert out == gold, f"{binary} differs from the reference on {name}"


@pytest.mark.parametrize("name", [k for k in cases.CASES if k in cases.REFERENCE_ONLY or k.endswith("_wide")])
def test_golden_inputs_unchanged(name):
    """Cases pinned on the reference's outputs alone: the seeded inputs that
    the GPU tests regenerate are still the ones the reference ran on."""
    with tempfile.TemporaryDirectory() as td:
        sha = cases.materialise(name, td)[4]
    with open(os.path.join(cases.HERE, f"{name}.sha256")) as f:
        assert f.read().strip() == sha


def test_reference_rebuild_agrees_if_present():
    """When the reference build is present, it still reproduces a golden file."""
    ref = os.path.join(cases.ROOT, "oracle", "_ref", "ref_dump")
    if not os.path.exists(ref):
        pytest.skip("oracle/_ref not built")
    with tempfile.TemporaryDirectory() as td:
        trp, tep, opts, mode, sha = cases.materialise("rbf_dense_small", td)
        out = subprocess.run([ref] + opts.split() + [trp, tep], check=True, capture_output=True, text=True).stdout
        with open(os.path.join(cases.HERE, "rbf_dense_small.ref.txt")) as f:
            assert out == f.read()
