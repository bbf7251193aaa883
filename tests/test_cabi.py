"""CPU checks of the drop-in boundary: the library loads, exports every
function include/*.h declares, has the reference's structure layout, and its
host-only functions (parameter check, model file I/O) behave exactly like the
reference's (oracle/_ref/libsvm_ref.so, built from the reference sources)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import cases
from helpers import param_from_opts, max_index
from svmb200 import cabi
from svmb200.lib import LIB_PATH, CLI_PATH, Engine

INCLUDE = os.path.join(cases.ROOT, "include")


def declared_functions():
    names = []
    for h in ("svm.h", "svm_b200.h"):
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[\w\s\*]*?\b(svm\w*|svmb\w*)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB_PATH), "libsvm_b200.so not built"
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    want = declared_functions()
    assert len(want) >= 30
    missing = [n for n in want if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    assert "libsvm_version" in exported
    lib = C.CDLL(LIB_PATH)
    assert C.c_int.in_dll(lib, "libsvm_version").value == 318


def test_struct_layout_matches_reference_abi():
    # offsets of the reference's structures (libsvm/svm.h:31-92, x86-64)
    src = r'''
    #include <stddef.h>
    #include <stdio.h>
    #include "svm.h"
    int main(void){
      printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(struct svm_node), sizeof(struct svm_problem),
        sizeof(struct svm_parameter), sizeof(struct svm_model), offsetof(struct svm_parameter, svm_type),
        offsetof(struct svm_parameter, shrinking), offsetof(struct svm_model, nr_class), offsetof(struct svm_model, free_sv));
      return 0; }'''
    ref_inc = os.path.join(os.environ.get("LIBSVM_REFERENCE", "/root/reference"), "libsvm")
    with tempfile.TemporaryDirectory() as td:
        res = {}
        for tag, inc in (("ours", INCLUDE), ("ref", ref_inc)):
            if tag == "ref" and not os.path.exists(os.path.join(ref_inc, "svm.h")):
                continue
            c = os.path.join(td, f"{tag}.c")
            open(c, "w").write(src)
            exe = os.path.join(td, tag)
            subprocess.run(["gcc", "-I", inc, c, "-o", exe], check=True)
            res[tag] = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
        if "ref" in res:
            assert res["ours"] == res["ref"]
        vals = [int(v) for v in res["ours"].split()]
        assert vals[:4] == [C.sizeof(cabi.svm_node), C.sizeof(cabi.svm_problem), C.sizeof(cabi.svm_parameter),
                            C.sizeof(cabi.svm_model)]


CHECK_CASES = [
    ("-s 0 -c 0", "C <= 0"), ("-s 1 -n 0", "nu <= 0 or nu > 1"), ("-s 1 -n 1.5", "nu <= 0 or nu > 1"),
    ("-s 9", "unknown svm type"), ("-t 7", "unknown kernel type"), ("-g -1", "gamma < 0"),
    ("-d -2", "degree of polynomial kernel < 0"), ("-m 0", "cache_size <= 0"), ("-e 0", "eps <= 0"),
    ("-h 2", "shrinking != 0 and shrinking != 1"), ("-b 3", "probability != 0 and probability != 1"),
    ("-s 2 -b 1", "one-class SVM probability output not supported yet"), ("-s 1 -n 0.99", "specified nu is infeasible"),
    ("-s 0 -c 1", None), ("-s 1 -n 0.2", None),
]


@pytest.mark.parametrize("opts,msg", CHECK_CASES)
def test_check_parameter_messages(opts, msg):
    import oracle_py
    tr, _ = cases.CASES["rbf_dense_small"][0]()
    # an unbalanced problem makes large nu infeasible
    tr.y[:200] = 1.0
    eng = Engine()
    prm = param_from_opts(opts, max_index(tr))
    assert eng.check_parameter(tr, prm) == msg
    ref = oracle_py.reference_lib()
    if ref is not None:
        rows = cabi.NodeRows(tr)
        r = ref.svm_check_parameter(C.byref(rows.prob), C.byref(prm))
        assert (r.decode() if r else None) == msg


def test_model_file_roundtrip_matches_reference_format(oracle):
    """svm_save_model writes the reference's format byte for byte; svm_load_model reads it back."""
    import oracle_py
    tr, _ = cases.CASES["multiclass_rbf"][0]()
    prm = param_from_opts(cases.CASES["multiclass_rbf"][1], max_index(tr))
    m, rows, arrays, _ = oracle.train(tr, prm)
    eng = Engine()
    with tempfile.TemporaryDirectory() as td:
        ours = os.path.join(td, "ours.model")
        assert eng.lib.svm_save_model(ours.encode(), m) == 0
        ref = oracle_py.reference_lib()
        if ref is not None:
            theirs = os.path.join(td, "ref.model")
            assert ref.svm_save_model(theirs.encode(), m) == 0
            assert open(ours).read() == open(theirs).read()
        loaded = eng.lib.svm_load_model(ours.encode())
        assert loaded
        a = cabi.model_arrays(loaded.contents)
        assert a["nr_class"] == arrays["nr_class"] and a["total_sv"] == arrays["total_sv"]
        assert np.array_equal(a["nsv"], arrays["nsv"]) and np.array_equal(a["labels"], arrays["labels"])
        np.testing.assert_allclose(a["sv_coef"], arrays["sv_coef"], rtol=1e-15, atol=0)
        np.testing.assert_allclose(a["rho"], arrays["rho"], rtol=1e-5)
        assert loaded.contents.free_sv == 1
        eng.lib.svm_free_and_destroy_model(C.byref(loaded))
    oracle.free(m)


def test_cli_usage_without_gpu():
    r = subprocess.run([CLI_PATH], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage: svm-train" in r.stdout


def test_no_gpu_fails_loudly_not_silently():
    """Without a device the engine refuses to train (no CPU fallback)."""
    eng = Engine()
    if eng.available():
        pytest.skip("a GPU is present")
    tr, _ = cases.CASES["rbf_dense_small"][0]()
    prm = param_from_opts("-c 1", max_index(tr))
    with pytest.raises(Exception):
        eng.train(tr, prm)
