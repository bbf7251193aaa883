"""The svm-train / svm-predict commands and the parallel text parser.

CPU tests: usage text, option errors and malformed-input messages (with exit
codes) equal those of the reference's own svm-train (oracle/_ref/svm-train,
built from the reference sources), and svmb_read_problem returns exactly the
rows a strict parse of the file gives, on files large enough to be cut into
one range per thread.

GPU tests: model files written by our svm-train equal, byte for byte, those of
the reference's svm-train on the golden inputs; cross-validation reports are
the same lines; svm-predict's output equals a reference-side harness
(oracle/_ref/ref_predict, the reference's svm_predict* row by row): the same
labels, and values within a few units in the last place (the device's double
exp and glibc's are not both correctly rounded)."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

import cases
from svmb200 import datagen
from svmb200.cabi import svm_node, svm_problem
from svmb200.lib import PKG_DIR

OUR_TRAIN = os.path.join(PKG_DIR, "svm-train")
OUR_PREDICT = os.path.join(PKG_DIR, "svm-predict")
REF_DIR = os.path.join(cases.ROOT, "oracle", "_ref")
REF_TRAIN = os.path.join(REF_DIR, "svm-train")
REF_PREDICT = os.path.join(REF_DIR, "ref_predict")

need_ref = pytest.mark.skipif(not os.path.exists(REF_TRAIN), reason="oracle/_ref not built")


def run(args, cwd=None):
    r = subprocess.run(args, capture_output=True, cwd=cwd, timeout=600)
    return r.returncode, r.stdout, r.stderr


MALFORMED = {
    "empty_line": "1 1:0.5\n\n-1 2:0.25\n",
    "blank_line": "1 1:0.5\n   \t \n",
    "unsorted_index": "1 1:0.5 3:0.1 2:0.2\n",
    "repeated_index": "1 2:0.5 2:0.1\n",
    "label_not_number": "abc 1:0.5\n",
    "label_trailing": "1.5x 1:0.5\n",
    "value_not_number": "1 1:abc\n",
    "value_trailing": "1 1:0.5x\n",
    "index_trailing": "1 1x:0.5\n",
    "index_space": "1 1 :0.5\n",
    "negative_index": "1 -1:0.5\n",
    "value_overflow": "1 1:1e400\n",
    "missing_value": "1 1:0.5 2:\n",
    "crlf_label_only": "1\r\n",
    "late_error": "".join(f"{1 if i % 2 else -1} 1:{i * 0.001} 2:0.5\n" for i in range(40000)) + "1 2:0.5 1:0.3\n",
}


@need_ref
@pytest.mark.parametrize("name", sorted(MALFORMED))
def test_malformed_input_reported_like_the_reference(name):
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "train.txt")
        with open(path, "w", newline="") as f:
            f.write(MALFORMED[name])
        ours = run([OUR_TRAIN, "-q", path, os.path.join(td, "m1")])
        ref = run([REF_TRAIN, "-q", path, os.path.join(td, "m2")])
    assert ours == ref


ACCEPTED_BUT_INVALID = {
    # parses (trailing text without ':' is ignored, index 0 allowed, CRLF,
    # tabs, a ':' without an index skipped), then svm_check_parameter refuses nu
    "lenient_forms": "+1 0:1 1:0.5 junk\r\n-1\t2:-2.5e-1\t \n1 3:1 :7\n",
}


@need_ref
@pytest.mark.parametrize("name", sorted(ACCEPTED_BUT_INVALID))
def test_accepted_forms_reach_the_parameter_check(name):
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "train.txt")
        with open(path, "w", newline="") as f:
            f.write(ACCEPTED_BUT_INVALID[name])
        ours = run([OUR_TRAIN, "-s", "1", "-n", "2", path, os.path.join(td, "m1")])
        ref = run([REF_TRAIN, "-s", "1", "-n", "2", path, os.path.join(td, "m2")])
    assert ours == ref
    assert b"nu <= 0 or nu > 1" in ours[2]


@need_ref
@pytest.mark.parametrize("args", [[], ["-q"], ["-z", "1", "f"], ["-v", "1", "f"], ["-c"], ["/nonexistent/file"],
                                  ["-q", "-s"]])
def test_usage_and_option_errors_like_the_reference(args):
    with tempfile.TemporaryDirectory() as td:
        assert run([OUR_TRAIN] + args, cwd=td) == run([REF_TRAIN] + args, cwd=td)


def _lib():
    lib = C.CDLL(os.path.join(PKG_DIR, "libsvm_b200.so"))
    lib.svmb_read_problem.argtypes = [C.c_char_p, C.POINTER(svm_problem), C.POINTER(C.POINTER(svm_node)),
                                      C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
    lib.svmb_free_problem.argtypes = [C.POINTER(svm_problem), C.POINTER(svm_node)]
    return lib


def _strict_parse(text):
    """Rows of a well-formed file as (label, [(index, value)])."""
    rows = []
    for line in text.splitlines():
        toks = line.split()
        rows.append((float(toks[0]), [(int(t.split(":")[0]), float(t.split(":")[1])) for t in toks[1:]]))
    return rows


@pytest.mark.parametrize("nrows", [50, 60000])
def test_parser_returns_the_file_rows(nrows):
    """Values are strtod numbers (bit-exact); the large file is parsed by many
    threads and must come back in file order."""
    rng = np.random.default_rng(nrows)
    lines = []
    for i in range(nrows):
        k = int(rng.integers(0, 6))
        idx = np.sort(rng.choice(40, size=k, replace=False)) + (i % 2)
        vals = rng.standard_normal(k) * 10.0 ** rng.integers(-5, 5, size=k)
        fmt = ["{!r}", "{:.3e}", "{:+.6f}"][i % 3]
        feats = " ".join(f"{j}:{fmt.format(float(v))}" for j, v in zip(idx, vals))
        lines.append(f"{(-1) ** i * (i % 7)} {feats}".rstrip() + ("  \n" if i % 5 == 0 else "\n"))
    text = "".join(lines)
    lib = _lib()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "f.txt")
        with open(path, "w") as f:
            f.write(text)
        prob = svm_problem()
        space = C.POINTER(svm_node)()
        maxi, bad = C.c_int(), C.c_longlong()
        assert lib.svmb_read_problem(path.encode(), C.byref(prob), C.byref(space), C.byref(maxi), C.byref(bad)) == 0
    want = _strict_parse(text)
    assert prob.l == len(want)
    assert maxi.value == max((r[1][-1][0] for r in want if r[1]), default=0)
    for i in range(prob.l):
        lab, feats = want[i]
        assert prob.y[i] == lab
        got = []
        j = 0
        while prob.x[i][j].index != -1:
            got.append((prob.x[i][j].index, prob.x[i][j].value))
            j += 1
        assert got == feats, i
    lib.svmb_free_problem(C.byref(prob), space)


# ---------------------------------------------------------------- GPU ------

MODEL_CASES = ["rbf_dense_small", "multiclass_rbf", "nu_rbf_dense", "weighted_rbf", "rbf_sparse",
               "prob_multiclass_rbf", "eps_svr_rbf", "nu_svr_rbf", "one_class_rbf", "prob_svr"]


@need_ref
@pytest.mark.gpu
@pytest.mark.parametrize("name", MODEL_CASES)
def test_model_file_identical_to_reference_svm_train(name):
    with tempfile.TemporaryDirectory() as td:
        trp, tep, opts, mode, _ = cases.materialise(name, td)
        ours, ref = os.path.join(td, "ours.model"), os.path.join(td, "ref.model")
        rc, out, err = run([OUR_TRAIN, "-q"] + opts.split() + [trp, ours])
        assert rc == 0, err
        rc, _, err = run([REF_TRAIN, "-q"] + opts.split() + [trp, ref])
        assert rc == 0, err
        assert open(ours, "rb").read() == open(ref, "rb").read()


@need_ref
@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cv_multiclass", "cv_svr", "cv_prob_multiclass"])
def test_cross_validation_report_identical(name):
    with tempfile.TemporaryDirectory() as td:
        trp, _, opts, mode, _ = cases.materialise(name, td)
        args = ["-q", "-v", mode[3:]] + opts.split() + [trp]
        rc1, out1, err1 = run([OUR_TRAIN] + args)
        rc2, out2, err2 = run([REF_TRAIN] + args)
    assert rc1 == rc2 == 0, (err1, err2)
    assert out1 == out2


@need_ref
@pytest.mark.gpu
@pytest.mark.parametrize("name,prob", [("multiclass_rbf", 0), ("prob_multiclass_rbf", 1), ("prob_binary_rbf", 1),
                                       ("eps_svr_rbf", 0), ("one_class_rbf", 0), ("rbf_sparse", 0)])
def test_svm_predict_output_identical_to_reference(name, prob):
    """Both predict from the model file the reference's svm-train wrote."""
    with tempfile.TemporaryDirectory() as td:
        trp, tep, opts, mode, _ = cases.materialise(name, td)
        model = os.path.join(td, "ref.model")
        rc, _, err = run([REF_TRAIN, "-q"] + opts.split() + [trp, model])
        assert rc == 0, err
        o1, o2 = os.path.join(td, "ours.out"), os.path.join(td, "ref.out")
        rc, out, err = run([OUR_PREDICT, "-b", str(prob), tep, model, o1])
        assert rc == 0, err
        assert (b"Accuracy = " in out) or (b"Mean squared error" in out)
        rc, _, err = run([REF_PREDICT, "-b", str(prob), tep, model, o2])
        assert rc == 0, err
        a, b = open(o1).read().splitlines(), open(o2).read().splitlines()
        assert len(a) == len(b)
        if prob:
            assert a[0] == b[0]                       # the "labels ..." header
            a, b = a[1:], b[1:]
        ours = np.array([[float(v) for v in line.split()] for line in a])
        ref = np.array([[float(v) for v in line.split()] for line in b])
        if not name.startswith("eps_svr"):
            assert np.array_equal(ours[:, 0], ref[:, 0]), "labels differ"
        # kernel values are float64 exp() of the same argument; the device's
        # exp and glibc's may differ in the last bit, so values agree to a
        # few units in the last place, not always bit for bit
        np.testing.assert_allclose(ours, ref, rtol=1e-13, atol=1e-15)
