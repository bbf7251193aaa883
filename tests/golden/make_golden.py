"""Regenerate the golden fixtures from the reference's own CPU solver.

Requires oracle/_ref/ref_dump and ref_dump_fp64 (built by `make -C oracle ref`
from the reference sources).  For each case in cases.py this writes
  <case>.ref.txt    output of the stock reference (float Q cache)
  <case>.fp64.txt   output of the reference with `typedef double Qfloat`
  <case>.sha256     checksum of the generated input text
Run:  python tests/golden/make_golden.py [case ...]
"""
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import cases  # noqa: E402

REF = os.path.join(cases.ROOT, "oracle", "_ref")


def run(binary, opts, trp, tep, mode):
    args = [os.path.join(REF, binary)]
    if mode.startswith("cv:"):
        args += ["-v", mode[3:]]
    args += opts.split() + [trp] + ([tep] if tep else [])
    return subprocess.run(args, check=True, capture_output=True, text=True).stdout


def main(names):
    names = names or list(cases.CASES)
    with tempfile.TemporaryDirectory() as td:
        for name in names:
            trp, tep, opts, mode, sha = cases.materialise(name, td)
            for binary, suffix in (("ref_dump", "ref"), ("ref_dump_fp64", "fp64")):
                out = run(binary, opts, trp, tep, mode)
                with open(os.path.join(HERE, f"{name}.{suffix}.txt"), "w") as f:
                    f.write(out)
            with open(os.path.join(HERE, f"{name}.sha256"), "w") as f:
                f.write(sha + "\n")
            print(name, "ok")


if __name__ == "__main__":
    main(sys.argv[1:])
