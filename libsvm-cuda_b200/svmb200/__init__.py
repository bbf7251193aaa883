"""Python bindings of the B200 SVM engine (libsvm_b200.so, include/svm.h + include/svm_b200.h).

The shared library is the product; this package only marshals arguments.  It
never falls back to another implementation: if the library or a GPU is
missing, calls raise EngineError.
"""
from .datagen import CSR  # noqa: F401
from .lib import Engine, EngineError, SolveStats  # noqa: F401
