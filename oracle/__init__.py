"""CPU oracle for the TCL4 L4(t) path -- test infrastructure only.

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package.  It wraps ``libtaco_oracle.so`` (a C++17 +
OpenMP restatement of the reference's CPU algorithm; see ``taco_oracle.h`` for
the parity status) with numpy-facing helpers.
"""
from .oracle import *  # noqa: F401,F403
