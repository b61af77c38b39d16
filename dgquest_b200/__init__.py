"""dgquest_b200: a B200-native state-vector simulator behind the QuEST C API.

The product is the shared library ``libdgq.so`` built in this directory
(C++ host planner + sm_100a CUDA kernels, C ABI declared in
``include/QuEST.h`` and ``include/dgq.h``). This package loads it and
mirrors the QuEST API in Python (``dgquest_b200.quest``) for tests and
benchmarks. There is no CPU fallback: importing the bindings fails loudly
when the library is missing.
"""
import ctypes
import os

__all__ = ["lib", "library_path", "load_library"]

_HERE = os.path.dirname(os.path.abspath(__file__))
library_path = os.path.join(_HERE, "libdgq.so")
_lib = None


def load_library():
    """Loads libdgq.so (built in-tree by ``dgquest_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(library_path):
            raise ImportError(
                f"libdgq.so not found at {library_path}; build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'` or `make -C dgquest_b200`")
        _lib = ctypes.CDLL(library_path, mode=ctypes.RTLD_GLOBAL)
    return _lib


def __getattr__(name):
    if name == "lib":
        return load_library()
    raise AttributeError(name)
