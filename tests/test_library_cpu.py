"""CPU tests of the C ABI: libdgq.so loads and exports every function that
include/QuEST.h and include/dgq.h declare (no GPU calls are made)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("QuEST.h", "dgq.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_headers_declare_the_required_api():
    names = declared_functions()
    required = {"createQuESTEnv", "destroyQuESTEnv", "createQureg", "destroyQureg", "initZeroState", "hadamard",
                "controlledNot", "controlledPhaseShift", "rotateX", "rotateY", "rotateZ", "compactUnitary",
                "multiQubitUnitary", "calcProbOfOutcome", "measure", "getAmp", "seedQuEST",
                "searchQuregTaskPartitions", "controlledPhaseFlip", "pauliX", "pauliZ", "SqX", "SqY", "SqW",
                "unitary", "swapGate"}
    assert required <= names, required - names


def test_library_exports_every_declared_symbol():
    from dgquest_b200 import library_path, load_library
    assert os.path.exists(library_path)
    lib = load_library()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_symbol():
    from dgquest_b200 import quest
    lib = quest._library()
    for name in declared_functions():
        assert hasattr(quest, name), name
    assert lib.getQuEST_PREC() == 2
