"""The C-ABI library loads and exports every function include/kfb.h declares
(no device calls: runs without a GPU)."""
import os
import re

from kernelforge_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "kfb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(kfb_[a-z0-9_]+)\s*\(", src)))


def test_header_and_binding_agree():
    names = declared_functions()
    assert names, "no declarations parsed"
    assert sorted(_lib.EXPORTS) == names


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.kfb_abi_version() == 1


def test_library_is_sm100a_only():
    # the build compiles for sm_100a only (no PTX for other targets)
    from kernelforge_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
