"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares (no compute calls)."""
import ctypes
import os
import re

import pytest

from ftspolysol_b200 import engine, host

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(ftsp_\w+)\s*\(", re.M)


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in sorted(os.listdir(inc)):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(inc, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)   # drop comments
        text = re.sub(r"typedef\s+struct\s+\w+\s*\{.*?\}\s*\w+\s*;", "", text, flags=re.S)
        names.update(DECL.findall(text))
    return sorted(names)


def test_headers_declare_the_known_entry_points():
    names = declared_functions()
    for n in engine.ABI_SYMBOLS + host.HOST_SYMBOLS:
        assert n in names, n
    assert len(names) == len(set(engine.ABI_SYMBOLS + host.HOST_SYMBOLS))


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports(name):
    if not os.path.exists(engine.library_path()):
        pytest.skip("libftsp.so not built")
    L = ctypes.CDLL(engine.library_path())
    assert hasattr(L, name), name
