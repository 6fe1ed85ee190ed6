"""The native library loads on a CPU-only machine and exports every function include/*.h declares."""
import ctypes as C
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(csu_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_exports(native):
    L = C.CDLL(os.path.join(ROOT, "csu_b200", "lib", "libcsu_b200.so"))
    names = declared()
    assert len(names) > 20
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_strerror(native):
    import csu_b200
    L = csu_b200.lib()
    assert L.csu_strerror(0) == b"ok"
    assert L.csu_strerror(4) == b"non-finite state"
