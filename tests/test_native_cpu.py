"""libpfflip.so loads without a GPU and exports every entry point of
include/pfflip.h (no compute calls here)."""

import ctypes
import os
import re

from pfflip import _native as N
from pfflip.poisson import level_dims

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(REPO, "include"))):
        if fn.endswith(".h"):
            src = open(os.path.join(REPO, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"\b(pf_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    names = declared_functions()
    missing = [n for n in names if n not in N.SIGNATURES]
    assert not missing, missing


def declared_arities():
    out = {}
    for fn in sorted(os.listdir(os.path.join(REPO, "include"))):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(REPO, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(pf_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", src):
            args = m.group(2).strip()
            out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_binding_arities_match_header():
    ar = declared_arities()
    assert len(ar) >= 20
    bad = {n: (a, len(N.SIGNATURES[n][1])) for n, a in ar.items() if len(N.SIGNATURES[n][1]) != a}
    assert not bad, bad


def test_host_only_entry_points():
    lib = N.lib()
    assert b"sm_100a" in lib.pf_version()
    assert lib.pf_mg_partials_count() > 0
    for res, md in (((128,) * 3, 4), ((24,) * 3, 4), ((25, 32, 32), 4), ((64, 32, 16), 4)):
        dims = (ctypes.c_int32 * 48)()
        n = lib.pf_mg_level_count(*res, md, dims)
        ref = level_dims(res, md)
        assert n == len(ref)
        assert [tuple(dims[3 * i: 3 * i + 3]) for i in range(n)] == [tuple(r) for r in ref]


def _c_layout():
    """Compile a probe against include/pfflip.h and read its struct layout."""
    import shutil
    import subprocess
    import tempfile

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        import pytest

        pytest.skip("no C compiler")
    fields = {"pf_grid": [f for f, _ in N.pf_grid._fields_], "pf_mg_level": [f for f, _ in N.pf_mg_level._fields_],
              "pf_mg_desc": [f for f, _ in N.pf_mg_desc._fields_]}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "pfflip.h"', "int main(void){"]
    for st, fs in fields.items():
        lines.append(f'printf("{st} size %zu\\n", sizeof({st}));')
        for f in fs:
            lines.append(f'printf("{st} {f} %zu\\n", offsetof({st}, {f}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "probe.c"), os.path.join(d, "probe")
        open(src, "w").write("\n".join(lines))
        subprocess.check_call([cc, "-I", os.path.join(REPO, "include"), src, "-o", exe])
        out = subprocess.check_output([exe], text=True)
    res = {}
    for ln in out.splitlines():
        st, f, v = ln.split()
        res[(st, f)] = int(v)
    return res


def test_struct_layouts_match_header():
    c = _c_layout()
    for cls in (N.pf_grid, N.pf_mg_level, N.pf_mg_desc):
        name = cls.__name__
        assert c[(name, "size")] == ctypes.sizeof(cls), name
        for f, _ in cls._fields_:
            assert c[(name, f)] == getattr(cls, f).offset, (name, f)
