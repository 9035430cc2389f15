"""The C-ABI library builds, loads and exports every symbol include/fos.h declares."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "fos.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fos_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib_path():
    from fos import build
    return build.build()


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "fos_jfa_run" in syms and "fos_frame_graph" in syms
    assert len(syms) >= 40


def test_library_exports_every_declared_symbol(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (fos_[a-z0-9_]+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing


def test_ctypes_binding_covers_header(lib_path):
    from fos import _lib
    lib = _lib.load()
    for s in declared_symbols():
        assert hasattr(lib, s), s
        assert s in _lib.SIGNATURES, f"{s} has no ctypes signature"


def declared_arities():
    """Parameter count of every function declared in include/fos.h."""
    src = open(os.path.join(ROOT, "include", "fos.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for name, params in re.findall(r"\b(fos_[a-z0-9_]+)\s*\(([^;{}]*?)\)\s*;", src, flags=re.S):
        params = " ".join(params.split())
        out[name] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_ctypes_argument_counts_match_header():
    """Every ctypes signature takes as many arguments as its declaration."""
    from fos import _lib
    ar = declared_arities()
    assert len(ar) >= 40
    bad = {k: (n, len(_lib.SIGNATURES[k])) for k, n in ar.items()
           if k in _lib.SIGNATURES and len(_lib.SIGNATURES[k]) != n}
    assert not bad, bad


def test_status_strings_without_gpu(lib_path):
    from fos import _lib
    lib = _lib.load()
    assert lib.fos_status_string(0) == b"FOS_OK"
    assert lib.fos_status_string(2) == b"FOS_E_CAPACITY"
    import ctypes as C
    p = _lib.FosParams()
    lib.fos_params_default(C.byref(p))
    assert p.t_add == 0.15 and p.t_drop == 0.10 and p.expected_face_scale == 1.5
    # argument validation needs no device
    assert lib.fos_ctx_create(None, 10, 64, 0, C.byref(C.c_void_p())) == 1
    assert lib.fos_set_resolution(None, 64) == 1


def test_ctypes_structures_match_header_layout(tmp_path):
    """Every ctypes structure of the binding has the size and field offsets of
    its C declaration in include/fos.h (a C probe compiled with gcc prints
    them), so no field is silently shifted across the boundary."""
    import ctypes as C
    from fos import _lib
    structs = {name: cls for name, cls in vars(_lib).items()
               if isinstance(cls, type) and issubclass(cls, C.Structure) and name.startswith("Fos")}
    assert len(structs) >= 10
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "fos.h"', "int main(void) {"]
    for name, cls in sorted(structs.items()):
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True, capture_output=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                   check=True).stdout.splitlines())
    for name, cls in structs.items():
        assert int(got[name]) == C.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert int(got[f"{name}.{fname}"]) == getattr(cls, fname).offset, f"{name}.{fname}"

