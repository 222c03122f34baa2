"""The drop-in boundary's signatures, checked against the reference's own source.

Three descriptions of the 89 ``api3_*`` entry points must agree with the reference core's
definitions (semiconductor_3d.c:4570-5353):

* the declarations of ``include/semisim_b200.h`` (the C side of this library);
* the ctypes table ``semiconductor_devices_simulator_b200/abi.py`` (its Python side);
* the bindings the reference's own Python makes, ``main.py:172-219`` and
  ``main.py:3490-3514`` (``_f`` / ``_opt``) and ``validate.py:31-53``, since those are
  what load this library in place of the reference core.

Return type and every argument type are compared (``const`` and parameter names
ignored).  The reference checkout is read as text (its Python is parsed, not run); the
test is skipped where the checkout is absent.
"""
import ast
import ctypes
import os
import re

import pytest

from semiconductor_devices_simulator_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("SEMISIM_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))
CORE = os.path.join(REF, "semiconductor_3d.c")

pytestmark = pytest.mark.skipif(not os.path.exists(CORE), reason="reference checkout not present")

_DEF = re.compile(r"(?m)^(void|int|double|long long)\s+(api3_\w+)\s*\(([^)]*)\)\s*\{")
_DECL = re.compile(r"(?m)^(void|int|double|long long)\s+(api3_\w+)\s*\(([^)]*)\)\s*;")

CT = {"void": None, "int": ctypes.c_int, "double": ctypes.c_double, "long long": ctypes.c_longlong,
      "int*": ctypes.POINTER(ctypes.c_int), "double*": ctypes.POINTER(ctypes.c_double),
      "long long*": ctypes.POINTER(ctypes.c_longlong)}


def c_type(decl):
    """'const double *xs' -> 'double*'; 'int n' -> 'int'; 'void' -> 'void'."""
    t = decl.replace("const", " ").strip()
    ptr = t.count("*")
    t = t.replace("*", " ")
    words = t.split()
    if len(words) > 1 and words[-1] not in ("int", "double", "long", "void"):
        words = words[:-1]                                 # drop the parameter name
    return " ".join(words) + "*" * ptr


def signatures(text, rx):
    out = {}
    for m in rx.finditer(text):
        ret, name, params = m.group(1), m.group(2), m.group(3).strip()
        args = [] if params in ("", "void") else [c_type(p) for p in params.split(",")]
        out[name] = (ret, args)
    return out


@pytest.fixture(scope="module")
def ref_sigs():
    sigs = signatures(open(CORE).read(), _DEF)
    assert len(sigs) == 89, sorted(sigs)
    return sigs


def test_header_matches_reference_definitions(ref_sigs):
    hdr = signatures(open(os.path.join(ROOT, "include", "semisim_b200.h")).read(), _DECL)
    missing = set(ref_sigs) - set(hdr)
    assert not missing, missing
    bad = {n: (hdr[n], ref_sigs[n]) for n in ref_sigs if hdr[n] != ref_sigs[n]}
    assert not bad, bad


def test_ctypes_table_matches_reference_definitions(ref_sigs):
    assert set(abi.API3) == set(ref_sigs)
    for name, (ret, args) in ref_sigs.items():
        res, argt = abi.API3[name]
        assert res == CT[ret], (name, res, ret)
        assert list(argt) == [CT[a] for a in args], (name, argt, args)


def _ctype_of(node, names):
    """ctypes type of a binding argument expression of main.py (Name, ctypes.X or
    ctypes.POINTER(X))."""
    if isinstance(node, ast.Constant) and node.value is None:
        return None
    if isinstance(node, ast.Name):
        return names[node.id]
    if isinstance(node, ast.Attribute) and isinstance(node.value, ast.Name) and node.value.id == "ctypes":
        return getattr(ctypes, node.attr)
    if (isinstance(node, ast.Call) and isinstance(node.func, ast.Attribute) and node.func.attr == "POINTER"):
        return ctypes.POINTER(_ctype_of(node.args[0], names))
    raise AssertionError(f"unexpected binding expression {ast.dump(node)}")


def main_py_bindings():
    tree = ast.parse(open(os.path.join(REF, "main.py")).read())
    names = {"D": ctypes.c_double, "I": ctypes.c_int, "V": None, "DP": ctypes.POINTER(ctypes.c_double),
             "IP": ctypes.POINTER(ctypes.c_int)}
    out = {}
    for node in ast.walk(tree):
        if (isinstance(node, ast.Call) and isinstance(node.func, ast.Name) and node.func.id in ("_f", "_opt")
                and node.args and isinstance(node.args[0], ast.Constant)
                and str(node.args[0].value).startswith("api3_")):
            vals = [_ctype_of(a, names) for a in node.args[1:]]
            out[node.args[0].value] = (node.lineno, vals[0], vals[1:])
    return out


def validate_py_bindings():
    tree = ast.parse(open(os.path.join(REF, "validate.py")).read())
    env = {"ctypes": ctypes, "_I": ctypes.c_int, "_D": ctypes.c_double, "None": None}
    out = {}
    for node in ast.walk(tree):
        if (isinstance(node, ast.Tuple) and len(node.elts) == 3 and isinstance(node.elts[0], ast.Constant)
                and str(node.elts[0].value).startswith("api3_")):
            res = eval(compile(ast.Expression(node.elts[1]), "validate.py", "eval"), env)
            args = eval(compile(ast.Expression(node.elts[2]), "validate.py", "eval"), env)
            out[node.elts[0].value] = (node.lineno, res, list(args))
    return out


def test_reference_python_bindings_match_ctypes_table():
    mp = main_py_bindings()
    vp = validate_py_bindings()
    assert len(mp) >= 50 and len(vp) >= 15, (len(mp), len(vp))
    for src, table in (("main.py", mp), ("validate.py", vp)):
        for name, (line, res, args) in table.items():
            assert name in abi.API3, f"{src}:{line} binds {name}, which the ABI table lacks"
            r, a = abi.API3[name]
            assert res == r, f"{src}:{line} {name} restype {res} != {r}"
            assert args == list(a), f"{src}:{line} {name} argtypes {args} != {a}"
