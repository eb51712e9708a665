"""The Fortran binding module (cice-evp1d_b200/fortran/evp1d_cuda.F90) against
the C-ABI it binds (include/evp1d.h).

No Fortran compiler exists on the build or test machines, so the module is
checked by reading it: every bind(C) interface must name an entry point the
header declares and the library exports, with the same number of arguments,
each of a kind the C prototype accepts under ISO_C_BINDING (int by value,
size_t by value, a pointer passed as c_ptr by value, a pointer-to-pointer
out-argument as c_ptr by reference, int32_t / double arrays, structs by
reference), and the same return kind; every bind(C) derived type must list
the C struct's fields in the same order with the same kinds and counts.
"""
import ctypes
import os
import re
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "cice-evp1d_b200", "fortran", "evp1d_cuda.F90")
HDR = os.path.join(ROOT, "include", "evp1d.h")
LIB = os.path.join(ROOT, "cice-evp1d_b200", "lib", "libevp1d.so")


# ---------------------------------------------------------------- Fortran side
def _fortran_lines():
    out, cur = [], ""
    for raw in open(F90):
        line = raw.split("!", 1)[0].rstrip()
        if not line.strip():
            continue
        s = line.strip()
        if cur:
            s = s[1:].lstrip() if s.startswith("&") else s
        if s.endswith("&"):
            cur += s[:-1] + " "
            continue
        out.append(cur + s)
        cur = ""
    return out


_DECL = re.compile(r"^(integer\(c_int\)|integer\(c_int32_t\)|integer\(c_size_t\)|"
                   r"real\(c_double\)|type\(c_ptr\)|type\((\w+)\))\s*(,[^:]*)?::\s*(.*)$", re.I)


def _items(lst):
    """'a, b(*), c(12)' -> [(name, dim)] with dim None, '*' or an int."""
    out = []
    for it in re.findall(r"(\w+)(?:\(([^)]*)\))?", lst):
        name, dim = it
        out.append((name, None if not dim else ("*" if dim.strip() == "*" else int(dim))))
    return out


def fortran_types():
    types, cur = {}, None
    for ln in _fortran_lines():
        m = re.match(r"^type\s*,\s*bind\(C\)\s*::\s*(\w+)$", ln, re.I)
        if m:
            cur = m.group(1)
            types[cur] = []
            continue
        if cur and re.match(r"^end\s+type", ln, re.I):
            cur = None
            continue
        if cur:
            d = _DECL.match(ln)
            assert d, f"unparsed field line in {cur}: {ln}"
            kind = "double" if d.group(1).lower() == "real(c_double)" else "ptr"
            for name, dim in _items(d.group(4)):
                types[cur].append((name.lower(), kind, dim or 1))
    return types


_HEAD = re.compile(r"^(integer\(c_int\)\s+function|type\(c_ptr\)\s+function|subroutine)\s+"
                   r"(\w+)\s*\(([^)]*)\)\s*bind\(C\s*,\s*name\s*=\s*\"(\w+)\"\)$", re.I)


def fortran_interfaces():
    out, cur = {}, None
    for ln in _fortran_lines():
        h = _HEAD.match(ln)
        if h:
            ret = {"integer(c_int) function": "int", "type(c_ptr) function": "ptr",
                   "subroutine": "void"}[re.sub(r"\s+", " ", h.group(1).lower())]
            dummies = [a.strip() for a in h.group(3).split(",") if a.strip()]
            cur = {"fname": h.group(2), "ret": ret, "dummies": dummies, "kind": {}}
            out[h.group(4)] = cur
            continue
        if cur is None:
            continue
        if re.match(r"^end\s+(function|subroutine)", ln, re.I):
            missing = [d for d in cur["dummies"] if d.lower() not in cur["kind"]]
            assert not missing, f"{cur['fname']}: undeclared dummies {missing}"
            cur = None
            continue
        if re.match(r"^import\b", ln, re.I):
            continue
        d = _DECL.match(ln)
        assert d, f"unparsed declaration in {cur['fname']}: {ln}"
        base, attrs = d.group(1).lower(), (d.group(3) or "").lower()
        value = "value" in attrs
        for name, dim in _items(d.group(4)):
            if base == "integer(c_int)":
                k = "int" if value else "ref:int"
            elif base == "integer(c_size_t)":
                k = "size_t" if value else "ref:size_t"
            elif base == "type(c_ptr)":
                k = "ptr" if value else "ptr_ref"
            elif base == "integer(c_int32_t)":
                k = "arr:int32_t" if dim == "*" else "ref:int32_t"
            elif base == "real(c_double)":
                k = "arr:double" if dim == "*" else "ref:double"
            else:
                k = "struct:" + d.group(2).lower()
            cur["kind"][name.lower()] = k
    assert cur is None, "unterminated interface"
    return out


# ---------------------------------------------------------------------- C side
def _header():
    return re.sub(r"/\*.*?\*/", " ", open(HDR).read(), flags=re.S)


def c_prototype(name):
    m = re.search(r"(?:^|[;}\n])\s*([\w\s\*]+?)\b" + name + r"\s*\(([^;{]*?)\)\s*;", _header(), re.S)
    assert m, f"{name} is not declared in include/evp1d.h"
    ret = " ".join(m.group(1).split())
    params = []
    for p in m.group(2).split(","):
        p = " ".join(p.split())
        if not p or p == "void":
            continue
        stars = p.count("*")
        toks = [t for t in re.findall(r"\w+", p) if t != "const"]
        params.append((toks[0], stars))
    return ret, params


def c_struct(name):
    m = re.search(r"typedef\s+struct\s+" + name + r"\s*\{(.*?)\}\s*" + name + r"\s*;", _header(), re.S)
    assert m, f"struct {name} not found"
    fields = []
    for decl in m.group(1).split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        head = re.match(r"^((?:const\s+)?\w+)\s+(.*)$", decl)
        for dcl in head.group(2).split(","):
            dm = re.match(r"^\s*(\**)\s*(?:const\s+)?(\w+)\s*(?:\[(\d+)\])?\s*$", dcl)
            kind = "ptr" if dm.group(1) else head.group(1).replace("const ", "")
            fields.append((dm.group(2).lower(), kind, int(dm.group(3) or 1)))
    return fields


def _compatible(fkind, ctype):
    base, stars = ctype
    if fkind == "int":
        return base == "int" and stars == 0
    if fkind == "size_t":
        return base == "size_t" and stars == 0
    if fkind == "ptr":
        return stars >= 1
    if fkind == "ptr_ref":
        return stars == 2
    if fkind.startswith("arr:"):
        return base == fkind[4:] and stars == 1
    if fkind.startswith("struct:"):
        return base.lower() == fkind[7:] and stars == 1
    return False


# ------------------------------------------------------------------- the tests
def test_every_interface_matches_its_c_prototype():
    ifs = fortran_interfaces()
    assert len(ifs) >= 18
    for cname, f in ifs.items():
        ret, params = c_prototype(cname)
        assert f["fname"] == cname, f"{f['fname']} binds {cname}"
        want_ret = {"int": "int", "void": "void"}.get(f["ret"])
        if want_ret:
            assert ret == want_ret, f"{cname}: returns {ret}, the interface says {f['ret']}"
        else:
            assert "*" in ret, f"{cname}: returns {ret}, the interface says a pointer"
        assert len(f["dummies"]) == len(params), (cname, f["dummies"], params)
        for dummy, cp in zip(f["dummies"], params):
            k = f["kind"][dummy.lower()]
            assert _compatible(k, cp), f"{cname}: argument {dummy} is {k}, C has {cp}"


@pytest.mark.parametrize("name", ["evp1d_params", "evp1d_fields", "evp1d_grads"])
def test_derived_types_match_the_c_structs(name):
    assert fortran_types()[name] == c_struct(name)


def test_the_library_exports_every_bound_entry_point():
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    lib = ctypes.CDLL(LIB)
    missing = [c for c in fortran_interfaces() if not hasattr(lib, c)]
    assert not missing, missing


def test_the_checker_rejects_a_wrong_binding(tmp_path, monkeypatch):
    """A binding with an argument of the wrong kind (ndte by reference) and
    one with an argument too few are both caught."""
    src = open(F90).read()
    bad = src.replace("""       type(c_ptr), value :: h
       integer(c_int), value :: ndte
       type(evp1d_fields), intent(in) :: io
     end function

     ! dyn_evp1d_finalize""", """       type(c_ptr), value :: h
       integer(c_int) :: ndte
       type(evp1d_fields), intent(in) :: io
     end function

     ! dyn_evp1d_finalize""")
    assert bad != src
    p = tmp_path / "bad.F90"
    p.write_text(bad)
    monkeypatch.setattr(sys.modules[__name__], "F90", str(p))
    with pytest.raises(AssertionError, match="evp1d_run: argument ndte"):
        test_every_interface_matches_its_c_prototype()
    bad2 = src.replace('function evp1d_finalize(h) bind(C, name="evp1d_finalize")',
                       'function evp1d_finalize() bind(C, name="evp1d_finalize")')
    bad2 = bad2.replace("""  import :: c_ptr, c_int
       type(c_ptr), value :: h
     end function

     ! evp1d_run split""", """  import :: c_ptr, c_int
     end function

     ! evp1d_run split""")
    p.write_text(bad2)
    with pytest.raises(AssertionError, match="evp1d_finalize"):
        test_every_interface_matches_its_c_prototype()


def test_integration_examples_use_the_module():
    """The Fortran snippets of INTEGRATION.md only call procedures the module
    binds (or defines) and only set fields that evp1d_fields has."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```fortran\n(.*?)```", text, re.S)
    assert blocks
    bound = {c.lower() for c in fortran_interfaces()} | {"evp1d_last_error_f"}
    fields = {f[0] for f in fortran_types()["evp1d_fields"]}
    for b in blocks:
        for name in re.findall(r"\b(evp1d_\w+)\s*\(", b):
            if re.search(r"(function|subroutine)\s+" + name, b):
                continue  # an interface written out in the snippet itself
            assert name.lower() in bound, f"INTEGRATION.md calls {name}, which the module does not bind"
        for f in re.findall(r"\bio%(\w+)", b):
            assert f.lower() in fields, f"INTEGRATION.md sets io%{f}, not a field of evp1d_fields"
