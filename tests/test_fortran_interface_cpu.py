"""The Fortran ISO_C_BINDING module include/owl_ssg.f90 against the C header
include/owl_ssg.h (no Fortran compiler exists here, so the two are compared
as text): every macro constant has a Fortran parameter of the same value,
every C struct a bind(c) type with the same fields in the same order and of
the matching C type and array length, and every function a bind(c)
interface with the same name, return kind and argument kinds (by value or by
reference) in the same order."""
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
INC = os.path.join(os.path.dirname(HERE), "include")


def _read(name):
    with open(os.path.join(INC, name)) as f:
        return f.read()


def _c_source():
    s = _read("owl_ssg.h")
    s = re.sub(r"/\*.*?\*/", " ", s, flags=re.S)
    return re.sub(r"//[^\n]*", " ", s)


def _f_source():
    lines = []
    for ln in _read("owl_ssg.f90").splitlines():
        ln = ln.split("!")[0].rstrip()
        if lines and lines[-1].endswith("&"):
            lines[-1] = lines[-1][:-1] + " " + ln.strip().lstrip("&")
        else:
            lines.append(ln)
    return lines


C_SCALAR = {"int": "int", "float": "float", "double": "double", "long long": "longlong"}
F_SCALAR = {"integer(c_int)": "int", "real(c_float)": "float", "real(c_double)": "double",
            "integer(c_long_long)": "longlong", "type(c_ptr)": "ptr"}


def c_constants():
    out = {}
    for m in re.finditer(r"#define\s+(OWL_\w+)\s+(.+)", _c_source()):
        v = m.group(2).strip()
        if re.fullmatch(r"[-()\d\s*]+", v):
            out[m.group(1)] = eval(v)
    return out


def f_constants():
    out = {}
    for ln in _f_source():
        m = re.match(r"\s*integer\(c_int\),\s*parameter\s*::\s*(\w+)\s*=\s*(.+)", ln)
        if m:
            out[m.group(1)] = eval(m.group(2))
    return out


def c_structs():
    out = {}
    for m in re.finditer(r"typedef\s+struct\s*\{(.*?)\}\s*(\w+)\s*;", _c_source(), flags=re.S):
        fields = []
        for decl in m.group(1).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            dm = re.match(r"(const\s+)?(long long|int|float|double|\w+)\s+(.*)", decl)
            base, rest = dm.group(2), dm.group(3)
            for name in rest.split(","):
                name = name.strip()
                ptr = name.startswith("*")
                name = name.lstrip("*").strip()
                nm = re.match(r"(\w+)(?:\[(\d+)\])?", name)
                kind = "ptr" if ptr else C_SCALAR[base]
                fields.append((nm.group(1), kind, int(nm.group(2) or 1)))
        out[m.group(2)] = fields
    return out


def f_types():
    out, cur = {}, None
    for ln in _f_source():
        m = re.match(r"\s*type,\s*bind\(c\)\s*::\s*(\w+)", ln)
        if m:
            cur = out.setdefault(m.group(1), [])
            continue
        if cur is not None and re.match(r"\s*end type", ln):
            cur = None
            continue
        if cur is not None and "::" in ln:
            kind, names = (x.strip() for x in ln.split("::"))
            for name in re.findall(r"\w+(?:\(\d+\))?", names):
                nm = re.match(r"(\w+)(?:\((\d+)\))?", name)
                cur.append((nm.group(1), F_SCALAR[kind], int(nm.group(2) or 1)))
    return out


def c_functions():
    out = {}
    src = " ".join(_c_source().split())
    for m in re.finditer(r"(int|void|float|const char \*)\s*(owl_\w+)\s*\(([^)]*)\)\s*;", src):
        args = [] if m.group(3).strip() in ("", "void") else [a.strip() for a in m.group(3).split(",")]
        kinds = []
        for a in args:
            if "*" in a:
                kinds.append("ref")
            else:
                base = re.match(r"(const\s+)?(long long|int|float|double)", a).group(2)
                kinds.append(C_SCALAR[base])
        ret = {"int": "int", "void": "none", "float": "float", "const char *": "ptr"}[m.group(1)]
        out[m.group(2)] = (ret, kinds)
    return out


def f_interfaces():
    out, cur, decls = {}, None, {}
    for ln in _f_source():
        m = re.match(r"\s*(?:(integer\(c_int\)|real\(c_float\)|type\(c_ptr\))\s+)?(function|subroutine)\s+(\w+)\s*"
                     r"\(([^)]*)\)\s*bind\(c,\s*name='(\w+)'\)", ln)
        if m:
            assert m.group(3) == m.group(5), ln
            ret = {"integer(c_int)": "int", "real(c_float)": "float", "type(c_ptr)": "ptr", None: "none"}[m.group(1)]
            cur = (m.group(3), ret, [a.strip() for a in m.group(4).split(",") if a.strip()])
            decls = {}
            continue
        if cur is not None and re.match(r"\s*end (function|subroutine)", ln):
            name, ret, args = cur
            kinds = []
            for a in args:
                kind, value = decls[a]
                if value:
                    kinds.append("ref" if kind == "ptr" else kind)
                else:
                    kinds.append("ref")
            out[name] = (ret, kinds)
            cur = None
            continue
        if cur is not None and "::" in ln and not ln.strip().startswith("import"):
            spec, names = (x.strip() for x in ln.split("::"))
            parts = [p.strip() for p in spec.split(",")]
            kind = F_SCALAR.get(parts[0], "derived")
            value = "value" in parts
            for name in re.findall(r"(\w+)(?:\(\*\))?", names):
                decls[name] = (kind, value)
    return out


def test_constants_match():
    c, f = c_constants(), f_constants()
    assert len(c) >= 60
    assert set(c) == set(f), (set(c) ^ set(f))
    for k in c:
        assert c[k] == f[k], k


def test_structs_match_field_by_field():
    c, f = c_structs(), f_types()
    assert len(c) == 7
    assert set(c) == set(f), (set(c) ^ set(f))
    for k in c:
        assert c[k] == f[k], (k, c[k], f[k])


def test_functions_match_argument_by_argument():
    c, f = c_functions(), f_interfaces()
    assert len(c) >= 25
    assert set(c) == set(f), (set(c) ^ set(f))
    for k in c:
        assert c[k] == f[k], (k, c[k], f[k])


def test_library_exports_every_interface():
    from owl_b200 import _lib as L
    lib = L.load()
    for name in f_interfaces():
        assert hasattr(lib, name), name
