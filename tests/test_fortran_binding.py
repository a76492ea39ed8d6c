"""The Fortran interface module include/semba_gpu_m.F90 against the C header.

No Fortran compiler is needed: both files are parsed as text.  Every entry
point the header declares must have a bind(C) interface of the same name and
argument count (a subroutine for void, a type(c_ptr) function for const
char*), and every struct must have a bind(C) derived type whose members are
the struct's members in order, with the matching interoperable kind and the
array extents reversed (C [a][b] is Fortran (b, a))."""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "semba_gpu.h"
MODULE = ROOT / "include" / "semba_gpu_m.F90"


def _c_source():
    return re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)


def c_functions():
    out = {}
    for m in re.finditer(r"(sgpu_status|void|const char\*)\s+(sgpu_\w+)\s*\(([^)]*)\)\s*;", _c_source()):
        args = [a.strip() for a in m.group(3).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(2)] = (m.group(1), args)
    return out


_C_KIND = {"int": "integer(c_int)", "float": "real(c_float)", "double": "real(c_double)"}


def c_structs():
    out = {}
    for m in re.finditer(r"typedef\s+struct\s*\{(.*?)\}\s*(sgpu_\w+)\s*;", _c_source(), flags=re.S):
        members = []
        for decl in m.group(1).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            t = re.match(r"(const\s+)?(\w+)\s*(.*)", decl)
            base, rest = t.group(2), t.group(3)
            for item in rest.split(","):
                item = item.strip()
                ptr = item.startswith("*")
                name = item.lstrip("*").strip()
                dims = [int(d) for d in re.findall(r"\[(\d+)\]", name)]
                name = re.sub(r"\[.*", "", name).strip()
                kind = "type(c_ptr)" if ptr else _C_KIND.get(base, f"type({base})")
                members.append((name, kind, tuple(reversed(dims))))
        out[m.group(2)] = members
    return out


def _fortran_source():
    # drop comments and join continuation lines
    lines = []
    for ln in MODULE.read_text().splitlines():
        ln = re.sub(r"!.*", "", ln).rstrip()
        if lines and lines[-1].endswith("&"):
            lines[-1] = lines[-1][:-1] + " " + ln.strip()
        else:
            lines.append(ln)
    return "\n".join(lines)


def f_interfaces():
    out = {}
    for m in re.finditer(r"^\s*(type\(c_ptr\)\s+function|integer\(c_int\)\s+function|subroutine)\s+(\w+)\s*\(([^)]*)\)"
                         r"\s*bind\(C,\s*name=\"(\w+)\"\)", _fortran_source(), flags=re.M):
        args = [a.strip() for a in m.group(3).split(",") if a.strip()]
        out[m.group(4)] = (m.group(1).split()[0], m.group(2), args)
    return out


def f_types():
    out = {}
    for m in re.finditer(r"type,\s*bind\(C\)\s*::\s*(\w+)\n(.*?)\n\s*end type", _fortran_source(), flags=re.S):
        members = []
        for ln in m.group(2).splitlines():
            ln = ln.strip()
            if not ln:
                continue
            kind, names = [x.strip() for x in ln.split("::")]
            for item in re.findall(r"\w+(?:\([^)]*\))?", names):
                nm = re.match(r"(\w+)", item).group(1)
                dims = tuple(int(d) for d in re.findall(r"\d+", item[len(nm):]))
                members.append((nm, kind, dims))
        out[m.group(1)] = members
    return out


def test_every_entry_point_has_an_interface():
    cf, fi = c_functions(), f_interfaces()
    assert len(cf) > 80
    missing = sorted(set(cf) - set(fi))
    assert not missing, f"no Fortran interface for {missing}"
    extra = sorted(set(fi) - set(cf))
    assert not extra, f"interfaces for names the header does not declare: {extra}"
    for name, (ret, args) in cf.items():
        kind, fname, fargs = fi[name]
        assert fname == name, name
        assert len(fargs) == len(args), f"{name}: {len(fargs)} Fortran arguments, {len(args)} in C"
        want = {"void": "subroutine", "const char*": "type(c_ptr)", "sgpu_status": "integer(c_int)"}[ret]
        assert kind == want, f"{name}: {kind} for a C {ret}"


def test_every_struct_has_a_matching_derived_type():
    cs, ft = c_structs(), f_types()
    assert len(cs) >= 15
    missing = sorted(set(cs) - set(ft))
    assert not missing, f"no bind(C) type for {missing}"
    for name, members in cs.items():
        assert ft[name] == members, f"{name}:\n C {members}\n F {ft[name]}"


def test_value_arguments_follow_the_c_prototypes():
    """A C scalar passed by value must be a `value` dummy; a pointer to a
    handle or an array must not be passed as a Fortran value integer."""
    src = _fortran_source()
    cf = c_functions()
    for name, (_, args) in cf.items():
        body = re.search(r"bind\(C,\s*name=\"%s\"\)(.*?)end (function|subroutine)" % name, src, flags=re.S).group(1)
        _, _, fargs = f_interfaces()[name]
        for ca, fa in zip(args, fargs):
            decl = re.search(r"^\s*(.*?)::[^\n]*\b%s\b" % fa, body, flags=re.M)
            assert decl, f"{name}: no declaration of {fa}"
            attrs = decl.group(1)
            by_value = "*" not in ca
            if by_value:
                assert "value" in attrs, f"{name}({fa}): C passes '{ca}' by value"
            elif "value" in attrs:
                assert "type(c_ptr)" in attrs, f"{name}({fa}): '{ca}' is a pointer"


def test_fixed_form_limits():
    for n, ln in enumerate(MODULE.read_text().splitlines(), 1):
        assert len(ln) <= 132, f"line {n} longer than 132 characters"
