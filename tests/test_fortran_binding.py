"""The Fortran binding module a maintainer adds to the reference (the
``ISO_C_BINDING`` module in INTEGRATION.md) against the C ABI it binds.

No Fortran compiler exists on the build or GPU machines, so the module is
checked here as text: every ``bind(c)`` interface names a function of
``include/lceqcd_gpu.h`` with the same number of arguments, each argument
passed by value exactly where the C parameter is a scalar and by reference
where it is a pointer, with a matching kind; the return kinds agree; and the
``bind(c)`` derived types mirror ``lce_params`` and ``lce_meas`` member by
member.
"""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _fortran_module():
    text = (ROOT / "INTEGRATION.md").read_text()
    m = re.search(r"```fortran\n(module lceqcd_gpu_mod\n.*?\nend module)\n```", text, re.S)
    assert m, "binding module not found"
    return m.group(1)


def _c_header():
    text = (ROOT / "include" / "lceqcd_gpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return "\n".join(line for line in text.splitlines() if not line.lstrip().startswith("#"))


def _c_prototypes():
    text = _c_header()
    protos = {}
    for m in re.finditer(r"\b((?:const\s+)?[A-Za-z_][\w\s]*?\**)\s*\b(lce_\w+)\s*\(([^;{)]*)\)\s*;", text):
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3).strip()
        if ret.startswith("typedef"):
            continue
        params = [] if args in ("", "void") else [a.strip() for a in args.split(",")]
        protos[name] = (ret, params)
    return protos


def _c_struct(name):
    text = _c_header()
    m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, re.S)
    assert m, name
    members = []
    for decl in m.group(1).split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        mm = re.match(r"((?:unsigned )?(?:long long|int|double|float|long))\s+(.*)", decl)
        assert mm, decl
        ctype = mm.group(1)
        for var in mm.group(2).split(","):
            var = var.strip()
            n = 1
            arr = re.match(r"(\w+)\[(\d+)\]", var)
            if arr:
                var, n = arr.group(1), int(arr.group(2))
            members.append((var, ctype, n))
    return members


F_KIND = {"integer(c_int)": "int", "real(c_double)": "double", "real(c_float)": "float",
          "integer(c_long)": "long", "integer(c_long_long)": "unsigned long long",
          "integer(c_size_t)": "size_t", "complex(c_float_complex)": "float",
          "complex(c_double_complex)": "double", "type(c_ptr)": "void*"}


def _fortran_interfaces():
    mod = _fortran_module()
    body = mod[mod.index("interface"):mod.index("end interface")]
    body = re.sub(r"&\s*\n\s*", " ", body)  # free-form continuation lines
    out = {}
    pat = re.compile(r"^\s*(?:(integer\(c_int\)|type\(c_ptr\))\s+function|subroutine)\s+(\w+)\(([^)]*)\)\s*bind\(c\)"
                     r"(.*?)^\s*end (?:function|subroutine)", re.S | re.M)
    for m in pat.finditer(body):
        ret, name, args, decls = m.group(1) or "void", m.group(2), m.group(3), m.group(4)
        argnames = [a.strip() for a in args.split(",") if a.strip()]
        types = {}
        for stmt in re.split(r"[;\n]", decls):
            stmt = stmt.strip()
            if not stmt or stmt == "import":
                continue
            dm = re.match(r"((?:integer|real|complex|type)\([\w]+\))\s*((?:,\s*[\w()]+)*)\s*::\s*(.*)", stmt)
            assert dm, (name, stmt)
            attrs = dm.group(2)
            for v in dm.group(3).split(","):
                v = v.strip()
                vn = re.match(r"(\w+)(\(.*\))?", v)
                types[vn.group(1)] = (dm.group(1), "value" in attrs, vn.group(2) is not None)
        out[name] = (ret, argnames, types)
    return out


def test_module_is_present_and_balanced():
    mod = _fortran_module()
    opened = len(re.findall(r"^\s*(?:integer\(c_int\)|type\(c_ptr\))\s+function\b", mod, re.M))
    assert opened == len(re.findall(r"^\s*end function\b", mod, re.M))
    assert len(re.findall(r"^\s*subroutine\b", mod, re.M)) == len(re.findall(r"^\s*end subroutine\b", mod, re.M))
    assert len(re.findall(r"\bbind\(c\)", mod)) >= 30


def test_every_binding_matches_the_c_prototype():
    protos = _c_prototypes()
    fifs = _fortran_interfaces()
    assert len(fifs) >= 28
    for name, (ret, argnames, types) in fifs.items():
        assert name in protos, f"{name}: no such C function"
        cret, cparams = protos[name]
        assert len(argnames) == len(cparams), f"{name}: {len(argnames)} arguments, C has {len(cparams)}"
        if ret == "void":
            assert cret == "void", name
        elif ret == "type(c_ptr)":
            assert cret.endswith("*"), name
        else:
            assert cret == "int", name
        for a, cp in zip(argnames, cparams):
            assert a in types, f"{name}: argument {a} undeclared"
            ftype, by_value, is_array = types[a]
            pointer = "*" in cp or "[" in cp
            cbase = " ".join(re.sub(r"\bconst\b|\*|\[.*?\]", " ", cp).split())
            cbase = re.sub(r"\s+\w+$", "", cbase)  # the parameter's name
            if ftype.startswith("type(") and ftype != "type(c_ptr)":
                # a bind(c) derived type: the C side takes a pointer to the struct
                assert pointer and not by_value, f"{name}({a})"
                assert ftype[5:-1] in cbase, f"{name}({a}): {ftype} vs {cp}"
                continue
            if ftype == "type(c_ptr)":
                assert by_value and pointer, f"{name}({a}): an opaque handle is a C pointer passed by value"
                continue
            assert by_value != pointer, f"{name}({a}): value attribute vs C parameter {cp!r}"
            want = F_KIND[ftype]
            if cbase in ("unsigned", "unsigned int"):
                cbase = "int"  # a counter read as a default integer (no unsigned kinds in Fortran)
            assert cbase == want, f"{name}({a}): Fortran {ftype} vs C {cp!r}"


@pytest.mark.parametrize("ftype,cname", [("lce_params", "lce_params"), ("lce_meas", "lce_meas")])
def test_derived_types_mirror_the_c_structs(ftype, cname):
    mod = _fortran_module()
    m = re.search(r"type, bind\(c\) :: %s\n(.*?)\n\s*end type" % ftype, mod, re.S)
    assert m, ftype
    fields = []
    for line in m.group(1).splitlines():
        line = line.split("!")[0].strip()
        if not line:
            continue
        dm = re.match(r"((?:integer|real)\(\w+\))\s*::\s*(.*)", line)
        assert dm, line
        for v in dm.group(2).split(","):
            v = v.strip()
            vn = re.match(r"(\w+)(?:\((\d+)\))?", v)
            fields.append((vn.group(1), F_KIND[dm.group(1)], int(vn.group(2) or 1)))
    cfields = _c_struct(cname)
    assert [(n, k) for n, _, k in fields] == [(n, k) for n, _, k in cfields]
    for (fn, fk, _), (cn, ck, _) in zip(fields, cfields):
        assert fn == cn
        assert fk == ck or (fk, ck) == ("unsigned long long", "unsigned long long"), (fn, fk, ck)
