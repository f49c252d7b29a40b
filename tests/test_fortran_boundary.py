"""The Fortran bind(C) module (fortran/gamgpu_mod.F90) matches the C ABI (include/gamgpu.h).

No Fortran compiler exists on this image, so the module is checked by reading it: every bind(C) derived
type has the C struct's fields in the same order with the same C types and array lengths, and its C
layout (offsets and size, computed with the C alignment rules that bind(C) follows) equals the struct's
as gcc lays it out (an offsetof table compiled from the header); every bind(C) interface names a function
the header declares, with the same number of arguments, passing each by value or by reference as the
C prototype does.
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gamgpu.h")
FMOD = os.path.join(ROOT, "fortran", "gamgpu_mod.F90")
STRUCTS = ("gam_model_c", "gam_grid_c", "gam_status_c")
# C type -> (size, alignment); bind(C) kinds map onto them
CTYPES = {"int": (4, 4), "unsigned": (4, 4), "double": (8, 8), "ptr": (8, 8), "long long": (8, 8)}
FKIND = {"integer(c_int)": "int", "real(c_double)": "double", "type(c_ptr)": "ptr",
         "integer(c_long_long)": "long long"}


def _strip_c(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def c_struct_fields(name):
    text = _strip_c(open(HEADER).read())
    m = re.search(r"typedef\s+struct\s*\{([^{}]*)\}\s*" + name + r"\s*;", text)
    assert m, name
    fields = []
    for decl in m.group(1).split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        mm = re.match(r"(const\s+)?(unsigned long long|long long|unsigned int|unsigned|int|double)\s*(\*?)\s*(.*)",
                      decl)
        assert mm, decl
        base = mm.group(2)
        for item in mm.group(4).split(","):
            item = item.strip()
            ptr = mm.group(3) == "*" or item.startswith("*")
            item = item.lstrip("*").strip()
            am = re.match(r"(\w+)\s*(?:\[(\d+)\])?$", item)
            assert am, item
            kind = "ptr" if ptr else ("int" if base in ("unsigned int", "unsigned") else base)
            fields.append((am.group(1).lower(), kind, int(am.group(2) or 1)))
    return fields


def fortran_type_fields(name):
    text = open(FMOD).read()
    m = re.search(r"type\s*,\s*bind\(C\)\s*::\s*" + name + r"\s*\n(.*?)end type " + name, text, flags=re.S | re.I)
    assert m, name
    fields = []
    for line in m.group(1).splitlines():
        line = line.split("!")[0].strip()
        if not line:
            continue
        decl, names = [s.strip() for s in line.split("::", 1)]
        kind = FKIND[decl.lower().replace(" ", "")]
        for item in re.split(r",(?![^(]*\))", names):
            item = item.split("=")[0].strip()
            am = re.match(r"(\w+)\s*(?:\((\d+)\))?$", item)
            assert am, item
            fields.append((am.group(1).lower(), kind, int(am.group(2) or 1)))
    return fields


def c_layout(fields):
    off, offs, align = 0, [], 1
    for _, kind, n in fields:
        size, al = CTYPES[kind]
        off = (off + al - 1) // al * al
        offs.append(off)
        off += size * n
        align = max(align, al)
    return offs, (off + align - 1) // align * align


@pytest.fixture(scope="module")
def gcc_layouts(tmp_path_factory):
    d = tmp_path_factory.mktemp("offsets")
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "gamgpu.h"', "int main(void) {"]
    for s in STRUCTS:
        src.append(f'printf("{s} size %zu\\n", sizeof({s}));')
        for fname, _, _ in c_struct_fields(s):
            real = next(f for f in re.findall(r"\w+", _strip_c(open(HEADER).read())) if f.lower() == fname)
            src.append(f'printf("{s} {fname} %zu\\n", offsetof({s}, {real}));')
    src.append("return 0; }")
    (d / "off.c").write_text("\n".join(src))
    exe = d / "off"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(d / "off.c"), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    tab = {}
    for line in out.splitlines():
        s, f, v = line.split()
        tab[(s, f)] = int(v)
    return tab


@pytest.mark.parametrize("name", STRUCTS)
def test_fortran_type_matches_c_struct(name, gcc_layouts):
    cf, ff = c_struct_fields(name), fortran_type_fields(name)
    assert [f[0] for f in ff] == [f[0] for f in cf], "field order"
    assert ff == cf, "types / array lengths"
    offs, size = c_layout(ff)
    assert size == gcc_layouts[(name, "size")]
    for (fname, _, _), off in zip(ff, offs):
        assert off == gcc_layouts[(name, fname)], fname


def c_prototypes():
    text = _strip_c(open(HEADER).read())
    protos = {}
    for m in re.finditer(r"\b(?:int|void|long long|const char\*)\s+\**(gam_\w+)\s*\(([^)]*)\)\s*;", text):
        params = [" ".join(p.split()) for p in m.group(2).split(",") if p.strip() and p.strip() != "void"]
        protos[m.group(1)] = params
    return protos


def fortran_interfaces():
    text = open(FMOD).read()
    body = re.search(r"\binterface\b(.*?)\bend interface\b", text, flags=re.S | re.I).group(1)
    out = {}
    for m in re.finditer(r"(?:function|subroutine)\s+(\w+)\s*\(([^)]*)\)[^\n]*?(?:&\s*\n\s*)?bind\(C,\s*name=\"(\w+)\"\)"
                         r"(.*?)end (?:function|subroutine)", body, flags=re.S | re.I):
        args = [a.strip().lower() for a in m.group(2).replace("&", " ").split(",") if a.strip()]
        decls = {}
        for line in m.group(4).splitlines():
            line = line.split("!")[0].strip()
            if "::" not in line or line.lower().startswith("import"):
                continue
            attrs, names = [s.strip().lower() for s in line.split("::", 1)]
            for nm in re.split(r",(?![^(]*\))", names):
                decls[nm.split("(")[0].strip()] = attrs
        out[m.group(3)] = (args, decls)
    return out


def test_fortran_interfaces_match_prototypes():
    protos, ifaces = c_prototypes(), fortran_interfaces()
    assert len(ifaces) >= 30
    for cname, (args, decls) in ifaces.items():
        assert cname in protos, cname
        params = protos[cname]
        assert len(args) == len(params), (cname, args, params)
        for a, p in zip(args, params):
            attrs = decls[a]
            by_value = "value" in attrs
            is_ptr = "*" in p
            if is_ptr:   # an address: a Fortran argument by reference, or a c_ptr passed by value
                assert (not by_value) or attrs.startswith("type(c_ptr)"), (cname, a, p, attrs)
            else:        # a scalar: by value, with the matching kind
                assert by_value, (cname, a, p, attrs)
                if p.startswith("double"):
                    assert attrs.startswith("real(c_double)"), (cname, a, p)
                elif p.startswith("long long"):
                    assert attrs.startswith("integer(c_long_long)"), (cname, a, p)
                else:
                    assert attrs.startswith("integer(c_int)"), (cname, a, p)
