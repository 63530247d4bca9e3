"""The Fortran iso_c_binding module (fortran/gitm_vert_iface.f90) against the C
header it mirrors (include/gitm_vert.h), without a Fortran compiler.

Every `type, bind(C)` of the module is laid out with C's rules (each member
at the next multiple of its alignment; c_int32_t 4 bytes, c_int64_t, c_double
and c_ptr 8; nested bind(C) types by their own size and alignment), and every
member's offset and each type's size are compared with offsetof / sizeof of
the C struct of the same name, compiled here with gcc from the header.  The
routines the module binds must be declared in the header with the same
number of arguments.
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "fortran", "gitm_vert_iface.f90")
HEADER = os.path.join(ROOT, "include", "gitm_vert.h")
KINDS = {"integer(c_int32_t)": (4, 4), "integer(c_int)": (4, 4), "integer(c_int64_t)": (8, 8),
         "real(c_double)": (8, 8), "type(c_ptr)": (8, 8)}


def _logical_lines(text):
    """Fortran free-form lines with comments removed and '&' continuations joined."""
    out, cur = [], ""
    for raw in text.splitlines():
        line = raw.split("!", 1)[0].rstrip()
        if not line.strip():
            continue
        if cur:
            line = line.lstrip()
            if line.startswith("&"):
                line = line[1:]
        if line.endswith("&"):
            cur += line[:-1] + " "
            continue
        out.append(cur + line)
        cur = ""
    return out


def parse_types(text):
    """{type name: [(member, kind spec, count)]} for every bind(C) derived type."""
    types, cur = {}, None
    for line in _logical_lines(text):
        s = line.strip()
        m = re.match(r"type\s*,\s*bind\s*\(\s*c\s*\)\s*::\s*(\w+)", s, re.I)
        if m:
            cur = m.group(1)
            types[cur] = []
            continue
        if cur and re.match(r"end\s*type", s, re.I):
            cur = None
            continue
        if cur:
            kind, names = [x.strip() for x in s.split("::", 1)]
            kind = re.sub(r"\s+", "", kind).lower()
            for item in re.findall(r"(\w+)\s*(\(\s*\d+\s*\))?", names):
                name, dim = item
                count = int(dim.strip("() ")) if dim else 1
                types[cur].append((name, kind, count))
    return types


def layout(types):
    """{type: (size, align, {member: offset})} by C's rules."""
    res = {}

    def one(t):
        if t in res:
            return res[t]
        off, align, offs = 0, 1, {}
        for name, kind, count in types[t]:
            nested = re.match(r"type\((\w+)\)", kind)
            by_lower = {n.lower(): n for n in types}  # Fortran names are case-insensitive
            if nested and nested.group(1) in by_lower:
                sz, al, _ = one(by_lower[nested.group(1)])
            else:
                assert kind in KINDS, f"{t}.{name}: kind {kind} not handled"
                sz, al = KINDS[kind]
            off = -(-off // al) * al
            offs[name] = off
            off += sz * count
            align = max(align, al)
        size = -(-off // align) * align
        res[t] = (size, align, offs)
        return res[t]

    for t in types:
        one(t)
    return res


def c_layout(types, tmp_path):
    """offsetof / sizeof of the C structs of the header, compiled with gcc."""
    lines = ['#include <stddef.h>', '#include <stdio.h>', f'#include "{HEADER}"', "int main(void) {"]
    for t, members in types.items():
        lines.append(f'  printf("%s size %zu\\n", "{t}", sizeof({t}));')
        for name, _, _ in members:
            lines.append(f'  printf("%s %s %zu\\n", "{t}", "{name}", offsetof({t}, {name}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    exe = tmp_path / "layout"
    src.write_text("\n".join(lines))
    subprocess.run(["gcc", "-std=c99", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    sizes, offs = {}, {}
    for line in out.splitlines():
        a, b, c = line.split()
        if b == "size":
            sizes[a] = int(c)
        else:
            offs[(a, b)] = int(c)
    return sizes, offs


def test_bind_c_types_match_the_header(tmp_path):
    types = parse_types(open(F90).read())
    assert {"GitmVertParams", "GitmFArray", "GitmFortranState"} <= set(types)
    mine = layout(types)
    sizes, offs = c_layout(types, tmp_path)
    for t, (size, _, members) in mine.items():
        assert sizes[t] == size, f"{t}: C sizeof {sizes[t]} != Fortran layout {size}"
        for name, off in members.items():
            assert offs[(t, name)] == off, f"{t}.{name}: C offset {offs[(t, name)]} != Fortran {off}"


def test_every_member_of_the_c_structs_is_bound():
    """No C member is missing from the Fortran types (same member count)."""
    types = parse_types(open(F90).read())
    header = open(HEADER).read()
    for t in types:
        m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (t, t), header, re.S)
        assert m, t
        body = re.sub(r"/\*.*?\*/", "", m.group(1), flags=re.S)
        c_names = []
        for decl in body.split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            # "int32_t a, b, c", "GitmFArray x, y", "double t[6]", "double* p"
            c_names += [re.sub(r"\[.*\]", "", v).strip(" *") for v in decl.split(None, 1)[1].split(",")]
        f_names = [n for n, _, _ in types[t]]
        assert f_names == c_names, f"{t}: Fortran {f_names} != C {c_names}"


def test_bound_routines_are_declared_with_the_same_arity():
    text = open(F90).read()
    header = open(HEADER).read()
    found = 0
    for m in re.finditer(r"(?:function|subroutine)\s+(\w+)\s*\(([^)]*)\)[\s&]*bind\s*\(\s*C\s*,\s*name\s*=\s*\"(\w+)\"",
                         text, re.I):
        fname, fargs, cname = m.groups()
        nf = len([a for a in fargs.replace("&", " ").split(",") if a.strip()])
        d = re.search(r"\b%s\s*\(([^)]*)\)\s*;" % cname, header)
        assert d, f"{cname} is not declared in {os.path.basename(HEADER)}"
        nc = len([a for a in d.group(1).split(",") if a.strip() and a.strip() != "void"])
        assert nf == nc, f"{cname}: Fortran binds {nf} arguments, C declares {nc}"
        found += 1
    assert found >= 5
