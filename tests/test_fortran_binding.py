"""The Fortran ISO_C_BINDING module (include/mps_linsolve_c.f90) against the C
header (include/mps_linsolve.h).

No Fortran compiler exists in this image, so the module is checked the way a
compiler would lay it out: bind(C) derived types follow the companion C
compiler's rules, so the offsets computed from the module's component list
must equal the offsets gcc reports for the header's structs.  Every function
the header declares must have a bind(C) interface with the same name and
argument count.
"""
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "include", "mps_linsolve_c.f90")
HDR = os.path.join(ROOT, "include", "mps_linsolve.h")

KINDS = {"integer(c_int)": (4, 4), "real(c_double)": (8, 8), "type(c_ptr)": (8, 8),
         "integer(c_long_long)": (8, 8)}


def _strip(src):
    return "\n".join(line.split("!")[0] for line in src.splitlines())


def fortran_types():
    src = _strip(open(F90).read())
    types = {}
    for m in re.finditer(r"type,\s*bind\(C\)\s*::\s*(\w+)(.*?)end type", src, re.S | re.I):
        name, body = m.group(1), m.group(2)
        comps = []
        for line in body.splitlines():
            line = line.strip()
            if not line:
                continue
            kind, names = [x.strip() for x in line.split("::")]
            for nm in [x.strip() for x in re.split(r",(?![^()]*\))", names)]:
                mm = re.match(r"(\w+)(?:\((\d+)\))?$", nm)
                comps.append((mm.group(1), kind.lower(), int(mm.group(2) or 1)))
        types[name] = comps
    return types


def layout(types, name):
    """(offsets, size, align) of a bind(C) type by the C layout rules."""
    off, align, out = 0, 1, {}
    for comp, kind, count in types[name]:
        if kind.startswith("type(mps_"):
            sub = kind[len("type("):-1]
            _, size, a = layout(types, sub)
        else:
            size, a = KINDS[kind]
        off = (off + a - 1) // a * a
        out[comp] = off
        off += size * count
        align = max(align, a)
    size = (off + align - 1) // align * align
    return out, size, align


def c_layout(struct, members):
    prog = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HDR}"', "int main(void){"]
    prog.append(f'printf("sizeof %zu\\n", sizeof({struct}));')
    for m in members:
        prog.append(f'printf("{m} %zu\\n", offsetof({struct}, {m}));')
    prog.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(c, "w").write("\n".join(prog))
        subprocess.check_call(["gcc", "-std=c11", "-o", exe, c])
        out = subprocess.check_output([exe], text=True)
    vals = dict(line.split() for line in out.strip().splitlines())
    return {k: int(v) for k, v in vals.items()}


@pytest.mark.parametrize("name", ["mps_grid", "mps_solver_opts", "mps_solve_info", "mps_profile", "mps_problem",
                                  "mps_plasma_step"])
def test_bind_c_types_match_header_layout(name):
    types = fortran_types()
    assert name in types, f"{name} missing from the Fortran module"
    offs, size, _ = layout(types, name)
    got = c_layout(name, list(offs))
    assert got.pop("sizeof") == size
    assert got == offs


def _header_functions():
    src = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    funcs = {}
    for m in re.finditer(r"^[\w\s\*]*?\b(mps_\w+)\s*\(([^;{]*?)\)\s*;", src, re.M | re.S):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        funcs[m.group(1)] = len(args)
    return funcs


def _fortran_functions():
    src = _strip(open(F90).read()).replace("&\n", " ")
    funcs = {}
    for m in re.finditer(r"(?:function|subroutine)\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)", src):
        args = [a for a in m.group(2).split(",") if a.strip()]
        assert m.group(1) == m.group(3)
        funcs[m.group(3)] = len(args)
    return funcs


def test_every_header_function_has_a_fortran_interface():
    hdr = _header_functions()
    f90 = _fortran_functions()
    assert len(hdr) >= 21
    missing = sorted(set(hdr) - set(f90))
    assert not missing, missing
    for name, n in hdr.items():
        assert f90[name] == n, (name, f90[name], n)
