"""The Fortran iso_c_binding layer against the C header and the Python mirror (text checks, CPU).

No Fortran compiler is on this image, so the bind(C) module
(more_benchmarks_dc_ocean_b200/fortran/redi_b200_c.F90) cannot be compiled
here. These tests hold it to the C-ABI instead: every bind(C) derived type has
the fields of its C struct in include/redi_b200.h, in the same order, with
matching kinds (integer(c_int) = int, real(c_double) = double, type(c_ptr) =
any pointer), and the same fields as the ctypes structure ocean_redi.py passes;
every bound procedure is declared in the header and exported by the library.
"""

import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "more_benchmarks_dc_ocean_b200", "fortran", "redi_b200_c.F90")
DROPIN = os.path.join(ROOT, "more_benchmarks_dc_ocean_b200", "fortran", "ocean_redi.F90")
HEADER = os.path.join(ROOT, "include", "redi_b200.h")
LIB = os.path.join(ROOT, "more_benchmarks_dc_ocean_b200", "libredi_b200.so")

KIND = {"integer(c_int)": "int", "real(c_double)": "double", "type(c_ptr)": "ptr"}


def _strip_f90(text):
    return "\n".join(line.split("!")[0] for line in text.splitlines())


def fortran_types():
    """{type name: [(field, kind)]} of every `type, bind(C)` block."""
    src = _strip_f90(open(F90).read())
    out = {}
    for m in re.finditer(r"type\s*,\s*bind\(C\)[^:]*::\s*(\w+)(.*?)end\s+type", src, re.S | re.I):
        fields = []
        for line in m.group(2).splitlines():
            line = line.strip()
            if not line:
                continue
            decl, names = line.split("::")
            kind = KIND[decl.strip().lower().replace(" ", "")]
            fields += [(n.strip(), kind) for n in names.split(",")]
        out[m.group(1)] = fields
    return out


def c_structs():
    """{struct name: [(field, kind)]} of every typedef struct in the header."""
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*(\w+)\s*;", src, re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            base = re.match(r"(const\s+)?(int|double|\w+)", decl).group(2)
            for part in decl[len(re.match(r"(const\s+)?\w+", decl).group(0)):].split(","):
                part = part.strip()
                name = re.sub(r"[*\s]|const", "", part)
                if "*" in part or base not in ("int", "double"):
                    kind = "ptr" if "*" in part else base
                else:
                    kind = base
                fields.append((name, kind))
        out[m.group(3)] = fields
    return out


def test_bind_c_types_match_the_header_field_by_field():
    ft, cs = fortran_types(), c_structs()
    assert set(ft) == {"redi_b200_grid", "redi_b200_metrics", "redi_b200_eos", "redi_b200_state", "redi_b200_bc",
                       "redi_b200_coeffs"}
    for name, fields in ft.items():
        assert name in cs, name
        assert [(n.lower(), k) for n, k in fields] == [(n.lower(), k) for n, k in cs[name]], name


def test_bind_c_types_match_the_python_mirror():
    from more_benchmarks_dc_ocean_b200 import ocean_redi as R

    mirror = {"redi_b200_grid": R._Grid, "redi_b200_metrics": R._Metrics, "redi_b200_eos": R._Eos,
              "redi_b200_state": R._State, "redi_b200_bc": R._BC, "redi_b200_coeffs": R._Coeffs}
    for name, fields in fortran_types().items():
        py = [f[0].lower() for f in mirror[name]._fields_]
        assert [n.lower() for n, _ in fields] == py, name


def test_bound_procedures_are_declared_and_exported():
    src = _strip_f90(open(F90).read())
    names = re.findall(r'bind\(C,\s*name="(\w+)"\)', src)
    assert len(names) >= 9
    header = open(HEADER).read()
    for n in names:
        assert re.search(rf"\b{n}\s*\(", header), n
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    syms = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in syms.splitlines() if line.strip()}
    for n in names:
        assert n in exported, n


def test_drop_in_module_keeps_the_reference_public_names():
    src = _strip_f90(open(DROPIN).read()).lower()
    assert re.search(r"^\s*module\s+ocean_redi\s*$", src, re.M)
    for name in ("ocean_redi_t", "redi_calc_coeffs", "redi_apply_flux"):
        assert re.search(rf"public\s*::\s*{name}\b", src), name
    # argument lists of the two entry points (redi/ocean_redi.F90:572, 927)
    assert re.search(r"subroutine\s+redi_calc_coeffs\(grid,\s*metrics,\s*eos,\s*this,\s*ms\)", src)
    assert re.search(r"subroutine\s+redi_apply_flux\(grid,\s*metrics,\s*this,\s*ms,\s*dt,\s*khtr_u_ext,\s*"
                     r"khtr_v_ext,\s*bc\)", src)
    for tbp in ("init", "destroy", "enter_data", "exit_data"):
        assert re.search(rf"procedure.*::\s*{tbp}\s*=>", src), tbp
