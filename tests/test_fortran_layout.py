"""The Fortran binding's bind(C) derived types against the C structs.

include/mfcfd_b200_mod.F90 declares mfcfd_grid and mfcfd_params as
``type, bind(C)`` copies of the C structs of include/mfcfd_b200.h.  No Fortran
compiler exists here, so the test lays the Fortran types out as ISO_C_BINDING
requires (the companion C struct's layout: fields in declaration order,
c_int 4, c_double 8 and c_ptr 8 bytes, each naturally aligned) and compares
field names, offsets and sizes with the C compiler's offsetof/sizeof of the
header's structs, and with the ctypes mirror the Python host uses.
"""
import os
import re
import shutil
import subprocess

import pytest

from mfcfd_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "include", "mfcfd_b200_mod.F90")
KINDS = {"integer(c_int)": 4, "real(c_double)": 8, "type(c_ptr)": 8}


def fortran_types():
    """{type name: [(field, size)]} of the bind(C) types, declaration order."""
    text = open(F90).read()
    out = {}
    for name, body in re.findall(r"type\s*,\s*bind\(C\)\s*::\s*(\w+)(.*?)end type", text,
                                 re.S | re.I):
        fields = []
        for line in body.splitlines():
            line = line.split("!", 1)[0].strip()
            if not line:
                continue
            m = re.match(r"(integer\(c_int\)|real\(c_double\)|type\(c_ptr\))\s*::\s*(.*)", line,
                         re.I)
            assert m, f"unparsed line in {name}: {line!r}"
            size = KINDS[m.group(1).lower()]
            fields += [(f.strip(), size) for f in m.group(2).split(",")]
        out[name] = fields
    return out


def c_layout(fields):
    """(offsets, size) of a C struct with these members (natural alignment)."""
    off, offsets, align = 0, {}, 1
    for name, size in fields:
        off = (off + size - 1) // size * size
        offsets[name] = off
        off += size
        align = max(align, size)
    return offsets, (off + align - 1) // align * align


def compiled_layout(struct, fields):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = [f'printf("{f} %zu\\n", offsetof({struct}, {f}));' for f, _ in fields]
    src = ("#include <stdio.h>\n#include <stddef.h>\n#include \"mfcfd_b200.h\"\nint main(void){"
           + "".join(lines) + f'printf("sizeof %zu\\n", sizeof({struct})); return 0;}}\n')
    work = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"layout_{struct}_{os.getpid()}")
    os.makedirs(work, exist_ok=True)
    with open(os.path.join(work, "l.c"), "w") as fh:
        fh.write(src)
    exe = os.path.join(work, "l")
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(work, "l.c")], check=True, capture_output=True)
    res = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    vals = dict(line.split() for line in res.strip().splitlines())
    return {k: int(v) for k, v in vals.items()}


@pytest.mark.parametrize("struct,ctype", [("mfcfd_grid", _lib.Grid),
                                          ("mfcfd_params", _lib.Params)])
def test_bind_c_types_match_the_header(struct, ctype):
    ftypes = fortran_types()
    assert struct in ftypes, f"{struct} not declared bind(C) in the Fortran module"
    fields = ftypes[struct]
    offsets, size = c_layout(fields)
    got = compiled_layout(struct, fields)  # fails to compile if a name differs
    for f, _ in fields:
        assert got[f] == offsets[f], f"{struct}.{f}: C offset {got[f]}, Fortran {offsets[f]}"
    assert got["sizeof"] == size
    # the ctypes mirror: same names in the same order at the same offsets
    assert [n for n, _ in ctype._fields_] == [f for f, _ in fields]
    for f, _ in fields:
        assert getattr(ctype, f).offset == offsets[f], f
    assert __import__("ctypes").sizeof(ctype) == size
