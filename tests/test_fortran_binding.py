"""The Fortran component module (monc_b200/fortran/gpudycore.F90) against the C header.

No Fortran compiler is available here, so the module is checked as text: the bind(C) derived
types mgpu_config and mgpu_reductions are parsed, laid out with the C rules a bind(C) type
follows (each component at the next multiple of its alignment, the size rounded up to the
largest alignment), and compared field by field -- name, kind, array length and byte offset --
with the structs of include/monc_gpu.h as gcc lays them out.  The C field list is parsed from
the header itself, so a field added to one side only fails here.  The interfaces the module
binds must name functions the header declares.
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "monc_gpu.h")
FORTRAN = os.path.join(ROOT, "monc_b200", "fortran", "gpudycore.F90")

C_KINDS = {"int32_t": ("i4", 4), "double": ("f8", 8)}
F_KINDS = {"integer(c_int32_t)": ("i4", 4), "real(c_double)": ("f8", 8)}


def _c_defines():
    out = {}
    for name, val in re.findall(r"#define\s+(MGPU_\w+)\s+\(?(\d+)", open(HEADER).read()):
        out[name] = int(val)
    return out


def c_struct(name):
    """[(field, kind, length)] of `typedef struct name {...} name;` in the header."""
    text = open(HEADER).read()
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    defs = _c_defines()
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        ctype, rest = decl.split(None, 1)
        kind = C_KINDS[ctype][0]
        for item in rest.split(","):
            item = item.strip()
            m = re.fullmatch(r"(\w+)(?:\[(\w+)\])?", item)
            assert m, f"unparsed C declarator {item!r}"
            n = m.group(2)
            length = 1 if n is None else (int(n) if n.isdigit() else defs[n])
            fields.append((m.group(1), kind, length))
    return fields


def f_type(name):
    """[(field, kind, length)] of `type, bind(C) :: name ... end type name` in the module."""
    text = open(FORTRAN).read()
    params = {k: int(v) for k, v in re.findall(r"\b(MGPU_MAX_\w+)\s*=\s*(\d+)", text)}
    body = re.search(r"type, bind\(C\) :: %s\n(.*?)\n\s*end type %s" % (name, name), text, re.S | re.I).group(1)
    fields = []
    for line in body.splitlines():
        line = line.split("!")[0].strip()
        if not line:
            continue
        ftype, names = (s.strip() for s in line.split("::"))
        kind = F_KINDS[ftype.replace(" ", "")][0]
        for item in re.findall(r"\w+(?:\([^)]*\))?", names):
            m = re.fullmatch(r"(\w+)(?:\((\w+)\))?", item)
            n = m.group(2)
            length = 1 if n is None else (int(n) if n.isdigit() else params[n])
            fields.append((m.group(1), kind, length))
    return fields


def c_layout(fields):
    """Offsets and size of a C struct of these fields (natural alignment)."""
    size = {"i4": 4, "f8": 8}
    off, offsets, align = 0, {}, 1
    for f, kind, length in fields:
        a = size[kind]
        off = (off + a - 1) // a * a
        offsets[f] = off
        off += a * length
        align = max(align, a)
    return offsets, (off + align - 1) // align * align


def gcc_offsets(tmp_path, struct, names):
    src = tmp_path / f"{struct}.c"
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "monc_gpu.h"', "int main(void){",
             f'printf("size %zu\\n", sizeof({struct}));']
    lines += [f'printf("{f} %zu\\n", offsetof({struct}, {f}));' for f in names]
    lines += ["return 0;}"]
    src.write_text("\n".join(lines))
    exe = tmp_path / struct
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    return {k: int(v) for k, v in (ln.split() for ln in out.strip().splitlines())}


@pytest.mark.parametrize("struct", ["mgpu_config", "mgpu_reductions"])
def test_fortran_type_matches_c_struct(tmp_path, struct):
    cf = c_struct(struct)
    ff = f_type(struct)
    assert [f for f, _, _ in ff] == [f for f, _, _ in cf], "field names or order differ"
    for (name, ck, cl), (_, fk, fl) in zip(cf, ff):
        assert (ck, cl) == (fk, fl), f"{struct}.{name}: C {ck}[{cl}] vs Fortran {fk}({fl})"
    f_off, f_size = c_layout(ff)
    g = gcc_offsets(tmp_path, struct, [f for f, _, _ in cf])
    assert f_size == g["size"], f"{struct}: Fortran layout {f_size} bytes, C {g['size']}"
    for name, _, _ in cf:
        assert f_off[name] == g[name], f"{struct}.{name}: offset {f_off[name]} vs {g[name]}"


def test_fortran_interfaces_bind_declared_functions():
    text = open(FORTRAN).read()
    bound = set(re.findall(r'bind\(C, name="(mgpu_\w+)"\)', text))
    header = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    declared = set(re.findall(r"\b(mgpu_\w+)\s*\(", header))
    assert bound, "no bound entry points"
    assert bound <= declared, sorted(bound - declared)
    for must in ("mgpu_config_defaults", "mgpu_create", "mgpu_step", "mgpu_upload_field", "mgpu_download_field",
                 "mgpu_destroy", "mgpu_last_error"):
        assert must in bound


def test_a_field_added_on_one_side_is_caught(tmp_path, monkeypatch):
    """The comparison fails when the header gains a field the module lacks."""
    fake = tmp_path / "monc_gpu.h"
    text = open(HEADER).read().replace("  double  ugal, vgal;                 /* the fixed frame",
                                       "  double  ugal, vgal, wgal;           /* the fixed frame")
    assert "wgal" in text
    fake.write_text(text)
    monkeypatch.setattr(__import__(__name__), "HEADER", str(fake))
    assert [f for f, _, _ in c_struct("mgpu_config")] != [f for f, _, _ in f_type("mgpu_config")]
