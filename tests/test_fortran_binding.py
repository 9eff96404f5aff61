"""The Fortran binding (fortran/smcrt_c.f90) against the C ABI (include/smcrt.h),
checked without a Fortran compiler: every bind(C) derived type has the size and
component offsets of its C struct (C layout rules applied to the Fortran
components, compared with a gcc probe of the header), and every C entry point
has a bind(C) interface of the same name, return kind and arity whose arguments
pass the way the C parameters do (scalars by value with the matching kind,
pointers by address or as a type(c_ptr) value)."""
import json
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
MODULE = ROOT / "fortran" / "smcrt_c.f90"
HEADER = ROOT / "include" / "smcrt.h"

KIND_SIZE = {"c_int32_t": 4, "c_int64_t": 8, "c_double": 8, "c_float": 4, "c_ptr": 8, "c_size_t": 8}


def _source_lines(path):
    """Fortran statements with comments stripped and continuation lines joined."""
    out, cur = [], ""
    for raw in path.read_text().splitlines():
        line = raw.split("!")[0].rstrip()
        if not line.strip():
            continue
        if cur:
            line = line.lstrip().lstrip("&")
        if line.endswith("&"):
            cur += line[:-1] + " "
            continue
        out.append((cur + line).strip())
        cur = ""
    return out


def fortran_types():
    """name -> [(component, kind, element count)] of every bind(C) derived type."""
    types, cur = {}, None
    for st in _source_lines(MODULE):
        m = re.match(r"type\s*,\s*bind\(C\)\s*::\s*(\w+)", st, re.I)
        if m:
            cur = m.group(1).lower()
            types[cur] = []
            continue
        if cur and re.match(r"end\s*type", st, re.I):
            cur = None
            continue
        if cur:
            m = re.match(r"(integer|real|type)\((\w+)\)\s*::\s*(.*)", st, re.I)
            assert m, st
            kind = m.group(2).lower()
            for name, dims in re.findall(r"(\w+)(\([^)]*\))?", m.group(3)):
                n = 1
                if dims:
                    for d in dims.strip("()").split(","):
                        n *= int(d)
                types[cur].append((name.lower(), kind, n))
    return types


def fortran_layout(comps):
    off, layout, align = 0, {}, 1
    for name, kind, n in comps:
        size = KIND_SIZE[kind]
        align = max(align, size)
        off = (off + size - 1) // size * size
        layout[name] = off
        off += size * n
    return (off + align - 1) // align * align, layout


def c_layout(tmp_path, types):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "smcrt.h"', "int main(void){", 'printf("{");']
    for i, (name, comps) in enumerate(types.items()):
        lines.append(f'printf("{"," if i else ""}\\"{name}\\":{{\\"size\\":%zu", sizeof({name}));')
        for comp, _, _ in comps:
            lines.append(f'printf(",\\"{comp}\\":%zu", offsetof({name}, {comp}));')
        lines.append('printf("}");')
    lines += ['printf("}\\n");', "return 0;}"]
    src = tmp_path / "flayout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "flayout"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    return json.loads(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout)


def test_every_c_struct_has_an_interoperable_fortran_type(tmp_path):
    types = fortran_types()
    c_structs = set(re.findall(r"typedef struct (\w+) \{", HEADER.read_text()))
    assert c_structs == set(types), c_structs ^ set(types)
    layout = c_layout(tmp_path, types)
    for name, comps in types.items():
        size, offs = fortran_layout(comps)
        assert size == layout[name]["size"], name
        for comp, off in offs.items():
            assert off == layout[name][comp], (name, comp)


def c_functions():
    """name -> (return type, [(parameter text)])."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    out = {}
    for m in re.finditer(r"^(int32_t|int64_t|void|const char\*)\s+(smcrt_\w+)\(([^)]*)\);", text, re.M):
        params = [p.strip() for p in m.group(3).replace("\n", " ").split(",")]
        out[m.group(2)] = (m.group(1), [] if params == ["void"] else params)
    return out


def fortran_interfaces():
    """name -> (return kind or None, [(argument, kind, attributes, is_array)])."""
    lines = _source_lines(MODULE)
    out, i = {}, 0
    while i < len(lines):
        st = lines[i]
        m = re.match(r"(?:(integer|real|type)\((\w+)\)\s+)?(function|subroutine)\s+(\w+)\(([^)]*)\)\s*bind\(C,\s*"
                     r"name=\"(\w+)\"\)", st, re.I)
        if m:
            ret = m.group(2).lower() if m.group(3).lower() == "function" else None
            args = [a.strip().lower() for a in m.group(5).split(",") if a.strip()]
            decl = {}
            i += 1
            while not re.match(r"end\s+(function|subroutine)", lines[i], re.I):
                d = re.match(r"(integer|real|type)\((\w+)\)\s*(,[^:]*)?::\s*(.*)", lines[i], re.I)
                if d:
                    attrs = (d.group(3) or "").lower()
                    for ent in re.findall(r"(\w+)(\([^)]*\))?", d.group(4)):
                        decl[ent[0].lower()] = (d.group(2).lower(), attrs, bool(ent[1]))
                i += 1
            out[m.group(6)] = (ret, [(a,) + decl[a] for a in args])
        i += 1
    return out


C_VALUE_KIND = {"int32_t": "c_int32_t", "uint32_t": "c_int32_t", "int64_t": "c_int64_t", "uint64_t": "c_int64_t",
                "double": "c_double", "float": "c_float"}
C_RETURN_KIND = {"int32_t": "c_int32_t", "int64_t": "c_int64_t", "const char*": "c_ptr", "void": None}


@pytest.mark.parametrize("name", sorted(c_functions()))
def test_every_c_entry_point_has_a_matching_fortran_interface(name):
    ret, params = c_functions()[name]
    ifaces = fortran_interfaces()
    assert name in ifaces, f"no Fortran interface for {name}"
    fret, fargs = ifaces[name]
    assert fret == C_RETURN_KIND[ret], (name, ret, fret)
    assert len(fargs) == len(params), (name, params, fargs)
    for p, (arg, kind, attrs, is_array) in zip(params, fargs):
        pointer = "*" in p or "[" in p
        if pointer:
            # by address, or the pointer itself as a type(c_ptr) value
            assert "value" not in attrs or kind == "c_ptr", (name, p, arg)
        else:
            ctype = p.rsplit(" ", 1)[0].replace("const ", "").strip()
            assert "value" in attrs and kind == C_VALUE_KIND[ctype], (name, p, arg, kind, attrs)
