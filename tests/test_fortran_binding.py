"""The Fortran binding module agrees with the C header, entry point by entry
point and field by field.

fortran/rp_gpu_mod.f90 is what the kept Fortran driver compiles to call the
library (the call that replaces update_particles is at ROMSPath.f90:529).
No Fortran compiler exists here, so this test reads both files as text:

* every function of include/romspath_gpu.h has one bind(C) interface with
  the same name, the same arguments in the same order (names compared
  without case) and a compatible Fortran declaration for each: a C scalar
  as a value argument of the same kind, rp_ctx* as type(c_ptr) by value,
  rp_ctx** and struct pointers by reference, data pointers as assumed-size
  arrays (or scalars) of the same kind or, where C may take NULL, as
  type(c_ptr) by value;
* every struct of the header has a bind(C) type with the same fields in
  the same order, and the C layout rules give both the same size and the
  same offset for every field -- which also equal the ctypes mirrors the
  Python side uses.
"""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "romspath_gpu.h")
MODULE = os.path.join(ROOT, "fortran", "rp_gpu_mod.f90")

C_SCALAR = {"int32_t": ("int", 4), "uint32_t": ("int", 4), "int64_t": ("int", 8), "uint64_t": ("int", 8),
            "double": ("real", 8), "float": ("real", 4), "char": ("char", 1), "int8_t": ("int", 1),
            "void": ("void", 0), "int": ("int", 4)}
F_KIND = {"integer(c_int32_t)": ("int", 4), "integer(c_int64_t)": ("int", 8), "integer(c_int)": ("int", 4),
          "real(c_double)": ("real", 8), "real(c_float)": ("real", 4), "character(kind=c_char)": ("char", 1)}
STRUCTS = ("rp_params", "rp_grid", "rp_frame", "rp_behavior", "rp_device_state", "rp_adj_step")
MACROS = {"RP_MAXNGRID": 5}


def _header():
    s = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    funcs = {}
    for m in re.finditer(r"\n(int|const char \*)\s*(rp_\w+)\s*\(([^)]*)\);", s):
        ret, name, args = m.group(1), m.group(2), " ".join(m.group(3).split())
        out = []
        if args != "void":
            for a in args.split(","):
                a = a.strip()
                dims = re.findall(r"\[(\w+)\]", a)
                a = re.sub(r"\[\w+\]", "", a)
                mm = re.match(r"(?:const\s+)?(\w+)\s*((?:\*\s*(?:const\s*)?)*)\s*(\w+)$", a)
                assert mm, a
                base, stars, an = mm.group(1), mm.group(2).count("*"), mm.group(3)
                out.append((base, stars + len(dims), an))
        funcs[name] = (ret, out)
    structs = {}
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} \1;", s, flags=re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            mm = re.match(r"(?:const\s+)?(\w+)\s+(.*)$", decl)
            base, rest = mm.group(1), mm.group(2)
            for item in rest.split(","):
                item = item.strip()
                ptr = item.startswith("*")
                item = item.lstrip("*").strip()
                dm = re.match(r"(\w+)(?:\[(\w+)\])?$", item)
                nm, dim = dm.group(1), dm.group(2)
                count = int(MACROS.get(dim, dim)) if dim else 1
                size = 8 if ptr else C_SCALAR[base][1]
                fields.append((nm, size, size, count))
        structs[m.group(1)] = fields
    return funcs, structs


def _module():
    src = open(MODULE).read()
    src = re.sub(r"!.*", "", src)
    src = re.sub(r"&\s*\n\s*", " ", src)
    lines = [" ".join(ln.split()) for ln in src.split("\n") if ln.strip()]
    funcs, types = {}, {}
    cur, kind = None, None
    for ln in lines:
        low = ln.lower()
        m = re.match(r"(integer\(c_int\)|type\(c_ptr\)) function (\w+)\(([^)]*)\) bind\(c, name=\"(\w+)\"\)", low)
        if m:
            assert m.group(2) == m.group(4), ln
            args = [a.strip() for a in m.group(3).split(",") if a.strip()]
            cur = {"ret": m.group(1), "args": args, "decl": {}}
            funcs[m.group(2)] = cur
            kind = "f"
            continue
        m = re.match(r"type, bind\(c\) :: (\w+)", low)
        if m:
            cur = {"fields": []}
            types[m.group(1)] = cur
            kind = "t"
            continue
        if low.startswith("end function") or low.startswith("end type"):
            cur, kind = None, None
            continue
        if cur is None or low.startswith("import"):
            continue
        m = re.match(r"([a-z_]+\([^)]*\))((?:,\s*[a-z]+(?:\([a-z]+\))?)*)\s*::\s*(.*)$", low)
        if not m:
            continue
        ftype, attrs, names = m.group(1), m.group(2), m.group(3)
        value = "value" in attrs
        for item in re.findall(r"(\w+)(\([^)]*\))?", names):
            nm, dim = item[0], item[1].strip("()") if item[1] else ""
            if kind == "f":
                cur["decl"][nm] = (ftype, value, dim)
            else:
                count = int(MACROS.get(dim.upper(), dim)) if dim else 1
                cur["fields"].append((nm, ftype, count))
    return funcs, types


def _f_size(ftype):
    if ftype == "type(c_ptr)":
        return 8
    return F_KIND[ftype][1]


def _layout(fields):
    """(name, offset, size) of each field and the struct size, C rules."""
    off, out, align = 0, [], 1
    for nm, size, al, count in fields:
        off = (off + al - 1) // al * al
        out.append((nm, off, size * count))
        off += size * count
        align = max(align, al)
    return out, (off + align - 1) // align * align


def test_every_entry_point_is_bound_with_matching_arguments():
    hfun, _ = _header()
    ffun, _ = _module()
    assert set(ffun) == set(hfun), (set(hfun) ^ set(ffun))
    for name, (ret, cargs) in hfun.items():
        f = ffun[name]
        assert f["ret"] == ("type(c_ptr)" if ret.startswith("const char") else "integer(c_int)"), name
        assert [a.lower() for _, _, a in cargs] == f["args"], name
        for (base, depth, an), fa in zip(cargs, f["args"]):
            ftype, value, dim = f["decl"][fa]
            where = f"{name}({an})"
            if base == "rp_ctx":
                assert ftype == "type(c_ptr)" and value == (depth == 1), where
            elif base in STRUCTS:
                assert depth == 1 and ftype == f"type({base})" and not value, where
            elif depth == 0:
                assert value and F_KIND[ftype] == C_SCALAR[base], where
            elif depth == 2:                       # const double *const *: an array of pointers
                assert ftype == "type(c_ptr)" and not value and dim == "*", where
            elif ftype == "type(c_ptr)":           # a pointer C may take as NULL
                assert value, where
            else:
                assert not value and F_KIND[ftype] == C_SCALAR[base], where
                if base == "char":
                    assert dim == "*", where


@pytest.mark.parametrize("struct", STRUCTS)
def test_struct_layouts_match(struct):
    from romspath_b200 import _lib
    _, hst = _header()
    _, ftypes = _module()
    hfields = hst[struct]
    ffields = [(nm, _f_size(ft), _f_size(ft), n) for nm, ft, n in ftypes[struct]["fields"]]
    assert [f[0].lower() for f in hfields] == [f[0] for f in ffields], struct
    hl, hsize = _layout(hfields)
    fl, fsize = _layout(ffields)
    assert [(o, s) for _, o, s in hl] == [(o, s) for _, o, s in fl], struct
    assert hsize == fsize, struct
    mirror = {"rp_params": _lib.RpParams, "rp_grid": _lib.RpGrid, "rp_frame": _lib.RpFrame,
              "rp_behavior": _lib.RpBehavior, "rp_device_state": _lib.RpDeviceState,
              "rp_adj_step": _lib.RpAdjStep}[struct]
    assert C.sizeof(mirror) == hsize, struct
    offs = [getattr(mirror, nm).offset for nm, _ in mirror._fields_]
    assert offs == [o for _, o, _ in hl], struct
