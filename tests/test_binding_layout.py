"""The struct mirrors of the C ABI against the library as compiled (CPU).

Three descriptions of each struct of include/xcal_b200.h must agree:
  * the library's own sizeof / offsetof (xcal_abi_layout, no device needed);
  * the ctypes mirror in xcalibre.jl_b200/_abi.py (what these tests use);
  * the Julia mirror in ext/XCALibre_B200Ext.jl (what XCALibre.jl's package
    extension passes to ccall), parsed from its struct declarations and laid
    out by the C rules Julia follows for isbits structs.
Field names and order are compared with the header's own declarations.  A
mirror that drifts from the header (a missing `dim`, a field out of order)
fails here instead of passing wrong memory at run time.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "xcal_b200.h")
JULIA_EXT = os.path.join(ROOT, "ext", "XCALibre_B200Ext.jl")

# (xcal_abi_layout selector, C typedef, ctypes class in _abi, Julia struct)
STRUCTS = [
    (0, "xcal_mesh_desc", "MeshDesc", "MeshDesc"),
    (1, "xcal_bc", "BCDesc", "BCDesc"),
    (2, "xcal_solver_setup", "SolverSetupDesc", "SolverSetupDesc"),
    (3, "xcal_schemes", "SchemesDesc", "SchemesDesc"),
    (4, "xcal_config", "ConfigDesc", "ConfigDesc"),
    (5, "xcal_polymesh_desc", "PolyMeshDesc", None),
    (6, "xcal_mesh_buffers", "MeshBuffers", None),
    (7, "xcal_term", "TermDesc", "TermDesc"),
    (8, "xcal_source", "SourceDesc", "SourceDesc"),
]


def header_fields(name):
    """Field names of `typedef struct { ... } name;` in declaration order."""
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    bodies = {m.group(2): m.group(1) for m in re.finditer(r"typedef struct \{([^{}]*)\}\s*(\w+)\s*;", src)}
    assert name in bodies, name
    names = []
    for decl in bodies[name].split(";"):
        decl = decl.strip()
        if not decl:
            continue
        # "double a, b, c" / "const xcal_bc* bc_U" / "double value[3]"
        head, *rest = [d.strip() for d in decl.split(",")]
        first = re.findall(r"([A-Za-z_]\w*)\s*(?:\[\d+\])?$", head)
        names.append(first[0])
        for r in rest:
            names.append(re.match(r"\**\s*([A-Za-z_]\w*)", r).group(1))
    return names


def julia_structs():
    """{struct name: [(field, type string)]} of ext/XCALibre_B200Ext.jl."""
    src = open(JULIA_EXT).read()
    out = {}
    for m in re.finditer(r"^struct (\w+)\n(.*?)^end", src, flags=re.S | re.M):
        fields = []
        for ln in m.group(2).splitlines():
            ln = ln.split("#")[0].strip()
            if ln:
                f, t = ln.split("::")
                fields.append((f.strip(), t.strip()))
        out[m.group(1)] = fields
    return out


def julia_layout(name, structs, memo):
    """(size, alignment, [offsets]) of a Julia isbits struct, C rules."""
    if name in memo:
        return memo[name]
    prim = {"Int32": (4, 4), "Int64": (8, 8), "Float64": (8, 8), "Float32": (4, 4), "UInt8": (1, 1)}

    def size_align(t):
        if t in prim:
            return prim[t]
        if t.startswith("Ptr{"):
            return 8, 8
        m = re.fullmatch(r"NTuple\{(\d+),\s*(\w+)\}", t)
        if m:
            s, a = size_align(m.group(2))
            return int(m.group(1)) * s, a
        s, a, _ = julia_layout(t, structs, memo)
        return s, a

    off, align, offs = 0, 1, []
    for _, t in structs[name]:
        s, a = size_align(t)
        off = (off + a - 1) // a * a
        offs.append(off)
        off += s
        align = max(align, a)
    size = (off + align - 1) // align * align
    memo[name] = (size, align, offs)
    return memo[name]


@pytest.fixture(scope="module")
def lib():
    from importlib import import_module
    import __graft_entry__ as ge
    ge.load_package()
    return import_module("xcalibre_b200._lib").lib()


def library_layout(lib, which):
    buf = (C.c_int64 * 128)()
    n = lib.xcal_abi_layout(which, buf, 128)
    assert n > 1, (which, n)
    return int(buf[0]), [int(v) for v in buf[1:n]]


@pytest.mark.parametrize("which,cname,pyname,jlname", STRUCTS)
def test_ctypes_mirror_matches_library(lib, x, which, cname, pyname, jlname):
    size, offs = library_layout(lib, which)
    cls = getattr(x._abi, pyname)
    names = [f[0] for f in cls._fields_]
    assert names == header_fields(cname), (cname, names)
    assert C.sizeof(cls) == size, (cname, C.sizeof(cls), size)
    assert [getattr(cls, n).offset for n in names] == offs, cname


@pytest.mark.parametrize("which,cname,pyname,jlname", [s for s in STRUCTS if s[3]])
def test_julia_mirror_matches_library(lib, which, cname, pyname, jlname):
    structs = julia_structs()
    assert jlname in structs, jlname
    assert [f for f, _ in structs[jlname]] == header_fields(cname), cname
    size, offs = library_layout(lib, which)
    jsize, _, joffs = julia_layout(jlname, structs, {})
    assert jsize == size, (cname, jsize, size)
    assert joffs == offs, (cname, joffs, offs)


def test_layout_rejects_unknown_and_short(lib):
    buf = (C.c_int64 * 4)()
    assert lib.xcal_abi_layout(99, buf, 4) < 0
    assert lib.xcal_abi_layout(4, buf, 4) < 0     # xcal_config needs more room


def test_julia_mirror_catches_a_drift():
    """The parse-and-lay-out check sees a field dropped from a mirror (the
    shape of a stale MeshDesc without `dim`)."""
    structs = julia_structs()
    bad = dict(structs)
    bad["MeshDesc"] = [f for f in structs["MeshDesc"] if f[0] != "dim"]
    assert [f for f, _ in bad["MeshDesc"]] != header_fields("xcal_mesh_desc")
    assert julia_layout("MeshDesc", bad, {})[0] < julia_layout("MeshDesc", structs, {})[0]
    assert np.all(np.diff(julia_layout("MeshDesc", structs, {})[2]) > 0)
