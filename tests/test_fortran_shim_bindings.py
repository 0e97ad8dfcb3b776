"""The Fortran shim's ISO_C_BINDING interfaces against the C ABI they bind.

No Fortran compiler exists on either machine, so the shim (omm-bundle_b200/fortran/) is
checked here statically: every `bind(c, name="...")` interface block is parsed, each dummy
argument is reduced to how it crosses the C boundary (by value or by reference, and its C
type), and the result must agree, argument by argument, with the prototype of the same name
in include/ommgpu.h; the symbol must also be exported by the built library."""
import ctypes as ct
import os
import re

import pytest

import ommgpu as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "omm-bundle_b200", "fortran", "MatrixSwitch_gpu.F90")
HEADER = os.path.join(ROOT, "include", "ommgpu.h")


def fortran_interfaces():
    """{c_name: (return kind, [argument kinds])} of every bind(c) interface body in the shim."""
    src = open(SHIM).read()
    src = re.sub(r"&\s*\n\s*", " ", src)  # join continuation lines
    out = {}
    for mt in re.finditer(r"(integer\(c_int\)|type\(c_ptr\))\s+function\s+(\w+)\(([^)]*)\)\s*bind\(c,\s*name=\"(\w+)\"\)"
                          r"(.*?)end function", src, re.S):
        ret, args, cname, body = mt.group(1), mt.group(3), mt.group(4), mt.group(5)
        decls = {}
        for line in body.splitlines():
            line = line.strip()
            if "::" not in line or line.startswith("import"):
                continue
            spec, names = line.split("::")
            for nm in names.split(","):
                decls[nm.strip().lower()] = spec.strip().lower()
        kinds = []
        for a in [x.strip().lower() for x in args.split(",") if x.strip()]:
            spec = decls[a]
            byval = "value" in spec
            dim = "dimension" in spec
            if spec.startswith("integer(c_int)"):
                k = "int" if byval else "int*"
            elif spec.startswith("real(c_double)"):
                k = "double" if byval else "double*"
            elif spec.startswith("complex(c_double_complex)"):
                assert not byval, (cname, a)
                k = "double*"  # a complex(dp) scalar by reference is the C ABI's double[2]
            elif spec.startswith("logical(c_bool)"):
                k = "bool" if byval else "bool*"
            elif spec.startswith("character(kind=c_char)"):
                k = "char*" if (dim or not byval) else "char"
            elif spec.startswith("type(c_ptr)"):
                k = "ptr" if (byval and not dim) else "ptr*"
            elif spec.startswith("type(c_funptr)"):
                assert byval
                k = "funptr"
            else:
                raise AssertionError("unhandled declaration %r in %s" % (spec, cname))
            kinds.append(k)
        out[cname] = ("ptr" if ret.startswith("type") else "int", kinds)
    return out


def c_prototypes():
    """{name: (return kind, [argument C types])} of the functions declared in the header."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = re.sub(r"^\s*#.*$", "", txt, flags=re.M)
    typedefs = set(re.findall(r"typedef\s+\w+\s*\(\*(\w+)\)", txt))
    out = {}
    for mt in re.finditer(r"([\w\s\*]+?)\b(\w+)\s*\(([^;{]*?)\)\s*;", txt, re.S):
        ret, name, params = mt.group(1).strip(), mt.group(2), mt.group(3)
        if ret.startswith("typedef") or name in typedefs:
            continue
        ps = [] if params.strip() in ("", "void") else [p.strip() for p in params.split(",")]
        out[name] = (ret, ps, typedefs)
    return out


def c_kind(p, typedefs):
    """How a C parameter crosses the boundary, in the Fortran-side vocabulary above."""
    p = re.sub(r"\s+", " ", p)
    ty = re.sub(r"\b\w+\s*(\[\w*\])?$", "", p).strip() if not p.endswith("*") else p
    arr = re.search(r"\[\w*\]$", p) is not None
    ptrs = ty.count("*") + (1 if arr else 0)
    base = ty.replace("*", "").replace("const", "").strip()
    if base in typedefs:
        return {"funptr"}
    if ptrs == 0:
        return {{"int": "int", "double": "double", "bool": "bool", "char": "char",
                 "long long": "int64", "unsigned long long": "uint64"}[base]}
    if ptrs == 2:
        return {"ptr*"}
    if base == "char":
        return {"char*"}
    if base == "double":
        return {"double*", "ptr"}
    if base == "int":
        return {"int*", "ptr"}
    if base == "bool":
        return {"bool*"}
    return {"ptr"}


def test_every_shim_binding_matches_the_header():
    fi = fortran_interfaces()
    cp = c_prototypes()
    assert len(fi) >= 52, len(fi)  # handle API (d and z), omm, omm_callback, key layer, omm_wrapper
    L = G.lib()
    for cname, (ret, kinds) in sorted(fi.items()):
        assert cname in cp, "shim binds %s, which the header does not declare" % cname
        cret, params, typedefs = cp[cname]
        assert len(params) == len(kinds), (cname, params, kinds)
        for i, (p, k) in enumerate(zip(params, kinds)):
            assert k in c_kind(p, typedefs), "%s argument %d: shim passes %s, header has %r" % (cname, i + 1, k, p)
        if ret == "ptr":
            assert "*" in cret, (cname, cret)
        else:
            assert cret == "int", (cname, cret)
        assert hasattr(L, cname), "%s is not exported by the library" % cname


@pytest.mark.parametrize("name", ["mm_zmultiply", "m_zadd", "m_ztrace", "mm_ztrace", "m_zscale", "m_zset",
                                  "m_zset_element", "m_zget_element", "m_register_szden", "m_register_pzcsc",
                                  "psp_zgemspm", "psp_zgespmm", "omm_wrapper", "ms_wrapper_open"])
def test_shim_has_complex_generics_and_key_layer(name):
    src = open(SHIM).read()
    assert re.search(r"subroutine\s+%s\(" % name, src), name


def test_shim_defaults_are_the_references():
    src = open(SHIM).read()
    # m_allocate without a label: 'sdden' (MatrixSwitch.F90:344-347), in both modules
    assert len(re.findall(r"lab = 'sdden'", src)) == 2
    assert "lab = 'gdden'" not in src
    # an operation without a label: the reference's 'ref'
    assert "c = ['r', 'e', 'f']" in src
