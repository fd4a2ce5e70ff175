"""Static check of the Fortran shim (maccpic_b200/fortran/em2g_shim.f90)
against the C ABI it binds (include/em2g.h).

No Fortran compiler exists here, so the shim cannot be built; what can go
wrong in an iso_c_binding interface is checked by reading it instead:

* every bind(c) function is declared in include/em2g.h with the same number
  of arguments, and each argument's Fortran kind and passing mode (value or
  reference) is the C parameter's type;
* the bind(c) derived type em2g_params has the members of struct
  em2g_params in the same order with the same C types and array lengths, so
  that its C layout (computed from the members) has the offsets gcc gives the
  C struct -- which the ctypes mirror in maccpic_b200/_lib.py must also have;
* the shim defines em2's move, curnt and fields with no arguments
  (pic/main.f90:154-169) and calls no library function it has not declared.
"""
import os
import re
import subprocess


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "maccpic_b200", "fortran", "em2g_shim.f90")
HEADER = os.path.join(ROOT, "include", "em2g.h")

# Fortran declaration -> (C base type, pointer depth)
F_KINDS = {
    ("integer(c_int)", True): ("int", 0), ("integer(c_int)", False): ("int", 1),
    ("integer(c_int32_t)", True): ("int", 0), ("integer(c_int32_t)", False): ("int", 1),
    ("integer(c_int64_t)", True): ("int64_t", 0), ("integer(c_int64_t)", False): ("int64_t", 1),
    ("real(c_double)", True): ("double", 0), ("real(c_double)", False): ("double", 1),
    ("type(c_ptr)", True): ("opaque", 1), ("type(c_ptr)", False): ("opaque", 2),
    ("type(em2g_params)", False): ("em2g_params", 1),
}
C_OPAQUE = {"em2g_ctx", "em2g_adj", "em2g_ens", "void"}
F_MEMBER = {"integer(c_int32_t)": ("int32_t", 4), "integer(c_int64_t)": ("int64_t", 8),
            "real(c_double)": ("double", 8)}


def _strip_fortran(src):
    return "\n".join(ln.split("!")[0] for ln in src.splitlines())


def _c_prototypes():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    protos = {}
    for ret, name, args in re.findall(r"(int|const char\s*\*)\s*(em2g_\w+)\s*\(([^)]*)\)\s*;",
                                      src):
        params = []
        args = args.strip()
        if args and args != "void":
            for a in args.split(","):
                a = a.replace("const", " ").strip()
                depth = a.count("*")
                base = a.replace("*", " ").split()[0]
                params.append(("opaque" if base in C_OPAQUE else base, depth))
        protos[name] = ("ptr" if "char" in ret else "int", params)
    return protos


def _fortran_interfaces():
    src = _strip_fortran(open(SHIM).read())
    block = src[src.index("interface"):src.index("end interface")]
    funcs = {}
    for m in re.finditer(r"(integer\(c_int\)|type\(c_ptr\))\s+function\s+(\w+)\s*\(([^)]*)\)"
                         r"\s*bind\(c\)(.*?)end function", block, flags=re.S):
        ret, name, args, body = m.groups()
        names = [a.strip() for a in args.split(",") if a.strip()]
        kinds = {}
        for ln in body.splitlines():
            ln = ln.strip()
            if "::" not in ln:
                continue
            decl, vars_ = ln.split("::")
            parts = [p.strip() for p in decl.split(",")]
            value = "value" in parts
            for v in vars_.split(","):
                v = v.strip()
                vname = v.split("(")[0].strip()
                kinds[vname] = F_KINDS[(parts[0], value)]
        funcs[name] = ("ptr" if ret == "type(c_ptr)" else "int", [kinds[n] for n in names])
    return funcs


def test_every_bind_c_function_matches_the_header():
    protos = _c_prototypes()
    funcs = _fortran_interfaces()
    assert len(funcs) >= 10
    for name, (ret, params) in funcs.items():
        assert name in protos, f"{name} is not declared in include/em2g.h"
        cret, cparams = protos[name]
        assert ret == cret, name
        assert params == cparams, (name, params, cparams)


def _fortran_params_members():
    src = _strip_fortran(open(SHIM).read())
    m = re.search(r"type,\s*bind\(c\)\s*::\s*em2g_params(.*?)end type", src, flags=re.S)
    members = []
    for ln in m.group(1).splitlines():
        if "::" not in ln:
            continue
        decl, vars_ = ln.split("::")
        ctype, size = F_MEMBER[decl.strip()]
        for v in re.findall(r"(\w+)(?:\((\d+)\))?", vars_):
            members.append((v[0], ctype, size, int(v[1]) if v[1] else 1))
    return members


def _c_layout(members):
    """Offsets of a C struct with these members (natural alignment)."""
    off, out = 0, {}
    for name, _, size, count in members:
        off = (off + size - 1) // size * size
        out[name] = off
        off += size * count
    align = max(m[2] for m in members)
    return out, (off + align - 1) // align * align


def test_params_type_matches_the_c_struct(tmp_path):
    members = _fortran_params_members()
    offsets, size = _c_layout(members)
    # the C struct as gcc lays it out
    prog = tmp_path / "off.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "em2g.h"', 'int main(void){',
             'printf("size %zu\\n", sizeof(em2g_params));']
    for name, *_ in members:
        lines.append(f'printf("{name} %zu %zu\\n", offsetof(em2g_params, {name}), '
                     f'sizeof(((em2g_params*)0)->{name}));')
    lines.append("return 0;}")
    prog.write_text("\n".join(lines))
    exe = tmp_path / "off"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(prog), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for ln in out.splitlines():
        k, *v = ln.split()
        got[k] = [int(x) for x in v]
    assert got["size"][0] == size
    for name, _, msize, count in members:
        assert got[name] == [offsets[name], msize * count], name
    # and the ctypes mirror of the Python host
    from maccpic_b200._lib import Em2gParams
    import ctypes
    assert ctypes.sizeof(Em2gParams) == size
    assert [f[0] for f in Em2gParams._fields_] == [m[0] for m in members]
    for name, *_ in members:
        assert getattr(Em2gParams, name).offset == offsets[name], name


def test_shim_defines_em2s_subroutines_and_calls_only_declared_functions():
    src = _strip_fortran(open(SHIM).read()).lower()
    for sub in ("move", "curnt", "fields"):
        assert re.search(rf"^\s*subroutine\s+{sub}\s*$", src, flags=re.M), sub
        assert re.search(rf"^\s*end subroutine\s+{sub}\s*$", src, flags=re.M), sub
    declared = set(_fortran_interfaces())
    body = src[src.index("end interface"):]
    called = set(re.findall(r"\b(em2g_[a-z_0-9]+)\s*\(", body))
    helpers = {"em2g_check"}
    assert called - helpers <= declared, called - helpers - declared
    # the output predicate of pic/main.f90:158-159 decides the downloads
    assert "(mod(it,isav) == 0) .or. (it == 1) .or. (mod(it,iphs) == 0) .or. (it == nt)" in src
