"""The ISO_C_BINDING module (wenostandalone_b200/fortran/m_weno_sb.f90)
against the C header it binds (include/weno_sb.h).  CPU only.

No Fortran compiler exists on the machines this suite runs on, so the module
is checked by reading it: every bind(C) interface names a function the
header declares, with the same number of arguments, and each argument is
passed the way the C prototype takes it -- a C scalar by VALUE with the
matching ISO_C_BINDING kind, a C pointer either as `type(c_ptr), value` or
by reference (a Fortran dummy without VALUE).  Every entry point of the
header except the test-suite diagnostics has an interface.
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "wenostandalone_b200", "fortran", "m_weno_sb.f90")
HDR = os.path.join(ROOT, "include", "weno_sb.h")

# test-suite diagnostics, deliberately not bound for Fortran drivers
DIAGNOSTICS = {"weno_sb_selftest_rcp", "weno_sb_selftest_timeout"}

C_SCALAR_KIND = {"int": "c_int", "unsigned": "c_int", "int64_t": "c_int64_t", "double": "c_double",
                 "int32_t": "c_int32_t", "size_t": "c_size_t"}


def c_prototypes():
    txt = open(HDR).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"([A-Za-z_][\w \*]*?)\b(weno_sb_\w+)\s*\(([^)]*)\)\s*;", txt):
        ret, name, params = m.group(1).strip(), m.group(2), m.group(3).strip()
        plist = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        args = []
        for p in plist:
            ptr = "*" in p
            base = re.sub(r"\b(const|struct)\b", "", p.split("*")[0]).split()
            args.append((ptr, base[0] if base else ""))
        out[name] = (ret, args)
    return out


def fortran_interfaces():
    txt = open(F90).read()
    block = txt[txt.index("interface"):txt.index("end interface")]
    out = {}
    pat = re.compile(r"(?:([\w()]+)\s+)?function\s+(\w+)\s*\(([^)]*)\)\s*&?\s*bind\(C,\s*name='(\w+)'\)(.*?)end function",
                     re.S)
    for m in pat.finditer(block.replace("&\n", " ")):
        rtype, fname, args, cname, body = m.groups()
        names = [a.strip().lower() for a in args.split(",") if a.strip()]
        decl = {}
        for line in body.splitlines():
            line = line.split("!")[0].strip()
            if "::" not in line:
                continue
            spec, vars_ = line.split("::", 1)
            for v in vars_.split(","):
                v = re.sub(r"\(.*\)", "", v).strip().lower()
                if v:
                    decl[v] = spec.strip().lower()
        out[cname] = (fname, rtype, names, decl)
    return out


def test_every_entry_point_has_an_interface():
    protos, ifs = c_prototypes(), fortran_interfaces()
    assert protos and ifs
    missing = sorted(set(protos) - set(ifs) - DIAGNOSTICS)
    assert not missing, f"no Fortran interface for {missing}"
    unknown = sorted(set(ifs) - set(protos))
    assert not unknown, f"interfaces bind names the header does not declare: {unknown}"


def test_interfaces_match_the_prototypes():
    protos, ifs = c_prototypes(), fortran_interfaces()
    for cname, (fname, rtype, names, decl) in ifs.items():
        ret, args = protos[cname]
        assert fname == cname, (fname, cname)
        assert len(names) == len(args), f"{cname}: {len(names)} Fortran args against {len(args)} in C"
        if "*" in ret:
            assert rtype and "c_ptr" in rtype, (cname, rtype)
        else:
            assert rtype and C_SCALAR_KIND[ret.split()[-1]] in rtype, (cname, rtype, ret)
        for a, (ptr, base) in zip(names, args):
            spec = decl.get(a)
            assert spec is not None, f"{cname}: argument {a} is not declared"
            by_value = re.search(r"\bvalue\b", spec) is not None
            if ptr:
                # a C pointer: a c_ptr passed by value, or any dummy by reference
                assert ("c_ptr" in spec) or not by_value, (cname, a, spec)
                if "c_ptr" not in spec and base in C_SCALAR_KIND:
                    assert C_SCALAR_KIND[base] in spec, (cname, a, spec, base)
                if base == "weno_sb_grid":
                    assert "type(weno_sb_grid)" in spec, (cname, a, spec)
            else:
                assert by_value, f"{cname}: C scalar {a} must be passed by value ({spec})"
                assert C_SCALAR_KIND[base] in spec, (cname, a, spec, base)


def test_bind_c_types_follow_the_structs():
    """Field order and kinds of the bind(C) derived types."""
    txt = open(F90).read().lower()
    grid = re.search(r"type, bind\(c\) :: weno_sb_grid(.*?)end type", txt, re.S).group(1)
    assert re.search(r"integer\(c_int32_t\) :: m_cells, n_cells, p_cells", grid)
    assert re.search(r"integer\(c_int32_t\) :: v_size, buff_size, scheme", grid)
    assert re.search(r"real\(c_double\) :: weno_eps, teno_ct", grid)
    face = re.search(r"type, bind\(c\) :: weno_sb_face_coefs(.*?)end type", txt, re.S).group(1)
    # C double polyL[3][5] is Fortran polyL(5, 3): the same 15 doubles
    assert "polyl(5, 3), polyr(5, 3)" in face and "dl(5), dr(5)" in face and "beta_coef(5, 6)" in face
    blk = re.search(r"type, bind\(c\) :: weno_sb_block(.*?)end type", txt, re.S).group(1)
    order = [ln.split("!")[0].split("::")[1].strip() for ln in blk.splitlines() if "::" in ln]
    assert order == ["grid", "dir, order", "flags", "dtype", "v_in", "coefs", "vl, vr"], order
