"""The Fortran binding (include/qqcd_gpu_f.f90) against the C header (include/qqcd_gpu.h).

No Fortran compiler exists here, so the module is checked by parsing both files:
every C prototype has a bind(C) interface of the same name, with the same number of
arguments, each passed by value exactly where C passes by value (scalars and the opaque
handles qq_ctx / qq_defl / qq_net / qq_eig), with the matching interoperable kind; every C struct
has a bind(C) derived type with the same members in the same order.  The shim module
keeps the reference's procedure names and argument lists (Q/diracops.f90:264-599,
Q/inverters.f90:302-487, 2871-3572, 4310-4465, Q/quark.f90:458-842), checked against the
lists below, which restate those signatures."""
import re
from pathlib import Path

import pytest

INC = Path(__file__).resolve().parent.parent / "include"
HANDLES = ("qq_ctx", "qq_defl", "qq_net", "qq_eig")


def strip_c_comments(s):
    return re.sub(r"/\*.*?\*/", " ", s, flags=re.S)


def c_prototypes():
    text = strip_c_comments((INC / "qqcd_gpu.h").read_text())
    protos = {}
    for m in re.finditer(r"(int|long long|const char\s*\*)\s*(qq_\w+)\s*\(([^)]*)\)\s*;", text):
        ret, name, args = m.group(1), m.group(2), m.group(3)
        alist = [] if args.strip() in ("", "void") else [a.strip() for a in args.split(",")]
        protos[name] = (ret.replace(" ", ""), alist)
    return protos


def c_structs():
    text = strip_c_comments((INC / "qqcd_gpu.h").read_text())
    out = {}
    for m in re.finditer(r"typedef struct (qq_\w+)\s*\{(.*?)\}\s*\1\s*;", text, flags=re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            tm = re.match(r"(const\s+)?(qq_ctx\s*\*|double\s*\*|qq_solve_info\s*\*|unsigned long long|"
                          r"long long|int|double)\s*(.*)", decl)
            assert tm, decl
            ctype = tm.group(2).replace(" ", "")
            if tm.group(1):
                ctype = "const" + ctype
            for var in tm.group(3).split(","):
                var = var.strip()
                vm = re.match(r"(\*?)(\w+)\s*(?:\[(.*)\])?", var)
                n = eval(vm.group(3)) if vm.group(3) else 1  # noqa: S307 -- "2 * 512" etc.
                fields.append((vm.group(2), ctype + vm.group(1), n))
        out[m.group(1)] = fields
    return out


def classify_c(arg):
    """(by_value, kind) of one C parameter."""
    a = " ".join(arg.replace("*", " * ").split())
    stars = a.count("*")
    arr = "[" in a
    base = a.replace("const ", "").replace("*", "").strip()
    base = re.sub(r"\s*\w+\s*(\[.*\])?$", "", base).strip()  # drop the parameter name
    if base in HANDLES and stars == 1:
        return True, "ptr"
    if stars == 2 or (base == "void" and stars >= 1):
        return False, "ptr"
    if stars == 0 and not arr:
        return True, {"int": "int", "double": "double", "unsigned long long": "llong", "long long": "llong"}[base]
    kind = {"int": "int", "double": "double", "long long": "llong", "char": "char",
            "qq_geom": "qq_geom", "qq_method": "qq_method", "qq_solve_info": "qq_solve_info",
            "qq_uneven_group": "qq_uneven_group"}[base]
    return False, kind


def fortran_text():
    src = (INC / "qqcd_gpu_f.f90").read_text()
    src = re.sub(r"!.*", "", src)
    return re.sub(r"&\s*\n\s*", " ", src)


def f_interfaces():
    src = fortran_text()
    out = {}
    pat = re.compile(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)\s*result\((\w+)\)(.*?)"
                     r"end function", flags=re.S)
    for m in pat.finditer(src):
        fname, args, cname, res, body = m.groups()
        dummies = [a.strip() for a in args.split(",") if a.strip()]
        decls = {}
        for line in body.splitlines():
            dm = re.match(r"\s*(type\((\w+)\)|integer\((\w+)\)|real\((\w+)\)|character\(kind=(\w+)\))(.*?)::(.*)",
                          line)
            if not dm:
                continue
            kind = dm.group(2) or dm.group(3) or dm.group(4) or dm.group(5)
            attrs = dm.group(6)
            for v in re.findall(r"(\w+)\s*(?:\([^)]*\))?", dm.group(7)):
                decls[v] = (kind, "value" in attrs)
        out[cname] = (fname, dummies, res, decls)
    return out


def f_types():
    src = fortran_text()
    out = {}
    for m in re.finditer(r"type,\s*bind\(C\)\s*::\s*(\w+)(.*?)end type", src, flags=re.S):
        comps = []
        for line in m.group(2).splitlines():
            dm = re.match(r"\s*(type\((\w+)\)|integer\((\w+)\)|real\((\w+)\))\s*::\s*(.*)", line)
            if not dm:
                continue
            kind = dm.group(2) or dm.group(3) or dm.group(4)
            for v in re.findall(r"(\w+)\s*(?:\((\d+)\))?", dm.group(5)):
                comps.append((v[0], kind, int(v[1]) if v[1] else 1))
        out[m.group(1)] = comps
    return out


F_KIND = {"int": "c_int", "double": "c_double", "llong": "c_long_long", "ptr": "c_ptr", "char": "c_char"}


def test_every_prototype_has_an_interface():
    protos, ifaces = c_prototypes(), f_interfaces()
    assert len(protos) >= 60
    assert sorted(protos) == sorted(ifaces), set(protos) ^ set(ifaces)
    for cname, (fname, _, _, _) in ifaces.items():
        assert fname == cname


@pytest.mark.parametrize("name", sorted(c_prototypes()))
def test_interface_matches_prototype(name):
    ret, cargs = c_prototypes()[name]
    fname, dummies, res, decls = f_interfaces()[name]
    assert len(dummies) == len(cargs), (name, dummies, cargs)
    want_ret = {"int": "c_int", "longlong": "c_long_long", "constchar*": "c_ptr"}[ret]
    assert decls[res][0] == want_ret, (name, decls[res])
    for d, a in zip(dummies, cargs):
        by_value, kind = classify_c(a)
        fk, fval = decls[d]
        assert fval == by_value, (name, d, a)
        assert fk == F_KIND.get(kind, kind), (name, d, a, fk)


@pytest.mark.parametrize("name", sorted(c_structs()))
def test_struct_layouts(name):
    cs = c_structs()[name]
    ft = f_types()[name]
    assert [f[0] for f in cs] == [f[0] for f in ft], name
    kinds = {"int": "c_int", "double": "c_double", "qq_ctx*": "c_ptr", "constdouble*": "c_ptr", "double*": "c_ptr",
             "qq_solve_info*": "c_ptr"}
    for (cn, ct, cnum), (fn, fk, fnum) in zip(cs, ft):
        assert kinds[ct] == fk, (name, cn, ct, fk)
        assert cnum == fnum, (name, cn, cnum, fnum)


# The reference's argument lists (restated from the cited signatures).
REFERENCE_SIGNATURES = {
    "Hsingle": "gout,u,gin,idag,coact,bc,gblclr,vecbl,vecblinv,myid,nn,ldiv,nms,lvbc,ib,lbd,iblv,MRT",  # diracops:554
    "Hdouble": "he,u,ge,idag,coact,kappa,bc,vecbl,vecblinv,myid,nn,ldiv,nms,lvbc,ib,lbd,iblv,MRT",  # diracops:264
    "Hdbletm": "he,u,GeeGooinv,ge,idag,coact,kappa,iflag,bc,vecbl,vecblinv,myid,nn,ldiv,nms,lvbc,ib,lbd,iblv,MRT",
    "gmresdr": "rwdir,phi,x,GMRES,resmax,itermin,itercount,u,GeeGooinv,iflag,kappa,coact,bc,vecbl,vecblinv,myid,nn,"
               "ldiv,nms,lvbc,ib,lbd,iblv,MRT,MRT2",  # inverters:2871
    "psc": "rwdir,b,x,GMRES,resmax,itermin,itercount,u,GeeGooinv,iflag,kappa,coact,bc,vecbl,vecblinv,myid,nn,ldiv,"
           "nms,lvbc,ib,lbd,iblv,MRT,MRT2",  # inverters:4310
    "bicgstab": "rwdir,phi,x,resmax,itermin,itercount,u,GeeGooinv,iflag,kappa,coact,bc,vecbl,vecblinv,myid,nn,ldiv,"
                "nms,lvbc,ib,lbd,iblv,MRT,MRT2",  # inverters:302
    "fermprop": "rwdir,be,bo,nkappa,kappa,cSW,inverter,coact,bc,resmax,itermin,omegaM3R,u,vectype,kGMRES,xe,xo,myid,"
                "nn,ldiv,nms,lvbc,lvcl,ib,lbd,iblv,vecbl,vecblinv,ntmqcd,hoption,MRT,MRT2",  # quark:458
}


@pytest.mark.parametrize("name", sorted(REFERENCE_SIGNATURES))
def test_shim_keeps_reference_signature(name):
    src = fortran_text()
    shim = src[src.index("module qqcd_gpu_shim"):]
    m = re.search(r"subroutine\s+%s\s*\(([^)]*)\)" % name, shim)
    assert m, name
    got = [a.strip() for a in m.group(1).split(",")]
    assert got == REFERENCE_SIGNATURES[name].split(","), name
    assert re.search(r"public\s*::.*\b%s\b" % name, shim), name


def test_shim_validates_and_checks_every_call():
    src = fortran_text()
    shim = src[src.index("module qqcd_gpu_shim"):]
    for name in REFERENCE_SIGNATURES:
        body = re.search(r"subroutine\s+%s\s*\(.*?end subroutine %s" % (name, name), shim, flags=re.S).group(0)
        assert "call qqgpu_validate(" in body, name
        assert "call qqgpu_prepare(" in body, name
        assert "call qqgpu_check(" in body, name
