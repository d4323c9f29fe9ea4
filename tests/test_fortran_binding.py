"""The Fortran drop-in binding (include/fortran/) checked against the C ABI
(include/st_b200.h) and against the reference's own routine signatures.

No Fortran compiler exists on this machine, so the files are checked by
parsing:
- every ISO_C_BINDING interface in st_b200_mod.f90 binds a function that
  include/st_b200.h declares, with the same number of arguments, each passed
  the same way (a C pointer <-> a by-reference dummy or a type(c_ptr) VALUE
  dummy; a C scalar <-> a VALUE dummy of the matching kind) and the same
  result type;
- the bind(c) type st_params_t lists the fields of st_params in order;
- each reference routine the library replaces has a wrapper of the same name
  and argument list in st_stubs_mf.f / st_stubs_periodic.f (the table below
  cites each reference signature);
- every library call in the wrappers names a public interface of the module
  with that interface's number of arguments;
- the wrappers obey fixed source form (72 columns, continuation in column 6).
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "st_b200.h")
FDIR = os.path.join(ROOT, "include", "fortran")
MOD = os.path.join(FDIR, "st_b200_mod.f90")
STUBS = {"mf": os.path.join(FDIR, "st_stubs_mf.f"), "periodic": os.path.join(FDIR, "st_stubs_periodic.f")}

# Reference signatures (name, arguments, where), case-insensitive as Fortran is.
D1 = ["F", "dF", "iadd", "cadd"]
D2 = ["F", "dF", "d2F", "iadd"]
TRI = ["A1", "B1", "C1", "R", "n", "lot", "nper", "ncom"]
PEN = ["A1", "B1", "C1", "D1", "E1", "R", "n", "lot", "nper", "ncom"]
REF_MF = [
    ("Setup_Derivatives_Sym", [], "src/derivCDopt6_sym_tri.f:9"),
    ("Setup_Derivatives_Asym", [], "src/derivCDopt6_asym_tri.f:9"),
    ("Init_Filters_sym", [], "src/filters_sym.f:9"),
    ("Init_Filters_asym", [], "src/filters_asym.f:9"),
    ("DFDX_sym", D1, "src/derivCDopt6_sym_tri.f:409"),
    ("D2FDX2_sym", D2, "src/derivCDopt6_sym_tri.f:538"),
    ("DFDY_sym", D1, "src/derivCDopt6_sym_tri.f:672"),
    ("D2FDY2_sym", D2, "src/derivCDopt6_sym_tri.f:801"),
    ("DFDZ_sym", D1, "src/derivCDopt6_sym_tri.f:932"),
    ("D2FDZ2_sym", D2, "src/derivCDopt6_sym_tri.f:1062"),
    ("DFDX_asym", D1, "src/derivCDopt6_asym_tri.f:412"),
    ("D2FDX2_asym", D2, "src/derivCDopt6_asym_tri.f:540"),
    ("DFDY_asym", D1, "src/derivCDopt6_asym_tri.f:670"),
    ("D2FDY2_asym", D2, "src/derivCDopt6_asym_tri.f:798"),
    ("DFDZ_asym", D1, "src/derivCDopt6_asym_tri.f:930"),
    ("D2FDZ2_asym", D2, "src/derivCDopt6_asym_tri.f:1061"),
    ("tridiagonal", TRI, "src/tridiagonal.f90:1"),
    ("pentadiagonal", PEN, "src/pentadiagonal.f90:1"),
    ("Compact_Filter", ["F", "F0", "N"], "src/filters_sym.f:398"),
    ("Compact_Filter_X_sym", ["F", "F0"], "src/filters_sym.f:436"),
    ("Compact_Filter_Y_sym", ["F", "F0"], "src/filters_sym.f:637"),
    ("Compact_Filter_Z_sym", ["F", "F0"], "src/filters_sym.f:838"),
    ("Compact_Filter_X_asym", ["F", "F0"], "src/filters_asym.f:388"),
    ("Compact_Filter_Y_asym", ["F", "F0"], "src/filters_asym.f:586"),
    ("Compact_Filter_Z_asym", ["F", "F0"], "src/filters_asym.f:783"),
    ("Gaussian_Filter", ["F", "Fg", "N"], "src/filters_sym.f:1046"),
    ("Gaussian_Filter_X", ["F", "Fg"], "src/filters_sym.f:1072"),
    ("Gaussian_Filter_Y", ["F", "Fg"], "src/filters_sym.f:1234"),
    ("Gaussian_Filter_Z", ["F", "Fg"], "src/filters_sym.f:1396"),
    ("Compute_gamma", ["Y"], "src/lddrk4_nonperiodic_mf.f:342"),
    ("RHS", ["Q", "Qrhs", "Y"], "src/rhsv_sym_mf.f:9"),
    ("Compute_hyper", ["Q", "Y"], "src/hyper_dynamic_sym_mf.f:166"),
    ("Hyper_RHS", ["Q", "Qrhs", "Y"], "src/hyper_rhs_sym_mf.f:12"),
    ("Species_RHS", ["Q", "Qrhs", "Y", "Yrhs"], "src/species_rhs_sym.f:9"),
    ("bc_RHS", ["Q", "Qrhs", "Y", "Yrhs", "time"], "src/bc_mf.f:11"),
    ("Sponge_Forcing", ["Q", "Qrhs", "Y", "Yrhs"], "src/sponge_mf.f:7"),
    ("Fix_Pressure", ["Q", "Y"], "pproc/pproc_mf.f:190"),
    ("Compute_CFL", ["Q", "cfl_stab_all", "cfl_resv_all", "step"], "src/lddrk4_nonperiodic_mf.f:7"),
    ("Compute_Tstep", ["Q", "Y", "cfl_resv", "step"], "src/lddrk4_nonperiodic_mf.f:75"),
    ("Compute_KE", ["Q"], "src/lddrk4_nonperiodic_mf.f:168"),
    ("Compute_Mom", ["Q"], "src/lddrk4_nonperiodic_mf.f:216"),
    ("Compute_Mass", ["Q", "Y"], "src/lddrk4_nonperiodic_mf.f:243"),
    ("Compute_Energy", ["Q"], "src/lddrk4_nonperiodic_mf.f:267"),
    ("Compute_Entropy", ["Q", "Y"], "src/lddrk4_nonperiodic_mf.f:288"),
    ("LDDRK4", ["time", "step"], "src/lddrk4_nonperiodic_mf.f:428"),
    ("Compute_Grad", [], "src/grad_sym.f:13"),
    ("Compute_SRM_Stats", ["step"], "pproc/pproc_mf.f:4"),
    ("Generate_Shock_Surface", [], "src/shock.f:163"),
    ("MakePaddedArrays", ["W", "xx", "yy", "zz", "nfields"], "src/vis_silo_mf.f:440"),
    ("Write_Visual_Silo", ["time", "step"], "src/vis_silo_mf.f:7"),
]
REF_PERIODIC = [
    ("Setup_Derivatives", [], "src/derivCDopt6_periodic.f:9"),
    ("Init_Filters", [], "src/filters_periodic.f:9"),
    ("DFDX", D1, "src/derivCDopt6_periodic.f:164"),
    ("D2FDX2", D2, "src/derivCDopt6_periodic.f:281"),
    ("DFDY", D1, "src/derivCDopt6_periodic.f:400"),
    ("D2FDY2", D2, "src/derivCDopt6_periodic.f:515"),
    ("DFDZ", D1, "src/derivCDopt6_periodic.f:631"),
    ("D2FDZ2", D2, "src/derivCDopt6_periodic.f:747"),
    ("tridiagonal", TRI, "src/tridiagonal.f90:1"),
    ("pentadiagonal", PEN, "src/pentadiagonal.f90:1"),
    ("Compact_Filter", ["F", "F0", "N"], "src/filters_periodic.f:90"),
    ("Compact_Filter_X", ["F", "F0"], "src/filters_periodic.f:115"),
    ("Compact_Filter_Y", ["F", "F0"], "src/filters_periodic.f:254"),
    ("Compact_Filter_Z", ["F", "F0"], "src/filters_periodic.f:393"),
    ("Gaussian_Filter", ["F", "Fg", "N"], "src/filters_periodic.f:540"),
    ("Gaussian_Filter_X", ["F", "Fg"], "src/filters_periodic.f:565"),
    ("Gaussian_Filter_Y", ["F", "Fg"], "src/filters_periodic.f:680"),
    ("Gaussian_Filter_Z", ["F", "Fg"], "src/filters_periodic.f:793"),
    ("RHS", ["Q", "Qrhs"], "src/rhsv_periodic_sf.f:9"),
    ("Compute_hyper", ["Q"], "src/hyper_dynamic.f:173"),
    ("Hyper_RHS", ["Q", "Qrhs"], "src/hyper_rhs.f:12"),
    ("Compute_CFL", ["Q", "cfl_stab_all", "cfl_resv_all", "step"], "src/lddrk4_periodic_sf.f:7"),
    ("Compute_Tstep", ["Q", "cfl_resv", "step"], "src/lddrk4_periodic_sf.f:74"),
    ("Compute_KE", ["Q"], "src/lddrk4_periodic_sf.f:153"),
    ("Compute_Mom", ["Q"], "src/lddrk4_periodic_sf.f:201"),
    ("Compute_Mass", ["Q"], "src/lddrk4_periodic_sf.f:228"),
    ("Compute_Energy", ["Q"], "src/lddrk4_periodic_sf.f:247"),
    ("Compute_Entropy", ["Q"], "src/lddrk4_periodic_sf.f:268"),
    ("LDDRK4", ["time", "step"], "src/lddrk4_periodic_sf.f:311"),
    ("Fix_Pressure", ["Q"], "src/lddrk4_periodic_sf.f:436"),
]


# ---- parsing ---------------------------------------------------------------
def split_top(s):
    """Split on commas outside parentheses and quotes."""
    out, depth, cur, q = [], 0, "", None
    for ch in s:
        if q:
            cur += ch
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
            continue
        cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def c_prototypes():
    text = re.sub(r"/\*.*?\*/", " ", open(HDR).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"^\s*(int|void|const\s+char\s*\*)\s*(\w+)\s*\(([^)]*)\)\s*;", text, re.M):
        ret, name, args = m.group(1), m.group(2), m.group(3).strip()
        params = [] if args in ("", "void") else [a.strip() for a in args.split(",")]
        protos[name] = ("ptr" if "*" in ret else ret, params)
    return protos


def c_struct_fields(struct):
    text = re.sub(r"/\*.*?\*/", " ", open(HDR).read(), flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\}" % struct, text, re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        typ, names = decl.split(None, 1)
        fields += [(typ, n.strip()) for n in names.split(",")]
    return fields


def fortran_free_lines(path):
    """Free-form source with continuations joined and comments removed."""
    lines, cur = [], ""
    for raw in open(path):
        line = raw.split("!")[0].rstrip() if "'" not in raw else raw.rstrip()
        if line.strip().startswith("!"):
            continue
        if cur:
            line = cur + " " + line.lstrip().lstrip("&")
            cur = ""
        if line.endswith("&"):
            cur = line[:-1]
            continue
        if line.strip():
            lines.append(line.strip())
    return lines


def module_interfaces():
    """{binding name: (fortran name, result kind, [(arg, kind, type)])}"""
    lines = fortran_free_lines(MOD)
    ifaces, cur = {}, None
    head = re.compile(r"^(?:(integer\(c_int\)|type\(c_ptr\))\s+)?(function|subroutine)\s+(\w+)\s*\(([^)]*)\)\s*"
                      r"bind\(c,\s*name='(\w+)'\)", re.I)
    for ln in lines:
        m = head.match(ln)
        if m:
            res = m.group(1) or "void"
            res = "int" if res.lower().startswith("integer") else ("ptr" if res.lower().startswith("type") else "void")
            args = [a.strip() for a in m.group(4).split(",") if a.strip()]
            cur = {"fname": m.group(3), "res": res, "args": args, "decl": {}, "bind": m.group(5)}
            continue
        if cur is None:
            continue
        if re.match(r"^end\s+(function|subroutine)", ln, re.I):
            ifaces[cur["bind"]] = cur
            cur = None
            continue
        m = re.match(r"^(.*?)::(.*)$", ln)
        if m and not ln.lower().startswith("import"):
            attrs = m.group(1).lower()
            for ent in split_top(m.group(2)):
                nm = re.match(r"(\w+)", ent).group(1)
                cur["decl"][nm.lower()] = attrs
    return ifaces


def fortran_arg_kind(attrs):
    typ = attrs.split(",")[0].strip().replace(" ", "")
    if "value" in attrs:
        return ("ptr", typ) if typ == "type(c_ptr)" else ("val", typ)
    return ("ptr", typ)


def c_arg_kind(param):
    if "*" in param or "[" in param:
        return ("ptr", None)
    typ = param.rsplit(None, 1)[0].replace("const", "").strip()
    return ("val", typ)


VAL_TYPES = {"int": "integer(c_int)", "double": "real(c_double)"}


def fixed_form_statements(path):
    """(line number, statement) of a fixed-form file, continuations joined."""
    stmts = []
    for no, raw in enumerate(open(path), 1):
        line = raw.rstrip("\n")
        if not line.strip() or line[0] in "*cC!":
            continue
        if len(line) > 5 and line[5] not in " 0" and not line[:5].strip():
            stmts[-1] = (stmts[-1][0], stmts[-1][1] + " " + line[6:].strip())
        else:
            stmts.append((no, line[6:].strip() if len(line) > 6 else ""))
    return stmts


def stub_subroutines(path):
    subs = {}
    for no, st in fixed_form_statements(path):
        m = re.match(r"^Subroutine\s+(\w+)\s*(?:\((.*)\))?\s*$", st, re.I)
        if m:
            args = [a.strip() for a in (m.group(2) or "").split(",") if a.strip()]
            subs[m.group(1).lower()] = (m.group(1), args, no)
    return subs


# ---- tests -----------------------------------------------------------------
def test_interfaces_match_the_c_header():
    protos = c_prototypes()
    ifaces = module_interfaces()
    assert len(ifaces) >= 60
    for bind, it in ifaces.items():
        if bind == "strlen":
            continue
        assert bind in protos, f"{bind} is not declared in include/st_b200.h"
        cres, cparams = protos[bind]
        assert it["res"] == cres, (bind, it["res"], cres)
        assert len(it["args"]) == len(cparams), (bind, it["args"], cparams)
        for a, cp in zip(it["args"], cparams):
            attrs = it["decl"].get(a.lower())
            assert attrs is not None, (bind, a, "argument without a declaration")
            fk, ft = fortran_arg_kind(attrs)
            ck, ct = c_arg_kind(cp)
            assert fk == ck, (bind, a, attrs, cp)
            if ck == "val":
                assert VAL_TYPES[ct] == ft, (bind, a, ft, ct)


def test_params_type_matches_the_c_struct():
    lines = fortran_free_lines(MOD)
    i = next(k for k, ln in enumerate(lines) if ln.lower().startswith("type, bind(c) :: st_params_t"))
    ffields = []
    for ln in lines[i + 1:]:
        if ln.lower().startswith("end type"):
            break
        typ, names = ln.split("::")
        ffields += [(typ.strip().replace(" ", ""), n.strip()) for n in names.split(",")]
    cfields = c_struct_fields("st_params")
    assert [n for _, n in ffields] == [n for _, n in cfields]
    for (ft, n), (ct, _) in zip(ffields, cfields):
        assert VAL_TYPES[ct] == ft, n


@pytest.mark.parametrize("family,table", [("mf", REF_MF), ("periodic", REF_PERIODIC)])
def test_every_replaced_routine_has_its_reference_signature(family, table):
    subs = stub_subroutines(STUBS[family])
    for name, args, where in table:
        assert name.lower() in subs, f"{name} ({where}) has no wrapper"
        _, got, _ = subs[name.lower()]
        assert [a.lower() for a in got] == [a.lower() for a in args], (name, where, got)


@pytest.mark.parametrize("family", ["mf", "periodic"])
def test_wrapper_calls_match_the_module(family):
    ifaces = {it["fname"].lower(): it for it in module_interfaces().values()}
    public = set()
    for ln in fortran_free_lines(MOD):
        m = re.match(r"^public\s*::\s*(.*)$", ln, re.I)
        if m:
            public |= {x.strip().lower() for x in m.group(1).split(",")}
    calls = 0
    for no, st in fixed_form_statements(STUBS[family]):
        for m in re.finditer(r"\b(st_\w+)\s*\(", st):
            name = m.group(1).lower()
            if name in ("st_check", "st_b200_init", "st_b200_monitors", "st_b200_pull_commons"):
                continue
            assert name in public, (no, name)
            depth, j = 0, m.end() - 1
            for j in range(m.end() - 1, len(st)):
                depth += {"(": 1, ")": -1}.get(st[j], 0)
                if depth == 0:
                    break
            args = split_top(st[m.end():j])
            assert len(args) == len(ifaces[name]["args"]), (no, name, args)
            calls += 1
    assert calls > 30


@pytest.mark.parametrize("family", ["mf", "periodic"])
def test_fixed_source_form(family):
    depth = 0
    for no, raw in enumerate(open(STUBS[family]), 1):
        line = raw.rstrip("\n")
        if not line.strip() or line[0] in "*cC!":
            continue
        assert len(line) <= 72, (no, len(line))
        assert line[:5].strip() == "" or line[:5].strip().isdigit(), (no, line)
    for no, st in fixed_form_statements(STUBS[family]):
        if re.match(r"^Subroutine\b", st, re.I):
            assert depth == 0, no
            depth = 1
        elif re.match(r"^End\s*$", st, re.I):
            assert depth == 1, no
            depth = 0
    assert depth == 0
