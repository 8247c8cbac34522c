"""include/m_calypso_b200.f90 (the Fortran host's iso_c_binding module)
agrees with include/calypso_b200.h: the bind(C) derived types match the C
structs field for field, every C entry point has an interface with the same
binding name, argument count, passing mode (value or address) and kind, and
the status constants are the header's.  No Fortran compiler is needed; where
one exists the module is also compiled."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "calypso_b200.h")
MOD = os.path.join(ROOT, "include", "m_calypso_b200.f90")

C_KIND = {"int": "c_int", "unsigned": "c_int", "double": "c_double", "float": "c_float",
          "size_t": "c_size_t", "long long": "c_long_long", "char": "c_char"}
HANDLES = {"cb2_ctx", "cb2_ensemble", "cb2_mlp", "void"}


def c_source():
    return re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)


def c_structs():
    out = {}
    for name, body in re.findall(r"typedef struct (\w+) \{(.*?)\}\s*\w+;", c_source(), flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            m = re.match(r"(const )?(long long|\w+)\s*(\*?)\s*(.*)$", decl)
            base, ptr, names = m.group(2), m.group(3), m.group(4)
            for nm in names.split(","):
                nm = nm.strip().lstrip("*")
                dim = re.search(r"\[(\d+)\]", nm)
                fields.append((re.sub(r"\[\d+\]", "", nm), "c_ptr" if ptr else C_KIND[base],
                               int(dim.group(1)) if dim else 0))
        out[name] = fields
    return out


def c_protos():
    out = {}
    for p in re.findall(r"^\s*((?:const\s+)?\w+\s*\*?\s*cb2_\w+\s*\([^;]*\))\s*;", c_source(), flags=re.M):
        p = " ".join(p.split())
        m = re.match(r"(.*?)\b(cb2_\w+)\s*\((.*)\)$", p)
        args = []
        if m.group(3).strip() != "void":
            for a in m.group(3).split(","):
                a = a.strip()
                mm = re.match(r"(const )?(long long|\w+)\s*(\**)\s*(\w+)(\[\d+\])?$", a)
                args.append((mm.group(2), len(mm.group(3)), bool(mm.group(5)), mm.group(4)))
        out[m.group(2)] = (m.group(1).strip(), args)
    return out


def f_source():
    # join continuation lines, drop comments
    txt = re.sub(r"!.*", "", open(MOD).read())
    return re.sub(r"&\s*\n\s*", " ", txt)


def f_types():
    out = {}
    for name, body in re.findall(r"type, bind\(C\) :: (\w+)\n(.*?)end type", f_source(), flags=re.S | re.I):
        fields = []
        for line in body.strip().split("\n"):
            m = re.match(r"\s*(integer|real|type)\((\w+)\)\s*::\s*(.*)$", line.strip())
            for nm in m.group(3).split(","):
                nm = nm.strip()
                dim = re.search(r"\((\d+)\)", nm)
                fields.append((re.sub(r"\(\d+\)", "", nm), m.group(2), int(dim.group(1)) if dim else 0))
        out[name] = fields
    return out


def f_interfaces():
    out = {}
    pat = r"function (\w+)\(([^)]*)\)\s*bind\(C, name='(\w+)'\) result\(rc\)(.*?)end function"
    for name, dummies, bname, body in re.findall(pat, f_source(), flags=re.S | re.I):
        decls = {}
        rtype = None
        for line in body.strip().split("\n"):
            line = line.strip()
            if not line or line == "import":
                continue
            m = re.match(r"(integer|real|type|character)\(([\w=]+)\)(.*?)::\s*(\w+)", line)
            kind = m.group(2).replace("kind=", "")
            attrs = m.group(3)
            if m.group(4) == "rc":
                rtype = kind
                continue
            decls[m.group(4).lower()] = (kind, "value" in attrs)
        names = [d.strip().lower() for d in dummies.split(",") if d.strip()]
        out[bname] = (name, names, decls, rtype)
    return out


def test_structs_match_field_for_field():
    cs, ft = c_structs(), f_types()
    for name in ("cb2_params", "cb2_sph_tables"):
        assert cs[name] == ft[name], name


def test_every_entry_point_has_a_matching_interface():
    protos, ifs = c_protos(), f_interfaces()
    assert set(protos) == set(ifs), set(protos) ^ set(ifs)
    for name, (ret, args) in protos.items():
        fname, dummies, decls, rtype = ifs[name]
        assert fname == name
        assert rtype == ("c_int" if ret == "int" else "c_ptr"), name
        assert len(dummies) == len(args), name
        for (base, nptr, is_arr, cname), dn in zip(args, dummies):
            assert dn == cname.lower(), (name, cname, dn)
            kind, by_value = decls[dn]
            if base in HANDLES:
                # a handle by value, or the address of one (constructors)
                assert kind == "c_ptr" and by_value == (nptr == 1), (name, cname)
            elif base in ("cb2_params", "cb2_sph_tables"):
                assert kind == base and not by_value, (name, cname)
            elif nptr == 0 and not is_arr:
                assert kind == C_KIND[base] and by_value, (name, cname)
            else:
                # an array: the host array itself, or a device address by value
                assert (kind == C_KIND[base] and not by_value) or (kind == "c_ptr" and by_value), (name, cname)


def test_constants_match_header():
    consts = dict(re.findall(r"#define (CB2_\w+) (-?\d+)", open(HDR).read()))
    fconst = dict(re.findall(r"parameter :: (CB2_\w+) = (-?\d+)", open(MOD).read()))
    assert consts == fconst


@pytest.mark.skipif(shutil.which("gfortran") is None, reason="no Fortran compiler in this image")
def test_module_compiles(tmp_path):
    r = subprocess.run(["gfortran", "-std=f2008", "-c", MOD, "-J", str(tmp_path), "-o", str(tmp_path / "m.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
