"""The Fortran ISO_C_BINDING module (fortran/astr_b200_mod.F90) against the C header
(include/astr_b200.h), checked as text (no Fortran compiler is needed): every entry point the
header declares has a bind(C) interface of the same name, the same number of arguments, and for
each argument the same passing convention -- a C pointer or array is either `type(c_ptr), value`
or a by-reference Fortran argument of the matching kind, a C scalar is a `value` argument of the
matching kind."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _c_decls():
    src = open(os.path.join(ROOT, "include", "astr_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"^\s*(int|const char\*)\s+(astr_\w+)\s*\(([^;]*?)\)\s*;", src, re.M | re.S):
        ret, name, args = m.group(1), m.group(2), m.group(3)
        params = []
        for a in [x.strip() for x in args.replace("\n", " ").split(",") if x.strip()]:
            ptr = "*" in a or "[" in a
            base = re.sub(r"\bconst\b", "", a.split("[")[0]).replace("*", " ").split()
            ctype = base[0] if len(base) > 1 else base[0]
            params.append((ctype, ptr))
        out[name] = (ret, params)
    return out


def _f_decls():
    src = open(os.path.join(ROOT, "fortran", "astr_b200_mod.F90")).read()
    src = re.sub(r"&\s*\n\s*", " ", src)
    out = {}
    for m in re.finditer(r"^\s*(integer\(c_int\)|type\(c_ptr\))\s+function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*"
                         r"name=\"(\w+)\"\)(.*?)end function", src, re.M | re.S):
        ret, fname, args, cname, body = m.groups()
        names = [a.strip() for a in args.split(",") if a.strip()]
        attrs = {}
        for line in body.splitlines():
            if "::" not in line or line.strip().startswith("import"):
                continue
            spec, vars_ = line.split("::")
            for v in vars_.split(","):
                v = v.strip().split("(")[0]
                if v:
                    attrs[v.lower()] = spec.strip().lower()
        out[cname] = (ret, [(n, attrs.get(n.lower(), "")) for n in names])
    return out


C_KIND = {"int": "c_int", "double": "c_double", "int64_t": "c_int64_t", "char": "c_char"}


def test_every_header_entry_point_has_a_fortran_interface():
    c, f = _c_decls(), _f_decls()
    assert len(c) >= 30
    missing = sorted(set(c) - set(f))
    assert not missing, missing
    extra = sorted(set(f) - set(c))
    assert not extra, extra


def test_argument_counts_and_conventions_match():
    c, f = _c_decls(), _f_decls()
    bad = []
    for name, (cret, cparams) in c.items():
        fret, fparams = f[name]
        if (cret == "int") != (fret == "integer(c_int)"):
            bad.append((name, "return", cret, fret))
        if len(cparams) != len(fparams):
            bad.append((name, "arity", len(cparams), len(fparams)))
            continue
        for i, ((ctype, ptr), (fname, spec)) in enumerate(zip(cparams, fparams)):
            is_value = "value" in spec
            is_cptr = "type(c_ptr)" in spec
            if not spec:
                bad.append((name, i, fname, "undeclared"))
            elif ptr:
                kind = C_KIND.get(ctype)
                ok = (is_cptr and is_value) or (not is_value and (is_cptr or kind is None or kind in spec))
                if not ok:
                    bad.append((name, i, fname, ctype + "*", spec))
            else:
                kind = C_KIND.get(ctype)
                if not is_value or is_cptr or (kind and kind not in spec):
                    bad.append((name, i, fname, ctype, spec))
    assert not bad, bad
