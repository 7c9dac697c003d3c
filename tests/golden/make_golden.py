"""Generate the known-answer fixtures under tests/golden/ from the reference's
own Fortran tests, read as text.

The reference pins its Fock build with four known-answer programs
(tests/fortran/test_h2_sonly.F90, test_interface_h2.F90, test_h2_ccpvdz.F90,
test_h2o_ccpvdz.F90).  Each builds a molecule and basis in local arrays,
disables screening with schwrz_int = 1e10, uses an identity density, and
compares every packed Fock element against hard-coded values at tol = 1e-10.
This script parses those assignments and the `fa_ref` arrays and writes one
JSON fixture per test, so the parity tests never need the reference tree.
It also writes h2o_ccpvtz.json from the f-shell known-answer program
(tests/fortran/test_h2o_ccpvtz.F90 with fa_h2o_ccpvtz_reference.dat), kept
for the f-shell classes.

Usage (needs the reference checkout; the fixtures are committed):
    python tests/golden/make_golden.py /path/to/gms_libERI
"""
import json
import math
import os
import re
import sys

TESTS = {
    "h2_sonly": "tests/fortran/test_h2_sonly.F90",
    "interface_h2": "tests/fortran/test_interface_h2.F90",
    "h2_ccpvdz": "tests/fortran/test_h2_ccpvdz.F90",
    "h2o_ccpvdz": "tests/fortran/test_h2o_ccpvdz.F90",
}

# the tests' pi_val literal and primitive norms (gto_norm_s/p/d in each test)
PI = 3.14159265358979323846264338327950288


def gto_norm(kind, a):
    base = (2.0 * a / PI) ** 0.75
    if kind == "s":
        return base
    if kind == "p":
        return 2.0 * math.sqrt(a) * base
    if kind == "d":
        return 4.0 * a * base
    if kind == "f":
        return 8.0 * a * math.sqrt(a) * base
    raise ValueError(kind)


REAL = r"[-+]?\d+\.?\d*(?:[dDeE][-+]?\d+)?(?:_dp)?"


def fnum(tok):
    tok = tok.strip().replace("_dp", "").replace("d", "e").replace("D", "e")
    return float(tok)


def eval_rhs(rhs):
    rhs = rhs.strip()
    m = re.fullmatch(r"(%s)\s*\*\s*gto_norm_([spd])\(\s*(%s)\s*\)" % (REAL, REAL), rhs)
    if m:
        return fnum(m.group(1)) * gto_norm(m.group(2), fnum(m.group(3)))
    if re.fullmatch(REAL, rhs):
        return fnum(rhs)
    return None


ALIASES = {
    "ang_mom_arr": "ang_mom", "contr_num_arr": "contr_num", "sh_loc_arr": "sh_loc",
    "atom_num_arr": "atom_num", "atom_loc_arr": "atom_loc", "start_bas_arr": "start_bas",
    "end_bas_arr": "end_bas", "exponents_arr": "exponents", "coords_arr": "coords",
    "contr_coef_s_arr": "coef_s", "contr_coef_p_arr": "coef_p", "contr_coef_d_arr": "coef_d",
    "contr_coef_f_arr": "coef_f", "contr_coef_s": "coef_s", "contr_coef_p": "coef_p",
    "contr_coef_d": "coef_d", "contr_coef_f": "coef_f",
}
INT_ARRAYS = {"ang_mom", "contr_num", "sh_loc", "atom_num", "atom_loc", "start_bas", "end_bas"}
SCALARS = {"nsh_val": "nsh", "natoms_val": "natoms", "num_bas_val": "num_bas", "mxgtot_val": "mxgtot"}


def parse(path):
    text = open(path).read()
    lines = text.splitlines()
    scal, arrs = {}, {}
    fa_ref, fa_line = [], None
    in_ref = False
    for ln, raw in enumerate(lines, 1):
        code = raw.split("!")[0]
        if "fa_ref(n_tri) = [" in code:
            in_ref, fa_line = True, ln
            continue
        if in_ref:
            fa_ref += [fnum(x) for x in re.findall(r"[-+]?\d+\.\d+[dD][-+]?\d+", code)]
            if "]" in code:
                in_ref = False
            continue
        for stmt in code.split(";"):
            stmt = stmt.strip()
            m = re.match(r"integer\s*,\s*parameter\s*::\s*(\w+)\s*=\s*(\d+)", stmt)
            if m and m.group(1) in SCALARS:
                scal[SCALARS[m.group(1)]] = int(m.group(2))
                continue
            m = re.fullmatch(r"(\w+)\s*=\s*(\d+)", stmt)
            if m and m.group(1) in SCALARS:
                scal[SCALARS[m.group(1)]] = int(m.group(2))
                continue
            m = re.fullmatch(r"(\w+)\((\d+)\)\s*=\s*(.+)", stmt)
            if m:
                name = ALIASES.get(m.group(1), m.group(1))
                val = eval_rhs(m.group(3))
                if val is None:
                    continue
                arrs.setdefault(name, {})[int(m.group(2))] = val
    return scal, arrs, fa_ref, fa_line


def build(ref_root, key, rel):
    scal, arrs, fa_ref, fa_line = parse(os.path.join(ref_root, rel))
    nsh, mx = scal["nsh"], scal["mxgtot"]
    out = dict(scal)
    for name in ["ang_mom", "contr_num", "sh_loc", "atom_num", "atom_loc", "start_bas", "end_bas"]:
        out[name] = [int(arrs[name][i]) for i in range(1, nsh + 1)]
    ncoef = mx * nsh
    for name in ["exponents", "coef_s", "coef_p", "coef_d", "coef_f"]:
        d = arrs.get(name, {})
        out[name] = [float(d.get(i, 0.0)) for i in range(1, ncoef + 1)]
    out["coords"] = [float(arrs["coords"][i]) for i in range(1, 3 * scal["natoms"] + 1)]
    n = scal["num_bas"]
    ntri = n * (n + 1) // 2
    assert len(fa_ref) == ntri, (key, len(fa_ref), ntri)
    out["schwrz"] = [1.0e10] * (nsh * (nsh + 1) // 2)
    dens = [0.0] * ntri
    for i in range(1, n + 1):
        dens[i * (i + 1) // 2 - 1] = 1.0
    out["density"] = dens
    out["fa_ref"] = fa_ref
    out["tol"] = 1.0e-10
    out["source"] = "%s (fa_ref at line %d)" % (rel, fa_line)
    return out


# ---- the f-shell known answer (tests/fortran/test_h2o_ccpvtz.F90) ------------
# That test fills its basis in two subroutines (oxygen; hydrogen with the atom
# and first shell as arguments) through integer variables, and reads its 2145
# reference values from fa_h2o_ccpvtz_reference.dat.  The small interpreter
# below runs exactly those statement forms; every expression is checked
# against a whitelist before evaluation (the reference is read as data).
F_TEST = "tests/fortran/test_h2o_ccpvtz.F90"
F_DAT = "tests/fortran/fa_h2o_ccpvtz_reference.dat"
_SAFE = re.compile(r"^[\w\s+\-*/().]*$")


def _fexpr(expr, env, arrs):
    expr = expr.strip()
    m = re.fullmatch(r"(%s)\s*\*\s*gto_norm_([spdf])\(\s*(%s)\s*\)" % (REAL, REAL), expr)
    if m:
        return fnum(m.group(1)) * gto_norm(m.group(2), fnum(m.group(3)))
    if re.fullmatch(REAL, expr):
        return fnum(expr)
    # integer arithmetic over the subroutine's variables and array reads
    expr = re.sub(r"(\w+_arr)\(([^()]*)\)",
                  lambda mm: repr(arrs[ALIASES[mm.group(1)]][int(_fexpr(mm.group(2), env, arrs))]), expr)
    if not _SAFE.match(expr):
        raise ValueError("unexpected expression: %r" % expr)
    for name in re.findall(r"[A-Za-z_]\w*", expr):
        if name not in env:
            raise ValueError("unknown name %r in %r" % (name, expr))
    return eval(expr, {"__builtins__": {}}, dict(env))


def _run_body(lines, env, arrs):
    active = [True]
    for raw in lines:
        code = raw.split("!")[0].strip()
        if not code:
            continue
        m = re.fullmatch(r"if\s*\((\w+)\s*==\s*(\d+)\)\s*then", code)
        if m:
            active.append(active[-1] and env[m.group(1)] == int(m.group(2)))
            continue
        if code == "else":
            active[-1] = active[-2] and not active[-1]
            continue
        if code in ("end if", "endif"):
            active.pop()
            continue
        if not active[-1] or code.startswith("integer"):
            continue
        for stmt in code.split(";"):
            stmt = stmt.strip()
            m = re.fullmatch(r"(\w+)\(([^=]*)\)\s*=\s*(.+)", stmt)
            if m and m.group(1) in ALIASES:
                idx = int(_fexpr(m.group(2), env, arrs))
                arrs.setdefault(ALIASES[m.group(1)], {})[idx] = _fexpr(m.group(3), env, arrs)
                continue
            m = re.fullmatch(r"(\w+)\s*=\s*(.+)", stmt)
            if m:
                env[m.group(1)] = int(_fexpr(m.group(2), env, arrs))
                continue
            raise ValueError("unexpected statement: %r" % stmt)


def build_f(ref_root):
    text = open(os.path.join(ref_root, F_TEST)).read().splitlines()
    subs, cur = {}, None
    for raw in text:
        code = raw.split("!")[0].strip()
        m = re.match(r"subroutine\s+(\w+)\s*\(([^)]*)\)", code)
        if m:
            cur = m.group(1)
            subs[cur] = ([a.strip() for a in m.group(2).split(",") if a.strip()], [])
            continue
        if code.startswith("end subroutine"):
            cur = None
            continue
        if cur:
            subs[cur][1].append(raw)
    scal, arrs, _, _ = parse(os.path.join(ref_root, F_TEST))  # scalars and coordinates
    for raw in text:
        m = re.match(r"\s*call\s+(setup_\w+)\s*\(([^)]*)\)", raw.split("!")[0])
        if not m:
            continue
        params, body = subs[m.group(1)]
        args = [int(a) for a in m.group(2).split(",") if a.strip()]
        _run_body(body, dict(zip(params, args)), arrs)
    vals = open(os.path.join(ref_root, F_DAT)).read().split()
    count, fa_ref = int(vals[0]), [fnum(v) for v in vals[1:]]
    assert count == len(fa_ref)
    nsh, mx = scal["nsh"], scal["mxgtot"]
    out = dict(scal)
    for name in ["ang_mom", "contr_num", "sh_loc", "atom_num", "atom_loc", "start_bas", "end_bas"]:
        out[name] = [int(arrs[name][i]) for i in range(1, nsh + 1)]
    for name in ["exponents", "coef_s", "coef_p", "coef_d", "coef_f"]:
        d = arrs.get(name, {})
        out[name] = [float(d.get(i, 0.0)) for i in range(1, mx * nsh + 1)]
    out["coords"] = [float(arrs["coords"][i]) for i in range(1, 3 * scal["natoms"] + 1)]
    n = scal["num_bas"]
    ntri = n * (n + 1) // 2
    assert len(fa_ref) == ntri, (len(fa_ref), ntri)
    out["schwrz"] = [1.0e10] * (nsh * (nsh + 1) // 2)
    dens = [0.0] * ntri
    for i in range(1, n + 1):
        dens[i * (i + 1) // 2 - 1] = 1.0
    out["density"] = dens
    out["fa_ref"] = fa_ref
    out["tol"] = 1.0e-10
    out["source"] = "%s (basis), %s (values)" % (F_TEST, F_DAT)
    return out


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LIBERI_REFERENCE", "")
    if not ref_root or not os.path.isdir(ref_root):
        sys.exit("usage: make_golden.py <reference checkout>")
    here = os.path.dirname(os.path.abspath(__file__))
    for key, rel in TESTS.items():
        fx = build(ref_root, key, rel)
        with open(os.path.join(here, key + ".json"), "w") as f:
            json.dump(fx, f, indent=0)
        print(key, "nsh", fx["nsh"], "nbf", fx["num_bas"], "values", len(fx["fa_ref"]))
    fx = build_f(ref_root)
    with open(os.path.join(here, "h2o_ccpvtz.json"), "w") as f:
        json.dump(fx, f, indent=0)
    print("h2o_ccpvtz", "nsh", fx["nsh"], "nbf", fx["num_bas"], "values", len(fx["fa_ref"]))


if __name__ == "__main__":
    main()
