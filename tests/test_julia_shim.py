"""CPU checks of the Julia shim (dav-qed2d_b200/julia/QED2d.jl), read as text
because Julia is not installed here:

* it exports every name the reference module exports (src/QED2d.jl:27-54) and
  defines each of them, plus the unexported functions the reference's own tests
  call qualified (QED2d.LuscherZ, test/rhmc_zolovarev_bound.jl:63);
* every ccall names a function that include/qed2d.h declares, passes as many
  values as it lists argument types, and its argument and return types are the
  C types of the declaration (pointer, int32, int64, uint32, uint64, double);
* the shim's mirrors of the C structs (CRhmc, CHmcResult) list the fields of
  qed2d_rhmc_params and qed2d_hmc_result with the same types in the same order;
* the Zolotarev helpers the shim exports (k, v, a_r, ... written on the library's
  elliptic functions) agree, through the Python mirror that shares their
  definitions, with the library's coefficients and with scipy."""
import os
import re

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(REPO, "dav-qed2d_b200", "julia", "QED2d.jl")
HEADER = os.path.join(REPO, "include", "qed2d.h")

# export lists of the reference module, src/QED2d.jl:27-54 (leapgrog! is the
# reference's own spelling; it defines leapfrog!)
REFERENCE_EXPORTS = """
LattParm KernelParm RHMCParm Integrators Leapfrog OMF4
plaquette! qtop! updt_fld! krnl_force!
HMC! Hamiltonian Action Plaquette Qtop OMF4! leapgrog! update_momenta!
unfold_fld! unfold_reflect!
gamm5Dw gamm5Dw_sqr gamm5Dw_sqr_msq tr_dQwdU gamm5Dw_sqr_musq gamm5Dw_sqr_sqr_musq gamm5Dw_sqr_sqr gamm5 Dw
CG save_gauge load_gauge
k v a_r c_r mu nu rho_mu P d A delta error get_rhmc_params power_method reweighting_factor R MultiCG
generate_pseudofermion!
plwv
""".split()
QUALIFIED = ["LuscherZ"]


def shim_text():
    return open(SHIM).read()


def strip_comments(src):
    return "\n".join(line.split("#", 1)[0] if not line.lstrip().startswith("#") else "" for line in src.split("\n"))


def exports(src):
    names = []
    lines = src.split("\n")
    i = 0
    while i < len(lines):
        line = lines[i].strip()
        if line.startswith("export "):
            body = line[len("export "):]
            while body.rstrip().endswith(",") and i + 1 < len(lines):
                i += 1
                body += " " + lines[i].strip()
            names += [n.strip() for n in body.split(",") if n.strip()]
        i += 1
    return names


def defined(src, name):
    n = re.escape(name)
    pats = [rf"^\s*function\s+{n}\s*\(", rf"^\s*{n}\s*\(.*\)\s*=", rf"^\s*const\s+{n}\s*=",
            rf"^\s*(mutable\s+)?struct\s+{n}\b", rf"^\s*abstract\s+type\s+{n}\b", rf"\(:{n},\s*:qed2d_\w+\)"]
    return any(re.search(p, src, re.M) for p in pats)


def split_top(s):
    """Split s at top-level commas (outside (), {}, [])."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def balanced(s, start):
    """s[start] == '('; return the text inside the matching parentheses."""
    depth = 0
    for i in range(start, len(s)):
        if s[i] == "(":
            depth += 1
        elif s[i] == ")":
            depth -= 1
            if depth == 0:
                return s[start + 1:i]
    raise ValueError("unbalanced")


def ccalls(src):
    """(symbols, return type, [argument types], number of values) of every ccall."""
    out = []
    for m in re.finditer(r"ccall\(", src):
        inner = balanced(src, m.end() - 1)
        parts = split_top(inner)
        target, ret, types = parts[0], parts[1], parts[2]
        values = parts[3:]
        assert types.startswith("(") and types.endswith(")"), types
        tl = split_top(types[1:-1])
        if "QuoteNode" in target:   # @eval loop: the symbols come from the loop's tuple list
            head = src[:m.start()]
            loop = head[head.rfind("for (jl, c) in"):]
            syms = re.findall(r":(qed2d_\w+)", loop)
        else:
            syms = re.findall(r":(qed2d_\w+)", target)
        assert syms, target
        out.append((syms, ret, tl, len(values)))
    return out


JL_TYPES = {"Cint": "i32", "Int32": "i32", "Int64": "i64", "UInt64": "u64", "UInt32": "u32", "Cdouble": "f64",
            "Float64": "f64", "Cstring": "ptr", "CPtrD": "ptr"}


def jl_kind(t):
    t = t.strip()
    if t.startswith(("Ptr{", "Ref{", "CUDA.CuPtr{")):
        return "ptr"
    return JL_TYPES[t]


def c_kind(t):
    t = t.strip()
    if "*" in t:
        return "ptr"
    t = t.replace("const ", "").strip()
    return {"int": "i32", "int32_t": "i32", "int64_t": "i64", "uint64_t": "u64", "uint32_t": "u32",
            "double": "f64"}[t]


def header_decls():
    txt = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    decls = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(qed2d_\w+)\s*\(([^;{]*?)\)\s*;", txt, re.S):
        ret, name, params = m.group(1), m.group(2), m.group(3)
        ps = [] if params.strip() in ("", "void") else [p for p in split_top(params)]
        kinds = []
        for p in ps:
            p = " ".join(p.split())
            typ = re.sub(r"\b\w+\s*$", "", p) if not p.endswith("*") else p   # drop the parameter name
            kinds.append(c_kind(typ))
        decls[name] = (c_kind(ret.strip().split("\n")[-1]), kinds)
    return decls


def test_shim_exports_the_reference_api():
    src = strip_comments(shim_text())
    ex = set(exports(src))
    missing = [n for n in REFERENCE_EXPORTS if n not in ex]
    assert not missing, missing
    undefined = [n for n in REFERENCE_EXPORTS + QUALIFIED if not defined(src, n)]
    assert not undefined, undefined


def test_shim_ccalls_match_the_header():
    src = strip_comments(shim_text())
    decls = header_decls()
    calls = ccalls(src)
    assert len(calls) > 30
    seen = set()
    for syms, ret, types, nvalues in calls:
        assert len(types) == nvalues, (syms, types, nvalues)
        kinds = [jl_kind(t) for t in types]
        for s in syms:
            assert s in decls, f"{s} is not declared in include/qed2d.h"
            cret, ckinds = decls[s]
            assert kinds == ckinds, (s, kinds, ckinds)
            assert jl_kind(ret) == cret, (s, ret, cret)
            seen.add(s)
    # every reference-facing entry point is reachable from Julia
    for s in ["qed2d_cg", "qed2d_cg_shift", "qed2d_hmc_nf2", "qed2d_hmc_rhmc", "qed2d_omf4_nf2",
              "qed2d_leapfrog_rhmc", "qed2d_update_momenta_rhmc", "qed2d_luscher_z", "qed2d_ellip_sncn"]:
        assert s in seen, s


def jl_struct(src, name):
    m = re.search(rf"^struct {name}\n(.*?)^end", src, re.S | re.M)
    fields = []
    for part in re.split(r"[;\n]", m.group(1)):
        part = part.strip()
        if part:
            fname, typ = part.split("::")
            t = typ.strip()
            tup = re.match(r"NTuple\{(\d+),\s*(\w+)\}", t)
            fields.append((fname.strip(), f"{JL_TYPES[tup.group(2)]}[{tup.group(1)}]" if tup else JL_TYPES[t]))
    return fields


def c_struct(name):
    txt = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    m = re.search(r"typedef struct \{([^{}]*)\}\s*" + name + ";", txt)
    fields = []
    for decl in m.group(1).split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        arr = re.match(r"(\w+) (\w+)\[(\w+)\]", decl)
        if arr:
            fields.append((arr.group(2), f"{c_kind(arr.group(1))}[32]"))
            assert arr.group(3) == "QED2D_MAXPOLES"
        else:
            typ, fname = decl.rsplit(" ", 1)
            fields.append((fname, c_kind(typ)))
    return fields


def test_shim_structs_match_the_header():
    src = strip_comments(shim_text())
    assert jl_struct(src, "CRhmc") == c_struct("qed2d_rhmc_params")
    assert jl_struct(src, "CHmcResult") == c_struct("qed2d_hmc_result")


def test_zolotarev_helpers_vs_library_and_scipy():
    """k, v, a_r, c_r, mu, nu, rho_mu, d, A, delta, P and error as the reference
    writes them (src/QED2dRHMC.jl:2-89), evaluated on the library's elliptic
    functions: equal to get_rhmc_params' coefficients, the elliptic functions
    equal to scipy's, and the approximation within delta on [r_a^2, r_b^2]."""
    from scipy.special import ellipj, ellipk

    import qed2d
    n, r_a, r_b = 7, 0.3, 4.0
    eps = (r_a / r_b) ** 2
    m = qed2d.k(eps) ** 2
    assert abs(qed2d.v(n, eps) - ellipk(m) / (2 * n + 1)) < 1e-14 * ellipk(m)
    for r in (1, 4, 2 * n + 1):
        sn, cn, _, _ = ellipj(r * qed2d.v(n, eps), m)
        assert abs(qed2d.c_r(r, n, eps) - sn ** 2) < 1e-13
        assert abs(qed2d.a_r(r, n, eps) - cn ** 2 / sn ** 2) < 1e-12 * (cn ** 2 / sn ** 2)
    p = qed2d.get_rhmc_params(n, r_a, r_b)
    for j in range(1, n + 1):
        assert qed2d.mu(j, n, eps, r_b) == pytest.approx(p.mu[j - 1], rel=1e-14)
        assert qed2d.nu(j, n, eps, r_b) == pytest.approx(p.nu[j - 1], rel=1e-14)
        assert qed2d.rho_mu(j, 1, n, n, eps, r_b) == pytest.approx(p.rho[j - 1], rel=1e-12)
    assert qed2d.delta(n, eps) == pytest.approx(p.delta, rel=1e-12)
    assert qed2d.A(n, eps) == pytest.approx(p.A, rel=1e-14)
    assert qed2d.rho_nu(2, 1, n, n, eps, r_b) != 0.0
    with pytest.raises(ValueError):
        qed2d.rho_mu(0, 1, n, n, eps, r_b)
    # |1 - sqrt(Y) (A / r_b) P(Y)| <= delta across the spectral interval
    for Y in np.geomspace(r_a ** 2, r_b ** 2, 25):
        approx = (qed2d.A(n, eps) / r_b) * qed2d.P(1, n, n, eps, r_b, Y)
        assert qed2d.error(Y, approx) <= qed2d.delta(n, eps) + 1e-14   # equioscillates: = delta at the ends
    # the C entry points reject a parameter outside [0, 1)
    import ctypes as C
    from qed2d import _lib
    out = C.c_double(0)
    assert _lib.lib().qed2d_ellip_K(1.0, C.byref(out)) == _lib.BAD_ARG
