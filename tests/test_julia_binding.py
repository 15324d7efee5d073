"""The Julia binding (julia/PeriDynB200.jl) against the C header.

No Julia toolchain exists where the library is built, so the binding is
checked as text: every `ccall((:name, LIB), Ret, (Args...), ...)` must name a
function declared in include/peridyn_b200.h with the same number of
arguments and matching types (Julia's `Int32`/`Int64`/`Float64`/`Ptr{T}`/
`Ref{T}`/`CuPtr{T}` against the C types; device-pointer arguments must be
`CuPtr`, host arrays `Ptr`), the `MaterialDesc` struct must list the fields
of `pd_material_desc` in order with matching types, the integer constants
must equal the header's enums, and the methods the reference's call sites
reach must exist with the reference's argument shapes (run! calls
`apply_solver!(env, solver)`, solvers.jl:148; force_density! calls
`force_density_T!(f, y, limits, mat, device)`, general_material.jl:245).
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "julia", "PeriDynB200.jl")
HDR = os.path.join(ROOT, "include", "peridyn_b200.h")


def _strip_c_comments(s):
    s = re.sub(r"/\*.*?\*/", " ", s, flags=re.S)
    return re.sub(r"//[^\n]*", " ", s)


def header_functions():
    src = _strip_c_comments(open(HDR).read())
    out = {}
    for m in re.finditer(r"PD_API\s+([^;(]+?)\s*\b(\w+)\s*\(([^)]*)\)\s*;", src, flags=re.S):
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3).strip()
        params = [] if args in ("", "void") else [a.strip() for a in args.split(",")]
        out[name] = (ret, params)
    return out


def header_struct(name):
    src = _strip_c_comments(open(HDR).read())
    m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), src, flags=re.S)
    fields = []
    for decl in m.group(1).split(";"):
        decl = decl.strip()
        if decl:
            fields.append(decl)
    return fields


def header_enums():
    src = _strip_c_comments(open(HDR).read())
    vals = {}
    for body in re.findall(r"enum\s*\{(.*?)\}", src, flags=re.S):
        for item in body.split(","):
            m = re.match(r"\s*(\w+)\s*=\s*(-?\d+)", item)
            if m:
                vals[m.group(1)] = int(m.group(2))
    m = re.search(r"#define PD_ABI_VERSION (\d+)", src)
    vals["PD_ABI_VERSION"] = int(m.group(1))
    return vals


def _split_top(s):
    """Split a Julia tuple body on top-level commas (braces nest)."""
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch == "{":
            depth += 1
        elif ch == "}":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        parts.append(cur.strip())
    return parts


def julia_ccalls():
    src = open(JL).read()
    calls = []
    for m in re.finditer(r"ccall\(\(:(\w+),\s*LIB\),\s*([\w{}]+),\s*\(([^()]*)\)", src, flags=re.S):
        calls.append((m.group(1), m.group(2), _split_top(" ".join(m.group(3).split()))))
    return calls


def c_param_type(param):
    """C parameter declaration -> normalised type (name dropped)."""
    p = " ".join(param.replace("*", " * ").split())
    toks = p.split(" ")
    if toks[-1] != "*" and len(toks) > 1:
        name = toks[-1]
        toks = toks[:-1]
    else:
        name = ""
    t = " ".join(toks).replace("const ", "").replace(" *", "*").replace(" ", "")
    return t, name


# Julia ccall type -> the C types it may stand for (host memory)
ALLOWED = {
    "Int32": {"int32_t", "pd_status", "int"},
    "Cint": {"int32_t", "int"},
    "Int64": {"int64_t"},
    "Float64": {"double"},
    "Ptr{Cvoid}": {"pd_env*", "void*"},
    "Ptr{Ptr{Cvoid}}": {"pd_env**", "void**"},
    "Ptr{Float64}": {"double*"},
    "Ptr{Int64}": {"int64_t*"},
    "Ptr{Int32}": {"int32_t*"},
    "Ptr{UInt8}": {"uint8_t*"},
    "Ref{Int64}": {"int64_t*"},
    "Ref{MaterialDesc}": {"pd_material_desc*"},
    "Cstring": {"char*"},
    "CuPtr{Cvoid}": {"double*"},
    "CuPtr{Float64}": {"double*"},
}


def test_every_ccall_matches_the_header():
    fns = header_functions()
    calls = julia_ccalls()
    assert len(calls) >= 20
    seen = set()
    for name, ret, jargs in calls:
        assert name in fns, f"{name} is not declared in the header"
        cret, cparams = fns[name]
        seen.add(name)
        cret_t = cret.replace("const ", "").replace(" ", "")
        assert cret_t in ALLOWED[ret], f"{name}: return {ret} vs {cret}"
        assert len(jargs) == len(cparams), f"{name}: {len(jargs)} arguments in Julia, {len(cparams)} in C"
        for k, (jt, cp) in enumerate(zip(jargs, cparams)):
            ct, cname = c_param_type(cp)
            assert jt in ALLOWED, f"{name} arg {k}: unknown Julia type {jt}"
            assert ct in ALLOWED[jt], f"{name} arg {k} ({cname}): Julia {jt} vs C {ct}"
            device = cname.endswith("_dev")
            assert device == jt.startswith("CuPtr"), f"{name} arg {k} ({cname}): device pointer needs CuPtr, host Ptr"
    for needed in ("pd_env_vv_steps", "pd_env_qsdrag", "pd_env_update_acc", "pd_force_density_device",
                   "pd_env_update_neighs", "pd_env_damage", "pd_env_get_state", "pd_env_set_state",
                   "pd_env_add_block", "pd_env_set_family", "pd_env_finalize"):
        assert needed in seen, f"the binding never calls {needed}"


def test_material_desc_matches_the_c_struct():
    cfields = header_struct("pd_material_desc")
    src = open(JL).read()
    m = re.search(r"struct MaterialDesc\n(.*?)\nend", src, flags=re.S)
    jfields = [ln.strip() for ln in m.group(1).splitlines() if "::" in ln]
    assert len(jfields) == len(cfields), (jfields, cfields)
    tmap = {"int32_t": "Int32", "int64_t": "Int64", "double": "Float64", "double*": "Ptr{Float64}"}
    for jf, cf in zip(jfields, cfields):
        jname, jt = [t.strip() for t in jf.split("::")]
        ct, cname = c_param_type(cf)
        assert jname == cname, f"field {jname} vs {cname}"
        assert tmap[ct] == jt, f"field {jname}: Julia {jt} vs C {ct}"


def test_constants_match_the_header():
    enums = header_enums()
    src = open(JL).read()
    consts = re.findall(r"const (PD_\w+) = (?:Int32\()?(-?\d+)\)?", src)
    assert len(consts) >= 10
    for name, val in consts:
        assert name in enums, name
        assert enums[name] == int(val), f"{name} = {val}, header {enums[name]}"


@pytest.mark.parametrize("pattern", [
    # run! (solvers.jl:148) calls apply_solver!(envs[id], solver): two positional arguments
    r"function apply_solver!\(env::PeriDyn\.GeneralEnvironment, solver::PeriDyn\.DSVelocityVerlet\)",
    r"function apply_solver!\(env::PeriDyn\.GeneralEnvironment, s::PeriDyn\.QSDrag\)",
    # force_density! (general_material.jl:245): force_density_T!(f, y, limits, mat, Val{:cuda}), no env keyword
    r"function force_density_T!\(f::CuMatrix\{Float64\}, y::CuMatrix\{Float64\}, limits, "
    r"mat::PeriDyn\.PeridynamicsMaterial,\s*::Type\{Val\{:cuda\}\}; particles=nothing\)",
    r"function update_acc!\(env::PeriDyn\.GeneralEnvironment\)",
    r"function update_neighs!\(envs::Vector\{PeriDyn\.GeneralEnvironment\}; max_part=30\)",
])
def test_methods_reached_from_the_reference_call_sites(pattern):
    src = open(JL).read()
    assert re.search(pattern, src), pattern
    # no method may require an env= keyword that the reference never passes
    assert "env=nothing" not in src
