"""CPU checks of the Julia backend files against the C ABI.

libnegf.jl_b200/julia/backend_nvidia.jl is the drop-in for LibNEGF.jl's
src/backend_cpu.jl and backend_nvidia_sweeps.jl overrides the algorithm
functions with whole-sweep library calls.  No Julia toolchain exists here, so
the files are checked as text: every ccall names a function that
include/negf_b200.h declares, with the same number of arguments and the same
kind (pointer, 32-bit integer, char, double, 64-bit integer) in each position,
and the backend defines every be_* function of backend_cpu.jl with the same
positional arity.
"""

import os
import re

import pytest

from conftest import ROOT

JULIA = os.path.join(ROOT, "libnegf.jl_b200", "julia")
HEADER = os.path.join(ROOT, "include", "negf_b200.h")

# the be_* functions of src/backend_cpu.jl:26-289 and their positional arity
REFERENCE_BE = {
    "be_copy_to_hw!": 2, "be_copy_to_hw": 1, "be_copy_from_hw!": 2, "be_copy_from_hw": 1, "be_copy_in_hw!": 2,
    "be_copy_in_hw": 1, "be_zero_array": 1, "be_identity": 1, "be_ctranspose!": 4, "be_ctranspose": 3,
    "be_random_array": 1, "be_fill!": 2, "be_A_from_LU": 1, "be_zero_lu": 1, "be_inv": 1, "be_lu!": 4, "be_lu": 3,
    "be_inv_from_lu!": 2, "be_mldivide!": 6, "be_gemm!": 9, "be_mul": 2, "be_getri!": 3, "be_trsm!": 9,
    "be_getrf!": 3, "be_potrf!": 4, "be_herk!": 8,
}
# the algorithm functions the sweeps file overrides, and their arity
REFERENCE_SWEEPS = {
    "bndiag_of_inv_rgf_local!": 5, "bndiag_of_inv_rgf_global!": 5, "keldyshndiag!": 5,
    "bndiag_of_inv_general_rgf!": 5, "Block_factorization!": 3, "Block_inverse!": 3, "bndiag_of_inv_ddrgf!": 5,
    "opt_params": 4,
}


def _split_top(s):
    """Split at commas outside brackets."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def _c_kind(t):
    t = t.strip()
    if "*" in t:
        return "ptr"
    t = re.sub(r"\b(const|unsigned)\b", "", t)
    t = re.sub(r"\s+\w+$", "", t.strip()).strip() if len(t.split()) > 1 else t
    return {"int32_t": "i32", "int": "i32", "char": "char", "double": "f64", "int64_t": "i64",
            "uint8_t": "u8", "void": "void", "CCscMatrix": "struct"}.get(t.strip(), "?" + t)


def _jl_kind(t):
    t = t.strip()
    if t.startswith(("Ptr{", "Ref{")) or t in ("Cstring", "Ptr"):
        return "ptr"
    return {"Int32": "i32", "Cint": "i32", "Cchar": "char", "Float64": "f64", "Cdouble": "f64", "Int64": "i64",
            "UInt8": "u8"}.get(t, "?" + t)


def _header_protos():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = "\n".join(line for line in text.splitlines() if not line.lstrip().startswith("#"))
    protos = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(negf_\w+|run_bndiag_wrapper)\s*\(([^;{]*?)\)\s*;", text, re.S):
        ret, name, args = m.group(1), m.group(2), " ".join(m.group(3).split())
        kinds = [] if args in ("", "void") else [_c_kind(a) for a in _split_top(args)]
        protos[name] = (_c_kind(ret + " x") if "*" not in ret else "ptr", kinds)
    return protos


def _ccalls(text):
    calls = []
    for m in re.finditer(r"ccall\(\(:(\w+),\s*LIBNEGF\),\s*", text):
        i = m.end()
        # return type up to the next top-level comma, then the argument type tuple
        depth, j = 0, i
        while not (text[j] == "," and depth == 0):
            depth += text[j] in "({[" and 1 or 0
            depth -= text[j] in ")}]" and 1 or 0
            j += 1
        ret = text[i:j].strip()
        k = text.index("(", j)
        depth, e = 0, k
        while True:
            depth += text[e] == "("
            depth -= text[e] == ")"
            if depth == 0:
                break
            e += 1
        types = _split_top(text[k + 1:e])
        calls.append((m.group(1), ret, [_jl_kind(t) for t in types if t]))
    return calls


def _jl_text():
    return "\n".join(open(os.path.join(JULIA, f)).read() for f in sorted(os.listdir(JULIA)) if f.endswith(".jl"))


def test_every_ccall_matches_the_header():
    protos = _header_protos()
    calls = _ccalls(_jl_text())
    assert len(calls) >= 12
    for name, ret, kinds in calls:
        assert name in protos, "ccall of %s, which include/negf_b200.h does not declare" % name
        cret, ckinds = protos[name]
        assert len(kinds) == len(ckinds), (name, kinds, ckinds)
        for a, (jk, ck) in enumerate(zip(kinds, ckinds)):
            assert jk == ck, "%s argument %d: Julia %s, C %s" % (name, a + 1, jk, ck)
        assert (ret == "Cstring" and cret == "ptr") or (ret == "Cint" and cret == "i32"), (name, ret, cret)


def _jl_functions(text):
    """name -> positional arity of every one-line or block method definition."""
    out = {}
    for m in re.finditer(r"^(?:function\s+)?([A-Za-z_][\w!]*)\(([^)]*)\)\s*(?:::\s*[\w{},]+\s*)?(?:=|$)", text,
                         re.M):
        name, args = m.group(1), m.group(2)
        pos = args.split(";")[0]
        out.setdefault(name, set()).add(len([a for a in _split_top(pos) if a]))
    return out


def test_backend_defines_every_be_function_of_backend_cpu():
    fns = _jl_functions(open(os.path.join(JULIA, "backend_nvidia.jl")).read())
    for name, arity in REFERENCE_BE.items():
        assert name in fns, "backend_nvidia.jl lacks %s (src/backend_cpu.jl)" % name
        assert arity in fns[name], (name, fns[name])


def test_sweeps_file_overrides_the_algorithm_functions():
    fns = _jl_functions(open(os.path.join(JULIA, "backend_nvidia_sweeps.jl")).read())
    for name, arity in REFERENCE_SWEEPS.items():
        assert name in fns and arity in fns[name], (name, fns.get(name))


@pytest.mark.parametrize("fname", ["backend_nvidia.jl", "backend_nvidia_sweeps.jl"])
def test_backend_has_no_cpu_compute(fname):
    """Compute reaches the GPU through ccall only: no LAPACK / BLAS / CPU
    linear algebra calls in the backend."""
    text = open(os.path.join(JULIA, fname)).read()
    code = "\n".join(line.split("#")[0] for line in text.splitlines())
    assert "LAPACK." not in code and "BLAS." not in code, fname
    assert not re.search(r"(?<![\w.!])(inv|lu|adjoint|mul!|ldiv!)\(", code), fname
