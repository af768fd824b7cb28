"""The Julia binding (pdcs_b200/julia/PDCSB200.jl) repeats the C structs of
include/pdcs.h for ccall.  Julia is not installed here, so the binding cannot
run; this test checks what can be checked without it: every struct the
binding passes to the library has the header's fields, in the header's
order, with the same widths, and every entry point it calls is exported by
the header."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pdcs.h")
JULIA = os.path.join(ROOT, "pdcs_b200", "julia", "PDCSB200.jl")

STRUCTS = {"pdcs_problem": "PdcsProblem", "pdcs_options": "PdcsOptions", "pdcs_result": "PdcsResult",
           "pdcs_batch_info": "PdcsBatchInfo", "pdcs_grad_options": "PdcsGradOptions",
           "pdcs_grad_info": "PdcsGradInfo"}
C2J = {"int64_t": "Int64", "int32_t": "Int32", "double": "Float64"}


def c_structs():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for body, name in re.findall(r"typedef struct\s*\{(.*?)\}\s*(\w+)\s*;", text, re.S):
        fields = []
        for decl in body.split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            decl = decl.replace("const ", "")
            m = re.match(r"(\w+)\s*(\**)\s*(.*)", decl)
            base, stars, names = m.group(1), m.group(2), m.group(3)
            for nm in names.split(","):
                nm = nm.strip()
                ptr = stars + "*" * nm.count("*")
                nm = nm.strip("* ")
                if ptr:
                    jt = "Ptr{Cvoid}" if base == "void" else "Ptr{%s}" % C2J[base]
                else:
                    jt = C2J[base]
                fields.append((nm, jt))
        out[name] = fields
    return out


def julia_structs():
    text = open(JULIA).read()
    out = {}
    for name, body in re.findall(r"^(?:mutable )?struct (\w+)\n(.*?)^end", text, re.S | re.M):
        fields = []
        for line in body.splitlines():
            m = re.match(r"\s+(\w+)::(\S+)\s*$", line)
            if m:
                fields.append((m.group(1), m.group(2)))
        out[name] = fields
    return out


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_julia_structs_match_header(cname):
    c = c_structs()[cname]
    j = julia_structs()[STRUCTS[cname]]
    assert j == c, (cname, [x for x in zip(c, j) if x[0] != x[1]][:3], len(c), len(j))


def test_julia_calls_only_exported_entry_points():
    header = open(HEADER).read()
    exported = set(re.findall(r"^\s*(?:int|void|const char\*)\s+(pdcs_\w+)\s*\(", header, re.M))
    called = set(re.findall(r"ccall\(\(:(pdcs_\w+),", open(JULIA).read()))
    assert called and called <= exported, called - exported
