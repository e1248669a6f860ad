"""The Julia ccall shim (pmf-glm_b200/julia/pmfmhd_shim.jl) cannot run here (no Julia in the
image); these checks keep it consistent with the C header and with INTEGRATION.md, which
quotes it."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "pmf-glm_b200", "julia", "pmfmhd_shim.jl")
HEADER = os.path.join(ROOT, "include", "pmfmhd.h")

C_TO_JULIA = {"int32_t": "Int32", "float": "Float32", "double": "Float64", "int64_t": "Int64"}


def header_grid_fields():
    text = open(HEADER).read()
    body = re.search(r"typedef struct pmfmhd_grid \{(.*?)\} pmfmhd_grid;", text, flags=re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        ctype, names = decl.split(None, 1)
        for name in names.split(","):
            name = name.strip()
            m = re.match(r"(\w+)\[(\d+)\]", name)
            if m:
                fields.append((m.group(1), f"NTuple{{{m.group(2)},{C_TO_JULIA[ctype]}}}"))
            else:
                fields.append((name, C_TO_JULIA[ctype]))
    return fields


def shim_grid_fields():
    text = open(SHIM).read()
    body = re.search(r"struct PmfGrid[^\n]*\n(.*?)\nend", text, flags=re.S).group(1)
    return re.findall(r"(\w+)::([\w{},]+)", body)


def test_pmfgrid_matches_the_c_struct():
    assert shim_grid_fields() == header_grid_fields()


def test_integration_notes_quote_the_shim_verbatim():
    notes = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    assert open(SHIM).read() in notes


def test_shim_binds_only_declared_symbols():
    header = open(HEADER).read()
    for sym in set(re.findall(r"ccall\(\(:(\w+),", open(SHIM).read())):
        assert re.search(r"\b%s\s*\(" % sym, header), sym
