"""The Julia backend package (lcs.jl_b200/LCSB200) against the C ABI and the
reference's package metadata, without Julia.

- Project.toml names every dependency with the reference's UUID (Project.toml
  [deps] of LCS.jl, extracted into tests/golden/known_answers.json), and the
  workspace packages resolve by path from a checkout in which LCSB200/ sits
  beside LCSCUDA/, as LCSCUDA/Project.toml [sources] does.
- Every `struct` of src/abi.jl has the layout of its C counterpart in
  include/lcs_b200.h (LcsConfig <-> lcs_config, ...): the same number of
  fields, each of the same size at the same offset, and the same total size.
  Julia lays out an isbits struct with C alignment, so the offsets follow from
  the field types.
"""

import json
import os
import re
import subprocess
import tempfile
import tomllib

import pytest

from conftest import ROOT

SHIM = os.path.join(ROOT, "lcs.jl_b200", "LCSB200")
HEADER = os.path.join(ROOT, "include", "lcs_b200.h")
KNOWN = json.load(open(os.path.join(ROOT, "tests", "golden", "known_answers.json")))["julia_packages"]


def test_project_uuids_and_sources():
    proj = tomllib.load(open(os.path.join(SHIM, "Project.toml"), "rb"))
    uuids = KNOWN["uuids"]
    for name, uuid in proj["deps"].items():
        assert name in uuids, f"{name} is not a dependency of LCS.jl"
        assert uuid == uuids[name], (name, uuid, uuids[name])
    # LCS and the workspace packages (lib/*) resolve by path from beside LCSCUDA/
    local = {"LCS": ".."} | {k: "../" + v for k, v in KNOWN["root_sources"].items()}
    for name in proj["deps"]:
        if name in local:
            assert proj["sources"][name]["path"] == local[name], name
    for name, path in KNOWN["lcscuda_sources"].items():
        if name in proj["deps"]:
            assert proj["sources"][name]["path"] == path


# ------------------------------------------------------------------ layouts
SCALARS = {"Int32": (4, 4), "Cint": (4, 4), "UInt32": (4, 4), "Int64": (8, 8), "Float64": (8, 8),
           "Cdouble": (8, 8), "Ptr{Cvoid}": (8, 8)}


def julia_structs():
    src = open(os.path.join(SHIM, "src", "abi.jl")).read()
    consts = {m.group(1): int(m.group(2)) for m in re.finditer(r"^const (\w+) = (\d+)\s*$", src, re.M)}
    structs = {}
    for m in re.finditer(r"^struct (\w+)\n(.*?)^end", src, re.M | re.S):
        fields = []
        for ln in m.group(2).splitlines():
            ln = ln.split("#")[0]
            for part in ln.split(";"):
                part = part.strip()
                if part:
                    name, typ = part.split("::")
                    fields.append((name.strip(), typ.strip()))
        structs[m.group(1)] = fields
    return structs, consts


def julia_layout(structs, consts, name, cache):
    """(size, alignment, [(offset, size) per field]) of an isbits struct."""
    if name in cache:
        return cache[name]

    def size_align(t):
        if t in SCALARS:
            return SCALARS[t]
        m = re.fullmatch(r"NTuple\{(.+),\s*(\w+)\}", t)
        if m:
            count = eval(m.group(1), {}, dict(consts))  # "RDF_MAX_BINS + 1" and the like
            s, a = size_align(m.group(2))
            return s * count, a
        s, a, _ = julia_layout(structs, consts, t, cache)
        return s, a

    off, align, out = 0, 1, []
    for _, t in structs[name]:
        s, a = size_align(t)
        off = (off + a - 1) // a * a
        out.append((off, s))
        off += s
        align = max(align, a)
    size = (off + align - 1) // align * align
    cache[name] = (size, align, out)
    return cache[name]


def c_fields(cname):
    """Member names of a struct of the header, in order."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    m = re.search(r"typedef struct " + cname + r"\s*\{(.*?)\}\s*" + cname + ";", text, re.S)
    assert m, cname
    names = []
    for decl in m.group(1).split(";"):
        decl = decl.strip()
        if not decl:
            continue
        toks = decl.split(None, 1)
        for d in toks[1].split(","):
            names.append(re.sub(r"\[.*\]", "", d).strip().lstrip("*").strip())
    return names


def c_layout(cname, names):
    prog = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {",
            f'printf("%zu\\n", sizeof({cname}));']
    for f in names:
        prog.append(f'printf("%zu %zu\\n", offsetof({cname}, {f}), sizeof((({cname}*)0)->{f}));')
    prog.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        open(src, "w").write("\n".join(prog))
        exe = os.path.join(d, "t")
        subprocess.run(["/usr/bin/gcc", src, "-o", exe], check=True)
        vals = [int(v) for v in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    return vals[0], list(zip(vals[1::2], vals[2::2]))


def snake(name):
    return re.sub(r"(?<!^)([A-Z])", r"_\1", name).lower()


def test_every_abi_struct_has_the_c_layout():
    structs, consts = julia_structs()
    assert {"LcsConfig", "LcsSpecies", "LcsLog", "LcsCoupleLog"} <= set(structs)
    header = open(HEADER).read()
    checked = []
    cache = {}
    for jname in structs:
        cname = snake(jname)
        assert f"typedef struct {cname}" in header, f"{jname}: no {cname} in the header"
        jsize, _, jfields = julia_layout(structs, consts, jname, cache)
        csize, cfields = c_layout(cname, c_fields(cname))
        assert len(jfields) == len(cfields), (jname, len(jfields), len(cfields))
        assert jfields == cfields, (jname, [(a, b) for a, b in zip(jfields, cfields) if a != b])
        assert jsize == csize, (jname, jsize, csize)
        checked.append(jname)
    assert len(checked) >= 7


def test_constants_match_the_header():
    _, consts = julia_structs()
    header = open(HEADER).read()
    for jname, cname in (("MAX_SPECIES", "LCS_MAX_SPECIES"), ("RDF_MAX_BINS", "LCS_RDF_MAX_BINS"),
                         ("SPECTRUM_MAX_SHELLS", "LCS_SPECTRUM_MAX_SHELLS")):
        m = re.search(r"#define " + cname + r"\s+(\d+)", header)
        assert m and int(m.group(1)) == consts[jname], jname


@pytest.mark.parametrize("fn", ["lcs_create", "lcs_timestep", "lcs_evolve", "lcs_step", "lcs_upload_flow",
                                "lcs_download_flow", "lcs_upload_particles", "lcs_download_particles",
                                "lcs_last_error", "lcs_destroy"])
def test_shim_binds_declared_entry_points(fn):
    """Every ccall of the shim names an entry point the header declares."""
    src = "".join(open(os.path.join(SHIM, "src", f)).read() for f in ("abi.jl", "LCSB200.jl"))
    called = set(re.findall(r"ccall\(\(:(\w+), LIB\)", src))
    declared = set(re.findall(r"^LCS_API [^(]*?\b(lcs_\w+)\(", open(HEADER).read(), re.M))
    assert called <= declared, called - declared
    assert fn in called
