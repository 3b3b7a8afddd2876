"""Extract the reference's deterministic known answers into known_answers.json.

The reference's golden arrays (test/references/*.jld2) are git-LFS pointer
stubs and its random inputs come from Julia's Xoshiro stream, so the only
reference-owned values that pin this path are the deterministic assertions in
its test files.  This script reads those files as text (it runs nothing from
the reference) and writes the values, with their file:line, to
tests/golden/known_answers.json.  The committed JSON is what the tests read;
rerun this script only to refresh it, with the path of an LCS.jl checkout:

    python tests/golden/make_known_answers.py <path of the LCS.jl checkout>
"""

import json
import os
import re
import sys


def find_line(lines, pattern):
    for no, ln in enumerate(lines, 1):
        if re.search(pattern, ln):
            return no, ln
    raise SystemExit(f"pattern not found: {pattern}")


def parse_julia_array3(text):
    """Parse a Julia 3-D literal `[a b; c d;;; e f; g h]` into nested lists [i][j][k]."""
    body = text.strip()[1:-1]
    slabs = [s for s in body.split(";;;")]
    mats = []
    for s in slabs:
        rows = [r.split() for r in s.strip().split(";") if r.strip()]
        mats.append([[int(v) for v in r] for r in rows])
    ni, nj, nk = len(mats[0]), len(mats[0][0]), len(mats)
    return [[[mats[k][i][j] for k in range(nk)] for j in range(nj)] for i in range(ni)]


def main(ref):
    out = {"_generated_by": "tests/golden/make_known_answers.py (reads the reference's test files as text)"}

    ft = os.path.join(ref, "lib/fouriertools/test/runtests.jl")
    lines = open(ft).read().splitlines()
    kc = {}
    for k in (1, 2):
        no, ln = find_line(lines, rf"FT\.kcount\({k}\) == \d+")
        kc[str(k)] = int(re.search(rf"FT\.kcount\({k}\) == (\d+)", ln).group(1))
        kc[f"source_{k}"] = f"lib/fouriertools/test/runtests.jl:{no}"
    out["kcount"] = kc
    no, _ = find_line(lines, r"Set\(FT\.kset\(1\)\) == Set")
    block = []
    for ln in lines[no:]:
        if "])" in ln:
            break
        block.append(ln)
    triples = re.findall(r"\((-?\d+), (-?\d+), (-?\d+)\)", "\n".join(block))
    out["kset1"] = {"set": [[int(a), int(b), int(c)] for a, b, c in triples],
                    "source": f"lib/fouriertools/test/runtests.jl:{no}"}
    canon = []
    for no, ln in enumerate(lines, 1):
        m = re.search(r"FT\.canon\(\((-?\d+), (-?\d+), (-?\d+)\)\) == \((-?\d+), (-?\d+), (-?\d+)\)", ln)
        if m:
            v = [int(x) for x in m.groups()]
            canon.append({"in": v[:3], "out": v[3:], "source": f"lib/fouriertools/test/runtests.jl:{no}"})
    out["canon"] = canon
    no, ln = find_line(lines, r"U_hat = fill\(one\(ComplexF64\) \* 16\^3, 9, 16, 16\)")
    out["enespe_constant"] = {"value": 16 ** 3, "shape": [9, 16, 16],
                              "expect": "enespe(k0) == kcount(k0) * 3 / 2 for k0 = 1, 2",
                              "source": f"lib/fouriertools/test/runtests.jl:{no}-{no + 2}"}
    no, ln = find_line(lines, r'@testset "sidft3"')
    out["sirdft_property"] = {"n": 8, "kmin": 2, "kmax": 3,
                              "expect": "sirdft over kmin..kmax equals irfft of the shell-masked spectrum",
                              "source": f"lib/fouriertools/test/runtests.jl:{no}"}

    pt = os.path.join(ref, "lib/parallel/test/runtests.jl")
    text = open(pt).read()
    lines = text.splitlines()
    for name in ("ref0x00", "ref0x01"):
        no, _ = find_line(lines, rf"{name} = \[")
        lit = []
        for ln in lines[no - 1:]:
            lit.append(ln.split("=", 1)[1] if name in ln else ln)
            if ln.strip().endswith("]"):
                break
        out[name] = {"axes": [2, 4], "array": parse_julia_array3(" ".join(lit)),
                     "source": f"lib/parallel/test/runtests.jl:{no}"}

    tp = os.path.join(ref, "test/test_particles.jl")
    lines = open(tp).read().splitlines()
    no1, _ = find_line(lines, r"P\.coeff\(P\.LinearDrag\(\), 1\.0\) == 1\.0")
    no2, ln2 = find_line(lines, r"P\.coeff\(P\.NonlinearDrag\(\), 1\.0\) == ")
    out["drag"] = {"linear_Rep1": 1.0, "nonlinear_Rep1": float(re.search(r"== ([0-9.]+)", ln2).group(1)),
                   "source": f"test/test_particles.jl:{no1}-{no2}"}

    tf = os.path.join(ref, "test/test_flows.jl")
    lines = open(tf).read().splitlines()
    no, _ = find_line(lines, r'@testset "boxmean"')
    out["boxmean"] = {"dims": [8, 8, 8], "coarse_dims": [2, 2, 2], "halo_size": 3,
                      "expect": "boxmean of repeat(reshape(1:8,2,2,2); inner=filter_dims) == reshape(1:8,2,2,2)",
                      "source": f"test/test_flows.jl:{no}-{no + 14}"}
    no, _ = find_line(lines, r"F\.EnergyPreserveRCF\(1\.0, 1, 2, 4\)")
    no2, _ = find_line(lines, r"F\.phase_shift\(forcing, grid\) == 2")
    out["rcf_helpers"] = {"grid": [16, 16, 16], "coarse_size": 4, "coarse_dims_g": [4, 4, 4], "filter_size": 4,
                          "phase_shift": 2.0, "source": f"test/test_flows.jl:{no}-{no2}"}
    tm = os.path.join(ref, "lib/topologies/test/test_mpi.jl")
    lines = open(tm).read().splitlines()
    no, _ = find_line(lines, r"indices_with_halo_periodic = ")
    out["halo_periodic"] = {"expect": "after synchalo!(FullHalo(h)) A == A_g[mod1.(i, n)...] on the haloed box",
                            "source": f"lib/topologies/test/test_mpi.jl:{no}"}
    tu = os.path.join(ref, "test/test_utils.jl")
    lines = open(tu).read().splitlines()
    no, _ = find_line(lines, r'@testset "searchedsort2"')
    samples = []
    for k, ln in enumerate(lines[no:no + 20], no + 1):
        m = re.match(r"\s*\(\[([0-9, ]*)\], (-?\d+)\),", ln)
        if m:
            v = [int(x) for x in m.group(1).split(",") if x.strip()]
            samples.append({"v": v, "x": int(m.group(2)), "source": f"test/test_utils.jl:{k}"})
    out["searchsorted"] = {"samples": samples,
                           "expect": "Utils.searchsortedfirst/last (src/utils/fast.jl:8-40) equal Base's"}
    sub = []
    for k, ln in enumerate(lines, 1):
        m = re.search(r"Utils\.sub2ind\(ranges, \((\d+), (\d+)\)\) == (\d+)", ln)
        if m:
            sub.append({"ranges": [[1, 3], [1, 4]], "sub": [int(m.group(1)), int(m.group(2))], "ind": int(m.group(3)),
                        "source": f"test/test_utils.jl:{k}"})
    no, _ = find_line(lines, r"hasher = Utils\.Hasher\(\(0:5, 0:5, 0:5\)\)")
    out["hasher"] = {"sub2ind": sub, "roundtrip_axes": [[0, 5], [0, 5], [0, 5]],
                     "expect": "encode(x) == LinearIndices((6,6,6))[x .+ 1] and decode(encode(x)) == x",
                     "source": f"test/test_utils.jl:{no}"}
    # the package UUIDs and path sources a backend package beside LCSCUDA/ binds to
    import tomllib

    root = tomllib.load(open(os.path.join(ref, "Project.toml"), "rb"))
    cuda = tomllib.load(open(os.path.join(ref, "LCSCUDA", "Project.toml"), "rb"))
    out["julia_packages"] = {
        "uuids": dict(root["deps"], LCS=root["uuid"]),
        "root_sources": {k: v["path"] for k, v in root["sources"].items()},
        "lcscuda_sources": {k: v["path"] for k, v in cuda["sources"].items()},
        "source": "Project.toml [deps], [sources]; LCSCUDA/Project.toml [sources]",
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_known_answers.py <path of the LCS.jl checkout>")
    main(sys.argv[1])
