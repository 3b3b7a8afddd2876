"""The C-ABI boundary: both libraries load and export every declared entry
point, the ctypes structs match the C layout, and the CUDA library refuses
to run (loudly) where there is no GPU."""

import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from conftest import ROOT, gpu_available
from helpers import make_config
from lcs_b200 import _abi

HEADER = os.path.join(ROOT, "include", "lcs_b200.h")


def declared_functions():
    names = re.findall(r"^LCS_API [^(]*?\b(lcs_\w+)\(", open(HEADER).read(), re.M)
    assert len(names) >= 30
    return names


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def test_cuda_library_exports_every_declared_symbol(cuda_lib_path):
    syms = exported(cuda_lib_path)
    missing = [n for n in declared_functions() if n not in syms]
    assert not missing, missing
    assert set(_abi.PROTOTYPES) == set(declared_functions())


def test_oracle_exports_every_declared_symbol(oracle_lib_path):
    syms = exported(oracle_lib_path)
    missing = [n for n in declared_functions() if n not in syms]
    assert not missing, missing


def test_libraries_load_and_bind(cuda_lib_path, oracle_lib_path):
    for p in (cuda_lib_path, oracle_lib_path):
        lib = _abi.bind(C.CDLL(p))
        assert lib.lcs_last_error(None) is not None


def test_struct_layout_matches_c():
    fields = [f for f, _ in _abi.Config._fields_]
    prog = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {",
            'printf("%zu %zu %zu %zu\\n", sizeof(lcs_config), sizeof(lcs_species), sizeof(lcs_log), sizeof(lcs_couple_log));']
    for f in fields:
        prog.append(f'printf("%zu\\n", offsetof(lcs_config, {f}));')
    for f, _ in _abi.Log._fields_:
        prog.append(f'printf("%zu\\n", offsetof(lcs_log, {f}));')
    prog.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        open(src, "w").write("\n".join(prog))
        exe = os.path.join(d, "t")
        subprocess.run(["/usr/bin/gcc", src, "-o", exe], check=True)
        vals = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    sizes = [int(v) for v in vals[:4]]
    assert sizes == [C.sizeof(_abi.Config), C.sizeof(_abi.Species), C.sizeof(_abi.Log), C.sizeof(_abi.CoupleLog)]
    offs = [int(v) for v in vals[4:]]
    cfg_offs = [getattr(_abi.Config, f).offset for f in fields]
    log_offs = [getattr(_abi.Log, f).offset for f, _ in _abi.Log._fields_]
    assert offs == cfg_offs + log_offs


@pytest.mark.parametrize("cname,pyname", [("lcs_server_config", "ServerConfig"), ("lcs_species_state", "SpeciesState"),
                                          ("lcs_request", "Request"), ("lcs_species_out", "SpeciesOut"),
                                          ("lcs_server_stats", "ServerStats"), ("lcs_flow_stats", "FlowStat")])
def test_serving_struct_layouts_match_c(cname, pyname):
    st = getattr(_abi, pyname)
    fields = [f for f, _ in st._fields_]
    prog = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {",
            f'printf("%zu\\n", sizeof({cname}));']
    prog += [f'printf("%zu\\n", offsetof({cname}, {f}));' for f in fields]
    prog.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        open(src, "w").write("\n".join(prog))
        exe = os.path.join(d, "t")
        subprocess.run(["/usr/bin/gcc", src, "-o", exe], check=True)
        vals = [int(v) for v in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    assert vals[0] == C.sizeof(st)
    assert vals[1:] == [getattr(st, f).offset for f in fields]


def test_footprint_and_validation_without_gpu(cuda_lib_path):
    lib = _abi.bind(C.CDLL(cuda_lib_path))
    b = C.c_int64()
    small = make_config(16)
    big = make_config(32)
    assert lib.lcs_footprint(C.byref(small), C.byref(b)) == 0
    fs = b.value
    assert lib.lcs_footprint(C.byref(big), C.byref(b)) == 0
    # 10 haloed FP64 fields grow with the grid; the fixed scratch does not
    assert b.value - fs >= 10 * 8 * (38 ** 3 - 22 ** 3)
    bad = make_config(15)
    assert lib.lcs_footprint(C.byref(bad), C.byref(b)) == _abi.EINVAL
    assert b"even" in lib.lcs_last_error(None)
    nocol = make_config(16, coloring=_abi.COLORING_NO)
    assert lib.lcs_footprint(C.byref(nocol), C.byref(b)) == _abi.EINVAL
    rcf = make_config(16, forcing=_abi.FORCING_RC_ENERGY, kmin=1, kmax=3, coarse=4)
    assert lib.lcs_footprint(C.byref(rcf), C.byref(b)) == _abi.EINVAL
    empty = make_config(16, species=[{"n": 0}])
    assert lib.lcs_footprint(C.byref(empty), C.byref(b)) == _abi.EINVAL


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU refusal")
def test_cuda_library_fails_loudly_without_gpu(cuda_lib_path):
    lib = _abi.bind(C.CDLL(cuda_lib_path))
    h = C.c_void_p()
    rc = lib.lcs_create(C.byref(make_config(16)), C.byref(h))
    assert rc == _abi.ECUDA
    assert b"no CUDA device" in lib.lcs_last_error(None)
    from lcs_b200 import Engine, LCSError

    with pytest.raises(LCSError):
        Engine(make_config(16))
