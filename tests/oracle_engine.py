"""The CPU oracle behind the same Python interface as the CUDA engine.

Test infrastructure: the oracle (oracle/liblcs_oracle.so) implements the same
C ABI, so a test drives both libraries with identical calls and compares.
"""

import ctypes as C
import os

from lcs_b200 import _abi
from lcs_b200.engine import Engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# LCS_ORACLE_LIBRARY selects another build of the oracle (the sanitizer builds
# of `make -C oracle asan|tsan`)
ORACLE_PATH = os.environ.get("LCS_ORACLE_LIBRARY") or os.path.join(ROOT, "oracle", "liblcs_oracle.so")

_lib = None


def load_oracle():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_PATH):
            import subprocess

            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
        lib = _abi.bind(C.CDLL(ORACLE_PATH))
        lib.lcs_oracle_kcount.restype = C.c_int
        lib.lcs_oracle_kcount.argtypes = [C.c_int]
        lib.lcs_oracle_kset.restype = C.c_int
        lib.lcs_oracle_kset.argtypes = [C.c_int, C.POINTER(C.c_int32), C.c_int]
        lib.lcs_oracle_enespe0.restype = C.c_double
        lib.lcs_oracle_enespe0.argtypes = [C.c_int, C.c_double]
        lib.lcs_oracle_boxmean.restype = None
        lib.lcs_oracle_boxmean.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
        lib.lcs_oracle_sirdft.restype = C.c_double
        lib.lcs_oracle_sirdft.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_int] + [C.c_double] * 6
        lib.lcs_oracle_sincospi.restype = None
        lib.lcs_oracle_sincospi.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.lcs_oracle_color_mask.restype = C.c_int
        lib.lcs_oracle_color_mask.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int,
                                              C.POINTER(C.c_int32)]  # coloring, block, lo, hi, color, out
        lib.lcs_oracle_enespe.restype = C.c_double
        lib.lcs_oracle_enespe.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_int, C.c_double]
        lib.lcs_oracle_phase_shift.restype = C.c_double
        lib.lcs_oracle_phase_shift.argtypes = [C.c_int, C.c_int]
        lib.lcs_oracle_threads.restype = C.c_int
        _lib = lib
    return _lib


class OracleEngine(Engine):
    """Engine over the CPU oracle (same ABI)."""

    @staticmethod
    def _load():
        return load_oracle()
