"""B200 backend of LCS.jl's time step: host side of the C ABI.

`simulate(config)` mirrors `LCS.simulate`; `Engine` exposes every entry point
of include/lcs_b200.h (the per-step `timestep`/`evolve`/`step` and the stage
functions) on numpy arrays.  All time-step arithmetic runs in the CUDA
library liblcs_b200.so; this package only prepares inputs and reads results.
"""

from . import _abi, config, inits
from .config import RunConfig, from_dict, readconfig, workload
from .engine import Engine, LCSError, footprint
from .serve import Batch, Server
from .simulate import init_engine, simulate

__all__ = ["Batch", "Server", "Engine", "LCSError", "RunConfig", "_abi", "config", "footprint", "from_dict", "init_engine", "inits",
           "readconfig", "simulate", "workload"]
