"""ctypes mirror of include/lcs_b200.h and the loader of liblcs_b200.so.

The structures below are byte-for-byte the C structs of the header; the test
``tests/test_abi.py`` checks their sizes and field offsets against a C
compilation of the header.
"""

from __future__ import annotations

import ctypes as C
import os

ABI_VERSION = 1
MAX_SPECIES = 16

OK = 0
EINVAL = -1
ENOMEM = -2
ECUDA = -3
ETIMEDOUT = -4
ENONFINITE = -5
ESTATE = -6

ERROR_NAMES = {
    EINVAL: "EINVAL",
    ENOMEM: "ENOMEM",
    ECUDA: "ECUDA",
    ETIMEDOUT: "ETIMEDOUT",
    ENONFINITE: "ENONFINITE",
    ESTATE: "ESTATE",
}

MODE_FLOW, MODE_FLOW_PARTICLE = 0, 1
COLORING_NO, COLORING_RED_BLACK, COLORING_RED_BLACK_FAST, COLORING_RED_BLACK_BLOCK = 0, 1, 2, 3
FORCING_NO, FORCING_LINEAR_POWER, FORCING_RC_ENERGY = 0, 1, 2
DRAG_LINEAR, DRAG_NONLINEAR = 0, 1
PRECISION_FP64, PRECISION_FP32_MIXED = 0, 1

FIELD_U, FIELD_V, FIELD_W, FIELD_U2, FIELD_V2, FIELD_W2, FIELD_P, FIELD_DUDT, FIELD_DVDT, FIELD_DWDT = range(10)
FIELD_NAMES = ["U", "V", "W", "U2", "V2", "W2", "P", "dUdt", "dVdt", "dWdt"]

(PROP_X, PROP_Y, PROP_Z, PROP_X2, PROP_Y2, PROP_Z2, PROP_U, PROP_V, PROP_W, PROP_U2, PROP_V2, PROP_W2,
 PROP_DUDT, PROP_DVDT, PROP_DWDT, PROP_DIAM) = range(16)
NPROP = 16
PROP_NAMES = ["x", "y", "z", "x2", "y2", "z2", "u", "v", "w", "u2", "v2", "w2", "dudt", "dvdt", "dwdt", "diam"]


class Species(C.Structure):
    _fields_ = [
        ("nvalid", C.c_int64),
        ("gravity", C.c_double),
        ("density_ratio", C.c_double),
        ("drag", C.c_int32),
        ("_pad", C.c_int32),
    ]


class Config(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("mode", C.c_int32),
        ("dims", C.c_int32 * 3),
        ("halo_size", C.c_int32),
        ("cfl", C.c_double),
        ("dtmax", C.c_double),
        ("U0", C.c_double),
        ("L0", C.c_double),
        ("NU", C.c_double),
        ("time_blocking", C.c_int32),
        ("overlap", C.c_int32),
        ("coloring", C.c_int32),
        ("coloring_block", C.c_int32),
        ("omega", C.c_double),
        ("epsp", C.c_double),
        ("itrmin", C.c_int32),
        ("itrmax", C.c_int32),
        ("forcing", C.c_int32),
        ("kmin", C.c_int32),
        ("kmax", C.c_int32),
        ("coarse_size", C.c_int32),
        ("power", C.c_double),
        ("energy", C.c_double),
        ("n_species", C.c_int32),
        ("precision", C.c_int32),
        ("species", Species * MAX_SPECIES),
        ("device", C.c_int32),
        ("use_graphs", C.c_int32),
    ]


class CoupleLog(C.Structure):
    _fields_ = [("itr", C.c_int32), ("sweeps", C.c_int32), ("div", C.c_double)]


class Log(C.Structure):
    _fields_ = [
        ("couple1", CoupleLog),
        ("couple2", CoupleLog),
        ("forcing_p", C.c_double),
        ("forcing_e10", C.c_double),
        ("dt", C.c_double),
        ("t", C.c_double),
        ("step", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {
            "couple1": {"itr": self.couple1.itr, "sweeps": self.couple1.sweeps, "div": self.couple1.div},
            "couple2": {"itr": self.couple2.itr, "sweeps": self.couple2.sweeps, "div": self.couple2.div},
            "forcing": {"p": self.forcing_p, "e10": self.forcing_e10},
            "dt": self.dt,
            "t": self.t,
            "step": self.step,
        }


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)


class FlowStat(C.Structure):
    _fields_ = [(f, C.c_double) for f in (
        "u_mean", "u_max", "u_min", "v_mean", "v_max", "v_min", "w_mean", "w_max", "w_min", "k", "epsilon",
        "tau_eta", "l_mu", "l_eta", "Re_lambda", "urms", "k_eta", "skewness", "flatness", "L", "C_epsilon")]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


# ---- particle statistics (include/lcs_b200.h: lcs_particles_stat) -----------
RDF_MAX_BINS = 1024
SPECTRUM_MAX_SHELLS = 19
SPECTRUM_MAX_SAMPLES = 1024


class ParticleStatConfig(C.Structure):
    """Cell, RDF and Spectrum of src/particles/config.jl:51-94."""
    _fields_ = [("grid_ratio", C.c_int32), ("bin_size", C.c_int32), ("search_cell_size", C.c_int32),
                ("max_wavenumber", C.c_int32), ("nsamples", C.c_int32), ("_pad", C.c_int32),
                ("contact_tolerance", C.c_double), ("min_radius", C.c_double)]


class Summary(C.Structure):
    _fields_ = [("mean", C.c_double), ("max", C.c_double), ("min", C.c_double)]


class ParticleStats(C.Structure):
    _fields_ = [(f, Summary) for f in ("x", "y", "z", "u", "v", "w", "diam")] + [
        ("taup", C.c_double), ("St", C.c_double), ("gr_contact", C.c_double), ("npairs_contact", C.c_int64),
        ("nbins", C.c_int32), ("nshells", C.c_int32), ("edges", C.c_double * (RDF_MAX_BINS + 1)),
        ("gr", C.c_double * RDF_MAX_BINS), ("npairs", C.c_int64 * RDF_MAX_BINS),
        ("wavenumbers", C.c_double * SPECTRUM_MAX_SHELLS), ("Enp", C.c_double * SPECTRUM_MAX_SHELLS)]

    def as_dict(self) -> dict:
        """ParticleStat (src/particles/stat.jl:62-75) as nested dicts and numpy arrays."""
        import numpy as np

        nb, ns = self.nbins, self.nshells
        out = {f: {"mean": getattr(self, f).mean, "max": getattr(self, f).max, "min": getattr(self, f).min}
               for f in ("x", "y", "z", "u", "v", "w", "diam")}
        out["taup"], out["St"] = self.taup, self.St
        out["rdf"] = {"gr_contact": self.gr_contact, "npairs_contact": self.npairs_contact,
                      "edges": np.array(self.edges[: nb + 1]), "gr": np.array(self.gr[:nb]),
                      "npairs": np.array(self.npairs[:nb], dtype=np.int64)}
        out["spectrum"] = {"wavenumbers": np.array(self.wavenumbers[:ns]), "Enp": np.array(self.Enp[:ns])}
        return out


# ---- batching and serving forms (include/lcs_b200.h) -----------------------
MAX_ASYNC_STEPS = 4096
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_active", C.c_int32), ("steps_per_slice", C.c_int32), ("_pad", C.c_int32),
                ("hbm_budget_bytes", C.c_int64)]


class SpeciesState(C.Structure):
    _fields_ = [("ids", _I64), ("diam", _D), ("x", _D), ("y", _D), ("z", _D), ("u", _D), ("v", _D), ("w", _D)]


class Request(C.Structure):
    _fields_ = [("config", Config), ("U", _D), ("V", _D), ("W", _D), ("P", _D),
                ("species", SpeciesState * MAX_SPECIES), ("interp_velocity", C.c_int32), ("_pad", C.c_int32),
                ("nsteps", C.c_int64)]


class SpeciesOut(C.Structure):
    _fields_ = [("x", _D), ("y", _D), ("z", _D), ("u", _D), ("v", _D), ("w", _D)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64), ("queued", C.c_int64),
                ("active", C.c_int64), ("bytes_in_use", C.c_int64), ("peak_bytes_in_use", C.c_int64),
                ("p50_latency_s", C.c_double), ("p99_latency_s", C.c_double), ("mean_latency_s", C.c_double),
                ("busy_s", C.c_double)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}

# name -> (restype, argtypes) for every entry point of include/lcs_b200.h
PROTOTYPES = {
    "lcs_create": (C.c_int, [C.POINTER(Config), C.POINTER(_P)]),
    "lcs_destroy": (None, [_P]),
    "lcs_last_error": (C.c_char_p, [_P]),
    "lcs_footprint": (C.c_int, [C.POINTER(Config), _I64]),
    "lcs_upload_flow": (C.c_int, [_P, _D, _D, _D, _D]),
    "lcs_download_flow": (C.c_int, [_P, _D, _D, _D, _D]),
    "lcs_field_set": (C.c_int, [_P, C.c_int32, _D, C.c_int32]),
    "lcs_field_get": (C.c_int, [_P, C.c_int32, _D, C.c_int32]),
    "lcs_upload_particles": (C.c_int, [_P, C.c_int32, C.c_int64, _I64, _D, _D, _D, _D, _D, _D, _D]),
    "lcs_download_particles": (C.c_int, [_P, C.c_int32, _I64, _D, _D, _D, _D, _D, _D, _D]),
    "lcs_prop_set": (C.c_int, [_P, C.c_int32, C.c_int32, _D]),
    "lcs_prop_get": (C.c_int, [_P, C.c_int32, C.c_int32, _D]),
    "lcs_set_state": (C.c_int, [_P, C.c_int64, C.c_double]),
    "lcs_get_state": (C.c_int, [_P, _I64, _D]),
    "lcs_timestep": (C.c_int, [_P, _D]),
    "lcs_evolve": (C.c_int, [_P, C.c_double, C.POINTER(Log)]),
    "lcs_step": (C.c_int, [_P, C.c_int32, C.POINTER(Log)]),
    "lcs_step_timed": (C.c_int, [_P, C.c_int32, C.POINTER(Log), _D]),
    "lcs_transfer_stats": (C.c_int, [_P, _I64, _I64]),
    "lcs_synchalo": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32]),
    "lcs_flow_rhs": (C.c_int, [_P, C.c_int32]),
    "lcs_flow_update": (C.c_int, [_P, C.c_int32, C.c_double]),
    "lcs_flow_rhs_update": (C.c_int, [_P, C.c_int32, C.c_double]),
    "lcs_flow_couple": (C.c_int, [_P, C.c_int32, C.c_double, C.POINTER(CoupleLog)]),
    "lcs_flow_forcing": (C.c_int, [_P, C.c_double, _D, _D]),
    "lcs_flow_timestep": (C.c_int, [_P, _D]),
    "lcs_particles_timestep": (C.c_int, [_P, _D]),
    "lcs_particles_boundary": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "lcs_particles_motion": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "lcs_particles_update": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_double]),
    "lcs_init_particle_velocity": (C.c_int, [_P, C.c_int32]),
    "lcs_profile_enable": (C.c_int, [_P, C.c_int32]),
    "lcs_profile_reset": (C.c_int, [_P]),
    "lcs_profile_count": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "lcs_profile_entry": (C.c_int, [_P, C.c_int32, C.c_char_p, C.c_int32, _D, _I64]),
    "lcs_launch_count": (C.c_int, [_P, _I64]),
    "lcs_synchronize": (C.c_int, [_P]),
    "lcs_flow_timestep_noalloc": (C.c_int, [_P, _P, _P, C.POINTER(C.c_int32), C.c_int32, C.c_double, C.c_double,
                                            C.c_double, _P, _P]),
    "lcs_flow_stat": (C.c_int, [_P, C.POINTER(FlowStat)]),
    "lcs_particles_makeindex": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32]),
    "lcs_set_particle_sort": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "lcs_particles_cellindex": (C.c_int, [_P, C.c_int32, _I64, _I64, _I64]),
    "lcs_particles_stat": (C.c_int, [_P, C.c_int32, C.POINTER(ParticleStatConfig), C.c_double,
                                     C.POINTER(ParticleStats)]),
    "lcs_particles_density": (C.c_int, [_P, C.c_int32, C.c_int32, _D]),
    "lcs_upload_flow_coarse": (C.c_int, [_P, _D, _D, _D, _D]),
    "lcs_group_create": (C.c_int, [C.POINTER(_P), C.c_int32, C.POINTER(_P)]),
    "lcs_group_step_begin": (C.c_int, [_P, C.c_int32]),
    "lcs_group_destroy": (None, [_P]),
    "lcs_get_config": (C.c_int, [_P, C.POINTER(Config)]),
    "lcs_measure_fp64_peak": (C.c_int, [C.c_int32, _D]),
    "lcs_flow_divergence": (C.c_int, [_P, _D, _D]),
    "lcs_debug_unreachable_waits": (C.c_int, [_P, C.c_int32]),
    "lcs_restart_save": (C.c_int, [_P, C.c_char_p]),
    "lcs_restart_load": (C.c_int, [_P, C.c_char_p]),
    "lcs_restart_load_coarse": (C.c_int, [_P, C.c_char_p]),
    "lcs_stat_state_save": (C.c_int, [C.c_char_p, C.c_int64, C.c_double, C.c_double]),
    "lcs_stat_save": (C.c_int, [C.c_char_p, C.c_int64, C.c_double, C.c_double, C.c_void_p, C.c_int32, C.c_void_p,
                                C.c_void_p, C.c_void_p]),
    "lcs_stat_state_load": (C.c_int, [C.c_char_p, C.c_int64, _D, _D]),
    "lcs_h5_dataset": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_int32), _I64, C.c_char_p, C.c_void_p,
                                 C.c_int64]),
    "lcs_h5_list": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int64]),
    "lcs_io_last_error": (C.c_char_p, []),
    "lcs_step_begin": (C.c_int, [_P, C.c_int32]),
    "lcs_step_poll": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "lcs_step_finish": (C.c_int, [_P, C.POINTER(Log)]),
    "lcs_device_bytes": (C.c_int, [_P, _I64]),
    "lcs_set_tuning": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_double]),
    "lcs_batch_create": (C.c_int, [C.POINTER(Config), C.c_int32, C.POINTER(_P)]),
    "lcs_batch_size": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "lcs_batch_member": (C.c_int, [_P, C.c_int32, C.POINTER(_P)]),
    "lcs_batch_step": (C.c_int, [_P, C.c_int32, C.POINTER(Log)]),
    "lcs_batch_destroy": (None, [_P]),
    "lcs_batch_tuning": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _D, _D]),
    "lcs_server_create": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(_P)]),
    "lcs_server_submit": (C.c_int, [_P, C.POINTER(Request), _I64]),
    "lcs_server_poll": (C.c_int, [_P, C.c_int64, C.POINTER(C.c_int32), _I64]),
    "lcs_server_result": (C.c_int, [_P, C.c_int64, _D, _D, _D, _D, C.POINTER(SpeciesOut), C.POINTER(Log), _D]),
    "lcs_server_release": (C.c_int, [_P, C.c_int64]),
    "lcs_server_stats_get": (C.c_int, [_P, C.POINTER(ServerStats)]),
    "lcs_server_drain": (C.c_int, [_P, C.c_double]),
    "lcs_server_destroy": (None, [_P]),
    "lcs_serve_last_error": (C.c_char_p, []),
}

NOALLOC_MAX_PLANES = 4096

PACKAGE_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBRARY_PATH = os.path.join(PACKAGE_DIR, "liblcs_b200.so")


def bind(lib: C.CDLL) -> C.CDLL:
    """Attach the prototypes of every ABI entry point to a loaded library."""
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_cuda_lib = None


def load_library() -> C.CDLL:
    """Load the in-tree CUDA library; raise if it was not built.

    There is no CPU fallback: the time step runs on the B200 kernels or not at
    all.
    """
    global _cuda_lib
    if _cuda_lib is None:
        if not os.path.exists(LIBRARY_PATH):
            raise RuntimeError(
                f"{LIBRARY_PATH} is missing: build it with `make -C lcs.jl_b200` "
                "(or __graft_entry__.build()); the B200 backend has no CPU fallback"
            )
        _cuda_lib = bind(C.CDLL(LIBRARY_PATH))
    return _cuda_lib
