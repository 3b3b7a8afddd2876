"""Restart files in the reference's HDF5 layout (src/LCSIO/save.jl:40-167,
load.jl:23-118) through the library's own reader and writer, over the CPU
oracle (the I/O is host code over the public ABI, linked into both libraries).

The reader is checked against a file written by the HDF5 library itself: the
MATLAB 7.3 test file that SciPy ships (a 512-byte user block, then HDF5 with
libhdf5's own layout), whose `testdouble` is pi * [0..8] / 4.  The writer uses
the same encodings, compared byte for byte where the two overlap.
"""

import ctypes as C
import math
import os
import struct

import numpy as np
import pytest

from helpers import make_config
from lcs_b200 import _abi, restart
from oracle_engine import OracleEngine, load_oracle


def libhdf5_file():
    import scipy

    p = os.path.join(os.path.dirname(scipy.__file__), "io", "matlab", "tests", "data", "testhdf5_7.4_GLNX86.mat")
    if not os.path.exists(p):
        pytest.skip("the SciPy HDF5 test file is not installed")
    return p


def test_reads_a_file_written_by_libhdf5():
    lib = load_oracle()
    p = libhdf5_file()
    assert restart.listing(lib, p) == ["testdouble"]
    a = restart.dataset(lib, p, "testdouble")
    assert a.shape == (9, 1)
    assert np.allclose(a.ravel(), math.pi * np.arange(9) / 4, rtol=0, atol=1e-15)


def engine_with_state(n=16, species=({"n": 300, "density_ratio": 843.0}, {"n": 120, "density_ratio": 100.0}),
                      seed=0, steps=2):
    cfg = make_config(n, species=list(species), Re=80.0, itrmax=6)
    e = OracleEngine(cfg)
    rng = np.random.default_rng(seed)
    nx = cfg.dims[0]
    e.upload_flow(*[rng.standard_normal((nx, nx, nx)) * 0.3 for _ in range(3)], np.zeros((nx, nx, nx)))
    for s in range(int(cfg.n_species)):
        m = int(cfg.species[s].nvalid)
        pos = [rng.random(m) * 2 * math.pi for _ in range(3)]
        e.upload_particles(s, np.full(m, 0.01), *pos, *[np.zeros(m)] * 3, ids=np.arange(1, m + 1) + 1000 * s)
        e.init_particle_velocity(s)
    e.step(steps)
    return cfg, e


def test_restart_round_trip_and_layout(tmp_path):
    lib = load_oracle()
    cfg, a = engine_with_state()
    path = str(tmp_path / "restart.h5.2")
    restart.save(a, path)
    assert restart.listing(lib, path) == ["flow", "particles"]
    assert restart.listing(lib, path, "flow") == ["P", "U", "V", "W"]
    assert restart.listing(lib, path, "particles") == ["1", "2"]
    assert restart.listing(lib, path, "particles/1") == ["counts", "diam", "id", "u", "v", "w", "x", "y", "z"]
    U = restart.dataset(lib, path, "flow/U")
    assert U.shape == (16, 16, 16) and U.dtype == np.float64
    assert np.array_equal(U, a.download_flow()[0])
    assert restart.dataset(lib, path, "particles/2/counts").tolist() == [120]
    assert np.array_equal(restart.dataset(lib, path, "particles/2/id"), a.download_particles(1)["ids"])
    b = OracleEngine(cfg)
    restart.load(b, path)
    for x, y in zip(a.download_flow(), b.download_flow()):
        assert np.array_equal(x, y)
    for s in range(2):
        pa, pb = a.download_particles(s), b.download_particles(s)
        for k in ("ids", "diam", "x", "y", "z", "u", "v", "w"):
            assert np.array_equal(pa[k], pb[k]), (s, k)
    a.close()
    b.close()


def test_writer_encodings_match_libhdf5(tmp_path):
    """The F64 datatype message, the symbol node and the local heap's
    end-of-free-list value as libhdf5 writes them (read from the SciPy file)."""
    ref = open(libhdf5_file(), "rb").read()
    base = 512
    lib = load_oracle()
    cfg = make_config(8, mode=_abi.MODE_FLOW)
    eng = OracleEngine(cfg)
    eng.upload_flow(*[np.zeros((8, 8, 8))] * 4)
    path = str(tmp_path / "r.h5")
    restart.save(eng, path)
    ours = open(path, "rb").read()
    eng.close()
    f64 = bytes.fromhex("11203f000800000000004000340b0034ff030000")
    assert f64 in ref and f64 in ours
    # superblock: version 0, 8-byte offsets/lengths, K = 4 / 16
    assert ours[:8] == ref[base:base + 8] and ours[8:16] == bytes([0, 0, 0, 0, 0, 8, 8, 0])
    assert struct.unpack("<HH", ours[16:20]) == struct.unpack("<HH", ref[base + 16:base + 20]) == (4, 16)
    # every local heap ends its free list with offset 1, as libhdf5 does
    for src, off in ((ours, 0), (ref, base)):
        i = src.find(b"HEAP")
        assert i >= 0 and src[i + 4] == 0
        free = struct.unpack("<Q", src[i + 16:i + 24])[0]
        assert free == 1 or free < struct.unpack("<Q", src[i + 8:i + 16])[0]
    assert ours.count(b"SNOD") >= 2 and ours[ours.find(b"SNOD") + 4] == 1
    assert restart.listing(lib, path, "/") == ["flow"]


def test_restart_load_coarse_upsamples(tmp_path):
    lib = load_oracle()
    coarse_cfg = make_config(16, mode=_abi.MODE_FLOW)
    c = OracleEngine(coarse_cfg)
    rng = np.random.default_rng(3)
    fields = [rng.standard_normal((16, 16, 16)) for _ in range(4)]
    c.upload_flow(*fields)
    path = str(tmp_path / "coarse.h5")
    restart.save(c, path)
    fine_cfg = make_config(32, mode=_abi.MODE_FLOW)
    a, b = OracleEngine(fine_cfg), OracleEngine(fine_cfg)
    restart.load_coarse(a, path)
    b.upload_flow_coarse(*fields)
    for x, y in zip(a.download_flow(), b.download_flow()):
        assert np.array_equal(x, y)
    for e in (a, b, c):
        e.close()


def test_stat_state_and_errors(tmp_path):
    lib = load_oracle()
    path = str(tmp_path / "stat.h5")
    restart.save_state(lib, path, 1200, 3.25, 0.0025)
    assert restart.load_state(lib, path, 1200) == (3.25, 0.0025)
    assert restart.dataset(lib, path, "1200/state/step").tolist() == 1200
    with pytest.raises(Exception):
        restart.load_state(lib, path, 7)
    cfg, a = engine_with_state(steps=0)
    rpath = str(tmp_path / "r.h5")
    restart.save(a, rpath)
    other = OracleEngine(make_config(24, species=[{"n": 300, "density_ratio": 843.0}]))
    with pytest.raises(Exception) as exc:
        restart.load(other, rpath)
    assert getattr(exc.value, "code", None) == _abi.EINVAL
    fewer = OracleEngine(make_config(16, species=[{"n": 299, "density_ratio": 843.0}]))
    with pytest.raises(Exception) as exc:
        restart.load(fewer, rpath)
    assert "counts" in str(exc.value)
    with pytest.raises(Exception):
        restart.load(a, str(tmp_path / "missing.h5"))
    open(str(tmp_path / "junk.h5"), "wb").write(b"not hdf5" * 100)
    with pytest.raises(Exception):
        restart.load(a, str(tmp_path / "junk.h5"))
    for e in (a, other, fewer):
        e.close()


def test_reader_survives_corrupted_files(tmp_path):
    """Truncated files and files with random bytes overwritten: every read
    either returns or fails with an error, and never reads outside the file or
    a message (a crash would end the test run)."""
    lib = load_oracle()
    cfg, a = engine_with_state(steps=0)
    good = str(tmp_path / "good.h5")
    restart.save(a, good)
    a.close()
    blob = open(good, "rb").read()
    rng = np.random.default_rng(5)
    bad = str(tmp_path / "bad.h5")
    cases = [blob[:k] for k in (0, 8, 96, 200, 800, 2000, len(blob) // 2, len(blob) - 1)]
    for _ in range(150):
        b = bytearray(blob)
        head = min(len(b), 4096)  # the superblock, headers, heaps and B-trees sit at the front
        for at in rng.integers(0, head, int(rng.integers(1, 6))):
            b[at] = int(rng.integers(0, 256))
        cases.append(bytes(b))
    outcomes = {"ok": 0, "error": 0}
    for c in cases:
        open(bad, "wb").write(c)
        for call in (lambda: restart.listing(lib, bad), lambda: restart.dataset(lib, bad, "flow/U"),
                     lambda: restart.dataset(lib, bad, "particles/1/x")):
            try:
                call()
                outcomes["ok"] += 1
            except Exception:
                outcomes["error"] += 1
    assert outcomes["error"] > 0 and outcomes["ok"] > 0


FLOW_NAMES = {"u", "v", "w", "k", "ϵ", "τη", "lμ", "lη", "Reλ", "urms", "kη", "skew",
              "flat", "L", "Cϵ"}
PARTICLE_NAMES = {"x", "y", "z", "u", "v", "w", "diam", "τp", "St", "rdf", "spectrum"}


def test_stat_file_holds_the_reference_tree(tmp_path):
    """lcs_stat_save: the `<step>` entry of LCSIO.savestat (state, stat, log)
    with the Julia field names, from the library's own Flows.stat and
    Particles.stat, and the other steps of the file kept."""
    lib = load_oracle()
    cfg, e = engine_with_state(steps=2)
    log = _abi.Log()
    e._check(lib.lcs_step(e.handle, 1, C.byref(log)))
    fs = _abi.FlowStat()
    e._check(lib.lcs_flow_stat(e.handle, C.byref(fs)))
    pcfg = _abi.ParticleStatConfig(grid_ratio=4, bin_size=8, search_cell_size=2, max_wavenumber=8, nsamples=16,
                                   contact_tolerance=0.01, min_radius=1e-3)
    pstats = []
    for s in range(2):
        ps = _abi.ParticleStats()
        e._check(lib.lcs_particles_stat(e.handle, s, C.byref(pcfg), fs.tau_eta, C.byref(ps)))
        pstats.append(ps)
    path = str(tmp_path / "stat.h5")
    restart.save_state(lib, path, 1, 0.01, 0.01)  # an earlier step, kept by the next save
    restart.save_stat(lib, path, 3, 0.03, 0.01, flow=fs, nvalid=[300, 120], particles=pstats, log=log)
    assert restart.listing(lib, path) == ["1", "3"]
    assert restart.listing(lib, path, "3") == ["log", "stat", "state"]
    assert set(restart.listing(lib, path, "3/stat")) == {"flow", "particles", "state"}
    assert set(restart.listing(lib, path, "3/stat/flow")) == FLOW_NAMES
    assert restart.dataset(lib, path, "3/stat/flow/ϵ").tolist() == fs.epsilon
    assert restart.dataset(lib, path, "3/stat/flow/Reλ").tolist() == fs.Re_lambda
    assert restart.dataset(lib, path, "3/stat/flow/u/max").tolist() == fs.u_max
    assert restart.listing(lib, path, "3/stat/particles") == ["1", "2"]
    for s, ps in enumerate(pstats):
        g = f"3/stat/particles/{s + 1}"
        assert set(restart.listing(lib, path, g)) == PARTICLE_NAMES
        assert restart.dataset(lib, path, g + "/τp").tolist() == ps.taup
        assert restart.dataset(lib, path, g + "/diam/mean").tolist() == ps.diam.mean
        nb, nsh = ps.nbins, ps.nshells
        assert np.array_equal(restart.dataset(lib, path, g + "/rdf/edges"), np.array(ps.edges[:nb + 1]))
        assert np.array_equal(restart.dataset(lib, path, g + "/rdf/npairs"), np.array(ps.npairs[:nb]))
        assert restart.dataset(lib, path, g + "/rdf/npairs_contact").tolist() == ps.npairs_contact
        assert np.array_equal(restart.dataset(lib, path, g + "/spectrum/Enp"), np.array(ps.Enp[:nsh]))
        assert restart.dataset(lib, path, f"3/state/particles/{s + 1}/nvalid").tolist() == (300, 120)[s]
    assert restart.dataset(lib, path, "3/log/flow/couple2/itr").tolist() == log.couple2.itr
    assert restart.dataset(lib, path, "3/log/flow/couple1/div").tolist() == log.couple1.div
    assert "forcing" not in restart.listing(lib, path, "3/log/flow")  # no forcing: its log is empty
    assert restart.load_state(lib, path, 3) == (0.03, 0.01) and restart.load_state(lib, path, 1) == (0.01, 0.01)
    # saving step 1 again replaces its group and keeps step 3
    restart.save_state(lib, path, 1, 0.5, 0.25)
    assert restart.load_state(lib, path, 1) == (0.5, 0.25)
    assert set(restart.listing(lib, path, "3/stat/flow")) == FLOW_NAMES
    e.close()


def test_stat_file_with_many_steps(tmp_path):
    """A root group of 600 steps (over 256 entries: a two-level group B-tree),
    every step read back; a file the reader cannot read is left unchanged."""
    lib = load_oracle()
    path = str(tmp_path / "stat.h5")
    for q in range(600):
        restart.save_state(lib, path, 10 * q, 0.5 * q, 0.25)
    names = restart.listing(lib, path)
    assert sorted(int(x) for x in names) == [10 * q for q in range(600)]
    for q in range(0, 600, 7):
        assert restart.load_state(lib, path, 10 * q) == (0.5 * q, 0.25)
    junk = str(tmp_path / "junk.h5")
    open(junk, "wb").write(b"x" * 1000)
    with pytest.raises(Exception):
        restart.save_state(lib, junk, 1, 0.0, 0.0)
    assert open(junk, "rb").read() == b"x" * 1000


def test_stat_save_rejects_bad_counts(tmp_path):
    lib = load_oracle()
    path = str(tmp_path / "stat.h5")
    bad = _abi.ParticleStats()
    bad.nbins = _abi.RDF_MAX_BINS + 1
    with pytest.raises(Exception) as exc:
        restart.save_stat(lib, path, 1, 0.0, 0.0, particles=[bad], nvalid=[1])
    assert getattr(exc.value, "code", None) == _abi.EINVAL and not os.path.exists(path)
    bad.nbins, bad.nshells = 4, _abi.SPECTRUM_MAX_SHELLS + 1
    with pytest.raises(Exception):
        restart.save_stat(lib, path, 1, 0.0, 0.0, particles=[bad], nvalid=[1])
    assert lib.lcs_stat_save(path.encode(), 1, 0.0, 0.0, None, _abi.MAX_SPECIES + 1, None, None, None) == _abi.EINVAL
    assert lib.lcs_stat_save(None, 1, 0.0, 0.0, None, 0, None, None, None) == _abi.EINVAL
    # everything optional: the state entries alone
    restart.save_stat(lib, path, 5, 1.5, 0.5)
    assert restart.listing(lib, path, "5") == ["stat", "state"] and restart.load_state(lib, path, 5) == (1.5, 0.5)
