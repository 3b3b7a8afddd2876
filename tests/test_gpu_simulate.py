"""simulate() on the CUDA library: the stat and restart files it writes, and a
run resumed from its restart (LCS_RESUME) ending where the uninterrupted run
ends, bit for bit (step graphs on, as the config's backend default)."""

import os

import numpy as np
import pytest

from lcs_b200 import Engine, restart
from lcs_b200.simulate import simulate
from test_config import small_run

pytestmark = pytest.mark.gpu


def test_resume_on_the_device(tmp_path):
    d = small_run(steps=3, interval=3)
    d["simulate"].update({"interval_restart": 3, "num_restart_files": 2})
    out = str(tmp_path / "run")
    eng, _ = simulate(d, quiet=True, engine_cls=Engine, save=True, outdir=out)
    eng.close()
    d6 = small_run(steps=6, interval=3)
    d6["simulate"].update({"interval_restart": 3, "num_restart_files": 2})
    resumed, rlogs = simulate(d6, quiet=True, engine_cls=Engine, save=True, outdir=out, resume=True)
    assert [lg["step"] for lg in rlogs] == [4, 5, 6, 7]  # state.step 3 : last_step 6
    assert sorted(os.listdir(out)) == ["restart.h5.3", "restart.h5.6", "stat.h5"]
    lib = resumed.lib
    assert restart.listing(lib, os.path.join(out, "stat.h5")) == ["3", "6"]
    whole, wlogs = simulate(d6, quiet=True, engine_cls=Engine)
    assert rlogs[-1]["t"] == wlogs[-1]["t"] and resumed.get_state() == whole.get_state()
    for a, b in zip(resumed.download_flow(), whole.download_flow()):
        assert np.array_equal(a, b)
    for s in range(2):
        pa, pb = resumed.download_particles(s), whole.download_particles(s)
        oa, ob = np.argsort(pa["ids"]), np.argsort(pb["ids"])
        for k in pa:
            assert np.array_equal(pa[k][oa], pb[k][ob]), (s, k)
    resumed.close()
    whole.close()
