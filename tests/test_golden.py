"""Golden fixture (tests/golden/make_golden.py): a committed tiny case in the reference's formats with
the oracle's outputs.  The oracle must reproduce them bit for bit; the GPU path within 1e-9."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import rel_close

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASE = os.path.join(GOLD, "mini_case")
FIELDS = ("rivsto", "fldsto", "rivout", "fldout", "rivdph", "flddph", "levsto", "damsto", "pthflw",
          "rivout_aavg", "storge_amax")


def _gold():
    return dict(np.load(os.path.join(GOLD, "golden_mini.npz")))


def test_golden_case_exercises_the_options():
    g = _gold()
    assert g["fldsto"].max() > 0 and np.any(g["pthflw"] != 0) and g["damsto"].max() > 0
    assert g["nt"].min() >= 2


def test_oracle_reproduces_golden_bit_exact():
    from oracle import Oracle

    g = _gold()
    o = Oracle(CASE)
    for k in range(len(g["nt"])):
        o.put_runoff(g["runoff"][k])
        nt, dt = o.advance()
        assert nt == g["nt"][k] and dt == g["dt"][k]
    for f in FIELDS:
        assert np.array_equal(o.d(f).view(np.int64), g[f].view(np.int64)), f


def test_host_core_loads_golden_case():
    from cmf_b200 import HostModel

    h = HostModel(CASE)
    assert h.dims.nseqall == _gold()["rivsto"].size
    assert h.opts.lpthout and h.opts.llevee and h.opts.ldamout


@pytest.mark.gpu
def test_gpu_matches_golden():
    from cmf_b200 import HostModel, PhysicsGPU

    g = _gold()
    h = HostModel(CASE)
    p = PhysicsGPU(h)
    for k in range(len(g["nt"])):
        p.put_runoff(g["runoff"][k])
        nt, dt, _ = p.advance()
        assert nt[0] == g["nt"][k] and dt[0] == g["dt"][k]
    st, dg = p.get_state(), p.get_diag()
    got = {"rivsto": st["rivsto"][0], "fldsto": st["fldsto"][0], "rivout": st["rivout"][0], "fldout": st["fldout"][0],
           "levsto": st["levsto"][0], "damsto": st["damsto"][0], "pthflw": st["pthflw"][0],
           "rivdph": dg["rivdph"][0], "flddph": dg["flddph"][0], "rivout_aavg": dg["rivout_aavg"][0],
           "storge_amax": dg["storge_amax"][0]}
    for f in FIELDS:
        ok, worst, bad = rel_close(got[f], g[f], 1e-9)
        assert ok, (f, worst, bad)
