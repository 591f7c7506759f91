"""The product's host model core (C++) reproduces the reference initialisation bit for bit:
CALC_1D_SEQ sequence order, I1NEXT/I1UPST, READ_BIFPARAM tables, SET_FLDSTG, CMF_LEVEE_INIT,
CMF_DAMOUT_INIT and STORAGE_SEA_SURFACE, checked against the oracle's independent restatement."""
from __future__ import annotations

import numpy as np
import pytest


def _bits(a):
    a = np.asarray(a)
    return a.view(np.int64) if a.dtype == np.float64 else a


@pytest.mark.parametrize("name", ["cfg0", "cfg1s", "stress"])
def test_host_init_bit_exact(case_dirs, name):
    from cmf_b200 import HostModel
    from oracle import Oracle

    h = HostModel(case_dirs[name])
    o = Oracle(case_dirs[name])
    assert (h.dims.nseqall, h.dims.nseqriv, h.dims.nseqmax) == (o.nseqall, o.nseqriv, o.nseqmax)
    assert np.array_equal(h.i1seqx, o.i("i1seqx")) and np.array_equal(h.i1seqy, o.i("i1seqy"))
    on = o.i("i1next")
    assert np.array_equal(h.map("i1next"), np.where(on >= 0, on + 1, on))
    assert np.array_equal(h.map("i1upn"), o.i("i1upn"))
    # I1UPST: Fortran column-major (NSEQMAX,UPNMAX) vs the oracle's row-major [i][k], 1-based vs 0-based
    N, U = h.dims.nseqmax, h.dims.upnmax
    hu = h.map("i1upst").reshape(U, N).T
    ou = o.i("i1upst").reshape(N, U)
    for i in range(N):
        n = o.i("i1upn")[i]
        assert np.array_equal(hu[i, :n], ou[i, :n] + 1)
    for nm in ["rivelv", "elevtn", "nxtdst", "rivwth", "rivhgt", "rivlen", "rivman", "grarea", "rivstomax",
               "fldstomax", "fldgrd", "dwnelv"]:
        assert np.array_equal(_bits(h.map(nm)), _bits(o.d(nm))), nm
    st = h.initial_state()
    for nm in ["rivsto", "fldsto", "rivdph_pre", "damsto"]:
        assert np.array_equal(_bits(st[nm]), _bits(o.d(nm))), nm
    if h.opts.llevee:
        for nm in ["levhgt", "levfrc", "bashgt", "levdst", "levbassto", "levtopsto", "levfilsto"]:
            assert np.array_equal(_bits(h.map(nm)), _bits(o.d(nm))), nm
    if h.opts.lpthout:
        for nm in ["pth_elv", "pth_wth", "pth_dst", "pth_man"]:
            assert np.array_equal(_bits(h.map(nm)), _bits(o.d(nm))), nm
        assert np.array_equal(h.map("pth_upst"), o.i("pth_upst"))
        assert np.array_equal(h.map("pth_down"), o.i("pth_down"))
        assert np.array_equal(h.map("i1p_outn"), o.i("i1p_outn"))
        assert np.array_equal(h.map("i1p_infn"), o.i("i1p_infn"))
    if h.opts.ldamout:
        assert np.array_equal(h.map("i1dam"), o.i("i1dam"))
        assert np.array_equal(h.map("i2mask"), o.i("i2mask"))
        for nm in ["qn", "qf", "qa", "convol", "fldvol", "emevol", "adjvol"]:
            assert np.array_equal(_bits(h.map("dam_" + nm)), _bits(o.d("dam_" + nm))), nm


def test_sequence_is_topological(case_dirs):
    from cmf_b200 import HostModel

    h = HostModel(case_dirs["cfg1s"])
    nxt = h.map("i1next")
    R = h.dims.nseqriv
    assert np.all(nxt[:R] > np.arange(1, R + 1))      # I1NEXT(i) > i for every river cell
    assert np.all(nxt[R:] < 0)                         # mouths keep the negative code


def test_conv_resol_matches_oracle(case_dirs):
    from cmf_b200 import HostModel
    from oracle import Oracle

    h = HostModel(case_dirs["cfg0"])
    o = Oracle(case_dirs["cfg0"])
    rng = np.random.default_rng(5)
    grid = rng.gamma(0.8, 2.5, size=h.nx * h.ny).astype(np.float32).astype(np.float64)
    grid[::17] = float(np.float32(1e20))   # RMIS cells -> zero runoff
    a = h.conv_resol(grid)
    o.put_runoff_map(grid)
    assert np.array_equal(a.view(np.int64), o.d("runoff").view(np.int64))


def test_bad_case_reports_io_error(tmp_path):
    from cmf_b200 import HostModel

    with pytest.raises(RuntimeError, match="status -4"):
        HostModel(str(tmp_path))
