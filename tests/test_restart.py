"""Restart hand-off in the reference's binary layout (CMF_RESTART_WRITE / CMF_RESTART_INIT,
src/cmf_ctrl_restart_mod.F90:91-482), the storage-only restart's flow reconstruction
(CMF_CALC_OUTPRE, src/cmf_opt_outflw_mod.F90:308-421) and the sea-level boundary
(CMF_BOUNDARY_UPDATE, src/cmf_ctrl_boundary_mod.F90:267-304).

CPU: the oracle's writer/reader restate the reference's records; the host library (the product's
restart I/O) must write byte-identical files and read identical arrays.  GPU: a run resumed from a
restart must equal the uninterrupted run bit for bit, and the GPU resumed from an oracle restart
(full and storage-only) and under a sea-level boundary must stay within the parity bar."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import rel_close, runoff_series

PROG = ("rivsto", "fldsto", "rivout_pre", "fldout_pre", "rivdph_pre", "fldsto_pre", "damsto", "levsto", "pthflw_pre")
CASE = "cfg1s"


def _oracle_run(case_dir, steps, seed=3):
    from oracle import Oracle

    o = Oracle(case_dir)
    gr = o.d("grarea")
    forc = list(runoff_series(gr, CASE, steps, seed=seed, hourly=True))
    for r in forc:
        o.put_runoff(r)
        o.advance()
    return o


def _oracle_state(o):
    return {k: o.d(k).copy() for k in PROG + ("rivout", "fldout", "pthflw", "daminf")}


@pytest.mark.parametrize("dbl", [True, False])
@pytest.mark.parametrize("stoonly", [False, True])
def test_host_writer_matches_oracle_bytes_and_reader(case_dirs, tmp_path, dbl, stoonly):
    from cmf_b200 import HostModel

    o = _oracle_run(case_dirs[CASE], 5)
    a, b = str(tmp_path / "orc.bin"), str(tmp_path / "host.bin")
    o.write_restart(a, dbl=dbl, stoonly=stoonly)
    h = HostModel(case_dirs[CASE])
    h.write_restart(b, _oracle_state(o), dbl=dbl, stoonly=stoonly)
    assert open(a, "rb").read() == open(b, "rb").read()
    assert open(a + ".pth", "rb").read() == open(b + ".pth", "rb").read()
    nrec = 2 + (0 if stoonly else 4) + int(h.opts.ldamout) + int(h.opts.llevee)
    assert os.path.getsize(a) == (8 if dbl else 4) * h.nx * h.ny * nrec
    got = h.read_restart(a, dbl=dbl, stoonly=stoonly)
    from oracle import Oracle

    o2 = Oracle(case_dirs[CASE])
    o2.read_restart(a, dbl=dbl, stoonly=stoonly)
    for k in PROG:
        assert np.array_equal(got[k].view(np.int64), o2.d(k).view(np.int64)), k
    for k in ("rivout", "fldout", "pthflw"):
        assert not np.any(got[k]) and not np.any(o2.d(k)), k     # the binary path leaves them zero


def test_restart_file_layout(case_dirs, tmp_path):
    from cmf_b200 import HostModel

    o = _oracle_run(case_dirs[CASE], 3)
    f = str(tmp_path / "r.bin")
    o.write_restart(f, dbl=True)
    h = HostModel(case_dirs[CASE])
    recs = np.fromfile(f, dtype=np.float64).reshape(-1, h.ny, h.nx)
    land = np.zeros((h.ny, h.nx), dtype=bool)
    land[h.i1seqy - 1, h.i1seqx - 1] = True
    assert np.all(recs[:, ~land] == 1.0e20)
    for k, name in enumerate(("rivsto", "fldsto", "rivout_pre", "fldout_pre", "rivdph_pre", "fldsto_pre", "damsto", "levsto")):
        assert np.array_equal(recs[k][h.i1seqy - 1, h.i1seqx - 1], o.d(name)), name
    pth = np.fromfile(f + ".pth", dtype=np.float64)
    assert np.array_equal(pth, o.d("pthflw_pre"))


def test_oracle_restart_resume_is_exact(case_dirs, tmp_path):
    """Oracle: run, write, read into a fresh model, continue -- prognostics identical to the
    uninterrupted run (only the first sub-step's velocity diagnostic may differ: the binary
    restart leaves D2RIVOUT at zero)."""
    from oracle import Oracle

    steps, more = 5, 4
    o = Oracle(case_dirs[CASE])
    gr = o.d("grarea")
    forc = list(runoff_series(gr, CASE, steps + more, seed=4, hourly=True))
    for r in forc[:steps]:
        o.put_runoff(r)
        o.advance()
    f = str(tmp_path / "r.bin")
    o.write_restart(f)
    o2 = Oracle(case_dirs[CASE])
    o2.read_restart(f)
    for r in forc[steps:]:
        o.put_runoff(r)
        o2.put_runoff(r)
        assert o.advance() == o2.advance()
    for k in PROG:
        assert np.array_equal(o.d(k).view(np.int64), o2.d(k).view(np.int64)), k


def test_oracle_outpre_restates_manning(case_dirs, tmp_path):
    """CMF_CALC_OUTPRE against an independent numpy statement of the same formulas."""
    from oracle import Oracle

    o = _oracle_run(case_dirs[CASE], 6)
    f = str(tmp_path / "r.bin")
    o.write_restart(f, stoonly=True)
    o2 = Oracle(case_dirs[CASE])
    o2.read_restart(f, stoonly=True)
    o2.physics_fldstg()
    o2.calc_outpre()
    R = int(o2.i("i1next").size)
    nxt = o2.i("i1next")
    nriv = int(np.sum(nxt >= 0))
    rivelv, rivdph, wth, man = o2.d("rivelv"), o2.d("rivdph"), o2.d("rivwth"), o2.d("rivman")
    sfc = rivelv + rivdph
    p23 = float(np.float32(2.0) / np.float32(3.0))
    j = nxt[:nriv]
    slope = (sfc[:nriv] - sfc[j]) * (1.0 / o2.d("nxtdst")[:nriv])
    dflw = np.maximum(sfc[:nriv], sfc[j]) - rivelv[:nriv]
    area = wth[:nriv] * dflw
    q = np.where(area > float(np.float32(1e-5)),
                 area * (((1.0 / man[:nriv]) * np.power(np.maximum(dflw, 0), p23)) * np.sqrt(np.abs(slope))), 0.0)
    q = np.where(slope < 0, -q, q)
    ok, worst, bad = rel_close(o2.d("rivout_pre")[:nriv], q, 1e-12)
    assert ok, (worst, bad)
    assert np.array_equal(o2.d("rivdph_pre"), o2.d("rivdph"))
    assert R == o2.d("rivsto").size


def test_oracle_boundary_update(case_dirs):
    from oracle import Oracle

    o = Oracle(case_dirs[CASE])
    n = o.d("elevtn").size
    rng = np.random.default_rng(0)
    sl, ms = rng.normal(0, 0.5, n), rng.normal(0, 0.2, n)
    o.update_boundary(sl, ms)
    assert np.array_equal(o.d("dwnelv"), (o.d("elevtn") + ms) + sl)
    o.update_boundary(None, None)
    assert np.array_equal(o.d("dwnelv"), o.d("elevtn"))


# ------------------------------------------------------------------------------------------ GPU
def _gpu_compare(g, o, tol=1e-9, fields=("rivsto", "fldsto", "rivout", "fldout")):
    st = g.get_state()
    for f in fields:
        ok, worst, bad = rel_close(st[f][0], o.d(f), tol)
        assert ok, (f, worst, bad)


@pytest.mark.gpu
def test_gpu_resume_from_own_restart_is_exact(case_dirs, tmp_path):
    from cmf_b200 import HostModel, PhysicsGPU

    h = HostModel(case_dirs[CASE])
    gr = h.map("grarea")
    forc = list(runoff_series(gr, CASE, 9, seed=5, hourly=True))
    a = PhysicsGPU(h)
    for r in forc[:5]:
        a.put_runoff(r)
        a.advance()
    f = str(tmp_path / "g.bin")
    a.write_restart(f)
    b = PhysicsGPU(h)
    b.read_restart(f)
    for r in forc[5:]:
        a.put_runoff(r)
        b.put_runoff(r)
        na, da, _ = a.advance()
        nb, db, _ = b.advance()
        assert na[0] == nb[0] and da[0] == db[0]
    sa, sb = a.get_state(), b.get_state()
    for k in PROG:
        assert np.array_equal(sa[k].view(np.int64), sb[k].view(np.int64)), k


@pytest.mark.gpu
@pytest.mark.parametrize("stoonly", [False, True])
def test_gpu_from_oracle_restart_matches_oracle(case_dirs, tmp_path, stoonly):
    from cmf_b200 import HostModel, PhysicsGPU
    from oracle import Oracle

    o = _oracle_run(case_dirs[CASE], 6, seed=6)
    f = str(tmp_path / "o.bin")
    o.write_restart(f, stoonly=stoonly)
    o2 = Oracle(case_dirs[CASE])
    o2.read_restart(f, stoonly=stoonly)
    h = HostModel(case_dirs[CASE])
    g = PhysicsGPU(h)
    g.read_restart(f, stoonly=stoonly)
    if stoonly:
        o2.physics_fldstg()
        o2.calc_outpre()
        st = g.get_state()
        for k in ("rivout_pre", "fldout_pre", "rivdph_pre", "pthflw_pre", "rivsto", "fldsto"):
            ok, worst, bad = rel_close(st[k][0], o2.d(k), 1e-9)
            assert ok, (k, worst, bad)
    gr = h.map("grarea")
    for r in runoff_series(gr, CASE, 5, seed=7, hourly=True):
        g.put_runoff(r)
        o2.put_runoff(r)
        nt, dt, _ = g.advance()
        assert (nt[0], dt[0]) == o2.advance()
    _gpu_compare(g, o2)


@pytest.mark.gpu
def test_gpu_sea_level_boundary_matches_oracle(case_dirs):
    from cmf_b200 import HostModel, PhysicsGPU
    from oracle import Oracle

    h = HostModel(case_dirs[CASE])
    o = Oracle(case_dirs[CASE])
    g = PhysicsGPU(h)
    n = h.dims.nseqall
    rng = np.random.default_rng(11)
    gr = h.map("grarea")
    for k, r in enumerate(runoff_series(gr, CASE, 6, seed=8, hourly=True)):
        sl = rng.normal(0.0, 0.8, n)            # sea-level anomaly of this step [m]
        ms = np.full(n, 0.3) if k % 2 else None
        g.update_boundary(sl, ms)
        o.update_boundary(sl, ms)
        g.put_runoff(r)
        o.put_runoff(r)
        nt, dt, _ = g.advance()
        assert (nt[0], dt[0]) == o.advance()
    _gpu_compare(g, o)
