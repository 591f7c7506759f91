"""Runoff interpolation (CMF_FORCING_PUT: ROFF_INTERP / CONV_RESOL, src/cmf_ctrl_forcing_mod.F90:716-831)
and the input-matrix reader (CMF_INPMAT_INIT_BIN, :418-458).

CPU: the host reader returns exactly what was written in the reference's record layout, and the
oracle's ROFF_INTERP equals an independent numpy statement of the sum bit for bit.  GPU: the device
interpolation of every member equals the oracle bit for bit (same multiplications, divisions and
summation order; no fused multiply-add), for fp64 and fp32 fields and with the GET cleaning."""
from __future__ import annotations

import numpy as np
import pytest

CASE = "cfg1s"


def _setup(case_dir, tmp_path=None):
    from cmf_b200 import HostModel, synth

    h = HostModel(case_dir)
    nxin, nyin, ix, iy, ia = synth.make_inpmat(h.nx, h.ny, h.i1seqx, h.i1seqy, h.map("grarea"), factor=2, inpn=3, seed=1)
    return h, (nxin, nyin, ix, iy, ia.astype(np.float64))


def _fields(nxin, nyin, members, seed, dirty=False):
    rng = np.random.default_rng(seed)
    g = rng.gamma(0.8, 2.5, (members, nyin, nxin))
    g[rng.random(g.shape) < 0.02] = np.float32(1.0e20)          # RMIS inputs are skipped
    if dirty:
        g[rng.random(g.shape) < 0.02] = np.nan
        g[rng.random(g.shape) < 0.05] *= -1.0
    return g


def _numpy_interp(grid, inpmat, drofunit, N):
    nxin, nyin, ix, iy, ia = inpmat
    out = np.zeros(N)
    rmis = float(np.float32(1.0e20))
    for k in range(ix.shape[0]):
        use = (ix[k] > 0) & (ix[k] <= nxin) & (iy[k] >= 1) & (iy[k] <= nyin)
        v = np.where(use, grid[np.clip(iy[k] - 1, 0, nyin - 1), np.clip(ix[k] - 1, 0, nxin - 1)], rmis)
        add = np.where(v != rmis, (v * ia[k]) / drofunit, 0.0)
        out = np.where(v != rmis, out + add, out)
    return out


def test_inpmat_reader_roundtrip(case_dirs, tmp_path):
    from cmf_b200 import synth

    h, (nxin, nyin, ix, iy, ia) = _setup(case_dirs[CASE])
    f = str(tmp_path / "inpmat.bin")
    synth.write_inpmat(f, h.nx, h.ny, h.i1seqx, h.i1seqy, ix, iy, ia.astype(np.float32))
    rx, ry, ra = h.read_inpmat(f, 3)
    assert np.array_equal(rx, ix) and np.array_equal(ry, iy) and np.array_equal(ra, ia)
    # mass conservation of the synthetic matrix: the areas of a cell sum to its area (fp32 rounding)
    assert np.allclose(ra.sum(0), h.map("grarea"), rtol=1e-6)


def test_oracle_roff_interp_equals_numpy(case_dirs):
    from oracle import Oracle

    h, inpmat = _setup(case_dirs[CASE])
    o = Oracle(case_dirs[CASE])
    g = _fields(inpmat[0], inpmat[1], 1, 3)[0]
    o.put_runoff_grid(g, inpmat)
    ref = _numpy_interp(g, inpmat, h.drofunit, h.dims.nseqall)
    assert np.array_equal(o.d("runoff").view(np.int64), ref.view(np.int64))
    # GET cleaning: NaN -> RMIS (skipped), negative -> 0
    gd = _fields(inpmat[0], inpmat[1], 1, 4, dirty=True)[0]
    o.put_runoff_grid(gd, inpmat, clean=True)
    gc = np.where(np.isnan(gd), float(np.float32(1e20)), gd)
    gc = np.maximum(gc, 0.0)
    assert np.array_equal(o.d("runoff"), _numpy_interp(gc, inpmat, h.drofunit, h.dims.nseqall))


def _device_runoff(p):
    from cmf_b200 import emulator as E

    v = E.Features(p, np.ones(p.N)).runoff_view()
    return v.cpu().numpy()


@pytest.mark.gpu
def test_gpu_roff_interp_matches_oracle_bit_exact(case_dirs):
    import torch

    from cmf_b200 import PhysicsGPU
    from oracle import Oracle

    h, inpmat = _setup(case_dirs[CASE])
    M = 3
    p = PhysicsGPU(h, nmembers=M)
    p.set_runoff_map(inpmat)
    o = Oracle(case_dirs[CASE])
    for clean in (False, True):
        g = _fields(inpmat[0], inpmat[1], M, 5, dirty=clean)
        p.put_runoff_grid(g, clean=clean)
        got = _device_runoff(p)
        for m in range(M):
            o.put_runoff_grid(g[m], inpmat, clean=clean)
            assert np.array_equal(got[m].view(np.int64), o.d("runoff").view(np.int64)), (clean, m)
    # fp32 fields (what the reference reads from its runoff files), from device memory
    g32 = _fields(inpmat[0], inpmat[1], M, 6).astype(np.float32)
    p.put_runoff_grid(torch.tensor(g32, device="cuda:0"))
    got = _device_runoff(p)
    for m in range(M):
        o.put_runoff_grid(g32[m].astype(np.float64), inpmat)
        assert np.array_equal(got[m].view(np.int64), o.d("runoff").view(np.int64)), m
    p.close()


@pytest.mark.gpu
def test_gpu_conv_resol_and_advance_match_oracle(case_dirs):
    from cmf_b200 import PhysicsGPU
    from conftest import rel_close
    from oracle import Oracle

    h, _ = _setup(case_dirs[CASE])
    p = PhysicsGPU(h)
    p.set_runoff_map(None)
    o = Oracle(case_dirs[CASE])
    rng = np.random.default_rng(9)
    for k in range(5):
        g = rng.gamma(0.8, 2.5 * 24.0, (1, h.ny, h.nx))
        p.put_runoff_grid(g)
        o.put_runoff_grid(g[0])
        assert np.array_equal(_device_runoff(p)[0].view(np.int64), o.d("runoff").view(np.int64))
        nt, dt, _ = p.advance()
        assert (nt[0], dt[0]) == o.advance()
    st = p.get_state()
    for f in ("rivsto", "fldsto", "rivout", "fldout"):
        ok, worst, bad = rel_close(st[f][0], o.d(f), 1e-9)
        assert ok, (f, worst, bad)
    p.close()
