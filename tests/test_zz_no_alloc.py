"""cmf_gpu_stage_noalloc: the stage scheme + CFL minimum for callers that cannot let the library
allocate device memory (their own pool owns it, or they run inside a stream capture).  The
caller owns every buffer; the library only uses its fixed per-GPU scratch array.

Checked on two calls in a row (so the second call also shows that the shared scratch array
carries nothing stale from the first) against
  - the context entry point (cmf_gpu_ctx_stage, which works in buffers the context allocated):
    DT_MIN bit for bit (NT depends on every bit of it), the fields within the parity tolerance;
  - the oracle's stage scheme and CALC_ADPSTP minimum (src/cmf_calc_fldstg_mod.F90:21-110,
    src/cmf_ctrl_physics_mod.F90:161-210) started from the same storage: DT_MIN bit for bit."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import rel_close, runoff_series

pytestmark = pytest.mark.gpu

RTOL = 1e-9


def test_stage_noalloc_matches_context_entry_point(case_dirs):
    import torch

    from cmf_b200 import HostModel, PhysicsGPU, _abi

    lib = _abi.load()
    h = HostModel(case_dirs["stress"])
    g = PhysicsGPU(h, opts_override={"llevee": 0})     # the variant implements the default stage scheme
    N, L = h.dims.nseqall, h.dims.nlfp
    dev = torch.device("cuda", 0)

    def dbuf(a):
        return torch.tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)

    maps = {k: dbuf(h.map(k)) for k in ("rivstomax", "rivlen", "rivwth", "grarea", "rivelv", "nxtdst")}
    maps["fldstomax"] = dbuf(h.map("fldstomax")[: L * N])
    maps["fldgrd"] = dbuf(h.map("fldgrd")[: L * N])
    i2mask = torch.tensor(h.map("i2mask"), dtype=torch.int32, device=dev)
    series = iter(runoff_series(h.map("grarea"), "stress", 40))
    for _ in range(12):                                 # reach a flooded state first
        g.put_runoff(next(series))
        g.advance()
    for call in range(2):
        before = g.get_state()
        dt_min_ctx = g.stage()[0]                        # existing entry point
        after = g.get_state()
        diag = g.get_diag()
        rivsto = dbuf(before["rivsto"][0])
        fldsto = dbuf(before["fldsto"][0])
        outs = {k: torch.full((N,), -1.0, dtype=torch.float64, device=dev)
                for k in ("rivdph", "flddph", "fldfrc", "fldare", "sfcelv", "storge")}
        dtmin = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
        a = _abi.StageDevArgs(nseqall=N, nseqriv=h.dims.nseqriv, nlfp=L, ladpstp=1, dt_def=h.dt,
                              pgrv=h.params.pgrv, pdstmth=h.params.pdstmth, pcadp=h.params.pcadp,
                              dfrcinc=h.params.dfrcinc)
        for k, t in maps.items():
            setattr(a, k, t.data_ptr())
        a.i2mask = i2mask.data_ptr()
        a.rivsto, a.fldsto = rivsto.data_ptr(), fldsto.data_ptr()
        for k, t in outs.items():
            setattr(a, k, t.data_ptr())
        a.dt_min_out = dtmin.data_ptr()
        a.stream = None
        torch.cuda.synchronize()
        rc = lib.cmf_gpu_stage_noalloc(C.byref(a))
        assert rc == 0, lib.cmf_gpu_last_error()
        torch.cuda.synchronize()
        assert dtmin.item() == dt_min_ctx, (call, dtmin.item(), dt_min_ctx)     # bit for bit
        for k, ref in (("rivsto", after["rivsto"][0]), ("fldsto", after["fldsto"][0])):
            got = (rivsto if k == "rivsto" else fldsto).cpu().numpy()
            ok, worst, bad = rel_close(got, ref, RTOL)
            assert ok, (call, k, worst, bad)
        for k, t in outs.items():
            ok, worst, bad = rel_close(t.cpu().numpy(), diag[k][0], RTOL)
            assert ok, (call, k, worst, bad)
        g.put_runoff(next(series))                       # a different state for the second call
        g.advance()


def _noalloc_stage(lib, h, maps, i2mask, rivsto_np, fldsto_np, dev):
    import torch

    from cmf_b200 import _abi

    N, L = h.dims.nseqall, h.dims.nlfp
    rivsto = torch.tensor(np.ascontiguousarray(rivsto_np, dtype=np.float64), device=dev)
    fldsto = torch.tensor(np.ascontiguousarray(fldsto_np, dtype=np.float64), device=dev)
    outs = {k: torch.full((N,), -1.0, dtype=torch.float64, device=dev)
            for k in ("rivdph", "flddph", "fldfrc", "fldare", "sfcelv", "storge")}
    dtmin = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    a = _abi.StageDevArgs(nseqall=N, nseqriv=h.dims.nseqriv, nlfp=L, ladpstp=1, dt_def=h.dt, pgrv=h.params.pgrv,
                          pdstmth=h.params.pdstmth, pcadp=h.params.pcadp, dfrcinc=h.params.dfrcinc)
    for k, t in maps.items():
        setattr(a, k, t.data_ptr())
    a.i2mask = i2mask.data_ptr()
    a.rivsto, a.fldsto = rivsto.data_ptr(), fldsto.data_ptr()
    for k, t in outs.items():
        setattr(a, k, t.data_ptr())
    a.dt_min_out = dtmin.data_ptr()
    a.stream = None
    torch.cuda.synchronize()
    rc = lib.cmf_gpu_stage_noalloc(C.byref(a))
    assert rc == 0, lib.cmf_gpu_last_error()
    torch.cuda.synchronize()
    res = {k: t.cpu().numpy() for k, t in outs.items()}
    res["rivsto"], res["fldsto"] = rivsto.cpu().numpy(), fldsto.cpu().numpy()
    return dtmin.item(), res


def test_stage_noalloc_matches_oracle(case_dirs):
    """The same entry point against the oracle's stage scheme and CFL minimum, both started from the
    oracle's storage after a flood (config-0 network, runoff x40 so that floodplain layers fill)."""
    import torch

    from cmf_b200 import HostModel, _abi
    from oracle import Oracle

    lib = _abi.load()
    h = HostModel(case_dirs["cfg0"])
    o = Oracle(case_dirs["cfg0"])
    N, L = h.dims.nseqall, h.dims.nlfp
    dev = torch.device("cuda", 0)

    def dbuf(a):
        return torch.tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)

    maps = {k: dbuf(h.map(k)) for k in ("rivstomax", "rivlen", "rivwth", "grarea", "rivelv", "nxtdst")}
    maps["fldstomax"] = dbuf(h.map("fldstomax")[: L * N])
    maps["fldgrd"] = dbuf(h.map("fldgrd")[: L * N])
    i2mask = torch.tensor(h.map("i2mask"), dtype=torch.int32, device=dev)
    series = iter(runoff_series(h.map("grarea"), "cfg0", 60))
    for _ in range(36):
        o.put_runoff(next(series) * 40.0)
        o.advance()
    flooded = 0
    for call in range(2):
        pre_r, pre_f = o.d("rivsto"), o.d("fldsto")
        dt_min_o = o.stage()                                    # stage + this domain's CFL minimum
        dt_min_g, got = _noalloc_stage(lib, h, maps, i2mask, pre_r, pre_f, dev)
        assert dt_min_g == dt_min_o, (call, dt_min_g, dt_min_o)   # bit for bit
        for k in ("rivsto", "fldsto", "rivdph", "flddph", "fldfrc", "fldare", "sfcelv", "storge"):
            ok, worst, bad = rel_close(got[k], o.d(k), RTOL)
            assert ok, (call, k, worst, bad)
        flooded = max(flooded, int(np.sum(o.d("fldsto") > 0)))
        o.put_runoff(next(series) * 40.0)
        o.advance()
    assert flooded > 0                                          # the floodplain branch ran


def test_stage_noalloc_rejects_oversized_domain():
    from cmf_b200 import _abi

    lib = _abi.load()
    a = _abi.StageDevArgs(nseqall=3_000_000, nseqriv=2_000_000, nlfp=10, ladpstp=1, dt_def=3600.0)
    for f, _ in a._fields_[9:-1]:
        setattr(a, f, 16)     # non-null placeholders: the size check runs before any device work
    rc = lib.cmf_gpu_stage_noalloc(C.byref(a))
    assert rc == -1 and b"scratch limit" in lib.cmf_gpu_last_error()
