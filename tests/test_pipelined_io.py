"""Pipelined host I/O (cmf_gpu_ctx_put_runoff_async / advance_async / wait / get_diag_async /
io_wait): the same steps as the synchronous calls, bit for bit, with the next step's runoff
uploaded while a step runs and each finished step's diagnostics read back while the next runs."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import runoff_series

FIELDS = ("outflw_aavg", "rivdph", "storge_amax")


@pytest.mark.gpu
def test_pipelined_io_equals_synchronous(case_dirs):
    import torch

    from cmf_b200 import HostModel, PhysicsGPU

    h = HostModel(case_dirs["cfg1s"])
    series = [np.ascontiguousarray(r, dtype=np.float64) for r in runoff_series(h.map("grarea"), "cfg1s", 12, hourly=True)]
    K = len(series)
    sync, pipe = PhysicsGPU(h), PhysicsGPU(h)
    ref = []
    for r in series:
        sync.put_runoff(r)
        nt, dt, bud = sync.advance()
        out = {f: np.zeros(h.dims.nseqall) for f in FIELDS}
        sync.get_diag_fields(out)
        ref.append((nt, dt, bud, out))
    # pinned host buffers, two per field so that a read-back never lands in a buffer being read
    outs = [{f: torch.zeros(h.dims.nseqall, dtype=torch.float64).pin_memory().numpy() for f in FIELDS} for _ in range(K)]
    pipe.put_runoff_async(series[0])
    got = []
    for k in range(K):
        pipe.advance_async()
        if k + 1 < K:
            pipe.put_runoff_async(series[k + 1])
        got.append(pipe.wait())
        pipe.get_diag_fields_async(outs[k])
    pipe.io_wait()
    # two steps in flight: step k+1 is queued before the host waits for step k
    two = PhysicsGPU(h)
    outs2 = [{f: torch.zeros(h.dims.nseqall, dtype=torch.float64).pin_memory().numpy() for f in FIELDS} for _ in range(K)]
    got2 = []
    two.put_runoff_async(series[0])
    two.advance_async()
    two.get_diag_fields_async(outs2[0])
    two.put_runoff_async(series[1])
    two.advance_async()
    for k in range(K):
        got2.append(two.wait())
        two.io_wait()                                  # step k's read-back (step k+1's is not queued yet)
        if k + 1 < K:
            two.get_diag_fields_async(outs2[k + 1])    # after step k+1's launch, before step k+2's
        if k + 2 < K:
            two.put_runoff_async(series[k + 2])
            two.advance_async()
    two.io_wait()
    for k in range(K):
        nt, dt, bud, out = ref[k]
        for nt2, dt2, bud2 in (got[k], got2[k]):
            assert np.array_equal(nt, nt2) and np.array_equal(dt, dt2), k
            assert bud == bud2, k
        for f in FIELDS:
            assert np.array_equal(out[f].view(np.uint64), outs2[k][f].view(np.uint64)), (k, f)
        nt2, dt2, bud2 = got[k]
        assert np.array_equal(nt, nt2) and np.array_equal(dt, dt2), k
        assert bud == bud2, k
        for f in FIELDS:
            assert np.array_equal(out[f].view(np.uint64), outs[k][f].view(np.uint64)), (k, f)
    s1, s2, s3 = sync.get_state(), pipe.get_state(), two.get_state()
    for key in ("rivsto", "fldsto", "rivout", "fldout"):
        assert np.array_equal(s1[key], s2[key]) and np.array_equal(s1[key], s3[key]), key
    sync.close()
    pipe.close()
    two.close()


@pytest.mark.gpu
def test_pipelined_io_call_order(case_dirs):
    """At most two launched steps; wait needs a launched step; the synchronous advance refuses
    while steps are in flight; a synchronous put_runoff replaces a staged field."""
    from cmf_b200 import HostModel, PhysicsGPU

    h = HostModel(case_dirs["cfg1s"])
    r = np.ascontiguousarray(next(runoff_series(h.map("grarea"), "cfg1s", 1, hourly=True)), dtype=np.float64)
    g, ref = PhysicsGPU(h), PhysicsGPU(h)
    with pytest.raises(RuntimeError):
        g.wait()
    g.put_runoff(r)
    g.advance_async()
    g.advance_async()
    with pytest.raises(RuntimeError):
        g.advance_async()
    with pytest.raises(RuntimeError):
        g.advance()
    g.wait()
    g.wait()
    ref.put_runoff(r)
    ref.advance()
    ref.advance()
    # a staged field, then a synchronous one: the synchronous field is the one the step uses
    g.put_runoff_async(np.zeros_like(r))
    g.put_runoff(r)
    g.advance()
    ref.put_runoff(r)
    ref.advance()
    assert np.array_equal(g.get_state()["rivsto"], ref.get_state()["rivsto"])
    g.close()
    ref.close()


def test_diag_buffers_checked_on_host():
    """The Python API checks each named host buffer's name, type and size before the library
    copies into it (a short buffer would be overrun by the read-back)."""
    from cmf_b200 import PhysicsGPU

    g = object.__new__(PhysicsGPU)          # host logic only: no device context
    g.M, g.N, g.P, g.Lp, g.h = 2, 10, 3, 4, None
    assert (g.diag_len("rivdph"), g.diag_len("pthflwsum_aavg"), g.diag_len("pthflw_aavg")) == (20, 6, 24)
    g._diag_ptrs({"rivdph": np.zeros(20), "pthflw_aavg": np.zeros(24)})
    for bad in ({"rivdph": np.zeros(19)}, {"rivdph": np.zeros(20, np.float32)}, {"nosuch": np.zeros(20)},
                {"pthflw_aavg": np.zeros(23)}, {"outflw_aavg": np.zeros(40)[::2]}):
        with pytest.raises(ValueError):
            g._diag_ptrs(bad)
