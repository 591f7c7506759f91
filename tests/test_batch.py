"""Batched multi-domain launch (regional domains of uneven size, each with its own members, one
graph launch per coupling step): every domain and member must come out exactly as when its
context advances alone -- same NT/DT each step, bit-identical state -- and the first domain must
also stay within the parity bar against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_close, runoff_series

STEPS = 8
DOMAINS = (("cfg0", 1), ("cfg1s", 3), ("stress", 2))   # (case, members), uneven sizes and options


def _runoff(h, name, members, k_seed):
    gr = h.map("grarea")
    gens = [list(runoff_series(gr, name, STEPS, seed=k_seed + 17 * m, hourly=True)) for m in range(members)]
    return [np.stack([gens[m][k] for m in range(members)]) for k in range(STEPS)]


def _state_bits(p):
    st, dg = p.get_state(), p.get_diag()
    out = {k: np.ascontiguousarray(v).view(np.int64) for k, v in st.items()}
    for k in ("rivdph", "flddph", "rivout_aavg", "outflw_aavg", "storge_amax"):
        out["diag_" + k] = np.ascontiguousarray(dg[k]).view(np.int64)
    return out


@pytest.mark.gpu
def test_batch_equals_each_domain_alone(case_dirs):
    from cmf_b200 import HostModel, PhysicsBatch, PhysicsGPU
    from oracle import Oracle

    hosts = [HostModel(case_dirs[name]) for name, _ in DOMAINS]
    forc = [_runoff(h, name, m, 100 + 7 * k) for k, ((name, m), h) in enumerate(zip(DOMAINS, hosts))]
    # one block size for both sides: the budgets are block-partial sums (state does not depend on it)
    alone = [PhysicsGPU(h, nmembers=m, block_size=256) for h, (_, m) in zip(hosts, DOMAINS)]
    batched = [PhysicsGPU(h, nmembers=m, block_size=256) for h, (_, m) in zip(hosts, DOMAINS)]
    batch = PhysicsBatch(batched)
    oracle = Oracle(case_dirs[DOMAINS[0][0]])
    for k in range(STEPS):
        for d in range(len(DOMAINS)):
            alone[d].put_runoff(forc[d][k])
            batched[d].put_runoff(forc[d][k])
        oracle.put_runoff(forc[0][k][0])
        res = batch.advance()
        nt_o, dt_o = oracle.advance()
        for d in range(len(DOMAINS)):
            nt, dt, bud = alone[d].advance()
            nt_b, dt_b, bud_b = res[d]
            assert np.array_equal(nt, nt_b) and np.array_equal(dt.view(np.int64), dt_b.view(np.int64)), (d, k)
            assert bud == bud_b, (d, k)
        assert res[0][0][0] == nt_o and res[0][1][0] == dt_o
    for d in range(len(DOMAINS)):
        a, b = _state_bits(alone[d]), _state_bits(batched[d])
        for f in a:
            assert np.array_equal(a[f], b[f]), (DOMAINS[d], f)
    st = batched[0].get_state()
    for f in ("rivsto", "fldsto", "rivout", "fldout"):
        ok, worst, bad = rel_close(st[f][0], oracle.d(f), 1e-9)
        assert ok, (f, worst, bad)
    # members differ (their forcing does), so a mix-up between members would have been caught
    st1 = batched[1].get_state()
    assert not np.array_equal(st1["rivsto"][0], st1["rivsto"][1])
    batch.close()
    for p in alone + batched:
        p.close()


def test_batch_rejects_bad_input():
    """Argument checks happen before any CUDA call (runs without a GPU)."""
    import ctypes as C

    from cmf_b200 import _abi

    lib = _abi.load()
    h = C.c_void_p()
    assert lib.cmf_gpu_batch_create(None, 1, C.byref(h)) == -1
    arr = (C.c_void_p * 1)(None)
    assert lib.cmf_gpu_batch_create(arr, 1, C.byref(h)) == -1
    assert lib.cmf_gpu_batch_launch(None, 3600.0) == -3
