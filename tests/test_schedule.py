"""Launch schedules and the online autotuner (cmf_gpu_ctx_get_schedule / _set_schedule).

Every schedule -- graph of phase kernels with any block sizes and occupancy profile, or the
persistent kernel -- must produce the same bits: prognostic state, NT/DT and the water budgets
(summed from per-warp partials, so they do not depend on the block size).  That is what lets the
autotuner switch schedules on real outer steps of the run."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import runoff_series

pytestmark = pytest.mark.gpu

CANDIDATES = [dict(mode=0, flux_block=bf, rate_block=bf, store_block=bs, profile=pr)
              for bf in (64, 128, 256) for bs in (128, 256) for pr in (0, 1)] + [dict(mode=2)]


def _same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.int64), np.ascontiguousarray(b).view(np.int64))


@pytest.mark.parametrize("name,members,nsteps", [("stress", 1, 20), ("cfg1s", 2, 12)])
def test_every_schedule_bit_identical(case_dirs, name, members, nsteps):
    from cmf_b200 import HostModel, PhysicsGPU

    h = HostModel(case_dirs[name])
    gr = h.map("grarea")
    series = [list(runoff_series(gr, name, nsteps, seed=s, hourly=True)) for s in range(members)]
    ref = None
    for cand in CANDIDATES:
        g = PhysicsGPU(h, nmembers=members, block_size=128)
        g.set_schedule(**cand)
        out = []
        for k in range(nsteps):
            g.put_runoff(np.stack([series[m][k] for m in range(members)]))
            nt, dt, bud = g.advance()
            out.append((nt.copy(), dt.copy(), [dict(b) for b in bud]))
        st = g.get_state()
        if ref is None:
            ref = (out, st)
            continue
        for k, ((na, da, ba), (nb, db, bb)) in enumerate(zip(out, ref[0])):
            assert np.array_equal(na, nb) and _same(da, db), (cand, k)
            for m in range(members):
                for f in ba[m]:
                    assert _same(np.float64(ba[m][f]), np.float64(bb[m][f])), (cand, k, m, f)
        for f in ("rivsto", "fldsto", "rivout", "fldout", "levsto", "damsto", "pthflw"):
            assert _same(st[f], ref[1][f]), (cand, f)
        g.close()


def test_online_autotuner_times_candidates_and_caches(case_dirs):
    """A launch_mode 0 context without a fixed block size tunes itself on its first outer steps
    (4 warm-up steps, then 2 per candidate) and keeps the fastest; a second context of the same
    network shape starts from the cached choice.  The trajectory equals a fixed schedule's."""
    from cmf_b200 import HostModel, PhysicsGPU, _abi

    _abi.load().cmf_gpu_schedule_cache_clear()        # earlier tests may have tuned this shape
    h = HostModel(case_dirs["cfg1s"])
    gr = h.map("grarea")
    tuned = PhysicsGPU(h)
    fixed = PhysicsGPU(h, block_size=128)
    q0 = tuned.schedule()
    assert q0["tuned"] == -1
    ncand = 9
    steps = 4 + 2 * ncand + 2
    for r in runoff_series(gr, "cfg1s", steps, hourly=True):
        tuned.put_runoff(r)
        fixed.put_runoff(r)
        a, _, ba = tuned.advance()
        b, _, bb = fixed.advance()
        assert a[0] == b[0] and ba[0]["stonew2"] == bb[0]["stonew2"]
    q = tuned.schedule()
    assert q["tuned"] == 1 and q["candidates"] == ncand, q
    assert 0 < q["best_us_per_substep"] <= q["worst_us_per_substep"]
    sa, sb = tuned.get_state(), fixed.get_state()
    for f in ("rivsto", "fldsto", "rivout", "fldout"):
        assert _same(sa[f], sb[f]), f
    again = PhysicsGPU(h)
    q2 = again.schedule()
    assert q2["tuned"] == 0 and all(q2[k] == q[k] for k in ("mode", "flux_block", "rate_block", "store_block", "profile"))
    print("tuned schedule:", q)
