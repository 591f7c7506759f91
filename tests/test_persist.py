"""The persistent schedule (launch_mode 2): one cooperative kernel per coupling step with grid
barriers between the phases and the cell tiles interleaved over the CTAs.

It runs the same per-cell arithmetic as the graph of phase kernels, so states, NT/DT and budgets
must equal that path bit for bit (the budgets with the same 256-cell partial blocks), and the oracle
within the parity tolerance.  Its bounded waits are checked by a barrier that cannot complete."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_close, runoff_series

pytestmark = pytest.mark.gpu

RTOL = 1e-9
STATE_KEYS = ("rivsto", "fldsto", "rivout", "fldout", "rivout_pre", "fldout_pre", "rivdph_pre", "fldsto_pre",
              "levsto", "damsto", "daminf", "pthflw")
DIAG_KEYS = ("rivdph", "flddph", "fldfrc", "fldare", "sfcelv", "storge", "rivvel", "rivinf", "fldinf", "pthout",
             "outflw", "pthflwsum", "levdph", "rivout_aavg", "fldout_aavg", "outflw_aavg", "rivvel_aavg",
             "pthout_aavg", "runoff_aavg", "daminf_aavg", "storge_amax", "outflw_amax", "rivdph_amax",
             "pthflw_aavg", "pthflwsum_aavg")


def _same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.int64), np.ascontiguousarray(b).view(np.int64))


@pytest.mark.parametrize("name,members,nsteps", [("stress", 1, 30), ("cfg1s", 3, 16), ("cfg0", 2, 30)])
def test_persistent_equals_graph_bit_for_bit(case_dirs, name, members, nsteps):
    """Every state and diagnostic array, NT, DT and the budgets of every step are bit-identical to
    the graph of phase kernels (block size 256, the persistent kernel's tile)."""
    from cmf_b200 import HostModel, PhysicsGPU

    h = HostModel(case_dirs[name])
    a = PhysicsGPU(h, nmembers=members, launch_mode=2, ldiag_output=True)
    b = PhysicsGPU(h, nmembers=members, launch_mode=0, block_size=256, ldiag_output=True)
    assert a.launch_mode == 2 and b.launch_mode == 0
    gr = h.map("grarea")
    series = [list(runoff_series(gr, name, nsteps, seed=s, hourly=(name != "cfg0"))) for s in range(members)]
    for k in range(nsteps):
        r = np.stack([series[m][k] for m in range(members)])
        a.put_runoff(r)
        b.put_runoff(r)
        na, da, ba = a.advance()
        nb, db, bb = b.advance()
        assert np.array_equal(na, nb) and _same(da, db), f"step {k}: NT/DT"
        for m in range(members):
            for f, v in ba[m].items():
                assert _same(np.float64(v), np.float64(bb[m][f])), f"step {k} member {m} budget {f}"
        if k == nsteps // 2:
            a.diag_output("getave")
            b.diag_output("getave")
            oa, ob = a.get_diag_output(), b.get_diag_output()
            for f in oa:
                assert _same(oa[f], ob[f]), f"output diagnostics {f}"
            a.diag_output("reset")
            b.diag_output("reset")
    sa, sb = a.get_state(), b.get_state()
    for f in STATE_KEYS:
        assert _same(sa[f], sb[f]), f
    ga, gb = a.get_diag(), b.get_diag()
    for f in DIAG_KEYS:
        assert _same(ga[f], gb[f]), f
    assert a.kernel_launches < b.kernel_launches


def test_persistent_vs_oracle(case_dirs):
    """Free-running parity of the persistent schedule against the oracle on config-1 laws (levees,
    dams, bifurcation channels), 48 hourly steps."""
    from cmf_b200 import HostModel, PhysicsGPU
    from oracle import Oracle

    h = HostModel(case_dirs["cfg1s"])
    g = PhysicsGPU(h, launch_mode=2)
    o = Oracle(case_dirs["cfg1s"])
    for k, r in enumerate(runoff_series(h.map("grarea"), "cfg1s", 48, hourly=True)):
        o.put_runoff(r)
        g.put_runoff(r)
        nt_o, dt_o = o.advance()
        nt_g, dt_g, _ = g.advance()
        assert nt_g[0] == nt_o and dt_g[0] == dt_o, f"step {k}"
    st = g.get_state()
    for f in ("rivsto", "fldsto", "rivout", "fldout", "levsto", "damsto", "pthflw"):
        ok, worst, bad = rel_close(st[f][0], o.d(f), RTOL)
        assert ok, (f, worst, bad)


def test_persistent_bounded_wait_returns_status(case_dirs):
    """A grid barrier that can never complete (its count is one arrival short) runs out its 2 ms
    bound on every CTA: the kernel returns, the host reads CMF_E_BARRIER, and the context then
    advances normally, equal to a context that never ran the check."""
    from cmf_b200 import HostModel, PhysicsGPU

    h = HostModel(case_dirs["cfg1s"])
    g = PhysicsGPU(h, launch_mode=2)
    ref = PhysicsGPU(h, launch_mode=2)
    series = list(runoff_series(h.map("grarea"), "cfg1s", 6, hourly=True))
    g.put_runoff(series[0])
    ref.put_runoff(series[0])
    g.advance()
    ref.advance()
    assert g.persist_selftest(2_000_000) == 5
    for r in series[1:]:
        g.put_runoff(r)
        ref.put_runoff(r)
        a, _, _ = g.advance()
        b, _, _ = ref.advance()
        assert a[0] == b[0]
    sa, sb = g.get_state(), ref.get_state()
    for f in ("rivsto", "fldsto", "rivout", "fldout"):
        assert _same(sa[f], sb[f]), f
