"""Surrogate-assisted ensemble vs the plain GPU path on the same ensemble (E4/E5 measurement).

Both start from the same spun-up plain state and see the same forcing.  The plain ensemble is the
truth; the surrogate ensemble advances with the emulator, the plain solver judging a rotating
subset of members every 24 h (re-sync, hand-back above tolerance).  Throughput is
cell-coupling-steps/s = NSEQALL * members * hours / device time (CUDA events on the working
streams); accuracy is the Nash-Sutcliffe efficiency of daily (and hourly) discharge at gauge cells.
"""
from __future__ import annotations

import time

import numpy as np

from . import emulator as E


def measure(host, device, members: int = 16, days: int = 4, judge_slots: int = 2, train_members: int = 4,
            train_hours: int = 48, train_iters: int = 2000, cells_per_snapshot: int | None = 65536, seed: int = 100,
            gauges: int = 100, tol_rel: float = 0.05) -> dict:
    import torch

    from .model import PhysicsGPU

    t0 = time.perf_counter()
    X, t = E.generate_trajectories(host, members=train_members, hours=train_hours, spinup=12, seed=seed,
                                   cells_per_snapshot=cells_per_snapshot)
    mlp = E.MLP(device, seed=0, lr=2e-3)
    hist = E.train(mlp, X, t, iters=train_iters, batch=8192, seed=0)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    del X, t
    N = host.dims.nseqall
    gr = host.map("grarea")
    qref = E.qref_from_host(host)
    river = np.arange(host.dims.nseqriv)
    G = river[np.argsort(-qref[river])][:gauges]
    gens = E.runoff_generators(N, members, seed + 1)
    H = days * 24
    plain = PhysicsGPU(host, nmembers=members)
    for _ in range(24):
        plain.put_runoff(E.runoff_step(gens, gr))
        plain.advance()
    runoff = np.stack([E.runoff_step(gens, gr) for _ in range(H)])          # [H, M, N]
    ens = E.SurrogateEnsemble(host, mlp, members=members, judge_slots=judge_slots, gauges=G, tol_rel=tol_rel)
    ens.set_state_from(plain)
    # ---- truth: the plain ensemble
    dev = device
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    truth = np.zeros((H, members, len(G)))
    buf = {"outflw_aavg": np.zeros(members * N)}
    plain_ms = 0.0
    stream = torch.cuda.ExternalStream(plain.stream, device=dev)
    for h in range(H):
        plain.put_runoff(runoff[h])
        ev[0].record(stream)
        plain.advance()
        ev[1].record(stream)
        ev[1].synchronize()
        plain_ms += ev[0].elapsed_time(ev[1])
        truth[h] = plain.get_diag_fields(buf)["outflw_aavg"].reshape(members, N)[:, G]
    # ---- surrogate ensemble (wall time of the whole controller loop, device-synchronised)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    est = ens.run(runoff)
    torch.cuda.synchronize()
    sur_s = time.perf_counter() - t1
    plain.close()
    daily_t = truth.reshape(days, 24, members, len(G)).mean(1)
    daily_e = est.reshape(days, 24, members, len(G)).mean(1)
    nse_daily = E.nse(daily_e.reshape(days, -1), daily_t.reshape(days, -1))
    nse_hourly = E.nse(est.reshape(H, -1), truth.reshape(H, -1))
    cells = N * members * H
    return {
        "members": members, "days": days, "gauges": len(G), "judge_slots": judge_slots,
        "plain_cell_coupling_steps_per_s": cells / (plain_ms / 1e3),
        "surrogate_cell_coupling_steps_per_s": cells / sur_s,
        "speedup_vs_plain": (plain_ms / 1e3) / sur_s,
        "nse_daily_median": float(np.median(nse_daily)), "nse_daily_mean": float(np.mean(nse_daily)),
        "nse_hourly_median": float(np.median(nse_hourly)),
        "judged": ens.stats["judged"], "fallback": ens.stats["fallback"],
        "train_loss_first_last": [hist[0][1], hist[-1][1]], "train_seconds": train_s,
        "timing": "plain: CUDA events around each coupling step; surrogate: host clock around the controller loop "
                  "(emulator, judging plain runs, hand-over copies, read-backs)",
    }
